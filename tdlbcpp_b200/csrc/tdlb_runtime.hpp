// Host-side runtime pieces that need no GPU: the immersed-boundary marker
// scheduler.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "tdlb_kernels.cuh"

namespace tdlb {

// Orders one segment [begin, end) of a marker list for the per-plane level
// walk of k_ibm_spread.
//
// The reference applies markers strictly in list order (Forcing.hpp:72-157).
// Two markers interact only when they share a stencil cell, which needs the
// same j-plane. Within a plane each marker gets
//     level = 1 + max(level of earlier markers of the segment sharing a cell)
// (0 when there is none). Markers of one level touch disjoint cells; any two
// that share a cell sit on increasing levels in list order, so applying the
// levels one after another reproduces the sequential result exactly. A list
// is split into at most two segments (non-rotating markers, then the
// rotating blades); the spread kernel walks all levels of the first segment
// of a plane before those of the second, which keeps their list order too.
//
// Rotation-invariant mode (rot_xz != nullptr, the markers' impeller-frame
// offsets, 2 per marker of the segment): blade cells change every step, so
// the segment is scheduled for EVERY impeller angle at once. Rotation about
// the j axis keeps distances, and two markers can share a stencil cell only
// when their positions are within 3*sqrt(2) (each nearest cell is within 0.5
// per axis, stencils reach 1 cell). A marker therefore goes one level above
// every earlier marker of its plane that is that close.
//
// Output (device-ready, absolute indices):
//   order[end-begin]  marker indices, sorted by (plane j, level, list index);
//                     the marker in order[t] occupies slot slot_base + t
//   level_ptr[L+1]    slot offsets of the segment's levels (level_ptr[0] = slot_base)
//   plane_lv[ny+1]    level numbers (from level_base) of each plane's levels
struct MarkerSchedule {
    std::vector<int> order;
    std::vector<int> level_ptr;
    std::vector<int> plane_lv;
    int max_levels_per_plane = 0;
    int nlevels = 0;

    // 3*sqrt(2) plus a hair: the farthest two markers sharing a stencil cell can be
    static constexpr double kReach = 4.2426407 + 1e-6;

    void build(const Marker* m, int begin, int end, int nx, int ny, int nz, int slot_base, int level_base,
               const double* rot_xz = nullptr) {
        const int n = end - begin;
        order.assign((size_t)n, 0);
        plane_lv.assign((size_t)ny + 1, 0);
        level_ptr.assign(1, slot_base);
        max_levels_per_plane = 0;

        // stable counting sort by plane
        std::vector<int> pcount((size_t)ny + 1, 0);
        for (int q = begin; q < end; q++) pcount[(size_t)m[q].j + 1]++;
        for (int j = 0; j < ny; j++) pcount[(size_t)j + 1] += pcount[(size_t)j];
        std::vector<int> by_plane((size_t)n);
        {
            std::vector<int> fill(pcount.begin(), pcount.end() - 1);
            for (int q = begin; q < end; q++) by_plane[(size_t)fill[(size_t)m[q].j]++] = q;
        }

        std::vector<int> last(rot_xz ? 0 : (size_t)nx * nz, -1);   // highest level touching each (i,k)
        std::vector<int> lev((size_t)n, 0);
        std::vector<int> lcount;
        int level = level_base;
        for (int j = 0; j < ny; j++) {
            plane_lv[(size_t)j] = level;
            const int b = pcount[(size_t)j], e = pcount[(size_t)j + 1];
            int nlev = 0;
            std::unordered_map<long long, std::vector<int>> buckets;
            for (int s = b; s < e; s++) {
                const int q = by_plane[(size_t)s];
                int l = 0;
                if (!rot_xz) {
                    int cells[9];
                    stencil(m[q], nx, nz, cells);
                    for (int c = 0; c < 9; c++) l = std::max(l, last[(size_t)cells[c]] + 1);
                    for (int c = 0; c < 9; c++) last[(size_t)cells[c]] = l;
                } else {
                    const double x0 = rot_xz[2 * (size_t)(q - begin)], z0 = rot_xz[2 * (size_t)(q - begin) + 1];
                    const long long bx = (long long)std::floor(x0 / kReach), bz = (long long)std::floor(z0 / kReach);
                    for (long long dx = -1; dx <= 1; dx++)
                        for (long long dz = -1; dz <= 1; dz++) {
                            auto it = buckets.find(key(bx + dx, bz + dz));
                            if (it == buckets.end()) continue;
                            for (int s2 : it->second) {
                                const int q2 = by_plane[(size_t)s2];
                                const double ex = rot_xz[2 * (size_t)(q2 - begin)] - x0;
                                const double ez = rot_xz[2 * (size_t)(q2 - begin) + 1] - z0;
                                if (ex * ex + ez * ez <= kReach * kReach) l = std::max(l, lev[(size_t)s2] + 1);
                            }
                        }
                    buckets[key(bx, bz)].push_back(s);
                }
                lev[(size_t)s] = l;
                nlev = std::max(nlev, l + 1);
            }
            // bucket the plane's markers by level, keeping list order inside a level
            lcount.assign((size_t)nlev + 1, 0);
            for (int s = b; s < e; s++) lcount[(size_t)lev[(size_t)s] + 1]++;
            for (int l = 0; l < nlev; l++) lcount[(size_t)l + 1] += lcount[(size_t)l];
            std::vector<int> fill(lcount.begin(), lcount.end() - 1);
            for (int s = b; s < e; s++) order[(size_t)(b + fill[(size_t)lev[(size_t)s]]++)] = by_plane[(size_t)s];
            for (int l = 0; l < nlev; l++) level_ptr.push_back(slot_base + b + lcount[(size_t)l + 1]);
            if (!rot_xz) {
                for (int s = b; s < e; s++) {   // reset this plane's cells
                    int cells[9];
                    stencil(m[by_plane[(size_t)s]], nx, nz, cells);
                    for (int c = 0; c < 9; c++) last[(size_t)cells[c]] = -1;
                }
            }
            level += nlev;
            max_levels_per_plane = std::max(max_levels_per_plane, nlev);
        }
        plane_lv[(size_t)ny] = level;
        nlevels = level - level_base;
    }

    static long long key(long long a, long long b) { return (a + (1LL << 30)) * (1LL << 31) + (b + (1LL << 30)); }

    // The 9 (i,k) cells of a marker's stencil with the periodic wrap of
    // Forcing.hpp:98-101, as i*nz + k.
    static void stencil(const Marker& mk, int nx, int nz, int* cells) {
        int c = 0;
        for (int k1 = -1; k1 <= 1; k1++)
            for (int i1 = -1; i1 <= 1; i1++, c++) {
                int i2 = (int)mk.i + i1, k2 = (int)mk.k + k1;
                if (i2 < 0) i2 += nx;
                if (i2 >= nx) i2 -= nx;
                if (k2 < 0) k2 += nz;
                if (k2 >= nz) k2 -= nz;
                cells[c] = i2 * nz + k2;
            }
    }
};

// Unique stencil cells of the first segment, per plane and sorted by
// (i, k), with each slot's 9 plane-local cell indices. The per-pass IBM
// work is then done once per cell instead of once per (marker, cell): every
// wall cell is shared by about three markers.
struct CellList {
    std::vector<int> cell_e;       // element index (row*kp + k) of each cell
    std::vector<int> plane_cell;   // [ny+1] cell range of each plane
    std::vector<int> mcell;        // [n0][9]: plane-local cell index of stencil cell c of slot p
    int max_plane_cells = 0;

    void build(const Marker* m, const MarkerSchedule& seg0, int nx, int ny, int nz, int kp) {
        const int n0 = (int)seg0.order.size();
        cell_e.clear();
        mcell.assign((size_t)9 * n0, 0);
        plane_cell.assign((size_t)ny + 1, 0);
        max_plane_cells = 0;
        std::vector<int> slot((size_t)nx * nz, -1);
        std::vector<int> cells;
        for (int j = 0; j < ny; j++) {
            const int p0 = seg0.level_ptr[(size_t)seg0.plane_lv[(size_t)j]];
            const int p1 = seg0.level_ptr[(size_t)seg0.plane_lv[(size_t)j + 1]];
            cells.clear();
            for (int p = p0; p < p1; p++) {
                int st[9];
                MarkerSchedule::stencil(m[seg0.order[(size_t)p]], nx, nz, st);
                for (int c = 0; c < 9; c++)
                    if (slot[(size_t)st[c]] == -1) {
                        slot[(size_t)st[c]] = -2;
                        cells.push_back(st[c]);
                    }
            }
            std::sort(cells.begin(), cells.end());
            const int base = (int)cell_e.size();
            for (size_t t = 0; t < cells.size(); t++) {
                slot[(size_t)cells[t]] = (int)t;
                const int i = cells[t] / nz, k = cells[t] - i * nz;
                cell_e.push_back((i * ny + j) * kp + k);
            }
            for (int p = p0; p < p1; p++) {
                int st[9];
                MarkerSchedule::stencil(m[seg0.order[(size_t)p]], nx, nz, st);
                for (int c = 0; c < 9; c++) mcell[(size_t)p * 9 + c] = slot[(size_t)st[c]];
            }
            for (int cc : cells) slot[(size_t)cc] = -1;
            plane_cell[(size_t)j + 1] = (int)cell_e.size();
            max_plane_cells = std::max(max_plane_cells, (int)cell_e.size() - base);
        }
    }
};

}  // namespace tdlb
