// Host-side runtime pieces that need no GPU: the immersed-boundary marker
// scheduler.
#pragma once
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "tdlb_kernels.cuh"

namespace tdlb {

// Orders a marker list for the per-plane level walk of k_ibm_spread.
//
// The reference applies markers strictly in list order (Forcing.hpp:72-157).
// Two markers interact only when they share a stencil cell, which needs the
// same j-plane. Within a plane each marker gets
//     level = 1 + max(level of earlier markers sharing one of its cells)
// (0 when there is none). Markers of one level touch disjoint cells; any
// two that share a cell sit on increasing levels in list order, so applying
// the levels one after another reproduces the sequential result exactly.
//
// Rotating tail (markers [rot_begin, n), given with their impeller-frame
// offsets rot_xz[2*(q - rot_begin)]): their cells change every step, so they
// are scheduled for EVERY impeller angle at once. Rotation about the j axis
// keeps distances, and two markers can share a stencil cell only when their
// positions are within 3*sqrt(2) (each nearest cell is within 0.5, stencils
// reach 1 cell). A tail marker therefore goes one level above every earlier
// tail marker of its plane closer than that, and above all non-rotating
// levels of its plane (which precede it in list order).
//
// Output (device-ready):
//   order[n]       marker indices, sorted by (plane j, level, list index)
//   level_ptr[L+1] slot offsets of each level (levels numbered across planes)
//   plane_lv[ny+1] first level of each plane
struct MarkerSchedule {
    std::vector<int> order;
    std::vector<int> level_ptr;
    std::vector<int> plane_lv;
    int max_levels_per_plane = 0;

    void build(const Marker* m, int n, int nx, int ny, int nz, int rot_begin = -1, const double* rot_xz = nullptr) {
        if (rot_begin < 0 || rot_begin > n || !rot_xz) rot_begin = n;
        order.assign((size_t)n, 0);
        plane_lv.assign((size_t)ny + 1, 0);
        level_ptr.clear();
        max_levels_per_plane = 0;

        // stable counting sort by plane
        std::vector<int> pcount((size_t)ny + 1, 0);
        for (int q = 0; q < n; q++) pcount[(size_t)m[q].j + 1]++;
        for (int j = 0; j < ny; j++) pcount[(size_t)j + 1] += pcount[(size_t)j];
        std::vector<int> by_plane((size_t)n);
        {
            std::vector<int> fill(pcount.begin(), pcount.end() - 1);
            for (int q = 0; q < n; q++) by_plane[(size_t)fill[(size_t)m[q].j]++] = q;
        }

        std::vector<int> last((size_t)nx * nz, -1);    // highest level touching each (i,k) of the plane
        std::vector<int> lev((size_t)n, 0);
        std::vector<int> lcount;
        int level_base = 0;
        level_ptr.push_back(0);
        for (int j = 0; j < ny; j++) {
            plane_lv[(size_t)j] = level_base;
            const int b = pcount[(size_t)j], e = pcount[(size_t)j + 1];
            int nlev = 0, nlev_fixed = -1;
            std::unordered_map<long long, std::vector<int>> buckets;   // rotating markers of this plane
            for (int s = b; s < e; s++) {
                const int q = by_plane[(size_t)s];
                const Marker& mk = m[q];
                int l = 0;
                if (q < rot_begin) {
                    int cells[9];
                    stencil(mk, nx, nz, cells);
                    for (int c = 0; c < 9; c++) l = std::max(l, last[(size_t)cells[c]] + 1);
                    for (int c = 0; c < 9; c++) last[(size_t)cells[c]] = l;
                } else {
                    if (nlev_fixed < 0) nlev_fixed = nlev;
                    l = nlev_fixed;
                    const double x0 = rot_xz[2 * (size_t)(q - rot_begin)], z0 = rot_xz[2 * (size_t)(q - rot_begin) + 1];
                    const long long bx = (long long)std::floor(x0 / kReach), bz = (long long)std::floor(z0 / kReach);
                    for (long long dx = -1; dx <= 1; dx++)
                        for (long long dz = -1; dz <= 1; dz++) {
                            auto it = buckets.find(key(bx + dx, bz + dz));
                            if (it == buckets.end()) continue;
                            for (int s2 : it->second) {
                                const int q2 = by_plane[(size_t)s2];
                                const double ex = rot_xz[2 * (size_t)(q2 - rot_begin)] - x0;
                                const double ez = rot_xz[2 * (size_t)(q2 - rot_begin) + 1] - z0;
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
            for (int l = 0; l < nlev; l++) level_ptr.push_back(b + lcount[(size_t)l + 1]);
            // reset the touched cells of this plane
            for (int s = b; s < e; s++) {
                if (by_plane[(size_t)s] >= rot_begin) continue;
                int cells[9];
                stencil(m[by_plane[(size_t)s]], nx, nz, cells);
                for (int c = 0; c < 9; c++) last[(size_t)cells[c]] = -1;
            }
            level_base += nlev;
            max_levels_per_plane = std::max(max_levels_per_plane, nlev);
        }
        plane_lv[(size_t)ny] = level_base;
    }

    // 3*sqrt(2) plus a hair: the farthest two markers sharing a stencil cell can be
    static constexpr double kReach = 4.2426407 + 1e-6;
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

}  // namespace tdlb
