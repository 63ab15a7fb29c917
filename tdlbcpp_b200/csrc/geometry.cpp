// Rushton-turbine stirred-tank marker generator (host, no GPU needed).
//
// The reference takes its markers from the tdLBGeometryRushtonTurbineLib
// submodule, which is not vendored (tdlbcpp/src/main.cpp:274-303, :409-426
// call RushtonTurbinePolarCPP::generateFixedGeometry / ...RotatingNonUpdating
// / ...RotatingGeometry / updateRotatingGeometry and
// calcThisStepImpellerIncrement). This file is this project's own geometry
// with the same three marker classes, fed identically to the GPU path and
// to the CPU oracle. Its spec (cell coordinates, j vertical):
//
//   tank        cylinder of diameter T about the lattice centre
//               ((x-1)/2, (z-1)/2); wall markers at radius T/2 - inset
//               so that no stencil wraps across the periodic i/k seam
//   baffles     n_baffles radial plates of width T/10 against the wall,
//               full height, at angles pi/4 + 2 pi b / n_baffles
//   impeller    D = T/3 at clearance T/3 above j = 0: a disk of diameter
//               3D/4 (filled, disk_thickness planes), a shaft of radius
//               max(1, D/10) from the disk to the top, and n_blades flat
//               blades spanning radius D/4 .. D/2 and height D/5
//   spacing     one marker per cell along every line / ring
//   classes     fixed = wall + baffles; rotating-non-updating = disk +
//               shaft (axisymmetric: positions fixed, tangential velocity);
//               rotating = blades (positions follow the impeller angle)
//   velocity    (uDelta, vDelta, wDelta) = omega x r about the j axis,
//               omega = delta angle per step
//   speed ramp  delta angle = (tip_speed / (D/2)) * min(1, step / startup)
//
// Marker ORDER within each class is chosen so that markers sharing a
// stencil cell are rare inside a run: markers are emitted grouped by
// (i mod 3, k mod 3) of their cell (fixed/non-updating) or by position along
// the blade line mod 5 (rotating), which keeps the number of
// immersed-boundary levels per plane small. The GPU path reproduces the
// sequential result for ANY order; the order only changes its speed.
#include "tdlb_b200.h"
#include "tdlb_geometry.hpp"
#include "tdlb_rotate.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace tdlb {
namespace {

struct P {
    double pi, pk;     // continuous cell coordinates in the i-k plane
    long long j;
    double r, theta;   // polar about the tank axis
    int color;
    long long seq;
};

tdlb_marker to_marker(const RushtonGeom& G, const P& p, double omega) {
    tdlb_marker m{};
    long long i = (long long)std::floor(p.pi + 0.5);
    long long k = (long long)std::floor(p.pk + 0.5);
    i = std::min<long long>(std::max<long long>(i, 0), G.x - 1);
    k = std::min<long long>(std::max<long long>(k, 0), G.z - 1);
    m.i = i;
    m.j = p.j;
    m.k = k;
    m.iCartFraction = (float)(p.pi - (double)i);
    m.kCartFraction = (float)(p.pk - (double)k);
    const double di = p.pi - G.ci, dk = p.pk - G.ck;
    m.uDelta = (float)(-omega * dk);
    m.vDelta = 0.f;
    m.wDelta = (float)(omega * di);
    return m;
}

void ring(const RushtonGeom& G, double r, long long j, double phase, std::vector<P>& out) {
    const long long n = r < 0.5 ? 1 : std::max<long long>(1, (long long)std::llround(2.0 * M_PI * r));
    for (long long q = 0; q < n; q++) {
        const double th = phase + 2.0 * M_PI * (double)q / (double)n;
        P p;
        p.r = r;
        p.theta = th;
        p.pi = G.ci + r * std::cos(th);
        p.pk = G.ck + r * std::sin(th);
        p.j = j;
        p.color = 0;
        p.seq = (long long)out.size();
        out.push_back(p);
    }
}

// Group by (i mod 3, k mod 3) of the nearest cell: markers in one group
// sit >= 3 cells apart in i or k unless they share a cell.
void color_by_cell(std::vector<P>& v) {
    for (auto& p : v) {
        const long long i = (long long)std::floor(p.pi + 0.5), k = (long long)std::floor(p.pk + 0.5);
        p.color = (int)(((i % 3) + 3) % 3 * 3 + ((k % 3) + 3) % 3);
    }
    std::stable_sort(v.begin(), v.end(), [](const P& a, const P& b) { return a.color < b.color; });
}

}  // namespace

RushtonGeom RushtonGeom::from(const tdlb_rushton& s) {
    RushtonGeom G;
    G.x = s.x; G.y = s.y; G.z = s.z;
    G.T = s.tank_diameter > 0 ? s.tank_diameter : (double)s.x;
    G.D = s.impeller_diameter > 0 ? s.impeller_diameter : G.T / 3.0;
    G.clearance = s.clearance > 0 ? s.clearance : G.T / 3.0;
    G.blade_h = s.blade_height > 0 ? s.blade_height : G.D / 5.0;
    G.disk_planes = s.disk_thickness > 0 ? (int)std::llround(s.disk_thickness) : 1;
    G.n_blades = s.n_blades > 0 ? s.n_blades : 6;
    G.n_baffles = s.n_baffles > 0 ? s.n_baffles : (s.n_baffles < 0 ? 0 : 4);   // -1: none
    G.baffle_w = s.baffle_width > 0 ? s.baffle_width : G.T / 10.0;
    G.inset = s.wall_inset > 0 ? s.wall_inset : 2.0;
    G.tip_speed = s.tip_speed;
    G.startup = s.startup_steps;
    G.ci = ((double)s.x - 1.0) / 2.0;
    G.ck = ((double)s.z - 1.0) / 2.0;
    G.R_wall = G.T / 2.0 - G.inset;
    G.j_disk = (long long)std::llround(G.clearance);
    return G;
}

int RushtonGeom::blade_outer_radius() const { return (int)(D / 2.0); }

double RushtonGeom::increment(unsigned long long step) const {
    const double omega = tip_speed / (D / 2.0);
    if (startup <= 0 || (long long)step >= startup) return omega;
    return omega * (double)step / (double)startup;
}

std::vector<tdlb_marker> RushtonGeom::fixed() const {
    // The wall ring and the baffle points are the same in every plane: they
    // are computed once, grouped by colour, and emitted colour by colour --
    // the wall in (plane, ring position) order, then the baffles in
    // (baffle, plane, radius) order, which is the order a stable sort by
    // colour of the plane-by-plane list gives.
    std::vector<P> wall;
    ring(*this, R_wall, 0, 0.0, wall);
    std::vector<std::vector<P>> baffle((size_t)std::max(n_baffles, 0));
    for (int b = 0; b < n_baffles; b++) {
        const double phi = M_PI / 4.0 + 2.0 * M_PI * b / n_baffles;
        for (double r = R_wall - 1.0; r >= R_wall - baffle_w - 1e-9; r -= 1.0) {
            P p;
            p.r = r; p.theta = phi;
            p.pi = ci + r * std::cos(phi);
            p.pk = ck + r * std::sin(phi);
            p.j = 0;
            p.seq = 0;
            baffle[(size_t)b].push_back(p);
        }
    }
    auto colour = [](const P& p) {
        const long long i = (long long)std::floor(p.pi + 0.5), k = (long long)std::floor(p.pk + 0.5);
        return (int)(((i % 3) + 3) % 3 * 3 + ((k % 3) + 3) % 3);
    };
    size_t per_plane = wall.size();
    for (const auto& bv : baffle) per_plane += bv.size();
    std::vector<tdlb_marker> out;
    out.reserve(per_plane * (size_t)std::max<long long>(y, 0));
    for (int c = 0; c < 9; c++) {
        std::vector<const P*> w;
        for (const P& p : wall)
            if (colour(p) == c) w.push_back(&p);
        for (long long j = 0; j < y; j++)
            for (const P* p : w) {
                P q = *p;
                q.j = j;
                out.push_back(to_marker(*this, q, 0.0));
            }
        for (const auto& bv : baffle) {
            std::vector<const P*> bb;
            for (const P& p : bv)
                if (colour(p) == c) bb.push_back(&p);
            for (long long j = 0; j < y; j++)
                for (const P* p : bb) {
                    P q = *p;
                    q.j = j;
                    out.push_back(to_marker(*this, q, 0.0));
                }
        }
    }
    return out;
}

std::vector<tdlb_marker> RushtonGeom::rotating_nonupdating(double delta_angle) const {
    std::vector<P> v;
    const double R_disk = 0.375 * D;
    for (int t = 0; t < disk_planes; t++) {
        const long long j = j_disk + t;
        if (j < 0 || j >= y) continue;
        for (double r = 0.0; r <= R_disk + 1e-9; r += 1.0) ring(*this, r, j, 0.0, v);
    }
    const double r_shaft = std::max(1.0, D / 10.0);
    for (long long j = j_disk + disk_planes; j < y; j++) ring(*this, r_shaft, j, 0.0, v);
    color_by_cell(v);
    std::vector<tdlb_marker> out;
    out.reserve(v.size());
    for (const auto& p : v) out.push_back(to_marker(*this, p, delta_angle));
    return out;
}

std::vector<RotatingPolar> RushtonGeom::rotating_polar() const {
    // blades: radial lines at every height of the blade, grouped by the
    // position along the line mod 5 (same-group markers of one line are 5
    // apart at every angle)
    std::vector<RotatingPolar> v;
    const double r0 = D / 4.0, r1 = D / 2.0;
    const long long jh0 = (long long)std::llround((double)j_disk - blade_h / 2.0);
    const long long jh1 = (long long)std::llround((double)j_disk + blade_h / 2.0);
    for (int c = 0; c < 5; c++)
        for (int b = 0; b < n_blades; b++) {
            const double th = 2.0 * M_PI * b / n_blades;
            const double cth = std::cos(th), sth = std::sin(th);
            for (long long j = std::max<long long>(jh0, 0); j <= std::min<long long>(jh1, y - 1); j++) {
                int q = 0;
                for (double r = r0; r <= r1 + 1e-9; r += 1.0, q++) {
                    if (q % 5 != c) continue;
                    RotatingPolar p;
                    p.x0 = r * cth;
                    p.z0 = r * sth;
                    p.j = j;
                    v.push_back(p);
                }
            }
        }
    return v;
}

std::vector<tdlb_marker> RushtonGeom::rotating(double angle, double delta_angle) const {
    const std::vector<RotatingPolar> pol = rotating_polar();
    const double ca = std::cos(angle), sa = std::sin(angle);
    std::vector<tdlb_marker> out;
    out.reserve(pol.size());
    for (const auto& q : pol) {
        const RotatedMarker r = rotate_marker(q.x0, q.z0, ca, sa, delta_angle, ci, ck, x, z);
        tdlb_marker m{};
        m.i = r.i; m.j = q.j; m.k = r.k;
        m.iCartFraction = r.iCartFraction;
        m.kCartFraction = r.kCartFraction;
        m.uDelta = r.uDelta;
        m.vDelta = 0.f;
        m.wDelta = r.wDelta;
        out.push_back(m);
    }
    return out;
}

}  // namespace tdlb

namespace {
int copy_out(const std::vector<tdlb_marker>& v, tdlb_marker* out, size_t cap, size_t* n) {
    if (n) *n = v.size();
    if (!out) return TDLB_OK;
    if (cap < v.size()) return TDLB_EINVAL;
    if (!v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(tdlb_marker));
    return TDLB_OK;
}
bool bad(const tdlb_rushton* s) { return !s || s->x < 1 || s->y < 1 || s->z < 1; }
}  // namespace

extern "C" {

int tdlb_rushton_fixed(const tdlb_rushton* spec, tdlb_marker* out, size_t cap, size_t* n) {
    if (bad(spec)) return TDLB_EINVAL;
    return copy_out(tdlb::RushtonGeom::from(*spec).fixed(), out, cap, n);
}

int tdlb_rushton_rotating_nonupdating(const tdlb_rushton* spec, double delta_angle, tdlb_marker* out, size_t cap,
                                      size_t* n) {
    if (bad(spec)) return TDLB_EINVAL;
    return copy_out(tdlb::RushtonGeom::from(*spec).rotating_nonupdating(delta_angle), out, cap, n);
}

int tdlb_rushton_rotating(const tdlb_rushton* spec, double angle, double delta_angle, tdlb_marker* out, size_t cap,
                          size_t* n) {
    if (bad(spec)) return TDLB_EINVAL;
    return copy_out(tdlb::RushtonGeom::from(*spec).rotating(angle, delta_angle), out, cap, n);
}

double tdlb_rushton_impeller_increment(const tdlb_rushton* spec, uint64_t step) {
    if (bad(spec)) return 0.0;
    return tdlb::RushtonGeom::from(*spec).increment(step);
}

int tdlb_rushton_blade_outer_radius(const tdlb_rushton* spec) {
    if (bad(spec)) return TDLB_EINVAL;
    return tdlb::RushtonGeom::from(*spec).blade_outer_radius();
}

}  // extern "C"
