// Rushton-turbine geometry (host side); see geometry.cpp for the spec.
#pragma once
#include <vector>

#include "tdlb_b200.h"

namespace tdlb {

// A blade marker in the impeller frame: its offset from the tank axis at
// impeller angle 0 (x0, z0 along i and k) and its plane.
struct RotatingPolar {
    double x0, z0;
    long long j;
};

// Position of a rotating marker at an impeller angle with cos/sin (ca, sa),
// shared verbatim by the host generator and the device rotation kernel so
// that both produce bit-identical markers (no fused multiply-add: every
// operation rounds on its own). omega = impeller angle increment per step.
struct RotatedMarker {
    long long i, k;
    float iCartFraction, kCartFraction, uDelta, wDelta;
};

struct RushtonGeom {
    long long x, y, z;
    double T, D, clearance, blade_h, baffle_w, inset, tip_speed;
    int disk_planes, n_blades, n_baffles;
    long long startup;
    double ci, ck, R_wall;
    long long j_disk;

    static RushtonGeom from(const tdlb_rushton& s);
    int blade_outer_radius() const;
    double increment(unsigned long long step) const;
    std::vector<tdlb_marker> fixed() const;
    std::vector<tdlb_marker> rotating_nonupdating(double delta_angle) const;
    std::vector<RotatingPolar> rotating_polar() const;
    std::vector<tdlb_marker> rotating(double angle, double delta_angle) const;
};

}  // namespace tdlb
