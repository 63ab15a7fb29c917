// Project-written stand-in for the geometry header that tdLBCpp includes from
// its (un-vendored, empty) tdLBGeometryRushtonTurbineLib submodule.
//
// Test infrastructure only: it exists so that the reference's own CPU
// ComputeUnit headers compile into the parity oracle under oracle/_ref/.
// It declares just the marker type and the geometry class name that the
// compute core names:
//   - PosPolar<tNi,T> is the marker read by forcing()
//     (tdlbcpp/src/Forcing.hpp:72-150 uses i, j, k, iCartFraction,
//     kCartFraction, uDelta, vDelta, wDelta);
//   - RushtonTurbinePolarCPP<tNi,T> appears only in the writeAllOutput
//     signature (tdlbcpp/src/ComputeUnit.h:153), which the oracle never calls.
// Marker generation itself lives in the product (tdlbcpp_b200/csrc/geometry.cpp);
// the same marker list is fed to this oracle and to the GPU path.
#pragma once

template <typename tNi, typename T>
struct PosPolar {
    tNi i = 0;
    tNi j = 0;
    tNi k = 0;
    T iCartFraction = 0;
    T kCartFraction = 0;
    T uDelta = 0;
    T vDelta = 0;
    T wDelta = 0;
};

template <typename tNi, typename T>
class RushtonTurbinePolarCPP {
public:
    int impellerStartupStepsUntilNormalSpeed = 0;
};
