// Project-written stand-in for the un-vendored RushtonTurbine header.
// Test infrastructure only (see GeomPolar.hpp beside it): the compute-core
// headers include it but use nothing from it.
#pragma once

struct RushtonTurbine {
    explicit RushtonTurbine(int gridX) : gridX(gridX) {}
    int gridX;
};
