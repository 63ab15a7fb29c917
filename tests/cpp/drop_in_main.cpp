// A main.cpp-shaped driver (tdlbcpp/src/main.cpp:241-455) written against
// the C++ mirror of the ComputeUnit API. Used by tests/test_cpp_adapter.py:
// without a GPU it must fail loudly; with one it runs a small tank and
// prints density and momentum sums.
#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "tdlb_compute_unit_b200.hpp"

// the reference's marker type (GeomPolar.hpp PosPolar<tNi,T> fields forcing() reads)
template <typename tNi, typename T>
struct PosPolar {
    tNi i, j, k;
    T iCartFraction, kCartFraction, uDelta, vDelta, wDelta;
};

int main(int argc, char** argv) {
    const std::string json = argc > 1 ? argv[1] : "";
    try {
        tdlb::ComputeUnitB200 lb(json, 0);
        tdlb_rushton spec{};
        spec.x = lb.x; spec.y = lb.y; spec.z = lb.z;
        spec.tip_speed = 0.1;
        const double dth = tdlb_rushton_impeller_increment(&spec, 1);
        auto gen = [&](double angle) {
            std::vector<tdlb_marker> all;
            size_t n = 0;
            tdlb_rushton_fixed(&spec, nullptr, 0, &n);
            all.resize(n);
            tdlb_rushton_fixed(&spec, all.data(), n, &n);
            size_t n2 = 0;
            tdlb_rushton_rotating_nonupdating(&spec, dth, nullptr, 0, &n2);
            all.resize(n + n2);
            tdlb_rushton_rotating_nonupdating(&spec, dth, all.data() + n, n2, &n2);
            size_t n3 = 0;
            tdlb_rushton_rotating(&spec, angle, dth, nullptr, 0, &n3);
            all.resize(n + n2 + n3);
            tdlb_rushton_rotating(&spec, angle, dth, all.data() + n + n2, n3, &n3);
            std::vector<PosPolar<long, float>> geom(all.size());
            for (size_t q = 0; q < all.size(); q++)
                geom[q] = {all[q].i, all[q].j, all[q].k, all[q].iCartFraction, all[q].kCartFraction,
                           all[q].uDelta, all[q].vDelta, all[q].wDelta};
            return geom;
        };
        double angle = 0.0;
        lb.initialise(1.0f);
        auto geomFORCING = gen(angle);
        lb.forcing(geomFORCING, 0.97f, 1.9f);
        for (int step = 2; step <= 6; step++) {
            angle += dth;
            geomFORCING = gen(angle);
            lb.collision();
            lb.bounceBackBoundary();
            lb.streamingPush();
            lb.moments();
            lb.forcing(geomFORCING, 0.97f, 1.9f);
        }
        std::vector<float> rho, ux, uy, uz;
        lb.velocity_density(rho, ux, uy, uz);
        double mass = 0, mom = 0;
        for (size_t c = 0; c < rho.size(); c++) {
            mass += rho[c];
            mom += std::fabs(ux[c]) + std::fabs(uy[c]) + std::fabs(uz[c]);
        }
        std::printf("ok cells=%zu markers=%zu mass=%.6f absmom=%.6e\n", rho.size(), geomFORCING.size(), mass, mom);
        return 0;
    } catch (const std::runtime_error& e) {
        std::printf("error: %s\n", e.what());
        return 3;
    }
}
