// Drives the reference's CPU ComputeUnit and the B200 specialisation
// (include/tdlb_compute_unit_arch_b200.hpp) side by side through
// ComputeUnitBase<float, 18, MemoryLayoutIJKL>*, in main.cpp's order
// (tdlbcpp/src/main.cpp:213-305 set-up, :409-454 per step), and prints the
// relative L2 differences of their fields. Built against the reference's own
// headers by tests/cpp/Makefile; run by tests/test_gpu_arch_b200.py.
//
//   arch_b200_main <Simple|Esotwist> <edge> <steps> <workdir>
//
// Output: one line "ok rho=<e> u=<e> F=<e> Nu=<e> even=<0|1> even_ref=<0|1>
// markers=<n> jpeg_xz=<0|1> jpeg_xy=<0|1>", or "error: <message>" with exit
// code 3 when the B200 unit cannot be created (no GPU) or a call fails.
#include <sys/stat.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "ComputeUnit.h"
#include "tdlb_compute_unit_arch_b200.hpp"

namespace {

using Base = ComputeUnitBase<float, QLen::D3Q19, MemoryLayoutIJKL>;

// The impeller's marker lists from the project's geometry (the reference's
// geometry library is not vendored), as PosPolar<tNi, float>.
struct Geometry {
    tdlb_rushton spec{};
    std::vector<PosPolar<tNi, float>> fixed, nonupdating;

    static std::vector<PosPolar<tNi, float>> convert(const std::vector<tdlb_marker>& m) {
        std::vector<PosPolar<tNi, float>> out(m.size());
        for (size_t q = 0; q < m.size(); q++) {
            out[q].i = m[q].i;
            out[q].j = m[q].j;
            out[q].k = m[q].k;
            out[q].iCartFraction = m[q].iCartFraction;
            out[q].kCartFraction = m[q].kCartFraction;
            out[q].uDelta = m[q].uDelta;
            out[q].vDelta = m[q].vDelta;
            out[q].wDelta = m[q].wDelta;
        }
        return out;
    }
    template <typename F>
    static std::vector<tdlb_marker> gen(F f) {
        size_t n = 0;
        if (f(nullptr, 0, &n) != TDLB_OK) throw std::runtime_error("geometry query failed");
        std::vector<tdlb_marker> m(n);
        if (f(m.data(), n, &n) != TDLB_OK) throw std::runtime_error("geometry generation failed");
        return m;
    }
    Geometry(long edge, double tip, long startup, double first_delta) {
        spec.x = spec.y = spec.z = edge;
        spec.tip_speed = tip;
        spec.startup_steps = startup;
        fixed = convert(gen([&](tdlb_marker* o, size_t c, size_t* n) { return tdlb_rushton_fixed(&spec, o, c, n); }));
        nonupdating = convert(gen([&](tdlb_marker* o, size_t c, size_t* n) {
            return tdlb_rushton_rotating_nonupdating(&spec, first_delta, o, c, n);
        }));
    }
    // geomFORCING of main.cpp:301-303 / :420-426
    std::vector<PosPolar<tNi, float>> forcing(double angle, double delta) {
        std::vector<PosPolar<tNi, float>> all = fixed;
        all.insert(all.end(), nonupdating.begin(), nonupdating.end());
        auto rot = convert(gen([&](tdlb_marker* o, size_t c, size_t* n) {
            return tdlb_rushton_rotating(&spec, angle, delta, o, c, n);
        }));
        all.insert(all.end(), rot.begin(), rot.end());
        return all;
    }
};

struct L2 {
    double num = 0, den = 0;
    void add(double got, double want) {
        num += (got - want) * (got - want);
        den += want * want;
    }
    double value() const { return den > 0 ? std::sqrt(num / den) : std::sqrt(num); }
};

bool file_exists(const std::string& p) {
    struct stat sb;
    return stat(p.c_str(), &sb) == 0 && sb.st_size > 0;
}

template <Streaming S>
int run(long edge, int steps, const std::string& work) {
    using CpuCU = ComputeUnit<float, QLen::D3Q19, MemoryLayoutIJKL, EgglesSomers, S, CPU>;
    using B200CU = ComputeUnit<float, QLen::D3Q19, MemoryLayoutIJKL, EgglesSomers, S, B200>;
    using AF = AccessField<float, QLen::D3Q19, MemoryLayoutIJKL, EgglesSomers, S>;

    // main.cpp:213-230
    ComputeUnitParams cu;
    cu.nodeID = 0;
    cu.deviceID = 0;
    cu.idi = cu.idj = cu.idk = 0;
    cu.x = cu.y = cu.z = edge;
    cu.i0 = cu.j0 = cu.k0 = 0;
    cu.ghost = 1;
    cu.resolution = 1;

    FlowParams<float> flow;
    flow.initialRho = 1.0f;
    flow.reMNonDimensional = 7300.0f;
    flow.uav = 0.1f;
    flow.cs0 = 0.1f;
    flow.g3 = 0.8f;
    flow.alpha = 0.97f;
    flow.beta = 1.9f;
    flow.useLES = true;
    flow.streaming = S == Simple ? "Simple" : "Esotwist";
    const long startup = 30;
    Geometry geom(edge, flow.uav, startup, 0.0);
    // the units get a physical nu (main.cpp:275 computes it only for its own copy)
    flow.calcNuAndRe_m(tdlb_rushton_blade_outer_radius(&geom.spec));

    OutputParams out(work + "/output");
    CheckpointParams chk;
    chk.checkpointWriteRootDir = work;
    chk.checkpointWriteDirPrefix = "chk";
    DiskOutputTree tree(out, chk);
    tree.setRunningDataFile(work, "running_data.txt");

    CpuCU* cpu = new CpuCU(cu, flow, tree);
    B200CU* gpu = new B200CU(cu, flow, tree);
    Base* units[2] = {cpu, gpu};

    RunningParams running;
    running.step = 1;
    running.angle = 0;
    const double d1 = tdlb_rushton_impeller_increment(&geom.spec, 1);
    geom = Geometry(edge, flow.uav, startup, d1);
    std::vector<PosPolar<tNi, float>> forcing = geom.forcing(running.angle, d1);
    for (Base* lb : units) {
        lb->initialise(flow.initialRho);           // main.cpp:261
        lb->forcing(forcing, flow.alpha, flow.beta);  // main.cpp:305
        lb->setOutputExcludePoints(geom.fixed);       // main.cpp:309
    }
    for (int s = 0; s < steps; s++) {
        running.step++;
        const double d = tdlb_rushton_impeller_increment(&geom.spec, running.step);
        running.angle += d;
        forcing = geom.forcing(running.angle, d);
        for (Base* lb : units) {                      // main.cpp:438-454
            lb->collision();
            lb->bounceBackBoundary();
            lb->streamingPush();
            lb->moments();
            lb->forcing(forcing, flow.alpha, flow.beta);
        }
    }

    // the B200 unit's output calls through the base pointer (main.cpp:462-496)
    const tNi cut = edge / 2 + 1;
    units[1]->calcVorticityXZ(cut, running, 100);
    units[1]->calcVorticityXY(cut, running, 100);
    const bool jpeg_xz = file_exists(tree.formatXZPlaneDir(running.step, cut) + ".jpeg");
    const bool jpeg_xy = file_exists(tree.formatXYPlaneDir(running.step, cut) + ".jpeg");

    std::vector<float> rho, ux, uy, uz, f3, nu;
    gpu->read_velocity_density(rho, ux, uy, uz);
    gpu->read_force(f3);
    gpu->read_nu(nu);
    L2 e_rho, e_u, e_f, e_nu;
    for (tNi i = 1; i <= edge; i++)
        for (tNi j = 1; j <= edge; j++)
            for (tNi k = 1; k <= edge; k++) {
                const size_t c = ((size_t)(i - 1) * edge + (j - 1)) * edge + (k - 1);
                QVec<float, QLen::D3Q19> q = AF::read(*cpu, i, j, k);
                const tNi idx = cpu->index(i, j, k);
                const Velocity<float> u = q.velocity(cpu->F[idx]);
                e_rho.add(rho[c], q.q[0]);
                e_u.add(ux[c], u.x);
                e_u.add(uy[c], u.y);
                e_u.add(uz[c], u.z);
                e_f.add(f3[3 * c + 0], cpu->F[idx].x);
                e_f.add(f3[3 * c + 1], cpu->F[idx].y);
                e_f.add(f3[3 * c + 2], cpu->F[idx].z);
                e_nu.add(nu[c], cpu->Nu[idx]);
            }
    std::printf("ok rho=%.6e u=%.6e F=%.6e Nu=%.6e even=%d even_ref=%d markers=%zu jpeg_xz=%d jpeg_xy=%d\n",
                e_rho.value(), e_u.value(), e_f.value(), e_nu.value(), (int)gpu->evenStep, (int)cpu->evenStep,
                forcing.size(), (int)jpeg_xz, (int)jpeg_xy);
    delete units[1];   // through the base pointer, as main.cpp's unit would be
    delete units[0];
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 5) {
        std::printf("usage: %s <Simple|Esotwist> <edge> <steps> <workdir>\n", argv[0]);
        return 2;
    }
    const std::string streaming = argv[1];
    const long edge = std::atol(argv[2]);
    const int steps = std::atoi(argv[3]);
    const std::string work = argv[4];
    try {
        return streaming == "Simple" ? run<Simple>(edge, steps, work) : run<Esotwist>(edge, steps, work);
    } catch (const std::exception& e) {
        std::printf("error: %s\n", e.what());
        return 3;
    }
}
