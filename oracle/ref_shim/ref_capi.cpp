// C-ABI wrapper that drives the reference's OWN CPU ComputeUnit, compiled in
// place from the reference sources (tdlbcpp/src) by oracle/Makefile into
// oracle/_ref/libtdlb_ref.so.
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product links or loads this file;
// only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
// and only as the checker / the timed reference arm.
//
// What it exposes:
//   * a ComputeUnit<T,18,IJKL,EgglesSomers,{Simple|Esotwist},CPU> instance
//     for T=float (the reference's production precision, main.cpp:50) and
//     T=double (the FP64 oracle), stepped through the reference's own virtuals
//     in main.cpp's order (main.cpp:438-455);
//   * field read/write in the reference's AoS layout (Field.hpp:18-42),
//     returned as double (float->double is exact);
//   * integer-coded known-answer tests on the reference's own code:
//     the Simple push golden vectors of tests/StreamingSimplePushTest.hpp,
//     and the Esotwist read/write/writeMoments maps (StreamingEsoteric.hpp:28-180).
#include <cstdint>
#include <type_traits>
#include <cstring>
#include <cstdlib>
#include <string>
#include <vector>
#include <iostream>
#include <sstream>
#include <fstream>

#include "Header.h"
#include "ComputeUnit.h"
#if TDLBREF_WITH_GOLDEN
#include "StreamingSimplePushTest.hpp"
#include "StreamingSimpleTest.hpp"
#endif

namespace {

struct MarkerC {  // layout of tdlb_marker in include/tdlb_b200.h
    int64_t i, j, k;
    float iCartFraction, kCartFraction, uDelta, vDelta, wDelta, pad;
};

struct FlowC {    // layout of tdlbref_flow below
    double initialRho, nu, cs0, g3, alpha, beta;
    int32_t useLES;
    int32_t pad;
};

// Silence the reference's directory-creation chatter on stdout while the
// ComputeUnit / DiskOutputTree are constructed.
struct MuteCout {
    std::streambuf* old;
    std::ostringstream sink;
    MuteCout() : old(std::cout.rdbuf(sink.rdbuf())) {}
    ~MuteCout() { std::cout.rdbuf(old); }
};

DiskOutputTree makeTree(const std::string& tmpdir) {
    OutputParams out(tmpdir + "/ref_output");
    CheckpointParams chk;
    chk.checkpointWriteRootDir = tmpdir;
    chk.checkpointWriteDirPrefix = "ref";
    DiskOutputTree tree(out, chk);
    // the reference's progress log goes below tmpdir, not into the caller's
    // working directory (DiskOutputTree.h:80, :273-280)
    tree.setRunningDataFile(tmpdir, "ref_running_data.txt");
    return tree;
}

ComputeUnitParams makeCuParams(long x, long y, long z) {
    ComputeUnitParams cu;
    cu.nodeID = 0; cu.deviceID = -1;
    cu.idi = cu.idj = cu.idk = 0;
    cu.x = x; cu.y = y; cu.z = z;
    cu.i0 = cu.j0 = cu.k0 = 0;
    cu.ghost = 1;           // main.cpp:225 (grid.multiStep = 1)
    cu.resolution = 1;
    return cu;
}

struct Handle {
    int precision;          // 4 or 8
    int streaming;          // 0 Simple, 1 Esotwist
    void* cu;               // ComputeUnitBase<T,18,IJKL>*
    std::string tmpdir;     // root of the DiskOutputTree (checkpoints go below it)
};

template <typename T>
using Base = ComputeUnitBase<T, QLen::D3Q19, MemoryLayoutIJKL>;

template <typename T>
Base<T>* create(int streaming, long x, long y, long z, const FlowC* f, const char* tmpdir) {
    FlowParams<T> flow;
    flow.initialRho = T(f->initialRho);
    flow.nu = T(f->nu);
    flow.cs0 = T(f->cs0);
    flow.g3 = T(f->g3);
    flow.alpha = T(f->alpha);
    flow.beta = T(f->beta);
    flow.useLES = f->useLES != 0;
    flow.streaming = streaming == 0 ? "Simple" : "Esotwist";
    MuteCout mute;
    DiskOutputTree tree = makeTree(tmpdir ? tmpdir : "/tmp");
    ComputeUnitParams cu = makeCuParams(x, y, z);
    if (streaming == 0)
        return new ComputeUnit<T, QLen::D3Q19, MemoryLayoutIJKL, EgglesSomers, Simple, CPU>(cu, flow, tree);
    return new ComputeUnit<T, QLen::D3Q19, MemoryLayoutIJKL, EgglesSomers, Esotwist, CPU>(cu, flow, tree);
}

template <typename T>
void forcing(Base<T>* cu, const MarkerC* m, long n, double alpha, double beta) {
    std::vector<PosPolar<tNi, T>> geom((size_t)n);
    for (long q = 0; q < n; q++) {
        geom[q].i = m[q].i; geom[q].j = m[q].j; geom[q].k = m[q].k;
        geom[q].iCartFraction = T(m[q].iCartFraction);
        geom[q].kCartFraction = T(m[q].kCartFraction);
        geom[q].uDelta = T(m[q].uDelta);
        geom[q].vDelta = T(m[q].vDelta);
        geom[q].wDelta = T(m[q].wDelta);
    }
    cu->forcing(geom, T(alpha), T(beta));
}

template <typename T> Base<T>* as(Handle* h) { return static_cast<Base<T>*>(h->cu); }

// Integer-coded fill of tests/Params/ParamsCommon.hpp:168-206 (offset 0,
// two-digit coordinates): Q(i,j,k,l) = ((i*100+j)*100+k)*100+l.
template <typename CU>
void fillCoded(CU& cu) {
    for (tNi i = 0; i < cu.xg; i++)
        for (tNi j = 0; j < cu.yg; j++)
            for (tNi k = 0; k < cu.zg; k++) {
                unsigned long base = ((i * 100ul + j) * 100ul + k) * 100ul;
                for (int l = 0; l < QLen::D3Q19; l++) cu.Q[cu.index(i, j, k)].q[l] = base + l;
                cu.F[cu.index(i, j, k)].x = base;
                cu.F[cu.index(i, j, k)].y = base + 1;
                cu.F[cu.index(i, j, k)].z = base + 2;
                cu.Nu[cu.index(i, j, k)] = base + 1;
                cu.O[cu.index(i, j, k)] = true;
            }
}

template <typename CU>
void dumpQ(CU& cu, uint64_t* out) {
    for (size_t c = 0; c < cu.size; c++)
        for (int l = 0; l < QLen::D3Q19; l++) out[c * 18 + l] = cu.Q[c].q[l];
}

// Interior moments as the reference reads them (AccessField<...>::read, the
// accessor collision() and forcing() use), out[((i*x..)...)*18 + l] over
// interior cells in (i, j, k) order.
template <typename T, Streaming S>
void readMoments(Base<T>* b, double* out) {
    using CU = ComputeUnitForcing<T, QLen::D3Q19, MemoryLayoutIJKL, EgglesSomers, S>;
    using AF = AccessField<T, QLen::D3Q19, MemoryLayoutIJKL, EgglesSomers, S>;
    CU& cu = *static_cast<CU*>(b);
    size_t c = 0;
    for (tNi i = 1; i <= cu.xg1; i++)
        for (tNi j = 1; j <= cu.yg1; j++)
            for (tNi k = 1; k <= cu.zg1; k++, c++) {
                QVec<T, QLen::D3Q19> q = AF::read(cu, i, j, k);
                for (int l = 0; l < 18; l++) out[c * 18 + l] = (double)q.q[l];
            }
}

}  // namespace

// checkpoint_write through the reference's own DiskOutputTree
// (ComputeUnit.hpp:389-439): its params are set as main.cpp:237 sets them,
// with the checkpoint root and prefix of makeTree(); returns the directory
// the reference chose (DiskOutputTree.h:560-570).
template <typename T>
std::string checkpointWrite(Base<T>* cu, const std::string& tmpdir, const char* unit, long step) {
    MuteCout mute;
    GridParams grid;
    grid.x = cu->xg - 2; grid.y = cu->yg - 2; grid.z = cu->zg - 2;
    grid.multiStep = 1;
    RunningParams run;
    run.step = step;
    OutputParams out(tmpdir + "/ref_output");
    CheckpointParams chk;
    chk.checkpointWriteRootDir = tmpdir;
    chk.checkpointWriteDirPrefix = "ref";
    cu->outputTree.setParams(makeCuParams(grid.x, grid.y, grid.z), grid.getJson(), cu->flow.getJson(), run.getJson(),
                             out.getJson(), chk.getJson());
    cu->checkpoint_write(unit, run);
    return cu->outputTree.getCheckpointDirName(run, false);
}

template <typename T>
void setExclude(Base<T>* cu, const MarkerC* m, long n, int exclude) {
    std::vector<PosPolar<tNi, T>> pts((size_t)n);
    for (long q = 0; q < n; q++) {
        pts[(size_t)q].i = m[q].i;
        pts[(size_t)q].j = m[q].j;
        pts[(size_t)q].k = m[q].k;
    }
    if (exclude) cu->setOutputExcludePoints(pts);
    else cu->unsetOutputExcludePoints(pts);
}

template <typename T>
std::string savePlane(Base<T>* cu, long j, long step) {
    MuteCout mute;
    OrthoPlaneParams plane;
    plane.cutAt = j;
    BinFileParams bin;
    RunningParams run;
    run.step = step;
    cu->template savePlaneXZ<float, 4>(plane, bin, run);
    return cu->outputTree.formatXZPlaneDir(run.step, plane.cutAt);
}

extern "C" {

typedef FlowC tdlbref_flow;
typedef MarkerC tdlbref_marker;

void* tdlbref_create(int precision, int streaming, long x, long y, long z,
                     const tdlbref_flow* flow, const char* tmpdir) {
    if ((precision != 4 && precision != 8) || (streaming != 0 && streaming != 1)) return nullptr;
    if (x < 1 || y < 1 || z < 1) return nullptr;
    Handle* h = new Handle{precision, streaming, nullptr, tmpdir ? tmpdir : "/tmp"};
    if (precision == 4) h->cu = create<float>(streaming, x, y, z, flow, tmpdir);
    else h->cu = create<double>(streaming, x, y, z, flow, tmpdir);
    return h;
}

void tdlbref_destroy(void* hv) {
    Handle* h = (Handle*)hv;
    if (!h) return;
    if (h->precision == 4) delete as<float>(h); else delete as<double>(h);
    delete h;
}

#define TDLBREF_DISPATCH(h, call) \
    do { if ((h)->precision == 4) { auto cu = as<float>(h); call; } else { auto cu = as<double>(h); call; } } while (0)

long tdlbref_size(void* hv) { Handle* h = (Handle*)hv; long s = 0; TDLBREF_DISPATCH(h, s = (long)cu->size); return s; }
int tdlbref_even_step(void* hv) { Handle* h = (Handle*)hv; int e = 0; TDLBREF_DISPATCH(h, e = cu->evenStep ? 1 : 0); return e; }
void tdlbref_set_even_step(void* hv, int even) { Handle* h = (Handle*)hv; TDLBREF_DISPATCH(h, cu->evenStep = (even != 0)); }
void tdlbref_set_nu(void* hv, double nu) { Handle* h = (Handle*)hv; TDLBREF_DISPATCH(h, cu->flow.nu = nu); }

void tdlbref_initialise(void* hv, double rho) { Handle* h = (Handle*)hv; TDLBREF_DISPATCH(h, cu->initialise(rho)); }
void tdlbref_collision(void* hv) { Handle* h = (Handle*)hv; TDLBREF_DISPATCH(h, cu->collision()); }
void tdlbref_bounce_back(void* hv) { Handle* h = (Handle*)hv; TDLBREF_DISPATCH(h, cu->bounceBackBoundary()); }
void tdlbref_streaming_push(void* hv) { Handle* h = (Handle*)hv; TDLBREF_DISPATCH(h, cu->streamingPush()); }
void tdlbref_moments(void* hv) { Handle* h = (Handle*)hv; TDLBREF_DISPATCH(h, cu->moments()); }
void tdlbref_forcing(void* hv, const tdlbref_marker* m, long n, double alpha, double beta) {
    Handle* h = (Handle*)hv;
    if (h->precision == 4) forcing<float>(as<float>(h), m, n, alpha, beta);
    else forcing<double>(as<double>(h), m, n, alpha, beta);
}

// One time step in main.cpp's order (main.cpp:438-454).
void tdlbref_step(void* hv, const tdlbref_marker* m, long n, double alpha, double beta) {
    tdlbref_collision(hv);
    tdlbref_bounce_back(hv);
    tdlbref_streaming_push(hv);
    tdlbref_moments(hv);
    tdlbref_forcing(hv, m, n, alpha, beta);
}

void tdlbref_get_q(void* hv, double* out) {
    Handle* h = (Handle*)hv;
    TDLBREF_DISPATCH(h, for (size_t c = 0; c < cu->size; c++) for (int l = 0; l < 18; l++) out[c * 18 + l] = (double)cu->Q[c].q[l]);
}
void tdlbref_set_q(void* hv, const double* in) {
    Handle* h = (Handle*)hv;
    TDLBREF_DISPATCH(h, for (size_t c = 0; c < cu->size; c++) for (int l = 0; l < 18; l++) cu->Q[c].q[l] = in[c * 18 + l]);
}
void tdlbref_get_f(void* hv, double* out) {
    Handle* h = (Handle*)hv;
    TDLBREF_DISPATCH(h, for (size_t c = 0; c < cu->size; c++) { out[c * 3] = cu->F[c].x; out[c * 3 + 1] = cu->F[c].y; out[c * 3 + 2] = cu->F[c].z; });
}
void tdlbref_set_f(void* hv, const double* in) {
    Handle* h = (Handle*)hv;
    TDLBREF_DISPATCH(h, for (size_t c = 0; c < cu->size; c++) { cu->F[c].x = in[c * 3]; cu->F[c].y = in[c * 3 + 1]; cu->F[c].z = in[c * 3 + 2]; });
}
void tdlbref_get_nu(void* hv, double* out) {
    Handle* h = (Handle*)hv;
    TDLBREF_DISPATCH(h, for (size_t c = 0; c < cu->size; c++) out[c] = cu->Nu[c]);
}
void tdlbref_set_nu_field(void* hv, const double* in) {
    Handle* h = (Handle*)hv;
    TDLBREF_DISPATCH(h, for (size_t c = 0; c < cu->size; c++) cu->Nu[c] = in[c]);
}

void tdlbref_get_moments(void* hv, double* out) {
    Handle* h = (Handle*)hv;
    if (h->precision == 4) {
        if (h->streaming == 0) readMoments<float, Simple>(as<float>(h), out); else readMoments<float, Esotwist>(as<float>(h), out);
    } else {
        if (h->streaming == 0) readMoments<double, Simple>(as<double>(h), out); else readMoments<double, Esotwist>(as<double>(h), out);
    }
}

// ---------------------------------------------------------------------------
// Integer-coded known-answer tests (T = unsigned long, as in
// tests/StreamingSimpleTest.cpp:74 and :110).
// ---------------------------------------------------------------------------

// Simple push (push=1) or pull (push=0) on the coded fill of an x*y*z
// interior with ghost 1. out: xg*yg*zg*18 values in AoS order.
int tdlbref_kat_simple_stream(int push, long x, long y, long z, uint64_t* out) {
    MuteCout mute;
    FlowParams<unsigned long> flow;
    DiskOutputTree tree = makeTree("/tmp");
    ComputeUnit<unsigned long, QLen::D3Q19, MemoryLayoutIJKL, EgglesSomers, Simple, CPU> cu(makeCuParams(x, y, z), flow, tree);
    if (cu.xg > 99 || cu.yg > 99 || cu.zg > 99) return 1;
    fillCoded(cu);
    if (push) cu.streamingPush(); else cu.streamingPull();
    dumpQ(cu, out);
    return 0;
}

// The reference's committed golden vectors (tests/StreamingSimplePushTest.hpp
// and tests/StreamingSimpleTest.hpp) for the 3x3x3 interior, ghost 1.
int tdlbref_kat_simple_golden(int push, uint64_t* out) {
#if TDLBREF_WITH_GOLDEN
    MuteCout mute;
    FlowParams<unsigned long> flow;
    DiskOutputTree tree = makeTree("/tmp");
    ComputeUnit<unsigned long, QLen::D3Q19, MemoryLayoutIJKL, EgglesSomers, Simple, CPU> cu(makeCuParams(3, 3, 3), flow, tree);
    if (push) TestUtils::fillExpectedComputeUnitValuesTestStreamingNievePush(cu);
    else TestUtils::fillExpectedComputeUnitValuesTestStreamingNieve(cu);
    dumpQ(cu, out);
    return 0;
#else
    (void)push; (void)out;
    return 2;
#endif
}

// Esotwist transport on the coded fill: nsteps times, for every interior
// cell, q = AccessField::read(i,j,k); AccessField::write(q,i,j,k); then flip
// evenStep as streamingPush does (StreamingEsoteric.hpp:15-18). With
// moments_map != 0 the step instead applies read + writeMoments (the map
// moments() uses, CollisionEgglesSomers.hpp:196,248) without a flip.
int tdlbref_kat_esotwist(long x, long y, long z, int start_even, int nsteps, int moments_map, uint64_t* out) {
    MuteCout mute;
    FlowParams<unsigned long> flow;
    DiskOutputTree tree = makeTree("/tmp");
    using CU = ComputeUnit<unsigned long, QLen::D3Q19, MemoryLayoutIJKL, EgglesSomers, Esotwist, CPU>;
    using AF = AccessField<unsigned long, QLen::D3Q19, MemoryLayoutIJKL, EgglesSomers, Esotwist>;
    CU cu(makeCuParams(x, y, z), flow, tree);
    if (cu.xg > 99 || cu.yg > 99 || cu.zg > 99) return 1;
    fillCoded(cu);
    cu.evenStep = start_even != 0;
    for (int s = 0; s < nsteps; s++) {
        for (tNi i = 1; i <= cu.xg1; i++)
            for (tNi j = 1; j <= cu.yg1; j++)
                for (tNi k = 1; k <= cu.zg1; k++) {
                    QVec<unsigned long, QLen::D3Q19> q = AF::read(cu, i, j, k);
                    if (moments_map) AF::writeMoments(cu, q, i, j, k);
                    else AF::write(cu, q, i, j, k);
                }
        if (!moments_map) cu.streamingPush();
    }
    dumpQ(cu, out);
    return 0;
}

// Esotwist read map alone: for every interior cell, the 18 values
// AccessField::read returns on the coded fill (parity even/odd).
// out: x*y*z*18 values, interior cells in (i,j,k) order.
int tdlbref_kat_esotwist_read(long x, long y, long z, int even, uint64_t* out) {
    MuteCout mute;
    FlowParams<unsigned long> flow;
    DiskOutputTree tree = makeTree("/tmp");
    using CU = ComputeUnit<unsigned long, QLen::D3Q19, MemoryLayoutIJKL, EgglesSomers, Esotwist, CPU>;
    using AF = AccessField<unsigned long, QLen::D3Q19, MemoryLayoutIJKL, EgglesSomers, Esotwist>;
    CU cu(makeCuParams(x, y, z), flow, tree);
    if (cu.xg > 99 || cu.yg > 99 || cu.zg > 99) return 1;
    fillCoded(cu);
    cu.evenStep = even != 0;
    size_t c = 0;
    for (tNi i = 1; i <= cu.xg1; i++)
        for (tNi j = 1; j <= cu.yg1; j++)
            for (tNi k = 1; k <= cu.zg1; k++, c++) {
                QVec<unsigned long, QLen::D3Q19> q = AF::read(cu, i, j, k);
                for (int l = 0; l < 18; l++) out[c * 18 + l] = q.q[l];
            }
    return 0;
}

// FlowParams<float>::calcNuAndRe_m (FlowParams.hpp:65-70) itself.
double tdlbref_calc_nu(double re, double uav, int radius) {
    FlowParams<float> f;
    f.reMNonDimensional = (float)re;
    f.uav = (float)uav;
    f.calcNuAndRe_m(radius);
    return (double)f.nu;
}

// The flow and grid a ComputeUnit built by main.cpp from an input file
// holds: the file parsed by the reference's own GridParams / FlowParams
// getParamsFromJson (main.cpp:133-164), FlowParams<float> as
// useQVecPrecision is float (main.cpp:50), and the unit constructed from
// that FlowParams before main.cpp:275 computes nu for its own copy -- so
// the unit keeps the file's nu. xyz[3] = GridParams x, y, z; *multistep =
// GridParams.multiStep (the ghost width, main.cpp:225); *streaming = 0 for
// "Simple", 1 otherwise (main.cpp:242-256). Returns 0, or -1 when the file
// cannot be read or parsed.
int tdlbref_read_input(const char* path, long* xyz, long* multistep, FlowC* out, int* streaming) {
    try {
        nlohmann::json j;
        std::ifstream in(path);
        if (!in) return -1;
        in >> j;
        GridParams grid;
        FlowParams<float> flow;
        MuteCout mute;
        grid.getParamsFromJson(j["GridParams"]);
        flow.getParamsFromJson(j["FlowParams"]);
        xyz[0] = (long)grid.x;
        xyz[1] = (long)grid.y;
        xyz[2] = (long)grid.z;
        *multistep = (long)grid.multiStep;
        out->initialRho = flow.initialRho;
        out->nu = flow.nu;
        out->cs0 = flow.cs0;
        out->g3 = flow.g3;
        out->alpha = flow.alpha;
        out->beta = flow.beta;
        out->useLES = flow.useLES ? 1 : 0;
        out->pad = 0;
        *streaming = flow.streaming == "Simple" ? 0 : 1;
    } catch (const std::exception&) {
        return -1;
    }
    return 0;
}

// setOutputExcludePoints / unsetOutputExcludePoints (ComputeUnitOutput.hpp:20-53).
void tdlbref_set_exclude(void* hv, const tdlbref_marker* m, long n, int exclude) {
    Handle* h = (Handle*)hv;
    if (h->precision == 4) setExclude<float>(as<float>(h), m, n, exclude);
    else setExclude<double>(as<double>(h), m, n, exclude);
}

// savePlaneXZ<float, 4> (ComputeUnitOutput.hpp:354-447) through the
// reference's own DiskOutputTree; returns the plot directory it wrote.
long tdlbref_save_plane_xz(void* hv, long j, long step, char* dir_out, long cap) {
    Handle* h = (Handle*)hv;
    std::string dir;
    try {
        dir = h->precision == 4 ? savePlane<float>(as<float>(h), j, step) : savePlane<double>(as<double>(h), j, step);
    } catch (const std::exception&) {
        return 0;
    }
    if ((long)dir.size() + 1 > cap) return 0;
    std::memcpy(dir_out, dir.c_str(), dir.size() + 1);
    return (long)dir.size();
}

// Checkpoint through the reference's own writer / reader. write returns the
// directory length (0 on failure) and copies the path into dir_out.
long tdlbref_checkpoint_write(void* hv, const char* unit, long step, char* dir_out, long cap) {
    Handle* h = (Handle*)hv;
    std::string dir;
    try {
        if (h->precision == 4) dir = checkpointWrite<float>(as<float>(h), h->tmpdir, unit, step);
        else dir = checkpointWrite<double>(as<double>(h), h->tmpdir, unit, step);
    } catch (const std::exception&) {
        return 0;
    }
    if ((long)dir.size() + 1 > cap) return 0;
    std::memcpy(dir_out, dir.c_str(), dir.size() + 1);
    return (long)dir.size();
}

int tdlbref_checkpoint_read(void* hv, const char* dir, const char* unit) {
    Handle* h = (Handle*)hv;
    try {
        MuteCout mute;
        TDLBREF_DISPATCH(h, cu->checkpoint_read(dir, unit));
    } catch (const std::exception&) {
        return -1;
    }
    return 0;
}

}  // extern "C"
