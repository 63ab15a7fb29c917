// Host runtime and C ABI (include/tdlb_b200.h) of the B200 lattice Boltzmann
// time step: device memory, the marker scheduler, launch sequencing and
// state bookkeeping. Kernels live in step_kernels.cu and ibm_kernels.cu.
#include "tdlb_b200.h"
#include "tdlb_kernels.cuh"
#include "tdlb_runtime.hpp"
#include "tdlb_geometry.hpp"

#include <nlohmann/json.hpp>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

using tdlb::Dims;
using tdlb::Planes;

namespace {

thread_local std::string g_create_error = "no error";

struct Fail {
    int code;
    std::string msg;
};

#define TDLB_CK(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            throw Fail{TDLB_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)};        \
    } while (0)

long long round_up(long long a, long long m) { return (a + m - 1) / m * m; }

}  // namespace

#include "tdlb_handle.hpp"

namespace {

void release(tdlb_lattice* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    cudaFree(h->bufA);
    cudaFree(h->bufB);
    cudaFree(h->Nu);
    cudaFree(h->F);
    cudaFree(h->mask);
    cudaFree(h->d_markers);
    cudaFree(h->d_sched);
    cudaFree(h->d_level_ptr);
    cudaFree(h->d_plane_lv0);
    cudaFree(h->d_plane_lv1);
    cudaFree(h->d_blade_planes);
    cudaFree(h->d_cell_e);
    cudaFree(h->d_cell_order);
    cudaFree(h->d_plane_cell);
    cudaFree(h->d_prep);
    cudaFree(h->d_cell_m);
    cudaFree(h->d_cell_F);
    cudaFree(h->d_tail);
    cudaFree(h->d_sums);
    cudaFree(h->d_mask_static);
    cudaFree(h->d_plane_list);
    cudaFree(h->d_exclude);
    cudaFree(h->d_zone_list);
    cudaFree(h->d_box_list);
    cudaFree(h->d_box_out);
    for (cudaEvent_t e : h->tev) cudaEventDestroy(e);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->ibm) cudaStreamDestroy(h->ibm);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    if (h->ev_outer) cudaEventDestroy(h->ev_outer);
    if (h->ev_inner) cudaEventDestroy(h->ev_inner);
    if (h->ev_sync) cudaEventDestroy(h->ev_sync);
    cudaFree(h->d_red);
    cudaFree(h->d_rot_xz);
    cudaFree(h->d_load);
    cudaFree(h->d_res[0]);
    cudaFree(h->d_res[1]);
    for (auto& st : h->pin) {
        cudaFreeHost(st.p);
        if (st.ev) cudaEventDestroy(st.ev);
    }
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    else if (h->stream) cudaStreamDestroy(h->stream);
}

void validate_config(const tdlb_config& c) {
    if (c.x < 1 || c.y < 1 || c.z < 1) throw Fail{TDLB_EINVAL, "grid extents must be >= 1"};
    if (c.x > 32767 || c.y > 32767 || c.z > 32767) throw Fail{TDLB_EINVAL, "grid extent above 32767"};
    if (c.streaming != TDLB_STREAMING_SIMPLE && c.streaming != TDLB_STREAMING_ESOTWIST)
        throw Fail{TDLB_EINVAL, "streaming must be Simple (0) or Esotwist (1)"};
    if (c.storage < TDLB_STORAGE_FP32 || c.storage > TDLB_STORAGE_BF16)
        throw Fail{TDLB_EINVAL, "storage must be FP32 (0), FP16 (1) or BF16 (2)"};
    if (c.storage != TDLB_STORAGE_FP32 && !(c.initialRho > 0.0))
        throw Fail{TDLB_EINVAL, "16-bit storage needs initialRho > 0 (deviations are taken from it)"};
    if (!(c.nu >= 0.0) || !std::isfinite(c.nu)) throw Fail{TDLB_EINVAL, "nu must be finite and >= 0"};
}

tdlb_lattice* build(const tdlb_config& c, int device) {
    validate_config(c);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        throw Fail{TDLB_ECUDA, "no CUDA device available (this library has no CPU path)"};
    if (device < 0 || device >= ndev) throw Fail{TDLB_EINVAL, "device index out of range"};
    cudaDeviceProp prop;
    TDLB_CK(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) throw Fail{TDLB_ECUDA, "this library is built for sm_100a (B200); device is sm_" +
                                                     std::to_string(prop.major) + std::to_string(prop.minor)};
    auto* h = new tdlb_lattice();
    try {
        h->cfg = c;
        h->device = device;
        h->vec = tdlb_rt::default_cells_per_thread(c);
        h->err.reserve(512);
        TDLB_CK(cudaSetDevice(device));
        TDLB_CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        // the forcing pass is the latency-bound critical path of a split
        // step: its streams get the highest priority, so its blocks are
        // scheduled ahead of the outer launch's as SMs free up
        int prio_lo = 0, prio_hi = 0;
        TDLB_CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
        TDLB_CK(cudaStreamCreateWithPriority(&h->side, cudaStreamNonBlocking, prio_hi));
        TDLB_CK(cudaStreamCreateWithPriority(&h->ibm, cudaStreamNonBlocking, prio_hi));
        TDLB_CK(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
        TDLB_CK(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
        TDLB_CK(cudaEventCreateWithFlags(&h->ev_outer, cudaEventDisableTiming));
        TDLB_CK(cudaEventCreateWithFlags(&h->ev_inner, cudaEventDisableTiming));
        TDLB_CK(cudaEventCreateWithFlags(&h->ev_sync, cudaEventDisableTiming));
        Dims& g = h->g;
        g = tdlb::make_dims((int)c.x, (int)c.y, (int)c.z);
        h->mask_words = round_up((long long)g.nx * g.ny * g.kw, 64);
        if ((long long)g.nx * g.ny * g.kp >= (1LL << 31) - 64)
            throw Fail{TDLB_EINVAL, "lattice too large: one population plane must stay below 2^31 elements"};
        if (tdlb::ibm_smem_bytes(g, 0) > 200 * 1024)
            throw Fail{TDLB_EINVAL, "x * ceil(z/32) too large for the per-plane IBM flag tile"};
        h->cp = tdlb::make_collide_params(c.nu, c.cs0, c.g3);
        tdlb::set_rest(h->cp, c.initialRho);

        const size_t pop_bytes = (size_t)tdlb::NQ * g.plane * h->esz();
        size_t free_b = 0, total_b = 0;
        TDLB_CK(cudaMemGetInfo(&free_b, &total_b));
        const size_t need = pop_bytes * (c.streaming == TDLB_STREAMING_SIMPLE ? 2 : 1) +
                            (size_t)5 * g.plane * sizeof(float) + 2 * h->mask_words * sizeof(uint32_t);   // F (float4), Nu
        if (need > free_b) throw Fail{TDLB_ENOMEM, "lattice needs " + std::to_string(need) + " B, " +
                                                       std::to_string(free_b) + " B free on device"};
        TDLB_CK(cudaMalloc(&h->bufA, pop_bytes));
        if (c.streaming == TDLB_STREAMING_SIMPLE) TDLB_CK(cudaMalloc(&h->bufB, pop_bytes));
        TDLB_CK(cudaMalloc(&h->Nu, (size_t)g.plane * sizeof(float)));
        TDLB_CK(cudaMalloc(&h->F, (size_t)4 * g.plane * sizeof(float)));
        TDLB_CK(cudaMalloc(&h->mask, (size_t)2 * h->mask_words * sizeof(uint32_t)));
        TDLB_CK(cudaMemsetAsync(h->bufA, 0, pop_bytes, h->stream));
        if (h->bufB) TDLB_CK(cudaMemsetAsync(h->bufB, 0, pop_bytes, h->stream));
        TDLB_CK(cudaMemsetAsync(h->Nu, 0, (size_t)g.plane * sizeof(float), h->stream));
        TDLB_CK(cudaMemsetAsync(h->F, 0, (size_t)4 * g.plane * sizeof(float), h->stream));
        TDLB_CK(cudaMemsetAsync(h->mask, 0, (size_t)2 * h->mask_words * sizeof(uint32_t), h->stream));
        TDLB_CK(cudaStreamSynchronize(h->stream));
    } catch (...) {
        release(h);
        delete h;
        throw;
    }
    return h;
}

// Reference JSON -> tdlb_config (main.cpp:135-164 reads these sections).
tdlb_config config_from_json(const char* text) {
    nlohmann::json j;
    try {
        j = nlohmann::json::parse(text);
    } catch (const std::exception& e) {
        throw Fail{TDLB_EJSON, std::string("input JSON: ") + e.what()};
    }
    tdlb_config c{};
    try {
        const auto& grid = j.at("GridParams");
        const auto& flow = j.at("FlowParams");
        c.x = (int64_t)grid.at("x").get<uint64_t>();
        c.y = (int64_t)grid.at("y").get<uint64_t>();
        c.z = (int64_t)grid.at("z").get<uint64_t>();
        const int64_t ghost = (int64_t)grid.value("multiStep", (uint64_t)1);
        if (ghost != 1) throw Fail{TDLB_EINVAL, "GridParams.multiStep (ghost width) must be 1"};
        c.initialRho = flow.at("initialRho").get<double>();
        c.nu = flow.at("nu").get<double>();
        c.cs0 = flow.at("cs0").get<double>();
        c.g3 = flow.at("g3").get<double>();
        c.alpha = flow.at("alpha").get<double>();
        c.beta = flow.at("beta").get<double>();
        c.useLES = flow.at("useLES").get<bool>() ? 1 : 0;
        // main.cpp:242-256: "Simple" selects Simple, anything else Esotwist
        c.streaming = flow.at("streaming").get<std::string>() == "Simple" ? TDLB_STREAMING_SIMPLE : TDLB_STREAMING_ESOTWIST;
        // nu as the file gives it: main.cpp constructs the ComputeUnit from
        // its FlowParams (:242-256) before calcNuAndRe_m (:275) sets nu in
        // main's own copy, so the reference's unit keeps the file's value.
        // The FlowParams fields are float in the reference (useQVecPrecision).
        c.initialRho = (double)(float)c.initialRho;
        c.nu = (double)(float)c.nu;
        c.cs0 = (double)(float)c.cs0;
        c.g3 = (double)(float)c.g3;
        c.alpha = (double)(float)c.alpha;
        c.beta = (double)(float)c.beta;
    } catch (const Fail&) {
        throw;
    } catch (const std::exception& e) {
        throw Fail{TDLB_EJSON, std::string("input JSON: ") + e.what()};
    }
    c.storage = TDLB_STORAGE_FP32;
    return c;
}

// Entry points run `fn` after joining the split-step stream (JOIN), so they
// see every queued step and forcing pass; the step loop's own calls
// (collision, forcing_resident, rotate_impeller, step) do not join.
template <bool JOIN = true, typename F>
int guarded(tdlb_lattice* h, F&& fn) {
    if (!h) return TDLB_EINVAL;
    try {
        cudaSetDevice(h->device);
        if (JOIN) TDLB_CK(tdlb_rt::join_side(h));
        fn();
        return TDLB_OK;
    } catch (const Fail& f) {
        h->err = f.msg;
        return f.code;
    } catch (const std::bad_alloc&) {
        h->err = "host allocation failed";
        return TDLB_ENOMEM;
    } catch (const std::exception& e) {
        h->err = e.what();
        return TDLB_EINVAL;
    }
}

void require_init(tdlb_lattice* h) {
    if (!h->initialised) throw Fail{TDLB_ESTATE, "call tdlb_initialise() first"};
}

tdlb::StepArgs step_args(tdlb_lattice* h, bool collide) {
    tdlb::StepArgs a{};
    a.A = h->planes(h->state_buf());
    if (h->cfg.streaming == TDLB_STREAMING_SIMPLE) a.B = h->planes(h->other_buf());
    a.Nu = h->Nu;
    a.F = reinterpret_cast<const float4*>(h->F);
    a.mask = h->mask_cur();
    a.g = h->g;
    a.p = h->cp;
    a.les = h->cfg.useLES;
    a.from_moments = h->holds_moments ? 1 : 0;
    a.collide = collide ? 1 : 0;
    a.even = h->even ? 1 : 0;
    a.vec = h->vec;
    a.l2_prefetch = h->l2_prefetch;
    a.storage = h->cfg.storage;
    // residual box (16-bit storage): Simple reads the state buffer's
    // residuals and writes the other buffer's; Esotwist updates its one set
    a.rr = h->rbox(h->state_index());
    a.rw = h->cfg.streaming == TDLB_STREAMING_SIMPLE ? h->rbox(1 - h->state_index()) : a.rr;
    return a;
}

// ---------------------------------------------------------------------------
// Split steps.
//
// The forcing pass reads and writes only cells inside the stencils of the
// markers, and the step reads F only there. The "zone" is a set of 32-element
// chunks of the flat row*kp + k index that holds every stencil cell of the
// resident markers at any impeller angle (and, for Esotwist, their 26
// neighbours: an Esotwist location of a stencil cell is also a location of
// its neighbours in the other parity). A step then runs as
//   stream: wait(inner of step s-1), outer chunks of step s
//   ibm:    forcing pass s-1 ... wait(outer of step s), inner chunks of step s,
//           forcing pass s
// so forcing pass s-1 runs concurrently with the outer chunks of step s:
// those cells neither read F nor share a population location with a stencil
// cell, and every cell computes exactly what the unsplit step computes.
// ---------------------------------------------------------------------------

// The split-step stream, ordered after everything queued on `stream` so far.
cudaStream_t loop_stream(tdlb_lattice* h) {
    if (!h->pending) {
        TDLB_CK(cudaEventRecord(h->ev_sync, h->stream));
        TDLB_CK(cudaStreamWaitEvent(h->ibm, h->ev_sync, 0));
        h->pending = true;
    }
    return h->ibm;
}

inline void mark_bit(std::vector<uint64_t>& b, long long e) { b[(size_t)(e >> 6)] |= 1ull << (e & 63); }
inline bool test_bit(const std::vector<uint64_t>& b, long long e) { return (b[(size_t)(e >> 6)] >> (e & 63)) & 1ull; }

// Every stencil cell of markers [b, e) lies in `core`.
bool stencils_inside(const tdlb_lattice* h, const tdlb_marker* m, size_t n, const std::vector<uint64_t>& core) {
    const Dims& g = h->g;
    for (size_t q = 0; q < n; q++) {
        int st[9];
        tdlb::MarkerSchedule::stencil(reinterpret_cast<const tdlb::Marker*>(m)[q], g.nx, g.nz, st);
        for (int c = 0; c < 9; c++) {
            const long long i = st[c] / g.nz, k = st[c] % g.nz;
            if (!test_bit(core, (i * g.ny + m[q].j) * g.kp + k)) return false;
        }
    }
    return true;
}

void build_zone(tdlb_lattice* h) {
    TDLB_CK(tdlb_rt::join_side(h));
    TDLB_CK(cudaStreamSynchronize(h->stream));   // no launch still reads the old zone
    const Dims& g = h->g;
    const long long nel = g.rows() * g.kp;
    std::vector<uint64_t> core((size_t)((nel + 63) / 64), 0ull);
    for (int e : h->cells.cell_e) mark_bit(core, e);   // first segment: its stencil cells, exactly
    const int n1 = h->n_markers - h->n0;
    const tdlb_marker* rot = h->h_markers.data() + h->n0;
    if (n1 > 0 && h->impeller_begin >= 0 && h->h_rot_xz.size() == 2 * (size_t)n1) {
        // Blades turn about (ci, ck). A blade marker at radius r rounds to the
        // nearest cell, and its stencil cells lie within 1.5 cells of that
        // position per axis, so within r +- 2.13 of the axis: mark, plane by
        // plane, the annulus between the smallest and the largest blade radius
        // widened by 3 cells.
        std::vector<double> rlo((size_t)g.ny, 1e300), rhi((size_t)g.ny, -1.0);
        for (int q = 0; q < n1; q++) {
            const double r = std::sqrt(h->h_rot_xz[2 * q] * h->h_rot_xz[2 * q] + h->h_rot_xz[2 * q + 1] * h->h_rot_xz[2 * q + 1]);
            const int j = (int)rot[q].j;
            rlo[(size_t)j] = std::min(rlo[(size_t)j], r);
            rhi[(size_t)j] = std::max(rhi[(size_t)j], r);
        }
        for (int j = 0; j < g.ny; j++) {
            if (rhi[(size_t)j] < 0) continue;
            const double lo = rlo[(size_t)j] - 3.0, hi = rhi[(size_t)j] + 3.0;
            const int i0 = std::max(0, (int)std::floor(h->rot_ci - hi)), i1 = std::min(g.nx - 1, (int)std::ceil(h->rot_ci + hi));
            const int k0 = std::max(0, (int)std::floor(h->rot_ck - hi)), k1 = std::min(g.nz - 1, (int)std::ceil(h->rot_ck + hi));
            for (int i = i0; i <= i1; i++)
                for (int k = k0; k <= k1; k++) {
                    const double d = std::sqrt((i - h->rot_ci) * (i - h->rot_ci) + (k - h->rot_ck) * (k - h->rot_ck));
                    if (d >= lo && d <= hi) mark_bit(core, ((long long)i * g.ny + j) * g.kp + k);
                }
        }
    } else {
        // blades set by the host without an attached impeller: their current cells
        for (int q = 0; q < n1; q++) {
            int st[9];
            tdlb::MarkerSchedule::stencil(reinterpret_cast<const tdlb::Marker*>(rot)[q], g.nx, g.nz, st);
            for (int c = 0; c < 9; c++) mark_bit(core, ((long long)(st[c] / g.nz) * g.ny + rot[q].j) * g.kp + st[c] % g.nz);
        }
    }
    std::vector<uint64_t> zone;
    if (h->cfg.streaming == TDLB_STREAMING_ESOTWIST) {
        zone.assign(core.size(), 0ull);
        for (size_t w = 0; w < core.size(); w++)
            for (uint64_t b = core[w]; b; b &= b - 1) {
                const long long e = (long long)w * 64 + __builtin_ctzll(b);
                const long long row = e / g.kp;
                const int k = (int)(e - row * g.kp), i = (int)(row / g.ny), j = (int)(row % g.ny);
                for (int di = -1; di <= 1; di++)
                    for (int dj = -1; dj <= 1; dj++)
                        for (int dk = -1; dk <= 1; dk++) {
                            const int a = (i + di + g.nx) % g.nx, b2 = (j + dj + g.ny) % g.ny, c = (k + dk + g.nz) % g.nz;
                            mark_bit(zone, ((long long)a * g.ny + b2) * g.kp + c);
                        }
            }
    } else {
        zone = core;
    }
    // 32-element chunks (half a word of `zone`): the inner ones (any element
    // in the zone), then the outer ones
    static_assert(tdlb::kSplitChunk == 32, "chunk = half a word of the zone bitset");
    const long long nchunks = (nel + 31) / 32;
    std::vector<uint32_t> bits((size_t)((nchunks + 31) / 32), 0u);
    std::vector<int> list, outer;
    long long inner_cells = 0;   // interior cells of the inner chunks
    for (long long c = 0; c < nchunks; c++) {
        const uint32_t half = (uint32_t)(zone[(size_t)(c >> 1)] >> ((c & 1) * 32));
        if (half) {
            bits[(size_t)(c >> 5)] |= 1u << (c & 31);
            list.push_back((int)c);
            for (long long e = c * 32; e < std::min(c * 32 + 32, nel); e++) inner_cells += (e % g.kp) < g.nz;
        } else {
            outer.push_back((int)c);
        }
    }
    const long long n_in = (long long)list.size();
    list.insert(list.end(), outer.begin(), outer.end());
    if ((long long)list.size() > h->zone_list_cap || !h->d_zone_list) {
        cudaFree(h->d_zone_list);
        h->d_zone_list = nullptr;
        TDLB_CK(cudaMalloc(&h->d_zone_list, list.size() * sizeof(int)));
        h->zone_list_cap = (long long)list.size();
    }
    TDLB_CK(cudaMemcpyAsync(h->d_zone_list, list.data(), list.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    TDLB_CK(cudaStreamSynchronize(h->stream));
    h->n_zone = (int)n_in;
    h->n_outer = (int)(nchunks - n_in);
    h->zone_small = (double)inner_cells <= 0.6 * (double)g.rows() * (double)g.nz;
    h->h_zone_bits = std::move(bits);
    h->zone_ok = stencils_inside(h, rot, (size_t)std::max(n1, 0), core);
    h->h_zone_core = std::move(core);
    h->zone_gen = h->marker_gen;
}

// Forcing passes may go to the split-step stream (the next step can split).
bool split_capable(tdlb_lattice* h) {
    if (!h->overlap || h->own_stream || h->vec != 1 || !h->markers_set || !h->resident) return false;
    if (h->zone_gen != h->marker_gen) build_zone(h);
    // a zone covering most of the lattice leaves little to overlap with
    return h->zone_ok && (h->zone_small || h->overlap == 2);
}

// (A step with a residual box runs unsplit: its box launch reads the box
// chunks' populations and Nu before the plain launch writes them.)
bool can_split(tdlb_lattice* h) {
    if (h->rbox_geom.n) return false;
    return !h->holds_moments && split_capable(h);
}

// The chunks with a cell near the residual box (ResidualBox::near), which the
// box launch of a step runs, and that launch's scratch outputs.
void build_box_list(tdlb_lattice* h) {
    if (h->box_list_gen == h->box_gen) return;
    TDLB_CK(tdlb_rt::join_side(h));
    TDLB_CK(cudaStreamSynchronize(h->stream));   // no launch still reads the old list
    const Dims& g = h->g;
    const tdlb::ResidualBox& b = h->rbox_geom;
    const long long nchunks = (g.rows() * g.kp + 31) / 32;
    std::vector<uint8_t> hit((size_t)nchunks, 0);
    for (int i = std::max(0, b.i0 - 1); i <= std::min(g.nx - 1, b.i0 + b.bx); i++)
        for (int j = std::max(0, b.j0 - 1); j <= std::min(g.ny - 1, b.j0 + b.by); j++)
            for (int k = std::max(0, b.k0 - 1); k <= std::min(g.nz - 1, b.k0 + b.bz); k++)
                if (b.around(i, j, k)) hit[(size_t)((((long long)i * g.ny + j) * g.kp + k) >> 5)] = 1;
    std::vector<int> list;
    for (long long c = 0; c < nchunks; c++)
        if (hit[(size_t)c]) list.push_back((int)c);
    if ((long long)list.size() > h->box_list_cap || !h->d_box_list) {
        cudaFree(h->d_box_list);
        h->d_box_list = nullptr;
        h->box_list_cap = 0;
        TDLB_CK(cudaMalloc(&h->d_box_list, std::max<size_t>(list.size(), 1) * sizeof(int)));
        h->box_list_cap = (long long)std::max<size_t>(list.size(), 1);
    }
    {
        // one entry per thread of the box launch (128-thread blocks)
        const long long need = (long long)(tdlb::NQ + 1) * (((long long)list.size() * 32 + 127) / 128 * 128);
        if (need > h->box_out_cap || !h->d_box_out) {
            cudaFree(h->d_box_out);
            h->d_box_out = nullptr;
            h->box_out_cap = 0;
            TDLB_CK(cudaMalloc(&h->d_box_out, (size_t)std::max<long long>(need, 1) * sizeof(float)));
            h->box_out_cap = std::max<long long>(need, 1);
        }
    }
    if (!list.empty())
        TDLB_CK(cudaMemcpyAsync(h->d_box_list, list.data(), list.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    TDLB_CK(cudaStreamSynchronize(h->stream));
    h->n_box = (int)list.size();
    h->box_list_gen = h->box_gen;
}

// Queue one step-kernel launch, bracketed by timing events when enabled.
template <typename L>
void timed_launch(tdlb_lattice* h, cudaStream_t st, L&& launch) {
    h->launches++;
    if (!h->timing) {
        TDLB_CK(launch());
        return;
    }
    cudaEvent_t a = nullptr, b = nullptr;
    TDLB_CK(cudaEventCreate(&a));
    if (cudaEventCreate(&b) != cudaSuccess) {
        cudaEventDestroy(a);
        throw Fail{TDLB_ECUDA, "cudaEventCreate failed"};
    }
    h->tev.push_back(a);
    h->tev.push_back(b);
    TDLB_CK(cudaEventRecord(a, st));
    TDLB_CK(launch());
    TDLB_CK(cudaEventRecord(b, st));
}

void run_step(tdlb_lattice* h, bool collide) {
    tdlb::StepArgs a = step_args(h, collide);
    const bool simple = h->cfg.streaming == TDLB_STREAMING_SIMPLE;
    auto launch = [&](const tdlb::StepArgs& x, cudaStream_t st) {
        return simple ? tdlb::launch_step_simple(x, st) : tdlb::launch_step_esotwist(x, st);
    };
    // With a residual box: the box launch (the chunks near the box, with
    // residuals, into scratch), the plain launch, then the commit of the box
    // chunks' outputs (step_kernels.cuh). Such a step is never split.
    const bool boxed = a.rr.on();
    if (boxed) build_box_list(h);
    tdlb::StepArgs bx = a;
    bx.box = 2;
    bx.part = 2;
    bx.vec = 1;   // the box launches run one cell per thread, whatever the plain launch's variant
    bx.zone = tdlb::StepPart{h->d_box_list, h->n_box};
    bx.bout = tdlb::BoxOut{h->d_box_out, ((long long)h->n_box * 32 + 127) / 128 * 128};
    const bool run_box = boxed && h->n_box > 0;
    if (collide && can_split(h)) {
        cudaStream_t side = loop_stream(h);
        if (h->inner_queued) TDLB_CK(cudaStreamWaitEvent(h->stream, h->ev_inner, 0));
        if (h->n_outer > 0) {
            a.part = 1;
            a.zone = tdlb::StepPart{h->d_zone_list + h->n_zone, h->n_outer};
            timed_launch(h, h->stream, [&] { return launch(a, h->stream); });
        }
        TDLB_CK(cudaEventRecord(h->ev_outer, h->stream));
        TDLB_CK(cudaStreamWaitEvent(side, h->ev_outer, 0));
        if (h->n_zone > 0) {
            a.part = 2;
            a.zone = tdlb::StepPart{h->d_zone_list, h->n_zone};
            timed_launch(h, side, [&] { return launch(a, side); });
        }
        TDLB_CK(cudaEventRecord(h->ev_inner, side));
        h->inner_queued = true;
    } else {
        TDLB_CK(tdlb_rt::join_side(h));
        if (run_box) timed_launch(h, h->stream, [&] { return launch(bx, h->stream); });
        timed_launch(h, h->stream, [&] { return launch(a, h->stream); });
        if (run_box) timed_launch(h, h->stream, [&] { return tdlb::launch_box_commit(bx, simple, h->stream); });
    }
    if (simple) h->cur ^= 1;
    else h->even = !h->even;   // StreamingEsoteric.hpp:15-18
    h->holds_moments = false;
}

tdlb::IbmArgs ibm_args(tdlb_lattice* h, float alpha, float beta);

void validate_markers(const Dims& g, const tdlb_marker* m, size_t n, size_t base) {
    for (size_t q = 0; q < n; q++) {
        if (m[q].i < 0 || m[q].i >= g.nx || m[q].j < 0 || m[q].j >= g.ny || m[q].k < 0 || m[q].k >= g.nz) {
            char buf[160];
            std::snprintf(buf, sizeof buf, "marker %zu at (%lld,%lld,%lld) outside the %dx%dx%d interior", base + q,
                          (long long)m[q].i, (long long)m[q].j, (long long)m[q].k, g.nx, g.ny, g.nz);
            throw Fail{TDLB_EINVAL, buf};
        }
    }
}

// Grow the level-pointer array, keeping its contents (the first segment's
// levels stay valid when only the blade schedule grows).
void ensure_level_cap(tdlb_lattice* h, long long need) {
    if (need <= h->level_cap && h->d_level_ptr) return;
    TDLB_CK(cudaStreamSynchronize(h->stream));
    const long long cap = std::max<long long>(round_up(need * 2, 1024), 1024);
    int* p = nullptr;
    TDLB_CK(cudaMalloc(&p, cap * sizeof(int)));
    if (h->d_level_ptr) {
        const cudaError_t e = cudaMemcpy(p, h->d_level_ptr, (size_t)h->level_cap * sizeof(int), cudaMemcpyDeviceToDevice);
        if (e != cudaSuccess) {
            cudaFree(p);
            TDLB_CK(e);
        }
        cudaFree(h->d_level_ptr);
    }
    h->d_level_ptr = p;
    h->level_cap = cap;
}

// Device copy of the second segment's schedule (slots n0.., levels L0..).
// The planes whose second segment (blades) has levels, for the blade launch
// of the forcing pass, and its shared memory; uploaded when they change.
void update_blade_planes(tdlb_lattice* h) {
    const Dims& g = h->g;
    const auto& lv = h->seg1.plane_lv;
    const auto& lp = h->seg1.level_ptr;
    const int L0 = h->seg0.nlevels;
    std::vector<int> planes;
    int words = 0;
    for (int j = 0; j < g.ny; j++) {
        if (lv[(size_t)j] == lv[(size_t)j + 1]) continue;
        planes.push_back(j);
        // the level ranges are global level indices; seg1's level_ptr starts at level L0
        const int nb = lp[(size_t)(lv[(size_t)j + 1] - L0)] - lp[(size_t)(lv[(size_t)j] - L0)];
        words = std::max(words, tdlb::blade_table_words(nb));
    }
    words = std::min(words, 220 * 1024 / 4);   // a plane beyond this walks its blades on global memory
    if (planes != h->h_blade_planes) {
        if (!h->d_blade_planes) TDLB_CK(cudaMalloc(&h->d_blade_planes, (size_t)std::max(g.ny, 1) * sizeof(int)));
        h->h_blade_planes = planes;
        if (!planes.empty())
            TDLB_CK(cudaMemcpyAsync(h->d_blade_planes, h->h_blade_planes.data(), planes.size() * sizeof(int),
                                    cudaMemcpyHostToDevice, h->stream));
        h->n_blade = (int)planes.size();
    }
    if (words > h->blade_words) TDLB_CK(tdlb::ibm_prepare_blades(words));
    h->blade_words = std::max(h->blade_words, words);
}

void upload_seg1(tdlb_lattice* h) {
    const Dims& g = h->g;
    update_blade_planes(h);
    const int L0 = h->seg0.nlevels;
    ensure_level_cap(h, (long long)L0 + h->seg1.nlevels + 1);
    const int n1 = h->n_markers - h->n0;
    if (n1) TDLB_CK(cudaMemcpyAsync(h->d_sched + h->n0, h->seg1.order.data(), (size_t)n1 * sizeof(int),
                                    cudaMemcpyHostToDevice, h->stream));
    TDLB_CK(cudaMemcpyAsync(h->d_level_ptr + L0, h->seg1.level_ptr.data(), h->seg1.level_ptr.size() * sizeof(int),
                            cudaMemcpyHostToDevice, h->stream));
    TDLB_CK(cudaMemcpyAsync(h->d_plane_lv1, h->seg1.plane_lv.data(), (size_t)(g.ny + 1) * sizeof(int),
                            cudaMemcpyHostToDevice, h->stream));
}

// Make `m[0, n)` the resident list: segment 0 = [0, n0) with exact levels,
// segment 1 = [n0, n), rotation-invariant when rot_xz is given.
void upload_markers(tdlb_lattice* h, const tdlb_marker* m, size_t n, size_t n0, const double* rot_xz) {
    if (n > 0 && !m) throw Fail{TDLB_EINVAL, "markers is NULL"};
    if (n > (size_t)0x7fffffff) throw Fail{TDLB_EINVAL, "too many markers"};
    const Dims& g = h->g;
    validate_markers(g, m, n, 0);
    static_assert(sizeof(tdlb_marker) == sizeof(tdlb::Marker), "marker layout");
    TDLB_CK(cudaStreamSynchronize(h->stream));   // host vectors below are read by queued copies
    h->h_markers.assign(m, m + n);
    const auto* mk = reinterpret_cast<const tdlb::Marker*>(h->h_markers.data());
    h->n_markers = (int)n;
    h->n0 = (int)n0;
    h->seg0.build(mk, 0, (int)n0, g.nx, g.ny, g.nz, 0, 0);
    h->seg1.build(mk, (int)n0, (int)n, g.nx, g.ny, g.nz, (int)n0, h->seg0.nlevels, rot_xz);
    if ((long long)n > h->marker_cap) {
        cudaFree(h->d_markers); cudaFree(h->d_sched); cudaFree(h->d_sums);
        h->d_markers = nullptr; h->d_sched = nullptr; h->d_sums = nullptr;
        const long long cap = std::max<long long>(round_up((long long)n, 1024), 1024);
        TDLB_CK(cudaMalloc(&h->d_markers, cap * sizeof(tdlb::Marker)));
        TDLB_CK(cudaMalloc(&h->d_sched, cap * sizeof(int)));
        TDLB_CK(cudaMalloc(&h->d_sums, (size_t)3 * cap * sizeof(float)));
        h->marker_cap = cap;
    }
    const long long ntail = (long long)n - (long long)n0;
    if (ntail > h->tail_cap) {
        cudaFree(h->d_tail);
        h->d_tail = nullptr;
        const long long cap = round_up(ntail, 256);
        TDLB_CK(cudaMalloc(&h->d_tail, (size_t)tdlb::TF_COUNT * cap * sizeof(float)));
        h->tail_cap = cap;
    }
    // first segment: unique cells per plane, slot data
    h->cells.build(mk, h->seg0, g.nx, g.ny, g.nz, g.kp);
    const long long C0 = (long long)h->cells.cell_e.size();
    cudaFree(h->d_cell_e); cudaFree(h->d_plane_cell); cudaFree(h->d_prep); cudaFree(h->d_cell_m); cudaFree(h->d_cell_F);
    h->d_cell_e = nullptr; h->d_plane_cell = nullptr; h->d_prep = nullptr; h->d_cell_m = nullptr; h->d_cell_F = nullptr;
    TDLB_CK(cudaMalloc(&h->d_plane_cell, (size_t)(g.ny + 1) * sizeof(int)));
    if (C0) {
        // 16 elements of padding: the spread's bulk copies and L2 prefetches
        // round a plane's cell range out to 16-byte boundaries
        TDLB_CK(cudaMalloc(&h->d_cell_e, (C0 + 16) * sizeof(int)));
        TDLB_CK(cudaMalloc(&h->d_cell_m, (4 * C0 + 16) * sizeof(float)));
        TDLB_CK(cudaMalloc(&h->d_cell_F, (3 * C0 + 16) * sizeof(float)));
    }
    if (n0) TDLB_CK(cudaMalloc(&h->d_prep, ((size_t)tdlb::PF_STRIDE * n0 + 16) * sizeof(float)));
    {
        // F tiles of the ordinary planes' launch: up to 6144 cells (72 KB)
        // of shared memory;
        // the tile is sized for the most crowded ordinary plane, at least
        // 4608 cells. Planes with more cells (an impeller disk) go to a
        // second, 512-thread launch with a tile for the largest of them
        // (global memory beyond the 227 KB shared-memory limit).
        int typical = 0;
        for (int j = 0; j < g.ny; j++) {
            const int nc = h->cells.plane_cell[(size_t)j + 1] - h->cells.plane_cell[(size_t)j];
            if (nc <= 6144) typical = std::max(typical, nc);
        }
        const int small_cap = std::max(4608, round_up(typical, 64) > 6144 ? 6144 : (int)round_up(typical, 64));
        std::vector<int> small, big;
        int big_max = 0;
        for (int j = 0; j < g.ny; j++) {
            const int nc = h->cells.plane_cell[(size_t)j + 1] - h->cells.plane_cell[(size_t)j];
            if (nc > small_cap) { big.push_back(j); big_max = std::max(big_max, nc); }
            else small.push_back(j);
        }
        h->smem_cells = small_cap;
        h->n_small = (int)small.size();
        h->n_big = (int)big.size();
        h->big_tile_cells = tdlb::big_bulk_bytes(big_max) <= 220 * 1024 ? big_max : 0;
        TDLB_CK(tdlb::ibm_prepare_smem(h->smem_cells, h->n_small, tdlb::big_bulk_bytes(h->big_tile_cells)));
        // cell order of the pass: the big planes' cells, then the others
        cudaFree(h->d_cell_order);
        h->d_cell_order = nullptr;
        h->ncell_big = 0;
        if (!big.empty() && C0) {
            std::vector<char> is_big((size_t)g.ny, 0);
            for (int j : big) is_big[(size_t)j] = 1;
            std::vector<int> order;
            order.reserve((size_t)C0);
            for (int pass = 1; pass >= 0; pass--)
                for (int j = 0; j < g.ny; j++)
                    if (is_big[(size_t)j] == pass)
                        for (int c = h->cells.plane_cell[(size_t)j]; c < h->cells.plane_cell[(size_t)j + 1]; c++)
                            order.push_back(c);
            for (int j : big) h->ncell_big += h->cells.plane_cell[(size_t)j + 1] - h->cells.plane_cell[(size_t)j];
            TDLB_CK(cudaMalloc(&h->d_cell_order, order.size() * sizeof(int)));
            TDLB_CK(cudaMemcpy(h->d_cell_order, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice));
        }
        small.insert(small.end(), big.begin(), big.end());
        if (!h->d_plane_list) TDLB_CK(cudaMalloc(&h->d_plane_list, (size_t)g.ny * sizeof(int)));
        TDLB_CK(cudaMemcpy(h->d_plane_list, small.data(), (size_t)g.ny * sizeof(int), cudaMemcpyHostToDevice));
        h->h_plane_list = small;
    }
    // static touched flags of the first segment
    {
        std::vector<uint32_t> ms((size_t)h->mask_words, 0u);
        for (int e : h->cells.cell_e) {
            const int row = e / g.kp, k = e - row * g.kp;
            ms[(size_t)row * g.kw + (k >> 5)] |= 1u << (k & 31);
        }
        if (!h->d_mask_static) TDLB_CK(cudaMalloc(&h->d_mask_static, (size_t)h->mask_words * sizeof(uint32_t)));
        TDLB_CK(cudaMemcpy(h->d_mask_static, ms.data(), ms.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    }
    if (!h->d_plane_lv0) {
        TDLB_CK(cudaMalloc(&h->d_plane_lv0, (size_t)(g.ny + 1) * sizeof(int)));
        TDLB_CK(cudaMalloc(&h->d_plane_lv1, (size_t)(g.ny + 1) * sizeof(int)));
    }
    ensure_level_cap(h, (long long)h->seg0.nlevels + h->seg1.nlevels + 1);
    if (n) TDLB_CK(cudaMemcpyAsync(h->d_markers, m, n * sizeof(tdlb::Marker), cudaMemcpyHostToDevice, h->stream));
    if (n0) TDLB_CK(cudaMemcpyAsync(h->d_sched, h->seg0.order.data(), n0 * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    TDLB_CK(cudaMemcpyAsync(h->d_level_ptr, h->seg0.level_ptr.data(), h->seg0.level_ptr.size() * sizeof(int),
                            cudaMemcpyHostToDevice, h->stream));
    TDLB_CK(cudaMemcpyAsync(h->d_plane_lv0, h->seg0.plane_lv.data(), (size_t)(g.ny + 1) * sizeof(int),
                            cudaMemcpyHostToDevice, h->stream));
    upload_seg1(h);
    TDLB_CK(cudaMemcpyAsync(h->d_plane_cell, h->cells.plane_cell.data(), (size_t)(g.ny + 1) * sizeof(int),
                            cudaMemcpyHostToDevice, h->stream));
    if (C0) TDLB_CK(cudaMemcpyAsync(h->d_cell_e, h->cells.cell_e.data(), C0 * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    if (n0) {
        // the 9 cell indices of each slot into its prep row
        TDLB_CK(cudaMemcpy2DAsync(h->d_prep + tdlb::PF_CELL, tdlb::PF_STRIDE * sizeof(float), h->cells.mcell.data(),
                                  9 * sizeof(int), 9 * sizeof(int), (size_t)n0, cudaMemcpyHostToDevice, h->stream));
        tdlb::IbmArgs a = ibm_args(h, 0.f, 0.f);
        TDLB_CK(tdlb::launch_ibm_prepare(a, h->d_prep, nullptr, h->stream));
    }
    TDLB_CK(cudaStreamSynchronize(h->stream));
    h->markers_set = true;
    h->rot_device = false;
    h->impeller_begin = -1;
    h->marker_gen++;
}

tdlb::IbmArgs ibm_args(tdlb_lattice* h, float alpha, float beta) {
    tdlb::IbmArgs a{};
    a.markers = h->d_markers;
    a.sched = h->d_sched;
    a.level_ptr = h->d_level_ptr;
    a.plane_lv0 = h->d_plane_lv0;
    a.plane_lv1 = h->d_plane_lv1;
    a.n = h->n_markers;
    a.n0 = h->n0;
    a.cell_e = h->d_cell_e;
    a.plane_cell = h->d_plane_cell;
    a.ncell = (int)h->cells.cell_e.size();
    a.cell_order = h->d_cell_order;
    a.ncell_big = h->ncell_big;
    a.prep = h->d_prep;
    a.cell_m = h->d_cell_m;
    a.cell_F = h->d_cell_F;
    a.tail = h->d_tail;
    a.tail_cap = h->tail_cap;
    a.sums = h->d_sums;
    a.smem_cells = h->smem_cells;
    a.plane_list = h->d_plane_list;
    a.n_small = h->n_small;
    a.n_big = h->n_big;
    a.blade_planes = h->d_blade_planes;
    a.n_blade = h->n_blade;
    a.blade_words = h->blade_words;
    a.big_tile_cells = h->big_tile_cells;
    a.side = h->side;
    a.ev_fork = h->ev_fork;
    a.ev_join = h->ev_join;
    a.A = h->planes(h->state_buf());
    a.state_mode = h->state_mode();
    a.even = h->even ? 1 : 0;
    a.F4 = reinterpret_cast<float4*>(h->F);
    a.mask_old = h->mask_cur();
    a.mask_new = h->mask_next();
    a.mask_static = h->d_mask_static;
    a.mask_bytes = (size_t)h->mask_words * sizeof(uint32_t);
    a.g = h->g;
    a.alpha = alpha;
    a.beta = beta;
    a.storage = h->cfg.storage;
    a.p = h->cp;
    a.rbox = h->rbox(h->state_index());
    return a;
}

// Stream of a forcing pass or blade rotation: the split-step stream when the
// next step can split, else the handle's stream.
cudaStream_t ibm_stream(tdlb_lattice* h) {
    if (split_capable(h)) return loop_stream(h);
    TDLB_CK(tdlb_rt::join_side(h));
    return h->stream;
}

void run_forcing(tdlb_lattice* h, float alpha, float beta) {
    if (!h->markers_set) throw Fail{TDLB_ESTATE, "no markers set (tdlb_set_markers / tdlb_forcing)"};
    TDLB_CK(tdlb::launch_ibm(ibm_args(h, alpha, beta), ibm_stream(h)));
    h->launches += (h->cells.cell_e.empty() ? 0 : 1) + (h->n_markers > h->n0 ? 1 : 0) + (h->n_small > 0 ? 1 : 0) +
                   (h->n_big > 0 ? 1 : 0) + (h->n_blade > 0 ? 1 : 0);
    h->pass++;
    h->last_beta = beta;
}

// Copy an interior-cell plane set (npl planes of the device layout) to a
// host AoS array out[cell*npl + l], cells in (i, j, k) order.
void planes_to_host_aos(tdlb_lattice* h, const float* dev, int npl, float* out) {
    const Dims& g = h->g;
    std::vector<float> tmp((size_t)npl * g.plane);
    TDLB_CK(cudaMemcpyAsync(tmp.data(), dev, tmp.size() * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    TDLB_CK(cudaStreamSynchronize(h->stream));
    size_t c = 0;
    for (int i = 0; i < g.nx; i++)
        for (int j = 0; j < g.ny; j++)
            for (int k = 0; k < g.nz; k++, c++) {
                const size_t e = ((size_t)i * g.ny + j) * g.kp + k;
                for (int l = 0; l < npl; l++) out[c * npl + l] = tmp[(size_t)l * g.plane + e];
            }
}

// The force field (one float4 per element) as (Fx, Fy, Fz) per interior cell.
void force_to_host(tdlb_lattice* h, float* out3) {
    const Dims& g = h->g;
    std::vector<float> tmp((size_t)4 * g.plane);
    TDLB_CK(cudaMemcpyAsync(tmp.data(), h->F, tmp.size() * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    TDLB_CK(cudaStreamSynchronize(h->stream));
    size_t c = 0;
    for (int i = 0; i < g.nx; i++)
        for (int j = 0; j < g.ny; j++)
            for (int k = 0; k < g.nz; k++, c++) {
                const size_t e = ((size_t)i * g.ny + j) * g.kp + k;
                for (int l = 0; l < 3; l++) out3[c * 3 + l] = tmp[4 * e + (size_t)l];
            }
}

void host_aos_to_planes(tdlb_lattice* h, const float* in, int npl, float* dev) {
    const Dims& g = h->g;
    std::vector<float> tmp((size_t)npl * g.plane, 0.f);
    size_t c = 0;
    for (int i = 0; i < g.nx; i++)
        for (int j = 0; j < g.ny; j++)
            for (int k = 0; k < g.nz; k++, c++) {
                const size_t e = ((size_t)i * g.ny + j) * g.kp + k;
                for (int l = 0; l < npl; l++) tmp[(size_t)l * g.plane + e] = in[c * npl + l];
            }
    TDLB_CK(cudaMemcpyAsync(dev, tmp.data(), tmp.size() * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    TDLB_CK(cudaStreamSynchronize(h->stream));
}

// Moments of the current state into a temporary 18-plane device buffer.
float* state_moments(tdlb_lattice* h) {
    float* M = nullptr;
    TDLB_CK(cudaMalloc(&M, (size_t)tdlb::NQ * h->g.plane * sizeof(float)));
    cudaError_t e = tdlb::launch_state_moments(h->planes(h->state_buf()), h->planes32(M), h->g, h->state_mode(),
                                               h->even ? 1 : 0, h->stream, h->cfg.storage, h->cp,
                                               h->rbox(h->state_index()));
    if (e != cudaSuccess) {
        cudaFree(M);
        throw Fail{TDLB_ECUDA, std::string("state moments: ") + cudaGetErrorString(e)};
    }
    return M;
}

struct DevBuf {
    float* p;
    ~DevBuf() { cudaFree(p); }
};

// ---------------------------------------------------------------------------
// Residual box of the 16-bit storage (tdlb::ResidualBox): exact deviations
// for every population location inside a box of cells.
// ---------------------------------------------------------------------------
void drop_rbox(tdlb_lattice* h) {
    cudaFree(h->d_res[0]);
    cudaFree(h->d_res[1]);
    h->d_res[0] = h->d_res[1] = nullptr;
    h->rbox_geom = tdlb::ResidualBox{};
    h->box_gen++;
}

// The box [i0, i1) x [j0, j1) x [k0, k1); an empty one removes the box. The
// residuals start at zero: every location holds its 16-bit value exactly,
// and steps refine the locations inside the box from then on.
void set_rbox(tdlb_lattice* h, long long i0, long long i1, long long j0, long long j1, long long k0, long long k1) {
    const Dims& g = h->g;
    if (i1 <= i0 || j1 <= j0 || k1 <= k0) {
        drop_rbox(h);
        return;
    }
    // a rejected box leaves the current one in place
    if (h->cfg.storage == TDLB_STORAGE_FP32) throw Fail{TDLB_EINVAL, "a residual box needs 16-bit storage (FP32 storage is exact)"};
    if (h->own_stream) throw Fail{TDLB_ESTATE, "a tank of a batch has no residual box"};
    // no box cell at index 0: an Esotwist location that wraps around the
    // lattice (index 0) then never lies in the box
    if (i0 < 1 || j0 < 1 || k0 < 1 || i1 > g.nx || j1 > g.ny || k1 > g.nz)
        throw Fail{TDLB_EINVAL, "the residual box must lie within [1, x) x [1, y) x [1, z)"};
    drop_rbox(h);
    tdlb::ResidualBox b;
    b.i0 = (int)i0; b.j0 = (int)j0; b.k0 = (int)k0;
    b.bx = (int)(i1 - i0); b.by = (int)(j1 - j0); b.bz = (int)(k1 - k0);
    b.n = (long long)b.bx * b.by * b.bz;
    const int sets = h->cfg.streaming == TDLB_STREAMING_SIMPLE ? 2 : 1;
    for (int q = 0; q < sets; q++) {
        const size_t bytes = (size_t)tdlb::NQ * (size_t)b.n * sizeof(float);
        cudaError_t e = cudaMalloc(&h->d_res[q], bytes);
        if (e != cudaSuccess) {
            drop_rbox(h);
            throw Fail{TDLB_ENOMEM, "residual box: " + std::string(cudaGetErrorString(e))};
        }
        TDLB_CK(cudaMemsetAsync(h->d_res[q], 0, bytes, h->stream));
    }
    h->rbox_geom = b;
    h->box_gen++;
}

// Residuals back to zero, after anything wrote the 16-bit planes without
// them (initialise, checkpoint read).
void clear_rbox(tdlb_lattice* h) {
    for (int q = 0; q < 2; q++)
        if (h->d_res[q])
            TDLB_CK(cudaMemsetAsync(h->d_res[q], 0, (size_t)tdlb::NQ * (size_t)h->rbox_geom.n * sizeof(float), h->stream));
}

// The impeller's swept volume with a margin of 4 cells: the blades' radius
// about the axis and their planes. There the 16-bit rounding of the stored
// deviations is what sets the velocity error against FP64 (FP32 storage in
// this volume alone brings FP16 from 2.2e-3 to about 6e-4 after 2000 steps
// of a 120^3 tank at Re 20000).
void auto_rbox(tdlb_lattice* h, const tdlb::RushtonGeom& G, const std::vector<tdlb::RotatingPolar>& pol, double rmax) {
    if (h->cfg.storage == TDLB_STORAGE_FP32 || !h->rbox_auto || h->own_stream || pol.empty()) return;
    long long jmin = pol[0].j, jmax = pol[0].j;
    for (const tdlb::RotatingPolar& p : pol) {
        jmin = std::min(jmin, p.j);
        jmax = std::max(jmax, p.j);
    }
    const double r = rmax + 4.0;
    const Dims& g = h->g;
    auto lo = [](double v) { return std::max(1LL, (long long)std::floor(v)); };
    set_rbox(h, lo(G.ci - r), std::min<long long>(g.nx, (long long)std::ceil(G.ci + r) + 1), std::max(1LL, jmin - 4),
             std::min<long long>(g.ny, jmax + 5), lo(G.ck - r), std::min<long long>(g.nz, (long long)std::ceil(G.ck + r) + 1));
}

}  // namespace

extern "C" {

int tdlb_create_config(const tdlb_config* cfg, int device, tdlb_handle* out) {
    if (!cfg || !out) {
        g_create_error = "NULL argument";
        return TDLB_EINVAL;
    }
    *out = nullptr;
    try {
        *out = build(*cfg, device);
        return TDLB_OK;
    } catch (const Fail& f) {
        g_create_error = f.msg;
        return f.code;
    } catch (const std::bad_alloc&) {
        g_create_error = "host allocation failed";
        return TDLB_ENOMEM;
    }
}

int tdlb_create(const char* params_json, int device, tdlb_handle* out) {
    if (!params_json || !out) {
        g_create_error = "NULL argument";
        return TDLB_EINVAL;
    }
    *out = nullptr;
    try {
        tdlb_config c = config_from_json(params_json);
        *out = build(c, device);
        return TDLB_OK;
    } catch (const Fail& f) {
        g_create_error = f.msg;
        return f.code;
    } catch (const std::bad_alloc&) {
        g_create_error = "host allocation failed";
        return TDLB_ENOMEM;
    }
}

int tdlb_config_from_json(const char* params_json, tdlb_config* out) {
    if (!params_json || !out) {
        g_create_error = "NULL argument";
        return TDLB_EINVAL;
    }
    try {
        *out = config_from_json(params_json);
        return TDLB_OK;
    } catch (const Fail& f) {
        g_create_error = f.msg;
        return f.code;
    }
}

int tdlb_lattice_bytes(const tdlb_config* c, int64_t* bytes) {
    if (!c || !bytes || c->x < 1 || c->y < 1 || c->z < 1) return TDLB_EINVAL;
    const long long kp = round_up(c->z, tdlb::kRowPitch), kw = (kp + 31) / 32;
    const long long plane = round_up(c->x * c->y * kp, 64);
    const long long mask_words = round_up(c->x * c->y * kw, 64);
    const long long esz = c->storage == TDLB_STORAGE_FP32 ? 4 : 2;
    const long long pops = (long long)tdlb::NQ * plane * esz * (c->streaming == TDLB_STREAMING_SIMPLE ? 2 : 1);
    // fields, flags, and the marker buffers of a tank-wall geometry
    // (about 8 markers per (i, j) column at most, 256 bytes each with
    // their schedule, stencil-cell and per-pass data)
    *bytes = pops + 5 * plane * 4 + 2 * mask_words * 4 + 8 * c->x * c->y * 256;   // F (float4) and Nu: 5 planes
    return TDLB_OK;
}

int tdlb_destroy(tdlb_handle h) {
    if (!h) return TDLB_EINVAL;
    release(h);
    delete h;
    return TDLB_OK;
}

const char* tdlb_last_error(tdlb_handle h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int tdlb_initialise(tdlb_handle h, float rho) {
    return guarded(h, [&] {
        const Dims& g = h->g;
        h->cur = 0;
        h->even = true;
        h->holds_moments = true;
        h->pass = 0;
        if (h->cfg.storage == TDLB_STORAGE_FP32) {
            TDLB_CK(tdlb::launch_fill_uniform_moments(h->planes(h->bufA), g, rho, h->stream));
        } else {
            // 16-bit storage holds populations only: the rest populations of
            // rho have the same moments (rho, 0, ..., 0) as the reference's Q
            TDLB_CK(tdlb::launch_fill_rest(h->planes(h->bufA), g.plane, rho, (float)h->cfg.initialRho, h->cfg.storage,
                                           h->cp, h->stream));
            h->holds_moments = false;
        }
        TDLB_CK(cudaMemsetAsync(h->Nu, 0, (size_t)g.plane * sizeof(float), h->stream));
        TDLB_CK(cudaMemsetAsync(h->F, 0, (size_t)4 * g.plane * sizeof(float), h->stream));
        TDLB_CK(cudaMemsetAsync(h->mask, 0, (size_t)2 * h->mask_words * sizeof(uint32_t), h->stream));
        clear_rbox(h);
        h->initialised = true;
    });
}

int tdlb_set_markers(tdlb_handle h, const tdlb_marker* markers, size_t n) {
    return guarded(h, [&] {
        upload_markers(h, markers, n, n, nullptr);
        h->resident = true;
    });
}

int tdlb_forcing_resident(tdlb_handle h, float alpha, float beta) {
    return guarded<false>(h, [&] {
        require_init(h);
        run_forcing(h, alpha, beta);
    });
}

int tdlb_forcing(tdlb_handle h, const tdlb_marker* markers, size_t n, float alpha, float beta) {
    return guarded(h, [&] {
        require_init(h);
        upload_markers(h, markers, n, n, nullptr);
        h->resident = false;   // a new list every pass: no split-step zone
        run_forcing(h, alpha, beta);
    });
}

int tdlb_collision(tdlb_handle h) {
    return guarded<false>(h, [&] {
        require_init(h);
        run_step(h, true);
    });
}

int tdlb_bounce_back(tdlb_handle h) { return h ? TDLB_OK : TDLB_EINVAL; }
int tdlb_streaming_push(tdlb_handle h) { return h ? TDLB_OK : TDLB_EINVAL; }
int tdlb_moments(tdlb_handle h) { return h ? TDLB_OK : TDLB_EINVAL; }

int tdlb_step(tdlb_handle h, float alpha, float beta) {
    return guarded<false>(h, [&] {
        require_init(h);
        run_step(h, true);
        run_forcing(h, alpha, beta);
    });
}

int tdlb_read_moments(tdlb_handle h, float* out) {
    return guarded(h, [&] {
        require_init(h);
        if (!out) throw Fail{TDLB_EINVAL, "out is NULL"};
        DevBuf M{state_moments(h)};
        planes_to_host_aos(h, M.p, tdlb::NQ, out);
    });
}

int tdlb_read_velocity_density(tdlb_handle h, float* rho, float* ux, float* uy, float* uz) {
    return guarded(h, [&] {
        require_init(h);
        const Dims& g = h->g;
        DevBuf M{state_moments(h)};
        const size_t ncell = (size_t)g.nx * g.ny * g.nz;
        std::vector<float> m(ncell * tdlb::NQ), f(ncell * 3);
        planes_to_host_aos(h, M.p, tdlb::NQ, m.data());
        force_to_host(h, f.data());
        std::vector<uint8_t> t(ncell);
        std::vector<uint32_t> words((size_t)h->mask_words);
        TDLB_CK(cudaMemcpy(words.data(), h->mask_cur(), words.size() * 4, cudaMemcpyDeviceToHost));
        for (size_t c = 0; c < ncell; c++) {
            const int k = (int)(c % g.nz);
            const size_t row = c / g.nz;
            const bool on = (words[row * g.kw + (k >> 5)] >> (k & 31)) & 1u;
            const float fx = on ? f[c * 3] : 0.f, fy = on ? f[c * 3 + 1] : 0.f, fz = on ? f[c * 3 + 2] : 0.f;
            const float r = m[c * tdlb::NQ];
            // QVec.hpp:385-394, in the reference's precision
            if (rho) rho[c] = r;
            if (ux) ux[c] = (float)((1.0 / r) * (m[c * tdlb::NQ + 1] + 0.5 * fx));
            if (uy) uy[c] = (float)((1.0 / r) * (m[c * tdlb::NQ + 2] + 0.5 * fy));
            if (uz) uz[c] = (float)((1.0 / r) * (m[c * tdlb::NQ + 3] + 0.5 * fz));
        }
    });
}

int tdlb_read_force(tdlb_handle h, float* f3) {
    return guarded(h, [&] {
        require_init(h);
        if (!f3) throw Fail{TDLB_EINVAL, "out is NULL"};
        const Dims& g = h->g;
        force_to_host(h, f3);
        std::vector<uint32_t> words((size_t)h->mask_words);
        TDLB_CK(cudaMemcpy(words.data(), h->mask_cur(), words.size() * 4, cudaMemcpyDeviceToHost));
        const size_t ncell = (size_t)g.nx * g.ny * g.nz;
        for (size_t c = 0; c < ncell; c++) {
            const int k = (int)(c % g.nz);
            const size_t row = c / g.nz;
            if (!((words[row * g.kw + (k >> 5)] >> (k & 31)) & 1u)) f3[c * 3] = f3[c * 3 + 1] = f3[c * 3 + 2] = 0.f;
        }
    });
}

int tdlb_read_nu(tdlb_handle h, float* nu) {
    return guarded(h, [&] {
        require_init(h);
        if (!nu) throw Fail{TDLB_EINVAL, "out is NULL"};
        planes_to_host_aos(h, h->Nu, 1, nu);
    });
}

int tdlb_read_touched(tdlb_handle h, uint8_t* flags) {
    return guarded(h, [&] {
        require_init(h);
        if (!flags) throw Fail{TDLB_EINVAL, "out is NULL"};
        const Dims& g = h->g;
        std::vector<uint32_t> words((size_t)h->mask_words);
        TDLB_CK(cudaMemcpyAsync(words.data(), h->mask_cur(), words.size() * 4, cudaMemcpyDeviceToHost, h->stream));
        TDLB_CK(cudaStreamSynchronize(h->stream));
        const size_t ncell = (size_t)g.nx * g.ny * g.nz;
        for (size_t c = 0; c < ncell; c++) {
            const int k = (int)(c % g.nz);
            const size_t row = c / g.nz;
            flags[c] = (uint8_t)((words[row * g.kw + (k >> 5)] >> (k & 31)) & 1u);
        }
    });
}

int tdlb_get_dims(tdlb_handle h, int64_t* x, int64_t* y, int64_t* z) {
    return guarded(h, [&] {
        if (x) *x = h->g.nx;
        if (y) *y = h->g.ny;
        if (z) *z = h->g.nz;
    });
}

int tdlb_get_even_step(tdlb_handle h, int* even) {
    return guarded(h, [&] {
        if (!even) throw Fail{TDLB_EINVAL, "out is NULL"};
        *even = h->even ? 1 : 0;
    });
}

int tdlb_set_cells_per_thread(tdlb_handle h, int v) {
    return guarded(h, [&] {
        if (v != 1 && v != 2 && v != 4) throw Fail{TDLB_EINVAL, "cells per thread must be 1, 2 or 4"};
        h->vec = v;
    });
}

int tdlb_set_l2_prefetch(tdlb_handle h, int on) {
    return guarded(h, [&] {
        if (on != 0 && on != 1) throw Fail{TDLB_EINVAL, "l2 prefetch must be 0 or 1"};
        h->l2_prefetch = on;
    });
}

int tdlb_set_overlap(tdlb_handle h, int mode) {
    return guarded(h, [&] {
        if (mode < 0 || mode > 2) throw Fail{TDLB_EINVAL, "overlap mode must be 0, 1 or 2"};
        h->overlap = mode;
    });
}

int tdlb_join(tdlb_handle h) {
    return guarded(h, [&] {});
}

int tdlb_read_zone(tdlb_handle h, uint8_t* flags) {
    return guarded(h, [&] {
        if (!flags) throw Fail{TDLB_EINVAL, "out is NULL"};
        if (!split_capable(h))
            throw Fail{TDLB_ESTATE, "no split step (needs resident markers, one cell per thread, overlap on and, in "
                                    "mode 1, inner chunks holding at most 60 % of the lattice)"};
        const Dims& g = h->g;
        const std::vector<uint32_t>& bits = h->h_zone_bits;
        size_t c = 0;
        for (long long i = 0; i < g.nx; i++)
            for (long long j = 0; j < g.ny; j++)
                for (long long k = 0; k < g.nz; k++, c++) {
                    const long long chunk = ((i * g.ny + j) * g.kp + k) / tdlb::kSplitChunk;
                    flags[c] = (uint8_t)((bits[(size_t)(chunk >> 5)] >> (chunk & 31)) & 1u);
                }
    });
}

int tdlb_kernel_launches(tdlb_handle h, int64_t* n) {
    return guarded(h, [&] {
        if (!n) throw Fail{TDLB_EINVAL, "out is NULL"};
        *n = (int64_t)h->launches;
    });
}

int tdlb_set_kernel_timing(tdlb_handle h, int on) {
    return guarded(h, [&] { h->timing = on != 0; });
}

int tdlb_kernel_time(tdlb_handle h, double* total_ms, int64_t* launches) {
    return guarded(h, [&] {
        TDLB_CK(cudaStreamSynchronize(h->stream));
        double ms = 0.0;
        for (size_t q = 0; q + 1 < h->tev.size(); q += 2) {
            float t = 0.f;
            TDLB_CK(cudaEventElapsedTime(&t, h->tev[q], h->tev[q + 1]));
            ms += t;
        }
        const int64_t n = (int64_t)(h->tev.size() / 2);
        for (cudaEvent_t e : h->tev) cudaEventDestroy(e);
        h->tev.clear();
        if (total_ms) *total_ms = ms;
        if (launches) *launches = n;
    });
}

int tdlb_reduce_fp64(tdlb_handle h, double* out4) {
    return guarded(h, [&] {
        require_init(h);
        if (!out4) throw Fail{TDLB_EINVAL, "out is NULL"};
        if (!h->d_red) TDLB_CK(cudaMalloc(&h->d_red, (size_t)(tdlb::kReduceBlocks * 4 + 4) * sizeof(double)));
        tdlb::IbmArgs a = ibm_args(h, 0.f, 0.f);
        TDLB_CK(tdlb::launch_reduce_fp64(a, h->mask_cur(), h->d_red, h->d_red + tdlb::kReduceBlocks * 4, h->stream));
        TDLB_CK(cudaMemcpyAsync(out4, h->d_red + tdlb::kReduceBlocks * 4, 4 * sizeof(double), cudaMemcpyDeviceToHost,
                                h->stream));
        TDLB_CK(cudaStreamSynchronize(h->stream));
    });
}

int tdlb_get_stream(tdlb_handle h, void** stream) {
    return guarded(h, [&] {
        if (!stream) throw Fail{TDLB_EINVAL, "out is NULL"};
        *stream = (void*)h->stream;
    });
}

int tdlb_synchronize(tdlb_handle h) {
    return guarded(h, [&] { TDLB_CK(cudaStreamSynchronize(h->stream)); });
}

int tdlb_attach_rushton(tdlb_handle h, const tdlb_rushton* spec, double nonupdating_delta_angle, double angle,
                        double delta_angle) {
    return guarded(h, [&] {
        if (!spec) throw Fail{TDLB_EINVAL, "spec is NULL"};
        if (spec->x != h->g.nx || spec->y != h->g.ny || spec->z != h->g.nz)
            throw Fail{TDLB_EINVAL, "Rushton spec extents differ from the lattice"};
        const tdlb::RushtonGeom G = tdlb::RushtonGeom::from(*spec);
        std::vector<tdlb_marker> all = G.fixed();
        const int n_fixed = (int)all.size();
        const std::vector<tdlb_marker> nonupd = G.rotating_nonupdating(nonupdating_delta_angle);
        all.insert(all.end(), nonupd.begin(), nonupd.end());
        const size_t n0 = all.size();
        const std::vector<tdlb_marker> rot = G.rotating(angle, delta_angle);
        all.insert(all.end(), rot.begin(), rot.end());
        const std::vector<tdlb::RotatingPolar> pol = G.rotating_polar();
        std::vector<double> xz(2 * pol.size());
        double rmax = 0;
        for (size_t q = 0; q < pol.size(); q++) {
            xz[2 * q] = pol[q].x0;
            xz[2 * q + 1] = pol[q].z0;
            rmax = std::max(rmax, std::sqrt(pol[q].x0 * pol[q].x0 + pol[q].z0 * pol[q].z0));
        }
        if (G.ci - rmax < 2.0 || G.ci + rmax > h->g.nx - 3.0 || G.ck - rmax < 2.0 || G.ck + rmax > h->g.nz - 3.0)
            throw Fail{TDLB_EINVAL, "impeller does not stay 2 cells inside the lattice"};
        upload_markers(h, all.data(), all.size(), n0, xz.data());
        h->resident = true;
        h->h_rot_xz = xz;
        cudaFree(h->d_rot_xz);
        h->d_rot_xz = nullptr;
        if (!xz.empty()) {
            TDLB_CK(cudaMalloc(&h->d_rot_xz, xz.size() * sizeof(double)));
            TDLB_CK(cudaMemcpy(h->d_rot_xz, xz.data(), xz.size() * sizeof(double), cudaMemcpyHostToDevice));
        }
        h->rot_device = true;
        h->rot_ci = G.ci;
        h->rot_ck = G.ck;
        h->impeller_begin = n_fixed;
        h->rspec = *spec;
        h->angle = angle;
        h->rstep = 1;
        auto_rbox(h, G, pol, rmax);
    });
}

int tdlb_set_residual_box(tdlb_handle h, int64_t i0, int64_t i1, int64_t j0, int64_t j1, int64_t k0, int64_t k1) {
    return guarded(h, [&] {
        set_rbox(h, i0, i1, j0, j1, k0, k1);
        h->rbox_auto = false;
    });
}

int tdlb_get_residual_box(tdlb_handle h, int64_t* box6) {
    return guarded<false>(h, [&] {
        if (!box6) throw Fail{TDLB_EINVAL, "box6 is NULL"};
        const tdlb::ResidualBox& b = h->rbox_geom;
        box6[0] = b.i0; box6[1] = b.i0 + b.bx;
        box6[2] = b.j0; box6[3] = b.j0 + b.by;
        box6[4] = b.k0; box6[5] = b.k0 + b.bz;
    });
}

int tdlb_rotate_impeller(tdlb_handle h, double angle, double delta_angle) {
    return guarded<false>(h, [&] {
        if (!h->rot_device) throw Fail{TDLB_ESTATE, "no impeller attached (tdlb_attach_rushton)"};
        // after the previous forcing pass, which reads the blades
        TDLB_CK(tdlb::launch_rotate_markers(h->d_rot_xz, h->d_markers + h->n0, h->n_markers - h->n0, std::cos(angle),
                                            std::sin(angle), delta_angle, h->rot_ci, h->rot_ck, h->g.nx, h->g.nz,
                                            ibm_stream(h)));
        h->launches++;
        h->angle = angle;
    });
}

int tdlb_set_rotating_markers(tdlb_handle h, const tdlb_marker* markers, size_t n) {
    return guarded(h, [&] {
        if (h->impeller_begin < 0) throw Fail{TDLB_ESTATE, "no impeller attached (tdlb_attach_rushton)"};
        if (n != (size_t)(h->n_markers - h->n0)) throw Fail{TDLB_EINVAL, "rotating marker count differs from the attached blades"};
        if (n && !markers) throw Fail{TDLB_EINVAL, "markers is NULL"};
        validate_markers(h->g, markers, n, (size_t)h->n0);
        // Host copies and the blade schedule for these positions; the uploads
        // go through a pinned buffer and are queued after the work already on
        // the stream (the previous forcing pass still reads the old blades),
        // so this call does not wait for the device.
        std::copy(markers, markers + n, h->h_markers.begin() + h->n0);
        const auto* mk = reinterpret_cast<const tdlb::Marker*>(h->h_markers.data());
        h->seg1.build(mk, h->n0, h->n_markers, h->g.nx, h->g.ny, h->g.nz, h->n0, h->seg0.nlevels, nullptr);
        update_blade_planes(h);
        const int L0 = h->seg0.nlevels;
        ensure_level_cap(h, (long long)L0 + h->seg1.nlevels + 1);
        const size_t b_mk = n * sizeof(tdlb::Marker);
        const size_t b_order = n * sizeof(int);
        const size_t b_lv = h->seg1.level_ptr.size() * sizeof(int);
        const size_t b_pl = (size_t)(h->g.ny + 1) * sizeof(int);
        const size_t need = b_mk + b_order + b_lv + b_pl;
        auto& st = h->pin[h->pin_cur];
        h->pin_cur ^= 1;
        if (st.ev) TDLB_CK(cudaEventSynchronize(st.ev));   // the copies of two calls ago read this buffer
        else TDLB_CK(cudaEventCreateWithFlags(&st.ev, cudaEventDisableTiming));
        if (need > st.cap) {
            cudaFreeHost(st.p);
            st.p = nullptr;
            st.cap = 0;
            TDLB_CK(cudaHostAlloc((void**)&st.p, need, cudaHostAllocDefault));
            st.cap = need;
        }
        char* q = st.p;
        std::memcpy(q, markers, b_mk);
        std::memcpy(q + b_mk, h->seg1.order.data(), b_order);
        std::memcpy(q + b_mk + b_order, h->seg1.level_ptr.data(), b_lv);
        std::memcpy(q + b_mk + b_order + b_lv, h->seg1.plane_lv.data(), b_pl);
        if (n) {
            TDLB_CK(cudaMemcpyAsync(h->d_markers + h->n0, q, b_mk, cudaMemcpyHostToDevice, h->stream));
            TDLB_CK(cudaMemcpyAsync(h->d_sched + h->n0, q + b_mk, b_order, cudaMemcpyHostToDevice, h->stream));
        }
        TDLB_CK(cudaMemcpyAsync(h->d_level_ptr + L0, q + b_mk + b_order, b_lv, cudaMemcpyHostToDevice, h->stream));
        TDLB_CK(cudaMemcpyAsync(h->d_plane_lv1, q + b_mk + b_order + b_lv, b_pl, cudaMemcpyHostToDevice, h->stream));
        TDLB_CK(cudaEventRecord(st.ev, h->stream));
        h->rot_device = false;   // the blades now follow the host's list
        // a split step needs every blade stencil cell inside the zone
        if (h->zone_gen == h->marker_gen)
            h->zone_ok = stencils_inside(h, h->h_markers.data() + h->n0, n, h->h_zone_core);
    });
}

// Queue the impeller load of the last forcing pass and its copy into out5.
void queue_impeller_load(tdlb_lattice* h, double* out5) {
    if (!out5) throw Fail{TDLB_EINVAL, "out is NULL"};
    if (h->impeller_begin < 0) throw Fail{TDLB_ESTATE, "no impeller attached (tdlb_attach_rushton)"};
    if (h->pass == 0) throw Fail{TDLB_ESTATE, "no forcing pass yet"};
    if (!h->d_load) TDLB_CK(cudaMalloc(&h->d_load, (size_t)(tdlb::kLoadBlocks * 5 + 5) * sizeof(double)));
    tdlb::IbmArgs a = ibm_args(h, 0.f, h->last_beta);
    TDLB_CK(tdlb::launch_marker_load(a, h->impeller_begin, h->rot_ci, h->rot_ck, h->d_load,
                                     h->d_load + tdlb::kLoadBlocks * 5, h->stream));
    TDLB_CK(cudaMemcpyAsync(out5, h->d_load + tdlb::kLoadBlocks * 5, 5 * sizeof(double), cudaMemcpyDefault,
                            h->stream));
}

int tdlb_impeller_load(tdlb_handle h, double* out5) {
    return guarded(h, [&] {
        queue_impeller_load(h, out5);
        TDLB_CK(cudaStreamSynchronize(h->stream));
    });
}

int tdlb_impeller_load_async(tdlb_handle h, double* out5) {
    return guarded(h, [&] { queue_impeller_load(h, out5); });
}

int tdlb_read_markers(tdlb_handle h, tdlb_marker* out, size_t cap, size_t* n) {
    return guarded(h, [&] {
        if (n) *n = (size_t)h->n_markers;
        if (!out) return;
        if (cap < (size_t)h->n_markers) throw Fail{TDLB_EINVAL, "cap smaller than the marker count"};
        if (h->n_markers)
            TDLB_CK(cudaMemcpyAsync(out, h->d_markers, (size_t)h->n_markers * sizeof(tdlb_marker), cudaMemcpyDeviceToHost,
                                    h->stream));
        TDLB_CK(cudaStreamSynchronize(h->stream));
    });
}

int tdlb_schedule_levels(const tdlb_marker* markers, size_t n, int64_t x, int64_t y, int64_t z, int32_t* level_out,
                         int32_t* max_levels_per_plane) {
    if ((n && !markers) || x < 1 || y < 1 || z < 1 || n > (size_t)0x7fffffff) return TDLB_EINVAL;
    for (size_t q = 0; q < n; q++)
        if (markers[q].i < 0 || markers[q].i >= x || markers[q].j < 0 || markers[q].j >= y || markers[q].k < 0 ||
            markers[q].k >= z)
            return TDLB_EINVAL;
    tdlb::MarkerSchedule s;
    s.build(reinterpret_cast<const tdlb::Marker*>(markers), 0, (int)n, (int)x, (int)y, (int)z, 0, 0);
    if (level_out) {
        // level within its plane, from the plane's first level
        for (int64_t j = 0; j < y; j++)
            for (int lv = s.plane_lv[(size_t)j]; lv < s.plane_lv[(size_t)j + 1]; lv++)
                for (int p = s.level_ptr[(size_t)lv]; p < s.level_ptr[(size_t)lv + 1]; p++)
                    level_out[s.order[(size_t)p]] = lv - s.plane_lv[(size_t)j];
    }
    if (max_levels_per_plane) *max_levels_per_plane = s.max_levels_per_plane;
    return TDLB_OK;
}

int tdlb_debug_get_state(tdlb_handle h, float* out) {
    return guarded(h, [&] {
        if (!out) throw Fail{TDLB_EINVAL, "out is NULL"};
        if (h->cfg.storage != TDLB_STORAGE_FP32) throw Fail{TDLB_EINVAL, "raw state access needs FP32 storage"};
        planes_to_host_aos(h, h->state_buf(), tdlb::NQ, out);
    });
}

int tdlb_debug_set_state(tdlb_handle h, const float* in, int holds_moments) {
    return guarded(h, [&] {
        if (!in) throw Fail{TDLB_EINVAL, "in is NULL"};
        if (h->cfg.storage != TDLB_STORAGE_FP32) throw Fail{TDLB_EINVAL, "raw state access needs FP32 storage"};
        host_aos_to_planes(h, in, tdlb::NQ, h->state_buf());
        h->holds_moments = holds_moments != 0;
        h->initialised = true;
    });
}

int tdlb_debug_transport(tdlb_handle h) {
    return guarded(h, [&] {
        require_init(h);
        if (h->cfg.storage != TDLB_STORAGE_FP32) throw Fail{TDLB_EINVAL, "transport-only steps need FP32 storage"};
        run_step(h, false);
    });
}

}  // extern "C"

namespace tdlb_rt {
void drop_residual_box(tdlb_lattice* h) { ::drop_rbox(h); }
void clear_residual_box(tdlb_lattice* h) { ::clear_rbox(h); }
tdlb::StepArgs step_args(tdlb_lattice* h, bool collide) { return ::step_args(h, collide); }
tdlb::IbmArgs ibm_args(tdlb_lattice* h, float alpha, float beta) { return ::ibm_args(h, alpha, beta); }
void borrow_stream(tdlb_lattice* h, cudaStream_t s) {
    if (join_side(h) == cudaSuccess) cudaStreamSynchronize(h->stream);
    if (!h->own_stream) h->own_stream = h->stream;
    h->stream = s;
}

void return_stream(tdlb_lattice* h) {
    if (!h->own_stream) return;
    h->stream = h->own_stream;
    h->own_stream = nullptr;
}

cudaError_t join_side(tdlb_lattice* h) {
    if (!h->pending) return cudaSuccess;
    cudaError_t e = cudaEventRecord(h->ev_sync, h->ibm);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(h->stream, h->ev_sync, 0);
    if (e != cudaSuccess) return e;
    h->pending = false;
    h->inner_queued = false;
    return cudaSuccess;
}
}  // namespace tdlb_rt
