// Batched form: many independent tanks of uneven sizes on one GPU.
//
// All tanks' fused steps run as ONE persistent launch (k_batch_step): a grid
// of a few blocks per SM loops over work items, each 128..256 consecutive
// quads of one tank, with that tank's step view staged in shared memory; so
// small tanks no longer leave most of the GPU idle. Per step the batch then
// runs every tank's immersed-boundary pass (on a pool of streams, so the
// tanks' passes overlap) and moves every attached impeller on the device
// from a per-step cos/sin table. Two consecutive steps (one A/B and parity
// cycle) are captured into a CUDA graph and replayed. The kernel shape --
// cells per thread, threads per block, resident blocks per SM -- is chosen
// by a small autotuner that times every candidate on the batch itself.
#include "tdlb_handle.hpp"
#include "tdlb_geometry.hpp"
#include "tdlb_rotate.hpp"
#include "step_kernels.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

namespace tdlb {

// One tank's view of one step (both streaming schemes).
struct TankStep {
    Planes A, B;                 // Simple: source / destination; Esotwist: A
    float* Nu;
    const float* Fx;
    const float* Fy;
    const float* Fz;
    const uint32_t* mask;
    Dims g;
    CollideParams p;
    int les, from_moments, even, pad;
};

template <int NT>
__device__ __forceinline__ void stage(TankStep& dst, const TankStep* src) {
    static_assert(sizeof(TankStep) % 4 == 0, "TankStep words");
    constexpr int words = sizeof(TankStep) / 4;
    for (int w = threadIdx.x; w < words; w += NT) reinterpret_cast<int*>(&dst)[w] = reinterpret_cast<const int*>(src)[w];
}

template <typename S, int V, bool ESO, bool LES, bool FM>
__device__ __forceinline__ void tank_quad(const TankStep& ts, unsigned t) {
    if constexpr (!ESO) {
        simple_quad<S, V, LES, FM, true>(ts.A, ts.B, ts.Nu, ts.Fx, ts.Fy, ts.Fz, ts.mask, ts.g, ts.p, t);
    } else {
        if (ts.even) esotwist_quad<S, V, LES, FM, true, true>(ts.A, ts.Nu, ts.Fx, ts.Fy, ts.Fz, ts.mask, ts.g, ts.p, t);
        else esotwist_quad<S, V, LES, FM, true, false>(ts.A, ts.Nu, ts.Fx, ts.Fy, ts.Fz, ts.mask, ts.g, ts.p, t);
    }
}

// Persistent batched step: block b takes work items b, b + grid, ...; an
// item is `NT` consecutive quads of one tank, whose step view is staged in
// shared memory. 16-bit storage never holds moments, so its from-moments
// bodies are not built.
template <typename S, int V, int NT, bool ESO>
__global__ void __launch_bounds__(NT) k_batch_step(const TankStep* __restrict__ tanks, const int2* __restrict__ work,
                                                   int nwork) {
    constexpr bool kFM = sizeof(S) == 4;
    __shared__ TankStep ts;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 wk = work[w];
        __syncthreads();
        stage<NT>(ts, tanks + wk.x);
        __syncthreads();
        const unsigned t = (unsigned)wk.y + threadIdx.x;
        if (ts.les) {
            if (kFM && ts.from_moments) tank_quad<S, V, ESO, true, kFM>(ts, t);
            else tank_quad<S, V, ESO, true, false>(ts, t);
        } else {
            if (kFM && ts.from_moments) tank_quad<S, V, ESO, false, kFM>(ts, t);
            else tank_quad<S, V, ESO, false, false>(ts, t);
        }
    }
}

// Blade rotation from a per-step table (cos a, sin a, delta a) indexed by
// the device step counter, so a captured graph can replay many steps.
__global__ void k_rotate_tab(const double* __restrict__ xz, Marker* __restrict__ out, int n,
                             const double* __restrict__ table, const int* __restrict__ step, double ci, double ck, int nx,
                             int nz) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const double* tb = table + 3 * (size_t)(*step);
    const RotatedMarker r = rotate_marker(xz[2 * q], xz[2 * q + 1], tb[0], tb[1], tb[2], ci, ck, nx, nz);
    Marker& m = out[q];
    m.i = r.i;
    m.k = r.k;
    m.iCartFraction = r.iCartFraction;
    m.kCartFraction = r.kCartFraction;
    m.uDelta = r.uDelta;
    m.vDelta = 0.f;
    m.wDelta = r.wDelta;
}

__global__ void k_counter_inc(int* step) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *step += 1;
}

using BatchFn = void (*)(const TankStep*, const int2*, int);

template <typename S, bool ESO>
BatchFn pick(int v, int nt) {
    if (v == 1) return nt == 256 ? (BatchFn)k_batch_step<S, 1, 256, ESO> : (BatchFn)k_batch_step<S, 1, 128, ESO>;
    if constexpr (sizeof(S) == 4)
        if (v == 2) return nt == 256 ? (BatchFn)k_batch_step<S, 2, 256, ESO> : (BatchFn)k_batch_step<S, 2, 128, ESO>;
    return nt == 256 ? (BatchFn)k_batch_step<S, 4, 256, ESO> : (BatchFn)k_batch_step<S, 4, 128, ESO>;
}

BatchFn batch_kernel(int storage, bool eso, int v, int nt) {
    if (storage == STORE_F16) return eso ? pick<__half, true>(v, nt) : pick<__half, false>(v, nt);
    if (storage == STORE_BF16) return eso ? pick<__nv_bfloat16, true>(v, nt) : pick<__nv_bfloat16, false>(v, nt);
    return eso ? pick<float, true>(v, nt) : pick<float, false>(v, nt);
}

}  // namespace tdlb

using tdlb::TankStep;

struct tdlb_batch_s {
    int device = 0;
    std::vector<tdlb_lattice*> tanks;
    cudaStream_t stream = nullptr;
    std::vector<cudaStream_t> pool;   // per-tank IBM passes run spread over these
    std::vector<cudaEvent_t> ev;      // fork/join events
    TankStep* d_steps = nullptr;      // [2][n]: views of an even and an odd step of a run
    int2* d_work = nullptr;
    int nwork = 0;
    int* d_step = nullptr;            // device step counter of a run
    std::vector<double*> d_table;     // per tank: [steps][3] cos, sin, delta
    std::vector<int> table_cap;
    int vec = 1, threads = 128, bps = 4;   // kernel shape
    int grid = 0;
    long long launches = 0;           // kernels run by tdlb_batch_run* so far
    std::string err = "no error";
};

namespace {

struct BFail {
    int code;
    std::string msg;
};

#define TDLB_BCK(call)                                                                          \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) throw BFail{TDLB_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

thread_local std::string g_batch_create_error = "no error";

template <typename F>
int bguard(tdlb_batch_s* b, F&& fn) {
    if (!b) return TDLB_EINVAL;
    try {
        cudaSetDevice(b->device);
        fn();
        return TDLB_OK;
    } catch (const BFail& f) {
        b->err = f.msg;
        return f.code;
    } catch (const std::exception& e) {
        b->err = e.what();
        return TDLB_EINVAL;
    }
}

int storage_of(const tdlb_batch_s* b) { return b->tanks[0]->cfg.storage; }
bool eso_of(const tdlb_batch_s* b) { return b->tanks[0]->cfg.streaming == TDLB_STREAMING_ESOTWIST; }

// Work list for the current kernel shape: (tank, first quad) per item.
void build_work(tdlb_batch_s* b) {
    std::vector<int2> w;
    for (int t = 0; t < (int)b->tanks.size(); t++) {
        const Dims& g = b->tanks[(size_t)t]->g;
        const long long nq = g.rows() * (g.kp / b->vec);
        for (long long q = 0; q < nq; q += b->threads) w.push_back(make_int2(t, (int)q));
    }
    TDLB_BCK(cudaStreamSynchronize(b->stream));   // queued launches may still read the old list
    cudaFree(b->d_work);
    b->d_work = nullptr;
    TDLB_BCK(cudaMalloc(&b->d_work, w.size() * sizeof(int2)));
    TDLB_BCK(cudaMemcpy(b->d_work, w.data(), w.size() * sizeof(int2), cudaMemcpyHostToDevice));
    b->nwork = (int)w.size();
    int sms = 0;
    TDLB_BCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
    b->grid = std::min(b->nwork, sms * b->bps);
}

TankStep view_of(tdlb_lattice* h) {
    const tdlb::StepArgs a = tdlb_rt::step_args(h, true);
    TankStep s{};
    s.A = a.A;
    s.B = a.B;
    s.Nu = a.Nu;
    s.Fx = a.Fx;
    s.Fy = a.Fy;
    s.Fz = a.Fz;
    s.mask = a.mask;
    s.g = a.g;
    s.p = a.p;
    s.les = a.les;
    s.from_moments = a.from_moments;
    s.even = a.even;
    return s;
}

// Advance every tank's host bookkeeping by one fused step.
void advance_step_state(tdlb_lattice* h) {
    if (h->cfg.streaming == TDLB_STREAMING_SIMPLE) h->cur ^= 1;
    else h->even = !h->even;
    h->holds_moments = false;
}

void launch_fused(tdlb_batch_s* b, const TankStep* d_views, cudaStream_t st) {
    const tdlb::BatchFn fn = tdlb::batch_kernel(storage_of(b), eso_of(b), b->vec, b->threads);
    fn<<<b->grid, b->threads, 0, st>>>(d_views, b->d_work, b->nwork);
    TDLB_BCK(cudaGetLastError());
}

// Kernels one immersed-boundary pass launches (tdlb::launch_ibm).
int ibm_kernels(const tdlb::IbmArgs& a) {
    return (a.ncell > 0) + (a.n > a.n0) + (a.n_big > 0) + (a.n_small > 0);
}

// One batched step as launches on b->stream (also used inside capture):
// rotate impellers, fused step (views = d_views), IBM pass per tank.
// Returns the number of kernels it queued.
int queue_step(tdlb_batch_s* b, const TankStep* d_views, float alpha, float beta, bool use_table) {
    const size_t n = b->tanks.size();
    const size_t P = b->pool.size();
    int kernels = 1;
    if (use_table) {
        for (size_t t = 0; t < n; t++) {
            tdlb_lattice* h = b->tanks[t];
            if (!h->rot_device || h->n_markers == h->n0) continue;
            const int nr = h->n_markers - h->n0;
            tdlb::k_rotate_tab<<<(nr + 255) / 256, 256, 0, b->stream>>>(h->d_rot_xz, h->d_markers + h->n0, nr,
                                                                         b->d_table[t], b->d_step, h->rot_ci, h->rot_ck,
                                                                         h->g.nx, h->g.nz);
            kernels++;
        }
        TDLB_BCK(cudaGetLastError());
    }
    launch_fused(b, d_views, b->stream);
    for (size_t t = 0; t < n; t++) advance_step_state(b->tanks[t]);
    // the tanks' IBM passes, spread over the stream pool
    TDLB_BCK(cudaEventRecord(b->ev[0], b->stream));
    for (size_t k = 0; k < P; k++) TDLB_BCK(cudaStreamWaitEvent(b->pool[k], b->ev[0], 0));
    for (size_t t = 0; t < n; t++) {
        tdlb_lattice* h = b->tanks[t];
        if (!h->markers_set) continue;
        cudaStream_t s = b->pool[t % P];
        const tdlb::IbmArgs ia = tdlb_rt::ibm_args(h, alpha, beta);
        TDLB_BCK(tdlb::launch_ibm(ia, s));
        kernels += ibm_kernels(ia);
        h->pass++;
        h->last_beta = beta;
    }
    for (size_t k = 0; k < P; k++) {
        TDLB_BCK(cudaEventRecord(b->ev[1 + k], b->pool[k]));
        TDLB_BCK(cudaStreamWaitEvent(b->stream, b->ev[1 + k], 0));
    }
    if (use_table) {
        tdlb::k_counter_inc<<<1, 32, 0, b->stream>>>(b->d_step);
        TDLB_BCK(cudaGetLastError());
        kernels++;
    }
    return kernels;
}

void upload_views(tdlb_batch_s* b) {
    // views of the next two steps (the host state is restored afterwards)
    const size_t n = b->tanks.size();
    std::vector<TankStep> v(2 * n);
    std::vector<int> cur(n), pass(n);
    std::vector<bool> even(n), hm(n);
    for (size_t t = 0; t < n; t++) {
        tdlb_lattice* h = b->tanks[t];
        cur[t] = h->cur; pass[t] = h->pass; even[t] = h->even; hm[t] = h->holds_moments;
    }
    for (int k = 0; k < 2; k++)
        for (size_t t = 0; t < n; t++) {
            tdlb_lattice* h = b->tanks[t];
            v[(size_t)k * n + t] = view_of(h);
            advance_step_state(h);
            h->pass++;
        }
    for (size_t t = 0; t < n; t++) {
        tdlb_lattice* h = b->tanks[t];
        h->cur = cur[t]; h->pass = pass[t]; h->even = even[t]; h->holds_moments = hm[t];
    }
    // stream-ordered: launches already queued read the previous views
    TDLB_BCK(cudaMemcpyAsync(b->d_steps, v.data(), v.size() * sizeof(TankStep), cudaMemcpyHostToDevice, b->stream));
}

// Per-step (cos, sin, delta) of every attached impeller for `steps` steps.
void build_tables(tdlb_batch_s* b, int steps) {
    for (size_t t = 0; t < b->tanks.size(); t++) {
        tdlb_lattice* h = b->tanks[t];
        if (!h->rot_device) continue;
        if (b->table_cap[t] < steps) {
            cudaFree(b->d_table[t]);
            b->d_table[t] = nullptr;
            TDLB_BCK(cudaMalloc(&b->d_table[t], (size_t)3 * steps * sizeof(double)));
            b->table_cap[t] = steps;
        }
        const tdlb::RushtonGeom G = tdlb::RushtonGeom::from(h->rspec);
        std::vector<double> tab((size_t)3 * steps);
        double angle = h->angle;
        unsigned long long st = h->rstep;
        for (int s = 0; s < steps; s++) {
            st++;
            const double d = G.increment(st);
            angle += d;
            tab[(size_t)3 * s] = std::cos(angle);
            tab[(size_t)3 * s + 1] = std::sin(angle);
            tab[(size_t)3 * s + 2] = d;
        }
        TDLB_BCK(cudaMemcpy(b->d_table[t], tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
}

void finish_tables(tdlb_batch_s* b, int steps) {
    for (tdlb_lattice* h : b->tanks) {
        if (!h->rot_device) continue;
        const tdlb::RushtonGeom G = tdlb::RushtonGeom::from(h->rspec);
        for (int s = 0; s < steps; s++) {
            h->rstep++;
            h->angle += G.increment(h->rstep);
        }
    }
}

void check_ready(tdlb_batch_s* b) {
    for (tdlb_lattice* h : b->tanks)
        if (!h->initialised) throw BFail{TDLB_ESTATE, "every tank must be initialised first"};
}

// Steps, eager or graph-replayed: the first step of a tank that still holds
// moments (right after initialise) always runs eagerly.
void run(tdlb_batch_s* b, int steps, float alpha, float beta, bool graph) {
    check_ready(b);
    TDLB_BCK(cudaStreamSynchronize(b->stream));   // the previous run may still read the tables
    build_tables(b, steps);
    TDLB_BCK(cudaMemsetAsync(b->d_step, 0, sizeof(int), b->stream));
    int done = 0;
    bool any_moments = false;
    for (tdlb_lattice* h : b->tanks) any_moments = any_moments || h->holds_moments;
    while (done < steps && (any_moments || !graph || steps - done < 2)) {
        upload_views(b);
        b->launches += queue_step(b, b->d_steps, alpha, beta, true);
        done++;
        any_moments = false;
    }
    if (done < steps) {
        upload_views(b);
        cudaGraph_t g = nullptr;
        int per_pair = 0;
        TDLB_BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        try {
            per_pair += queue_step(b, b->d_steps, alpha, beta, true);
            per_pair += queue_step(b, b->d_steps + b->tanks.size(), alpha, beta, true);
        } catch (...) {
            cudaStreamEndCapture(b->stream, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        TDLB_BCK(cudaStreamEndCapture(b->stream, &g));
        cudaGraphExec_t ge = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        TDLB_BCK(ie);
        // the capture advanced the host state by two steps; each replay is two steps
        const int pairs = (steps - done) / 2;
        for (tdlb_lattice* h : b->tanks) h->pass -= 2;
        for (int r = 0; r < pairs; r++) {
            const cudaError_t le = cudaGraphLaunch(ge, b->stream);
            if (le != cudaSuccess) {
                cudaGraphExecDestroy(ge);
                TDLB_BCK(le);
            }
        }
        cudaGraphExecDestroy(ge);
        for (tdlb_lattice* h : b->tanks) h->pass += 2 * pairs;
        b->launches += (long long)per_pair * pairs;
        done += 2 * pairs;
        if (done < steps) {   // an odd step left
            upload_views(b);
            b->launches += queue_step(b, b->d_steps, alpha, beta, true);
            done++;
        }
    }
    finish_tables(b, steps);
}

void release(tdlb_batch_s* b) {
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (tdlb_lattice* h : b->tanks) tdlb_destroy(h);
    for (cudaStream_t s : b->pool) cudaStreamDestroy(s);
    for (cudaEvent_t e : b->ev) cudaEventDestroy(e);
    for (double* p : b->d_table) cudaFree(p);
    cudaFree(b->d_steps);
    cudaFree(b->d_work);
    cudaFree(b->d_step);
    if (b->stream) cudaStreamDestroy(b->stream);
}

}  // namespace

extern "C" {

int tdlb_batch_create(const tdlb_config* cfgs, int n, int device, tdlb_batch* out) {
    if (!cfgs || n < 1 || !out) {
        g_batch_create_error = "bad arguments";
        return TDLB_EINVAL;
    }
    *out = nullptr;
    auto* b = new tdlb_batch_s();
    b->device = device;
    try {
        for (int t = 0; t < n; t++) {
            if (cfgs[t].streaming != cfgs[0].streaming || cfgs[t].storage != cfgs[0].storage)
                throw BFail{TDLB_EINVAL, "all tanks of a batch share one streaming scheme and one storage precision"};
            tdlb_handle h = nullptr;
            const int rc = tdlb_create_config(&cfgs[t], device, &h);
            if (rc != TDLB_OK) throw BFail{rc, std::string("tank ") + std::to_string(t) + ": " + tdlb_last_error(nullptr)};
            b->tanks.push_back(h);
        }
        TDLB_BCK(cudaSetDevice(device));
        TDLB_BCK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        for (tdlb_lattice* h : b->tanks) tdlb_rt::borrow_stream(h, b->stream);
        const int P = std::min(n, 16);
        b->pool.resize((size_t)P);
        for (auto& s : b->pool) TDLB_BCK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        b->ev.resize((size_t)P + 1);
        for (auto& e : b->ev) TDLB_BCK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        TDLB_BCK(cudaMalloc(&b->d_steps, (size_t)2 * n * sizeof(TankStep)));
        TDLB_BCK(cudaMalloc(&b->d_step, sizeof(int)));
        b->d_table.assign((size_t)n, nullptr);
        b->table_cap.assign((size_t)n, 0);
        b->vec = cfgs[0].streaming == TDLB_STREAMING_SIMPLE ? 1 : 4;
        build_work(b);
    } catch (const BFail& f) {
        g_batch_create_error = f.msg;
        release(b);
        delete b;
        return f.code;
    }
    *out = b;
    return TDLB_OK;
}

int tdlb_batch_destroy(tdlb_batch b) {
    if (!b) return TDLB_EINVAL;
    release(b);
    delete b;
    return TDLB_OK;
}

const char* tdlb_batch_last_error(tdlb_batch b) { return b ? b->err.c_str() : g_batch_create_error.c_str(); }

int tdlb_batch_size(tdlb_batch b, int* n) {
    return bguard(b, [&] {
        if (!n) throw BFail{TDLB_EINVAL, "out is NULL"};
        *n = (int)b->tanks.size();
    });
}

int tdlb_batch_tank(tdlb_batch b, int t, tdlb_handle* out) {
    return bguard(b, [&] {
        if (!out || t < 0 || t >= (int)b->tanks.size()) throw BFail{TDLB_EINVAL, "tank index out of range"};
        *out = b->tanks[(size_t)t];
    });
}

int tdlb_batch_set_shape(tdlb_batch b, int cells_per_thread, int threads, int blocks_per_sm) {
    return bguard(b, [&] {
        if (cells_per_thread != 1 && cells_per_thread != 2 && cells_per_thread != 4)
            throw BFail{TDLB_EINVAL, "cells per thread must be 1, 2 or 4"};
        if (cells_per_thread == 2 && storage_of(b) != TDLB_STORAGE_FP32)
            throw BFail{TDLB_EINVAL, "16-bit storage runs 1 or 4 cells per thread"};
        if (threads != 128 && threads != 256) throw BFail{TDLB_EINVAL, "threads must be 128 or 256"};
        if (blocks_per_sm < 1 || blocks_per_sm > 16) throw BFail{TDLB_EINVAL, "blocks per SM must be 1..16"};
        b->vec = cells_per_thread;
        b->threads = threads;
        b->bps = blocks_per_sm;
        for (tdlb_lattice* h : b->tanks) h->vec = cells_per_thread;
        build_work(b);
    });
}

int tdlb_batch_get_shape(tdlb_batch b, int* cells_per_thread, int* threads, int* blocks_per_sm) {
    return bguard(b, [&] {
        if (cells_per_thread) *cells_per_thread = b->vec;
        if (threads) *threads = b->threads;
        if (blocks_per_sm) *blocks_per_sm = b->bps;
    });
}

// Times the fused batched launch for every candidate shape on the batch's
// own (initialised) tanks and keeps the fastest. The timed launches write
// the populations the next step would overwrite anyway, but they also
// update the LES eddy viscosity; callers re-initialise afterwards.
int tdlb_batch_autotune(tdlb_batch b, int trials, double* best_ms) {
    return bguard(b, [&] {
        check_ready(b);
        if (trials < 1) trials = 3;
        struct Cand { int v, nt, bps; };
        std::vector<Cand> cands;
        const bool h16 = storage_of(b) != TDLB_STORAGE_FP32;
        for (int v : {1, 2, 4}) {
            if (h16 && v == 2) continue;
            for (int nt : {128, 256})
                for (int bps : {2, 4, 8}) {
                    if (nt == 256 && bps == 8) continue;
                    cands.push_back({v, nt, bps});
                }
        }
        upload_views(b);
        cudaEvent_t e0, e1;
        TDLB_BCK(cudaEventCreate(&e0));
        TDLB_BCK(cudaEventCreate(&e1));
        float best = 1e30f;
        Cand win = cands[0];
        for (const Cand& c : cands) {
            b->vec = c.v; b->threads = c.nt; b->bps = c.bps;
            build_work(b);
            launch_fused(b, b->d_steps, b->stream);   // warm-up
            TDLB_BCK(cudaEventRecord(e0, b->stream));
            for (int r = 0; r < trials; r++) launch_fused(b, b->d_steps, b->stream);
            TDLB_BCK(cudaEventRecord(e1, b->stream));
            TDLB_BCK(cudaEventSynchronize(e1));
            float ms = 0.f;
            TDLB_BCK(cudaEventElapsedTime(&ms, e0, e1));
            ms /= trials;
            if (ms < best) { best = ms; win = c; }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        b->vec = win.v; b->threads = win.nt; b->bps = win.bps;
        for (tdlb_lattice* h : b->tanks) h->vec = win.v;
        build_work(b);
        if (best_ms) *best_ms = best;
    });
}

int tdlb_batch_run(tdlb_batch b, int steps, float alpha, float beta) {
    return bguard(b, [&] {
        if (steps < 0) throw BFail{TDLB_EINVAL, "steps must be >= 0"};
        if (steps) run(b, steps, alpha, beta, true);
    });
}

int tdlb_batch_run_eager(tdlb_batch b, int steps, float alpha, float beta) {
    return bguard(b, [&] {
        if (steps < 0) throw BFail{TDLB_EINVAL, "steps must be >= 0"};
        if (steps) run(b, steps, alpha, beta, false);
    });
}

int tdlb_batch_kernel_launches(tdlb_batch b, long long* n) {
    return bguard(b, [&] {
        if (!n) throw BFail{TDLB_EINVAL, "out is NULL"};
        *n = b->launches;
    });
}

int tdlb_batch_synchronize(tdlb_batch b) {
    return bguard(b, [&] { TDLB_BCK(cudaStreamSynchronize(b->stream)); });
}

int tdlb_batch_get_stream(tdlb_batch b, void** stream) {
    return bguard(b, [&] {
        if (!stream) throw BFail{TDLB_EINVAL, "out is NULL"};
        *stream = (void*)b->stream;
    });
}

}  // extern "C"
