// Batched form: many independent tanks of uneven sizes on one GPU.
//
// The tanks are split into two groups of about equal cell count, each with
// its own stream. One batched step is, per group, a fixed set of launches
// whatever the number of tanks:
//   1. k_rotate_batch   every attached impeller's blades at the step's angle,
//                       read from a per-step (cos, sin, delta) table indexed
//                       by a device step counter;
//   2. k_batch_step     the group's fused collision + streaming: work items
//                       of eight chunks of 128 or 256 quads of one tank, with
//                       that tank's step view staged in shared memory once
//                       per item; one block per item or a persistent grid of
//                       a few blocks per SM looping over the items (block 0
//                       also advances the step counter);
//   3-7. the immersed-boundary passes of the group's tanks
//                       (launch_ibm_batch) on a high-priority stream: cells,
//                       blade gathers, touched-flag copies, small-plane and
//                       large-plane spreads, each one launch over the group.
// The groups' fused launches take turns, so each group's forcing pass runs
// while the other group's fused launch streams through HBM. Four step pairs
// (A/B and parity cycles), and single pairs for the rest of a run, are
// captured into CUDA graphs that stay instantiated between runs while the
// batch's launch shapes, work lists and device arrays are unchanged. The
// fused launch's shape -- cells per thread, threads per block, blocks per SM
// or one block per item -- is chosen by an autotuner that times every
// candidate on the batch itself.
#include "tdlb_handle.hpp"
#include "tdlb_geometry.hpp"
#include "tdlb_rotate.hpp"
#include "step_kernels.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace tdlb {

// One tank's view of one step (both streaming schemes).
struct TankStep {
    Planes A, B;                 // Simple: source / destination; Esotwist: A
    float* Nu;
    const float4* F;
    const uint32_t* mask;
    Dims g;
    CollideParams p;
    int les, from_moments, even, pad;
};

// One tank's impeller for the rotation launch.
struct TankRotor {
    const double* xz;            // blade offsets in the impeller frame
    Marker* out;                 // the blades of the resident marker list
    const double* table;         // [steps][3] cos a, sin a, delta a
    double ci, ck;
    int n, nx, nz, pad;
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
        simple_quad<S, V, LES, FM, true>(ts.A, ts.B, ts.Nu, ts.F, ts.mask, ts.g, ts.p, t);
    } else {
        if (ts.even) esotwist_quad<S, V, LES, FM, true, true>(ts.A, ts.Nu, ts.F, ts.mask, ts.g, ts.p, t);
        else esotwist_quad<S, V, LES, FM, true, false>(ts.A, ts.Nu, ts.F, ts.mask, ts.g, ts.p, t);
    }
}

// Quads of `NT` threads a work item covers: the tank's view is staged in
// shared memory once per item.
constexpr int kBatchChunks = 8;
// How far ahead of the chunk a block starts it prefetches into L2: about this
// many cells, at least one chunk (a chunk is NT x V cells). Measured on B200:
// the 64-tank Esotwist batch at its autotuned shapes (FP32 256-cell chunks,
// FP16 1024-cell chunks; fused launch, ms): FP32 1.381 without, 1.267 one
// chunk ahead, 1.318 two; FP16 1.027, 1.011, 1.016. The server's batches at
// the default shape (128-cell chunks), the first 64 requests of the serving
// stream: 20,623 MLUPS without, 20,373 one chunk ahead, 21,243 two. (A
// prefetch one wave of resident blocks ahead, as in the plain kernels, spans
// 8-chunk items and overran L2: 1.52 ms.)
constexpr int kBatchPrefetchCells = 256;

// L2 prefetch of the chunk of NT quads from quad q0 of the staged tank: NQ + 1
// threads issue one bulk prefetch each (plane d's source span of the chunk's
// elements, shifted as the pull reads them, and Nu's with LES), as the plain
// kernels do one wave ahead (prefetch_ahead). The from-moments step reads its
// own cells and takes the same spans.
template <typename S, int V, int NT, bool ESO>
__device__ __forceinline__ void prefetch_chunk(const TankStep& ts, unsigned q0) {
    const int d = (int)threadIdx.x;
    if (d > NQ || (d == NQ && !ts.les)) return;
    const Dims& g = ts.g;
    const long long e0 = (long long)q0 * V, e1 = e0 + (long long)NT * V;
    if (d == NQ) return prefetch_span(ts.Nu, 4, g.plane, e0, e1);
    const long long rs = (long long)g.ny * g.kp;
    long long sh;
    if (ESO) {
        const int sg = ts.even ? -1 : 1;
        sh = (sg * cx_of(d) > 0 ? rs : 0) + (sg * cy_of(d) > 0 ? g.kp : 0);
    } else {
        sh = -(cx_of(d) * rs + cy_of(d) * g.kp);
    }
    prefetch_span(ts.A.p[d], (int)sizeof(S), g.plane, e0 + sh - 1, e1 + sh + 1);
}

// Batched step: block b takes work items b, b + grid, ...; an item is
// kBatchChunks x NT consecutive quads of one tank (fewer at the end of a
// tank), whose step view is staged in shared memory; as it starts chunk c of
// an item, the block prefetches chunk c + ahead into L2 (ahead > 0). 16-bit storage
// never holds moments, so its from-moments bodies are not built. `counter` (may be
// NULL) is advanced once: this launch runs after the step's rotation, which
// reads it.
template <typename S, int V, int NT, bool ESO>
__global__ void __launch_bounds__(NT, (ESO ? kEsotwistBlocksPerSM<V> : 4) * 128 / NT) k_batch_step(const TankStep* __restrict__ tanks, const int2* __restrict__ work,
                                                   int nwork, int* counter, int ahead) {
    constexpr bool kFM = sizeof(S) == 4;
    __shared__ TankStep ts;
    if (counter && blockIdx.x == 0 && threadIdx.x == 0) *counter += 1;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 wk = work[w];
        __syncthreads();
        stage<NT>(ts, tanks + wk.x);
        __syncthreads();
        const unsigned nquads = (unsigned)ts.g.nx * (unsigned)ts.g.ny * (unsigned)(ts.g.kp / V);
        for (int c = 0; c < kBatchChunks; c++) {
            const unsigned t0 = (unsigned)wk.y + (unsigned)(c * NT);
            if (t0 >= nquads) break;   // uniform over the block
            if (ahead > 0 && c + ahead < kBatchChunks) prefetch_chunk<S, V, NT, ESO>(ts, t0 + (unsigned)(ahead * NT));
            const unsigned t = t0 + threadIdx.x;
            if (ts.les) {
                if (kFM && ts.from_moments) tank_quad<S, V, ESO, true, kFM>(ts, t);
                else tank_quad<S, V, ESO, true, false>(ts, t);
            } else {
                if (kFM && ts.from_moments) tank_quad<S, V, ESO, false, kFM>(ts, t);
                else tank_quad<S, V, ESO, false, false>(ts, t);
            }
        }
    }
}

// Blade rotation of every tank: work item = (tank, first of 256 blades).
__global__ void __launch_bounds__(256) k_rotate_batch(const TankRotor* __restrict__ rotors, const int2* __restrict__ work,
                                                      const int* __restrict__ step) {
    const int2 w = work[blockIdx.x];
    const TankRotor& r = rotors[w.x];
    const int q = w.y + threadIdx.x;
    if (q >= r.n) return;
    const double* tb = r.table + 3 * (size_t)(*step);
    const RotatedMarker m = rotate_marker(r.xz[2 * q], r.xz[2 * q + 1], tb[0], tb[1], tb[2], r.ci, r.ck, r.nx, r.nz);
    Marker& o = r.out[q];
    o.i = m.i;
    o.k = m.k;
    o.iCartFraction = m.iCartFraction;
    o.kCartFraction = m.kCartFraction;
    o.uDelta = m.uDelta;
    o.vDelta = 0.f;
    o.wDelta = m.wDelta;
}

using BatchFn = void (*)(const TankStep*, const int2*, int, int*, int);

template <typename S, bool ESO>
BatchFn pick(int v, int nt) {
    if (v == 1) return nt == 256 ? (BatchFn)k_batch_step<S, 1, 256, ESO> : (BatchFn)k_batch_step<S, 1, 128, ESO>;
    if constexpr (sizeof(S) == 4)
        if (v == 2) return nt == 256 ? (BatchFn)k_batch_step<S, 2, 256, ESO> : (BatchFn)k_batch_step<S, 2, 128, ESO>;
    return nt == 256 ? (BatchFn)k_batch_step<S, 4, 256, ESO> : (BatchFn)k_batch_step<S, 4, 128, ESO>;
}

BatchFn batch_kernel(int storage, bool eso, int v, int nt) {
    return with_storage(storage, [&](auto s) {
        using S = decltype(s);
        return eso ? pick<S, true>(v, nt) : pick<S, false>(v, nt);
    });
}

}  // namespace tdlb

using tdlb::TankRotor;
using tdlb::TankStep;

namespace {

// A device array of int2 work items, regrown as needed.
struct WorkList {
    int2* d = nullptr;
    int n = 0, cap = 0;
};

}  // namespace

// The tanks of a batch are split into two groups of about equal cell count,
// each with its own stream. A step runs, per group, the blade rotation, the
// fused step and the forcing pass; group 1's fused step waits for group 0's
// and group 0's next fused step for group 1's, so each group's forcing pass
// (latency-bound) runs while the other group's fused step (bandwidth-bound)
// has the GPU. Tanks are independent, so every tank computes what it
// computes alone.
struct BatchGroup {
    std::vector<int> tanks;            // indices into tdlb_batch_s::tanks
    WorkList work;                     // fused-step items (tank, first quad)
    WorkList rot_work;                 // (tank, first blade)
    std::vector<int2> rot_items;       // host copy of rot_work
    WorkList cells, tails, copies, small, big;   // immersed-boundary items
    int small_tile = 0, big_tile = 0;
    cudaStream_t stream = nullptr;     // group 0: the batch's stream
    cudaStream_t side = nullptr;       // large-plane spreads
    cudaStream_t ibm = nullptr;        // the forcing pass (high priority, as `side`)
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_fused = nullptr, ev_ibm = nullptr;
};

struct tdlb_batch_s {
    int device = 0;
    int storage = TDLB_STORAGE_FP32;   // shared by every tank
    int streaming = TDLB_STREAMING_SIMPLE;
    std::vector<tdlb_lattice*> tanks;
    int view_cap = 0;                  // tanks the per-tank device arrays hold
    bool members_changed = true;       // work lists and arrays must follow the tank list
    cudaStream_t stream = nullptr;     // the batch's stream (group 0's)
    cudaEvent_t ev_split = nullptr, ev_merge = nullptr;
    TankStep* d_steps = nullptr;       // [2][n]: views of an even and an odd step of a run
    tdlb::IbmArgs* d_ibm = nullptr;    // [2][n]: forcing passes of the same two steps
    WorkList work;                     // fused-step items of every tank (autotuner)
    BatchGroup grp[2];
    int* d_step = nullptr;             // [2] device step counters of a run (one per group)
    double* d_tables = nullptr;        // per rotating tank: [steps][3] cos, sin, delta, back to back
    size_t tables_cap = 0;             // doubles d_tables holds
    TankRotor* d_rotors = nullptr;     // [n]
    // Instantiated graphs of kPairsPerGraph step pairs (0) and of one pair
    // (1), kept while everything their launches name stays the same (key).
    struct CachedGraph {
        cudaGraphExec_t ge = nullptr;
        std::vector<uintptr_t> key;
        int kernels = 0;
    } graphs[2];
    std::vector<unsigned> ibm_gen;     // marker generation the IBM lists were built for
    int vec = 1, threads = 128, bps = 0;   // fused-launch shape (bps 0: one block per work item)
    int sms = 0;                           // SMs of the device
    int ibm_priority = 0;                  // the device's highest stream priority
    long long launches = 0;            // kernels run by tdlb_batch_run* so far
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

int storage_of(const tdlb_batch_s* b) { return b->storage; }
bool eso_of(const tdlb_batch_s* b) { return b->streaming == TDLB_STREAMING_ESOTWIST; }

// Upload `items` into `w` (the stream is idle: callers synchronise first).
void put(WorkList& w, const std::vector<int2>& items) {
    if ((int)items.size() > w.cap) {
        cudaFree(w.d);
        w.d = nullptr;
        w.cap = 0;
        TDLB_BCK(cudaMalloc(&w.d, std::max<size_t>(items.size(), 1) * sizeof(int2)));
        w.cap = (int)items.size();
    }
    if (!items.empty()) TDLB_BCK(cudaMemcpy(w.d, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice));
    w.n = (int)items.size();
}

void drop(WorkList& w) {
    cudaFree(w.d);
    w = WorkList{};
}

// The two groups: tanks by decreasing cell count, each to the group with
// fewer cells so far.
void assign_groups(tdlb_batch_s* b) {
    std::vector<int> order(b->tanks.size());
    for (size_t t = 0; t < order.size(); t++) order[t] = (int)t;
    auto cells = [&](int t) { return b->tanks[(size_t)t]->g.rows() * (long long)b->tanks[(size_t)t]->g.nz; };
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cells(x) > cells(y); });
    long long sum[2] = {0, 0};
    b->grp[0].tanks.clear();
    b->grp[1].tanks.clear();
    for (int t : order) {
        const int k = sum[1] < sum[0] ? 1 : 0;
        b->grp[k].tanks.push_back(t);
        sum[k] += cells(t);
    }
    for (BatchGroup& G : b->grp) std::sort(G.tanks.begin(), G.tanks.end());
}

// Waits for the batch's own two streams, not the whole device: tanks set up on
// their own streams (for tdlb_batch_adopt) keep running meanwhile.
cudaError_t quiesce(tdlb_batch_s* b) {
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e == cudaSuccess && b->grp[1].stream && b->grp[1].stream != b->stream) e = cudaStreamSynchronize(b->grp[1].stream);
    return e;
}

// Fused-step work lists for the current shape: (tank, first quad) per item,
// for every tank and per group.
void build_work(tdlb_batch_s* b) {
    auto items = [&](const std::vector<int>& ts) {
        std::vector<int2> w;
        for (int t : ts) {
            const Dims& g = b->tanks[(size_t)t]->g;
            const long long nq = g.rows() * (g.kp / b->vec);
            for (long long q = 0; q < nq; q += (long long)b->threads * tdlb::kBatchChunks) w.push_back(make_int2(t, (int)q));
        }
        return w;
    };
    std::vector<int> all(b->tanks.size());
    for (size_t t = 0; t < all.size(); t++) all[t] = (int)t;
    TDLB_BCK(quiesce(b));   // queued launches may still read the old lists
    put(b->work, items(all));
    for (BatchGroup& G : b->grp) put(G.work, items(G.tanks));
}

// Immersed-boundary work lists per group; rebuilt when a tank's markers changed.
void build_ibm_work(tdlb_batch_s* b) {
    bool same = true;
    for (size_t t = 0; t < b->tanks.size(); t++) same = same && b->ibm_gen[t] == b->tanks[t]->marker_gen;
    if (same) return;
    TDLB_BCK(quiesce(b));
    int small_all = 0, big_all = 0;
    for (BatchGroup& G : b->grp) {
        std::vector<int2> cells, tails, copies, small, big;
        int small_tile = 0, big_tile = 0;
        for (int t : G.tanks) {
            const tdlb_lattice* h = b->tanks[(size_t)t];
            if (!h->markers_set) continue;
            const int ncell = (int)h->cells.cell_e.size();
            for (int c = 0; c < ncell; c += 256) cells.push_back(make_int2(t, c));
            for (int q = 0; q < h->n_markers - h->n0; q += 128) tails.push_back(make_int2(t, q));
            for (long long wd = 0; wd < h->mask_words; wd += tdlb::kMaskCopyWords) copies.push_back(make_int2(t, (int)wd));
            for (int s = 0; s < h->n_small; s++) small.push_back(make_int2(t, h->h_plane_list[(size_t)s]));
            for (int s = 0; s < h->n_big; s++) big.push_back(make_int2(t, h->h_plane_list[(size_t)(h->n_small + s)]));
            small_tile = std::max(small_tile, h->smem_cells);
            if (h->n_big) big_tile = std::max(big_tile, h->big_tile_cells);
        }
        put(G.cells, cells);
        put(G.tails, tails);
        put(G.copies, copies);
        put(G.small, small);
        put(G.big, big);
        G.small_tile = small_tile;
        G.big_tile = big_tile;
        small_all = std::max(small_all, small_tile);
        big_all = std::max(big_all, big_tile);
    }
    TDLB_BCK(tdlb::ibm_batch_prepare_smem(tdlb::ibm_smem_bytes(Dims{}, small_all), tdlb::ibm_smem_bytes(Dims{}, big_all)));
    for (size_t t = 0; t < b->tanks.size(); t++) b->ibm_gen[t] = b->tanks[t]->marker_gen;
}

TankStep view_of(tdlb_lattice* h) {
    const tdlb::StepArgs a = tdlb_rt::step_args(h, true);
    TankStep s{};
    s.A = a.A;
    s.B = a.B;
    s.Nu = a.Nu;
    s.F = a.F;
    s.mask = a.mask;
    s.g = a.g;
    s.p = a.p;
    s.les = a.les;
    s.from_moments = a.from_moments;
    s.even = a.even;
    return s;
}

// Advance a tank's host bookkeeping over one fused step.
void advance_step_state(tdlb_lattice* h) {
    if (h->cfg.streaming == TDLB_STREAMING_SIMPLE) h->cur ^= 1;
    else h->even = !h->even;
    h->holds_moments = false;
}

// The fused launch over `work`: persistent blocks (bps per SM, each taking
// items b, b + grid, ...) or, with bps = 0, one block per item, so that the
// block scheduler fills the SMs the other group's forcing pass leaves free.
// A block prefetches the chunk about kBatchPrefetchCells cells after the one
// it starts, within its item.
void launch_fused(tdlb_batch_s* b, const TankStep* d_views, const WorkList& work, int* counter, cudaStream_t st) {
    if (work.n == 0) return;
    const tdlb::BatchFn fn = tdlb::batch_kernel(storage_of(b), eso_of(b), b->vec, b->threads);
    const int grid = b->bps > 0 ? std::min(work.n, b->sms * b->bps) : work.n;
    const int ahead = std::max(1, tdlb::kBatchPrefetchCells / (b->threads * b->vec));
    fn<<<grid, b->threads, 0, st>>>(d_views, work.d, work.n, counter, ahead);
    TDLB_BCK(cudaGetLastError());
}

// One batched step of both groups (also used inside capture). `k` selects
// the uploaded views (0: first step of the pair, 1: second); `first`: no
// earlier step of this sequence, so group 0 need not wait for group 1.
// Returns the number of kernels it queued.
int queue_step(tdlb_batch_s* b, int k, bool first) {
    const size_t n = b->tanks.size();
    int kernels = 0;
    for (int gi = 0; gi < 2; gi++) {
        BatchGroup& G = b->grp[gi];
        BatchGroup& other = b->grp[gi ^ 1];
        if (G.tanks.empty()) continue;
        if (G.rot_work.n) {
            tdlb::k_rotate_batch<<<G.rot_work.n, 256, 0, G.stream>>>(b->d_rotors, G.rot_work.d, b->d_step + gi);
            TDLB_BCK(cudaGetLastError());
            kernels++;
        }
        // the fused steps of the two groups take turns
        if (!other.tanks.empty() && (gi == 1 || !first)) TDLB_BCK(cudaStreamWaitEvent(G.stream, other.ev_fused, 0));
        launch_fused(b, b->d_steps + (size_t)k * n, G.work, b->d_step + gi, G.stream);
        TDLB_BCK(cudaEventRecord(G.ev_fused, G.stream));
        kernels++;
        // the forcing pass runs on a high-priority stream, so that its
        // latency-bound blocks get SM slots ahead of the other group's fused
        // launch; the group's next rotation waits for it
        TDLB_BCK(cudaStreamWaitEvent(G.ibm, G.ev_fused, 0));
        tdlb::IbmBatch ib{};
        ib.args = b->d_ibm + (size_t)k * n;
        ib.cells = G.cells.d; ib.n_cells = G.cells.n;
        ib.tails = G.tails.d; ib.n_tails = G.tails.n;
        ib.copies = G.copies.d; ib.n_copies = G.copies.n;
        ib.small = G.small.d; ib.n_small = G.small.n;
        ib.big = G.big.d; ib.n_big = G.big.n;
        ib.small_tile = G.small_tile;
        ib.big_tile = G.big_tile;
        ib.storage = storage_of(b);
        TDLB_BCK(tdlb::launch_ibm_batch(ib, G.ibm, G.side, G.ev_fork, G.ev_join));
        kernels += (ib.n_cells > 0) + (ib.n_tails > 0) + (ib.n_copies > 0) + (ib.n_small > 0) + (ib.n_big > 0);
        TDLB_BCK(cudaEventRecord(G.ev_ibm, G.ibm));
        TDLB_BCK(cudaStreamWaitEvent(G.stream, G.ev_ibm, 0));
    }
    for (tdlb_lattice* h : b->tanks) {
        advance_step_state(h);
        if (h->markers_set) h->pass++;
    }
    return kernels;
}

// Group 1's stream joins the batch's stream (fork) and leaves it (merge).
void split_streams(tdlb_batch_s* b) {
    TDLB_BCK(cudaEventRecord(b->ev_split, b->stream));
    TDLB_BCK(cudaStreamWaitEvent(b->grp[1].stream, b->ev_split, 0));
}
void merge_streams(tdlb_batch_s* b) {
    TDLB_BCK(cudaEventRecord(b->ev_merge, b->grp[1].stream));
    TDLB_BCK(cudaStreamWaitEvent(b->stream, b->ev_merge, 0));
}

// Views and forcing arguments of the next two steps, uploaded in stream
// order (launches already queued read the previous ones). The host state is
// left as it was.
void upload_views(tdlb_batch_s* b, float alpha, float beta) {
    const size_t n = b->tanks.size();
    std::vector<TankStep> v(2 * n);
    std::vector<tdlb::IbmArgs> ia(2 * n);
    std::vector<int> cur(n), pass(n);
    std::vector<char> even(n), hm(n);
    for (size_t t = 0; t < n; t++) {
        tdlb_lattice* h = b->tanks[t];
        cur[t] = h->cur; pass[t] = h->pass; even[t] = h->even; hm[t] = h->holds_moments;
    }
    for (int k = 0; k < 2; k++)
        for (size_t t = 0; t < n; t++) {
            tdlb_lattice* h = b->tanks[t];
            v[(size_t)k * n + t] = view_of(h);
            advance_step_state(h);
            ia[(size_t)k * n + t] = tdlb_rt::ibm_args(h, alpha, beta);
            if (h->markers_set) h->pass++;
        }
    for (size_t t = 0; t < n; t++) {
        tdlb_lattice* h = b->tanks[t];
        h->cur = cur[t]; h->pass = pass[t]; h->even = even[t]; h->holds_moments = hm[t];
    }
    TDLB_BCK(cudaMemcpyAsync(b->d_steps, v.data(), v.size() * sizeof(TankStep), cudaMemcpyHostToDevice, b->stream));
    TDLB_BCK(cudaMemcpyAsync(b->d_ibm, ia.data(), ia.size() * sizeof(tdlb::IbmArgs), cudaMemcpyHostToDevice, b->stream));
}

// Per-step (cos, sin, delta) of every attached impeller for `steps` steps,
// and the rotation launch's tank table: one allocation and two asynchronous
// copies on the batch's stream (run() has waited for the previous run, the
// only reader). The rotation work lists are rebuilt only when they change.
void build_tables(tdlb_batch_s* b, int steps) {
    const size_t n = b->tanks.size();
    std::vector<TankRotor> rot(n);
    std::vector<size_t> off(n, 0);
    size_t total = 0;
    for (size_t t = 0; t < n; t++) {
        const tdlb_lattice* h = b->tanks[t];
        if (!h->rot_device || h->n_markers == h->n0) continue;
        off[t] = total;
        total += (size_t)3 * steps;
    }
    if (total > b->tables_cap) {
        cudaFree(b->d_tables);
        b->d_tables = nullptr;
        b->tables_cap = 0;
        TDLB_BCK(cudaMalloc(&b->d_tables, total * sizeof(double)));
        b->tables_cap = total;
    }
    std::vector<double> tab(total);
    for (size_t t = 0; t < n; t++) {
        tdlb_lattice* h = b->tanks[t];
        rot[t] = TankRotor{};
        if (!h->rot_device || h->n_markers == h->n0) continue;
        const tdlb::RushtonGeom G = tdlb::RushtonGeom::from(h->rspec);
        double* tt = tab.data() + off[t];
        double angle = h->angle;
        unsigned long long st = h->rstep;
        for (int s = 0; s < steps; s++) {
            st++;
            const double d = G.increment(st);
            angle += d;
            tt[(size_t)3 * s] = std::cos(angle);
            tt[(size_t)3 * s + 1] = std::sin(angle);
            tt[(size_t)3 * s + 2] = d;
        }
        const int nr = h->n_markers - h->n0;
        rot[t] = TankRotor{h->d_rot_xz, h->d_markers + h->n0, b->d_tables + off[t], h->rot_ci, h->rot_ck, nr, h->g.nx,
                           h->g.nz, 0};
    }
    if (total) TDLB_BCK(cudaMemcpyAsync(b->d_tables, tab.data(), total * sizeof(double), cudaMemcpyHostToDevice, b->stream));
    // (copies from pageable memory are staged before the calls return)
    TDLB_BCK(cudaMemcpyAsync(b->d_rotors, rot.data(), n * sizeof(TankRotor), cudaMemcpyHostToDevice, b->stream));
    for (BatchGroup& G : b->grp) {
        std::vector<int2> items;
        for (int t : G.tanks)
            for (int q = 0; q < rot[(size_t)t].n; q += 256) items.push_back(make_int2(t, q));
        const bool same = items.size() == G.rot_items.size() &&
                          (items.empty() || std::memcmp(items.data(), G.rot_items.data(), items.size() * sizeof(int2)) == 0);
        if (!same) {
            put(G.rot_work, items);
            G.rot_items = items;
        }
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

// Per-tank device arrays for at least the current number of tanks.
void ensure_capacity(tdlb_batch_s* b) {
    const int n = (int)b->tanks.size();
    if (n <= b->view_cap) return;
    const int cap = std::max(n, 2 * b->view_cap);
    TDLB_BCK(cudaStreamSynchronize(b->stream));
    cudaFree(b->d_steps);
    cudaFree(b->d_ibm);
    cudaFree(b->d_rotors);
    b->d_steps = nullptr;
    b->d_ibm = nullptr;
    b->d_rotors = nullptr;
    b->view_cap = 0;
    TDLB_BCK(cudaMalloc(&b->d_steps, (size_t)2 * cap * sizeof(TankStep)));
    TDLB_BCK(cudaMalloc(&b->d_ibm, (size_t)2 * cap * sizeof(tdlb::IbmArgs)));
    TDLB_BCK(cudaMalloc(&b->d_rotors, (size_t)cap * sizeof(TankRotor)));
    b->view_cap = cap;
}

// After tanks joined or left: arrays, fused work list and (through the
// generation check) the immersed-boundary lists follow the new tank list.
void sync_members(tdlb_batch_s* b) {
    if (!b->members_changed) return;
    ensure_capacity(b);
    assign_groups(b);
    build_work(b);
    for (auto& g : b->ibm_gen) g = ~0u;
    b->members_changed = false;
}

tdlb_lattice* add_tank(tdlb_batch_s* b, const tdlb_config& cfg) {
    if (cfg.streaming != b->streaming || cfg.storage != b->storage)
        throw BFail{TDLB_EINVAL, "all tanks of a batch share one streaming scheme and one storage precision"};
    tdlb_handle h = nullptr;
    const int rc = tdlb_create_config(&cfg, b->device, &h);
    if (rc != TDLB_OK) throw BFail{rc, std::string("tank: ") + tdlb_last_error(nullptr)};
    tdlb_rt::borrow_stream(h, b->stream);
    h->vec = b->vec;
    b->tanks.push_back(h);
    b->ibm_gen.push_back(~0u);
    b->members_changed = true;
    return h;
}

// A lattice created and prepared on its own stream joins the batch: its
// stream is drained and replaced by the batch's (as for add_tank), and the
// batch owns it from then on.
void adopt_tank(tdlb_batch_s* b, tdlb_lattice* h) {
    if (!h) throw BFail{TDLB_EINVAL, "handle is NULL"};
    if (h->own_stream) throw BFail{TDLB_ESTATE, "the lattice already belongs to a batch"};
    if (h->cfg.streaming != b->streaming || h->cfg.storage != b->storage)
        throw BFail{TDLB_EINVAL, "all tanks of a batch share one streaming scheme and one storage precision"};
    if (h->device != b->device) throw BFail{TDLB_EINVAL, "the lattice lives on another device"};
    // the batched step keeps no 16-bit residuals: the tank continues at its
    // storage precision everywhere
    tdlb_rt::drop_residual_box(h);
    tdlb_rt::borrow_stream(h, b->stream);
    h->vec = b->vec;
    b->tanks.push_back(h);
    b->ibm_gen.push_back(~0u);
    b->members_changed = true;
}

// The inverse of adopt_tank: tank t leaves the batch without being
// destroyed, once the batch's streams are idle, and runs on its own stream
// again; the caller owns it. Later tanks move down by one.
tdlb_lattice* detach_tank(tdlb_batch_s* b, int t) {
    if (t < 0 || t >= (int)b->tanks.size()) throw BFail{TDLB_EINVAL, "tank index out of range"};
    TDLB_BCK(quiesce(b));
    tdlb_lattice* h = b->tanks[(size_t)t];
    tdlb_rt::return_stream(h);
    h->vec = tdlb_rt::default_cells_per_thread(h->cfg);
    b->tanks.erase(b->tanks.begin() + t);
    b->ibm_gen.erase(b->ibm_gen.begin() + t);
    b->members_changed = true;
    return h;
}

void remove_tank(tdlb_batch_s* b, int t) {
    if (t < 0 || t >= (int)b->tanks.size()) throw BFail{TDLB_EINVAL, "tank index out of range"};
    TDLB_BCK(cudaStreamSynchronize(b->stream));
    tdlb_destroy(b->tanks[(size_t)t]);
    b->tanks.erase(b->tanks.begin() + t);
    b->ibm_gen.erase(b->ibm_gen.begin() + t);
    b->members_changed = true;
}

void check_ready(tdlb_batch_s* b) {
    for (tdlb_lattice* h : b->tanks)
        if (!h->initialised) throw BFail{TDLB_ESTATE, "every tank must be initialised first"};
}

// Pairs of steps per captured graph: the two groups' pipeline drains at the
// end of each replay.
constexpr int kPairsPerGraph = 4;

// One eager step: uploads follow every queued launch of both groups.
void eager_step(tdlb_batch_s* b, float alpha, float beta) {
    merge_streams(b);
    upload_views(b, alpha, beta);
    split_streams(b);
    b->launches += queue_step(b, 0, true);
}

// Everything a captured step pair names on the host side: launch shapes,
// work lists, device arrays, streams. A cached graph is replayed only while
// its key is unchanged (the views, tables and rotors it reads are device
// arrays rewritten before every run).
std::vector<uintptr_t> graph_key(const tdlb_batch_s* b, int P) {
    std::vector<uintptr_t> k = {(uintptr_t)P, b->tanks.size(), (uintptr_t)b->vec, (uintptr_t)b->threads,
                                (uintptr_t)b->bps, (uintptr_t)b->d_steps, (uintptr_t)b->d_ibm,
                                (uintptr_t)b->d_rotors, (uintptr_t)b->d_step};
    for (const BatchGroup& G : b->grp) {
        k.push_back(G.tanks.size());
        k.push_back((uintptr_t)G.stream);
        k.push_back((uintptr_t)G.side);
        for (const WorkList* w : {&G.work, &G.rot_work, &G.cells, &G.tails, &G.copies, &G.small, &G.big}) {
            k.push_back((uintptr_t)w->d);
            k.push_back((uintptr_t)w->n);
        }
        k.push_back((uintptr_t)G.small_tile);
        k.push_back((uintptr_t)G.big_tile);
    }
    return k;
}

// Sets the launch priority of every kernel node of g except those of `keep`.
cudaError_t prioritise_nodes(cudaGraph_t g, const void* keep, int priority) {
    size_t n = 0;
    cudaError_t e = cudaGraphGetNodes(g, nullptr, &n);
    if (e != cudaSuccess) return e;
    std::vector<cudaGraphNode_t> nodes(n);
    e = cudaGraphGetNodes(g, nodes.data(), &n);
    if (e != cudaSuccess) return e;
    for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType type;
        e = cudaGraphNodeGetType(nd, &type);
        if (e != cudaSuccess) return e;
        if (type != cudaGraphNodeTypeKernel) continue;
        cudaKernelNodeParams kp{};
        e = cudaGraphKernelNodeGetParams(nd, &kp);
        if (e != cudaSuccess) return e;
        if (kp.func == keep) continue;
        cudaLaunchAttributeValue v{};
        v.priority = priority;
        e = cudaGraphKernelNodeSetAttribute(nd, cudaLaunchAttributePriority, &v);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// The instantiated graph of P step pairs for the current batch: the cached
// one while its key holds, else a new capture (the old one is destroyed).
cudaGraphExec_t graph_for(tdlb_batch_s* b, int P, int& kernels) {
    tdlb_batch_s::CachedGraph& c = b->graphs[P == 1 ? 1 : 0];
    std::vector<uintptr_t> key = graph_key(b, P);
    if (c.ge && c.key == key) {
        kernels = c.kernels;
        return c.ge;
    }
    if (c.ge) {
        cudaGraphExecDestroy(c.ge);
        c.ge = nullptr;
    }
    cudaGraph_t g = nullptr;
    int per_graph = 0;
    TDLB_BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    try {
        split_streams(b);
        for (int p = 0; p < P; p++) {
            per_graph += queue_step(b, 0, p == 0);
            per_graph += queue_step(b, 1, false);
        }
        merge_streams(b);
    } catch (...) {
        cudaStreamEndCapture(b->stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    TDLB_BCK(cudaStreamEndCapture(b->stream, &g));
    // the capture advanced the host state by 2P steps (the parity is back
    // where it was); the replays run them
    for (tdlb_lattice* h : b->tanks)
        if (h->markers_set) h->pass -= 2 * P;
    // every kernel but the fused launch (forcing passes, rotations) keeps the
    // high priority of the streams it was captured from
    cudaError_t pe = prioritise_nodes(g, (const void*)tdlb::batch_kernel(storage_of(b), eso_of(b), b->vec, b->threads),
                                      b->ibm_priority);
    cudaGraphExec_t ge = nullptr;
    const cudaError_t ie = pe != cudaSuccess ? pe : cudaGraphInstantiateWithFlags(&ge, g, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(g);
    TDLB_BCK(ie);
    c.ge = ge;
    c.key = std::move(key);
    c.kernels = per_graph;
    kernels = per_graph;
    return ge;
}

// `steps` steps, eager or graph-replayed. A step whose state still holds
// moments (right after initialise) runs eagerly: its views differ from the
// repeating pair's.
void run(tdlb_batch_s* b, int steps, float alpha, float beta, bool graph) {
    if (b->tanks.empty()) return;
    check_ready(b);
    TDLB_BCK(quiesce(b));   // the previous run may still read the tables and lists
    sync_members(b);
    build_ibm_work(b);
    build_tables(b, steps);
    TDLB_BCK(cudaMemsetAsync(b->d_step, 0, 2 * sizeof(int), b->stream));
    int done = 0;
    bool any_moments = false;
    for (tdlb_lattice* h : b->tanks) any_moments = any_moments || h->holds_moments;
    while (done < steps && (any_moments || !graph || steps - done < 2)) {
        eager_step(b, alpha, beta);
        done++;
        any_moments = false;
    }
    int pairs = (steps - done) / 2;
    if (pairs > 0) {
        merge_streams(b);
        upload_views(b, alpha, beta);
        // graphs of kPairsPerGraph pairs, then of one pair; both read the
        // views just uploaded (an even number of steps ends on the parity it
        // started from)
        for (int P : {kPairsPerGraph, 1}) {
            const int replays = pairs / P;
            if (replays == 0) continue;
            int kernels = 0;
            const cudaGraphExec_t ge = graph_for(b, P, kernels);
            for (int r = 0; r < replays; r++) TDLB_BCK(cudaGraphLaunch(ge, b->stream));
            for (tdlb_lattice* h : b->tanks)
                if (h->markers_set) h->pass += 2 * P * replays;
            b->launches += (long long)kernels * replays;
            done += 2 * P * replays;
            pairs -= P * replays;
        }
        if (done < steps) eager_step(b, alpha, beta);   // an odd last step
    }
    merge_streams(b);
    finish_tables(b, steps);
    for (tdlb_lattice* h : b->tanks)
        if (h->markers_set) h->last_beta = beta;   // for tdlb_impeller_load
}

void release(tdlb_batch_s* b) {
    cudaSetDevice(b->device);
    cudaDeviceSynchronize();
    for (tdlb_lattice* h : b->tanks) tdlb_destroy(h);
    for (auto& c : b->graphs)
        if (c.ge) cudaGraphExecDestroy(c.ge);
    cudaFree(b->d_tables);
    drop(b->work);
    for (BatchGroup& G : b->grp) {
        for (WorkList* w : {&G.work, &G.rot_work, &G.cells, &G.tails, &G.copies, &G.small, &G.big}) drop(*w);
        if (G.ev_fork) cudaEventDestroy(G.ev_fork);
        if (G.ev_join) cudaEventDestroy(G.ev_join);
        if (G.ev_fused) cudaEventDestroy(G.ev_fused);
        if (G.ev_ibm) cudaEventDestroy(G.ev_ibm);
        if (G.side) cudaStreamDestroy(G.side);
        if (G.ibm) cudaStreamDestroy(G.ibm);
        if (G.stream && G.stream != b->stream) cudaStreamDestroy(G.stream);
    }
    cudaFree(b->d_steps);
    cudaFree(b->d_ibm);
    cudaFree(b->d_rotors);
    cudaFree(b->d_step);
    if (b->ev_split) cudaEventDestroy(b->ev_split);
    if (b->ev_merge) cudaEventDestroy(b->ev_merge);
    if (b->stream) cudaStreamDestroy(b->stream);
}

// Streams, events and the step counters of a new batch.
void init_streams(tdlb_batch_s* b) {
    TDLB_BCK(cudaSetDevice(b->device));
    TDLB_BCK(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device));
    int least = 0;
    TDLB_BCK(cudaDeviceGetStreamPriorityRange(&least, &b->ibm_priority));
    TDLB_BCK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    TDLB_BCK(cudaEventCreateWithFlags(&b->ev_split, cudaEventDisableTiming));
    TDLB_BCK(cudaEventCreateWithFlags(&b->ev_merge, cudaEventDisableTiming));
    for (int gi = 0; gi < 2; gi++) {
        BatchGroup& G = b->grp[gi];
        if (gi == 0) G.stream = b->stream;
        else TDLB_BCK(cudaStreamCreateWithFlags(&G.stream, cudaStreamNonBlocking));
        TDLB_BCK(cudaStreamCreateWithPriority(&G.side, cudaStreamNonBlocking, b->ibm_priority));
        TDLB_BCK(cudaStreamCreateWithPriority(&G.ibm, cudaStreamNonBlocking, b->ibm_priority));
        TDLB_BCK(cudaEventCreateWithFlags(&G.ev_fork, cudaEventDisableTiming));
        TDLB_BCK(cudaEventCreateWithFlags(&G.ev_join, cudaEventDisableTiming));
        TDLB_BCK(cudaEventCreateWithFlags(&G.ev_fused, cudaEventDisableTiming));
        TDLB_BCK(cudaEventCreateWithFlags(&G.ev_ibm, cudaEventDisableTiming));
    }
    TDLB_BCK(cudaMalloc(&b->d_step, 2 * sizeof(int)));
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
    b->storage = cfgs[0].storage;
    b->streaming = cfgs[0].streaming;
    b->vec = 1;
    try {
        init_streams(b);
        for (int t = 0; t < n; t++) add_tank(b, cfgs[t]);
        sync_members(b);
    } catch (const BFail& f) {
        g_batch_create_error = f.msg;
        release(b);
        delete b;
        return f.code;
    }
    *out = b;
    return TDLB_OK;
}

int tdlb_batch_create_empty(int device, int streaming, int storage, tdlb_batch* out) {
    if (!out || (streaming != TDLB_STREAMING_SIMPLE && streaming != TDLB_STREAMING_ESOTWIST) ||
        storage < TDLB_STORAGE_FP32 || storage > TDLB_STORAGE_BF16) {
        g_batch_create_error = "bad arguments";
        return TDLB_EINVAL;
    }
    *out = nullptr;
    auto* b = new tdlb_batch_s();
    b->device = device;
    b->storage = storage;
    b->streaming = streaming;
    b->vec = 1;
    try {
        init_streams(b);
    } catch (const BFail& f) {
        g_batch_create_error = f.msg;
        release(b);
        delete b;
        return f.code;
    }
    *out = b;
    return TDLB_OK;
}

int tdlb_batch_add(tdlb_batch b, const tdlb_config* cfg, int* index) {
    return bguard(b, [&] {
        if (!cfg) throw BFail{TDLB_EINVAL, "cfg is NULL"};
        add_tank(b, *cfg);
        if (index) *index = (int)b->tanks.size() - 1;
    });
}

int tdlb_batch_adopt(tdlb_batch b, tdlb_handle h, int* index) {
    return bguard(b, [&] {
        adopt_tank(b, h);
        if (index) *index = (int)b->tanks.size() - 1;
    });
}

int tdlb_batch_detach(tdlb_batch b, int index, tdlb_handle* out) {
    return bguard(b, [&] {
        if (!out) throw BFail{TDLB_EINVAL, "out is NULL"};
        *out = detach_tank(b, index);
    });
}

int tdlb_batch_remove(tdlb_batch b, int index) {
    return bguard(b, [&] { remove_tank(b, index); });
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
        if (blocks_per_sm < 0 || blocks_per_sm > 16) throw BFail{TDLB_EINVAL, "blocks per SM must be 0..16"};
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
// own (initialised) tanks and keeps the fastest. The timed launches repeat
// the next step's view, so they change the fields; callers initialise again.
int tdlb_batch_autotune(tdlb_batch b, int trials, double* best_ms) {
    return bguard(b, [&] {
        if (b->tanks.empty()) throw BFail{TDLB_ESTATE, "the batch has no tanks"};
        check_ready(b);
        sync_members(b);
        if (trials < 1) trials = 3;
        struct Cand { int v, nt, bps; };
        std::vector<Cand> cands;
        const bool h16 = storage_of(b) != TDLB_STORAGE_FP32;
        for (int v : {1, 2, 4}) {
            if (h16 && v == 2) continue;
            for (int nt : {128, 256})
                for (int bps : {0, 4, 8}) cands.push_back({v, nt, bps});
        }
        TDLB_BCK(quiesce(b));
        upload_views(b, 0.f, 0.f);
        cudaEvent_t e0, e1;
        TDLB_BCK(cudaEventCreate(&e0));
        TDLB_BCK(cudaEventCreate(&e1));
        float best = 1e30f;
        Cand win = cands[0];
        try {
            for (const Cand& c : cands) {
                b->vec = c.v; b->threads = c.nt; b->bps = c.bps;
                        build_work(b);
                launch_fused(b, b->d_steps, b->work, nullptr, b->stream);   // warm-up
                TDLB_BCK(cudaEventRecord(e0, b->stream));
                for (int r = 0; r < trials; r++) launch_fused(b, b->d_steps, b->work, nullptr, b->stream);
                TDLB_BCK(cudaEventRecord(e1, b->stream));
                TDLB_BCK(cudaEventSynchronize(e1));
                float ms = 0.f;
                TDLB_BCK(cudaEventElapsedTime(&ms, e0, e1));
                ms /= trials;
                if (ms < best) { best = ms; win = c; }
            }
        } catch (...) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
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
    return bguard(b, [&] {
        TDLB_BCK(cudaStreamSynchronize(b->stream));
        TDLB_BCK(cudaStreamSynchronize(b->grp[1].stream));
    });
}

int tdlb_batch_get_stream(tdlb_batch b, void** stream) {
    return bguard(b, [&] {
        if (!stream) throw BFail{TDLB_EINVAL, "out is NULL"};
        *stream = (void*)b->stream;
    });
}

}  // extern "C"
