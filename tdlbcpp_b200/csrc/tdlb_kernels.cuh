// Internal interface between the host runtime (tdlb_capi.cu) and the kernels.
#pragma once
#include <atomic>
#include "tdlb_common.cuh"

namespace tdlb {

// Chunks of a split step (32 consecutive elements of the flat row*kp + k
// index, one warp each): the launch takes chunks[0, count). A full launch
// (part 0) takes no list; l2_ahead > 0 turns on its L2 prefetch, that many
// CTAs ahead of the walk (step_kernels.cuh).
struct StepPart {
    const int* chunks;
    int count;
    int l2_ahead;
};
constexpr int kSplitChunk = 32;

// One wave of resident 128-thread CTAs of kernel K on the current device (the
// occupancy its register count allows, times the SMs): the L2 prefetch
// distance of a full launch. Queried once per kernel; 0 (prefetch off) if the
// query fails.
template <auto K>
int wave_ctas() {
    static std::atomic<int> n{0};
    int v = n.load(std::memory_order_relaxed);
    if (v == 0) {
        int dev = 0, sms = 0, per = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, K, 128, 0) == cudaSuccess && per > 0 && sms > 0) {
            v = per * sms;
            n.store(v, std::memory_order_relaxed);
        }
    }
    return v;
}

// Arguments of one fused step launch.
struct StepArgs {
    Planes A;               // Simple: source buffer; Esotwist: the single buffer
    Planes B;               // Simple: destination buffer (unused for Esotwist)
    float* Nu;
    const float4* F;        // force, one float4 (Fx, Fy, Fz, unused) per element
    const uint32_t* mask;   // IBM-touched flags of the forcing pass this step uses
    Dims g;
    CollideParams p;
    int les;                // Smagorinsky LES on/off (FlowParams::useLES)
    int from_moments;       // state holds moments (after initialise / checkpoint load)
    int collide;            // 0: transport only (identity collision; known-answer tests)
    int even;               // Esotwist parity (evenStep)
    int vec;                // cells per thread: 1, 2 or 4 (float, float2, float4 traffic)
    int l2_prefetch;        // full launches of the population form: L2 prefetch one wave ahead
    int storage;            // StorageKind of the population planes
    int part;               // 0: every cell; 1: outer chunks; 2: inner chunks (vec == 1, populations)
    StepPart zone;          // the chunks of part 1 or 2 (box == 2: the chunks near the residual box)
    ResidualBox rr;         // 16-bit storage, one cell per thread: residuals of the locations read ...
    ResidualBox rw;         // ... and written (Simple: of buffer A and B; Esotwist: the same box)
    int box;                // 0: no residual box; 2: the box launch over `zone` (the chunks near the box, part 2)
    BoxOut bout;            // box launch: its scratch outputs
};

// The StepPart a launch of kernel K takes: the chunk list (parts 1 and 2) or,
// for a full launch of the population form (FULL) with a.l2_prefetch on, the
// L2 prefetch distance of one wave of K's resident CTAs.
template <auto K, bool FULL>
StepPart launch_walk(const StepArgs& a) {
    StepPart w = a.zone;
    w.l2_ahead = FULL && a.part == 0 && a.l2_prefetch ? wave_ctas<K>() : 0;
    return w;
}

cudaError_t launch_step_simple(const StepArgs& a, cudaStream_t st);
cudaError_t launch_step_esotwist(const StepArgs& a, cudaStream_t st);
cudaError_t launch_step_simple_h16(const StepArgs& a, cudaStream_t st);
cudaError_t launch_step_esotwist_h16(const StepArgs& a, cudaStream_t st);
// After the plain launch of a step with a residual box: the box launch's
// outputs (a.bout) to the cells of a.zone (k_box_commit).
cudaError_t launch_box_commit(const StepArgs& a, bool simple, cudaStream_t st);
cudaError_t launch_fill_uniform_moments(Planes Q, const Dims& g, float rho, cudaStream_t st);
cudaError_t launch_state_moments(Planes A, Planes M, const Dims& g, int mode, int even, cudaStream_t st, int storage,
                                 const CollideParams& p, const ResidualBox& rb = ResidualBox{});

// ---- immersed boundary ----

// Marker record, identical in layout to tdlb_marker (include/tdlb_b200.h).
struct Marker {
    long long i, j, k;
    float iCartFraction, kCartFraction, uDelta, vDelta, wDelta, pad;
};
static_assert(sizeof(Marker) == 48, "Marker layout");

// Blade (second-segment) scratch written by k_ibm_gather_tail, read by the
// spread walk; field-major over the segment's slots.
enum TailField {
    TF_W = 0,               // 9 stencil weights, (k1, i1) order
    TF_RHO = 9,             // 9 densities
    TF_MX = 18, TF_MY = 27, TF_MZ = 36,   // 9 momenta each
    TF_U = 45, TF_V = 46, TF_WV = 47,     // marker velocity
    TF_CELL = 48,           // 9 packed (i << 16 | k) cells (int32 bit patterns)
    TF_COUNT = 57
};

// First-segment (static markers) data prepared once per upload, per slot
// p < n0: 9 weights, 9 plane-local cell indices, the marker velocity.
enum PrepField {
    PF_W = 0,
    PF_CELL = 9,            // int32 bit patterns
    PF_U = 18, PF_V = 19, PF_WV = 20,
    PF_STRIDE = 24          // floats per marker: marker-major rows of 96 bytes (six float4 loads)
};

struct IbmArgs {
    const Marker* markers;      // device copy of the marker list (list order)
    const int* sched;           // execution order: marker index per slot
    const int* level_ptr;       // [nlevels+1] slot offsets of each level
    const int* plane_lv0;       // [ny+1] levels of each j-plane, first segment
    const int* plane_lv1;       // [ny+1] levels of each j-plane, second segment (walked after the first)
    int n;                      // number of markers
    int n0;                     // markers (slots) of the first segment
    // first segment: unique stencil cells, sorted by (j, i, k)
    const int* cell_e;          // [C0] element index of each cell
    const int* plane_cell;      // [ny+1] cell range of each plane
    int ncell;                  // C0
    const int* cell_order;      // [C0] the big planes' cells, then the others (NULL: no big plane)
    int ncell_big;              // cells of the big planes
    const float* prep;          // PF_STRIDE * n0: one row per first-segment slot
    float* cell_m;              // C0 float4: rho, jx, jy, jz of each cell this pass
    float* cell_F;              // 3 * C0: F of each cell at the start of this pass
    float* tail;                // TF_COUNT * ntail_cap
    long long tail_cap;
    float* sums;                // 3 * n: each slot's spread sums (for the impeller load)
    int smem_cells;             // F tile capacity of the small-plane launch
    const int* plane_list;      // [ny] small planes first, then the big ones
    int n_small, n_big;         // planes in each launch
    const int* blade_planes;    // the planes with blade levels (the blade launch)
    int n_blade, blade_words;   // their count; shared-memory floats of the blade launch
    int big_tile_cells;         // F tile capacity of the big-plane launch
    cudaStream_t side;          // stream of the big-plane launch
    cudaEvent_t ev_fork, ev_join;
    Planes A;                   // current state
    int state_mode;             // 0 Simple pops, 1 moments, 2 Esotwist pops, 3 Esotwist moments
    int even;                   // Esotwist parity of the state's read map
    float4* F4;                 // force, one float4 (Fx, Fy, Fz, unused) per element
    const uint32_t* mask_old;   // touched flags of the previous forcing pass
    uint32_t* mask_new;         // touched flags of this pass (fully written)
    const uint32_t* mask_static;   // touched flags of the first segment (every pass)
    size_t mask_bytes;
    Dims g;
    float alpha, beta;
    int storage;                // StorageKind of the state planes
    CollideParams p;            // rest offsets of the 16-bit storage
    ResidualBox rbox;           // residuals of the state's locations (16-bit storage; off: res == NULL)
};

cudaError_t launch_ibm(const IbmArgs& a, cudaStream_t st);

// Immersed-boundary passes of many lattices in one set of launches: device
// IbmArgs per lattice and work lists of (lattice, first index) items --
// cells: 256 first-segment cells; tails: 128 blade markers; copies: 1024
// touched-flag words; small / big: one j-plane (128 / 512 threads).
struct IbmBatch {
    const IbmArgs* args;
    const int2* cells; int n_cells;
    const int2* tails; int n_tails;
    const int2* copies; int n_copies;
    const int2* small; int n_small;
    const int2* big; int n_big;
    int small_tile, big_tile;   // dynamic F tiles (cells) of the two spread launches
    int storage;
};
constexpr int kMaskCopyWords = 1024;
cudaError_t launch_ibm_batch(const IbmBatch& b, cudaStream_t st, cudaStream_t side, cudaEvent_t fork, cudaEvent_t join);
cudaError_t ibm_batch_prepare_smem(size_t small_bytes, size_t big_bytes);
// Per-upload preparation of the first segment (weights, velocities).
cudaError_t launch_ibm_prepare(const IbmArgs& a, float* prep, const int* mcell, cudaStream_t st);
// Shared memory the spread kernel needs: the plane's touched-flag tile plus
// an F tile of `cells` cells.
size_t ibm_smem_bytes(const Dims& g, int cells);
// Opt the spread kernels in to the dynamic shared memory of the ordinary
// planes' launch (tiles of `small_cells` cells) and of the big planes'
// launch (`big_bytes`).
cudaError_t ibm_prepare_smem(int small_cells, int n_small, size_t big_bytes);
// Shared memory of the big planes' launch for a tile of `big_cells` cells.
size_t big_bulk_bytes(int big_cells);
// Shared-memory floats of the blade launch for a plane of nb blade markers,
// and the opt-in to that many.
int blade_table_words(int nb);
cudaError_t ibm_prepare_blades(int words);
// FP64 force and torque of markers [begin, n) (by list index) of the last
// forcing pass: out[0..2] = -beta * sum of spread sums, out[3] = torque about
// the tank axis (ci, ck), out[4] = number of markers summed. `partial` holds
// kLoadBlocks * 5 doubles.
constexpr int kLoadBlocks = 128;
// FP64 mass/momentum reduction: out[0] = sum rho, out[1..3] = sum (j + F/2).
// `partial` holds kReduceBlocks * 4 doubles.
constexpr int kReduceBlocks = 592;
cudaError_t launch_reduce_fp64(const IbmArgs& a, const uint32_t* mask, double* partial, double* out, cudaStream_t st);
// Rest state at density rho for the 16-bit storage.
cudaError_t launch_fill_rest(Planes Q, long long plane, float rho, float rho0, int storage, const CollideParams& p,
                             cudaStream_t st);
cudaError_t launch_marker_load(const IbmArgs& a, int begin, double ci, double ck, double* partial, double* out,
                               cudaStream_t st);
// Recompute n rotating markers (offsets xz[2n]) for cos/sin (ca, sa).
cudaError_t launch_rotate_markers(const double* xz, Marker* out, int n, double ca, double sa, double omega, double ci,
                                  double ck, int nx, int nz, cudaStream_t st);

}  // namespace tdlb
