// Resolution doubling on the device (ComputeUnitBase::doubleResolutionFullCU,
// ComputeUnit.hpp:258-316, with indexPreviousResolution :480-502 and
// copyFieldsWithScaling :229-254).
//
// The reference doubles x, y and z, reallocates, zeroes every field and
// copies Q and Nu from the old lattice with the index map
// from = n/2 + n%2 in ghosted coordinates -- for interior cells, new cell n
// (0-based) takes old cell n/2: every old cell fills a 2x2x2 block. It runs
// at the top of a main-loop step, when Q holds moments, so the copy is of
// moments; F, the touched flags and the excluded points start at zero, and
// the caller regenerates the geometry for the new size (main.cpp:349-397).
// (The reference's copy loop runs l < 19 over 18-entry records; only the 18
// moments are meaningful and only they are copied here.)
//
// Here one kernel computes each new cell's parent moments from the current
// state and writes them as the state of the new lattice: at the cell for
// Simple, in the writeMoments places of the current parity for Esotwist. The
// state then holds moments, as after initialise. FP32 storage only.
#include "tdlb_handle.hpp"
#include "step_kernels.cuh"

#include <string>

namespace tdlb {

__global__ void __launch_bounds__(256) k_double_resolution(Planes A, Dims g, int mode, int even, CollideParams p,
                                                           const float* __restrict__ nu_old, Planes N, Dims h,
                                                           float* __restrict__ nu_new, int esotwist) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= h.rows() * h.nz) return;
    const int k = (int)(t % h.nz);
    const long long row = t / h.nz;
    const int j = (int)(row % h.ny);
    const int i = (int)(row / h.ny);
    const int pi = i >> 1, pj = j >> 1, pk = k >> 1;
    float m[NQ];
    state_moments18<float>(A, g, mode, even, p, pi, pj, pk, m);
    nu_new[row * h.kp + k] = nu_old[((long long)pi * g.ny + pj) * g.kp + pk];
    if (!esotwist) {
#pragma unroll
        for (int d = 0; d < NQ; d++) N.p[d][row * h.kp + k] = m[d];
        return;
    }
    const int i1 = i + 1 == h.nx ? 0 : i + 1, j1 = j + 1 == h.ny ? 0 : j + 1, k1 = k + 1 == h.nz ? 0 : k + 1;
#pragma unroll
    for (int d = 0; d < NQ; d++) {
        const long long li = cx_of(d) < 0 ? i1 : i, lj = cy_of(d) < 0 ? j1 : j, lk = cz_of(d) < 0 ? k1 : k;
        N.p[even ? d : (d ^ 1)][(li * h.ny + lj) * h.kp + lk] = m[d];
    }
}

}  // namespace tdlb

namespace {

struct RFail {
    int code;
    std::string msg;
};

#define TDLB_RCK(call)                                                                                      \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess) throw RFail{TDLB_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

long long round_up_ll(long long a, long long m) { return (a + m - 1) / m * m; }

// Frees a device pointer and clears it.
template <typename T>
void drop(T*& p) {
    cudaFree(p);
    p = nullptr;
}

}  // namespace

extern "C" {

int tdlb_double_resolution(tdlb_handle h) {
    if (!h) return TDLB_EINVAL;
    float* A = nullptr;
    float* B = nullptr;
    float* Nu = nullptr;
    float* F = nullptr;
    uint32_t* mask = nullptr;
    try {
        cudaSetDevice(h->device);
        TDLB_RCK(tdlb_rt::join_side(h));
        TDLB_RCK(cudaStreamSynchronize(h->stream));   // the old buffers are freed below
        if (!h->initialised) throw RFail{TDLB_ESTATE, "not initialised (tdlb_initialise)"};
        if (h->own_stream) throw RFail{TDLB_ESTATE, "a tank of a batch cannot change size"};
        if (h->cfg.storage != TDLB_STORAGE_FP32) throw RFail{TDLB_EINVAL, "resolution doubling needs FP32 storage"};
        const Dims g = h->g;
        if ((long long)g.nx * 2 > 32767 || (long long)g.ny * 2 > 32767 || (long long)g.nz * 2 > 32767)
            throw RFail{TDLB_EINVAL, "doubled grid extent above 32767"};
        const Dims n = tdlb::make_dims(g.nx * 2, g.ny * 2, g.nz * 2);
        if ((long long)n.nx * n.ny * n.kp >= (1LL << 31) - 64)
            throw RFail{TDLB_EINVAL, "doubled lattice too large: one plane must stay below 2^31 elements"};
        const long long words = round_up_ll((long long)n.nx * n.ny * n.kw, 64);
        const bool simple = h->cfg.streaming == TDLB_STREAMING_SIMPLE;
        const size_t pop = (size_t)tdlb::NQ * n.plane * sizeof(float);
        size_t free_b = 0, total_b = 0;
        TDLB_RCK(cudaMemGetInfo(&free_b, &total_b));
        const size_t need = pop * (simple ? 2 : 1) + (size_t)5 * n.plane * sizeof(float) + 2 * words * sizeof(uint32_t);
        if (need > free_b)
            throw RFail{TDLB_ENOMEM, "doubled lattice needs " + std::to_string(need) + " B, " + std::to_string(free_b) +
                                         " B free"};
        TDLB_RCK(cudaMalloc(&A, pop));
        if (simple) TDLB_RCK(cudaMalloc(&B, pop));
        TDLB_RCK(cudaMalloc(&Nu, (size_t)n.plane * sizeof(float)));
        TDLB_RCK(cudaMalloc(&F, (size_t)4 * n.plane * sizeof(float)));   // one float4 per element
        TDLB_RCK(cudaMalloc(&mask, (size_t)2 * words * sizeof(uint32_t)));
        TDLB_RCK(cudaMemsetAsync(A, 0, pop, h->stream));
        if (B) TDLB_RCK(cudaMemsetAsync(B, 0, pop, h->stream));
        TDLB_RCK(cudaMemsetAsync(Nu, 0, (size_t)n.plane * sizeof(float), h->stream));
        TDLB_RCK(cudaMemsetAsync(F, 0, (size_t)4 * n.plane * sizeof(float), h->stream));
        TDLB_RCK(cudaMemsetAsync(mask, 0, (size_t)2 * words * sizeof(uint32_t), h->stream));
        Planes dst;
        for (int d = 0; d < tdlb::NQ; d++) dst.p[d] = A + (size_t)d * n.plane;
        const long long cells = n.rows() * n.nz;
        tdlb::k_double_resolution<<<(unsigned)((cells + 255) / 256), 256, 0, h->stream>>>(
            h->planes(h->state_buf()), g, h->state_mode(), h->even ? 1 : 0, h->cp, h->Nu, dst, n, Nu, simple ? 0 : 1);
        TDLB_RCK(cudaGetLastError());
        TDLB_RCK(cudaStreamSynchronize(h->stream));
    } catch (const RFail& f) {
        cudaFree(A); cudaFree(B); cudaFree(Nu); cudaFree(F); cudaFree(mask);
        h->err = f.msg;
        return f.code;
    }
    // swap in the new lattice; the geometry is regenerated by the caller
    cudaFree(h->bufA); cudaFree(h->bufB); cudaFree(h->Nu); cudaFree(h->F); cudaFree(h->mask);
    h->bufA = A;
    h->bufB = B;
    h->Nu = Nu;
    h->F = F;
    h->mask = mask;
    Dims& g = h->g;
    g = tdlb::make_dims(g.nx * 2, g.ny * 2, g.nz * 2);
    h->mask_words = round_up_ll((long long)g.nx * g.ny * g.kw, 64);
    h->cfg.x *= 2;
    h->cfg.y *= 2;
    h->cfg.z *= 2;
    h->cur = 0;
    h->pass = 0;
    h->holds_moments = true;
    // markers, schedules and every per-plane or per-cell buffer belong to the old size
    h->markers_set = false;
    h->rot_device = false;
    h->impeller_begin = -1;
    h->n_markers = 0;
    h->n0 = 0;
    h->h_markers.clear();
    h->cells = tdlb::CellList{};
    drop(h->d_plane_lv0);
    drop(h->d_plane_lv1);
    drop(h->d_plane_cell);
    drop(h->d_plane_list);
    drop(h->d_cell_order);
    h->ncell_big = 0;
    drop(h->d_mask_static);
    drop(h->d_exclude);
    h->h_exclude.clear();
    h->h_plane_list.clear();
    drop(h->d_rot_xz);
    h->marker_gen++;
    h->resident = false;
    h->inner_queued = false;
    h->h_rot_xz.clear();
    return TDLB_OK;
}

}  // extern "C"
