// Fused lattice Boltzmann step kernels for sm_100a.
//
// One launch performs the reference's collision() + bounceBackBoundary() +
// streamingPush() + moments() sequence (main.cpp:438-451) for every interior
// cell: gather the 18 streamed populations, form the moments, apply the
// Eggels-Somers/LES collision with the immersed-boundary force, and store the
// 18 post-collision populations. Two streaming schemes:
//
//  * Simple (A/B buffers, pull). The reference's in-place push
//    (StreamingSimple.hpp:77-126) moves f*_d(y) to y + c_d for interior y and
//    its ghost-face writes (Boundary.hpp) are never read back, so the streamed
//    value at interior x is f*_d(x - c_d) when x - c_d is interior, and the
//    cell's OWN post-collision f*_d(x) otherwise (no reversal).
//  * Esotwist (one buffer, in place). For parity p, slot s of cell x lives at
//    cell x + o_s with o_s = max(-c_s, 0) (even) or max(+c_s, 0) (odd), +1
//    wrapping to 0 (StreamingEsoteric.hpp:28-130). Even steps read f_d from
//    slot d and write f*_d to slot opp(d); odd steps read slot opp(d) and
//    write slot d. Each cell reads and writes the same 18 locations, so
//    cells are independent.
//
// FROM_MOMENTS instantiations read the state as moments instead of
// populations: the state after initialise() (ComputeUnit.hpp:175-190) or a
// checkpoint load holds moments, exactly as the reference's Q does between
// moments() and collision().
#include "step_kernels.cuh"

namespace tdlb {


__device__ __forceinline__ int wrap_up(int a, int n) { return a + 1 == n ? 0 : a + 1; }

// ---------------------------------------------------------------------------
// Moment-form state after initialise(rho): slot 0 = rho, others 0 at every
// cell (QVec.hpp:406-411). For Esotwist with evenStep = true the reference's
// read map returns slot 0 of the cell itself, so the same fill serves both.
// ---------------------------------------------------------------------------
__global__ void k_fill_uniform_moments(Planes Q, Dims g, float rho) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = g.plane;
    if (t >= n) return;
    Q.p[0][t] = rho;
#pragma unroll
    for (int d = 1; d < NQ; d++) Q.p[d][t] = 0.f;
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
static inline unsigned blocks_for(long long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// Grid of a launch: every quad (part 0) or one warp per listed chunk (1, 2).
static inline unsigned step_blocks(const StepArgs& a, int V) {
    if (a.part != 0) return blocks_for((long long)a.zone.count * 32, 128);
    return blocks_for(a.g.rows() * (a.g.kp / V), 128);
}

template <int V>
static cudaError_t launch_simple_v(const StepArgs& a, cudaStream_t st) {
    const dim3 grid(step_blocks(a, V)), block(128);
#define TDLB_SIMPLE(LES, FM, COL, PART)                                                                       \
    k_step_simple<float, V, LES, FM, COL, PART><<<grid, block, 0, st>>>(                                   \
        a.A, a.B, a.Nu, a.F, a.mask, a.g, a.p,                                                               \
        launch_walk<k_step_simple<float, V, LES, FM, COL, PART>, COL && !FM>(a), ResidualBox{}, BoxOut{})
    if (!a.collide) TDLB_SIMPLE(false, false, false, 0);
    else if (a.from_moments) { if (a.les) TDLB_SIMPLE(true, true, true, 0); else TDLB_SIMPLE(false, true, true, 0); }
    else if constexpr (V == 1) {
        if (a.les) {
            if (a.part == 1) TDLB_SIMPLE(true, false, true, 1);
            else if (a.part == 2) TDLB_SIMPLE(true, false, true, 2);
            else TDLB_SIMPLE(true, false, true, 0);
        } else {
            if (a.part == 1) TDLB_SIMPLE(false, false, true, 1);
            else if (a.part == 2) TDLB_SIMPLE(false, false, true, 2);
            else TDLB_SIMPLE(false, false, true, 0);
        }
    } else {
        if (a.les) TDLB_SIMPLE(true, false, true, 0); else TDLB_SIMPLE(false, false, true, 0);
    }
#undef TDLB_SIMPLE
    return cudaGetLastError();
}

template <int V, bool LES, bool FM, bool COL, int PART>
static void eso_launch(const StepArgs& a, dim3 grid, cudaStream_t st) {
    if (a.even)
        k_step_esotwist<float, V, LES, FM, COL, true, PART><<<grid, 128, 0, st>>>(
            a.A, a.Nu, a.F, a.mask, a.g, a.p, launch_walk<k_step_esotwist<float, V, LES, FM, COL, true, PART>, COL && !FM>(a),
            ResidualBox{}, BoxOut{});
    else
        k_step_esotwist<float, V, LES, FM, COL, false, PART><<<grid, 128, 0, st>>>(
            a.A, a.Nu, a.F, a.mask, a.g, a.p, launch_walk<k_step_esotwist<float, V, LES, FM, COL, false, PART>, COL && !FM>(a),
            ResidualBox{}, BoxOut{});
}

template <int V>
static cudaError_t launch_esotwist_v(const StepArgs& a, cudaStream_t st) {
    const dim3 grid(step_blocks(a, V));
    if (!a.collide) eso_launch<V, false, false, false, 0>(a, grid, st);
    else if (a.from_moments) {
        if (a.les) eso_launch<V, true, true, true, 0>(a, grid, st); else eso_launch<V, false, true, true, 0>(a, grid, st);
    } else if constexpr (V == 1) {
        if (a.les) {
            if (a.part == 1) eso_launch<1, true, false, true, 1>(a, grid, st);
            else if (a.part == 2) eso_launch<1, true, false, true, 2>(a, grid, st);
            else eso_launch<1, true, false, true, 0>(a, grid, st);
        } else {
            if (a.part == 1) eso_launch<1, false, false, true, 1>(a, grid, st);
            else if (a.part == 2) eso_launch<1, false, false, true, 2>(a, grid, st);
            else eso_launch<1, false, false, true, 0>(a, grid, st);
        }
    } else {
        if (a.les) eso_launch<V, true, false, true, 0>(a, grid, st); else eso_launch<V, false, false, true, 0>(a, grid, st);
    }
    return cudaGetLastError();
}

cudaError_t launch_step_simple(const StepArgs& a, cudaStream_t st) {
    if (a.part != 0 && (a.vec != 1 || a.from_moments || !a.collide)) return cudaErrorInvalidValue;
    if (a.storage != STORE_F32) return launch_step_simple_h16(a, st);
    if (a.box != 0) return cudaErrorInvalidValue;   // no residual box for FP32 storage
    switch (a.vec) {
        case 1: return launch_simple_v<1>(a, st);
        case 2: return launch_simple_v<2>(a, st);
        default: return launch_simple_v<4>(a, st);
    }
}

cudaError_t launch_step_esotwist(const StepArgs& a, cudaStream_t st) {
    if (a.part != 0 && (a.vec != 1 || a.from_moments || !a.collide)) return cudaErrorInvalidValue;
    if (a.storage != STORE_F32) return launch_step_esotwist_h16(a, st);
    if (a.box != 0) return cudaErrorInvalidValue;   // no residual box for FP32 storage
    switch (a.vec) {
        case 1: return launch_esotwist_v<1>(a, st);
        case 2: return launch_esotwist_v<2>(a, st);
        default: return launch_esotwist_v<4>(a, st);
    }
}

cudaError_t launch_fill_uniform_moments(Planes Q, const Dims& g, float rho, cudaStream_t st) {
    k_fill_uniform_moments<<<blocks_for(g.plane, 256), 256, 0, st>>>(Q, g, rho);
    return cudaGetLastError();
}

cudaError_t launch_state_moments(Planes A, Planes M, const Dims& g, int mode, int even, cudaStream_t st, int storage,
                                 const CollideParams& p, const ResidualBox& rb) {
    const unsigned blocks = blocks_for(g.rows() * g.nz, 256);
    with_storage(storage, [&](auto s) {
        k_state_moments<decltype(s)><<<blocks, 256, 0, st>>>(A, M, g, mode, even, p, rb);
    });
    return cudaGetLastError();
}

}  // namespace tdlb
