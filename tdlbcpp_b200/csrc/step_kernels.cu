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
#include "tdlb_kernels.cuh"

namespace tdlb {

__device__ __forceinline__ bool mask_bit(const uint32_t* __restrict__ mask, const Dims& g, long long row, int k) {
    return (__ldg(mask + row * g.kw + (k >> 5)) >> (k & 31)) & 1u;
}

// ---------------------------------------------------------------------------
// Simple (A/B), one cell per thread.
// ---------------------------------------------------------------------------
template <bool LES, bool FROM_MOMENTS, bool COLLIDE>
__global__ void __launch_bounds__(256) k_step_simple(Planes A, Planes B, float* __restrict__ Nu,
                                                     const float* __restrict__ Fx, const float* __restrict__ Fy,
                                                     const float* __restrict__ Fz, const uint32_t* __restrict__ mask,
                                                     Dims g, CollideParams p) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = g.rows() * g.nz;
    if (t >= total) return;
    const int k = (int)(t % g.nz);
    const long long row = t / g.nz;
    const int j = (int)(row % g.ny);
    const int i = (int)(row / g.ny);
    const long long e = row * g.kp + k;

    float q[NQ];
#pragma unroll
    for (int d = 0; d < NQ; d++) {
        if (FROM_MOMENTS) {
            q[d] = __ldg(A.p[d] + e);
        } else {
            const int si = i - cx_of(d), sj = j - cy_of(d), sk = k - cz_of(d);
            const bool in = (unsigned)si < (unsigned)g.nx && (unsigned)sj < (unsigned)g.ny && (unsigned)sk < (unsigned)g.nz;
            const long long src = in ? ((long long)si * g.ny + sj) * g.kp + sk : e;
            q[d] = __ldg(A.p[d] + src);
        }
    }
    if (COLLIDE) {
        float m[NQ];
        if (FROM_MOMENTS) {
#pragma unroll
            for (int d = 0; d < NQ; d++) m[d] = q[d];
        } else {
            moments_of(q, m);
        }
        float fx = 0.f, fy = 0.f, fz = 0.f;
        if (mask_bit(mask, g, row, k)) {
            fx = __ldg(Fx + e); fy = __ldg(Fy + e); fz = __ldg(Fz + e);
        }
        float nu = LES ? Nu[e] : 0.f;
        collide<LES>(m, fx, fy, fz, nu, p, q);
        if (LES) Nu[e] = nu;
    }
#pragma unroll
    for (int d = 0; d < NQ; d++) B.p[d][e] = q[d];
}

// ---------------------------------------------------------------------------
// Esotwist (single buffer, in place), one cell per thread.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int wrap_up(int a, int n) { return a + 1 == n ? 0 : a + 1; }

template <bool LES, bool FROM_MOMENTS, bool COLLIDE, bool EVEN>
__global__ void __launch_bounds__(256) k_step_esotwist(Planes Q, float* __restrict__ Nu,
                                                       const float* __restrict__ Fx, const float* __restrict__ Fy,
                                                       const float* __restrict__ Fz, const uint32_t* __restrict__ mask,
                                                       Dims g, CollideParams p) {
    constexpr bool even = EVEN;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = g.rows() * g.nz;
    if (t >= total) return;
    const int k = (int)(t % g.nz);
    const long long row = t / g.nz;
    const int j = (int)(row % g.ny);
    const int i = (int)(row / g.ny);
    const int i1 = wrap_up(i, g.nx), j1 = wrap_up(j, g.ny), k1 = wrap_up(k, g.nz);
    const long long e = row * g.kp + k;

    // location of slot s for this cell: x + o_s
    long long loc[NQ];
#pragma unroll
    for (int s = 0; s < NQ; s++) {
        const int sg = even ? -1 : 1;
        const bool oi = sg * cx_of(s) > 0, oj = sg * cy_of(s) > 0, ok = sg * cz_of(s) > 0;
        loc[s] = ((long long)(oi ? i1 : i) * g.ny + (oj ? j1 : j)) * g.kp + (ok ? k1 : k);
    }
    float q[NQ];
#pragma unroll
    for (int d = 0; d < NQ; d++) {
        const int s = even ? d : (d ^ 1);
        q[d] = Q.p[s][loc[s]];
    }
    if (COLLIDE) {
        float m[NQ];
        if (FROM_MOMENTS) {
#pragma unroll
            for (int d = 0; d < NQ; d++) m[d] = q[d];
        } else {
            moments_of(q, m);
        }
        float fx = 0.f, fy = 0.f, fz = 0.f;
        if (mask_bit(mask, g, row, k)) {
            fx = __ldg(Fx + e); fy = __ldg(Fy + e); fz = __ldg(Fz + e);
        }
        float nu = LES ? Nu[e] : 0.f;
        collide<LES>(m, fx, fy, fz, nu, p, q);
        if (LES) Nu[e] = nu;
    }
#pragma unroll
    for (int d = 0; d < NQ; d++) {
        const int s = even ? (d ^ 1) : d;
        Q.p[s][loc[s]] = q[d];
    }
}

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

// Moments of the current state at every interior cell (what the reference's
// Q holds after moments()), written to 18 output planes of the same layout.
// mode: 0 = Simple populations in A (pull), 1 = moments in A (own cell),
//       2 = Esotwist populations (read map, parity `even`),
//       3 = Esotwist moments (read map, parity `even`).
__global__ void __launch_bounds__(256) k_state_moments(Planes A, Planes M, Dims g, int mode, int even) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = g.rows() * g.nz;
    if (t >= total) return;
    const int k = (int)(t % g.nz);
    const long long row = t / g.nz;
    const int j = (int)(row % g.ny);
    const int i = (int)(row / g.ny);
    const long long e = row * g.kp + k;
    float q[NQ], m[NQ];
    if (mode <= 1) {
#pragma unroll
        for (int d = 0; d < NQ; d++) {
            long long src = e;
            if (mode == 0) {
                const int si = i - cx_of(d), sj = j - cy_of(d), sk = k - cz_of(d);
                const bool in = (unsigned)si < (unsigned)g.nx && (unsigned)sj < (unsigned)g.ny && (unsigned)sk < (unsigned)g.nz;
                if (in) src = ((long long)si * g.ny + sj) * g.kp + sk;
            }
            q[d] = A.p[d][src];
        }
    } else {
        const int i1 = wrap_up(i, g.nx), j1 = wrap_up(j, g.ny), k1 = wrap_up(k, g.nz);
#pragma unroll
        for (int d = 0; d < NQ; d++) {
            const int s = even ? d : (d ^ 1);
            const int sg = even ? -1 : 1;
            const bool oi = sg * cx_of(s) > 0, oj = sg * cy_of(s) > 0, ok = sg * cz_of(s) > 0;
            q[d] = A.p[s][((long long)(oi ? i1 : i) * g.ny + (oj ? j1 : j)) * g.kp + (ok ? k1 : k)];
        }
    }
    if (mode == 0 || mode == 2) moments_of(q, m);
    else {
#pragma unroll
        for (int d = 0; d < NQ; d++) m[d] = q[d];
    }
#pragma unroll
    for (int d = 0; d < NQ; d++) M.p[d][e] = m[d];
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
static inline unsigned blocks_for(long long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

cudaError_t launch_step_simple(const StepArgs& a, cudaStream_t st) {
    const long long n = a.g.rows() * a.g.nz;
    const dim3 grid(blocks_for(n, 256)), block(256);
#define TDLB_SIMPLE(LES, FM, COL) k_step_simple<LES, FM, COL><<<grid, block, 0, st>>>(a.A, a.B, a.Nu, a.Fx, a.Fy, a.Fz, a.mask, a.g, a.p)
    if (!a.collide) TDLB_SIMPLE(false, false, false);
    else if (a.les) { if (a.from_moments) TDLB_SIMPLE(true, true, true); else TDLB_SIMPLE(true, false, true); }
    else { if (a.from_moments) TDLB_SIMPLE(false, true, true); else TDLB_SIMPLE(false, false, true); }
#undef TDLB_SIMPLE
    return cudaGetLastError();
}

cudaError_t launch_step_esotwist(const StepArgs& a, cudaStream_t st) {
    const long long n = a.g.rows() * a.g.nz;
    const dim3 grid(blocks_for(n, 256)), block(256);
#define TDLB_ESO(LES, FM, COL)                                                                                   \
    do {                                                                                                         \
        if (a.even) k_step_esotwist<LES, FM, COL, true><<<grid, block, 0, st>>>(a.A, a.Nu, a.Fx, a.Fy, a.Fz, a.mask, a.g, a.p); \
        else k_step_esotwist<LES, FM, COL, false><<<grid, block, 0, st>>>(a.A, a.Nu, a.Fx, a.Fy, a.Fz, a.mask, a.g, a.p); \
    } while (0)
    if (!a.collide) TDLB_ESO(false, false, false);
    else if (a.les) { if (a.from_moments) TDLB_ESO(true, true, true); else TDLB_ESO(true, false, true); }
    else { if (a.from_moments) TDLB_ESO(false, true, true); else TDLB_ESO(false, false, true); }
#undef TDLB_ESO
    return cudaGetLastError();
}

cudaError_t launch_fill_uniform_moments(Planes Q, const Dims& g, float rho, cudaStream_t st) {
    k_fill_uniform_moments<<<blocks_for(g.plane, 256), 256, 0, st>>>(Q, g, rho);
    return cudaGetLastError();
}

cudaError_t launch_state_moments(Planes A, Planes M, const Dims& g, int mode, int even, cudaStream_t st) {
    k_state_moments<<<blocks_for(g.rows() * g.nz, 256), 256, 0, st>>>(A, M, g, mode, even);
    return cudaGetLastError();
}

}  // namespace tdlb
