// Immersed-boundary forcing (Rushton-turbine markers) for sm_100a.
//
// Reference semantics (tdlbcpp/src/Forcing.hpp:56-176): markers are applied
// one after another in list order. Each marker
//   1. weights its 3x3 stencil in the i-k plane with the 3-point smoothed
//      delta (calcWeight, :18-35), indices wrapping periodically in i and k;
//   2. interpolates rho and (j + F/2) with the CURRENT F, i.e. including the
//      updates of earlier markers that share a cell (:91-121);
//   3. subtracts rho_sum * (uDelta, vDelta, wDelta) (:126-128);
//   4. spreads F = alpha*F - beta*w*sum into its 9 cells (:131-155).
// Cells no marker touched end with F = 0 (:162-174).
//
// Parallel form with the same result: a marker only interacts with markers
// of the same j-plane that share a stencil cell. The host scheduler assigns
// each marker a level = 1 + the highest level of an earlier marker sharing a
// cell, so markers of one level touch disjoint cells and every pair that
// shares a cell keeps its list order. One CTA per j-plane walks its levels
// with a barrier between them.
//
// "F = 0 where untouched" needs no full-grid sweep: the touched cells of each
// pass are recorded as one bit per cell (mask_new). The step kernel reads F
// only where the bit is set, and the next pass treats F as zero where neither
// the previous pass (mask_old) nor the current one has touched the cell.
//
// Two launches: k_ibm_gather (all markers in parallel: weights and the
// moments of the 9 stencil cells, which no marker changes) and k_ibm_spread
// (per plane, per level: the order-dependent F updates).
#include "tdlb_kernels.cuh"
#include "tdlb_rotate.hpp"

namespace tdlb {

// 3-point smoothed delta (Forcing.hpp:18-35).
__device__ __forceinline__ float calc_weight(float x) {
    x = fabsf(x);
    float w = 0.f;
    if (x <= 1.5f) {
        if (x <= 0.5f) w = (1.f / 3.f) * (1.f + sqrtf(fmaf(-3.f * x, x, 1.f)));
        else {
            const float y = 1.f - x;
            w = (1.f / 6.f) * (5.f - 3.f * x - sqrtf(fmaf(-3.f * y, y, 1.f)));
        }
    }
    return w;
}

__device__ __forceinline__ int wrap_i(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }

// rho and momentum of the state at interior cell (i, j, k).
__device__ __forceinline__ void cell_moments4(const Planes& A, int mode, int even, const Dims& g, int i, int j, int k,
                                              float* m4) {
    if (mode == 1) {
        const long long e = ((long long)i * g.ny + j) * g.kp + k;
#pragma unroll
        for (int s = 0; s < 4; s++) m4[s] = A.p[s][e];
        return;
    }
    float q[NQ];
    if (mode == 0) {
#pragma unroll
        for (int d = 0; d < NQ; d++) {
            const int si = i - cx_of(d), sj = j - cy_of(d), sk = k - cz_of(d);
            const bool in = (unsigned)si < (unsigned)g.nx && (unsigned)sj < (unsigned)g.ny && (unsigned)sk < (unsigned)g.nz;
            const long long src = in ? ((long long)si * g.ny + sj) * g.kp + sk : ((long long)i * g.ny + j) * g.kp + k;
            q[d] = A.p[d][src];
        }
        moments4_of(q, m4);
        return;
    }
    const int i1 = i + 1 == g.nx ? 0 : i + 1, j1 = j + 1 == g.ny ? 0 : j + 1, k1 = k + 1 == g.nz ? 0 : k + 1;
    const int nread = mode == 3 ? 4 : NQ;
#pragma unroll
    for (int d = 0; d < NQ; d++) {
        if (d >= nread) break;
        const int s = even ? d : (d ^ 1);
        const int sg = even ? -1 : 1;
        const bool oi = sg * cx_of(s) > 0, oj = sg * cy_of(s) > 0, ok = sg * cz_of(s) > 0;
        q[d] = A.p[s][((long long)(oi ? i1 : i) * g.ny + (oj ? j1 : j)) * g.kp + (ok ? k1 : k)];
    }
    if (mode == 3) {
#pragma unroll
        for (int s = 0; s < 4; s++) m4[s] = q[s];
    } else {
        moments4_of(q, m4);
    }
}

__global__ void __launch_bounds__(128) k_ibm_gather(IbmArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    const Marker mk = a.markers[a.sched[p]];
    const int i = (int)mk.i, j = (int)mk.j, k = (int)mk.k;
    float* s = a.scratch;
    const long long cap = a.cap;
    int c = 0;
    for (int k1 = -1; k1 <= 1; k1++) {
        for (int i1 = -1; i1 <= 1; i1++, c++) {
            const float w = calc_weight(-mk.iCartFraction + (float)i1) * calc_weight(-mk.kCartFraction + (float)k1);
            const int i2 = wrap_i(i + i1, a.g.nx), k2 = wrap_i(k + k1, a.g.nz);
            float m4[4];
            cell_moments4(a.A, a.state_mode, a.even, a.g, i2, j, k2, m4);
            s[(SF_W + c) * cap + p] = w;
            s[(SF_RHO + c) * cap + p] = m4[0];
            s[(SF_MX + c) * cap + p] = m4[1];
            s[(SF_MY + c) * cap + p] = m4[2];
            s[(SF_MZ + c) * cap + p] = m4[3];
            s[(SF_CELL + c) * cap + p] = __int_as_float((i2 << 16) | k2);
        }
    }
    s[SF_U * cap + p] = mk.uDelta;
    s[SF_V * cap + p] = mk.vDelta;
    s[SF_WV * cap + p] = mk.wDelta;
}

__global__ void __launch_bounds__(256) k_ibm_spread(IbmArgs a) {
    extern __shared__ uint32_t touched[];   // this plane's mask words, [nx][kw]
    const int j = blockIdx.x;
    const Dims g = a.g;
    const int nwords = g.nx * g.kw;
    for (int w = threadIdx.x; w < nwords; w += blockDim.x) touched[w] = 0u;
    __syncthreads();

    const float* s = a.scratch;
    const long long cap = a.cap;
    const int lv0 = a.plane_lv[j], lv1 = a.plane_lv[j + 1];
    for (int lv = lv0; lv < lv1; lv++) {
        const int p0 = a.level_ptr[lv], p1 = a.level_ptr[lv + 1];
        for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
            float w[9];
            long long e[9];
            int sw[9];
            uint32_t bit[9];
            float rhoSum = 0.f, xSum = 0.f, ySum = 0.f, zSum = 0.f;
#pragma unroll
            for (int c = 0; c < 9; c++) {
                w[c] = s[(SF_W + c) * cap + p];
                const int packed = __float_as_int(s[(SF_CELL + c) * cap + p]);
                const int i2 = packed >> 16, k2 = packed & 0xffff;
                const long long row = (long long)i2 * g.ny + j;
                e[c] = row * g.kp + k2;
                sw[c] = i2 * g.kw + (k2 >> 5);
                bit[c] = 1u << (k2 & 31);
                const bool live = (touched[sw[c]] & bit[c]) || (a.mask_old[row * g.kw + (k2 >> 5)] & bit[c]);
                const float fx = live ? a.Fx[e[c]] : 0.f;
                const float fy = live ? a.Fy[e[c]] : 0.f;
                const float fz = live ? a.Fz[e[c]] : 0.f;
                rhoSum = fmaf(w[c], s[(SF_RHO + c) * cap + p], rhoSum);
                xSum = fmaf(w[c], fmaf(0.5f, fx, s[(SF_MX + c) * cap + p]), xSum);
                ySum = fmaf(w[c], fmaf(0.5f, fy, s[(SF_MY + c) * cap + p]), ySum);
                zSum = fmaf(w[c], fmaf(0.5f, fz, s[(SF_MZ + c) * cap + p]), zSum);
            }
            xSum = fmaf(-rhoSum, s[SF_U * cap + p], xSum);
            ySum = fmaf(-rhoSum, s[SF_V * cap + p], ySum);
            zSum = fmaf(-rhoSum, s[SF_WV * cap + p], zSum);
#pragma unroll
            for (int c = 0; c < 9; c++) {
                // re-evaluated per cell: a stencil that wraps onto itself
                // (extent < 3) sees its own earlier update, as in the reference
                const long long row = e[c] / g.kp;
                const int k2 = (int)(e[c] - row * g.kp);
                const bool live = (touched[sw[c]] & bit[c]) || (a.mask_old[row * g.kw + (k2 >> 5)] & bit[c]);
                const float fx = live ? a.Fx[e[c]] : 0.f;
                const float fy = live ? a.Fy[e[c]] : 0.f;
                const float fz = live ? a.Fz[e[c]] : 0.f;
                const float bw = a.beta * w[c];
                a.Fx[e[c]] = fmaf(a.alpha, fx, -bw * xSum);
                a.Fy[e[c]] = fmaf(a.alpha, fy, -bw * ySum);
                a.Fz[e[c]] = fmaf(a.alpha, fz, -bw * zSum);
                atomicOr(&touched[sw[c]], bit[c]);
            }
        }
        __syncthreads();
    }
    // publish this plane's touched flags (planes without markers publish zeros)
    for (int w = threadIdx.x; w < nwords; w += blockDim.x) {
        const int i = w / g.kw, wk = w - i * g.kw;
        a.mask_new[((long long)i * g.ny + j) * g.kw + wk] = touched[w];
    }
}

// Impeller rotation on the device: recomputes the blade markers of the
// resident list for a new angle (main.cpp:409-426 does this on the host and
// re-uploads the whole list every step).
__global__ void k_rotate_markers(const double* __restrict__ xz, Marker* __restrict__ out, int n, double ca, double sa,
                                 double omega, double ci, double ck, int nx, int nz) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const RotatedMarker r = rotate_marker(xz[2 * q], xz[2 * q + 1], ca, sa, omega, ci, ck, nx, nz);
    Marker& m = out[q];
    m.i = r.i;
    m.k = r.k;
    m.iCartFraction = r.iCartFraction;
    m.kCartFraction = r.kCartFraction;
    m.uDelta = r.uDelta;
    m.vDelta = 0.f;
    m.wDelta = r.wDelta;
}

cudaError_t launch_rotate_markers(const double* xz, Marker* out, int n, double ca, double sa, double omega, double ci,
                                  double ck, int nx, int nz, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_rotate_markers<<<(n + 255) / 256, 256, 0, st>>>(xz, out, n, ca, sa, omega, ci, ck, nx, nz);
    return cudaGetLastError();
}

size_t ibm_smem_bytes(const Dims& g) { return (size_t)g.nx * g.kw * sizeof(uint32_t); }

cudaError_t ibm_prepare_smem(size_t bytes) {
    return cudaFuncSetAttribute(k_ibm_spread, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

cudaError_t launch_ibm(const IbmArgs& a, cudaStream_t st) {
    if (a.n > 0) {
        k_ibm_gather<<<(a.n + 127) / 128, 128, 0, st>>>(a);
        cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess) return err;
    }
    const size_t smem = ibm_smem_bytes(a.g);
    k_ibm_spread<<<a.g.ny, 256, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace tdlb
