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
// Per pass (launch_ibm): k_ibm_cells (moments and starting F of every unique
// stencil cell of the static markers; it also starts mask_new as the static
// touched flags), k_ibm_gather_tail (weights and stencil moments of every
// blade marker, which no marker changes), k_ibm_spread_bulk (one plane per
// group of threads: the static markers' levels on an F tile in shared
// memory), then k_ibm_blades (the blade levels of the planes that have
// blades, on a shared-memory hash table of the plane's blade cells). The
// batched passes run the same steps per lattice, with the blade levels
// inside their spread.
#include "tdlb_kernels.cuh"
#include "tdlb_rotate.hpp"

#include <algorithm>
#include <map>
#include <mutex>
#include <utility>

namespace tdlb {

// 3-point smoothed delta (Forcing.hpp:18-35). The reference evaluates it
// in double (its literals promote the float argument) and rounds the result
// to float; every operation here is an explicitly rounded double operation
// in the reference's order, so no kernel can contract it differently and
// the weights equal the reference's bit for bit.
__device__ __forceinline__ float calc_weight(float xf) {
    const double x = (double)fabsf(xf);
    if (x > 1.5) return 0.f;
    double w;
    if (x <= 0.5) {
        const double r = __dsqrt_rn(__dadd_rn(__dmul_rn(__dmul_rn(-3.0, x), x), 1.0));
        w = __dmul_rn(1.0 / 3.0, __dadd_rn(1.0, r));
    } else {
        const double y = __dsub_rn(1.0, x);
        const double r = __dsqrt_rn(__dadd_rn(__dmul_rn(-3.0, __dmul_rn(y, y)), 1.0));
        w = __dmul_rn(1.0 / 6.0, __dsub_rn(__dsub_rn(5.0, __dmul_rn(3.0, x)), r));
    }
    return __double2float_rn(w);
}

// Weight of stencil offset (i1, k1) for a marker at fractions (icf, kcf):
// the product of the two 1-D weights, rounded to float (Forcing.hpp:37-48).
__device__ __forceinline__ float stencil_weight(float icf, float kcf, int i1, int k1) {
    return __fmul_rn(calc_weight(__fadd_rn(-icf, (float)i1)), calc_weight(__fadd_rn(-kcf, (float)k1)));
}

__device__ __forceinline__ int wrap_i(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }

template <typename S>
__device__ __forceinline__ float ld_state(const float* plane, long long e) {
    if constexpr (sizeof(S) == 4) return plane[e];
    else return Storage<S>::dec(reinterpret_cast<const S*>(plane)[e]);
}

// rho and momentum of the state at interior cell (i, j, k). With a residual
// box, a cell near it adds the residuals of its locations inside the box
// after its 18 loads (the other cells take no box code).
template <typename S>
__device__ __forceinline__ void cell_moments4(const Planes& A, int mode, int even, const Dims& g, int i, int j, int k,
                                              const CollideParams& p, float* m4, const ResidualBox& rb) {
    if (mode == 1) {
        const long long e = ((long long)i * g.ny + j) * g.kp + k;
#pragma unroll
        for (int s = 0; s < 4; s++) m4[s] = ld_state<S>(A.p[s], e);
        return;
    }
    float q[NQ];
    const bool near_box = Storage<S>::deviation && rb.near(i, j, k);
    if (mode == 0) {
#pragma unroll
        for (int d = 0; d < NQ; d++) {
            const int si = i - cx_of(d), sj = j - cy_of(d), sk = k - cz_of(d);
            const bool in = (unsigned)si < (unsigned)g.nx && (unsigned)sj < (unsigned)g.ny && (unsigned)sk < (unsigned)g.nz;
            const long long src = in ? ((long long)si * g.ny + sj) * g.kp + sk : ((long long)i * g.ny + j) * g.kp + k;
            q[d] = ld_state<S>(A.p[d], src) + (Storage<S>::deviation ? (is_face(d) ? p.wface : p.wedge) : 0.f);
        }
        if (near_box) {   // residual box: the exact deviations
#pragma unroll
            for (int d = 0; d < NQ; d++) {
                const int si = i - cx_of(d), sj = j - cy_of(d), sk = k - cz_of(d);
                const bool in = (unsigned)si < (unsigned)g.nx && (unsigned)sj < (unsigned)g.ny && (unsigned)sk < (unsigned)g.nz;
                const int li = in ? si : i, lj = in ? sj : j, lk = in ? sk : k;
                if (rb.contains(li, lj, lk)) q[d] += *rb.at(d, li, lj, lk);
            }
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
        q[d] = ld_state<S>(A.p[s], ((long long)(oi ? i1 : i) * g.ny + (oj ? j1 : j)) * g.kp + (ok ? k1 : k)) +
               (mode == 2 && Storage<S>::deviation ? (is_face(d) ? p.wface : p.wedge) : 0.f);
    }
    if (mode == 2 && near_box) {   // residual box: the exact deviations
#pragma unroll
        for (int d = 0; d < NQ; d++) {
            const int s = even ? d : (d ^ 1);
            const int sg = even ? -1 : 1;
            const bool oi = sg * cx_of(s) > 0, oj = sg * cy_of(s) > 0, ok = sg * cz_of(s) > 0;
            if (rb.contains(oi ? i1 : i, oj ? j1 : j, ok ? k1 : k)) q[d] += *rb.at(s, oi ? i1 : i, oj ? j1 : j, ok ? k1 : k);
        }
    }
    if (mode == 3) {
#pragma unroll
        for (int s = 0; s < 4; s++) m4[s] = q[s];
    } else {
        moments4_of(q, m4);
    }
}

// ---------------------------------------------------------------------------
// First segment (markers that do not move), prepared once per upload.
// ---------------------------------------------------------------------------
__global__ void k_ibm_prepare(IbmArgs a, float* __restrict__ prep) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n0) return;
    const Marker mk = a.markers[a.sched[p]];
    float* row = prep + (size_t)p * PF_STRIDE;
    int c = 0;
    for (int k1 = -1; k1 <= 1; k1++)
        for (int i1 = -1; i1 <= 1; i1++, c++)
            row[PF_W + c] = stencil_weight(mk.iCartFraction, mk.kCartFraction, i1, k1);
    row[PF_U] = mk.uDelta;
    row[PF_V] = mk.vDelta;
    row[PF_WV] = mk.wDelta;
}

// Per pass: rho and momentum of every unique stencil cell of the first
// segment (cells sorted by row, so neighbouring threads pull neighbouring
// cells), and the F each cell starts the pass with (zero unless the previous
// pass touched it, Forcing.hpp:162-174).
template <typename S>
__device__ __forceinline__ void ibm_cell(const IbmArgs& a, int c) {
    const Dims& g = a.g;
    const int e = a.cell_e[c];
    const int row = e / g.kp;
    const int k = e - row * g.kp;
    const int i = row / g.ny;
    const int j = row - i * g.ny;
    float m4[4];
    cell_moments4<S>(a.A, a.state_mode, a.even, g, i, j, k, a.p, m4, a.rbox);
    const long long C = a.ncell;
    reinterpret_cast<float4*>(a.cell_m)[c] = make_float4(m4[0], m4[1], m4[2], m4[3]);
    const bool live = (a.mask_old[(long long)row * g.kw + (k >> 5)] >> (k & 31)) & 1u;
    const float4 f = live ? a.F4[e] : make_float4(0.f, 0.f, 0.f, 0.f);
    a.cell_F[c] = f.x;
    a.cell_F[C + c] = f.y;
    a.cell_F[2 * C + c] = f.z;
}

// Cells [first, first + count) of a.cell_order (of the cell list itself
// when there is no order).
// copy_mask: the launch also starts mask_new as the first segment's touched
// flags (mask_static, a multiple of 16 bytes), so that the pass needs no
// separate copy.
template <typename S>
__global__ void __launch_bounds__(256) k_ibm_cells(IbmArgs a, int first, int count, int copy_mask) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (copy_mask) {
        const long long n4 = (long long)(a.mask_bytes / 16);
        for (long long w = t; w < n4; w += (long long)gridDim.x * blockDim.x)
            reinterpret_cast<uint4*>(a.mask_new)[w] = reinterpret_cast<const uint4*>(a.mask_static)[w];
    }
    if (t >= count) return;
    ibm_cell<S>(a, a.cell_order ? a.cell_order[first + t] : first + t);
}

// Second segment (the blades): weights and the moments of the 9 stencil
// cells of every blade marker.
template <typename S>
__device__ __forceinline__ void ibm_tail_marker(const IbmArgs& a, int t) {
    const Marker mk = a.markers[a.sched[a.n0 + t]];
    const int i = (int)mk.i, j = (int)mk.j, k = (int)mk.k;
    float* s = a.tail;
    const long long cap = a.tail_cap;
    int c = 0;
    for (int k1 = -1; k1 <= 1; k1++) {
        for (int i1 = -1; i1 <= 1; i1++, c++) {
            const float w = stencil_weight(mk.iCartFraction, mk.kCartFraction, i1, k1);
            const int i2 = wrap_i(i + i1, a.g.nx), k2 = wrap_i(k + k1, a.g.nz);
            float m4[4];
            cell_moments4<S>(a.A, a.state_mode, a.even, a.g, i2, j, k2, a.p, m4, a.rbox);
            s[(TF_W + c) * cap + t] = w;
            s[(TF_RHO + c) * cap + t] = m4[0];
            s[(TF_MX + c) * cap + t] = m4[1];
            s[(TF_MY + c) * cap + t] = m4[2];
            s[(TF_MZ + c) * cap + t] = m4[3];
            s[(TF_CELL + c) * cap + t] = __int_as_float((i2 << 16) | k2);
        }
    }
    s[TF_U * cap + t] = mk.uDelta;
    s[TF_V * cap + t] = mk.vDelta;
    s[TF_WV * cap + t] = mk.wDelta;
}

// One thread per (blade marker t, stencil cell c): thread u takes c = u /
// ntail, t = u % ntail (c = 3 (k1 + 1) + (i1 + 1), as ibm_tail_marker), so
// the 9 cells of a marker are gathered in parallel; c = 0 also writes the
// marker velocity.
template <typename S>
__global__ void __launch_bounds__(128) k_ibm_gather_tail(IbmArgs a) {
    const int ntail = a.n - a.n0;
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= 9 * ntail) return;
    const int c = u / ntail, t = u - c * ntail;
    const Marker mk = a.markers[a.sched[a.n0 + t]];
    const int k1 = c / 3 - 1, i1 = c - 3 * (c / 3) - 1;
    const int i2 = wrap_i((int)mk.i + i1, a.g.nx), j = (int)mk.j, k2 = wrap_i((int)mk.k + k1, a.g.nz);
    float m4[4];
    cell_moments4<S>(a.A, a.state_mode, a.even, a.g, i2, j, k2, a.p, m4, a.rbox);
    float* s = a.tail;
    const long long cap = a.tail_cap;
    s[(TF_W + c) * cap + t] = stencil_weight(mk.iCartFraction, mk.kCartFraction, i1, k1);
    s[(TF_RHO + c) * cap + t] = m4[0];
    s[(TF_MX + c) * cap + t] = m4[1];
    s[(TF_MY + c) * cap + t] = m4[2];
    s[(TF_MZ + c) * cap + t] = m4[3];
    s[(TF_CELL + c) * cap + t] = __int_as_float((i2 << 16) | k2);
    if (c == 0) {
        s[TF_U * cap + t] = mk.uDelta;
        s[TF_V * cap + t] = mk.vDelta;
        s[TF_WV * cap + t] = mk.wDelta;
    }
}

// Bulk asynchronous copies global -> shared memory with an mbarrier
// (cp.async.bulk, no multicast): one thread issues them, the group waits on
// the barrier's transaction count. Source and destination 16-byte aligned,
// sizes a multiple of 16 bytes.
__device__ unsigned g_ibm_bulk_timeouts = 0;   // waits that gave up (then the tile is loaded by plain loads)

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect(uint64_t* bar, unsigned bytes) {
    asm volatile("{ .reg .b64 st; mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1; }" ::"r"(smem_addr(bar)),
                 "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_to_smem(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}
// Wait for phase 0 of the barrier, at most `limit` polls; false when it gave up.
__device__ __forceinline__ bool mbar_wait0(uint64_t* bar, int limit) {
    for (int it = 0; it < limit; it++) {
        unsigned done;
        asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; selp.u32 %0, 1, 0, p; }"
                     : "=r"(done) : "r"(smem_addr(bar)) : "memory");
        if (done) return true;
    }
    return false;
}
// The 16-byte aligned span of elements [c0, c0 + n) of a 4-byte array:
// the first element copied, its offset from c0 and the bytes to copy.
struct BulkSpan {
    const void* src;
    int off;
    unsigned bytes;
};
__device__ __forceinline__ BulkSpan bulk_span(const void* base, int c0, int n) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(base) + 4ull * (unsigned)c0;
    const uintptr_t lo = a & ~uintptr_t(15), hi = (a + 4ull * (unsigned)n + 15) & ~uintptr_t(15);
    return BulkSpan{reinterpret_cast<const void*>(lo), (int)((a - lo) >> 2), (unsigned)(hi - lo)};
}
// Floats between the three F arrays of a bulk tile of `cells` cells: room
// for the 16-byte rounding of each copy, and a multiple of 4, so that every
// array (a bulk copy's destination) starts on a 16-byte boundary.
__host__ __device__ constexpr int bulk_tile_stride(int cells) { return (cells + 8 + 3) & ~3; }

// Element i of a row held as float4 registers (i a compile-time constant
// after unrolling).
template <int N>
__device__ __forceinline__ float f4_lane(const float4 (&r)[N], int i) {
    const float4 v = r[i >> 2];
    return (i & 3) == 0 ? v.x : (i & 3) == 1 ? v.y : (i & 3) == 2 ? v.z : v.w;
}

// Bring elements [c0, c0 + n) of a 4-byte array into L2 (cp.async.bulk
// prefetch: no completion to wait for). The span is rounded out to 16 bytes;
// every array prefetched this way is allocated with 16 elements of padding.
__device__ __forceinline__ void prefetch_l2(const void* base, int c0, int n) {
    if (n <= 0) return;
    const BulkSpan sp = bulk_span(base, c0, n);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(sp.src), "r"(sp.bytes) : "memory");
}
// The per-marker and per-cell data a group's walk of plane j reads, into L2
// while the group fills its tile: the first segment's weights, cells and
// velocities (markers [pm0, pm1) of the prep arrays), the plane's cell
// moments and elements, and the blade markers' gathered stencils. One array
// per lane.
template <typename GRP>
__device__ __forceinline__ void prefetch_plane(const IbmArgs& a, int j, int c0, int nc, const GRP grp) {
    const int lane = grp.tid();
    if (lane >= 32) return;
    const int pm0 = a.level_ptr[a.plane_lv0[j]], pm1 = a.level_ptr[a.plane_lv0[j + 1]];
    const int q0 = a.level_ptr[a.plane_lv1[j]] - a.n0, q1 = a.level_ptr[a.plane_lv1[j + 1]] - a.n0;
    for (int f = lane; f < 3 + TF_COUNT; f += 32) {
        if (f == 0) prefetch_l2(a.prep, pm0 * PF_STRIDE, (pm1 - pm0) * PF_STRIDE);
        else if (f == 1) prefetch_l2(a.cell_m, 4 * c0, 4 * nc);
        else if (f == 2) prefetch_l2(a.cell_e, c0, nc);
        else prefetch_l2(a.tail + (size_t)(f - 3) * a.tail_cap, q0, q1 - q0);
    }
}

// A group of NT threads (whole warps) that walks one j-plane. Several groups
// can share a CTA, each synchronising on its own named barrier (bar.sync id,
// NT), so that the planes of one CTA advance independently; a group that is
// the whole CTA uses barrier 0 (__syncthreads).
template <int NT, bool NAMED = false>
struct PlaneGroup {
    int base;  // the group's first thread in the CTA
    int bar;   // named barrier id (NAMED), else the CTA barrier
    // thread index within the group (read from threadIdx each time, so that
    // it occupies no register of the register-bound walks)
    __device__ __forceinline__ int tid() const { return NAMED ? (int)threadIdx.x - base : (int)threadIdx.x; }
    __device__ __forceinline__ void sync() const {
        if constexpr (NAMED) asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(NT) : "memory");
        else __syncthreads();
    }
};

// Blade levels of plane j on global memory: F and the touched flags are
// read back from L2 (__ldcg), since earlier levels of this CTA wrote them.
// Used when the plane's blade stencils do not fit the shared-memory table;
// a called function rather than inlined, so that this rare fallback costs
// the register-bound walks around it no registers.
template <int NT, typename GRP>
__device__ __noinline__ void blade_levels_global(const IbmArgs& a, int j, const GRP grp) {
    const Dims g = a.g;
    const float* s = a.tail;
    const long long cap = a.tail_cap;
    for (int lv = a.plane_lv1[j]; lv < a.plane_lv1[j + 1]; lv++) {
        const int p0 = a.level_ptr[lv], p1 = a.level_ptr[lv + 1];
#pragma unroll 1
        for (int p = p0 + grp.tid(); p < p1; p += NT) {
            const int t = p - a.n0;
            float rhoSum = 0.f, xSum = 0.f, ySum = 0.f, zSum = 0.f;
#pragma unroll
            for (int c = 0; c < 9; c++) {
                const float w = s[(TF_W + c) * cap + t];
                const int packed = __float_as_int(s[(TF_CELL + c) * cap + t]);
                const int i2 = packed >> 16, k2 = packed & 0xffff;
                const long long row = (long long)i2 * g.ny + j;
                const long long e = row * g.kp + k2;
                const long long wd = row * g.kw + (k2 >> 5);
                const uint32_t bit = 1u << (k2 & 31);
                const bool live = (__ldcg(a.mask_new + wd) & bit) || (a.mask_old[wd] & bit);
                const float4 v = live ? __ldcg(a.F4 + e) : make_float4(0.f, 0.f, 0.f, 0.f);
                const float vx = v.x, vy = v.y, vz = v.z;
                rhoSum = fmaf(w, s[(TF_RHO + c) * cap + t], rhoSum);
                xSum = fmaf(w, fmaf(0.5f, vx, s[(TF_MX + c) * cap + t]), xSum);
                ySum = fmaf(w, fmaf(0.5f, vy, s[(TF_MY + c) * cap + t]), ySum);
                zSum = fmaf(w, fmaf(0.5f, vz, s[(TF_MZ + c) * cap + t]), zSum);
            }
            xSum = fmaf(-rhoSum, s[TF_U * cap + t], xSum);
            ySum = fmaf(-rhoSum, s[TF_V * cap + t], ySum);
            zSum = fmaf(-rhoSum, s[TF_WV * cap + t], zSum);
            a.sums[p] = xSum;
            a.sums[a.n + p] = ySum;
            a.sums[2 * a.n + p] = zSum;
#pragma unroll
            for (int c = 0; c < 9; c++) {
                const int packed = __float_as_int(s[(TF_CELL + c) * cap + t]);
                const int i2 = packed >> 16, k2 = packed & 0xffff;
                const long long row = (long long)i2 * g.ny + j;
                const long long e = row * g.kp + k2;
                const long long wd = row * g.kw + (k2 >> 5);
                const uint32_t bit = 1u << (k2 & 31);
                const bool live = (__ldcg(a.mask_new + wd) & bit) || (a.mask_old[wd] & bit);
                const float4 v = live ? __ldcg(a.F4 + e) : make_float4(0.f, 0.f, 0.f, 0.f);
                const float bw = a.beta * s[(TF_W + c) * cap + t];
                a.F4[e] = make_float4(fmaf(a.alpha, v.x, -bw * xSum), fmaf(a.alpha, v.y, -bw * ySum),
                                      fmaf(a.alpha, v.z, -bw * zSum), 0.f);
                atomicOr(&a.mask_new[wd], bit);
            }
        }
        grp.sync();
    }
}

// Blade levels of plane j on a shared-memory table. The plane's 9 x nb
// stencil references (nb blade markers) go into an open-addressing hash
// table keyed by the packed cell (i << 16 | k), H >= 9 nb entries of (key,
// Fx, Fy, Fz), so every insert ends within H probes. Each cell's F is loaded
// once -- zero unless this pass (mask_new: the first segment's cells) or the
// previous one touched it -- the levels run on the table, and the cells go
// back to F with their touched flags. The walk reads and writes the same
// values in the same order as blade_levels_global; only the L2 round trips
// between levels go. Needs 4 H + 9 nb words of `tile`; returns false, having
// done nothing, when they do not fit.
template <int THREADS, typename GRP>
__device__ __forceinline__ bool blade_levels_tile(const IbmArgs& a, int j, float* tile, int tile_words,
                                                  const GRP grp) {
    const int lv0 = a.plane_lv1[j], lv1 = a.plane_lv1[j + 1];
    const int q0 = a.level_ptr[lv0], q1 = a.level_ptr[lv1];
    const int nref = 9 * (q1 - q0);
    int lg = 5;
    while ((1 << lg) < nref) lg++;
    const int H = 1 << lg;
    if (4LL * H + nref > (long long)tile_words) return false;
    int* keys = reinterpret_cast<int*>(tile);
    float* hx = tile + H;
    float* hy = tile + 2 * H;
    float* hz = tile + 3 * H;
    int* ref = reinterpret_cast<int*>(tile + 4 * H);
    const Dims g = a.g;
    const float* s = a.tail;
    const long long cap = a.tail_cap;
    const bool distinct = g.nx >= 3 && g.nz >= 3;   // the 9 stencil cells of a marker differ

    for (int h = grp.tid(); h < H; h += THREADS) keys[h] = -1;
    grp.sync();
    // inserts, four references per thread at a time (their keys loaded
    // together)
    for (int r0 = grp.tid(); r0 < nref; r0 += 4 * THREADS) {
        int kk[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int r = r0 + u * THREADS;
            const int m = r / 9, c = r - 9 * m;
            kk[u] = r < nref ? __float_as_int(s[(TF_CELL + c) * cap + (q0 + m - a.n0)]) : -1;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int r = r0 + u * THREADS;
            if (r >= nref) break;
            const int key = kk[u];
            unsigned h = ((unsigned)key * 2654435761u) >> (32 - lg);
            for (int probe = 0; probe < H; probe++) {
                const int prev = atomicCAS(&keys[h], -1, key);
                if (prev == -1 || prev == key) break;
                h = (h + 1) & (unsigned)(H - 1);
            }
            ref[r] = (int)h;
        }
    }
    grp.sync();
    // each table cell's F, four entries per thread at a time: F is read
    // whatever the flags say (e is a lattice cell), so that the flag and F
    // loads of the four make one round trip
    for (int h0 = grp.tid(); h0 < H; h0 += 4 * THREADS) {
        float vx[4], vy[4], vz[4];
        bool live[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int h = h0 + u * THREADS;
            const int key = h < H ? keys[h] : -1;
            const int i2 = key >> 16, k2 = key & 0xffff;
            const long long row = (long long)i2 * g.ny + j;
            const long long e = row * g.kp + k2;
            const long long wd = row * g.kw + (k2 >> 5);
            const uint32_t bit = 1u << (k2 & 31);
            live[u] = false;
            vx[u] = vy[u] = vz[u] = 0.f;
            if (key >= 0) {
                const float4 v = __ldcg(a.F4 + e);
                vx[u] = v.x;
                vy[u] = v.y;
                vz[u] = v.z;
                live[u] = (__ldcg(a.mask_new + wd) & bit) || (a.mask_old[wd] & bit);
            }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int h = h0 + u * THREADS;
            if (h < H && keys[h] >= 0) {
                hx[h] = live[u] ? vx[u] : 0.f;
                hy[h] = live[u] ? vy[u] : 0.f;
                hz[h] = live[u] ? vz[u] : 0.f;
            }
        }
    }
    grp.sync();
    for (int lv = lv0; lv < lv1; lv++) {
        const int p0 = a.level_ptr[lv], p1 = a.level_ptr[lv + 1];
#pragma unroll 1
        for (int p = p0 + grp.tid(); p < p1; p += THREADS) {
            const int t = p - a.n0;
            const int* rf = ref + 9 * (p - q0);
            float rhoSum = 0.f, xSum = 0.f, ySum = 0.f, zSum = 0.f;
            float w[9], ox[9], oy[9], oz[9];
            int hh[9];
#pragma unroll
            for (int c = 0; c < 9; c++) {
                w[c] = s[(TF_W + c) * cap + t];
                hh[c] = rf[c];
                ox[c] = hx[hh[c]];
                oy[c] = hy[hh[c]];
                oz[c] = hz[hh[c]];
                rhoSum = fmaf(w[c], s[(TF_RHO + c) * cap + t], rhoSum);
                xSum = fmaf(w[c], fmaf(0.5f, ox[c], s[(TF_MX + c) * cap + t]), xSum);
                ySum = fmaf(w[c], fmaf(0.5f, oy[c], s[(TF_MY + c) * cap + t]), ySum);
                zSum = fmaf(w[c], fmaf(0.5f, oz[c], s[(TF_MZ + c) * cap + t]), zSum);
            }
            xSum = fmaf(-rhoSum, s[TF_U * cap + t], xSum);
            ySum = fmaf(-rhoSum, s[TF_V * cap + t], ySum);
            zSum = fmaf(-rhoSum, s[TF_WV * cap + t], zSum);
            a.sums[p] = xSum;
            a.sums[a.n + p] = ySum;
            a.sums[2 * a.n + p] = zSum;
            if (distinct) {   // 9 different cells: independent updates
#pragma unroll
                for (int c = 0; c < 9; c++) {
                    const float bw = a.beta * w[c];
                    hx[hh[c]] = fmaf(a.alpha, ox[c], -bw * xSum);
                    hy[hh[c]] = fmaf(a.alpha, oy[c], -bw * ySum);
                    hz[hh[c]] = fmaf(a.alpha, oz[c], -bw * zSum);
                }
            } else {
#pragma unroll
                for (int c = 0; c < 9; c++) {   // sequential: a wrapped stencil sees its own update
                    const float bw = a.beta * w[c];
                    hx[hh[c]] = fmaf(a.alpha, hx[hh[c]], -bw * xSum);
                    hy[hh[c]] = fmaf(a.alpha, hy[hh[c]], -bw * ySum);
                    hz[hh[c]] = fmaf(a.alpha, hz[hh[c]], -bw * zSum);
                }
            }
        }
        grp.sync();
    }
    for (int h = grp.tid(); h < H; h += THREADS) {
        const int key = keys[h];
        if (key < 0) continue;
        const int i2 = key >> 16, k2 = key & 0xffff;
        const long long row = (long long)i2 * g.ny + j;
        const long long e = row * g.kp + k2;
        a.F4[e] = make_float4(hx[h], hy[h], hz[h], 0.f);
        atomicOr(&a.mask_new[row * g.kw + (k2 >> 5)], 1u << (k2 & 31));
    }
    return true;
}

// One group per j-plane: the plane's first-segment levels on an F tile in
// shared memory (planes with more cells than the tile holds work on cell_F
// in place), write-back to F, then (BLADES) the blade levels, on a
// shared-memory table when they fit the tile, else on global F. The touched
// flags of the first segment never change, so each pass starts mask_new as
// a copy of them (mask_static) and the blade walk adds its cells.
// BULK: the group's tile is [3][bulk_tile_stride(tile_cells)] words (F x, y,
// z), filled by bulk copies of the plane's cell range (bar: the group's
// mbarrier).
// Otherwise the tile is [3][tile_cells] and filled by plain loads.
template <int THREADS, bool BULK = false, typename GRP = PlaneGroup<THREADS>, bool PIPE = false, bool BLADES = true>
__device__ __forceinline__ void ibm_spread_plane(const IbmArgs& a, int j, int tile_cells, float* tile, const GRP grp,
                                                 uint64_t* bar = nullptr, int* bulk_fail = nullptr) {
    const int c0 = a.plane_cell[j], nc = a.plane_cell[j + 1] - c0;
    const long long C = a.ncell;
    const bool in_smem = nc <= tile_cells;
    float *fx, *fy, *fz;
    prefetch_plane(a, j, c0, nc, grp);
    if (BULK && in_smem && nc > 0) {
        const int tc = bulk_tile_stride(tile_cells);
        const BulkSpan sx = bulk_span(a.cell_F + c0, 0, nc), sy = bulk_span(a.cell_F + C + c0, 0, nc),
                       sz = bulk_span(a.cell_F + 2 * C + c0, 0, nc);
        if (grp.tid() == 0) {
            mbar_init(bar);
            *bulk_fail = 0;
        }
        grp.sync();
        if (grp.tid() == 0) {
            mbar_expect(bar, sx.bytes + sy.bytes + sz.bytes);
            bulk_to_smem(tile, sx.src, sx.bytes, bar);
            bulk_to_smem(tile + tc, sy.src, sy.bytes, bar);
            bulk_to_smem(tile + 2 * tc, sz.src, sz.bytes, bar);
        }
        fx = tile + sx.off; fy = tile + tc + sy.off; fz = tile + 2 * tc + sz.off;
        // bounded wait; the group decides together whether it gave up, so
        // that every thread takes the same barriers
        if (!mbar_wait0(bar, 1 << 20)) *bulk_fail = 1;
        grp.sync();
        if (*bulk_fail) {
            // should not happen: count it, give the copies more time, then
            // load the tile with plain loads
            if (grp.tid() == 0) atomicAdd(&g_ibm_bulk_timeouts, 1u);
            mbar_wait0(bar, 1 << 22);
            grp.sync();
            for (int t = grp.tid(); t < nc; t += THREADS) {
                fx[t] = a.cell_F[c0 + t];
                fy[t] = a.cell_F[C + c0 + t];
                fz[t] = a.cell_F[2 * C + c0 + t];
            }
        }
    } else if (in_smem) {
        fx = tile; fy = tile + tile_cells; fz = tile + 2 * tile_cells;
#pragma unroll 4
        for (int t = grp.tid(); t < nc; t += THREADS) {
            fx[t] = a.cell_F[c0 + t];
            fy[t] = a.cell_F[C + c0 + t];
            fz[t] = a.cell_F[2 * C + c0 + t];
        }
    } else {
        fx = a.cell_F + c0; fy = a.cell_F + C + c0; fz = a.cell_F + 2 * C + c0;
    }
    grp.sync();

    // ---- first segment: each marker in list order relative to every marker
    //      it shares a cell with (level walk). With x and z at least 3 the 9
    //      stencil cells of a marker differ (the stencil wraps onto itself
    //      only on a narrower lattice).
    const bool distinct = a.g.nx >= 3 && a.g.nz >= 3;
    const float4* cm = reinterpret_cast<const float4*>(a.cell_m) + c0;   // rho, jx, jy, jz
    // PIPE: each thread's next slot row (the next slot of this level, else
    // its first slot of the next level) is loaded while the current slot is
    // processed, so a level's rounds wait for the cell moments only (it takes
    // 24 more registers: launches of at most 384 threads).
    const int lvb = a.plane_lv0[j], lve = a.plane_lv0[j + 1];
    float4 r[PF_STRIDE / 4];
    int rp = -1;   // the slot r holds
    for (int lv = lvb; lv < lve; lv++) {
        const int p0 = a.level_ptr[lv], p1 = a.level_ptr[lv + 1];
        const int p2 = lv + 1 < lve ? a.level_ptr[lv + 2] : p1;
#pragma unroll 1
        for (int p = p0 + grp.tid(); p < p1; p += THREADS) {
            float rhoSum = 0.f, xSum = 0.f, ySum = 0.f, zSum = 0.f;
            float w[9], ox[9], oy[9], oz[9];
            int li[9];
            if (rp != p) {
#pragma unroll
                for (int u = 0; u < PF_STRIDE / 4; u++) r[u] = reinterpret_cast<const float4*>(a.prep + (size_t)p * PF_STRIDE)[u];
            }
            int pn = p + THREADS, pe = p1;
            if (pn >= p1) {
                pn = p1 + grp.tid();
                pe = p2;
            }
            float4 rn[PF_STRIDE / 4];
            if (PIPE && pn < pe) {
#pragma unroll
                for (int u = 0; u < PF_STRIDE / 4; u++) rn[u] = reinterpret_cast<const float4*>(a.prep + (size_t)pn * PF_STRIDE)[u];
            }
#pragma unroll
            for (int c = 0; c < 9; c++) {
                w[c] = f4_lane(r, PF_W + c);
                li[c] = __float_as_int(f4_lane(r, PF_CELL + c));
            }
#pragma unroll
            for (int c = 0; c < 9; c++) {
                const float4 m = cm[li[c]];
                ox[c] = fx[li[c]];
                oy[c] = fy[li[c]];
                oz[c] = fz[li[c]];
                rhoSum = fmaf(w[c], m.x, rhoSum);
                xSum = fmaf(w[c], fmaf(0.5f, ox[c], m.y), xSum);
                ySum = fmaf(w[c], fmaf(0.5f, oy[c], m.z), ySum);
                zSum = fmaf(w[c], fmaf(0.5f, oz[c], m.w), zSum);
            }
            xSum = fmaf(-rhoSum, f4_lane(r, PF_U), xSum);
            ySum = fmaf(-rhoSum, f4_lane(r, PF_V), ySum);
            zSum = fmaf(-rhoSum, f4_lane(r, PF_WV), zSum);
            a.sums[p] = xSum;
            a.sums[a.n + p] = ySum;
            a.sums[2 * a.n + p] = zSum;
            if (distinct) {
                // 9 different cells: each update starts from the value read
                // above, so the 27 stores are independent
#pragma unroll
                for (int c = 0; c < 9; c++) {
                    const float bw = a.beta * w[c];
                    fx[li[c]] = fmaf(a.alpha, ox[c], -bw * xSum);
                    fy[li[c]] = fmaf(a.alpha, oy[c], -bw * ySum);
                    fz[li[c]] = fmaf(a.alpha, oz[c], -bw * zSum);
                }
            } else {
#pragma unroll
                for (int c = 0; c < 9; c++) {   // sequential: a wrapped stencil sees its own update
                    const float bw = a.beta * w[c];
                    fx[li[c]] = fmaf(a.alpha, fx[li[c]], -bw * xSum);
                    fy[li[c]] = fmaf(a.alpha, fy[li[c]], -bw * ySum);
                    fz[li[c]] = fmaf(a.alpha, fz[li[c]], -bw * zSum);
                }
            }
            if constexpr (PIPE) {
#pragma unroll
                for (int u = 0; u < PF_STRIDE / 4; u++) r[u] = rn[u];
                rp = pn < pe ? pn : -1;
            }
        }
        grp.sync();
    }
    // ---- write the plane's cells back to F (eight element loads in flight
    //      per thread)
    {
        int t = grp.tid();
        for (; t + 7 * THREADS < nc; t += 8 * THREADS) {
            int e[8];
#pragma unroll
            for (int u = 0; u < 8; u++) e[u] = a.cell_e[c0 + t + u * THREADS];
#pragma unroll
            for (int u = 0; u < 8; u++)
                a.F4[e[u]] = make_float4(fx[t + u * THREADS], fy[t + u * THREADS], fz[t + u * THREADS], 0.f);
        }
        for (; t < nc; t += THREADS) {
            const int e = a.cell_e[c0 + t];
            a.F4[e] = make_float4(fx[t], fy[t], fz[t], 0.f);
        }
    }
    grp.sync();

    // ---- second segment (blades), unless a separate launch walks them
    if (!BLADES || a.plane_lv1[j] == a.plane_lv1[j + 1]) return;
    const int words = BULK ? 3 * bulk_tile_stride(tile_cells) : 3 * tile_cells;
    if (!blade_levels_tile<THREADS>(a, j, tile, words, grp)) blade_levels_global<THREADS>(a, j, grp);
}

// G planes per CTA: group g (NT threads, its own barrier) walks plane
// planes[blockIdx.x * G + g] on its own tile, which bulk copies fill with one
// latency whatever the group's size. The ordinary planes run G = 1..4 groups
// of 128 threads, so all planes of a large lattice are resident at once; the
// big planes (an impeller disk) one group of 512.
template <int NT, int G, bool BLADES = true>
__global__ void __launch_bounds__(NT * G, 1) k_ibm_spread_bulk(IbmArgs a, const int* __restrict__ planes, int nplanes,
                                                              int tile_cells) {
    extern __shared__ __align__(128) float btile[];             // [G][3][bulk_tile_stride(tile_cells)]
    __shared__ uint64_t bars[G];
    __shared__ int fails[G];
    const int g = G == 1 ? 0 : (int)threadIdx.x / NT;
    const int q = (int)blockIdx.x * G + g;
    if (q >= nplanes) return;
    const PlaneGroup<NT, (G > 1)> grp{g * NT, g + 1};
    ibm_spread_plane<NT, true, PlaneGroup<NT, (G > 1)>, (NT * G <= 384), BLADES>(
        a, planes[q], tile_cells, btile + (size_t)g * 3 * bulk_tile_stride(tile_cells), grp, &bars[g],
                               &fails[g]);
}

// The blade levels of the planes that have blades, one plane per CTA of NT
// threads, after both first-segment spreads have written their planes' F:
// the blade planes' walks then run wide instead of holding up the
// 128-thread groups of the ordinary planes' launch. `words` floats of
// shared memory hold the plane's hash table.
template <int NT>
__global__ void __launch_bounds__(NT, 1) k_ibm_blades(IbmArgs a, const int* __restrict__ planes, int nplanes,
                                                      int words) {
    extern __shared__ __align__(16) float btab[];
    if ((int)blockIdx.x >= nplanes) return;
    const int j = planes[blockIdx.x];
    const PlaneGroup<NT> grp{0, 0};
    if (!blade_levels_tile<NT>(a, j, btab, words, grp)) blade_levels_global<NT>(a, j, grp);
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

// Deterministic FP64 reduction of the marker forces: fixed grid, fixed
// per-thread stride, fixed shared-memory tree, then one block sums the
// partials in order.
__global__ void __launch_bounds__(256) k_marker_load(IbmArgs a, int begin, double ci, double ck, double* partial) {
    __shared__ double red[5][256];
    double acc[5] = {0, 0, 0, 0, 0};
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += gridDim.x * blockDim.x) {
        const int q = a.sched[p];
        if (q < begin) continue;
        const Marker mk = a.markers[q];
        const double fx = -(double)a.beta * (double)a.sums[p];
        const double fy = -(double)a.beta * (double)a.sums[a.n + p];
        const double fz = -(double)a.beta * (double)a.sums[2 * a.n + p];
        const double di = (double)mk.i + (double)mk.iCartFraction - ci;
        const double dk = (double)mk.k + (double)mk.kCartFraction - ck;
        acc[0] += fx;
        acc[1] += fy;
        acc[2] += fz;
        acc[3] += dk * fx - di * fz;   // (r x F) along j, r = (di, 0, dk)
        acc[4] += 1.0;
    }
    for (int c = 0; c < 5; c++) red[c][threadIdx.x] = acc[c];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int c = 0; c < 5; c++) red[c][threadIdx.x] += red[c][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 5; c++) partial[blockIdx.x * 5 + c] = red[c][0];
}

// Ordered sum of the block partials: the warp stages them in shared memory
// (coalesced, all loads in flight at once), then one thread adds them in
// block order, so the result does not depend on the launch.
template <int NC, int NB>
__device__ __forceinline__ void ordered_final(const double* __restrict__ partial, int nblocks, double* out) {
    __shared__ double v[NB * NC];
    const int n = nblocks * NC;
    for (int q = threadIdx.x; q < n; q += blockDim.x) v[q] = partial[q];
    __syncthreads();
    if (threadIdx.x != 0) return;
    double acc[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) acc[c] = 0.0;
    for (int b = 0; b < nblocks; b++)
#pragma unroll
        for (int c = 0; c < NC; c++) acc[c] += v[b * NC + c];
#pragma unroll
    for (int c = 0; c < NC; c++) out[c] = acc[c];
}

__global__ void k_marker_load_final(const double* partial, int nblocks, double* out) {
    ordered_final<5, kLoadBlocks>(partial, nblocks, out);
}

cudaError_t launch_marker_load(const IbmArgs& a, int begin, double ci, double ck, double* partial, double* out,
                               cudaStream_t st) {
    k_marker_load<<<kLoadBlocks, 256, 0, st>>>(a, begin, ci, ck, partial);
    k_marker_load_final<<<1, 32, 0, st>>>(partial, kLoadBlocks, out);
    return cudaGetLastError();
}

// FP64 mass and momentum over all interior cells, deterministic: a fixed
// grid of kReduceBlocks blocks, a fixed per-thread stride, a fixed tree,
// then one thread sums the block partials in order.
template <typename S>
__global__ void __launch_bounds__(256) k_reduce_fp64(IbmArgs a, const uint32_t* __restrict__ mask, double* partial) {
    __shared__ double red[4][256];
    const Dims g = a.g;
    const long long total = g.rows() * g.nz;
    double acc[4] = {0, 0, 0, 0};
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % g.nz);
        const long long row = t / g.nz;
        const int j = (int)(row % g.ny), i = (int)(row / g.ny);
        float m4[4];
        cell_moments4<S>(a.A, a.state_mode, a.even, g, i, j, k, a.p, m4, a.rbox);
        const long long e = row * g.kp + k;
        const bool on = (mask[row * g.kw + (k >> 5)] >> (k & 31)) & 1u;
        acc[0] += m4[0];
        const float4 f = on ? a.F4[e] : make_float4(0.f, 0.f, 0.f, 0.f);
        acc[1] += (double)m4[1] + (on ? 0.5 * (double)f.x : 0.0);
        acc[2] += (double)m4[2] + (on ? 0.5 * (double)f.y : 0.0);
        acc[3] += (double)m4[3] + (on ? 0.5 * (double)f.z : 0.0);
    }
    for (int c = 0; c < 4; c++) red[c][threadIdx.x] = acc[c];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int c = 0; c < 4; c++) red[c][threadIdx.x] += red[c][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 4; c++) partial[blockIdx.x * 4 + c] = red[c][0];
}

__global__ void k_reduce_fp64_final(const double* partial, int nblocks, double* out) {
    ordered_final<4, kReduceBlocks>(partial, nblocks, out);
}

cudaError_t launch_reduce_fp64(const IbmArgs& a, const uint32_t* mask, double* partial, double* out, cudaStream_t st) {
    with_storage(a.storage, [&](auto s) {
        k_reduce_fp64<decltype(s)><<<kReduceBlocks, 256, 0, st>>>(a, mask, partial);
    });
    k_reduce_fp64_final<<<1, 32, 0, st>>>(partial, kReduceBlocks, out);
    return cudaGetLastError();
}

// Rest state of the 16-bit storage at density rho: every population
// w_d * rho, stored as its deviation from w_d * rho0.
template <typename S>
__global__ void k_fill_rest(Planes Q, long long plane, float rho_ratio_m1, CollideParams p) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= plane) return;
#pragma unroll
    for (int d = 0; d < NQ; d++)
        reinterpret_cast<S*>(Q.p[d])[t] = Storage<S>::enc(rho_ratio_m1 * (is_face(d) ? p.wface : p.wedge));
}

cudaError_t launch_fill_rest(Planes Q, long long plane, float rho, float rho0, int storage, const CollideParams& p,
                             cudaStream_t st) {
    const unsigned b = (unsigned)((plane + 255) / 256);
    const float r = rho / rho0 - 1.f;
    with_storage(storage, [&](auto s) { k_fill_rest<decltype(s)><<<b, 256, 0, st>>>(Q, plane, r, p); });
    return cudaGetLastError();
}

size_t ibm_smem_bytes(const Dims& g, int cells) {
    (void)g;
    return (size_t)3 * cells * sizeof(float);
}

// The dynamic shared-memory limit is a per-kernel, per-device attribute that
// every lattice and batch shares: it only ever grows, so that a smaller
// lattice set up later cannot lower it below what a larger one launches with.
cudaError_t raise_smem_limit(const void* fn, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> set;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    size_t& cur = set[{fn, dev}];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

// Ordinary planes per CTA: as few 128-thread groups as put every plane on
// the GPU at once (nplanes / SMs, rounded up), at most as many as their F
// tiles (12 bytes per cell) fit in the 227 KB of shared memory a CTA may use,
// and at most 4: groups of one CTA share its SM's load/store pipe. (At 400^3
// the 399 ordinary planes hold 5214 cells each: 3 groups, 133 CTAs.)
static int sm_count() {
    static int n[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (n[dev] == 0) {
        int v = 0;
        n[dev] = cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0 ? v : 148;
    }
    return n[dev];
}
int spread_groups(int tile_cells, int nplanes) {
    const size_t per = (size_t)12 * bulk_tile_stride(tile_cells);
    int G = (int)((227 * 1024 - 64) / per);
    G = G < 1 ? 1 : (G > 4 ? 4 : G);
    const int sms = sm_count();
    const int want = nplanes > 0 ? (nplanes + sms - 1) / sms : 1;
    return want < G ? (want < 1 ? 1 : want) : G;
}

template <int G>
static const void* spread_bulk_fn() { return (const void*)k_ibm_spread_bulk<128, G, false>; }

template <int G>
static void spread_small(const IbmArgs& a, cudaStream_t st) {
    const unsigned grid = (unsigned)((a.n_small + G - 1) / G);
    const size_t bytes = (size_t)G * 12 * bulk_tile_stride(a.smem_cells);
    k_ibm_spread_bulk<128, G, false><<<grid, 128 * G, bytes, st>>>(a, a.plane_list, a.n_small, a.smem_cells);
}

// Shared memory (floats) of the blade launch for a plane of nb blade
// markers: blade_levels_tile's table of H >= 9 nb entries (a power of two,
// at least 32) of four words, and 9 nb references.
int blade_table_words(int nb) {
    const int nref = 9 * nb;
    int H = 32;
    while (H < nref) H *= 2;
    return 4 * H + nref;
}

cudaError_t ibm_prepare_blades(int words) {
    return raise_smem_limit((const void*)k_ibm_blades<512>, (size_t)words * sizeof(float));
}

// Shared memory of the big planes' launch (one 512-thread group, a bulk
// tile of big_cells cells; none when the tile does not fit).
size_t big_bulk_bytes(int big_cells) { return big_cells > 0 ? (size_t)12 * bulk_tile_stride(big_cells) : 0; }

cudaError_t ibm_prepare_smem(int small_cells, int n_small, size_t big_bytes) {
    const int G = spread_groups(small_cells, n_small);
    const void* fn = G == 4 ? spread_bulk_fn<4>() : G == 3 ? spread_bulk_fn<3>() : G == 2 ? spread_bulk_fn<2>()
                                                                                       : spread_bulk_fn<1>();
    cudaError_t e = raise_smem_limit(fn, (size_t)G * 12 * bulk_tile_stride(small_cells));
    if (e != cudaSuccess) return e;
    return raise_smem_limit((const void*)k_ibm_spread_bulk<512, 1, false>, big_bytes);
}

cudaError_t launch_ibm_prepare(const IbmArgs& a, float* prep, const int* mcell, cudaStream_t st) {
    (void)mcell;
    if (a.n0 <= 0) return cudaSuccess;
    k_ibm_prepare<<<(a.n0 + 255) / 256, 256, 0, st>>>(a, prep);
    return cudaGetLastError();
}

cudaError_t launch_ibm(const IbmArgs& a, cudaStream_t st) {
    bool mask_copied = false;
    auto cells = [&](int first, int count, bool copy_mask, cudaStream_t cs) {
        if (count <= 0) return;
        with_storage(a.storage, [&](auto s) {
            k_ibm_cells<decltype(s)><<<(count + 255) / 256, 256, 0, cs>>>(a, first, count, copy_mask ? 1 : 0);
        });
        mask_copied |= copy_mask;
    };
    auto tail = [&](cudaStream_t ts) {
        if (a.n <= a.n0) return;
        const unsigned b = (unsigned)((9LL * (a.n - a.n0) + 127) / 128);
        with_storage(a.storage, [&](auto s) { k_ibm_gather_tail<decltype(s)><<<b, 128, 0, ts>>>(a); });
    };
    // mask_new starts as the first segment's (static) touched cells: copied
    // by the (largest) cells launch, else by a copy; only the blade walk
    // reads or sets mask_new, at the end of the pass.
    // Side stream: the blade markers' gather (which reads only the state and
    // is needed only by the blade walk) and the planes with many cells (an
    // impeller disk): their cells, then their spread with a full-size tile
    // and 512 threads, started before the ordinary planes' spread places its
    // blocks over the SMs. Handle's stream: the other planes' cells and
    // spread, then, after the side stream, the blade walk.
    cudaError_t err = cudaSuccess;
    const bool split = a.n_big > 0 && a.cell_order != nullptr;
    if (!split) cells(0, a.ncell, true, st);   // (before the fork: a big planes' spread reads them)
    err = cudaEventRecord(a.ev_fork, st);
    if (err != cudaSuccess) return err;
    err = cudaStreamWaitEvent(a.side, a.ev_fork, 0);
    if (err != cudaSuccess) return err;
    if (split) cells(0, a.ncell_big, false, a.side);
    tail(a.side);
    if (a.n_big > 0) {
        k_ibm_spread_bulk<512, 1, false><<<a.n_big, 512, big_bulk_bytes(a.big_tile_cells), a.side>>>(
            a, a.plane_list + a.n_small, a.n_big, a.big_tile_cells);
        err = cudaGetLastError();
        if (err != cudaSuccess) return err;
    }
    err = cudaEventRecord(a.ev_join, a.side);
    if (err != cudaSuccess) return err;
    if (split) cells(a.ncell_big, a.ncell - a.ncell_big, true, st);
    if (!mask_copied) {
        err = cudaMemcpyAsync(a.mask_new, a.mask_static, a.mask_bytes, cudaMemcpyDeviceToDevice, st);
        if (err != cudaSuccess) return err;
    }
    if (a.n_small > 0) {
        switch (spread_groups(a.smem_cells, a.n_small)) {
            case 4: spread_small<4>(a, st); break;
            case 3: spread_small<3>(a, st); break;
            case 2: spread_small<2>(a, st); break;
            default: spread_small<1>(a, st); break;
        }
    }
    err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    err = cudaStreamWaitEvent(st, a.ev_join, 0);
    if (err != cudaSuccess) return err;
    // the blade levels, once every plane's first segment is in F
    if (a.n_blade > 0) {
        k_ibm_blades<512><<<a.n_blade, 512, (size_t)a.blade_words * sizeof(float), st>>>(a, a.blade_planes, a.n_blade,
                                                                                      a.blade_words);
        err = cudaGetLastError();
    }
    return err;
}

// ---------------------------------------------------------------------------
// Batched passes: the immersed-boundary passes of many lattices in one set of
// launches. Every block takes one work item (lattice, first index); the
// lattice's IbmArgs is staged in shared memory and the single-lattice body
// runs on it, so each lattice's result equals its own launch_ibm.
// ---------------------------------------------------------------------------
template <int NT>
__device__ __forceinline__ void stage_args(IbmArgs& dst, const IbmArgs* src) {
    static_assert(sizeof(IbmArgs) % 8 == 0, "IbmArgs words");
    constexpr int words = sizeof(IbmArgs) / 8;
    for (int w = threadIdx.x; w < words; w += NT)
        reinterpret_cast<unsigned long long*>(&dst)[w] = reinterpret_cast<const unsigned long long*>(src)[w];
}

template <typename S>
__global__ void __launch_bounds__(256) k_ibm_cells_batch(const IbmArgs* __restrict__ args, const int2* __restrict__ work) {
    __shared__ IbmArgs sa;
    const int2 w = work[blockIdx.x];
    stage_args<256>(sa, args + w.x);
    __syncthreads();
    const int c = w.y + threadIdx.x;
    if (c < sa.ncell) ibm_cell<S>(sa, c);
}

template <typename S>
__global__ void __launch_bounds__(128) k_ibm_tail_batch(const IbmArgs* __restrict__ args, const int2* __restrict__ work) {
    __shared__ IbmArgs sa;
    const int2 w = work[blockIdx.x];
    stage_args<128>(sa, args + w.x);
    __syncthreads();
    const int t = w.y + threadIdx.x;
    if (t < sa.n - sa.n0) ibm_tail_marker<S>(sa, t);
}

// mask_new = mask_static, kMaskCopyWords words per work item
__global__ void __launch_bounds__(256) k_mask_copy_batch(const IbmArgs* __restrict__ args, const int2* __restrict__ work) {
    const int2 w = work[blockIdx.x];
    const IbmArgs& a = args[w.x];
    const long long words = (long long)(a.mask_bytes / sizeof(uint32_t));
    uint32_t* dst = a.mask_new;
    const uint32_t* src = a.mask_static;
    for (int q = threadIdx.x; q < kMaskCopyWords; q += 256) {
        const long long e = (long long)w.y + q;
        if (e < words) dst[e] = src[e];
    }
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS, THREADS == 128 ? 3 : 1) k_ibm_spread_batch(const IbmArgs* __restrict__ args,
                                                                             const int2* __restrict__ work, int big) {
    extern __shared__ float tile[];
    __shared__ IbmArgs sa;
    const int2 w = work[blockIdx.x];
    stage_args<THREADS>(sa, args + w.x);
    __syncthreads();
    const PlaneGroup<THREADS> grp{0, 0};
    ibm_spread_plane<THREADS>(sa, w.y, big ? sa.big_tile_cells : sa.smem_cells, tile, grp);
}

// The batch's ordinary planes, G work items (lattice, plane) per CTA: each
// group stages its lattice's arguments and walks its plane on a tile that
// bulk copies fill, as k_ibm_spread_bulk does for one lattice. region_cells:
// the largest tile of the batch's lattices (the group's share of shared
// memory); each lattice's walk uses its own tile size within it.
// (One group per CTA: at most 170 registers, so that three such CTAs fit an
// SM beside the other tank group's fused launch -- 64 tanks: 20,433 -> 21,000
// MLUPS FP32; 128 registers spill and measured slower.)
template <int NT, int G>
__global__ void __launch_bounds__(NT * G, G == 1 ? 3 : 1) k_ibm_spread_batch_bulk(const IbmArgs* __restrict__ args,
                                                                    const int2* __restrict__ work, int nwork,
                                                                    int region_cells) {
    extern __shared__ __align__(128) float btile[];             // [G][3][bulk_tile_stride(region_cells)]
    __shared__ IbmArgs sa[G];
    __shared__ uint64_t bars[G];
    __shared__ int fails[G];
    const int g = G == 1 ? 0 : (int)threadIdx.x / NT;
    const int q = (int)blockIdx.x * G + g;
    if (q >= nwork) return;
    const PlaneGroup<NT, (G > 1)> grp{g * NT, g + 1};
    const int2 w = work[q];
    constexpr int words = sizeof(IbmArgs) / 8;
    for (int i = grp.tid(); i < words; i += NT)
        reinterpret_cast<unsigned long long*>(&sa[g])[i] = reinterpret_cast<const unsigned long long*>(args + w.x)[i];
    grp.sync();
    ibm_spread_plane<NT, true, PlaneGroup<NT, (G > 1)>, (NT * G <= 384)>(
        sa[g], w.y, sa[g].smem_cells, btile + (size_t)g * 3 * bulk_tile_stride(region_cells), grp, &bars[g],
                               &fails[g]);
}

// Work items per CTA of the batched ordinary-plane spread: one. The batch's
// forcing pass runs beside the other tank group's fused launch, and a CTA of
// G groups holds G x 128 threads' registers (128-255 each) for its whole
// walk; measured on B200 (64 tanks, 20 steps): G <= 4 18,082 MLUPS FP32,
// G <= 2 19,086, G = 1 19,442 (FP16: 22,863 at G = 1).
static int batch_spread_groups(int cells) {
    (void)cells;
    return 1;
}

template <int G>
static const void* batch_bulk_fn() { return (const void*)k_ibm_spread_batch_bulk<128, G>; }

cudaError_t ibm_batch_prepare_smem(size_t small_bytes, size_t big_bytes) {
    (void)small_bytes;
    // every variant may be launched (tank groups with smaller tiles take more
    // work items per CTA): each gets the dynamic shared memory its widest
    // launch can use
    const void* fns[4] = {batch_bulk_fn<1>(), batch_bulk_fn<2>(), batch_bulk_fn<3>(), batch_bulk_fn<4>()};
    for (int G = 1; G <= 4; G++) {
        const size_t bytes = 227 * 1024 - (size_t)G * (sizeof(IbmArgs) + 16) - 256;
        cudaError_t e = raise_smem_limit(fns[G - 1], bytes);
        if (e != cudaSuccess) return e;
    }
    return raise_smem_limit((const void*)k_ibm_spread_batch<512>, big_bytes);
}

template <int G>
static void batch_spread_small(const IbmBatch& b, cudaStream_t st) {
    const unsigned grid = (unsigned)((b.n_small + G - 1) / G);
    const size_t bytes = (size_t)G * 12 * bulk_tile_stride(b.small_tile);
    k_ibm_spread_batch_bulk<128, G><<<grid, 128 * G, bytes, st>>>(b.args, b.small, b.n_small, b.small_tile);
}

cudaError_t launch_ibm_batch(const IbmBatch& b, cudaStream_t st, cudaStream_t side, cudaEvent_t fork, cudaEvent_t join) {
    if (b.n_cells > 0) {
        with_storage(b.storage, [&](auto s) {
            k_ibm_cells_batch<decltype(s)><<<b.n_cells, 256, 0, st>>>(b.args, b.cells);
        });
    }
    if (b.n_tails > 0) {
        with_storage(b.storage, [&](auto s) {
            k_ibm_tail_batch<decltype(s)><<<b.n_tails, 128, 0, st>>>(b.args, b.tails);
        });
    }
    if (b.n_copies > 0) k_mask_copy_batch<<<b.n_copies, 256, 0, st>>>(b.args, b.copies);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    if (b.n_big > 0) {
        err = cudaEventRecord(fork, st);
        if (err != cudaSuccess) return err;
        err = cudaStreamWaitEvent(side, fork, 0);
        if (err != cudaSuccess) return err;
        k_ibm_spread_batch<512><<<b.n_big, 512, ibm_smem_bytes(Dims{}, b.big_tile), side>>>(b.args, b.big, 1);
        err = cudaGetLastError();
        if (err != cudaSuccess) return err;
        err = cudaEventRecord(join, side);
        if (err != cudaSuccess) return err;
    }
    if (b.n_small > 0) {
        switch (batch_spread_groups(b.small_tile)) {
            case 4: batch_spread_small<4>(b, st); break;
            case 3: batch_spread_small<3>(b, st); break;
            case 2: batch_spread_small<2>(b, st); break;
            default: batch_spread_small<1>(b, st); break;
        }
    }
    err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    if (b.n_big > 0) return cudaStreamWaitEvent(st, join, 0);
    return cudaSuccess;
}

}  // namespace tdlb
