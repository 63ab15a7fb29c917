// Step-kernel templates (Simple pull and Esotwist in place), generic in the
// population storage type S (float, __half, __nv_bfloat16) and in V, the
// cells per thread. Instantiated by step_kernels.cu (FP32 storage) and
// step_kernels_h16.cu (16-bit deviation storage). See step_kernels.cu for
// the streaming semantics.
#pragma once
#include <cstring>

#include "tdlb_kernels.cuh"

namespace tdlb {

// ---------------------------------------------------------------------------
// Thread mapping shared by both schemes: V consecutive cells of one row per
// thread ("quad"), quads numbered row-major over (row, kq); a warp covers 32
// consecutive quads, so neighbouring lanes hold neighbouring cells of the
// same row except at row ends (where the wall rule or the periodic wrap
// applies anyway). V in {1, 2, 4}; populations move as float/float2/float4.
// ---------------------------------------------------------------------------
constexpr unsigned FULL = 0xffffffffu;

// FP32 vector helpers (F, Nu and FP32 populations)
template <int V>
__device__ __forceinline__ void vload(const float* __restrict__ p, float (&v)[V]) {
    if constexpr (V == 4) {
        const float4 t = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else if constexpr (V == 2) {
        const float2 t = __ldg(reinterpret_cast<const float2*>(p));
        v[0] = t.x; v[1] = t.y;
    } else {
        v[0] = __ldg(p);
    }
}
template <int V>
__device__ __forceinline__ void vstore(float* p, const float (&v)[V]) {
    if constexpr (V == 4) *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    else if constexpr (V == 2) *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
    else *p = v[0];
}
// Streaming stores (st.global.cs: first out of L2), for data the kernel does
// not read again -- Simple's destination buffer and Nu, FP32 storage.
// Measured on B200 at 400^3: k_step_simple 1.554 -> 1.528-1.535 ms; the
// in-place Esotwist kernel, which stores to the lines it has just read,
// measured slower with them (1.676 -> 1.724 ms), and so did the 16-bit Simple
// step (1.541 -> 1.574 ms whole step); those keep plain stores.
template <int V>
__device__ __forceinline__ void vstore_cs(float* p, const float (&v)[V]) {
    if constexpr (V == 4) __stcs(reinterpret_cast<float4*>(p), make_float4(v[0], v[1], v[2], v[3]));
    else if constexpr (V == 2) __stcs(reinterpret_cast<float2*>(p), make_float2(v[0], v[1]));
    else __stcs(p, v[0]);
}

// Population plane access in storage type S: V elements from element e,
// decoded to FP32 (RO: read-only, non-coherent path).
template <typename S, int V, bool RO>
__device__ __forceinline__ void pload(const float* plane, int e, float (&v)[V]) {
    if constexpr (sizeof(S) == 4) {
        const float* p = plane + e;
        if constexpr (V == 4) {
            const float4 t = RO ? __ldg(reinterpret_cast<const float4*>(p)) : *reinterpret_cast<const float4*>(p);
            v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
        } else if constexpr (V == 2) {
            const float2 t = RO ? __ldg(reinterpret_cast<const float2*>(p)) : *reinterpret_cast<const float2*>(p);
            v[0] = t.x; v[1] = t.y;
        } else {
            v[0] = RO ? __ldg(p) : *p;
        }
    } else {
        const S* p = reinterpret_cast<const S*>(plane) + e;
        if constexpr (V == 4) {
            const uint2 t = RO ? __ldg(reinterpret_cast<const uint2*>(p)) : *reinterpret_cast<const uint2*>(p);
            S s4[4];
            memcpy(s4, &t, sizeof t);
#pragma unroll
            for (int k = 0; k < 4; k++) v[k] = Storage<S>::dec(s4[k]);
        } else if constexpr (V == 2) {
            const unsigned t = RO ? __ldg(reinterpret_cast<const unsigned*>(p)) : *reinterpret_cast<const unsigned*>(p);
            S s2[2];
            memcpy(s2, &t, sizeof t);
            v[0] = Storage<S>::dec(s2[0]);
            v[1] = Storage<S>::dec(s2[1]);
        } else {
            const unsigned short t = RO ? __ldg(reinterpret_cast<const unsigned short*>(p))
                                        : *reinterpret_cast<const unsigned short*>(p);
            S s1;
            memcpy(&s1, &t, sizeof t);
            v[0] = Storage<S>::dec(s1);
        }
    }
}
template <typename S, bool RO>
__device__ __forceinline__ float pload1(const float* plane, int e) {
    float v[1];
    pload<S, 1, RO>(plane, e, v);
    return v[0];
}
template <typename S, int V, bool CS = false>
__device__ __forceinline__ void pstore(float* plane, int e, const float (&v)[V]) {
    if constexpr (sizeof(S) == 4) {
        if constexpr (CS) vstore_cs<V>(plane + e, v);
        else vstore<V>(plane + e, v);
    } else {
        S* p = reinterpret_cast<S*>(plane) + e;
        if constexpr (V == 4) {
            S s4[4];
#pragma unroll
            for (int k = 0; k < 4; k++) s4[k] = Storage<S>::enc(v[k]);
            uint2 t;
            memcpy(&t, s4, sizeof t);
            if constexpr (CS) __stcs(reinterpret_cast<uint2*>(p), t);
            else *reinterpret_cast<uint2*>(p) = t;
        } else if constexpr (V == 2) {
            S s2[2] = {Storage<S>::enc(v[0]), Storage<S>::enc(v[1])};
            unsigned t;
            memcpy(&t, s2, sizeof t);
            if constexpr (CS) __stcs(reinterpret_cast<unsigned*>(p), t);
            else *reinterpret_cast<unsigned*>(p) = t;
        } else {
            if constexpr (CS) {
                const S enc = Storage<S>::enc(v[0]);
                unsigned short t;
                memcpy(&t, &enc, sizeof t);
                __stcs(reinterpret_cast<unsigned short*>(p), t);
            } else {
                *p = Storage<S>::enc(v[0]);
            }
        }
    }
}
template <typename S>
__device__ __forceinline__ void pstore1(float* plane, int e, float v) {
    const float a[1] = {v};
    pstore<S, 1>(plane, e, a);
}
// rest-population offset of direction/slot d in the deviation storage
template <typename S>
__device__ __forceinline__ float rest_of(int d, const CollideParams& p) {
    return Storage<S>::deviation ? (is_face(d) ? p.wface : p.wedge) : 0.f;
}

struct Quad {
    int i, j, k0;     // cell (i, j, k0 .. k0+V-1)
    int row;          // i*ny + j
    int e0;           // element index of (row, k0)
    bool active;      // k0 < nz (the quad holds at least one cell)
};

// MUL_DIV: divide by multiply-high (Dims::by_kp16, by_ny). Measured on B200
// at 400^3: 5 % faster for the 16-bit kernels (issue-bound), but 4-11 %
// slower for the FP32 ones, whose loads the compiler then schedules worse;
// the FP32 kernels keep the hardware division sequence.
template <int V, bool MUL_DIV>
__device__ __forceinline__ Quad quad_of(const Dims& g, int nq, unsigned t) {
    Quad q;
    const unsigned total = (unsigned)g.nx * (unsigned)g.ny * (unsigned)nq;
    const unsigned tc = t < total ? t : total - 1;   // keep spare lanes on a valid quad
    // tc / nq = (tc / (16 / V)) / (kp / 16), nq = kp / V
    constexpr unsigned kShift = V == 1 ? 4 : V == 2 ? 3 : V == 4 ? 2 : 1;
    static_assert(V == 1 || V == 2 || V == 4 || V == 8, "cells per thread");
    unsigned row;
    if (MUL_DIV) {
        row = g.by_kp16.div(tc >> kShift);
        q.i = (int)g.by_ny.div(row);
    } else {
        row = tc / (unsigned)nq;
        q.i = (int)(row / (unsigned)g.ny);
    }
    const int kq = (int)(tc - row * (unsigned)nq);
    q.row = (int)row;
    q.j = (int)row - q.i * g.ny;
    q.k0 = kq * V;
    q.e0 = (int)row * g.kp + q.k0;
    q.active = t < total && q.k0 < g.nz;
    return q;
}

// FORCE = false: the cells are known to lie outside every immersed-boundary
// stencil (the outer part of a split step), so F is zero without reading the
// touched flags.
template <int V, bool LES, bool COLLIDE, bool DEV, bool FORCE = true, bool FAST = false>
__device__ __forceinline__ void collide_quad(float (&f)[NQ][V], const Quad& q, float* __restrict__ Nu,
                                             const float4* __restrict__ F, const uint32_t* __restrict__ mask,
                                             const Dims& g, const CollideParams& p, bool from_moments, float (&nu)[V]) {
    if (!COLLIDE) return;
    float fx[V], fy[V], fz[V];
    const uint32_t bits =
        FORCE ? (__ldg(mask + (size_t)q.row * g.kw + (q.k0 >> 5)) >> (q.k0 & 31)) & ((1u << V) - 1u) : 0u;
    if (bits) {
#pragma unroll
        for (int e = 0; e < V; e++) {
            const float4 v = F[q.e0 + e];
            fx[e] = v.x;
            fy[e] = v.y;
            fz[e] = v.z;
        }
#pragma unroll
        for (int e = 0; e < V; e++)
            if (!((bits >> e) & 1u)) fx[e] = fy[e] = fz[e] = 0.f;
    } else {
#pragma unroll
        for (int e = 0; e < V; e++) fx[e] = fy[e] = fz[e] = 0.f;
    }
    if (LES) vload<V>(Nu + q.e0, nu);
    if constexpr (DEV && V >= 2) {
        // 16-bit storage, several cells per thread: two cells at a time in
        // packed FP32x2 arithmetic (the state always holds populations)
#pragma unroll
        for (int e = 0; e < V; e += 2) {
            F2 qv[NQ], m[NQ];
#pragma unroll
            for (int d = 0; d < NQ; d++) qv[d] = f2(f[d][e], f[d][e + 1]);
            moments_of(qv, m);
            F2 n = LES ? f2(nu[e], nu[e + 1]) : f2(0.f);
            collide<LES, DEV, FAST>(m, f2(fx[e], fx[e + 1]), f2(fy[e], fy[e + 1]), f2(fz[e], fz[e + 1]), n, p, qv);
            if (LES) {
                nu[e] = n.v.x;
                nu[e + 1] = n.v.y;
            }
#pragma unroll
            for (int d = 0; d < NQ; d++) {
                f[d][e] = qv[d].v.x;
                f[d][e + 1] = qv[d].v.y;
            }
        }
    } else {
#pragma unroll
        for (int e = 0; e < V; e++) {
            float qv[NQ], m[NQ];
#pragma unroll
            for (int d = 0; d < NQ; d++) qv[d] = f[d][e];
            if (from_moments) {
#pragma unroll
                for (int d = 0; d < NQ; d++) m[d] = qv[d];
            } else {
                moments_of(qv, m);
            }
            float n = LES ? nu[e] : 0.f;
            collide<LES, DEV, FAST>(m, fx[e], fy[e], fz[e], n, p, qv);
            if (LES) nu[e] = n;
#pragma unroll
            for (int d = 0; d < NQ; d++) f[d][e] = qv[d];
        }
    }
}

// ---------------------------------------------------------------------------
// Residual box (16-bit storage, one cell per thread; tdlb::ResidualBox).
// A step with a box runs three launches:
//   the box launch (BOX = 2): the 32-cell chunks with a cell near the box,
//     from a list, with the residuals of their locations (the code below,
//     inlined), into a scratch array (BoxOut) -- before the plain launch
//     overwrites their populations (Esotwist) and their Nu, which the LES
//     collision reads;
//   the plain launch: every cell, without residuals;
//   k_box_commit: the box chunks' exact outputs over the plain ones, with the
//     residuals of the locations inside the box.
// The plain kernel so stays as it is. f holds the cell's 18 values in
// direction order.
// ---------------------------------------------------------------------------
// Simple: add the residuals of the source locations inside the box (x - c_d,
// or the cell itself where x - c_d is off the lattice).
__device__ __forceinline__ void box_pull_simple(const ResidualBox& rr, int i, int j, int k, const Dims& g,
                                                float (&f)[NQ][1]) {
#pragma unroll
    for (int d = 0; d < NQ; d++) {
        const int si = i - cx_of(d), sj = j - cy_of(d), sk = k - cz_of(d);
        const bool in = (unsigned)si < (unsigned)g.nx && (unsigned)sj < (unsigned)g.ny && (unsigned)sk < (unsigned)g.nz;
        const int li = in ? si : i, lj = in ? sj : j, lk = in ? sk : k;
        if (rr.contains(li, lj, lk)) f[d][0] += *rr.at(d, li, lj, lk);
    }
}
// Esotwist: slot s of cell (i, j, k) lives at (li, lj, lk); on reading, it
// holds direction EVEN ? s : s ^ 1, on writing EVEN ? s ^ 1 : s.
template <bool EVEN>
__device__ __forceinline__ void eso_location(int s, int i, int j, int k, int i1, int j1, int k1, int& li, int& lj,
                                             int& lk) {
    const int sg = EVEN ? -1 : 1;
    li = sg * cx_of(s) > 0 ? i1 : i;
    lj = sg * cy_of(s) > 0 ? j1 : j;
    lk = sg * cz_of(s) > 0 ? k1 : k;
}
template <bool EVEN>
__device__ __forceinline__ void box_read_eso(const ResidualBox& rb, int i, int j, int k, int i1, int j1, int k1,
                                             float (&f)[NQ][1]) {
#pragma unroll
    for (int s = 0; s < NQ; s++) {
        int li, lj, lk;
        eso_location<EVEN>(s, i, j, k, i1, j1, k1, li, lj, lk);
        if (rb.contains(li, lj, lk)) f[EVEN ? s : (s ^ 1)][0] += *rb.at(s, li, lj, lk);
    }
}
// ---------------------------------------------------------------------------
// Simple (A/B, pull).
//
// All loads of a thread are issued as one straight-line batch (no branch
// between them), so the 18 population fetches of a quad are in flight
// together. V = 1 pulls every population directly from x - c_d. V > 1 loads
// aligned vectors of the upstream rows and moves k-shifted values between
// lanes with shuffles; the values a lane cannot get from a neighbour (warp
// edges) and the own values the wall rule needs at row ends come from
// scalar loads issued in the same batch (in bounds for every lane; the ones
// a lane does not need hit L1).
// ---------------------------------------------------------------------------
template <typename S, int V, bool LES, bool FROM_MOMENTS, bool COLLIDE, bool FORCE = true, int BOX = 0>
__device__ __forceinline__ void simple_quad(const Planes& A, const Planes& B, float* __restrict__ Nu,
                                            const float4* __restrict__ F, const uint32_t* __restrict__ mask,
                                            const Dims& g, const CollideParams& p, unsigned t,
                                            const ResidualBox rr = ResidualBox{}, const BoxOut out = BoxOut{}) {
    static_assert(!(Storage<S>::deviation && FROM_MOMENTS), "16-bit state always holds populations");
    static_assert(BOX == 0 || (Storage<S>::deviation && V == 1), "the residual box serves 16-bit storage, one cell per thread");
    const int nq = g.kp / V;
    const Quad q = quad_of<V, sizeof(S) == 2>(g, nq, t);
    const int lane = threadIdx.x & 31;
    const int rs = g.ny * g.kp;   // elements per i step
    const bool i_lo = q.i == 0, i_hi = q.i == g.nx - 1, j_lo = q.j == 0, j_hi = q.j == g.ny - 1;
    const bool k_first = q.k0 == 0, k_last = q.k0 + V >= g.nz;
    float f[NQ][V];
    if (FROM_MOMENTS) {
#pragma unroll
        for (int d = 0; d < NQ; d++) pload<S, V, true>(A.p[d], q.e0, f[d]);
    } else if (V == 1) {
        // direct (unaligned) read-only loads: the texture path serves the
        // k-shifted rows better here than aligned loads plus lane shuffles
#pragma unroll
        for (int d = 0; d < NQ; d++) {
            const int cx = cx_of(d), cy = cy_of(d), cz = cz_of(d);
            // upstream cell x - c_d; off the lattice -> the cell keeps its own value
            const bool in = !((cx > 0 && i_lo) || (cx < 0 && i_hi) || (cy > 0 && j_lo) || (cy < 0 && j_hi) ||
                              (cz > 0 && k_first) || (cz < 0 && k_last));
            const int off = in ? -(cx * rs + cy * g.kp + cz) : 0;
            f[d][0] = pload1<S, true>(A.p[d], q.e0 + off);
        }
        if constexpr (BOX == 2) {
            // residual box: the exact deviation of every source location inside it
            if (q.active && rr.near(q.i, q.j, q.k0)) box_pull_simple(rr, q.i, q.j, q.k0, g, f);
        }
    } else {
        float hal[NQ], own[NQ];
        // batch 1: every load
#pragma unroll
        for (int d = 0; d < NQ; d++) {
            const int cx = cx_of(d), cy = cy_of(d), cz = cz_of(d);
            const bool row_ok = !((cx > 0 && i_lo) || (cx < 0 && i_hi) || (cy > 0 && j_lo) || (cy < 0 && j_hi));
            const int soff = row_ok ? -(cx * rs + cy * g.kp) : 0;
            const int src = q.e0 + soff;
            pload<S, V, true>(A.p[d], src, f[d]);
            if (cz > 0) {
                hal[d] = pload1<S, true>(A.p[d], (lane == 0 && !k_first) ? src - 1 : src);
                own[d] = (cx != 0 || cy != 0) ? pload1<S, true>(A.p[d], q.e0) : 0.f;
            } else if (cz < 0) {
                hal[d] = pload1<S, true>(A.p[d], (lane == 31 && !k_last) ? src + V : src);
                int le = g.nz - 1 - q.k0;
                le = le < 0 ? 0 : (le > V - 1 ? V - 1 : le);
                own[d] = (cx != 0 || cy != 0) ? pload1<S, true>(A.p[d], q.e0 + le) : 0.f;
            }
        }
        // batch 2: shift along k
#pragma unroll
        for (int d = 0; d < NQ; d++) {
            const int cx = cx_of(d), cy = cy_of(d), cz = cz_of(d);
            const bool row_ok = !((cx > 0 && i_lo) || (cx < 0 && i_hi) || (cy > 0 && j_lo) || (cy < 0 && j_hi));
            if (cz > 0) {                          // source k - 1
                float left = __shfl_up_sync(FULL, f[d][V - 1], 1);
                if (lane == 0) left = hal[d];
                const float own0 = (cx != 0 || cy != 0) ? own[d] : f[d][0];
                if (row_ok) {
#pragma unroll
                    for (int e = V - 1; e > 0; e--) f[d][e] = f[d][e - 1];
                    f[d][0] = k_first ? own0 : left;
                }
            } else if (cz < 0) {                   // source k + 1
                float right = __shfl_down_sync(FULL, f[d][0], 1);
                if (lane == 31) right = hal[d];
                const int le = g.nz - 1 - q.k0;   // element of the row's last cell when k_last
                float ownl = own[d];
                if (cx == 0 && cy == 0) {
#pragma unroll
                    for (int e = 0; e < V; e++)
                        if (e == le) ownl = f[d][e];
                }
                if (row_ok) {
#pragma unroll
                    for (int e = 0; e < V - 1; e++) f[d][e] = f[d][e + 1];
                    f[d][V - 1] = right;
                    if (k_last) {
#pragma unroll
                        for (int e = 0; e < V; e++)
                            if (e == le) f[d][e] = ownl;
                    }
                }
            }
        }
    }
    float nu[V];
    // 16-bit storage: approximate reciprocals and square root (measured on
    // B200 at 400^3: FP16 step 1.28 -> 1.19 ms; the Esotwist kernel, which
    // keeps IEEE rounding, measured slower with them, 1.38 -> 1.47 ms)
    collide_quad<V, LES, COLLIDE, Storage<S>::deviation, FORCE, Storage<S>::deviation>(f, q, Nu, F, mask, g,
                                                                                       p, FROM_MOMENTS, nu);
    if constexpr (BOX == 2) {
        // box launch: the exact outputs and Nu to the scratch array (entry
        // blockIdx.x * 128 + threadIdx.x of the chunk list)
        const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
        for (int d = 0; d < NQ; d++) out.v[(long long)d * out.n + o] = f[d][0];
        out.v[(long long)NQ * out.n + o] = nu[0];
        return;
    }
    if (!q.active) return;
#pragma unroll
    for (int d = 0; d < NQ; d++) pstore<S, V, sizeof(S) == 4>(B.p[d], q.e0, f[d]);
    if constexpr (sizeof(S) == 4) {
        if (COLLIDE && LES) vstore_cs<V>(Nu + q.e0, nu);
    } else {
        if (COLLIDE && LES) vstore<V>(Nu + q.e0, nu);
    }
}

// ---------------------------------------------------------------------------
// Esotwist (single buffer, in place).
//
// Slot s of cell x lives at x + o_s, o_s = max(-c_s, 0) (even) or
// max(+c_s, 0) (odd), +1 wrapping to 0; a cell reads and writes the same 18
// locations. V = 1 addresses them directly. For V > 1, where o_s has a k
// component the V locations of a quad are k0+1 .. k0+V: loads take the
// aligned vector at k0 and the next lane's first element; stores write the
// aligned vector at k0 holding the previous lane's last value, and the lane
// that owns the last cell of a warp (or of a row, where the location wraps to
// k = 0) stores that one value alone. A __syncwarp() separates every lane's
// loads from any lane's stores, so a location is always read by its owner
// before a neighbour overwrites it.
// ---------------------------------------------------------------------------
template <typename S, int V, bool LES, bool FROM_MOMENTS, bool COLLIDE, bool EVEN, bool FORCE = true, int BOX = 0>
__device__ __forceinline__ void esotwist_quad(const Planes& Q, float* __restrict__ Nu, const float4* __restrict__ F,
                                              const uint32_t* __restrict__ mask, const Dims& g, const CollideParams& p,
                                              unsigned t, const ResidualBox rb = ResidualBox{},
                                              const BoxOut out = BoxOut{}) {
    static_assert(!(Storage<S>::deviation && FROM_MOMENTS), "16-bit state always holds populations");
    static_assert(BOX == 0 || (Storage<S>::deviation && V == 1), "the residual box serves 16-bit storage, one cell per thread");
    const int nq = g.kp / V;
    const Quad q = quad_of<V, sizeof(S) == 2>(g, nq, t);
    const int lane = threadIdx.x & 31;
    const int i1 = q.i + 1 == g.nx ? 0 : q.i + 1;
    const int j1 = q.j + 1 == g.ny ? 0 : q.j + 1;
    const bool k_last = q.k0 + V >= g.nz;
    const int last_e = g.nz - 1 - q.k0;   // element holding the row's last cell (if < V)
    float f[NQ][V];
    if (V == 1) {
        // Slots with a k offset read element k + 1: every lane loads its own
        // (aligned) element k and takes k + 1 from the next lane; the lane at
        // a warp's end or a row's end loads its element itself. (Padding
        // lanes, k >= nz, load element 0 of their row: in bounds, unused.)
        const bool row_end = q.k0 == g.nz - 1;
        const bool warp_end = lane == 31;
        const int k1 = (row_end || q.k0 >= g.nz) ? 0 : q.k0 + 1;
        float v[NQ], x[NQ];
#pragma unroll
        for (int s = 0; s < NQ; s++) {
            const int sg = EVEN ? -1 : 1;
            const bool oi = sg * cx_of(s) > 0, oj = sg * cy_of(s) > 0, ok = sg * cz_of(s) > 0;
            const int base = ((oi ? i1 : q.i) * g.ny + (oj ? j1 : q.j)) * g.kp;
            v[s] = pload1<S, false>(Q.p[s], base + q.k0);
            if (ok) x[s] = (warp_end || row_end) ? pload1<S, false>(Q.p[s], base + k1) : 0.f;
        }
#pragma unroll
        for (int s = 0; s < NQ; s++) {
            const int sg = EVEN ? -1 : 1;
            const bool ok = sg * cz_of(s) > 0;
            const int d = EVEN ? s : (s ^ 1);
            if (ok) {
                const float right = __shfl_down_sync(FULL, v[s], 1);
                f[d][0] = (warp_end || row_end) ? x[s] : right;
            } else {
                f[d][0] = v[s];
            }
        }
        if constexpr (BOX == 2) {
            // residual box: the exact deviation of every location inside it
            // (slot s of this cell lives at cell (li, lj, lk))
            if (q.active && rb.near(q.i, q.j, q.k0)) box_read_eso<EVEN>(rb, q.i, q.j, q.k0, i1, j1, k1, f);
        }
    } else {
        float hal[NQ], wrap[NQ];
#pragma unroll
        for (int s = 0; s < NQ; s++) {
            const int sg = EVEN ? -1 : 1;
            const bool oi = sg * cx_of(s) > 0, oj = sg * cy_of(s) > 0, ok = sg * cz_of(s) > 0;
            const int d = EVEN ? s : (s ^ 1);
            const int base = ((oi ? i1 : q.i) * g.ny + (oj ? j1 : q.j)) * g.kp;
            pload<S, V, false>(Q.p[s], base + q.k0, f[d]);
            if (ok) {
                hal[s] = pload1<S, false>(Q.p[s], base + ((lane == 31 && !k_last) ? q.k0 + V : q.k0));
                wrap[s] = pload1<S, false>(Q.p[s], base);
            }
        }
#pragma unroll
        for (int s = 0; s < NQ; s++) {
            const int sg = EVEN ? -1 : 1;
            const bool ok = sg * cz_of(s) > 0;
            const int d = EVEN ? s : (s ^ 1);
            if (!ok) continue;
            float right = __shfl_down_sync(FULL, f[d][0], 1);
            if (lane == 31) right = hal[s];
#pragma unroll
            for (int e = 0; e < V - 1; e++) f[d][e] = f[d][e + 1];
            f[d][V - 1] = right;
            if (k_last) {                          // k = nz-1 wraps to 0
#pragma unroll
                for (int e = 0; e < V; e++)
                    if (e == last_e) f[d][e] = wrap[s];
            }
        }
    }
    __syncwarp();
    float nu[V];
    collide_quad<V, LES, COLLIDE, Storage<S>::deviation, FORCE>(f, q, Nu, F, mask, g, p, FROM_MOMENTS, nu);
    if constexpr (BOX == 2) {
        // box launch: the exact outputs, slot by slot, and Nu to the scratch
        // array (entry blockIdx.x * 128 + threadIdx.x of the chunk list)
        const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
        for (int s = 0; s < NQ; s++) out.v[(long long)s * out.n + o] = f[EVEN ? (s ^ 1) : s][0];
        out.v[(long long)NQ * out.n + o] = nu[0];
        return;
    }
    if (V == 1) {
        // Slots with a k offset write element k + 1: lane l writes element k
        // with the value of the previous lane (cell k - 1, same row), so the
        // warp's store is aligned; the lane at a warp's end or a row's end
        // writes its own element k + 1 (k = nz - 1: element 0) itself.
        const bool row_end = q.k0 == g.nz - 1;
        const bool warp_end = lane == 31;
        const int k1 = (row_end || q.k0 >= g.nz) ? 0 : q.k0 + 1;
#pragma unroll
        for (int s = 0; s < NQ; s++) {
            const int sg = EVEN ? -1 : 1;
            const bool oi = sg * cx_of(s) > 0, oj = sg * cy_of(s) > 0, ok = sg * cz_of(s) > 0;
            const int d = EVEN ? (s ^ 1) : s;
            const int base = ((oi ? i1 : q.i) * g.ny + (oj ? j1 : q.j)) * g.kp;
            if (!ok) {
                if (q.active) pstore1<S>(Q.p[s], base + q.k0, f[d][0]);
                continue;
            }
            const float left = __shfl_up_sync(FULL, f[d][0], 1);
            if (lane > 0 && q.k0 > 0 && q.k0 <= g.nz - 1 && q.active)
                pstore1<S>(Q.p[s], base + q.k0, left);
            if (q.active && (warp_end || row_end)) pstore1<S>(Q.p[s], base + k1, f[d][0]);
        }
        if (COLLIDE && LES && q.active) Nu[q.e0] = nu[0];
        return;
    }
    const bool k_first = q.k0 == 0;
#pragma unroll
    for (int s = 0; s < NQ; s++) {
        const int sg = EVEN ? -1 : 1;
        const bool oi = sg * cx_of(s) > 0, oj = sg * cy_of(s) > 0, ok = sg * cz_of(s) > 0;
        const int d = EVEN ? (s ^ 1) : s;      // direction written to slot s
        const int base = ((oi ? i1 : q.i) * g.ny + (oj ? j1 : q.j)) * g.kp;
        if (!ok) {
            if (q.active) pstore<S, V>(Q.p[s], base + q.k0, f[d]);
            continue;
        }
        float w[V];
        const float prev = __shfl_up_sync(FULL, f[d][V - 1], 1);
        w[0] = prev;
#pragma unroll
        for (int e = 1; e < V; e++) w[e] = f[d][e - 1];
        if (!q.active) continue;
        if (lane != 0 && !k_first) {
            pstore<S, V>(Q.p[s], base + q.k0, w);
        } else {
#pragma unroll
            for (int e = 1; e < V; e++) pstore1<S>(Q.p[s], base + q.k0 + e, w[e]);
        }
        if (k_last) {                          // the wrap location of k = nz-1
#pragma unroll
            for (int e = 0; e < V; e++)
                if (e == last_e) pstore1<S>(Q.p[s], base, f[d][e]);
        } else if (lane == 31) {
            pstore1<S>(Q.p[s], base + q.k0 + V, f[d][V - 1]);
        }
    }
    if (COLLIDE && LES && q.active) vstore<V>(Nu + q.e0, nu);
}


// Split step (one cell per thread). The immersed-boundary pass of a step
// touches a thin set of cells, so a step can run as two launches over
// 32-cell chunks of the flat (row, k) index, one warp per listed chunk:
//   PART 1 (outer): the chunks outside the zone; F is zero there, so these
//     warps read neither F nor the touched flags;
//   PART 2 (inner): the chunks of the zone.
// PART 0 runs every cell. The outer launch of a step depends on the previous
// step's populations only, so it can run while the previous forcing pass is
// still in flight.
// L2 prefetch ahead of a full launch's walk. CTA b covers elements
// [128 V b, 128 V (b + 1)) of the flat row * kp + k index. Every
// kPrefetchTiles-th CTA, as it starts, has NQ + 1 of its threads issue one
// cp.async.bulk.prefetch.L2 each, for the kPrefetchTiles tiles that begin
// `ahead` CTAs later: the span of plane d the pull reads (Simple: the tiles
// shifted by -c_d; Esotwist: shifted to the row of slot d's location) and
// Nu's span (LES). With `ahead` one wave of resident CTAs, the populations
// are in L2 when those CTAs load them, so the loads -- whose latency bounds
// the kernels at their occupancy -- wait for the L2, not for the DRAM.
// Measured on B200 at 400^3 (step kernel alone, ms): FP32 Simple 1.530 ->
// 1.483, FP32 Esotwist 1.677 -> 1.496, 16-bit Simple (four cells per thread)
// 1.26 -> 1.08, 16-bit Esotwist (two cells per thread) 1.55 -> 1.35.
// Spans are clamped to the plane and rounded out to 16 bytes (planes start
// 16-byte aligned and hold a multiple of 64 elements); a prefetch changes no
// result.
constexpr int kPrefetchTiles = 8;
__device__ __forceinline__ void prefetch_span(const void* base, int es, long long plane, long long e0,
                                              long long e1) {
    e0 = e0 < 0 ? 0 : e0;
    e1 = e1 > plane ? plane : e1;
    if (e0 >= e1) return;
    const uintptr_t lo = (reinterpret_cast<uintptr_t>(base) + (uintptr_t)(e0 * es)) & ~(uintptr_t)15;
    const uintptr_t hi = (reinterpret_cast<uintptr_t>(base) + (uintptr_t)(e1 * es) + 15) & ~(uintptr_t)15;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(lo), "r"((unsigned)(hi - lo)) : "memory");
}
template <typename S, int V, bool LES, bool ESO, bool EVEN>
__device__ __forceinline__ void prefetch_ahead(const Planes& A, const float* Nu, const Dims& g, int ahead) {
    const int d = (int)threadIdx.x;
    if (ahead <= 0 || d >= (LES ? NQ + 1 : NQ) || blockIdx.x % kPrefetchTiles) return;
    constexpr long long tile = 128LL * V;
    const long long e0 = ((long long)blockIdx.x + ahead) * tile, e1 = e0 + kPrefetchTiles * tile;
    if (e0 >= g.rows() * g.kp) return;
    if (d == NQ) return prefetch_span(Nu, 4, g.plane, e0, e1);
    const long long rs = (long long)g.ny * g.kp;
    long long sh;
    if (ESO) {
        const int sg = EVEN ? -1 : 1;
        sh = (sg * cx_of(d) > 0 ? rs : 0) + (sg * cy_of(d) > 0 ? g.kp : 0);
    } else {
        sh = -(cx_of(d) * rs + cy_of(d) * g.kp);
    }
    // one element either side: the k +- 1 neighbours
    prefetch_span(A.p[d], (int)sizeof(S), g.plane, e0 + sh - 1, e1 + sh + 1);
}

template <int PART>
__device__ __forceinline__ bool part_thread(const StepPart& part, unsigned& t) {
    t = blockIdx.x * blockDim.x + threadIdx.x;
    if (PART != 0) {
        const unsigned w = t >> 5;
        if (w >= (unsigned)part.count) return false;   // whole warps
        t = (unsigned)__ldg(part.chunks + w) * kSplitChunk + (threadIdx.x & 31u);
    }
    return true;
}

template <typename S, int V, bool LES, bool FROM_MOMENTS, bool COLLIDE, int PART = 0, int BOX = 0>
__global__ void __launch_bounds__(128, 4) k_step_simple(Planes A, Planes B, float* __restrict__ Nu,
                                                       const float4* __restrict__ F, const uint32_t* __restrict__ mask,
                                                       Dims g, CollideParams p, StepPart part, ResidualBox rr,
                                                       BoxOut out) {
    static_assert(PART == 0 || V == 1, "split steps run one cell per thread");
    static_assert(BOX != 2 || PART != 0, "the box path runs a chunk list");
    if constexpr (PART == 0 && COLLIDE && !FROM_MOMENTS)
        prefetch_ahead<S, V, LES, false, false>(A, Nu, g, part.l2_ahead);
    unsigned t;
    if (!part_thread<PART>(part, t)) return;   // whole warps
    simple_quad<S, V, LES, FROM_MOMENTS, COLLIDE, PART != 1, BOX>(A, B, Nu, F, mask, g, p, t, rr, out);
}

// Resident 128-thread blocks per SM the Esotwist kernel is built for: the
// register cap that follows (64 at one cell per thread) keeps enough loads in
// flight; measured on B200 at 400^3, 8 blocks beat 4 by about 5%.
template <int V>
constexpr int kEsotwistBlocksPerSM = V == 1 ? 8 : (V == 2 ? 6 : 4);

template <typename S, int V, bool LES, bool FROM_MOMENTS, bool COLLIDE, bool EVEN, int PART = 0, int BOX = 0>
__global__ void __launch_bounds__(128, BOX == 2 ? 4 : kEsotwistBlocksPerSM<V>) k_step_esotwist(Planes Q, float* __restrict__ Nu,
                                                         const float4* __restrict__ F, const uint32_t* __restrict__ mask,
                                                         Dims g, CollideParams p, StepPart part, ResidualBox rb,
                                                         BoxOut out) {
    static_assert(PART == 0 || V == 1, "split steps run one cell per thread");
    static_assert(BOX != 2 || PART != 0, "the box path runs a chunk list");
    if constexpr (PART == 0 && COLLIDE && !FROM_MOMENTS)
        prefetch_ahead<S, V, LES, true, EVEN>(Q, Nu, g, part.l2_ahead);
    unsigned t;
    if (!part_thread<PART>(part, t)) return;   // whole warps
    esotwist_quad<S, V, LES, FROM_MOMENTS, COLLIDE, EVEN, PART != 1, BOX>(Q, Nu, F, mask, g, p, t, rb, out);
}

// After the plain launch of a step with a residual box: every cell of the box
// chunks takes the outputs its box launch computed (entry blockIdx.x * 128 +
// threadIdx.x of `out`): Simple stores direction d to its own cell of plane d
// of Q (the destination buffer), Esotwist slot s to the slot's location;
// the residuals of the locations inside the box (rb: the destination's set)
// and Nu go with them.
template <typename S, bool SIMPLE, bool EVEN>
__global__ void __launch_bounds__(128) k_box_commit(Planes Q, float* __restrict__ Nu, Dims g, StepPart part,
                                                    ResidualBox rb, BoxOut out, int les) {
    unsigned t;
    if (!part_thread<2>(part, t)) return;
    const Quad q = quad_of<1, true>(g, g.kp, t);
    if (!q.active) return;
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i1 = q.i + 1 == g.nx ? 0 : q.i + 1;
    const int j1 = q.j + 1 == g.ny ? 0 : q.j + 1;
    const int k1 = q.k0 + 1 == g.nz ? 0 : q.k0 + 1;
#pragma unroll
    for (int s = 0; s < NQ; s++) {
        int li = q.i, lj = q.j, lk = q.k0;
        if (!SIMPLE) eso_location<EVEN>(s, q.i, q.j, q.k0, i1, j1, k1, li, lj, lk);
        const float v = out.v[(long long)s * out.n + o];
        const S enc = Storage<S>::enc(v);
        reinterpret_cast<S*>(Q.p[s])[((long long)li * g.ny + lj) * g.kp + lk] = enc;
        if (rb.contains(li, lj, lk)) *rb.at(s, li, lj, lk) = v - Storage<S>::dec(enc);
    }
    if (les) Nu[q.e0] = out.v[(long long)NQ * out.n + o];
}

// Moments of the current state at every interior cell (what the reference's
// Q holds after moments()), written to 18 FP32 output planes of the same
// layout. mode: 0 = Simple populations (pull), 1 = moments (own cell),
// 2 = Esotwist populations (read map, parity `even`), 3 = Esotwist moments.
template <typename S>
__device__ __forceinline__ void state_moments18(const Planes& A, const Dims& g, int mode, int even, const CollideParams& p,
                                                int i, int j, int k, float (&m)[NQ],
                                                const ResidualBox rb = ResidualBox{}) {
    const int e = (int)(((long long)i * g.ny + j) * g.kp + k);
    float q[NQ];
    if (mode <= 1) {
#pragma unroll
        for (int d = 0; d < NQ; d++) {
            int src = e;
            if (mode == 0) {
                const int si = i - cx_of(d), sj = j - cy_of(d), sk = k - cz_of(d);
                const bool in = (unsigned)si < (unsigned)g.nx && (unsigned)sj < (unsigned)g.ny && (unsigned)sk < (unsigned)g.nz;
                if (in) src = (si * g.ny + sj) * g.kp + sk;
                if (Storage<S>::deviation && rb.on()) {
                    const int li = in ? si : i, lj = in ? sj : j, lk = in ? sk : k;
                    if (rb.contains(li, lj, lk)) {
                        q[d] = pload1<S, false>(A.p[d], src) + *rb.at(d, li, lj, lk) + rest_of<S>(d, p);
                        continue;
                    }
                }
            }
            q[d] = pload1<S, false>(A.p[d], src) + (mode == 0 ? rest_of<S>(d, p) : 0.f);
        }
    } else {
        const int i1 = i + 1 == g.nx ? 0 : i + 1, j1 = j + 1 == g.ny ? 0 : j + 1, k1 = k + 1 == g.nz ? 0 : k + 1;
#pragma unroll
        for (int d = 0; d < NQ; d++) {
            const int s = even ? d : (d ^ 1);
            const int sg = even ? -1 : 1;
            const bool oi = sg * cx_of(s) > 0, oj = sg * cy_of(s) > 0, ok = sg * cz_of(s) > 0;
            q[d] = pload1<S, false>(A.p[s], ((oi ? i1 : i) * g.ny + (oj ? j1 : j)) * g.kp + (ok ? k1 : k)) +
                   (mode == 2 ? rest_of<S>(d, p) : 0.f);
            if (Storage<S>::deviation && mode == 2 && rb.on() && rb.contains(oi ? i1 : i, oj ? j1 : j, ok ? k1 : k))
                q[d] += *rb.at(s, oi ? i1 : i, oj ? j1 : j, ok ? k1 : k);
        }
    }
    if (mode == 0 || mode == 2) moments_of(q, m);
    else {
#pragma unroll
        for (int d = 0; d < NQ; d++) m[d] = q[d];
    }
}

template <typename S>
__global__ void __launch_bounds__(256) k_state_moments(Planes A, Planes M, Dims g, int mode, int even, CollideParams p,
                                                       ResidualBox rb) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = g.rows() * g.nz;
    if (t >= total) return;
    const int k = (int)(t % g.nz);
    const long long row = t / g.nz;
    const int j = (int)(row % g.ny);
    const int i = (int)(row / g.ny);
    float m[NQ];
    state_moments18<S>(A, g, mode, even, p, i, j, k, m, rb);
    const long long e = row * g.kp + k;
#pragma unroll
    for (int d = 0; d < NQ; d++) M.p[d][e] = m[d];
}

}  // namespace tdlb
