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

// ---------------------------------------------------------------------------
// Thread mapping shared by both schemes: V consecutive cells of one row per
// thread ("quad"), quads numbered row-major over (row, kq); a warp covers 32
// consecutive quads, so neighbouring lanes hold neighbouring cells of the
// same row except at row ends (where the wall rule or the periodic wrap
// applies anyway). V in {1, 2, 4}; populations move as float/float2/float4.
// ---------------------------------------------------------------------------
constexpr unsigned FULL = 0xffffffffu;

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
// plain (coherent) loads for the in-place Esotwist buffer
template <int V>
__device__ __forceinline__ void vload_rw(const float* p, float (&v)[V]) {
    if constexpr (V == 4) {
        const float4 t = *reinterpret_cast<const float4*>(p);
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else if constexpr (V == 2) {
        const float2 t = *reinterpret_cast<const float2*>(p);
        v[0] = t.x; v[1] = t.y;
    } else {
        v[0] = *p;
    }
}
template <int V>
__device__ __forceinline__ void vstore(float* p, const float (&v)[V]) {
    if constexpr (V == 4) *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    else if constexpr (V == 2) *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
    else *p = v[0];
}

struct Quad {
    int i, j, k0;     // cell (i, j, k0 .. k0+V-1)
    int row;          // i*ny + j
    int e0;           // element index of (row, k0)
    bool active;      // k0 < nz (the quad holds at least one cell)
};

template <int V>
__device__ __forceinline__ Quad quad_of(const Dims& g, int nq) {
    Quad q;
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned total = (unsigned)g.nx * (unsigned)g.ny * (unsigned)nq;
    const unsigned tc = t < total ? t : total - 1;   // keep spare lanes on a valid quad
    const unsigned row = tc / (unsigned)nq;
    const int kq = (int)(tc - row * (unsigned)nq);
    q.row = (int)row;
    q.i = (int)(row / (unsigned)g.ny);
    q.j = (int)row - q.i * g.ny;
    q.k0 = kq * V;
    q.e0 = (int)row * g.kp + q.k0;
    q.active = t < total && q.k0 < g.nz;
    return q;
}

template <int V, bool LES, bool COLLIDE>
__device__ __forceinline__ void collide_quad(float (&f)[NQ][V], const Quad& q, float* __restrict__ Nu,
                                             const float* __restrict__ Fx, const float* __restrict__ Fy,
                                             const float* __restrict__ Fz, const uint32_t* __restrict__ mask,
                                             const Dims& g, const CollideParams& p, bool from_moments, float (&nu)[V]) {
    if (!COLLIDE) return;
    float fx[V], fy[V], fz[V];
    const uint32_t bits = (__ldg(mask + (size_t)q.row * g.kw + (q.k0 >> 5)) >> (q.k0 & 31)) & ((1u << V) - 1u);
    if (bits) {
        vload<V>(Fx + q.e0, fx);
        vload<V>(Fy + q.e0, fy);
        vload<V>(Fz + q.e0, fz);
#pragma unroll
        for (int e = 0; e < V; e++)
            if (!((bits >> e) & 1u)) fx[e] = fy[e] = fz[e] = 0.f;
    } else {
#pragma unroll
        for (int e = 0; e < V; e++) fx[e] = fy[e] = fz[e] = 0.f;
    }
    if (LES) vload<V>(Nu + q.e0, nu);
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
        collide<LES>(m, fx[e], fy[e], fz[e], n, p, qv);
        if (LES) nu[e] = n;
#pragma unroll
        for (int d = 0; d < NQ; d++) f[d][e] = qv[d];
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
template <int V, bool LES, bool FROM_MOMENTS, bool COLLIDE>
__global__ void __launch_bounds__(128, 4) k_step_simple(Planes A, Planes B, float* __restrict__ Nu,
                                                       const float* __restrict__ Fx, const float* __restrict__ Fy,
                                                       const float* __restrict__ Fz, const uint32_t* __restrict__ mask,
                                                       Dims g, CollideParams p) {
    const int nq = g.kp / V;
    const Quad q = quad_of<V>(g, nq);
    const int lane = threadIdx.x & 31;
    const int rs = g.ny * g.kp;   // elements per i step
    const bool i_lo = q.i == 0, i_hi = q.i == g.nx - 1, j_lo = q.j == 0, j_hi = q.j == g.ny - 1;
    const bool k_first = q.k0 == 0, k_last = q.k0 + V >= g.nz;
    float f[NQ][V];
    if (FROM_MOMENTS) {
#pragma unroll
        for (int d = 0; d < NQ; d++) vload<V>(A.p[d] + q.e0, f[d]);
    } else if (V == 1) {
#pragma unroll
        for (int d = 0; d < NQ; d++) {
            const int cx = cx_of(d), cy = cy_of(d), cz = cz_of(d);
            // upstream cell x - c_d; off the lattice -> the cell keeps its own value
            const bool in = !((cx > 0 && i_lo) || (cx < 0 && i_hi) || (cy > 0 && j_lo) || (cy < 0 && j_hi) ||
                              (cz > 0 && k_first) || (cz < 0 && k_last));
            const int off = in ? -(cx * rs + cy * g.kp + cz) : 0;
            f[d][0] = __ldg(A.p[d] + q.e0 + off);
        }
    } else {
        float hal[NQ], own[NQ];
        // batch 1: every load
#pragma unroll
        for (int d = 0; d < NQ; d++) {
            const int cx = cx_of(d), cy = cy_of(d), cz = cz_of(d);
            const bool row_ok = !((cx > 0 && i_lo) || (cx < 0 && i_hi) || (cy > 0 && j_lo) || (cy < 0 && j_hi));
            const int soff = row_ok ? -(cx * rs + cy * g.kp) : 0;
            const float* src = A.p[d] + q.e0 + soff;
            vload<V>(src, f[d]);
            if (cz > 0) {
                hal[d] = __ldg((lane == 0 && !k_first) ? src - 1 : src);
                own[d] = (cx != 0 || cy != 0) ? __ldg(A.p[d] + q.e0) : 0.f;
            } else if (cz < 0) {
                hal[d] = __ldg((lane == 31 && !k_last) ? src + V : src);
                int le = g.nz - 1 - q.k0;
                le = le < 0 ? 0 : (le > V - 1 ? V - 1 : le);
                own[d] = (cx != 0 || cy != 0) ? __ldg(A.p[d] + q.e0 + le) : 0.f;
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
    collide_quad<V, LES, COLLIDE>(f, q, Nu, Fx, Fy, Fz, mask, g, p, FROM_MOMENTS, nu);
    if (!q.active) return;
#pragma unroll
    for (int d = 0; d < NQ; d++) vstore<V>(B.p[d] + q.e0, f[d]);
    if (COLLIDE && LES) vstore<V>(Nu + q.e0, nu);
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
template <int V, bool LES, bool FROM_MOMENTS, bool COLLIDE, bool EVEN>
__global__ void __launch_bounds__(128, 4) k_step_esotwist(Planes Q, float* __restrict__ Nu,
                                                         const float* __restrict__ Fx, const float* __restrict__ Fy,
                                                         const float* __restrict__ Fz, const uint32_t* __restrict__ mask,
                                                         Dims g, CollideParams p) {
    const int nq = g.kp / V;
    const Quad q = quad_of<V>(g, nq);
    const int lane = threadIdx.x & 31;
    const int i1 = q.i + 1 == g.nx ? 0 : q.i + 1;
    const int j1 = q.j + 1 == g.ny ? 0 : q.j + 1;
    const bool k_last = q.k0 + V >= g.nz;
    const int last_e = g.nz - 1 - q.k0;   // element holding the row's last cell (if < V)
    float f[NQ][V];
    if (V == 1) {
        const int k1 = q.k0 + 1 == g.nz ? 0 : q.k0 + 1;
#pragma unroll
        for (int s = 0; s < NQ; s++) {
            const int sg = EVEN ? -1 : 1;
            const bool oi = sg * cx_of(s) > 0, oj = sg * cy_of(s) > 0, ok = sg * cz_of(s) > 0;
            const int d = EVEN ? s : (s ^ 1);
            f[d][0] = Q.p[s][((oi ? i1 : q.i) * g.ny + (oj ? j1 : q.j)) * g.kp + (ok ? k1 : q.k0)];
        }
    } else {
        float hal[NQ], wrap[NQ];
#pragma unroll
        for (int s = 0; s < NQ; s++) {
            const int sg = EVEN ? -1 : 1;
            const bool oi = sg * cx_of(s) > 0, oj = sg * cy_of(s) > 0, ok = sg * cz_of(s) > 0;
            const int d = EVEN ? s : (s ^ 1);
            const float* base = Q.p[s] + ((oi ? i1 : q.i) * g.ny + (oj ? j1 : q.j)) * g.kp;
            vload_rw<V>(base + q.k0, f[d]);
            if (ok) {
                hal[s] = base[(lane == 31 && !k_last) ? q.k0 + V : q.k0];
                wrap[s] = base[0];
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
    collide_quad<V, LES, COLLIDE>(f, q, Nu, Fx, Fy, Fz, mask, g, p, FROM_MOMENTS, nu);
    if (V == 1) {
        if (!q.active) return;
        const int k1 = q.k0 + 1 == g.nz ? 0 : q.k0 + 1;
#pragma unroll
        for (int s = 0; s < NQ; s++) {
            const int sg = EVEN ? -1 : 1;
            const bool oi = sg * cx_of(s) > 0, oj = sg * cy_of(s) > 0, ok = sg * cz_of(s) > 0;
            const int d = EVEN ? (s ^ 1) : s;
            Q.p[s][((oi ? i1 : q.i) * g.ny + (oj ? j1 : q.j)) * g.kp + (ok ? k1 : q.k0)] = f[d][0];
        }
        if (COLLIDE && LES) Nu[q.e0] = nu[0];
        return;
    }
    const bool k_first = q.k0 == 0;
#pragma unroll
    for (int s = 0; s < NQ; s++) {
        const int sg = EVEN ? -1 : 1;
        const bool oi = sg * cx_of(s) > 0, oj = sg * cy_of(s) > 0, ok = sg * cz_of(s) > 0;
        const int d = EVEN ? (s ^ 1) : s;      // direction written to slot s
        float* base = Q.p[s] + ((oi ? i1 : q.i) * g.ny + (oj ? j1 : q.j)) * g.kp;
        if (!ok) {
            if (q.active) vstore<V>(base + q.k0, f[d]);
            continue;
        }
        float w[V];
        const float prev = __shfl_up_sync(FULL, f[d][V - 1], 1);
        w[0] = prev;
#pragma unroll
        for (int e = 1; e < V; e++) w[e] = f[d][e - 1];
        if (!q.active) continue;
        if (lane != 0 && !k_first) {
            vstore<V>(base + q.k0, w);
        } else {
#pragma unroll
            for (int e = 1; e < V; e++) base[q.k0 + e] = w[e];
        }
        if (k_last) {                          // the wrap location of k = nz-1
#pragma unroll
            for (int e = 0; e < V; e++)
                if (e == last_e) base[0] = f[d][e];
        } else if (lane == 31) {
            base[q.k0 + V] = f[d][V - 1];
        }
    }
    if (COLLIDE && LES && q.active) vstore<V>(Nu + q.e0, nu);
}

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

template <int V>
static cudaError_t launch_simple_v(const StepArgs& a, cudaStream_t st) {
    const long long nquads = a.g.rows() * (a.g.kp / V);
    const dim3 grid(blocks_for(nquads, 128)), block(128);
#define TDLB_SIMPLE(LES, FM, COL) k_step_simple<V, LES, FM, COL><<<grid, block, 0, st>>>(a.A, a.B, a.Nu, a.Fx, a.Fy, a.Fz, a.mask, a.g, a.p)
    if (!a.collide) TDLB_SIMPLE(false, false, false);
    else if (a.les) { if (a.from_moments) TDLB_SIMPLE(true, true, true); else TDLB_SIMPLE(true, false, true); }
    else { if (a.from_moments) TDLB_SIMPLE(false, true, true); else TDLB_SIMPLE(false, false, true); }
#undef TDLB_SIMPLE
    return cudaGetLastError();
}

template <int V>
static cudaError_t launch_esotwist_v(const StepArgs& a, cudaStream_t st) {
    const long long nquads = a.g.rows() * (a.g.kp / V);
    const dim3 grid(blocks_for(nquads, 128)), block(128);
#define TDLB_ESO(LES, FM, COL)                                                                                        \
    do {                                                                                                              \
        if (a.even) k_step_esotwist<V, LES, FM, COL, true><<<grid, block, 0, st>>>(a.A, a.Nu, a.Fx, a.Fy, a.Fz, a.mask, a.g, a.p); \
        else k_step_esotwist<V, LES, FM, COL, false><<<grid, block, 0, st>>>(a.A, a.Nu, a.Fx, a.Fy, a.Fz, a.mask, a.g, a.p); \
    } while (0)
    if (!a.collide) TDLB_ESO(false, false, false);
    else if (a.les) { if (a.from_moments) TDLB_ESO(true, true, true); else TDLB_ESO(true, false, true); }
    else { if (a.from_moments) TDLB_ESO(false, true, true); else TDLB_ESO(false, false, true); }
#undef TDLB_ESO
    return cudaGetLastError();
}

cudaError_t launch_step_simple(const StepArgs& a, cudaStream_t st) {
    switch (a.vec) {
        case 1: return launch_simple_v<1>(a, st);
        case 2: return launch_simple_v<2>(a, st);
        default: return launch_simple_v<4>(a, st);
    }
}

cudaError_t launch_step_esotwist(const StepArgs& a, cudaStream_t st) {
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

cudaError_t launch_state_moments(Planes A, Planes M, const Dims& g, int mode, int even, cudaStream_t st) {
    k_state_moments<<<blocks_for(g.rows() * g.nz, 256), 256, 0, st>>>(A, M, g, mode, even);
    return cudaGetLastError();
}

}  // namespace tdlb
