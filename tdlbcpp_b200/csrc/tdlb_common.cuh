// Shared device definitions for the B200 lattice Boltzmann time step.
//
// Lattice: D3Q19-style with 18 moving populations and no rest population
// (tdlbcpp/src/Header.h:35, :64-100). Population slot d has lattice vector
// (CX[d], CY[d], CZ[d]); opposite(d) = d ^ 1.
//
// Device layout (one lattice = one "tank"):
//   * interior cells only (the reference's ghost layer is never read by the
//     step, so it is not stored);
//   * cell (i, j, k), 0 <= i < nx, 0 <= j < ny, 0 <= k < nz, row r = i*ny + j,
//     element e = r*kp + k, kp = row pitch = nz rounded up to kRowPitch
//     elements (16: every FP32 row starts on a 64-byte boundary);
//   * 18 population planes (SoA), each `plane` elements long and 256-byte
//     aligned, addressed through an 18-pointer table;
//   * F as one float4 (Fx, Fy, Fz, unused) per element -- the forcing pass
//     reads and writes it at scattered stencil cells, where one 16-byte
//     access replaces three 4-byte ones in three planes --, Nu as one plane,
//     and the IBM "touched" flags as one bit per cell: word r*kw + k/32,
//     bit k%32.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace tdlb {

constexpr int NQ = 18;

// Lattice vectors in slot order Q01..Q18 (Header.h:70-100).
__host__ __device__ constexpr int cx_of(int d) {
    return d == 0 ? 1 : d == 1 ? -1 : d == 6 ? 1 : d == 7 ? -1 : d == 8 ? 1 : d == 9 ? -1
         : d == 12 ? 1 : d == 13 ? -1 : d == 14 ? 1 : d == 15 ? -1 : 0;
}
__host__ __device__ constexpr int cy_of(int d) {
    return d == 2 ? 1 : d == 3 ? -1 : d == 6 ? 1 : d == 7 ? -1 : d == 10 ? 1 : d == 11 ? -1
         : d == 12 ? -1 : d == 13 ? 1 : d == 16 ? 1 : d == 17 ? -1 : 0;
}
__host__ __device__ constexpr int cz_of(int d) {
    return d == 4 ? 1 : d == 5 ? -1 : d == 8 ? 1 : d == 9 ? -1 : d == 10 ? 1 : d == 11 ? -1
         : d == 14 ? -1 : d == 15 ? 1 : d == 16 ? -1 : d == 17 ? 1 : 0;
}

// Division of n < 2^31 by a fixed divisor d >= 1 as one multiply-high, an
// add and a shift (Granlund and Montgomery, "Division by invariant integers
// using multiplication", PLDI 1994, the round-up method with l = ceil(log2 d)
// and m = floor(2^32 (2^l - d) / d) + 1): q = (mulhi(n, m) + n) >> l.
struct DivU31 {
    unsigned mul, shift;
    __device__ __forceinline__ unsigned div(unsigned n) const { return (__umulhi(n, mul) + n) >> shift; }
};
__host__ inline DivU31 make_div_u31(unsigned d) {
    unsigned l = 0;
    while ((1ull << l) < d) l++;
    DivU31 r;
    r.mul = (unsigned)((((1ull << l) - d) << 32) / d + 1);
    r.shift = l;
    return r;
}

// Row pitch granule in elements. 16 FP32 elements = 64-byte rows. 32 (every
// FP32 row on its own 128-byte L2 line) measured 4 % slower on B200 at 400^3
// (FP32 Simple step kernel 1.600 -> 1.664 ms, Esotwist 1.670 -> 1.737 ms,
// FP16 alike): the step's time follows the padded row length (416 against
// 400 elements) and the line alignment buys nothing back. (Build parameter.)
#ifndef TDLB_ROW_PITCH
#define TDLB_ROW_PITCH 16
#endif
constexpr int kRowPitch = TDLB_ROW_PITCH;
static_assert(kRowPitch % 16 == 0, "the row pitch is a multiple of 16 elements");

struct Dims {
    int nx, ny, nz;     // interior extent
    int kp;             // row pitch in elements (multiple of kRowPitch)
    int kw;             // bitmask words per row
    long long plane;    // elements per population plane (multiple of 64)
    DivU31 by_ny;       // n / ny
    DivU31 by_kp16;     // n / (kp / 16)
    __host__ __device__ long long rows() const { return (long long)nx * ny; }
};

// Extent, row pitch, plane size and divisors of an nx x ny x nz lattice.
__host__ inline Dims make_dims(int nx, int ny, int nz) {
    Dims g{};
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.kp = (nz + kRowPitch - 1) / kRowPitch * kRowPitch;
    g.kw = (g.kp + 31) / 32;
    g.plane = ((long long)nx * ny * g.kp + 63) / 64 * 64;
    g.by_ny = make_div_u31((unsigned)ny);
    g.by_kp16 = make_div_u31((unsigned)(g.kp / 16));
    return g;
}

// 18 plane base pointers of one population buffer. With 16-bit storage the
// pointers address __half / __nv_bfloat16 elements (kernels cast them).
struct Planes {
    float* p[NQ];
};

// Population storage. FP32 stores f itself; the 16-bit forms store the
// deviation f - w_d * rho0 from the rest weight of the direction's class
// (w = 1/12 for faces, 1/24 for edges: the populations the Eggels-Somers
// inverse filter gives at rest), and all arithmetic stays FP32.
enum StorageKind { STORE_F32 = 0, STORE_F16 = 1, STORE_BF16 = 2 };

template <typename S>
struct Storage;
template <>
struct Storage<float> {
    static constexpr bool deviation = false;
    __device__ __forceinline__ static float dec(float x) { return x; }
    __device__ __forceinline__ static float enc(float x) { return x; }
};
template <>
struct Storage<__half> {
    static constexpr bool deviation = true;
    __device__ __forceinline__ static float dec(__half x) { return __half2float(x); }
    __device__ __forceinline__ static __half enc(float x) { return __float2half_rn(x); }
};
template <>
struct Storage<__nv_bfloat16> {
    static constexpr bool deviation = true;
    __device__ __forceinline__ static float dec(__nv_bfloat16 x) { return __bfloat162float(x); }
    __device__ __forceinline__ static __nv_bfloat16 enc(float x) { return __float2bfloat16_rn(x); }
};
// Calls f with a value of the storage type of `kind` (float, __half,
// __nv_bfloat16), so that one generic lambda launches the matching kernel
// instance.
template <typename F>
inline auto with_storage(int kind, F&& f) {
    switch (kind) {
        case STORE_F16: return f(__half());
        case STORE_BF16: return f(__nv_bfloat16());
        default: return f(float());
    }
}

// rest population of slot/direction d for the deviation storage
__host__ __device__ constexpr bool is_face(int d) { return d < 6; }

// Residual box of the 16-bit storage: for every population location (cell,
// slot) inside the box [i0, i0+bx) x [j0, j0+by) x [k0, k0+bz) the FP32
// residual of its 16-bit rounding is kept as well, so that such a location
// holds its deviation exactly: dec(stored) + residual. Placed over the
// impeller's swept volume it keeps the stirred flow's most sensitive cells at
// FP32 storage precision (there the 16-bit rounding dominates the velocity
// error against FP64). res == nullptr: no box. Residual plane s (one per
// slot) starts at res + s * n.
struct ResidualBox {
    float* res = nullptr;
    long long n = 0;
    int i0 = 0, j0 = 0, k0 = 0, bx = 0, by = 0, bz = 0;
    __host__ __device__ bool on() const { return res != nullptr; }
    __device__ __forceinline__ bool contains(int i, int j, int k) const {
        return (unsigned)(i - i0) < (unsigned)bx && (unsigned)(j - j0) < (unsigned)by && (unsigned)(k - k0) < (unsigned)bz;
    }
    // the 3x3x3 neighbourhood of (i, j, k) meets the box (geometry only) ...
    __host__ __device__ __forceinline__ bool around(int i, int j, int k) const {
        return (unsigned)(i - i0 + 1) < (unsigned)(bx + 2) && (unsigned)(j - j0 + 1) < (unsigned)(by + 2) &&
               (unsigned)(k - k0 + 1) < (unsigned)(bz + 2);
    }
    // ... of a set box
    __host__ __device__ __forceinline__ bool near(int i, int j, int k) const { return res && around(i, j, k); }
    __device__ __forceinline__ float* at(int s, int i, int j, int k) const {
        return res + (long long)s * n + ((long long)(i - i0) * by + (j - j0)) * bz + (k - k0);
    }
};

// Scratch outputs of an Esotwist box launch: 19 arrays (the 18 slots' values
// and Nu) of n entries, one entry per thread of the launch.
struct BoxOut {
    float* v = nullptr;
    long long n = 0;
};

// Collision constants (FlowParams fields the step reads).
struct CollideParams {
    float nu;       // molecular viscosity
    float b0, c0;   // 1/(1+6 nu), 1-6 nu  (CollisionEgglesSomers.hpp:31-32)
    float cs0sq;    // Smagorinsky cs0^2
    float g3;       // third-order relaxation
    float wface;    // rest populations rho0/12 and rho0/24 (16-bit storage offsets)
    float wedge;
    float rho0;     // 6 wface + 12 wedge: the density of the rest populations
};

// Rest populations of the deviation storage for initial density rho0.
__host__ inline void set_rest(CollideParams& p, double rho0) {
    p.wface = (float)(rho0 / 12.0);
    p.wedge = (float)(rho0 / 24.0);
    p.rho0 = (float)(6.0 * (double)p.wface + 12.0 * (double)p.wedge);
}

__host__ inline CollideParams make_collide_params(double nu, double cs0, double g3) {
    CollideParams p;
    p.nu = (float)nu;
    p.b0 = (float)(1.0 / (1.0 + 6.0 * (double)(float)nu));
    p.c0 = (float)(1.0 - 6.0 * (double)(float)nu);
    p.cs0sq = (float)cs0 * (float)cs0;
    p.g3 = (float)g3;
    set_rest(p, 1.0);
    return p;
}

// ---------------------------------------------------------------------------
// Two cells' values in one register pair, computed with Blackwell's packed
// FP32x2 instructions (fma/add/mul .rn.f32x2: one instruction for both
// lanes, each lane rounded as the scalar IEEE operation). The moment and
// collision templates below take T = float (one cell) or T = F2 (two cells);
// with T = float they are the plain scalar code. The packed form serves the
// 16-bit storage kernels, which are bound by instruction issue rather than
// by memory; products and sums are not contracted into FMAs there except
// where madd() asks for one, so its rounding differs from the scalar form's
// by FP32 ulps, far below the 16-bit storage rounding.
// ---------------------------------------------------------------------------
struct F2 {
    float2 v;
};
__device__ __forceinline__ F2 f2(float a, float b) { return F2{make_float2(a, b)}; }
__device__ __forceinline__ F2 f2(float a) { return F2{make_float2(a, a)}; }
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2{__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return F2{__ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v)}; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return F2{__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator*(float s, F2 b) { return F2{__fmul2_rn(make_float2(s, s), b.v)}; }
__device__ __forceinline__ F2 operator*(F2 a, float s) { return F2{__fmul2_rn(a.v, make_float2(s, s))}; }
__device__ __forceinline__ F2 operator+(F2 a, float s) { return F2{__fadd2_rn(a.v, make_float2(s, s))}; }
__device__ __forceinline__ F2 operator-(F2 a, float s) { return F2{__fadd2_rn(a.v, make_float2(-s, -s))}; }

// a * b + c with one rounding
__device__ __forceinline__ float madd(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ F2 madd(F2 a, F2 b, F2 c) { return F2{__ffma2_rn(a.v, b.v, c.v)}; }
__device__ __forceinline__ F2 madd(float a, F2 b, F2 c) { return F2{__ffma2_rn(make_float2(a, a), b.v, c.v)}; }
__device__ __forceinline__ F2 madd(float a, F2 b, float c) {
    return F2{__ffma2_rn(make_float2(a, a), b.v, make_float2(c, c))};
}

// a per-lane function of a pair
template <typename Fn>
__device__ __forceinline__ F2 lanewise(F2 a, Fn fn) { return F2{make_float2(fn(a.v.x), fn(a.v.y))}; }

// ---------------------------------------------------------------------------
// Moments of 18 populations (the linear map of CollisionEgglesSomers.hpp:
// 186-256), factored through sums/differences of opposite pairs so that each
// moment costs a few adds. m[0] = rho, m[1..3] = momentum, m[4..9] second
// order (M05..M10), m[10..15] third order (M11..M16), m[16..17] fourth order.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void moments_of(const T* q, T* m) {
    const T s01 = q[0] + q[1], d01 = q[0] - q[1];
    const T s03 = q[2] + q[3], d03 = q[2] - q[3];
    const T s05 = q[4] + q[5], d05 = q[4] - q[5];
    // xy edges: Q07 (+,+) Q08 (-,-) Q13 (+,-) Q14 (-,+)
    const T xa = q[6] + q[7], xb = q[6] - q[7], xc = q[12] + q[13], xd = q[12] - q[13];
    // xz edges: Q09 (+,+) Q10 (-,-) Q15 (+,-) Q16 (-,+)
    const T ya = q[8] + q[9], yb = q[8] - q[9], yc = q[14] + q[15], yd = q[14] - q[15];
    // yz edges: Q11 (+,+) Q12 (-,-) Q17 (+,-) Q18 (-,+)
    const T za = q[10] + q[11], zb = q[10] - q[11], zc = q[16] + q[17], zd = q[16] - q[17];

    const T exy = xa + xc, exz = ya + yc, eyz = za + zc;
    const T px = xb + xd, py = xb - xd;        // xy-edge x and y momentum
    const T qx = yb + yd, qz = yb - yd;        // xz-edge x and z momentum
    const T ry = zb + zd, rz = zb - zd;        // yz-edge y and z momentum

    m[0] = s01 + s03 + s05 + exy + exz + eyz;
    m[1] = d01 + px + qx;
    m[2] = d03 + py + ry;
    m[3] = d05 + qz + rz;
    m[4] = exy + exz - s03 - s05;
    m[5] = xa - xc;
    m[6] = exy + eyz - s01 - s05;
    m[7] = ya - yc;
    m[8] = za - zc;
    m[9] = exz + eyz - s01 - s03;
    m[10] = 2.f * px - d01 - qx;
    m[11] = 2.f * py - d03 - ry;
    m[12] = 3.f * (qx - d01);
    m[13] = 3.f * (ry - d03);
    m[14] = qz + rz - 2.f * d05;
    m[15] = 3.f * (rz - qz);
    m[16] = 0.5f * (s01 + s03 + exz + eyz) - s05 - exy;
    m[17] = 1.5f * (s01 - s03 - exz + eyz);
}

// rho and momentum only (what the immersed boundary interpolates).
__device__ __forceinline__ void moments4_of(const float* q, float* m) {
    const float s01 = q[0] + q[1], d01 = q[0] - q[1];
    const float s03 = q[2] + q[3], d03 = q[2] - q[3];
    const float s05 = q[4] + q[5], d05 = q[4] - q[5];
    const float xa = q[6] + q[7], xb = q[6] - q[7], xc = q[12] + q[13], xd = q[12] - q[13];
    const float ya = q[8] + q[9], yb = q[8] - q[9], yc = q[14] + q[15], yd = q[14] - q[15];
    const float za = q[10] + q[11], zb = q[10] - q[11], zc = q[16] + q[17], zd = q[16] - q[17];
    m[0] = s01 + s03 + s05 + xa + xc + ya + yc + za + zc;
    m[1] = d01 + (xb + xd) + (yb + yd);
    m[2] = d03 + (xb - xd) + (zb + zd);
    m[3] = d05 + (yb - yd) + (zb - zd);
}

// ---------------------------------------------------------------------------
// Eggels-Somers collision with optional Smagorinsky LES
// (CollisionEgglesSomers.hpp:27-176) for one cell, in FP32.
//   m      : 18 pre-collision moments
//   fx..fz : IBM force at the cell (zero where the cell was not touched)
//   nu     : in = previous eddy viscosity, out = new one (LES only)
//   out    : 18 post-collision populations
// The inverse filter (:137-171) is applied through the even/odd structure of
// each group of opposite directions. alpha[M17] = alpha[M18] = 0, so the
// fourth-order columns drop out.
//
// FAST: hardware-approximate reciprocals and square root (16-bit forms).
// DEV (16-bit deviation storage): the populations in and out are deviations
// f - w rho0. The moments of the rest populations are (rho0, 0, ..., 0) and
// the inverse filter maps alpha0 = rho0 / 24 back to them, so m[0] holds
// rho - rho0 and alpha0 is taken as (rho - rho0) / 24: every output is then
// the deviation itself, without adding and removing the rest weights.
// ---------------------------------------------------------------------------
// Hardware approximations (PTX rcp.approx / sqrt.approx, flush-to-zero):
// one instruction each instead of the IEEE-rounded sequences. Only for the
// 16-bit storage forms, whose state is rounded to 11 significant bits on
// every store, far above the approximations' few-ulp FP32 error; the FP32
// form keeps IEEE rounding.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
template <bool FAST>
__device__ __forceinline__ float rcp_of(float x) { return FAST ? rcp_approx(x) : __frcp_rn(x); }
template <bool FAST>
__device__ __forceinline__ F2 rcp_of(F2 x) { return lanewise(x, [](float a) { return rcp_of<FAST>(a); }); }
template <bool FAST>
__device__ __forceinline__ float sqrt_abs(float x) { return FAST ? sqrt_approx(fabsf(x)) : sqrtf(fabsf(x)); }
template <bool FAST>
__device__ __forceinline__ F2 sqrt_abs(F2 x) { return lanewise(x, [](float a) { return sqrt_abs<FAST>(a); }); }
template <typename T>
__device__ __forceinline__ T splat(float a);
template <>
__device__ __forceinline__ float splat<float>(float a) { return a; }
template <>
__device__ __forceinline__ F2 splat<F2>(float a) { return f2(a); }

template <bool LES, bool DEV = false, bool FAST = false, typename T = float>
__device__ __forceinline__ void collide(const T* m, T fx, T fy, T fz, T& nu, const CollideParams& p, T* out) {
    const T rho = DEV ? m[0] + p.rho0 : m[0];
    const T inv_rho = rcp_of<FAST>(rho);
    const T jx = madd(0.5f, fx, m[1]);
    const T jy = madd(0.5f, fy, m[2]);
    const T jz = madd(0.5f, fz, m[3]);
    const T ux = inv_rho * jx, uy = inv_rho * jy, uz = inv_rho * jz;

    T b, c;
    if (LES) {
        // fct = 3 / (rho (1 + 6 (Nu + nu)))       (:52)
        const T fct = 3.f * rcp_of<FAST>(rho * madd(6.f, nu + p.nu, 1.f));
        // literal grouping of :55-65: m + 0.5*F*u - m
        const T dudx = fct * (madd(0.5f * fx, ux, m[1]) - m[4]);
        const T dvdy = fct * (madd(0.5f * fy, uy, m[2]) - m[6]);
        const T dwdz = fct * (madd(0.5f * fz, uz, m[3]) - m[9]);
        const T divv = dudx + dvdy + dwdz;
        const T sxy = 2.f * fct * (madd(0.5f * fy, ux, m[2]) - m[5]);
        const T sxz = 2.f * fct * (madd(0.5f * fz, ux, m[3]) - m[7]);
        const T syz = 2.f * fct * (madd(0.5f * fz, uy, m[3]) - m[8]);
        const T sh = 2.f * (dudx * dudx + dvdy * dvdy + dwdz * dwdz) + sxy * sxy + sxz * sxz + syz * syz
                       - (2.f / 3.f) * divv * divv;
        nu = p.cs0sq * sqrt_abs<FAST>(sh);   // (:74)
        const T nut = nu + p.nu;
        b = rcp_of<FAST>(madd(6.f, nut, 1.f));
        c = madd(-6.f, nut, 1.f);
    } else {
        b = splat<T>(p.b0);
        c = splat<T>(p.c0);
    }

    constexpr float r24 = 1.f / 24.f;
    const T a0 = m[0] * r24;
    const T a1 = (m[1] + fx) * r24;
    const T a2 = (m[2] + fy) * r24;
    const T a3 = (m[3] + fz) * r24;
    const T br = b * r24;
    const T a4 = (2.f * jx * ux - m[4] * c) * br;
    const T a5 = (2.f * jx * uy - m[5] * c) * br;
    const T a6 = (2.f * jy * uy - m[6] * c) * br;
    const T a7 = (2.f * jx * uz - m[7] * c) * br;
    const T a8 = (2.f * jy * uz - m[8] * c) * br;
    const T a9 = (2.f * jz * uz - m[9] * c) * br;
    const float g = -p.g3 * r24;   // scalar constant
    const T a10 = g * m[10], a11 = g * m[11], a12 = g * m[12];
    const T a13 = g * m[13], a14 = g * m[14], a15 = g * m[15];

    // faces
    const T e01 = 2.f * a0 + 3.f * (a4 - a6 - a9);
    const T o01 = 4.f * a1 - 2.f * (a10 + a12);
    out[0] = e01 + o01;
    out[1] = e01 - o01;
    const T e03 = 2.f * a0 + 3.f * (a6 - a4 - a9);
    const T o03 = 4.f * a2 - 2.f * (a11 + a13);
    out[2] = e03 + o03;
    out[3] = e03 - o03;
    const T e05 = 2.f * a0 + 3.f * (a9 - a4 - a6);
    const T o05 = 4.f * (a3 - a14);
    out[4] = e05 + o05;
    out[5] = e05 - o05;
    // xy edges: Q07 (+x+y) Q14 (-x+y) Q08 (-x-y) Q13 (+x-y)
    const T exy = a0 + 1.5f * (a4 + a6 - a9);
    const T X = 2.f * (a1 + a10), Y = 2.f * (a2 + a11), Z = 6.f * a5;
    out[6] = exy + X + Y + Z;
    out[13] = exy - X + Y - Z;
    out[7] = exy - X - Y + Z;
    out[12] = exy + X - Y - Z;
    // xz edges: Q09 (+x+z) Q16 (-x+z) Q10 (-x-z) Q15 (+x-z)
    const T exz = a0 + 1.5f * (a4 - a6 + a9);
    const T Xp = 2.f * a1 - a10 + a12, Zp = 2.f * a3 + a14 - a15, W = 6.f * a7;
    out[8] = exz + Xp + Zp + W;
    out[15] = exz - Xp + Zp - W;
    out[9] = exz - Xp - Zp + W;
    out[14] = exz + Xp - Zp - W;
    // yz edges: Q11 (+y+z) Q18 (-y+z) Q12 (-y-z) Q17 (+y-z)
    const T eyz = a0 + 1.5f * (a6 - a4 + a9);
    const T Yp = 2.f * a2 - a11 + a13, Zq = 2.f * a3 + a14 + a15, Wp = 6.f * a8;
    out[10] = eyz + Yp + Zq + Wp;
    out[17] = eyz - Yp + Zq - Wp;
    out[11] = eyz - Yp - Zq + Wp;
    out[16] = eyz + Yp - Zq - Wp;
}

}  // namespace tdlb
