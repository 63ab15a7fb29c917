// Rotation of an impeller marker, shared by the host geometry generator
// (geometry.cpp) and the device rotation kernel (ibm_kernels.cu).
//
// Every double operation is written as its own rounded step (the device
// uses the _rn intrinsics, which are never fused into multiply-adds; the host
// build has no FMA contraction), so host and device produce bit-identical
// markers for the same (x0, z0, cos, sin, omega).
#pragma once

#include <cmath>

#include "tdlb_geometry.hpp"

#if defined(__CUDACC__)
#define TDLB_HD __host__ __device__
#else
#define TDLB_HD
#endif

namespace tdlb {

TDLB_HD inline double dmul(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
TDLB_HD inline double dadd(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
TDLB_HD inline double dsub(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}

// Marker at impeller angle a (ca = cos a, sa = sin a) for a blade point with
// offset (x0, z0) from the tank axis (ci, ck); nearest cell clamped to the
// lattice, fractions in [-0.5, 0.5], velocity omega x r about the j axis.
TDLB_HD inline RotatedMarker rotate_marker(double x0, double z0, double ca, double sa, double omega, double ci,
                                           double ck, long long nx, long long nz) {
    const double di = dsub(dmul(x0, ca), dmul(z0, sa));
    const double dk = dadd(dmul(x0, sa), dmul(z0, ca));
    const double pi = dadd(ci, di);
    const double pk = dadd(ck, dk);
    long long i = (long long)floor(dadd(pi, 0.5));
    long long k = (long long)floor(dadd(pk, 0.5));
    i = i < 0 ? 0 : (i > nx - 1 ? nx - 1 : i);
    k = k < 0 ? 0 : (k > nz - 1 ? nz - 1 : k);
    RotatedMarker r;
    r.i = i;
    r.k = k;
    r.iCartFraction = (float)dsub(pi, (double)i);
    r.kCartFraction = (float)dsub(pk, (double)k);
    r.uDelta = (float)dmul(-omega, dsub(pk, ck));
    r.wDelta = (float)dmul(omega, dsub(pi, ci));
    return r;
}

}  // namespace tdlb
