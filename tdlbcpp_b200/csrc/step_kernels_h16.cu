// 16-bit deviation storage (FP16 and BF16) instances of the step kernels
// (step_kernels.cuh). Populations are stored as f - w_d * rho0; collision and
// LES run in FP32. One and four cells per thread.
#include "step_kernels.cuh"

namespace tdlb {

static inline unsigned blocks16(long long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

template <typename S, int V>
static cudaError_t simple16(const StepArgs& a, cudaStream_t st) {
    const dim3 grid(blocks16(a.g.rows() * (a.g.kp / V), 128)), block(128);
    if (a.les) k_step_simple<S, V, true, false, true><<<grid, block, 0, st>>>(a.A, a.B, a.Nu, a.Fx, a.Fy, a.Fz, a.mask, a.g, a.p);
    else k_step_simple<S, V, false, false, true><<<grid, block, 0, st>>>(a.A, a.B, a.Nu, a.Fx, a.Fy, a.Fz, a.mask, a.g, a.p);
    return cudaGetLastError();
}

template <typename S, int V>
static cudaError_t eso16(const StepArgs& a, cudaStream_t st) {
    const dim3 grid(blocks16(a.g.rows() * (a.g.kp / V), 128)), block(128);
    if (a.les) {
        if (a.even) k_step_esotwist<S, V, true, false, true, true><<<grid, block, 0, st>>>(a.A, a.Nu, a.Fx, a.Fy, a.Fz, a.mask, a.g, a.p);
        else k_step_esotwist<S, V, true, false, true, false><<<grid, block, 0, st>>>(a.A, a.Nu, a.Fx, a.Fy, a.Fz, a.mask, a.g, a.p);
    } else {
        if (a.even) k_step_esotwist<S, V, false, false, true, true><<<grid, block, 0, st>>>(a.A, a.Nu, a.Fx, a.Fy, a.Fz, a.mask, a.g, a.p);
        else k_step_esotwist<S, V, false, false, true, false><<<grid, block, 0, st>>>(a.A, a.Nu, a.Fx, a.Fy, a.Fz, a.mask, a.g, a.p);
    }
    return cudaGetLastError();
}

cudaError_t launch_step_simple_h16(const StepArgs& a, cudaStream_t st) {
    if (!a.collide || a.from_moments) return cudaErrorInvalidValue;   // 16-bit state is always populations
    return with_storage(a.storage, [&](auto s) {
        using S = decltype(s);
        if constexpr (sizeof(S) == 4) return cudaErrorInvalidValue;
        else return a.vec == 1 ? simple16<S, 1>(a, st) : simple16<S, 4>(a, st);
    });
}

cudaError_t launch_step_esotwist_h16(const StepArgs& a, cudaStream_t st) {
    if (!a.collide || a.from_moments) return cudaErrorInvalidValue;
    return with_storage(a.storage, [&](auto s) {
        using S = decltype(s);
        if constexpr (sizeof(S) == 4) return cudaErrorInvalidValue;
        else return a.vec == 1 ? eso16<S, 1>(a, st) : eso16<S, 4>(a, st);
    });
}

}  // namespace tdlb
