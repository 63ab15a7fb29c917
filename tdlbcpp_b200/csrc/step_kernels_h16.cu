// 16-bit deviation storage (FP16 and BF16) instances of the step kernels
// (step_kernels.cuh). Populations are stored as f - w_d * rho0; collision and
// LES run in FP32. One, two and four cells per thread.
#include "step_kernels.cuh"

namespace tdlb {

static inline unsigned blocks16(long long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

static inline unsigned grid16(const StepArgs& a, int V) {
    if (a.part != 0) return blocks16((long long)a.zone.count * 32, 128);
    return blocks16(a.g.rows() * (a.g.kp / V), 128);
}

// One launch; BOX as StepArgs::box (2 only at one cell per thread, over a
// chunk list).
template <typename S, int V, bool LES, int PART, int BOX>
static void simple16_part(const StepArgs& a, cudaStream_t st) {
    k_step_simple<S, V, LES, false, true, PART, BOX><<<grid16(a, V), 128, 0, st>>>(
        a.A, a.B, a.Nu, a.F, a.mask, a.g, a.p, launch_walk<k_step_simple<S, V, LES, false, true, PART, BOX>, true>(a),
        a.rr, a.bout);
}

template <typename S, int V, bool LES>
static void simple16_les(const StepArgs& a, cudaStream_t st) {
    if constexpr (V == 1) {
        if (a.box == 2) return simple16_part<S, 1, LES, 2, 2>(a, st);
        if (a.part == 1) return simple16_part<S, 1, LES, 1, 0>(a, st);
        if (a.part == 2) return simple16_part<S, 1, LES, 2, 0>(a, st);
    }
    simple16_part<S, V, LES, 0, 0>(a, st);
}

template <typename S, int V>
static cudaError_t simple16(const StepArgs& a, cudaStream_t st) {
    if (a.les) simple16_les<S, V, true>(a, st);
    else simple16_les<S, V, false>(a, st);
    return cudaGetLastError();
}

template <typename S, int V, bool LES, int PART, int BOX>
static void eso16_part(const StepArgs& a, cudaStream_t st) {
    const unsigned grid = grid16(a, V);
    if (a.even)
        k_step_esotwist<S, V, LES, false, true, true, PART, BOX><<<grid, 128, 0, st>>>(
            a.A, a.Nu, a.F, a.mask, a.g, a.p, launch_walk<k_step_esotwist<S, V, LES, false, true, true, PART, BOX>, true>(a),
            a.rr, a.bout);
    else
        k_step_esotwist<S, V, LES, false, true, false, PART, BOX><<<grid, 128, 0, st>>>(
            a.A, a.Nu, a.F, a.mask, a.g, a.p, launch_walk<k_step_esotwist<S, V, LES, false, true, false, PART, BOX>, true>(a),
            a.rr, a.bout);
}

template <typename S, int V, bool LES>
static void eso16_les(const StepArgs& a, cudaStream_t st) {
    if constexpr (V == 1) {
        if (a.box == 2) return eso16_part<S, 1, LES, 2, 2>(a, st);
        if (a.part == 1) return eso16_part<S, 1, LES, 1, 0>(a, st);
        if (a.part == 2) return eso16_part<S, 1, LES, 2, 0>(a, st);
    }
    eso16_part<S, V, LES, 0, 0>(a, st);
}

template <typename S, int V>
static cudaError_t eso16(const StepArgs& a, cudaStream_t st) {
    if (a.les) eso16_les<S, V, true>(a, st);
    else eso16_les<S, V, false>(a, st);
    return cudaGetLastError();
}

// The box launch: one cell per thread over a chunk list (part 2), with the
// residual planes and the scratch outputs.
static bool box_args_ok(const StepArgs& a) {
    if (a.box == 0) return true;
    return a.box == 2 && a.vec == 1 && a.part == 2 && a.rr.on() && a.rw.on() && a.bout.v;
}

cudaError_t launch_step_simple_h16(const StepArgs& a, cudaStream_t st) {
    if (!a.collide || a.from_moments || !box_args_ok(a)) return cudaErrorInvalidValue;   // 16-bit state is always populations
    return with_storage(a.storage, [&](auto s) {
        using S = decltype(s);
        if constexpr (sizeof(S) == 4) return cudaErrorInvalidValue;
        else return a.vec == 1 ? simple16<S, 1>(a, st) : a.vec == 2 ? simple16<S, 2>(a, st) : simple16<S, 4>(a, st);
    });
}

cudaError_t launch_step_esotwist_h16(const StepArgs& a, cudaStream_t st) {
    if (!a.collide || a.from_moments || !box_args_ok(a)) return cudaErrorInvalidValue;
    return with_storage(a.storage, [&](auto s) {
        using S = decltype(s);
        if constexpr (sizeof(S) == 4) return cudaErrorInvalidValue;
        else return a.vec == 1 ? eso16<S, 1>(a, st) : a.vec == 2 ? eso16<S, 2>(a, st) : eso16<S, 4>(a, st);
    });
}

cudaError_t launch_box_commit(const StepArgs& a, bool simple, cudaStream_t st) {
    if (!box_args_ok(a) || a.box != 2) return cudaErrorInvalidValue;
    if (a.zone.count <= 0) return cudaSuccess;
    return with_storage(a.storage, [&](auto s) {
        using S = decltype(s);
        if constexpr (sizeof(S) == 4) return cudaErrorInvalidValue;
        else {
            const unsigned grid = grid16(a, 1);
            if (simple) k_box_commit<S, true, true><<<grid, 128, 0, st>>>(a.B, a.Nu, a.g, a.zone, a.rw, a.bout, a.les);
            else if (a.even) k_box_commit<S, false, true><<<grid, 128, 0, st>>>(a.A, a.Nu, a.g, a.zone, a.rr, a.bout, a.les);
            else k_box_commit<S, false, false><<<grid, 128, 0, st>>>(a.A, a.Nu, a.g, a.zone, a.rr, a.bout, a.les);
            return cudaGetLastError();
        }
    });
}

}  // namespace tdlb
