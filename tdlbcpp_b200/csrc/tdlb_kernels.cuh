// Internal interface between the host runtime (tdlb_capi.cu) and the kernels.
#pragma once
#include "tdlb_common.cuh"

namespace tdlb {

// Arguments of one fused step launch.
struct StepArgs {
    Planes A;               // Simple: source buffer; Esotwist: the single buffer
    Planes B;               // Simple: destination buffer (unused for Esotwist)
    float* Nu;
    const float* Fx;
    const float* Fy;
    const float* Fz;
    const uint32_t* mask;   // IBM-touched flags of the forcing pass this step uses
    Dims g;
    CollideParams p;
    int les;                // Smagorinsky LES on/off (FlowParams::useLES)
    int from_moments;       // state holds moments (after initialise / checkpoint load)
    int collide;            // 0: transport only (identity collision; known-answer tests)
    int even;               // Esotwist parity (evenStep)
};

cudaError_t launch_step_simple(const StepArgs& a, cudaStream_t st);
cudaError_t launch_step_esotwist(const StepArgs& a, cudaStream_t st);
cudaError_t launch_fill_uniform_moments(Planes Q, const Dims& g, float rho, cudaStream_t st);
cudaError_t launch_state_moments(Planes A, Planes M, const Dims& g, int mode, int even, cudaStream_t st);

// ---- immersed boundary ----

// Marker record, identical in layout to tdlb_marker (include/tdlb_b200.h).
struct Marker {
    long long i, j, k;
    float iCartFraction, kCartFraction, uDelta, vDelta, wDelta, pad;
};
static_assert(sizeof(Marker) == 48, "Marker layout");

// Per-marker scratch written by the gather phase, read by the spread phase,
// field-major so consecutive markers of a level load contiguously.
enum ScratchField {
    SF_W = 0,               // 9 stencil weights, (k1, i1) order
    SF_RHO = 9,             // 9 densities
    SF_MX = 18, SF_MY = 27, SF_MZ = 36,   // 9 momenta each
    SF_U = 45, SF_V = 46, SF_WV = 47,     // marker velocity
    SF_CELL = 48,           // 9 cell element indices (int32 bit patterns)
    SF_COUNT = 57
};

struct IbmArgs {
    const Marker* markers;      // device copy of the marker list (list order)
    const int* sched;           // execution order: marker index per slot
    const int* level_ptr;       // [nlevels+1] slot offsets of each level
    const int* plane_lv;        // [ny+1] first level of each j-plane
    int n;                      // number of markers
    float* scratch;             // SF_COUNT * cap floats
    long long cap;              // scratch stride (>= n)
    Planes A;                   // current state
    int state_mode;             // 0 Simple pops, 1 moments, 2 Esotwist pops, 3 Esotwist moments
    int even;                   // Esotwist parity of the state's read map
    float* Fx; float* Fy; float* Fz;
    const uint32_t* mask_old;   // touched flags of the previous forcing pass
    uint32_t* mask_new;         // touched flags of this pass (fully written)
    Dims g;
    float alpha, beta;
};

cudaError_t launch_ibm(const IbmArgs& a, cudaStream_t st);
size_t ibm_smem_bytes(const Dims& g);
// Opt the spread kernel in to `bytes` of dynamic shared memory (> 48 KiB).
cudaError_t ibm_prepare_smem(size_t bytes);
// Recompute n rotating markers (offsets xz[2n]) for cos/sin (ca, sa).
cudaError_t launch_rotate_markers(const double* xz, Marker* out, int n, double ca, double sa, double omega, double ci,
                                  double ck, int nx, int nz, cudaStream_t st);

}  // namespace tdlb
