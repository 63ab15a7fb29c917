// The handle behind tdlb_handle (include/tdlb_b200.h): one lattice on one
// GPU with its device buffers, resident markers and state bookkeeping.
// Shared by the C-ABI translation units.
#pragma once

#include <string>
#include <vector>

#include "tdlb_b200.h"
#include "tdlb_kernels.cuh"
#include "tdlb_runtime.hpp"

using tdlb::Dims;
using tdlb::Planes;

struct tdlb_lattice {
    tdlb_config cfg{};
    Dims g{};
    int device = 0;
    cudaStream_t stream = nullptr;       // all of the handle's work is queued here
    cudaStream_t own_stream = nullptr;   // set when `stream` is borrowed from a batch
    tdlb::CollideParams cp{};

    float* bufA = nullptr;       // 18 planes
    float* bufB = nullptr;       // 18 planes (Simple only)
    float* Nu = nullptr;
    float* F = nullptr;          // 3 planes: Fx, Fy, Fz
    uint32_t* mask = nullptr;    // 2 x (rows * kw) words
    long long mask_words = 0;

    // state
    int cur = 0;                 // Simple: which buffer holds the state (0 A, 1 B)
    bool holds_moments = true;   // state is in moment form (after initialise)
    bool even = true;            // Esotwist parity (ComputeUnit.hpp:116)
    int pass = 0;                // forcing passes so far; mask[pass & 1] is current
    int vec = 4;                 // cells per thread of the step kernels (set per scheme in build())
    int l2_prefetch = 1;         // full step launches prefetch one wave ahead into L2 (tdlb_set_l2_prefetch)
    bool initialised = false;

    // markers: the resident list and its two-segment schedule
    tdlb::Marker* d_markers = nullptr;
    int* d_sched = nullptr;
    int* d_level_ptr = nullptr;
    int* d_plane_lv0 = nullptr;
    int* d_plane_lv1 = nullptr;
    // first-segment cell lists and per-pass IBM buffers
    tdlb::CellList cells;
    int* d_cell_e = nullptr;
    int* d_cell_order = nullptr;  // the big planes' cells first (NULL without big planes)
    int ncell_big = 0;
    int* d_plane_cell = nullptr;
    float* d_prep = nullptr;      // PF_STRIDE * n0
    float* d_cell_m = nullptr;    // 4 * C0 (float4 per cell)
    float* d_cell_F = nullptr;    // 3 * C0
    float* d_tail = nullptr;      // TF_COUNT * tail_cap
    long long tail_cap = 0;
    float* d_sums = nullptr;      // 3 * marker_cap
    int smem_cells = 0;
    int* d_plane_list = nullptr;  // small planes, then big planes
    std::vector<int> h_plane_list;   // host copy of d_plane_list
    unsigned marker_gen = 0;      // bumped by every marker upload
    int n_small = 0, n_big = 0, big_tile_cells = 0;
    // the planes with blade levels, walked by their own launch
    std::vector<int> h_blade_planes;
    int* d_blade_planes = nullptr;
    int n_blade = 0, blade_words = 0;
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    uint32_t* d_mask_static = nullptr;   // first segment's touched cells
    uint32_t* d_exclude = nullptr;       // excluded output points (1 bit per cell), when set
    std::vector<uint32_t> h_exclude;
    double* d_red = nullptr;             // FP64 reduction partials + result
    long long marker_cap = 0;
    long long level_cap = 0;
    int n_markers = 0;      // list length
    int n0 = 0;             // markers of the first segment (the rest rotate)
    std::vector<tdlb_marker> h_markers;   // host copy of the resident list
    tdlb::MarkerSchedule seg0, seg1;
    bool markers_set = false;
    float last_beta = 0.f;        // beta of the last forcing pass (for the load)
    // resident impeller: markers [n0, n_markers) are blades
    double* d_rot_xz = nullptr;   // their impeller-frame offsets (device rotation)
    bool rot_device = false;
    double rot_ci = 0, rot_ck = 0;
    int impeller_begin = -1;      // first marker of the impeller (-1: none)
    tdlb_rushton rspec{};         // the attached impeller's spec
    double angle = 0.0;           // impeller angle of the last rotation
    unsigned long long rstep = 1; // main-loop step the angle belongs to (main.cpp:336 starts at 1)
    double* d_load = nullptr;     // kLoadBlocks*5 partials + 5 results
    // pinned staging of the per-step blade upload (markers and their
    // schedule), two buffers used in turn; each buffer's event marks the end
    // of the copies that read it
    struct PinStage {
        char* p = nullptr;
        size_t cap = 0;
        cudaEvent_t ev = nullptr;
    } pin[2];
    int pin_cur = 0;
    std::vector<double> h_rot_xz; // host copy of d_rot_xz

    // Split steps: the outer chunks of a step run on `stream` while the
    // previous forcing pass and the inner chunks run on `ibm`.
    cudaStream_t ibm = nullptr;
    cudaEvent_t ev_outer = nullptr, ev_inner = nullptr, ev_sync = nullptr;
    int overlap = 0;              // split steps: 0 off, 1 when the zone is small, 2 always (tdlb_set_overlap)
    bool zone_small = false;      // inner chunks hold at most 60 % of the elements
    bool pending = false;         // `ibm` holds work that `stream` has not waited for
    bool inner_queued = false;    // ev_inner marks the inner launch of the last step
    bool resident = false;        // markers kept for many passes (set/attach), so a zone pays
    unsigned zone_gen = ~0u;      // marker_gen the zone was built for
    bool zone_ok = false;         // every stencil cell of the current markers lies in the zone
    std::vector<uint64_t> h_zone_core;   // 1 bit per element: the stencil cells the zone covers
    std::vector<uint32_t> h_zone_bits;   // 1 bit per 32-element chunk, set for the inner chunks
    int* d_zone_list = nullptr;          // the inner chunks, then the outer chunks, each ascending
    int n_zone = 0, n_outer = 0;
    long long zone_list_cap = 0;
    // 16-bit storage: the residual box (tdlb::ResidualBox) and its residuals,
    // one set per population buffer (Simple: A and B; Esotwist: one)
    tdlb::ResidualBox rbox_geom{};        // geometry only (res unused)
    float* d_res[2] = {nullptr, nullptr};
    bool rbox_auto = true;                // set from the impeller by tdlb_attach_rushton
    unsigned box_gen = 0;                 // bumped by every change of the box
    // chunks with a cell near the box (the box launch of a step), ascending,
    // and the Esotwist box launch's scratch outputs (NQ + 1 floats per
    // thread of that launch)
    int* d_box_list = nullptr;
    int n_box = 0;
    long long box_list_cap = 0;
    float* d_box_out = nullptr;
    long long box_out_cap = 0;            // floats
    unsigned box_list_gen = ~0u;          // box_gen the list was built for
    // step-kernel timing (tdlb_set_kernel_timing): start/stop event pairs
    bool timing = false;
    std::vector<cudaEvent_t> tev;
    long long launches = 0;       // kernels queued by the step loop (tdlb_kernel_launches)

    std::string err = "no error";

    size_t esz() const { return cfg.storage == TDLB_STORAGE_FP32 ? 4 : 2; }   // bytes per population
    Planes planes(float* base) const {
        Planes p;
        for (int d = 0; d < tdlb::NQ; d++)
            p.p[d] = reinterpret_cast<float*>(reinterpret_cast<char*>(base) + (size_t)d * (size_t)g.plane * esz());
        return p;
    }
    // FP32 planes of a moment buffer (always FP32)
    Planes planes32(float* base) const {
        Planes p;
        for (int d = 0; d < tdlb::NQ; d++) p.p[d] = base + (size_t)d * (size_t)g.plane;
        return p;
    }
    // residual box of population buffer `buf` (0: bufA, 1: bufB); off when
    // no box is set
    tdlb::ResidualBox rbox(int buf) const {
        tdlb::ResidualBox b = rbox_geom;
        b.res = d_res[buf];
        return b;
    }
    int state_index() const { return cfg.streaming == TDLB_STREAMING_SIMPLE && cur == 1 ? 1 : 0; }
    float* state_buf() const { return cfg.streaming == TDLB_STREAMING_SIMPLE && cur == 1 ? bufB : bufA; }
    float* other_buf() const { return cur == 1 ? bufA : bufB; }
    uint32_t* mask_cur() const { return mask + (size_t)(pass & 1) * mask_words; }
    uint32_t* mask_next() const { return mask + (size_t)((pass + 1) & 1) * mask_words; }
    int state_mode() const {
        if (cfg.streaming == TDLB_STREAMING_SIMPLE) return holds_moments ? 1 : 0;
        return holds_moments ? 3 : 2;
    }
};


// Runtime helpers shared by the C-ABI translation units (tdlb_capi.cu).
namespace tdlb_rt {
// Default cells per thread of a lattice's step kernel. Measured on B200 at
// 400^3 with the L2 prefetch on (step kernel alone): FP32 storage is fastest
// with one cell per thread; 16-bit storage with packed FP32x2 arithmetic,
// Simple with four (1.08 ms), Esotwist with two (1.35 ms; one: 1.48, four:
// 1.39).
inline int default_cells_per_thread(const tdlb_config& c) {
    if (c.storage == TDLB_STORAGE_FP32) return 1;
    return c.streaming == TDLB_STREAMING_SIMPLE ? 4 : 2;
}
tdlb::StepArgs step_args(tdlb_lattice* h, bool collide);
tdlb::IbmArgs ibm_args(tdlb_lattice* h, float alpha, float beta);
// Queue h's work on `s` instead of its own stream (batches share one).
void borrow_stream(tdlb_lattice* h, cudaStream_t s);
// Undo borrow_stream: h's work goes to its own stream again.
void return_stream(tdlb_lattice* h);
// Make `stream` wait for the forcing pass and inner launches queued on the
// split-step stream (every entry point other than the step loop calls it).
cudaError_t join_side(tdlb_lattice* h);
// Remove the residual box (a tank joining a batch, whose step kernel keeps
// none), or set its residuals to zero (after the planes were written
// without them).
void drop_residual_box(tdlb_lattice* h);
void clear_residual_box(tdlb_lattice* h);
}  // namespace tdlb_rt
