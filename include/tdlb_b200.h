/*
 * tdlb_b200.h -- C ABI of the B200-native lattice Boltzmann time step.
 *
 * A drop-in for the hot path of TurbulentDynamics/tdLBCpp: one ComputeUnit
 * (D3Q19 with 18 moving populations, Eggels-Somers collision with optional
 * Smagorinsky LES, Simple or Esotwist streaming, the reference's wall rule,
 * Rushton-turbine immersed-boundary forcing) held on one GPU.
 *
 * Each entry point names the reference interface it replaces
 * (tdlbcpp/src/<file>:<line>). Plain pointers and sizes only; every call
 * returns 0 on success or a negative TDLB_E* code, and tdlb_last_error()
 * gives the message of the last failure on that handle. There is no CPU
 * fallback: a process without a usable sm_100 GPU gets TDLB_ECUDA from
 * tdlb_create().
 *
 * Threading: a handle owns one CUDA stream; calls on one handle must not
 * race each other. Results of device work are visible to the host after the
 * reading calls (tdlb_read_*, tdlb_checkpoint_write, tdlb_synchronize).
 */
#ifndef TDLB_B200_H
#define TDLB_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TDLB_ABI_VERSION 1

/* status codes */
#define TDLB_OK 0
#define TDLB_EINVAL (-1)   /* bad argument (sizes, marker out of range, bad JSON value) */
#define TDLB_ECUDA (-2)    /* CUDA runtime error / no usable device */
#define TDLB_ENOMEM (-3)   /* device or host allocation failed */
#define TDLB_EIO (-4)      /* file missing, unreadable or truncated */
#define TDLB_ESTATE (-5)   /* call not valid in the current state */
#define TDLB_EJSON (-6)    /* input JSON malformed or missing a required key */

/* streaming schemes (FlowParams::streaming, main.cpp:242-256) */
#define TDLB_STREAMING_SIMPLE 0
#define TDLB_STREAMING_ESOTWIST 1

/* population storage precision: FP32 populations, or 16-bit deviations
 * f_i - w_i*rho0 from the rest weights (w = 1/12 faces, 1/24 edges;
 * rho0 = initialRho) with all arithmetic in FP32 */
#define TDLB_STORAGE_FP32 0
#define TDLB_STORAGE_FP16 1
#define TDLB_STORAGE_BF16 2

typedef struct tdlb_lattice* tdlb_handle;

/* An immersed-boundary marker: the fields of the reference's
 * PosPolar<tNi,T> that forcing() reads (Forcing.hpp:72-150), cell indices in
 * interior coordinates (0 <= i < x, 0 <= j < y, 0 <= k < z; the reference adds
 * its ghost width). 48 bytes. */
typedef struct tdlb_marker {
    int64_t i, j, k;
    float iCartFraction;
    float kCartFraction;
    float uDelta, vDelta, wDelta;
    float pad;
} tdlb_marker;

/* Programmatic configuration: the GridParams / FlowParams keys the time step
 * reads (Params/GridParams.hpp:24-32, Params/FlowParams.hpp:24-61). */
typedef struct tdlb_config {
    int64_t x, y, z;          /* interior lattice (GridParams x, y, z) */
    int32_t streaming;        /* TDLB_STREAMING_* */
    int32_t storage;          /* TDLB_STORAGE_* */
    double initialRho;
    double nu;                /* kinematic viscosity (FlowParams::nu, set by calcNuAndRe_m) */
    double cs0;               /* Smagorinsky constant */
    double g3;                /* third-order relaxation */
    double alpha, beta;       /* IBM force relaxation (forcing(geom, alpha, beta)) */
    int32_t useLES;
    int32_t reserved;
} tdlb_config;

/* Replaces: the ComputeUnit constructor + allocateMemory
 * (ComputeUnit.hpp:125-133, ComputeUnitGpu.hpp:31-47) as driven by main.cpp
 * from the input JSON (main.cpp:135-164, :213-256). `params_json` is the text
 * of the reference's input file (GridParams, FlowParams, RunningParams ... ;
 * keys as in input_debug_gridx60_numSteps20.json). The unit takes the
 * FlowParams fields as the file gives them (rounded to float, the
 * reference's FlowParams<float>), nu included: main.cpp builds its unit
 * before calcNuAndRe_m (main.cpp:275) sets nu in main's own copy, so the
 * reference's unit also keeps the file's nu. A caller that wants
 * calcNuAndRe_m's nu writes it into the file or uses tdlb_create_config. */
int tdlb_create(const char* params_json, int device, tdlb_handle* out);

/* The configuration tdlb_create builds from params_json, without a GPU
 * (host only; same errors as tdlb_create, message in tdlb_last_error(NULL)).
 * Replaces: GridParams/FlowParams::getParamsFromJson as main.cpp:150-153
 * calls them. */
int tdlb_config_from_json(const char* params_json, tdlb_config* out);

/* Same, from a filled tdlb_config (nu used as given). */
int tdlb_create_config(const tdlb_config* cfg, int device, tdlb_handle* out);

/* Device bytes a lattice of this config takes (fields, flags, and the marker
 * buffers of a tank-wall geometry; an upper estimate). No counterpart in the
 * reference (its checkEnoughMemory only compares, ComputeUnitGpu.hpp:15-30). */
int tdlb_lattice_bytes(const tdlb_config* cfg, int64_t* bytes);

/* Replaces: ~ComputeUnitBase / freeMemory (ComputeUnit.hpp:150-154). */
int tdlb_destroy(tdlb_handle h);

/* Message of the last failed call on h (or of the last failed create when
 * h is NULL). Never NULL. */
const char* tdlb_last_error(tdlb_handle h);

/* Replaces: ComputeUnitBase::initialise(T rho) (ComputeUnit.hpp:175-190,
 * GPU ComputeUnitGpu.hpp:209-222): moments (rho, 0, ..., 0), F = Nu = 0,
 * Esotwist parity even. */
int tdlb_initialise(tdlb_handle h, float rho);

/* Replaces: forcing(std::vector<PosPolar>&, alfa, beta)
 * (ComputeUnit.h:113, Forcing.hpp:56-176, GPU ComputeUnitGpu.hpp:279-294).
 * Uploads the markers (host pointer, list order = application order),
 * schedules them and runs the immersed-boundary kernels on the current
 * moments. The marker list stays resident for tdlb_forcing_resident(). */
int tdlb_forcing(tdlb_handle h, const tdlb_marker* markers, size_t n, float alpha, float beta);

/* Upload + schedule markers without applying them. */
int tdlb_set_markers(tdlb_handle h, const tdlb_marker* markers, size_t n);

/* forcing() with the resident marker list. */
int tdlb_forcing_resident(tdlb_handle h, float alpha, float beta);

/* Replaces: collision() (CollisionEgglesSomers.hpp:27-181, GPU
 * CollisionEgglesSomers.cuh:17-154) TOGETHER WITH the streaming and
 * moments that follow it: one fused launch streams, forms moments and
 * collides every cell. */
int tdlb_collision(tdlb_handle h);

/* Replace: bounceBackBoundary() (Boundary.hpp:13-35), streamingPush()
 * (StreamingSimple.hpp:257-307, StreamingEsoteric.hpp:14-18) and moments()
 * (CollisionEgglesSomers.hpp:185-256). Their work is inside
 * tdlb_collision(); these keep the reference's call sequence valid and
 * return 0 (streamingPush() flips the Esotwist parity in the reference; here
 * the fused launch does). */
int tdlb_bounce_back(tdlb_handle h);
int tdlb_streaming_push(tdlb_handle h);
int tdlb_moments(tdlb_handle h);

/* One reference time step, main.cpp:438-454 order: collision (fused) then
 * forcing with the resident markers. */
int tdlb_step(tdlb_handle h, float alpha, float beta);

/* Interior moments as the reference's Q holds them after moments()
 * (QVec slots M01..M18), AoS: out[((i*y + j)*z + k)*18 + l]. */
int tdlb_read_moments(tdlb_handle h, float* out);

/* Density and velocity u = (j + F/2)/rho (QVec.hpp:385-394) of every
 * interior cell, each array x*y*z in (i, j, k) order. Any pointer may be
 * NULL. */
int tdlb_read_velocity_density(tdlb_handle h, float* rho, float* ux, float* uy, float* uz);

/* Interior F (3 per cell, AoS; zero where no marker touched the cell), the
 * eddy viscosity Nu (1 per cell) and the touched flags of the last forcing
 * pass (1 byte per cell). */
int tdlb_read_force(tdlb_handle h, float* f3);
int tdlb_read_nu(tdlb_handle h, float* nu);
int tdlb_read_touched(tdlb_handle h, uint8_t* flags);

/* Lattice shape and state. */
int tdlb_get_dims(tdlb_handle h, int64_t* x, int64_t* y, int64_t* z);
int tdlb_get_even_step(tdlb_handle h, int* even);

/* FP64 sums over all interior cells (a project-defined diagnostic; the
 * reference has none): out[0] = mass (sum of rho), out[1..3] = momentum
 * (sum of j + F/2). Deterministic: fixed launch shape and summation order. */
int tdlb_reduce_fp64(tdlb_handle h, double* out4);

/* Make all queued device work complete. */
int tdlb_synchronize(tdlb_handle h);

/* Replaces: ComputeUnitBase::doubleResolutionFullCU() (ComputeUnit.hpp:
 * 258-316): x, y, z double; every new cell takes the moments and Nu of old
 * cell (i/2, j/2, k/2); F, the touched flags and the excluded points start
 * at zero; the state then holds moments, as after tdlb_initialise. The
 * markers are dropped: set the geometry of the new size (as main.cpp:
 * 349-397 does). FP32 storage, handles outside a batch. */
int tdlb_double_resolution(tdlb_handle h);

/* ---- output: excluded points, vorticity slices, plane dump ---- */

/* Replaces: setOutputExcludePoints / unsetOutputExcludePoints
 * (ComputeUnitOutput.hpp:20-53): the cells of the markers (i, j, k) become
 * (exclude = 1) or stop being (0) excluded output points. */
int tdlb_set_output_exclude(tdlb_handle h, const tdlb_marker* markers, size_t n, int exclude);

/* Replaces: calcVorticityXZ(j) / calcVorticityXY(k) (ComputeUnitOutput.hpp:
 * 113-285; GPU ComputeUnitOutput.cuh:10-64) up to the picture: the float
 * field log |curl u|^2, u = j / rho of the current moments, central
 * differences; -1 at excluded points. XZ: out[i*z + k] (x*z floats); XY:
 * out[j*x + i] (x*y floats). A neighbour beyond a lattice face is replaced
 * by the cell itself (the reference reads its ghost layer there). */
int tdlb_vorticity_xz(tdlb_handle h, int64_t j, float* out);
int tdlb_vorticity_xy(tdlb_handle h, int64_t k, float* out);

/* tDiskGrid<float, 4> and tDiskGrid<float, 3> (Output.hpp:22-26): cell
 * coordinates and 4 moments / 3 force components, 24 and 20 bytes. */
typedef struct tdlb_disk_grid4 {
    uint16_t iGrid, jGrid, kGrid, pad;
    float q[4];
} tdlb_disk_grid4;
typedef struct tdlb_disk_grid3 {
    uint16_t iGrid, jGrid, kGrid, pad;
    float q[3];
} tdlb_disk_grid3;

/* Replaces: savePlaneXZ<float, 4> (ComputeUnitOutput.hpp:354-447) up to the
 * files: the records of the plane j, in (i, k) order -- every non-excluded
 * cell's Q slots 0..3 as the reference holds them (Simple: the first four
 * moments; Esotwist: the raw slots of the writeMoments placement, i.e.
 * moments of neighbouring cells), and F where F is non-zero. Coordinates as the
 * reference writes them: iGrid = i, kGrid = k, jGrid = j for the moments and
 * j + 1 for F. q_n / f_n return the counts; with q_out / f_out NULL only the
 * counts are computed. The caller writes the records as the reference's
 * QVec.bin / F3.bin files. */
int tdlb_plane_xz(tdlb_handle h, int64_t j, tdlb_disk_grid4* q_out, size_t q_cap, size_t* q_n, tdlb_disk_grid3* f_out,
                  size_t f_cap, size_t* f_n);

/* Replaces: ComputeUnitBase::checkpoint_write(unit_name, RunningParams)
 * (ComputeUnit.hpp:389-439) with the directory given instead of derived
 * (DiskOutputTree.h:560-570). Writes, in the reference's layout and names
 * (DiskOutputTree.h:572-589), <dir>/checkpoint_grid.<id>.<unit>.{Q,F,Nu}
 * over the ghosted grid (Q: the 18 moments as the reference's Q holds them
 * between steps -- at the cell for Simple, in the writeMoments places for
 * Esotwist; ghost cells zero) and <dir>/AllParams.<id>.<unit>.json. <id> is
 * idi.idj.idk of params_json's ComputeUnitParams (default 0.0.0).
 * params_json (may be NULL) holds the run's params sections (RunningParams
 * with the step and angle, ...); missing sections are filled from the
 * handle. Extension: "StreamingState": {"evenStep"} records the Esotwist
 * parity, which the reference's checkpoint drops. <dir> is created if
 * missing (one level). Any storage precision. */
int tdlb_checkpoint_write(tdlb_handle h, const char* dir, const char* unit_name, const char* params_json);

/* Replaces: ComputeUnitBase::checkpoint_read(dirname, unit_name)
 * (ComputeUnit.hpp:318-386): reads <dir>/AllParams.0.0.0.<unit>.json and
 * the Q, F and Nu files. The lattice size must match the handle; the flow
 * params (nu, cs0, g3, alpha, beta, useLES, initialRho) are taken from the
 * file as the reference does (:341). Afterwards the state holds moments,
 * as after tdlb_initialise; Esotwist parity from "StreamingState.evenStep"
 * (true when absent). A missing or short file is TDLB_EIO (the reference
 * prints and continues). FP32 storage only. */
int tdlb_checkpoint_read(tdlb_handle h, const char* dir, const char* unit_name);

/* Step-kernel variant: cells per thread (1, 2 or 4 -- float2 / float4
 * traffic). Default: 1 for FP32 storage; for 16-bit storage 4 with Simple
 * streaming, 2 with Esotwist (the fastest on B200 at 400^3 for each). Split steps (tdlb_set_overlap) need
 * one cell per thread. FP32
 * storage: all variants compute identical results; 16-bit storage: 2 and 4
 * cells per thread use packed FP32x2 arithmetic (results within FP32
 * rounding). A residual box works with every variant (its own launches run
 * one cell per thread). */
int tdlb_set_cells_per_thread(tdlb_handle h, int v);

/* L2 prefetch of the step kernels (on by default; no counterpart in the
 * reference). A full step launch walks the lattice in 128-thread tiles of
 * the flat row-major cell index; every eighth tile's CTA, as it starts,
 * issues bulk L2 prefetches of the population spans (and Nu) that the tiles
 * one wave of resident CTAs further on will read, so their loads hit L2.
 * Results are identical either way (a prefetch moves no data the kernel
 * sees); the switch is for measurement. on: 0 or 1 (else TDLB_EINVAL). */
int tdlb_set_l2_prefetch(tdlb_handle h, int on);

/* Residual box of the 16-bit storage forms (no counterpart in the
 * reference, whose storage is FP32). For every population location of the
 * cells [i0, i1) x [j0, j1) x [k0, k1) the library keeps, beside the 16-bit
 * deviation, the FP32 residual of its rounding, so these locations are
 * stored exactly: the stirred tank's velocity error against FP64 comes
 * mostly from the 16-bit rounding in the impeller's swept volume. The box
 * costs 72 (Esotwist) or 144 (Simple) bytes of device memory per box cell,
 * plus 76 bytes of scratch per cell of the 32-cell chunks within one cell of
 * it, and traffic only there: a step with a box adds two launches over those
 * chunks (they are stepped with the residuals before the plain launch and
 * committed after it) and never splits (tdlb_set_overlap).
 * tdlb_attach_rushton sets it over the blades' swept volume with a 4-cell
 * margin, unless a box was set (or removed) with this call; an empty box
 * (i1 <= i0) removes it. Requires 16-bit storage (TDLB_EINVAL), a lattice
 * outside a batch (TDLB_ESTATE; a lattice joining a batch loses its box),
 * and i0, j0, k0 >= 1. Read-back (moments, velocity), the forcing pass and
 * the FP64 sums include the residuals. */
int tdlb_set_residual_box(tdlb_handle h, int64_t i0, int64_t i1, int64_t j0, int64_t j1, int64_t k0, int64_t k1);
/* The current box as {i0, i1, j0, j1, k0, k1} (all zero: none). */
int tdlb_get_residual_box(tdlb_handle h, int64_t* box6);

/* Split steps. mode 0 (default): off; 1: on when the inner chunks hold at
 * most 60 % of the lattice (large tanks; a small one is mostly stencil
 * cells); 2: on whenever possible. With resident markers (tdlb_set_markers
 * or tdlb_attach_rushton) and one cell per thread, a step runs as two launches:
 * the cells outside every marker stencil (the "outer" chunks, which read no
 * force) on the handle's stream, and the stencil cells and their neighbours
 * (the "inner" chunks) on a second stream, after the forcing pass. The
 * previous step's forcing pass then runs while the outer cells of the next
 * step are computed. Every cell computes what the single launch computes,
 * so results are bit-identical with overlap on and off. Measured on B200
 * at 400^3 (Rushton tank): whole steps 0-4 % faster, because the two
 * launches over scattered chunks lose most of what the overlap hides, hence
 * off by default. A step with a residual box (tdlb_set_residual_box) runs
 * unsplit. Entry points other
 * than tdlb_collision, tdlb_forcing_resident, tdlb_rotate_impeller and
 * tdlb_step first order the handle's stream after that second stream. */
int tdlb_set_overlap(tdlb_handle h, int mode);

/* Order the handle's stream (tdlb_get_stream) after every queued step and
 * forcing pass, without waiting on the host. */
int tdlb_join(tdlb_handle h);

/* Per-cell flags (interior cells in (i, j, k) order) of the split-step zone:
 * 1 where the cell belongs to an inner chunk. TDLB_ESTATE when the handle
 * does not split its steps (see tdlb_set_overlap). */
int tdlb_read_zone(tdlb_handle h, uint8_t* flags);

/* Step-kernel timing: when on, every step-kernel launch (both launches of a
 * split step) is bracketed by CUDA events on its own stream.
 * tdlb_kernel_time waits for the device, returns the summed launch time in
 * ms and the number of launches since the last call, and resets both. */
int tdlb_set_kernel_timing(tdlb_handle h, int on);
/* Kernels the handle's step loop has queued so far (step launches, forcing
 * passes, blade rotations). */
int tdlb_kernel_launches(tdlb_handle h, int64_t* n);
int tdlb_kernel_time(tdlb_handle h, double* total_ms, int64_t* launches);

/* The cudaStream_t (as void*) all of h's device work is queued on, for
 * callers that time it with CUDA events or order their own work after it. */
int tdlb_get_stream(tdlb_handle h, void** stream);

/* ---- Rushton-turbine geometry (host only; no GPU needed) ----
 * Replaces the un-vendored tdLBGeometryRushtonTurbineLib calls of main.cpp
 * (RushtonTurbinePolarCPP::generateFixedGeometry, :289-290;
 * generateRotatingNonUpdatingGeometry, :293-294; generateRotatingGeometry /
 * updateRotatingGeometry, :297-298 and :424-425; calcThisStepImpellerIncrement,
 * :286 and :409; RushtonTurbine::impellers[0].blades.outerRadius, :275).
 * This is the project's own geometry (spec in tdlbcpp_b200/csrc/geometry.cpp);
 * zero-valued fields take their defaults (T = x, D = T/3, clearance T/3,
 * blade height D/5, 1 disk plane, 6 blades, 4 baffles of width T/10, wall
 * inset 2 cells). Each generator writes at most `cap` markers to `out` and
 * the full count to *n; out == NULL only queries the count. */
typedef struct tdlb_rushton {
    int64_t x, y, z;
    double tank_diameter;
    double impeller_diameter;
    double clearance;
    double blade_height;
    double disk_thickness;
    int32_t n_blades;
    int32_t n_baffles;
    double baffle_width;
    double wall_inset;
    double tip_speed;          /* FlowParams::uav */
    int64_t startup_steps;     /* RunningParams::impellerStartupStepsUntilNormalSpeed */
} tdlb_rushton;

int tdlb_rushton_fixed(const tdlb_rushton* spec, tdlb_marker* out, size_t cap, size_t* n);
int tdlb_rushton_rotating_nonupdating(const tdlb_rushton* spec, double delta_angle, tdlb_marker* out, size_t cap, size_t* n);
int tdlb_rushton_rotating(const tdlb_rushton* spec, double angle, double delta_angle, tdlb_marker* out, size_t cap, size_t* n);
double tdlb_rushton_impeller_increment(const tdlb_rushton* spec, uint64_t step);
int tdlb_rushton_blade_outer_radius(const tdlb_rushton* spec);

/* Resident impeller (replaces main.cpp:409-426, which regenerates the
 * rotating markers on the host and re-uploads the whole list every step):
 * generates the spec's fixed, rotating-non-updating (velocities from
 * nonupdating_delta_angle, as main.cpp:293) and rotating markers at
 * (angle, delta_angle), keeps them on the device in that list order, and
 * schedules the blades for every angle at once. Afterwards
 * tdlb_rotate_impeller() moves the blades on the device and
 * tdlb_forcing_resident()/tdlb_step() apply the list. The impeller must sit
 * at least 2 cells inside the lattice at every angle. */
int tdlb_attach_rushton(tdlb_handle h, const tdlb_rushton* spec, double nonupdating_delta_angle, double angle,
                        double delta_angle);
int tdlb_rotate_impeller(tdlb_handle h, double angle, double delta_angle);

/* Host-driven alternative to tdlb_rotate_impeller(), the way main.cpp does
 * it (:424-426): replace the attached blades with n host-generated markers
 * (same count and order as attached; e.g. tdlb_rushton_rotating at the new
 * angle). Only the blades are copied and rescheduled. */
int tdlb_set_rotating_markers(tdlb_handle h, const tdlb_marker* markers, size_t n);

/* FP64 load on the attached impeller (rotating-non-updating + rotating
 * markers) from the last forcing pass: out[0..2] = force the markers apply
 * to the fluid, -beta * sum of each marker's (interpolated - target)
 * momentum; out[3] = its torque about the tank axis (j); out[4] = markers
 * summed. A project-defined diagnostic: the reference computes none. */
int tdlb_impeller_load(tdlb_handle h, double* out5);
/* The same load, queued on the handle's stream with its copy into out5
 * (pinned host memory or device memory), without waiting: out5 holds it once
 * the stream has reached this point (tdlb_synchronize, or an event recorded
 * on the stream after this call). Lets a caller prepare the next step on the
 * host while the device finishes this one. The first call allocates the
 * reduction's device scratch. */
int tdlb_impeller_load_async(tdlb_handle h, double* out5);

/* The same FP64 impeller load for callers that cannot allocate device
 * memory once their run has started: a host application that hands the
 * whole GPU to its own memory pool up front (a cudaMalloc of the library's
 * would fail or break its accounting), or a real-time loop that forbids
 * allocation after start-up (cudaMalloc can synchronise the device and takes
 * unbounded time). It calls no cudaMalloc, cudaFree or other allocating
 * routine, and writes the 5 doubles to the caller's DEVICE buffer d_out5 on
 * h's stream (nothing is synchronised). No counterpart in the reference.
 * Its scratch is a fixed 40 KiB array compiled into the library, so lists of
 * more than 1,048,576 markers are rejected (TDLB_EINVAL). The first call on
 * each device looks that array up (cudaGetSymbolAddress) and keeps the
 * address: make that first call before any stream capture. A device reset
 * (cudaDeviceReset) invalidates the kept address: do not call this after
 * one in the same process. All calls on a device share the array and it
 * keeps the last call's contents; calls that overlap on the GPU race. */
int tdlb_impeller_load_noalloc(tdlb_handle h, double* d_out5);

/* Copy of the resident marker list as the device holds it (list order). */
int tdlb_read_markers(tdlb_handle h, tdlb_marker* out, size_t cap, size_t* n);

/* Immersed-boundary schedule of a marker list (host only): the per-plane
 * level of every marker (level_out[n], may be NULL) and the largest number
 * of levels in one plane. Markers of one level share no stencil cell. */
int tdlb_schedule_levels(const tdlb_marker* markers, size_t n, int64_t x, int64_t y, int64_t z,
                         int32_t* level_out, int32_t* max_levels_per_plane);

/* ---- batched form: many independent tanks on one GPU ----
 * No counterpart in the reference (it runs one lattice per process,
 * main.cpp:336-454). A batch owns its tanks; every tank is an ordinary
 * handle (tdlb_batch_tank) for initialise, attach_rushton, set_markers and
 * the read functions, and all tanks share the batch's stream. All tanks of a
 * batch use one streaming scheme and one storage precision; sizes, nu, LES
 * and markers differ freely. A run splits the tanks into two groups of about
 * equal cell count on two streams whose fused steps take turns, so one
 * group's forcing pass overlaps the other group's fused step; the batch's
 * stream waits for both before tdlb_batch_run returns. */
typedef struct tdlb_batch_s* tdlb_batch;

int tdlb_batch_create(const tdlb_config* cfgs, int n, int device, tdlb_batch* out);
/* A batch with no tanks yet, for tanks added later (tdlb_batch_add). */
int tdlb_batch_create_empty(int device, int streaming, int storage, tdlb_batch* out);
int tdlb_batch_destroy(tdlb_batch b);
/* Last error of b; of the calling thread's last failed create if b is NULL. */
const char* tdlb_batch_last_error(tdlb_batch b);
int tdlb_batch_size(tdlb_batch b, int* n);
/* A tank joins (index: its position) or leaves the batch between runs; a
 * removed tank's handle is destroyed and later tanks move down by one. */
int tdlb_batch_add(tdlb_batch b, const tdlb_config* cfg, int* index);
/* A lattice created with tdlb_create* and prepared on its own stream
 * (markers attached, initialised, first forcing pass) joins the batch as its
 * last tank: its stream is drained, it runs on the batch's streams from then
 * on and the batch owns it (tdlb_batch_remove or tdlb_batch_destroy destroys
 * it; the caller must not). Its streaming scheme, storage and device must be
 * the batch's. Setting a tank up this way overlaps a running batch, where
 * tdlb_batch_add's tank is set up on the batch's stream after it. No
 * counterpart in the reference, which runs one lattice per process. */
int tdlb_batch_adopt(tdlb_batch b, tdlb_handle h, int* index);
/* The inverse of tdlb_batch_adopt: tank `index` leaves the batch without
 * being destroyed (after the batch's queued work), runs on its own stream
 * again and belongs to the caller (tdlb_destroy). Later tanks move down by
 * one. Lets a caller read a finished tank and free it while the batch runs
 * on. No counterpart in the reference. */
int tdlb_batch_detach(tdlb_batch b, int index, tdlb_handle* out);
int tdlb_batch_remove(tdlb_batch b, int index);
int tdlb_batch_tank(tdlb_batch b, int t, tdlb_handle* out);
/* Shape of the fused batched launch: cells per thread (1, 2, 4; 16-bit
 * storage 1 or 4), threads per block (128 or 256) and blocks per SM: 1..16
 * makes the launch persistent (grid = min(work items, SMs x blocks_per_sm),
 * each block taking items b, b + grid, ...); 0 (the default) runs one block
 * per work item, which the block scheduler balances against the other
 * group's forcing pass. A work item is eight chunks of `threads` quads of
 * one tank. */
int tdlb_batch_set_shape(tdlb_batch b, int cells_per_thread, int threads, int blocks_per_sm);
int tdlb_batch_get_shape(tdlb_batch b, int* cells_per_thread, int* threads, int* blocks_per_sm);
/* Times every shape on the initialised batch and keeps the fastest
 * (best_ms: its fused-launch time, may be NULL). The timed launches change
 * the fields: initialise the tanks again afterwards. */
int tdlb_batch_autotune(tdlb_batch b, int trials, double* best_ms);
/* `steps` time steps of every tank, the reference's main-loop step each
 * (main.cpp:409-454): impeller rotation (tanks with tdlb_attach_rushton, the
 * angle advanced by tdlb_rushton_impeller_increment of the step), fused
 * collision + streaming, immersed-boundary forcing (tanks with markers) with
 * alpha, beta. Pairs of steps replay captured CUDA graphs (four pairs, then
 * single pairs), kept between runs while the batch's tanks and shape stay
 * the same. */
int tdlb_batch_run(tdlb_batch b, int steps, float alpha, float beta);
/* Same steps, every launch issued eagerly (no graph). */
int tdlb_batch_run_eager(tdlb_batch b, int steps, float alpha, float beta);
/* Kernels the batch's runs have launched since it was created (graph
 * replays counted per kernel node). */
int tdlb_batch_kernel_launches(tdlb_batch b, long long* n);
int tdlb_batch_synchronize(tdlb_batch b);
int tdlb_batch_get_stream(tdlb_batch b, void** stream);

/* ---- serving form: a request loop over resident, batched tanks ----
 * No counterpart in the reference. A server runs two threads. A helper
 * admits submitted requests in arrival order while a slot is free and the
 * tank's device bytes (tdlb_lattice_bytes) fit the free HBM (less 1 GiB)
 * and the budget, and builds each admitted tank (a Rushton turbine filling
 * the lattice, tip speed and Re as requested, LES with Cs = 0.1, rho = 1,
 * forced once as main.cpp:305 does) on the tank's own stream while the
 * resident tanks step. The worker adopts built tanks into the resident
 * batch of their precision and scheme (tdlb_batch_adopt) between chunks,
 * advances every resident tank in chunks of min(chunk_steps, smallest
 * remaining step count) with alpha = 0.97, beta = 1.9, and detaches
 * finished tanks (tdlb_batch_detach), which the helper reads out and frees
 * while the next chunk runs. A tank's result does not depend on what else
 * is resident. */
typedef struct tdlb_server_s* tdlb_server;

typedef struct tdlb_request {
    int64_t id;               /* caller's tag, returned in the result */
    int64_t x, y, z;          /* lattice; the tank diameter is x */
    double tip_speed;         /* impeller tip speed (lattice units) */
    double reynolds;          /* nu from calcNuAndRe_m (FlowParams.hpp:65-70) */
    int64_t steps;
    int32_t storage;          /* TDLB_STORAGE_* */
    int32_t streaming;        /* TDLB_STREAMING_* */
    int32_t les;              /* Smagorinsky LES on/off */
    int32_t pad;
    float* out_rho;           /* optional host buffers (x*y*z each), filled */
    float* out_ux;            /* at completion; must stay valid until then */
    float* out_uy;
    float* out_uz;
} tdlb_request;

typedef struct tdlb_result {
    int64_t id;
    int32_t status;           /* TDLB_OK, or why the request failed */
    int32_t pad;
    double t_submit, t_admit, t_done;   /* seconds since the server started */
    int64_t cells, steps;
    double mass, momentum[3];           /* FP64 sums at the end (tdlb_reduce_fp64) */
    double force[3], torque;            /* FP64 impeller load of the last pass */
    double power_number;                /* |torque * omega| / (N^3 D^5), N = omega / 2 pi, rho = 1 */
} tdlb_result;

typedef struct tdlb_server_stats {
    int64_t submitted, completed, queued, active, admitted, chunks, bytes_in_use;
    double lattice_updates;   /* cell updates done so far */
    double busy_s;            /* wall time spent stepping */
    double elapsed_s;         /* since the server started */
} tdlb_server_stats;

/* hbm_budget_bytes: 0 = free HBM only; max_active: resident tank slots. */
int tdlb_server_create(int device, int64_t hbm_budget_bytes, int max_active, int chunk_steps, tdlb_server* out);
int tdlb_server_destroy(tdlb_server s);   /* unfinished requests end with TDLB_ESTATE */
const char* tdlb_server_last_error(tdlb_server s);
/* Thread-safe; the request is copied (its output buffers are not). */
int tdlb_server_submit(tdlb_server s, const tdlb_request* r);
/* Up to cap finished results, in completion order; n: how many. */
int tdlb_server_poll(tdlb_server s, tdlb_result* out, int cap, int* n);
/* Wait until every submitted request has finished (TDLB_ESTATE on timeout). */
int tdlb_server_wait_idle(tdlb_server s, double timeout_s);
int tdlb_server_get_stats(tdlb_server s, tdlb_server_stats* st);

/* ---- known-answer-test support (integer-coded transport) ----
 * Raw population state: for Simple the current buffer, for Esotwist the
 * single in-place buffer. Layout: out[((i*y + j)*z + k)*18 + slot]. */
int tdlb_debug_get_state(tdlb_handle h, float* out);
int tdlb_debug_set_state(tdlb_handle h, const float* in, int holds_moments);
/* One transport-only step (identity collision): streaming and, for
 * Esotwist, the parity flip, exactly as a step with f* = f. */
int tdlb_debug_transport(tdlb_handle h);

#ifdef __cplusplus
}
#endif
#endif /* TDLB_B200_H */
