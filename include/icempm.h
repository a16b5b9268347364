/*
 * icempm.h -- C ABI of the B200-native 2D APIC MPM sea-ice step.
 *
 * This is the drop-in boundary for the reference's GPU driver path
 * (simulation/gpu_implementation5.{h,cpp}, simulation/gpu_partition.{h,cpp},
 * simulation/kernels.cuh of igorg520b/iceMPM_2d_sp).  Every entry point takes
 * plain pointers and sizes; no C++ or torch types cross it.  The caller owns
 * all host buffers; the library owns the device arrays and its CUDA stream.
 *
 * Return convention (all functions): 0 = ok, negative = API/CUDA error
 * (ICEMPM_E_*; icempm_last_error() gives the message of the calling thread).
 * Device-side simulation errors are reported separately as the reference's
 * bitmask (ICEMPM_ERR_*) through icempm_get_status().
 *
 * Threading: a handle is not re-entrant; calls on one handle must be
 * serialised by the caller (the reference drives GPU_Implementation5 from a
 * single thread: cli/main.cpp:55-59, gui/backgroundworker.cpp:37-63).
 * Separate handles are independent.
 */
#ifndef ICEMPM_H
#define ICEMPM_H

#include <stddef.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#if defined(__GNUC__)
#define ICEMPM_API __attribute__((visibility("default")))
#else
#define ICEMPM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* SimParams: byte-for-byte mirror of `struct SimParams`                    */
/* (simulation/parameters_sim.h:36-127).  Field order, types and therefore  */
/* the x86-64 layout (328 bytes) are identical, so a caller holding the     */
/* reference struct can pass its address directly.  The static members of  */
/* the reference struct are the ICEMPM_* constants below.                   */
/* ------------------------------------------------------------------------ */
typedef struct icempm_simparams {
    int32_t tpb_P2G, tpb_Upd, tpb_G2P;
    uint32_t nPartitions;
    int32_t nPtsInitial;
    int64_t SimulationStartUnixTime;
    double InitialTimeStep, SimulationEndTime;
    double AnimationFramePeriod;
    int32_t SimulationStep;
    double SimulationTime;
    bool SaveSnapshots;
    int32_t SnapshotPeriod;
    int32_t GridXTotal, GridYTotal;
    int32_t ModeledRegionOffsetX, ModeledRegionOffsetY;
    int32_t InitializationImageSizeX, InitializationImageSizeY;
    double DimensionHorizontal;
    double windDragCoeff_airDensity;
    bool UseWindData, UseCurrentData;
    double sea_water_density;
    double waterDragEffectiveLinear, waterDragEffectiveQuadratic;
    double IceDensity, PoissonsRatio, YoungsModulus;
    double IceCompressiveStrength, IceTensileStrength, IceShearStrength, IceTensileStrength2;
    double DP_phi, DP_threshold_p;
    double RidgeFormationCoeff;
    double cellsize;
    double ParticleVolume, ParticleViewSize;
    double dt_vol_Dpinv, vmax;
    double lambda, mu, kappa;
    double ParticleMass;
    double cellsize_inv, Dp_inv;
    int32_t UpdateEveryNthStep;
} icempm_simparams_t;

/* static constexpr members of SimParams (parameters_sim.h:39-76) */
#define ICEMPM_DISABLED_PTS_PROPORTION_THRESHOLD 0.05f
#define ICEMPM_PI 3.14159265358979323846
#define ICEMPM_GRAVITY 9.8
#define ICEMPM_MAX_REGIONS 100

/* grid arrays (parameters_sim.h:49-58); node index = y + x*GridYTotal */
enum {
    ICEMPM_GRID_MASS = 0, ICEMPM_GRID_PX = 1, ICEMPM_GRID_PY = 2,
    ICEMPM_GRID_NX = 3, ICEMPM_GRID_NY = 4,
    ICEMPM_GRID_CURRENT_VX = 5, ICEMPM_GRID_CURRENT_VY = 6,
    ICEMPM_GRID_FX = 7, ICEMPM_GRID_FY = 8,
    ICEMPM_N_GRID_ARRAYS = 9
};

/* HSSOA rows (parameters_sim.h:65-76): point i, row j lives at
 * buf[i + capacity*j], all rows f64.  Rows 0-2 hold a uint32 in the low 4
 * bytes of the double slot (the reference reinterpret_casts them). */
enum {
    ICEMPM_IDX_UTILITY = 0, ICEMPM_IDX_CELL = 1, ICEMPM_IDX_POINT = 2,
    ICEMPM_IDX_P = 3, ICEMPM_IDX_Q = 4, ICEMPM_IDX_JP_INV = 5,
    ICEMPM_IDX_POSX = 6, ICEMPM_IDX_VELX = 8, ICEMPM_IDX_FE00 = 10,
    ICEMPM_IDX_BP00 = 14, ICEMPM_IDX_THICKNESS = 18,
    ICEMPM_N_PTS_ARRAYS = 19
};

/* point flags in the utility word (kernels.cuh:11-13) */
#define ICEMPM_STATUS_CRUSHED  0x10000u
#define ICEMPM_STATUS_DISABLED 0x20000u
#define ICEMPM_STATUS_ERROR    0x40000u

/* device error bitmask, same values as kernels.cuh:17-26 */
#define ICEMPM_ERR_POINT_POS_NAN      0x0001u
#define ICEMPM_ERR_POINT_VEL_NAN      0x0002u
#define ICEMPM_ERR_POINT_JUMP_CELLS   0x0004u
#define ICEMPM_ERR_POINT_LEFT_AREA    0x0008u
#define ICEMPM_ERR_POINT_BP_NAN       0x0010u
#define ICEMPM_ERR_POINT_FE_NAN       0x0020u
#define ICEMPM_ERR_GRID_P2G_NAN_VEL   0x0100u
#define ICEMPM_ERR_GRID_P2G_NAN_MASS  0x0200u
#define ICEMPM_ERR_GRID_NAN           0x0400u
/* bits added by this library (no reference counterpart) */
#define ICEMPM_ERR_FIXED_OVERFLOW     0x1000u  /* a P2G term exceeded the fixed-point range */
#define ICEMPM_ERR_BARRIER_TIMEOUT    0x2000u  /* a bounded device wait gave up */

/* API error codes (negative returns) */
#define ICEMPM_OK            0
#define ICEMPM_E_ARG        (-1)
#define ICEMPM_E_CUDA       (-2)
#define ICEMPM_E_NOMEM      (-3)
#define ICEMPM_E_STATE      (-4)
#define ICEMPM_E_CAPACITY   (-5)
#define ICEMPM_E_UNSUPPORTED (-6)

/* ------------------------------------------------------------------------ */
/* Options (no reference counterpart: the reference has one FP64 path).      */
/* ------------------------------------------------------------------------ */
enum {
    ICEMPM_VARIANT_FIXED = 0, /* FP32 state, int64 fixed-point P2G (deterministic) */
    ICEMPM_VARIANT_FP32  = 1, /* FP32 state, FP32 atomics                           */
    ICEMPM_VARIANT_FP64  = 2, /* FP64 state and arithmetic, FP64 atomics            */
    ICEMPM_VARIANT_TEXTBOOK = 3 /* the plain FP32 baseline: three unfused kernels, one point or
                                   node per thread, 27 global FP32 atomics per point in P2G
                                   (for comparison; never faster) */
};
enum {
    ICEMPM_FORCING_COMPAT   = 0, /* reference grid update: effective drag + current ramp (kernels.cuh:141-169) */
    ICEMPM_FORCING_EXTENDED = 1  /* quadratic water drag (rho_w, Cd) + wind stress (rho_a, Ca) */
};
enum { ICEMPM_WIND_NONE = 0, ICEMPM_WIND_UNIFORM = 1, ICEMPM_WIND_RANKINE = 2 };

typedef struct icempm_options {
    int32_t variant;          /* ICEMPM_VARIANT_* */
    int32_t forcing;          /* ICEMPM_FORCING_* */
    int32_t sort_every;       /* internal locality re-sort cadence in steps; 0 = only at upload */
    int32_t use_graphs;       /* capture step chunks in CUDA graphs (1 = yes) */
    int32_t block_threads;    /* particle kernel CTA size: 128, 256 or 512 (0 = default) */
    int32_t warp_reduce;      /* same-cell warp pre-reduction in P2G (1 = yes) */
    int32_t device;           /* CUDA device ordinal */
    int32_t reserved0;
    /* extended forcing only */
    double water_density, water_drag_coeff;   /* rho_w [kg/m^3], Cd */
    double air_density, air_drag_coeff;       /* rho_a [kg/m^3], Ca */
    int32_t wind_kind;                        /* ICEMPM_WIND_* */
    int32_t reserved1;
    double wind_u, wind_v;                    /* uniform wind [m/s] */
    double wind_cx, wind_cy;                  /* Rankine centre [m, world coords] */
    double wind_vmax, wind_radius;            /* Rankine peak speed [m/s] and radius [m] */
} icempm_options_t;

typedef struct icempm_context icempm_t;

/* Fill `opts` with the defaults (fixed-point variant, compat forcing). */
ICEMPM_API void icempm_default_options(icempm_options_t *opts);

/* Create a context for one scene on one GPU.
 * Replaces GPU_Implementation5::initialize + GPU_Partition::allocate +
 * transfer_grid_data_to_device + update_current_field
 * (gpu_implementation5.cpp:94-128,165-184; gpu_partition.cpp:108-137,174-196,259-293).
 *   prms          : SimParams with helper variables computed (ComputeHelperVariables)
 *   grid_status   : GridX*GridY bytes, node index y + x*GridY (100 = modelled water)
 *   current_vxvy  : 2*GridX*GridY doubles (vx block then vy block) or NULL (zero current)
 *   capacity      : maximum number of points the device arrays hold
 *   opts          : NULL for defaults */
ICEMPM_API int icempm_create(const icempm_simparams_t *prms, const uint8_t *grid_status,
                  const double *current_vxvy, uint32_t capacity,
                  const icempm_options_t *opts, icempm_t **out);

/* Destroy a context and free its device memory (GPU_Partition::~GPU_Partition,
 * gpu_partition.cpp:214-232). NULL is accepted. */
ICEMPM_API int icempm_destroy(icempm_t *ctx);

/* Upload `size` points from a reference-layout HSSOA buffer (19 rows of
 * `capacity` doubles).  Replaces GPU_Partition::transfer_points_from_soa_to_device
 * (gpu_partition.cpp:81-106).  disabled_count seeds the device counter. */
ICEMPM_API int icempm_upload_points(icempm_t *ctx, const double *hssoa, uint32_t capacity,
                         uint32_t size, int32_t disabled_count);

/* Re-read SimParams (GPU_Partition::update_constants, gpu_partition.cpp:140-170).
 * Also clears the device error word as the reference does. */
ICEMPM_API int icempm_update_constants(icempm_t *ctx, const icempm_simparams_t *prms);

/* Replace the current field (GPU_Partition::update_current_field,
 * gpu_partition.cpp:174-196): 2*GridX*GridY doubles, vx block then vy block. */
ICEMPM_API int icempm_set_current(icempm_t *ctx, const double *current_vxvy);

/* Time-varying current and wind.  The reference reads one static current
 * field (WindAndCurrentInterpolator::ReadStaticFlowData,
 * windandcurrentinterpolator.cpp:20-63), leaves SetTime unfinished (66-70:
 * "return whether data needs to be copied to GPU") and keeps a wind that is
 * bilinear in space and linear in time between two frames commented out
 * (get_wind_vector, kernels.cuh:580-622).  Here both frames live on the
 * device and icempm_set_forcing_time blends them in one kernel.
 *
 * icempm_set_flow_frames: current frames a and b, 2*GridX*GridY doubles each
 * (vx block, vy block, as icempm_set_current); b NULL repeats a; both NULL
 * drops the frames (the current set last stays in force). */
ICEMPM_API int icempm_set_flow_frames(icempm_t *ctx, const double *current_a, const double *current_b);

/* Wind frames on a coarse grid: rows x cols samples of 4 floats {u_a, v_a,
 * u_b, v_b} (m/s), row-major, row along y and column along x (the reference's
 * wgrid[lat][lon][4]); sample (r, c) sits at world (x0 + c*cell, y0 + r*cell)
 * metres.  wind NULL drops the frames (the static wind of the options stays
 * in force).  Rejects rows or cols < 1, cell <= 0 or non-finite values. */
ICEMPM_API int icempm_set_wind_frames(icempm_t *ctx, const float *wind, int32_t rows, int32_t cols, double cell,
                                      double x0, double y0);

/* Blend the frames into the forcing the next sub-steps read: current =
 * (1-tc)*a + tc*b at every node; with wind frames, wind = (1-tw)*W_a + tw*W_b,
 * W bilinear at the node's world position (x*cellsize, y*cellsize; clamped
 * to the wind grid), and wind stress rho_air*C_air*|U|*U (extended forcing).
 * Weights outside [0, 1] are rejected; ICEMPM_E_STATE when no frames are set.
 * Asynchronous on the context's stream; under the extended forcing the next
 * step scatters from the new forcing. */
ICEMPM_API int icempm_set_forcing_time(icempm_t *ctx, double tc, double tw);

/* The forcing tables the sub-steps read: current (2*GridX*GridY doubles, vx
 * block then vy block) and the extended forcing's wind stress (same layout,
 * Pa); either pointer may be NULL.  Synchronises the stream. */
ICEMPM_API int icempm_get_forcing(icempm_t *ctx, double *current_vxvy, double *wind_stress_xy);

/* Advance `nsteps` sub-steps starting at step index `first_step`.  Step k runs
 * reset_grid, p2g, update_nodes(t = dt*k rounded to float) and
 * g2p(recordPQ = (k % UpdateEveryNthStep == 0)), exactly as the loop in
 * Model::Step (model.cpp:18-39).  Asynchronous: returns after enqueueing. */
ICEMPM_API int icempm_step(icempm_t *ctx, int32_t nsteps, int32_t first_step);

/* Download all points into a reference-layout HSSOA buffer, in the slot order
 * of the last upload (or of the last icempm_sort_compact).  Replaces
 * GPU_Partition::transfer_from_device's point part (gpu_partition.cpp:17-38).
 * Synchronises the stream.  *size receives the number of points. */
ICEMPM_API int icempm_download_points(icempm_t *ctx, double *hssoa, uint32_t capacity, uint32_t *size);

/* The same download without waiting for it: the state at this point of the
 * stream is converted into the context's staging buffer, and its copy into
 * `hssoa` runs on a second stream, so icempm_step calls made next overlap the
 * copy (the reference's GPU_Implementation5 carries a
 * transfer_completion_callback for this purpose, gpu_implementation5.h:45,
 * unused there).  `hssoa` must stay valid and unread until
 * icempm_download_wait returns; page-locked memory (icempm_host_register)
 * lets the copy overlap.  *size receives the number of points at once. */
ICEMPM_API int icempm_download_points_async(icempm_t *ctx, double *hssoa, uint32_t capacity, uint32_t *size);

/* Wait for the last icempm_download_points_async copy to land in host
 * memory (sub-steps enqueued after it keep running).  Returns at once when
 * no copy is outstanding. */
ICEMPM_API int icempm_download_wait(icempm_t *ctx);

/* Fetch the device error bitmask and disabled-point counter
 * (gpu_partition.cpp:40-48).  Synchronises the stream. */
ICEMPM_API int icempm_get_status(icempm_t *ctx, uint32_t *error_bits, int32_t *disabled_count);

/* Zero the boundary-force accumulators (GPU_Partition::clear_force_accumulator,
 * gpu_partition.cpp:310-319). */
ICEMPM_API int icempm_clear_force_accumulator(icempm_t *ctx);

/* Download the accumulated boundary forces into fxfy (2*GridX*GridY doubles,
 * fx block then fy block) divided by elapsed_steps*dt, as
 * GPU_Implementation5::transfer_from_device does (gpu_implementation5.cpp:188-224). */
ICEMPM_API int icempm_get_boundary_forces(icempm_t *ctx, double *fxfy, int32_t elapsed_steps);

/* Remove disabled points and sort the rest by cell index x*GridY+y, on the
 * device.  Same result as HostSideSOA::RemoveDisabledAndSort followed by a
 * re-upload (host_side_soa.cpp:36-47, model.cpp:63-72); ties keep their
 * previous relative order.  Resets the disabled counter to 0. */
ICEMPM_API int icempm_sort_compact(icempm_t *ctx);

/* Sort cadence from a measurement on the live scene (no reference
 * counterpart: the reference re-sorts only when it compacts, host_side_soa.cpp:36-47).
 * Advances the scene 2 * trial_steps sub-steps from first_step: trial_steps in
 * the current point order, one locality sort (timed), trial_steps in the
 * sorted order.  Cadence k in {100, 400} is kept when the sorted order's
 * ms/step plus the sort's ms / k beats the current order's ms/step, else 0;
 * the choice becomes the context's sort_every and is returned. */
ICEMPM_API int icempm_tune_sort_cadence(icempm_t *ctx, int32_t trial_steps, int32_t first_step, int32_t *sort_every);

/* Device time of the last icempm_step call, in ms: [0] total, [1] grid
 * update kernels, [2] fused G2P+P2G kernels, [3] locality re-sorts.
 * Synchronises the stream. (GPU_Partition::record_timings, gpu_partition.cpp:370-436) */
ICEMPM_API int icempm_timings(icempm_t *ctx, float ms[4]);

/* Run `nsteps` further sub-steps launched one by one (no CUDA graph) with a
 * CUDA event pair around every kernel, and report the summed device time of
 * the grid-update kernels and of the fused G2P+P2G kernels.  Continues from
 * the device step counter; used for per-kernel profiling. (No reference
 * counterpart beyond the phase columns of GPU_Partition::record_timings.) */
ICEMPM_API int icempm_phase_times(icempm_t *ctx, int32_t nsteps, float *update_ms, float *fused_ms);

/* Fixed-point scales of the P2G accumulators (value * scale -> int64) of the
 * FIXED variant.  No reference counterpart. */
ICEMPM_API int icempm_fixed_point_scales(icempm_t *ctx, double *scale_mass, double *scale_momentum);

/* Page-lock a caller-owned host range for asynchronous copies
 * (cudaHostRegister) and release it again.  No reference counterpart. */
ICEMPM_API int icempm_host_register(void *ptr, size_t bytes);
ICEMPM_API int icempm_host_unregister(void *ptr);

/* Number of visible CUDA devices (0 with a negative return when none). */
ICEMPM_API int icempm_device_count(int *count);

/* Number of points currently on the device (including disabled ones). */
ICEMPM_API int icempm_point_count(icempm_t *ctx, uint32_t *n);

/* CUDA stream the context enqueues on (cudaStream_t), for event timing. */
ICEMPM_API int icempm_get_stream(icempm_t *ctx, void **stream);

/* Number of kernel launches this context has enqueued since creation. */
ICEMPM_API int icempm_launch_count(icempm_t *ctx, uint64_t *count);

/* Test hook of the bounded device waits (no counterpart in the reference,
 * whose kernels do not wait on copies).  The fused kernel waits on a barrier
 * for each chunk's point state; with extra_bytes > 0 every such barrier
 * expects extra_bytes more than the copies deliver, so the wait runs out
 * after wait_limit_us although every copy has landed, and the step raises
 * ICEMPM_ERR_BARRIER_TIMEOUT instead of hanging.  (0, 0) restores the
 * production setting (exact byte counts, 1 s limit).  The context stays
 * usable: icempm_update_constants clears the error word. */
ICEMPM_API int icempm_debug_barrier_timeout(icempm_t *ctx, uint32_t extra_bytes, uint32_t wait_limit_us);

/* Largest point count icempm_cell_order_noalloc accepts. */
#define ICEMPM_NOALLOC_MAX_POINTS (1u << 20)

/* Compaction order without device allocation.  No counterpart in the
 * reference.  For callers that must not allocate device memory -- code whose
 * host framework owns every device byte through its own pool, or that issues
 * work into a stream it cannot synchronise around cudaMalloc/cudaFree -- this
 * computes the order icempm_sort_compact applies: d_order[0..*d_count) are the
 * indices of the points without ICEMPM_STATUS_DISABLED, sorted by cell index
 * x*grid_y + y of the cell word d_cell[i] ((y << 16) | x), ties in index
 * order.  Inputs d_cell, d_utility (n words each) and outputs d_order (n
 * words) and d_count (1 word) are the caller's device buffers.  All
 * intermediate storage is one static device array of 36 MiB that every GPU
 * loading this library keeps until exit; n above ICEMPM_NOALLOC_MAX_POINTS is
 * rejected with ICEMPM_E_CAPACITY.  The first call on a device resolves that
 * array's address (set-up), so make it before any stream capture.  Calls share
 * the array: calls that overlap on the GPU race.  Asynchronous on `stream`
 * (cudaStream_t, NULL = default stream); allocates nothing. */
ICEMPM_API int icempm_cell_order_noalloc(const uint32_t *d_cell, const uint32_t *d_utility, uint32_t n,
                                         int32_t grid_y, uint32_t *d_order, uint32_t *d_count, void *stream);

/* Grid arrays of a saved frame (SnapshotManager::PrepareFrameArrays,
 * snapshotmanager.cpp:623-765), computed on the GPU from the points on the
 * device.  Each pointer is a host buffer of the caller (NULL skips that
 * array): G = GridXTotal * GridYTotal floats for the ten channels, 3G bytes
 * of interleaved colour, G bytes of mass mask and of points per cell, and
 * 2 * ICEMPM_MAX_REGIONS floats of (fx, fy) boundary force per region. */
typedef struct icempm_frame_t {
    float *point_density, *mass, *vx, *vy, *Jpinv, *P, *Q, *r, *g, *b;
    uint8_t *rgb;
    uint8_t *mass_mask;
    uint8_t *count;
    float *forces_per_region;
} icempm_frame_t;

/* point_colors_rgb[pid] = 0xRRGGBB by point id (GPU_Implementation5::
 * point_colors_rgb); NULL or ids >= ncolors colour points white.  The boundary
 * forces are divided by elapsed_steps * dt as icempm_get_boundary_forces does. */
ICEMPM_API int icempm_prepare_frame(icempm_t *ctx, const uint32_t *point_colors_rgb, uint32_t ncolors,
                                    int32_t elapsed_steps, icempm_frame_t *out);

/* ---- Ensembles (many scenes per launch; no counterpart in the reference) ---
 * Many independent scenes advanced together: one launch of the grid update
 * and one of the fused kernel per sub-step cover every scene of the batch,
 * captured in CUDA graphs.  Each scene is an ordinary context (created,
 * uploaded, downloaded, queried, sorted and compacted through the calls
 * above); all contexts of a batch share the variant and the device and must
 * outlive the batch.  The batch advances all scenes in lockstep: sub-step
 * index first_step .. first_step+nsteps-1 for each, at each scene's own dt. */
typedef struct icempm_batch icempm_batch_t;

typedef struct icempm_batch_tuning_t {
    int32_t tile_nodes;    /* shared scatter tile of the fused kernel: 0 (none: node sums go
                              straight to the global accumulators), 512 or 1024 nodes */
    int32_t stages;        /* bulk-copy stages of point state: 1 or 2 (2 without a tile only) */
    int32_t sort_every;    /* locality sort of every scene each this many sub-steps; 0 = never */
    int32_t graph_steps;   /* sub-steps per CUDA graph; 0 = direct launches */
    float ms_per_step;     /* set by icempm_batch_autotune: the chosen form's time per sub-step */
    int32_t reserved[3];
} icempm_batch_tuning_t;

ICEMPM_API int icempm_batch_create(icempm_t *const *contexts, int32_t count, icempm_batch_t **out);
ICEMPM_API int icempm_batch_destroy(icempm_batch_t *batch);
/* Blocks until the sub-steps are done (the contexts' own calls may follow). */
ICEMPM_API int icempm_batch_step(icempm_batch_t *batch, int32_t nsteps, int32_t first_step);
/* Project autotuner: times the kernel shapes and sort cadences on the live
 * scenes (which advance by 4 * trial_steps sub-steps, indices from first_step)
 * and keeps the fastest; the choice is returned in *out (may be NULL). */
ICEMPM_API int icempm_batch_autotune(icempm_batch_t *batch, int32_t trial_steps, int32_t first_step,
                                     icempm_batch_tuning_t *out);
ICEMPM_API int icempm_batch_set_tuning(icempm_batch_t *batch, const icempm_batch_tuning_t *tuning);
ICEMPM_API int icempm_batch_get_tuning(icempm_batch_t *batch, icempm_batch_tuning_t *tuning);
/* ms[0] = device time of the last icempm_batch_step; ms[1..3] = 0. */
ICEMPM_API int icempm_batch_timings(icempm_batch_t *batch, float ms[4]);
ICEMPM_API int icempm_batch_launch_count(icempm_batch_t *batch, uint64_t *count);

/* ---- Learned return map (no counterpart in the reference) -----------------
 * An MLP 4 -> 64 -> 64 -> 3 (SiLU) that stands in for the projection of a
 * trial state onto the Drucker-Prager yield surface (wolper_dp's case 3,
 * kernels.cuh:411-467).  A trial state is 4 floats (sigma1 >= sigma2 of Fe,
 * Jp_inv, thickness); inputs x = (log sigma1, log sigma2, log Jp_inv,
 * log thickness), outputs y = (log sigma1'/sigma1, log sigma2'/sigma2,
 * log Jp_inv'/Jp_inv), both standardised: norm[14] = x mean[4], x std[4],
 * y mean[3], y std[3].  Parameters: 4675 floats, row-major W1[64][4] b1[64]
 * W2[64][64] b2[64] W3[3][64] b3[3].  All pointers d_* are device memory of
 * the caller; calls are asynchronous on `stream` (cudaStream_t, NULL =
 * default). */
ICEMPM_API int icempm_mlp_param_count(void);
/* d_grad += gradient of mean_s sum_o (y_o - y_ref_o)^2 over n standardised
 * samples d_x[n][4], d_y[n][3]; *d_loss += that loss. */
ICEMPM_API int icempm_mlp_grad(const float *d_params, const float *d_x, const float *d_y, uint32_t n,
                               float *d_grad, float *d_loss, void *stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8; t counts from 1). */
ICEMPM_API int icempm_mlp_adam(float *d_params, const float *d_grad, float *d_m, float *d_v, int32_t t, float lr,
                               void *stream);
/* FP32 forward of the standardised outputs d_y[n][3]. */
ICEMPM_API int icempm_mlp_forward(const float *d_params, const float *d_x, uint32_t n, float *d_y, void *stream);
/* The exact map on trial states d_trial[n][4] -> d_out[n][4] (sigma1',
 * sigma2', Jp_inv', 0), in FP32 or (fp64 != 0) FP64 arithmetic. */
ICEMPM_API int icempm_return_map_exact(const icempm_simparams_t *prms, const float *d_trial, uint32_t n,
                                       float *d_out, int32_t fp64, void *stream);
/* The learned map: BF16 tensor-core inference with FP32 accumulation for the
 * trial states that project onto the yield surface; the others take the exact
 * closed forms.  A network answer whose yield residual |q' - q_yield(p')| /
 * q_yield(p') exceeds tol is replaced by the exact map (counted in
 * *d_fallbacks, which the call adds to).  d_out[n][4] = (sigma1', sigma2',
 * Jp_inv', 0 exact / 1 network / 2 fallback). */
ICEMPM_API int icempm_return_map_learned(const icempm_simparams_t *prms, const float *d_params, const float *d_norm,
                                         const float *d_trial, uint32_t n, float tol, float *d_out,
                                         uint32_t *d_fallbacks, void *stream);
/* The learned map on the step path: from now on the fused kernel sends every
 * crushed point's projection onto the yield surface (wolper_dp case 3,
 * kernels.cuh:400-467, as called from partition_kernel_g2p, kernels.cuh:271-283)
 * to the network, evaluated in place by BF16 tensor-core MMAs with FP32
 * accumulation over the warp's points; an answer off the yield surface by
 * more than tol (as icempm_return_map_learned) is replaced by the exact map.
 * d_params (ICEMPM mlp parameters) and d_norm (14 floats) are device
 * pointers, packed at the call; d_params NULL switches the network off.
 * FP32-state variants only.  Resets the counts below. */
ICEMPM_API int icempm_set_learned_map(icempm_t *ctx, const float *d_params, const float *d_norm, float tol);
/* Projections the network answered (*kept) and those that fell back to the
 * exact map (*fallbacks) since icempm_set_learned_map.  Synchronises. */
ICEMPM_API int icempm_learned_map_counts(icempm_t *ctx, uint64_t *kept, uint64_t *fallbacks);
/* Training data from a run: from now on the fused kernel records up to
 * `capacity` projections (trial, projected) of crushed points with
 * (index + sub-step) % stride == 0.  icempm_harvest_end copies the records
 * (8 floats each: sigma1, sigma2, Jp_inv, thickness, sigma1', sigma2',
 * Jp_inv', 3) to `records`, sets *count to the number offered (may exceed
 * capacity) and stops recording. */
ICEMPM_API int icempm_harvest_begin(icempm_t *ctx, uint32_t capacity, int32_t stride);
ICEMPM_API int icempm_harvest_end(icempm_t *ctx, float *records, uint32_t capacity, uint32_t *count);

/* Message of the last failing call on this thread ("" if none). */
ICEMPM_API const char *icempm_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* ICEMPM_H */
