/*
 * fenix_cuda.h — C ABI of libfenixcuda.so, a B200 (sm_100a) CUDA implementation of
 * fenix's per-frame combustion-volume simulation step.
 *
 * Each entry point replaces one member of the reference's simulation object,
 * `CombustionVolumeSimulation`
 * (src/engine/simulation/runtime/combustion-volume-simulation/types.ts:62-76),
 * created by `createCombustionVolumeSimulation(device, options)`
 * (src/engine/simulation/runtime/createCombustionVolumeSimulation.ts:39-53).
 * Each declaration below cites the reference member it replaces.
 *
 * Conventions
 *  - All functions are `extern "C"`. They take plain pointers and sizes and return
 *    fx_status (0 = FX_OK, < 0 = FX_ERR_*). No C++ exception crosses the ABI.
 *  - A handle is thread-affine: use one host thread per fx_sim.
 *  - fx_sim_step only enqueues work on the simulation's CUDA stream and does not
 *    wait for it. This matches the reference, where step() records into the
 *    caller's encoder and the caller submits. Calls that return data to the host
 *    (read_field, get_stats with counts, synchronize) wait for the stream.
 *  - After the first failure a handle keeps a sticky error string
 *    (fx_sim_last_error). Failures before a handle exists are reported through
 *    fx_last_error().
 *  - Device pointers are returned as uint64_t (a bigint under bun:ffi).
 *  - Parameters are latched at the next fx_sim_step, as in the reference.
 */
#ifndef FENIX_CUDA_H
#define FENIX_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FX_ABI_VERSION 1

typedef int32_t fx_status;
#define FX_OK 0
#define FX_ERR_INVALID_ARGUMENT (-1)
#define FX_ERR_CUDA (-2)
#define FX_ERR_OUT_OF_MEMORY (-3)
#define FX_ERR_STATE (-4)
#define FX_ERR_TIMEOUT (-5)
#define FX_ERR_UNSUPPORTED (-6)

typedef struct fx_sim fx_sim;

/* ScalarAdvectionMode (types.ts:4): 'semi-lagrangian' | 'maccormack'. */
#define FX_ADVECT_SEMI_LAGRANGIAN 0
#define FX_ADVECT_MACCORMACK 1

/* SimulationQualitySettings (types.ts:6-14). Values are JS numbers in the
 * reference, so they are doubles here. Setters round and clamp them exactly as
 * createSimulationQualitySettings does (types.ts:26-44). A NaN is rejected with
 * FX_ERR_INVALID_ARGUMENT. */
typedef struct fx_quality {
  double pressure_interval;    /* 1..16 */
  double vorticity_interval;   /* 1..16 */
  double fine_pre_iterations;  /* 0..32 */
  double fine_post_iterations; /* 0..32 */
  double mid_pre_iterations;   /* 0..32 */
  double mid_post_iterations;  /* 0..32 */
  double coarse_iterations;    /* 0..64 */
} fx_quality;

#define FX_QUALITY_PRESSURE_INTERVAL (1u << 0)
#define FX_QUALITY_VORTICITY_INTERVAL (1u << 1)
#define FX_QUALITY_FINE_PRE (1u << 2)
#define FX_QUALITY_FINE_POST (1u << 3)
#define FX_QUALITY_MID_PRE (1u << 4)
#define FX_QUALITY_MID_POST (1u << 5)
#define FX_QUALITY_COARSE (1u << 6)
#define FX_QUALITY_ALL (0x7Fu)

/* SimulationRuntimeParams (types.ts:46-58). A field mask stands for Partial<>. */
typedef struct fx_runtime_params {
  double wind[3];
  double wind_strength;
  double gravity[3];
  double gravity_strength;
  double buoyancy;
  double vorticity_strength;
  double vorticity_constant_mask;
  double vorticity_velocity_mask;
  double vorticity_heat_mask;
  double vorticity_density_mask;
  double world_size;
} fx_runtime_params;

#define FX_PARAM_WIND (1u << 0)
#define FX_PARAM_WIND_STRENGTH (1u << 1)
#define FX_PARAM_GRAVITY (1u << 2)
#define FX_PARAM_GRAVITY_STRENGTH (1u << 3)
#define FX_PARAM_BUOYANCY (1u << 4)
#define FX_PARAM_VORTICITY_STRENGTH (1u << 5)
#define FX_PARAM_VORTICITY_CONSTANT_MASK (1u << 6)
#define FX_PARAM_VORTICITY_VELOCITY_MASK (1u << 7)
#define FX_PARAM_VORTICITY_HEAT_MASK (1u << 8)
#define FX_PARAM_VORTICITY_DENSITY_MASK (1u << 9)
#define FX_PARAM_WORLD_SIZE (1u << 10)
#define FX_PARAM_ALL (0x7FFu)

/* Kernel paths. Both compute the reference step and give identical results. */
#define FX_KERNELS_FUSED 0 /* default: fused, brick-list-driven kernels */
#define FX_KERNELS_PLAIN 1 /* one kernel per reference WGSL pass (the plain FP32 step) */

/* Option flags (extensions). The first two do not change results. */
#define FX_OPT_DEBUG_FIELDS (1u << 0) /* always write vorticity, |vorticity|, |F_conf| */
#define FX_OPT_NO_GRAPHS (1u << 1)    /* launch kernels directly instead of CUDA graphs */
/* FP16 storage of the scalar sets (density, temperature, fuel, reaction); fused
 * kernels only (FX_ERR_UNSUPPORTED with FX_KERNELS_PLAIN). Arithmetic stays f32;
 * every value a reference pass stores into a scalar buffer is rounded to
 * binary16, stochastically unless FX_OPT_F16_ROUND_NEAREST (below) is given.
 * Velocity and pressure stay f32. Field reads
 * and writes still exchange f32 (writes are rounded), and the render buffers
 * report FX_DTYPE_F16. */
#define FX_OPT_SCALARS_F16 (1u << 2)
/* With FX_OPT_SCALARS_F16: round every binary16 scalar store to nearest (ties to
 * even). Without it the stores round stochastically: to one of the two
 * neighbouring binary16 values, up with probability equal to the distance from
 * the lower one in units of their spacing, by a hash of the voxel, the store
 * site and the step index. Round-to-nearest holds a value still when a step
 * changes it by less than half a binary16 spacing (slow smoke decay), a bias
 * that stochastic rounding removes. */
#define FX_OPT_F16_ROUND_NEAREST (1u << 4)
/* Sparse mode (extension; fused kernels and the reference pressure schedule
 * only). The reference computes velocity advection, curl, confinement,
 * divergence, the fine pressure sweeps and the projection over the whole grid
 * (runtime/createCombustionVolumeSimulation.ts:270-296). In sparse mode velocity
 * advection runs in the bricks flagged in the current scalar set, and the
 * others in U = the bricks flagged in the current or the next set; velocity and
 * the fine pressure and divergence are 0 outside those bricks. Scalar passes,
 * injection and the mid and coarse pressure levels are unchanged. Results
 * differ from the reference where the velocity outside the active bricks
 * matters; fx_sim_set_sparse switches it at run time. */
#define FX_OPT_SPARSE (1u << 3)

/* CombustionVolumeSimulationOptions (createCombustionVolumeSimulation.ts:39-48).
 * Fill with fx_sim_options_default() and then override fields. */
typedef struct fx_sim_options {
  uint32_t struct_size;           /* sizeof(fx_sim_options) */
  uint32_t width, height, depth;  /* resolution; 0 = reference default 128 x 256 x 128 */
  int32_t scalar_advection_mode;  /* FX_ADVECT_*; default maccormack */
  uint32_t runtime_mask;          /* FX_PARAM_* bits of `runtime` that are given */
  fx_runtime_params runtime;      /* options.wind/windStrength/gravity/gravityStrength/worldSize (+ the rest) */
  uint32_t quality_mask;          /* FX_QUALITY_* bits of `quality` that are given */
  fx_quality quality;             /* options.qualitySettings */
  int32_t device;                 /* CUDA device ordinal */
  int32_t kernels;                /* FX_KERNELS_* */
  uint32_t flags;                 /* FX_OPT_* */
  void* stream;                   /* cudaStream_t to enqueue on; NULL = the simulation's own stream */
} fx_sim_options;

/* getRenderBuffers() (createCombustionVolumeSimulation.ts:306-312): the current
 * scalar set, the current brick flags and the packed brick layout
 * (sim/sparse/createSparseBrickLayout.ts:28-38). Device pointers stay valid until
 * fx_sim_destroy; which buffers form the current set alternates every step. */
typedef struct fx_render_buffers {
  uint64_t density;
  uint64_t temperature;
  uint64_t fuel;
  uint64_t reaction;
  uint64_t active_brick_flags; /* uint32 per brick, 1 = active */
  uint32_t active_brick_info[8];
  uint32_t width, height, depth;
  int32_t dtype; /* FX_DTYPE_F32, or FX_DTYPE_F16 (IEEE binary16) with FX_OPT_SCALARS_F16 */
} fx_render_buffers;

#define FX_DTYPE_F32 0
#define FX_DTYPE_F16 1

/* getDebugBuffers() (createCombustionVolumeSimulation.ts:313-326). */
typedef struct fx_debug_buffers {
  fx_render_buffers render;
  uint64_t velocity_magnitude;
  uint64_t divergence;
  uint64_t pressure;
  uint64_t vorticity_magnitude;
  uint64_t confinement_force_magnitude;
} fx_debug_buffers;

/* Field ids for fx_sim_read_field / fx_sim_write_field. Scalar and velocity fields
 * are f32 of width*height*depth voxels (x fastest); flags are uint32 per brick;
 * pressure-level fields have the level's own voxel count. */
enum {
  FX_FIELD_DENSITY = 0, FX_FIELD_TEMPERATURE, FX_FIELD_FUEL, FX_FIELD_REACTION,
  FX_FIELD_PREV_DENSITY, FX_FIELD_PREV_TEMPERATURE, FX_FIELD_PREV_FUEL, FX_FIELD_PREV_REACTION,
  FX_FIELD_VELOCITY_X, FX_FIELD_VELOCITY_Y, FX_FIELD_VELOCITY_Z,
  FX_FIELD_VELOCITY_SCRATCH_X, FX_FIELD_VELOCITY_SCRATCH_Y, FX_FIELD_VELOCITY_SCRATCH_Z,
  FX_FIELD_VORTICITY_X, FX_FIELD_VORTICITY_Y, FX_FIELD_VORTICITY_Z,
  FX_FIELD_VORTICITY_MAGNITUDE, FX_FIELD_CONFINEMENT_MAGNITUDE, FX_FIELD_VELOCITY_MAGNITUDE,
  FX_FIELD_BRICK_FLAGS, FX_FIELD_PREV_BRICK_FLAGS,
  FX_FIELD_FINE_DIVERGENCE, FX_FIELD_FINE_PRESSURE_A, FX_FIELD_FINE_PRESSURE_B,
  FX_FIELD_MID_DIVERGENCE, FX_FIELD_MID_PRESSURE_A, FX_FIELD_MID_PRESSURE_B,
  FX_FIELD_COARSE_DIVERGENCE, FX_FIELD_COARSE_PRESSURE_A, FX_FIELD_COARSE_PRESSURE_B,
  FX_FIELD_PRESSURE,
  FX_FIELD_COUNT
};

/* Host-visible counters of a simulation. */
typedef struct fx_stats {
  int64_t step_index;          /* simulationStepIndex */
  int32_t current_scalar_set;  /* currentScalarSet (0 or 1) */
  int32_t last_pressure_buffer;/* lastPressureBuffer: 0 = 'a', 1 = 'b' */
  uint32_t brick_count;        /* bricks of 8^3 voxels */
  uint32_t active_bricks;      /* bricks flagged in the current flags (waits for the stream) */
  uint32_t kernels_per_step;   /* kernels the last step launched */
  uint32_t flags;              /* FX_STATS_* */
} fx_stats;

#define FX_STATS_GRAPH (1u << 0)      /* the last step replayed a captured CUDA graph */
#define FX_STATS_GRAPHS_OFF (1u << 1) /* graphs are off (FX_OPT_NO_GRAPHS, or capture failed) */

/* Version of this ABI (FX_ABI_VERSION). */
int32_t fx_abi_version(void);

/* Message of the last failure on this thread that had no handle to record it. */
const char* fx_last_error(void);

/* Fills `opt` with the reference defaults (createCombustionVolumeSimulation.ts:54,
 * 181,194-204; types.ts:16-24). */
void fx_sim_options_default(fx_sim_options* opt);

/* createCombustionVolumeSimulation(device, options)
 * (createCombustionVolumeSimulation.ts:50-401). Allocates and zeroes every buffer. */
fx_status fx_sim_create(const fx_sim_options* opt, fx_sim** out);

/* dispose() (createCombustionVolumeSimulation.ts:384-399). NULL is ignored. */
void fx_sim_destroy(fx_sim* sim);

/* step(encoder, elapsedSeconds, stepSeconds) (createCombustionVolumeSimulation.ts:230-305).
 * Enqueues one step on the simulation's stream. */
fx_status fx_sim_step(fx_sim* sim, double elapsed_seconds, double step_seconds);

/* getRenderBuffers() (createCombustionVolumeSimulation.ts:306-312). */
fx_status fx_sim_get_render_buffers(fx_sim* sim, fx_render_buffers* out);

/* getDebugBuffers() (createCombustionVolumeSimulation.ts:313-326). Like the
 * reference, this requests the |v| debug pass on the next step. */
fx_status fx_sim_get_debug_buffers(fx_sim* sim, fx_debug_buffers* out);

/* getScalarAdvectionMode() / setScalarAdvectionMode(mode)
 * (createCombustionVolumeSimulation.ts:327-337). */
fx_status fx_sim_get_scalar_advection_mode(fx_sim* sim, int32_t* mode);
fx_status fx_sim_set_scalar_advection_mode(fx_sim* sim, int32_t mode);

/* getRuntimeParams() / setRuntimeParams(Partial<params>)
 * (createCombustionVolumeSimulation.ts:338-365). `mask` selects the given fields. */
fx_status fx_sim_get_runtime_params(fx_sim* sim, fx_runtime_params* out);
fx_status fx_sim_set_runtime_params(fx_sim* sim, const fx_runtime_params* params, uint32_t mask);

/* getQualitySettings() / setQualitySettings(Partial<settings>)
 * (createCombustionVolumeSimulation.ts:366-377). */
fx_status fx_sim_get_quality(fx_sim* sim, fx_quality* out);
fx_status fx_sim_set_quality(fx_sim* sim, const fx_quality* quality, uint32_t mask);

/* updateSources(sources) (createCombustionVolumeSimulation.ts:378-380 →
 * runtime/passes/SourceInjectionPass.ts:71-83). `packed` holds count * 32 floats in
 * the layout of sim/emitters/packEmitterSources.ts:13-77 (128 bytes per source). */
fx_status fx_sim_update_sources(fx_sim* sim, const float* packed, uint32_t count);

/* reset() (createCombustionVolumeSimulation.ts:381-383 → doReset :206-226). */
fx_status fx_sim_reset(fx_sim* sim);

/* resolution (types.ts:63). */
fx_status fx_sim_get_resolution(fx_sim* sim, uint32_t* width, uint32_t* height, uint32_t* depth);

/* Readback and upload of one field (no reference counterpart: the reference
 * reads buffers only through its renderer). Waits for the stream. `bytes` must
 * equal the field's size. */
fx_status fx_sim_field_size(fx_sim* sim, int32_t field_id, size_t* bytes);
fx_status fx_sim_read_field(fx_sim* sim, int32_t field_id, void* host_dst, size_t bytes);
fx_status fx_sim_write_field(fx_sim* sim, int32_t field_id, const void* host_src, size_t bytes);

/* Saved state (extension). The state is what doReset of
 * createCombustionVolumeSimulation.ts:206-226 re-initialises and the next step
 * reads: the host clock (current scalar set, step index, start and last elapsed
 * seconds, the initialized flag, the latest pressure buffer), the current scalar
 * set as stored (f32 or binary16), the velocity, the fine pressure of the latest
 * solve (the V-cycle's warm start) and the brick flags of both sets. Settings
 * (quality, runtime parameters, sources, solver, kernels) are not part of it.
 * fx_sim_state_bytes gives the size of the blob; save copies it to `dst` (host
 * or device memory, waits for the stream). Load accepts a blob of a simulation
 * with the same resolution and scalar storage (else FX_ERR_INVALID_ARGUMENT,
 * reported through fx_last_error, and the simulation is unchanged and usable),
 * clears everything else as fx_sim_reset does, and
 * the steps that follow give the same bits as the steps that followed the save. */
fx_status fx_sim_state_bytes(fx_sim* sim, uint64_t* bytes);
fx_status fx_sim_save_state(fx_sim* sim, void* dst, uint64_t bytes);
fx_status fx_sim_load_state(fx_sim* sim, const void* src, uint64_t bytes);

/* Waits until all enqueued work of the simulation has finished. */
fx_status fx_sim_synchronize(fx_sim* sim);

/* Counters; active_bricks waits for the stream. */
fx_status fx_sim_get_stats(fx_sim* sim, fx_stats* out);

/* Instrumentation (no reference counterpart; the reference's only timing is a
 * stats-gl overlay, src/engine/render/renderer/createViewportRuntime.ts:236-268).
 * FX_INSTR_KERNEL_TIMES brackets every kernel with CUDA events on the
 * simulation's stream; FX_INSTR_COUNT_ACTIVE adds, after every step, the step's
 * active bricks and their voxels to device-side counters. */
#define FX_INSTR_KERNEL_TIMES (1u << 0)
#define FX_INSTR_COUNT_ACTIVE (1u << 1)
#define FX_INSTR_SOLVER_NORMS (1u << 2) /* FP64 solver statistics after the reference schedule too */

typedef struct fx_kernel_time {
  char name[48];
  uint32_t launches;
  uint32_t reserved;
  double total_ms;
} fx_kernel_time;

fx_status fx_sim_set_instrumentation(fx_sim* sim, uint32_t flags);

/* Per-kernel totals since the last call (waits for the stream, then resets).
 * Writes up to `capacity` entries and the number of distinct kernels to *count. */
fx_status fx_sim_read_kernel_times(fx_sim* sim, fx_kernel_time* out, uint32_t capacity, uint32_t* count);

/* Active bricks and active voxels summed over the steps since the last call
 * (waits for the stream, then resets). */
fx_status fx_sim_read_active_counters(fx_sim* sim, uint64_t* brick_steps, uint64_t* voxel_steps);

/* The CUDA stream the simulation enqueues on (cudaStream_t). */
fx_status fx_sim_get_stream(fx_sim* sim, void** stream);

/* The sticky error message of a handle ("" when none). */
const char* fx_sim_last_error(fx_sim* sim);

/* Pressure solver (extension; no counterpart in the reference, whose solve is the
 * fixed schedule of sim/runtime/passes/PressureSolvePass.ts:68-84, set through
 * fx_quality). FX_SOLVER_VCYCLE runs weighted-Jacobi V-cycles over `levels`
 * levels (the reference's level sizes, buffers.ts:10-16): `pre_sweeps` and
 * `post_sweeps` per level, `coarse_sweeps` on the coarsest, the coarse
 * right-hand side 4 x the mean of the 8 fine residuals, the reference's
 * trilinear prolongation. It stops when ||div - A p||_2 <= tolerance * ||div||_2
 * (both FP64, on the device) or after max_cycles cycles, and can start from the
 * previous step's pressure. Both kernel paths: the fused one's loop is a
 * conditional WHILE node decided on the device under CUDA graphs; the plain
 * one's is a host loop over one-voxel kernels. tolerance 0 with max_cycles N
 * is a fixed schedule of N cycles per step. Not in sparse mode. */
#define FX_SOLVER_REFERENCE 0
#define FX_SOLVER_VCYCLE 1

typedef struct fx_solver_settings {
  int32_t mode;          /* FX_SOLVER_*; default FX_SOLVER_REFERENCE */
  int32_t levels;        /* 2..6; default 5 */
  int32_t pre_sweeps;    /* 0..32; default 4 */
  int32_t post_sweeps;   /* 0..32; default 4 */
  int32_t coarse_sweeps; /* 0..256; default 20 */
  int32_t max_cycles;    /* 1..1000; default 30 */
  int32_t warm_start;    /* 1: start from the previous pressure; default 1 */
  int32_t reserved;
  double omega;          /* Jacobi weight in (0, 1]; default 2/3 */
  double tolerance;      /* relative residual; default 1e-5 */
} fx_solver_settings;

void fx_solver_settings_default(fx_solver_settings* out);
fx_status fx_sim_set_solver(fx_sim* sim, const fx_solver_settings* settings);
fx_status fx_sim_get_solver(fx_sim* sim, fx_solver_settings* out);

/* FP64 statistics of the latest pressure solve (waits for the stream): the
 * norms of the divergence and of the final residual, their ratio, the max
 * |div u| of the projected velocity over interior voxels, and the V-cycles run.
 * Filled by FX_SOLVER_VCYCLE steps, and by reference-schedule steps while
 * FX_INSTR_SOLVER_NORMS is set. */
typedef struct fx_solver_stats {
  double rhs_l2;
  double residual_l2;
  double relative_residual;
  double max_abs_divergence;
  int32_t cycles;
  int32_t converged;
} fx_solver_stats;

fx_status fx_sim_read_solver_stats(fx_sim* sim, fx_solver_stats* out);

/* Sparse mode on (1) or off (0) from the next step (see FX_OPT_SPARSE). No
 * counterpart in the reference. FX_ERR_UNSUPPORTED with the plain kernels or
 * the V-cycle solver. */
fx_status fx_sim_set_sparse(fx_sim* sim, int32_t on);
fx_status fx_sim_get_sparse(fx_sim* sim, int32_t* on);

/* Autotuning (extension): times every sweep kernel variant of the pressure
 * solve on each level (fine, mid, coarse) of this simulation's grid and keeps
 * the fastest for its later steps, where it beats the level's default by at
 * least 3 % (else the default). All variants give the same bits. Waits for
 * the stream; overwrites the pressure buffers that are not current (the
 * non-current fine buffer and the mid/coarse levels, which every solve
 * rewrites from zero). */
typedef struct fx_autotune_report {
  int32_t sweep_variant[3]; /* chosen variant per level (0..8) */
  float sweep_us[3];        /* its time per sweep */
  float default_us[3];      /* the default variant's time per sweep */
} fx_autotune_report;

fx_status fx_sim_autotune(fx_sim* sim, fx_autotune_report* out);
/* Sets the sweep variant of each level directly (a cached autotuning result):
 * -1 keeps the default; a variant that does not fit the level's width is
 * FX_ERR_INVALID_ARGUMENT. Variants: 0-2 one x per thread at z-depth 2/4/8,
 * 3-4 two x per thread (even widths) at z-depth 2/4, 5-7 four x per thread
 * (widths divisible by 4) at z-depth 2/4/1, 8 four x per thread marching runs
 * of planes with the next plane's loads in flight (widths divisible by 4). */
fx_status fx_sim_set_sweep_variants(fx_sim* sim, const int32_t variants[3]);
fx_status fx_sim_get_sweep_variants(fx_sim* sim, int32_t variants[3]);

/* Grids of the brick-list kernels (extension; the reference dispatches one
 * workgroup of 4^3 threads per 4^3 voxels, runtime/combustion-volume-simulation/
 * constants.ts:3 and runtime/shared/createVolumeDispatch.ts:5-38). Each such
 * kernel runs SMs x ctas_per_sm blocks (at most one per brick), every block
 * walking the brick list with a stride of the grid, so the results do not
 * depend on the choice. Index: FX_BK_*. 0 keeps the default (8); else 1..64. */
#define FX_BRICK_KERNELS 11
#define FX_BK_INJECT 0
#define FX_BK_ADVECT_SCALARS 1
#define FX_BK_COMBUSTION 2
#define FX_BK_BUOYANCY 3
#define FX_BK_SPARSE_ADVECT_VELOCITY 4
#define FX_BK_SPARSE_VORTICITY 5
#define FX_BK_SPARSE_CONFINEMENT 6
#define FX_BK_SPARSE_DIV_FIRST_SWEEP 7
#define FX_BK_SPARSE_SWEEP 8
#define FX_BK_SPARSE_PROLONG_FINE 9
#define FX_BK_SPARSE_PROJECT 10
fx_status fx_sim_set_brick_ctas(fx_sim* sim, const int32_t ctas_per_sm[FX_BRICK_KERNELS]);
fx_status fx_sim_get_brick_ctas(fx_sim* sim, int32_t ctas_per_sm[FX_BRICK_KERNELS]);

/* Times the brick kernels' grids and keeps the fastest per kernel (extension).
 * The timing runs on a clone: a second simulation with this one's settings,
 * sources and saved state (fx_sim_save_state), stepped `steps` times (1..64,
 * after one warm-up step) from that state for each of 2, 4, 8, 16 and 32 CTAs
 * per SM, with per-kernel CUDA events. The simulation itself is only read (its
 * stream is waited for), and the clone is destroyed before the call returns;
 * it needs the memory of a second simulation for that time. A grid replaces the
 * default only when it is at least 3 % faster. Kernels that did not run (the
 * sparse ones in dense mode) keep the default and report 0 us. Fused kernels
 * only. The choice enters the step's CUDA-graph key. */
typedef struct fx_brick_tune_report {
  int32_t ctas_per_sm[FX_BRICK_KERNELS]; /* chosen (8 where the default stays) */
  float us[FX_BRICK_KERNELS];            /* its time per step */
  float default_us[FX_BRICK_KERNELS];    /* the default grid's time per step */
} fx_brick_tune_report;

fx_status fx_sim_autotune_bricks(fx_sim* sim, double step_seconds, int32_t steps, fx_brick_tune_report* out);

/* Batches (extension; the reference steps one simulation per device): many
 * independent simulations, each with its own options (sizes may differ), stepped
 * together. Every fx_batch_step is one CUDA graph in which each simulation's
 * device work is a separate branch, so they run concurrently from one launch.
 * The members are ordinary fx_sim handles owned by the batch: use them for
 * params, quality, sources, solver, field reads and writes; do not destroy them.
 * fx_sim_step on a member steps that member alone. Fused kernels only. */
typedef struct fx_batch fx_batch;

fx_status fx_batch_create(const fx_sim_options* const* options, uint32_t count, fx_batch** out);
void fx_batch_destroy(fx_batch* batch);
fx_status fx_batch_size(fx_batch* batch, uint32_t* count);
fx_status fx_batch_get_sim(fx_batch* batch, uint32_t index, fx_sim** sim);
/* One step of every member (each member's reference schedule, parameters and
 * sources), enqueued on the batch stream. */
fx_status fx_batch_step(fx_batch* batch, double elapsed_seconds, double step_seconds);
fx_status fx_batch_synchronize(fx_batch* batch);
fx_status fx_batch_get_stream(fx_batch* batch, void** stream);
const char* fx_batch_last_error(fx_batch* batch);

/* Volume raymarch: the reference's VolumeRaymarchPass
 * (src/engine/render/passes/createVolumeRaymarchPass.ts:15-29), whose fragment
 * shader (:300-726) runs as a CUDA kernel into a headless RGBA device buffer
 * instead of a WebGPU render target. It reads a simulation's render buffers
 * (the current scalar set and brick flags, f32 or FP16) and skips inactive
 * bricks as the shader does. */
#define FX_MAX_RENDER_LIGHTS 3
#define FX_LIGHT_DIRECTIONAL 0
#define FX_LIGHT_POINT 1

/* OrbitCameraSnapshot (src/engine/scene/camera/createOrbitCameraController.ts:11-19). */
typedef struct fx_camera {
  double position[3];
  double target[3];
  double forward[3];
  double right[3];
  double up[3];
  double aspect;
  double tan_half_fov_y;
} fx_camera;

/* RenderLight (src/engine/render/lighting/renderLight.ts:3-9). */
typedef struct fx_render_light {
  int32_t type; /* FX_LIGHT_* */
  int32_t reserved;
  double direction[3];
  double position[3];
  double color[3];
  double intensity;
} fx_render_light;

/* RaymarchRenderParams (createVolumeRaymarchPass.ts:8-13); the mask stands for
 * Partial<>, and the values are clamped as setRenderParams does (:268-281). */
typedef struct fx_raymarch_params {
  uint32_t mask;        /* FX_RM_* */
  uint32_t light_count; /* with FX_RM_LIGHTS: lights[0..light_count) (at most 3 are kept) */
  double step_count;    /* rounded, then clamped to [32, 4096] (the reference has no upper bound) */
  double scattering_forward; /* clamped to [0, 0.98] */
  double scattering_back;    /* clamped to [-0.98, 0] */
  fx_render_light lights[FX_MAX_RENDER_LIGHTS];
} fx_raymarch_params;

#define FX_RM_STEP_COUNT (1u << 0)
#define FX_RM_LIGHTS (1u << 1)
#define FX_RM_SCATTER_FORWARD (1u << 2)
#define FX_RM_SCATTER_BACK (1u << 3)

/* VolumeDisplayMode (src/engine/render/volumetrics/volumeDisplayMode.ts). */
#define FX_DISPLAY_TEMPERATURE 0
#define FX_DISPLAY_DENSITY 1
#define FX_DISPLAY_FUEL 2

#define FX_PIXELS_RGBA16F 0 /* 4 x IEEE binary16 per pixel */
#define FX_PIXELS_RGBA32F 1 /* 4 x float per pixel */
#define FX_PIXELS_RGBA8 2   /* 4 x unorm8 per pixel (the canvas): round(clamp(x, 0, 1) * 255) */

typedef struct fx_raymarch fx_raymarch;

/* createVolumeRaymarchPass(device, format, resolution) (:81-91): world bounds
 * and the default step count of the resolution, the default light. */
fx_status fx_raymarch_create(uint32_t width, uint32_t height, uint32_t depth, fx_raymarch** out);
void fx_raymarch_destroy(fx_raymarch* pass);
/* setRenderParams (:268-281). */
fx_status fx_raymarch_set_params(fx_raymarch* pass, const fx_raymarch_params* params);
/* render(encoder, view, buffers, camera, displayMode, width, height, elapsed)
 * (:184-266): fills `pixels`, a device buffer of render_width * render_height
 * RGBA pixels (row 0 at the top, premultiplied colour; (0, 0, 0, 0) where the
 * reference's fragment discards), on the simulation's stream. The simulation
 * must have the pass's resolution. */
fx_status fx_raymarch_render(fx_raymarch* pass, fx_sim* sim, const fx_camera* camera, int32_t display_mode, uint32_t render_width,
                             uint32_t render_height, double elapsed_seconds, void* pixels, int32_t pixel_format);

/* Bloom: the reference's BloomPass (src/engine/render/passes/createBloomPass.ts),
 * from the raymarch's HDR image (RGBA16F, or RGBA32F) to the canvas image: a
 * soft threshold into a half-resolution RGBA16F texture, a 9-tap gaussian blur
 * along x then y, and the composite with pow(., 0.92) (or the blit when
 * disabled). textureSample is bilinear with exact f32 weights and clamp-to-edge
 * addressing. The pass owns its half-resolution textures (allocated on the
 * first render of a size). */
typedef struct fx_bloom_params { /* BloomParams (createBloomPass.ts:1-6) */
  int32_t enabled;
  int32_t reserved;
  double threshold;
  double strength;
  double radius;
} fx_bloom_params;

typedef struct fx_bloom fx_bloom;
fx_status fx_bloom_create(fx_bloom** out);  /* createBloomPass(device, canvasFormat), on the current device */
void fx_bloom_destroy(fx_bloom* pass);
/* render(encoder, sourceView, targetView, width, height, params) (:96-130):
 * `hdr` and `out` are device buffers of width * height pixels (row 0 at the
 * top); out_format FX_PIXELS_RGBA8 or FX_PIXELS_RGBA32F; stream: cudaStream_t. */
fx_status fx_bloom_render(fx_bloom* pass, const void* hdr, int32_t hdr_format, uint32_t width, uint32_t height,
                          const fx_bloom_params* params, void* out, int32_t out_format, void* stream);

/* Differentiable rollout: an extension with no counterpart in the reference.
 * K FP32 steps of a simulation (f32 storage, the reference pressure schedule,
 * MacCormack advection, pressure and vorticity intervals of 1) from its current
 * state, with a control patch of per-voxel
 * inflow velocity: after inject-velocity, every step sets velocity.y at
 * (inflow_x0 + i, inflow_y, inflow_z0 + k) to inflow[i + inflow_nx * k]. The loss
 * is sum over voxels of (density_K - target)^2 (FP64 accumulation). Step k runs
 * at elapsed = start_elapsed + k * step_seconds with step = step_seconds.
 *
 * The adjoint differentiates the plain step; with FX_KERNELS_FUSED the forward
 * and the recomputed (taped) steps run the fused kernels, which give the same
 * bits (unless an inflow value exceeds the speed limit, when every step is
 * plain).
 * fx_rollout_forward leaves the simulation in its final state and keeps a state
 * checkpoint every checkpoint_interval steps; fx_rollout_backward returns the
 * gradient of the loss with respect to the inflow values and the initial
 * velocity field by the adjoint of every pass, recomputing each segment from its
 * checkpoint, and leaves the simulation in the forward's final state again.
 * The recomputation records each step's tape (27 fields of width * height *
 * depth floats per step of a segment, allocated by fx_rollout_create when they
 * take at most half of the device's free memory); without that allocation each
 * step is re-run taped just before its adjoint, with the same result.
 * Brick flags, emitter sources and the step uniform are constants of the
 * differentiation; a branch (min, max, clamp, the MacCormack limiter) passes the
 * adjoint of the operand it selected. */
typedef struct fx_rollout_desc {
  uint32_t struct_size;
  uint32_t steps;               /* K (default 64) */
  uint32_t checkpoint_interval; /* k (default 8) */
  uint32_t reserved0;
  double start_elapsed;         /* elapsed seconds of step 0 */
  double step_seconds;          /* default 1/60 */
  uint32_t inflow_x0, inflow_y, inflow_z0;
  uint32_t inflow_nx, inflow_nz; /* 0 x 0: no control patch */
  uint32_t reserved1;
} fx_rollout_desc;

typedef struct fx_rollout fx_rollout;
void fx_rollout_desc_default(fx_rollout_desc* desc);
/* The rollout borrows `sim`: every call but fx_rollout_destroy needs it alive. */
fx_status fx_rollout_create(fx_sim* sim, const fx_rollout_desc* desc, fx_rollout** out);
void fx_rollout_destroy(fx_rollout* rollout);
/* target: width * height * depth host floats (x fastest). */
fx_status fx_rollout_set_target(fx_rollout* rollout, const float* target);
/* inflow: inflow_nx * inflow_nz host floats; *loss receives the loss. */
fx_status fx_rollout_forward(fx_rollout* rollout, const float* inflow, double* loss);
/* grad_inflow: inflow_nx * inflow_nz host floats; grad_velocity: NULL or
 * 3 * width * height * depth host floats (the x, y, z planes). */
fx_status fx_rollout_backward(fx_rollout* rollout, float* grad_inflow, float* grad_velocity);

/* Brick flags of caller-owned fields, allocating nothing. No counterpart in the
 * reference. It computes what compute-active-bricks.wgsl.ts:35-58 computes, for
 * the density, temperature and reaction fields (width*height*depth floats each,
 * x fastest) on the current device. It writes one uint32 flag (0 or 1) per 8^3
 * brick to `flags` (ceil(w/8)*ceil(h/8)*ceil(d/8) entries, x fastest) and
 * enqueues on `stream` (cudaStream_t, NULL for the legacy stream).
 *
 * It is for callers that cannot allocate device memory at the time of the
 * call: a per-frame loop, where a cudaFree would wait for the whole device, or
 * a process whose device memory its own arena has already reserved. It calls no
 * cudaMalloc or cudaFree and no allocating library routine. Its scratch is a
 * 1 MiB static device array, one summary byte per brick, so grids above
 * 1,048,576 bricks are rejected with FX_ERR_INVALID_ARGUMENT before any CUDA
 * call. The first call on a device is its set-up: it looks up that array's
 * address (cudaGetSymbolAddress) with the device current, and, as CUDA 12
 * loads modules lazily by default, that is when the driver loads the module
 * holding the array and the kernels onto the device. So make one call (any
 * small grid) before an arena reserves the rest of device memory, or set
 * CUDA_MODULE_LOADING=EAGER; later calls take no device memory. The first call
 * should also come before any stream capture. The address is cached per device
 * ordinal and does not survive cudaDeviceReset. Nothing has to start at zero.
 * There is one scratch array per device, so two calls in flight at once on one
 * device race; calls on one stream are ordered. Launch errors come from the
 * launches themselves, so an error pending from earlier unrelated work is left
 * alone. Errors go to fx_last_error(). */
fx_status fx_brick_flags_noalloc(const float* density, const float* temperature, const float* reaction, uint32_t width,
                                 uint32_t height, uint32_t depth, uint32_t* flags, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FENIX_CUDA_H */
