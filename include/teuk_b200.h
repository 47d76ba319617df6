/*
 * teuk_b200.h -- C ABI of the B200 (sm_100a) engine for the teuk-kokkos RK4
 * right-hand-side hot path: the spin -2 Teukolsky spatial pipeline
 * (SBP radial operators, fixed-m spin-weighted-harmonic transforms with the
 * implicit Kerr ell-coupling, band projection) and its classical RK4 stage
 * update.
 *
 * Every entry point replaces one member of the reference's C++ interface:
 *
 *   teuk_b200_create            SpatialPipeline::SpatialPipeline
 *                               (include/teuk/spatial_pipeline.hpp:163-363)
 *   teuk_b200_destroy           ~SpatialPipeline
 *   teuk_b200_shape             SpatialPipelineStorage::snapshot_shape
 *                               (include/teuk/pipeline_storage.hpp:114-117)
 *   teuk_b200_set_state         Kokkos::deep_copy into storage().state()
 *                               (include/teuk/pipeline_bands.hpp:215-231)
 *   teuk_b200_get_state         deep_copy out of storage().state()
 *                               (include/teuk/pipeline_checkpoint.hpp:820-830)
 *   teuk_b200_evaluate_rhs      SpatialPipeline::evaluate_rhs_at_time
 *                               (include/teuk/spatial_pipeline.hpp:458-588)
 *   teuk_b200_step              SpatialPipeline::step, repeated
 *                               (include/teuk/spatial_pipeline.hpp:590-620;
 *                               include/teuk/device_rk4.hpp:84-128)
 *   teuk_b200_initialize_gaussian
 *                               initialize_compactified_gaussian_pulse
 *                               (include/teuk/pipeline_initial_data.hpp:211-339)
 *   teuk_b200_sample_endpoint   EndpointWaveformSampler::sample
 *                               (include/teuk/waveform_output.hpp:75-160)
 *   teuk_b200_get_activation / teuk_b200_restore_activation /
 *   teuk_b200_reset_activation  SpatialPipeline::source_activation_state /
 *                               restore_source_activation /
 *                               reset_source_activation
 *                               (include/teuk/spatial_pipeline.hpp:386-420)
 *   teuk_b200_last_error        the std::invalid_argument / runtime_error
 *                               message the reference would throw
 *   teuk_b200_checkpoint_write / teuk_b200_checkpoint_load
 *                               write_pipeline_checkpoint /
 *                               load_pipeline_checkpoint_verified
 *                               (include/teuk/pipeline_checkpoint.hpp:782-936)
 *   teuk_b200_diagnostics_sample
 *                               PipelineDiagnostics::sample_pipeline
 *                               (include/teuk/pipeline_diagnostics.hpp:143-345)
 *   teuk_b200_parse_run_config / teuk_b200_resolved_config
 *                               parse_run_configuration_text /
 *                               resolved_configuration_text
 *                               (include/teuk/config.hpp:683-831)
 *   teuk_b200_step_static_scratch
 *                               no counterpart: teuk_b200_step with its RK
 *                               slopes in a static device array
 *
 * Batched variants (teuk_b200_batch_*) pack many independent solves of
 * uneven shape into one set of stage launches, and the server
 * (teuk_b200_server_*) admits, advances and retires such solves
 * continuously; neither has a counterpart in the reference, whose driver
 * runs one pipeline per process (include/teuk/solver_driver.hpp:86-353).
 *
 * Conventions.  State arrays are complex128 stored as interleaved
 * (real, imag) doubles in the reference's (mode, field, radial, theta)
 * order with theta contiguous and 13 fields (include/teuk/fields.hpp:27-28,
 * include/teuk/pipeline_storage.hpp:18-33).  A `memory` argument says
 * whether a pointer is host (TEUK_B200_HOST) or CUDA device
 * (TEUK_B200_DEVICE) memory.  Every call returns TEUK_B200_OK or a negative
 * status; teuk_b200_last_error() then holds the message (thread-local).
 * No call falls back to a CPU implementation: when the CUDA kernels cannot
 * run, create fails with TEUK_B200_ERR_CUDA.
 */
#ifndef TEUK_B200_H
#define TEUK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TEUK_B200_ABI_VERSION 1

enum teuk_b200_status {
  TEUK_B200_OK = 0,
  TEUK_B200_ERR_INVALID_ARGUMENT = -1, /* std::invalid_argument */
  TEUK_B200_ERR_RUNTIME = -2,          /* std::runtime_error */
  TEUK_B200_ERR_CUDA = -3,             /* CUDA launch / allocation failure */
  TEUK_B200_ERR_UNSUPPORTED = -4,      /* valid reference input not yet
                                          built on the B200 path */
  TEUK_B200_ERR_OUT_OF_MEMORY = -5
};

enum teuk_b200_memory { TEUK_B200_HOST = 0, TEUK_B200_DEVICE = 1 };

/* include/teuk/radial_discretization.hpp:17 */
enum teuk_b200_discretization {
  TEUK_B200_D42 = 0,
  TEUK_B200_D84 = 1,
  TEUK_B200_D105 = 2
};

/* include/teuk/teukolsky.hpp:148-151 */
enum teuk_b200_reduction {
  TEUK_B200_FREE_DAMPED = 0,
  TEUK_B200_STAGE_CONSTRAINED = 1
};

/* include/teuk/spatial_pipeline.hpp:40-53 */
enum teuk_b200_source_mode {
  TEUK_B200_SOURCE_DISABLED = 0,
  TEUK_B200_SOURCE_CONSTRAINT_AWARE = 1,
  TEUK_B200_SOURCE_UNRESTRICTED = 2
};

/* Field slots of the 13-field state (include/teuk/pipeline_storage.hpp:18-33) */
enum teuk_b200_field {
  TEUK_B200_FIRST_P = 0,
  TEUK_B200_FIRST_Q = 1,
  TEUK_B200_FIRST_PSI = 2,
  TEUK_B200_FIELD_COUNT = 13
};

enum teuk_b200_boundary { TEUK_B200_SCRI = 0, TEUK_B200_HORIZON = 1 };

/* Constructor arguments of SpatialPipeline plus the ModeRegistry lists
 * (include/teuk/modes.hpp:42-80).  Mode lists may be given in any order;
 * they are sorted and checked exactly like ModeRegistry does. */
typedef struct teuk_b200_config {
  int abi_version; /* TEUK_B200_ABI_VERSION */
  double mass;
  double spin;
  double compactification_length;
  int radial_points;  /* nr: uniform grid on [0, L^2 / r_+] */
  int theta_nodes;    /* Gauss-Legendre nodes */
  int ell_max_first;  /* PipelineAngularBands::ell_max_first */
  int ell_max_second; /* PipelineAngularBands::ell_max_second */
  int mode_count;
  const int* modes;   /* stored signed m */
  int parent_count;
  const int* parents; /* first-order modes */
  int target_count;
  const int* targets; /* second-order modes */
  double reduction_damping;
  double dissipation;
  int reduction;      /* enum teuk_b200_reduction */
  int discretization; /* enum teuk_b200_discretization */
  int source_mode;    /* enum teuk_b200_source_mode */
  double source_start_time;
  double normalized_constraint_tolerance;
  int required_consecutive_passes;
} teuk_b200_config;

/* SourceActivationState (include/teuk/source_activation.hpp) */
typedef struct teuk_b200_activation {
  int active;
  double activation_time;
  int consecutive_passes;
  double last_eligibility_time;
} teuk_b200_activation;

/* GaussianPulseMode / PipelineGaussianPulse
 * (include/teuk/pipeline_initial_data.hpp:24-57).  center and width are
 * compactified radii (not fractions of R_H). */
typedef struct teuk_b200_gaussian_mode {
  int ell;
  int m;
  double amplitude_real;
  double amplitude_imag;
} teuk_b200_gaussian_mode;

typedef struct teuk_b200_gaussian {
  double center;
  double width;
  int compact_support;
  int mode_count;
  const teuk_b200_gaussian_mode* modes;
} teuk_b200_gaussian;

/* One endpoint waveform record (include/teuk/waveform_output.hpp:23-32). */
typedef struct teuk_b200_waveform_record {
  int boundary; /* enum teuk_b200_boundary */
  int order;    /* 1 = first-order field, 2 = second-order field */
  int m;
  int ell;
  double rescaled_real;
  double rescaled_imag;
  double endpoint_real;
  double endpoint_imag;
} teuk_b200_waveform_record;

typedef struct teuk_b200_pipeline teuk_b200_pipeline;
typedef struct teuk_b200_batch teuk_b200_batch;

const char* teuk_b200_last_error(void);
int teuk_b200_abi_version(void);
/* The CUDA device that pipelines, batches and servers created afterwards on
 * the calling thread use (cudaSetDevice inside the engine).  The engine links
 * the CUDA runtime statically, so a device chosen through another copy of
 * the runtime (a framework's, an application's) does not reach it; a
 * process driving one GPU per rank or thread selects it here.  No
 * counterpart in the reference (its execution space picks the device at
 * Kokkos::initialize). */
int teuk_b200_set_device(int device);
int teuk_b200_get_device(int* device);

/* ---- single pipeline (one solve) ------------------------------------- */
int teuk_b200_create(const teuk_b200_config* config,
                     teuk_b200_pipeline** out);
int teuk_b200_destroy(teuk_b200_pipeline* pipeline);
/* shape[4] = {modes, 13, radial, theta} */
int teuk_b200_shape(const teuk_b200_pipeline* pipeline, size_t shape[4]);
/* Values count = modes*13*radial*theta complex numbers. */
int teuk_b200_set_state(teuk_b200_pipeline* pipeline, const double* state,
                        size_t complex_count, int memory);
int teuk_b200_get_state(teuk_b200_pipeline* pipeline, double* state,
                        size_t complex_count, int memory);
/* RHS of a caller-supplied stage (same layout).  Stage fields that lie
 * outside the retained fixed-m bands are projected onto them first; every
 * stage the pipeline itself produces is already in band. */
int teuk_b200_evaluate_rhs(teuk_b200_pipeline* pipeline, const double* stage,
                           double* output, size_t complex_count, double time,
                           int memory);
/* Advance `steps` classical RK4 steps of size dt from `time`. */
int teuk_b200_step(teuk_b200_pipeline* pipeline, double time, double dt,
                   int steps);
/* Same steps as teuk_b200_step without allocating device memory: the three
 * RK slope buffers come from one static device array of 3 x 524,288
 * complex128 values (24 MiB) instead of the pipeline's own.  No counterpart
 * in the reference, which always steps through a workspace it allocated.
 * - For callers that cannot allocate at step time (a framework allocator
 *   that already holds the device, a latency budget without room for a
 *   driver allocation call).
 * - Linear (disabled-source) pipelines whose band state holds at most
 *   524,288 complex values; larger ones, and second-order pipelines, are
 *   rejected (TEUK_B200_ERR_INVALID_ARGUMENT / _UNSUPPORTED) before any
 *   device work.
 * - The first call on each device resolves the array's address (a module
 *   load); make it once before any stream capture.
 * - The array is shared by every pipeline on a device: calls that overlap
 *   in time on one device (other threads, other streams) race on it.
 *   Serialize them.
 * - Nothing in the array needs to start at zero.
 * - The array's device address is cached per device for the life of the
 *   process.  A cudaDeviceReset in the host process frees the array with
 *   the context and leaves that address stale: do not call this entry
 *   point on a device after resetting it. */
int teuk_b200_step_static_scratch(teuk_b200_pipeline* pipeline, double time,
                                  double dt, int steps);

/* Failure-detection test hook, not for production use.  Batches and
 * pipelines built after a call with chunk >= 0 withhold that chunk from CTA
 * 0 of their stage-1 streaming launches: the kernel's bounded waits for it
 * run out (about 2 s) and the step reports TEUK_B200_ERR_CUDA ("stage kernel
 * pipeline wait timed out") with the CUDA context still usable.  chunk = -1
 * (the initial value) switches it off.  Process-wide. */
int teuk_b200_test_withhold_chunk(int chunk);
int teuk_b200_initialize_gaussian(teuk_b200_pipeline* pipeline,
                                  const teuk_b200_gaussian* pulse);
/* Records for the scri then horizon endpoints of the first-order field and
 * then the second-order field, in the reference's order.  `capacity` is the
 * number of records `out` can hold; `count` receives the number written. */
int teuk_b200_sample_endpoint(teuk_b200_pipeline* pipeline,
                              teuk_b200_waveform_record* out,
                              size_t capacity, size_t* count);
int teuk_b200_get_activation(const teuk_b200_pipeline* pipeline,
                             teuk_b200_activation* out);
int teuk_b200_restore_activation(teuk_b200_pipeline* pipeline,
                                 const teuk_b200_activation* state);
int teuk_b200_reset_activation(teuk_b200_pipeline* pipeline);
/* Bind the pipeline's launches to a caller cudaStream_t (NULL = the
 * pipeline's own stream). */
int teuk_b200_set_stream(teuk_b200_pipeline* pipeline, void* cuda_stream);
int teuk_b200_synchronize(teuk_b200_pipeline* pipeline);
/* Pipeline checkpoint format v5 of the reference: `directory` receives
 * metadata.txt (key=value provenance, geometry, activation, progress and
 * the FNV-1a 64 checksum) and state.bin (the 13-field state as interleaved
 * little-endian binary64).  `time_step` is the run's step, recorded as
 * provenance.  write_pipeline_checkpoint
 * (include/teuk/pipeline_checkpoint.hpp:782-857). */
int teuk_b200_checkpoint_write(teuk_b200_pipeline* pipeline,
                               const char* directory, double time_step,
                               double time, uint64_t step);
/* load_pipeline_checkpoint_verified (pipeline_checkpoint.hpp:869-936):
 * format, registry, numerical configuration (incl. time_step), geometry,
 * size, checksum and band-limit checks all pass before the pipeline's
 * state and activation latch change; *time and *step receive the recorded
 * progress. */
int teuk_b200_checkpoint_load(teuk_b200_pipeline* pipeline,
                              const char* directory, double time_step,
                              double* time, uint64_t* step);
/* PipelineDiagnostics::sample_pipeline (include/teuk/pipeline_diagnostics.hpp
 * :143-345): RMS and maximum of every stored field and of its last stored
 * right-hand side, of the two reduction constraints Q - D psi, of the
 * source and the forcing, plus the latch and source-constraint summary.
 * All reductions run on the device; a nonfinite value fails the call with
 * the reference's message. */
typedef struct teuk_b200_norm {
  double rms;
  double maximum;
} teuk_b200_norm;

typedef struct teuk_b200_diagnostics {
  teuk_b200_norm state[TEUK_B200_FIELD_COUNT];
  teuk_b200_norm rhs[TEUK_B200_FIELD_COUNT];
  teuk_b200_norm first_reduction_constraint;
  teuk_b200_norm second_reduction_constraint;
  teuk_b200_norm source_over_r3;
  teuk_b200_norm forcing;
  double independent_reconstruction_constraint_maximum;
  /* SourceConstraintNorms of the last latch check: psi3 Bianchi, psi2
   * Bianchi, h_ll reality */
  double constraint_absolute_maximum[3];
  double constraint_normalized_maximum[3];
  double constraint_weighted_rms[3];
  double constraint_normalized_weighted[3];
  double constraint_controlling_normalized;
  int constraints_finite;
  teuk_b200_activation activation;
  int second_order_source_active;
  size_t point_count;
  int scri_finite;
  int horizon_finite;
  int all_finite;
} teuk_b200_diagnostics;

int teuk_b200_diagnostics_sample(teuk_b200_pipeline* pipeline,
                                 teuk_b200_diagnostics* out);
/* Device bytes held by one pipeline built from `config` (admission). */
int teuk_b200_footprint_bytes(const teuk_b200_config* config,
                              size_t* bytes);

/* ---- batched solves: one set of stage launches for all instances -----
 * Linear solves (source disabled) of any mix of shapes and
 * discretizations.  Second-order solves batch only as identical
 * configurations with the Unrestricted source from t = 0: they become the
 * replicas of one nodal pipeline, whose RHS launches serve all of them at
 * once; each replica's results equal the solve alone bit for bit.  Such a
 * batch starts at t = 0 and keeps its own time; it shares one dt across its
 * instances, has no band endpoint coefficients (Unsupported) and no fixed
 * launch count (Unsupported).  Any other batch holding a second-order
 * configuration is Unsupported. */
int teuk_b200_batch_create(const teuk_b200_config* configs, int count,
                           teuk_b200_batch** out);

/* Launch choices of a batch.  None of them changes a result bit: bands do
 * not couple, every radial row gets the same sums in the same order however
 * the rows are split into strips, and the split-precision transforms are a
 * separate, stated precision (TEUK_B200_PRECISION_SPLIT).  No counterpart in
 * the reference (kernel selection and tuning of this engine). */
enum teuk_b200_stage_kernel_choice {
  TEUK_B200_KERNEL_AUTO = 0, /* streaming kernel for every band that fits */
  TEUK_B200_KERNEL_TILE = 1  /* tile kernel for every band */
};
enum teuk_b200_precision {
  /* FP64 transforms and ell-coupling (the reference's arithmetic) */
  TEUK_B200_PRECISION_FP64 = 0,
  /* split-precision tensor-core transforms: FP64 operands cut into BF16
   * slices, FP32 accumulation, FP64 recombination; everything else FP64 */
  TEUK_B200_PRECISION_SPLIT = 1
};
typedef struct teuk_b200_batch_options {
  int abi_version;  /* TEUK_B200_ABI_VERSION */
  int stage_kernel; /* teuk_b200_stage_kernel_choice */
  int precision;    /* teuk_b200_precision */
  /* streaming-kernel strip length in radial rows (0: the autotuner's or the
   * built-in choice; otherwise at least 64) */
  int strip_rows;
  /* 1: time the candidate strip lengths (64 to 4096 rows) of every
   * streaming launch group at build and keep the fastest (cached per shape
   * class for the process) */
  int autotune;
} teuk_b200_batch_options;
/* teuk_b200_create with launch choices (one solve; the second-order
 * pipeline reads `precision` only). */
int teuk_b200_create_with_options(const teuk_b200_config* config,
                                  const teuk_b200_batch_options* options,
                                  teuk_b200_pipeline** out);
int teuk_b200_batch_create_with_options(const teuk_b200_config* configs,
                                        int count,
                                        const teuk_b200_batch_options* options,
                                        teuk_b200_batch** out);
/* Strip length (rows) each streaming launch group of the batch uses, in
 * launch-group order; `count` gets the number of groups written (at most
 * `capacity`).  Groups that run the tile kernel report 0. */
int teuk_b200_batch_strip_rows(const teuk_b200_batch* batch, int* rows,
                               int capacity, int* count);
int teuk_b200_batch_destroy(teuk_b200_batch* batch);
int teuk_b200_batch_size(const teuk_b200_batch* batch, int* count);
int teuk_b200_batch_shape(const teuk_b200_batch* batch, int instance,
                          size_t shape[4]);
int teuk_b200_batch_set_state(teuk_b200_batch* batch, int instance,
                              const double* state, size_t complex_count,
                              int memory);
int teuk_b200_batch_get_state(teuk_b200_batch* batch, int instance,
                              double* state, size_t complex_count,
                              int memory);
int teuk_b200_batch_initialize_gaussian(teuk_b200_batch* batch, int instance,
                                        const teuk_b200_gaussian* pulse);
/* One RK4 step of size dt[i] for every instance i, `steps` times.  With
 * graph != 0 the four stage launches of a step are replayed from a
 * captured CUDA graph. */
int teuk_b200_batch_step(teuk_b200_batch* batch, const double* dt, int steps,
                         int graph);
int teuk_b200_batch_sample_endpoint(teuk_b200_batch* batch, int instance,
                                    teuk_b200_waveform_record* out,
                                    size_t capacity, size_t* count);
/* Per-instance endpoint Psi modal coefficients gathered on the device for
 * every instance at once: (instance, boundary, mode, ell) complex values in
 * the batch's packed order; `count` receives the complex count. */
int teuk_b200_batch_endpoint_modal(teuk_b200_batch* batch, double* out,
                                   size_t capacity, size_t* count,
                                   int memory);
int teuk_b200_batch_set_stream(teuk_b200_batch* batch, void* cuda_stream);
int teuk_b200_batch_synchronize(teuk_b200_batch* batch);
/* Kernel launches issued per RK4 step (for launch accounting). */
int teuk_b200_batch_launches_per_step(const teuk_b200_batch* batch,
                                      int* launches);
/* Launch groups (per discretization, reduction and kernel) whose stages run
 * a streaming kernel (persistent CTAs over radial strips: n_ell <= 16 and at
 * most 32 Gauss-Legendre nodes, or, free-damped, n_ell <= 24 and at most 48
 * nodes) and those that run the tile kernel.  No counterpart in the
 * reference: kernel selection of this engine. */
int teuk_b200_batch_stage_kernels(const teuk_b200_batch* batch,
                                  int* streaming_groups, int* tile_groups);

/* ---- runtime configuration (.cfg) --------------------------------------
 * The teuk_solver schema (include/teuk/config.hpp): `key = value` lines,
 * '#' comments, `key=value` command-line overrides, unknown keys rejected,
 * the reference's defaults, validation order and messages.  The plus2
 * companion keys are accepted and validated as schema only. */
#define TEUK_B200_MAX_MODES 64
#define TEUK_B200_MAX_SEEDS 64
#define TEUK_B200_PATH_CAPACITY 1024

typedef struct teuk_b200_run_config {
  int abi_version;                /* TEUK_B200_ABI_VERSION */
  double mass, spin, compactification_length;
  int radial_points, theta_nodes, ell_max_first, ell_max_second;
  int mode_count, modes[TEUK_B200_MAX_MODES];       /* stored registry */
  int parent_count, parents[TEUK_B200_MAX_MODES];   /* first_order_modes */
  int target_count, targets[TEUK_B200_MAX_MODES];   /* second_order_modes */
  double reduction_damping, dissipation;
  int reduction, discretization;
  int source_mode;  /* disabled unless second_order.enabled */
  double source_start_time, normalized_constraint_tolerance;
  int required_consecutive_passes;
  double final_time;
  int steps;
  double cfl;
  double time_step;               /* final_time / steps */
  int initial_data_type;          /* 0 gaussian, 1 checkpoint */
  double center, width;           /* compactified radii (fraction * R_H) */
  int compact_support;
  int seed_count;                 /* after the sharp-partner expansion */
  teuk_b200_gaussian_mode seeds[TEUK_B200_MAX_SEEDS];
  char checkpoint_directory[TEUK_B200_PATH_CAPACITY];
  char output_directory[TEUK_B200_PATH_CAPACITY];
  int diagnostic_every, checkpoint_every;
} teuk_b200_run_config;

/* parse_run_configuration_text: `text` is the .cfg content, `overrides`
 * are `key=value` strings applied on top. */
int teuk_b200_parse_run_config(const char* text, const char* const* overrides,
                               int override_count, teuk_b200_run_config* out);
/* The pipeline configuration of a parsed run (make_run_mode_registry,
 * make_source_policy); its mode pointers refer to `run`'s arrays. */
int teuk_b200_run_pipeline_config(const teuk_b200_run_config* run,
                                  teuk_b200_config* out);
/* resolved_configuration_text of the parsed run (the body of
 * resolved_config.cfg); *length receives the byte count (excluding the
 * terminating zero written when it fits). */
int teuk_b200_resolved_config(const char* text, const char* const* overrides,
                              int override_count, char* out, size_t capacity,
                              size_t* length);

/* ---- serving: continuous batching of solve requests --------------------
 * No counterpart in the reference (one solve per process).  Requests are
 * queued by teuk_b200_server_submit and admitted in arrival order while
 * the device footprint of the admitted set stays within the budget; every
 * admitted solve keeps its state on the device and advances inside the
 * shared batched RK4 step; a solve that reaches its step count leaves the
 * batch with its endpoint waveform records, and its memory and tile slots
 * go to the next queued requests.  Linear (disabled-source) solves only.
 * Device memory: every buffer of the batch comes from the server's own
 * CUDA memory pool (stream-ordered on the server's stream), warmed with
 * min(budget, 4 GiB) at creation; memory a layout change frees stays in the
 * pool until teuk_b200_server_destroy, so a membership change makes no
 * driver allocation and no device-wide free. */
typedef struct teuk_b200_server teuk_b200_server;

typedef struct teuk_b200_server_options {
  int abi_version;          /* TEUK_B200_ABI_VERSION */
  size_t hbm_budget_bytes;  /* device bytes the admitted solves may hold */
  int max_active;           /* cap on concurrent solves (0 = no cap) */
  int graph;                /* replay each batched step from a CUDA graph */
  int precision;            /* teuk_b200_precision of every admitted solve */
} teuk_b200_server_options;

typedef struct teuk_b200_server_stats {
  int queued;                 /* submitted, not admitted yet */
  int active;                 /* in the batch */
  int finished;               /* results ready */
  long long steps;            /* batched steps run */
  double grid_point_updates;  /* sum over solves of steps * modes * nr * ntheta */
  double device_seconds;      /* device time of the batched steps */
  size_t resident_bytes;      /* device bytes of the current batch */
  int rebuilds;               /* batch layouts built on membership changes */
  double rebuild_seconds;     /* host time spent building them (incl.
                                 initial data of admitted solves) */
} teuk_b200_server_stats;

int teuk_b200_server_create(const teuk_b200_server_options* options,
                            teuk_b200_server** out);
int teuk_b200_server_destroy(teuk_b200_server* server);
/* Queue one solve: Gaussian initial data `pulse`, `steps` RK4 steps of
 * size dt from time 0.  Validation (the reference's constructor checks and
 * the budget) happens here; *id identifies the request. */
int teuk_b200_server_submit(teuk_b200_server* server,
                            const teuk_b200_config* config,
                            const teuk_b200_gaussian* pulse, double dt,
                            int steps, uint64_t* id);
/* Admit queued requests that fit, run up to `steps` batched RK4 steps
 * (fewer when every admitted solve finishes), retire finished solves.
 * *active receives the number of solves still in the batch. */
int teuk_b200_server_advance(teuk_b200_server* server, int steps,
                             int* active);
/* Endpoint waveform records of a finished request (the records
 * teuk_b200_sample_endpoint gives after the same steps) and its
 * time-to-waveform in seconds from submit to retirement.  Returns
 * TEUK_B200_ERR_INVALID_ARGUMENT with "request is not finished" while it
 * is queued or running. */
int teuk_b200_server_result(teuk_b200_server* server, uint64_t id,
                            teuk_b200_waveform_record* out, size_t capacity,
                            size_t* count, double* latency_seconds);
int teuk_b200_server_stats_get(const teuk_b200_server* server,
                               teuk_b200_server_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* TEUK_B200_H */
