/* pvb200.h — C ABI of the B200-native point-vortex backend (libpvb200.so).
 *
 * The library evaluates the direct O(N^2) Biot–Savart velocity of point vortices in the
 * three geometries of jplaurie/PointVortex (infinite plane with core radius, Weiss–McWilliams
 * periodic square box, disk with circle-theorem images) on an NVIDIA B200 (sm_100a), and runs
 * the reference's RK4 and DOPRI5 steps with the state resident in GPU memory.
 *
 * Every entry point replaces one member of the reference's link-time backend interface
 * (src/backend.h:9-16) or of its VelocityKernel class (src/compute.h:18-36); the comment above
 * each one names it. Plain pointers and sizes only; all arrays are structure-of-arrays
 * doubles (src/vortex.h:15-51). Unless stated otherwise pointers are HOST pointers.
 *
 * Errors: every function returns a pv_status. The codes map one to one onto the exception
 * types the reference throws (std::invalid_argument, std::out_of_range, std::runtime_error,
 * std::logic_error); pv_last_error() returns the message, which follows the reference's text.
 *
 * Threading: a context belongs to one host thread at a time. Work is ordered on the
 * context's own CUDA stream; functions that return results to the host synchronise it.
 */
#ifndef PVB200_H
#define PVB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PVB200_ABI_VERSION 1

typedef enum pv_status {
    PV_OK = 0,
    PV_ERROR_INVALID_ARGUMENT = 1, /* std::invalid_argument */
    PV_ERROR_OUT_OF_RANGE = 2,     /* std::out_of_range */
    PV_ERROR_RUNTIME = 3,          /* std::runtime_error (non-finite, coincident, DOPRI5 failure) */
    PV_ERROR_LOGIC = 4,            /* std::logic_error (hook used out of order) */
    PV_ERROR_CUDA = 5,             /* CUDA runtime failure; the message names the call */
    PV_ERROR_CAPACITY = 6          /* batch admission: no free slot or no room in the arena */
} pv_status;

typedef enum pv_geometry {
    PV_GEOMETRY_INFINITE = 0, /* boundaryCondition infinite (src/params.h:56) */
    PV_GEOMETRY_PERIODIC = 1, /* boundaryCondition periodic */
    PV_GEOMETRY_DISK = 2      /* boundaryCondition disk */
} pv_geometry;

typedef enum pv_precision {
    PV_PRECISION_FP64 = 0, /* plain FP64 pair sums (the reference's arithmetic) */
    PV_PRECISION_FP32C = 1 /* FP32 bulk pair sums, compensated, FP64 where cancellation needs it */
} pv_precision;

/* The SimParams fields (src/params.h:37-78) that the velocity path reads. */
typedef struct pv_params {
    int geometry;          /* pv_geometry */
    double core_radius;    /* coreRadius (infinite plane only) */
    double box_length_x;   /* boxLengthX (periodic) */
    double box_length_y;   /* boxLengthY (periodic; must equal boxLengthX) */
    int image_layers;      /* periodicImageLayers, 0..64 */
    double disk_radius;    /* diskRadius (disk) */
    int precision;         /* pv_precision */
} pv_params;

/* StepResult, src/compute.h:11-16 */
typedef struct pv_step_result {
    double accepted_time_step;
    double suggested_time_step;
    double normalized_error;
    unsigned rejected_steps;
} pv_step_result;

/* One close-dipole candidate of DipoleManager::process (src/dipole.cpp:49-78):
 * second == population marks a disk wall-image candidate. */
typedef struct pv_dipole_candidate {
    uint64_t first;
    uint64_t second;
    double distance_squared;
} pv_dipole_candidate;

typedef struct pv_context pv_context;

/* ---- lifecycle -------------------------------------------------------------------------- */

/* makeBackendKernel (src/backend.h:16) with the kernel constructors' validation
 * (src/compute.cpp:50-56, 165-173, 258-261). device: CUDA ordinal. */
pv_status pv_context_create(const pv_params *params, int device, pv_context **out);
/* ~VelocityKernel; frees every device buffer of the context. */
void pv_context_destroy(pv_context *ctx);
/* Message of the last failure on ctx, or, when ctx is NULL, of the calling thread's last failed
 * call that takes no context. Valid until the next call on the same context/thread. */
const char *pv_last_error(const pv_context *ctx);
/* backendName (src/backend.h:13). */
const char *pv_backend_name(void);
/* backendRuntimeDetails (src/backend.h:14): "key value" lines, NUL-terminated in buf. */
pv_status pv_runtime_details(int device, char *buf, size_t len);

/* ---- host-array evaluation ---------------------------------------------------------------- */

/* VelocityKernel::evaluateRange (src/compute.h:26-28; src/compute.cpp:88, 203, 286):
 * velocities of targets [begin, end) due to all n sources, written to u[0..end-begin) and
 * v[0..end-begin). Does not touch the context's device-resident state. */
pv_status pv_evaluate_range(pv_context *ctx, const double *x, const double *y,
                            const double *circulation, size_t n, size_t begin, size_t end,
                            double *u, double *v);
/* VelocityKernel::evaluate (src/compute.cpp:57-69): full range plus the finiteness check. */
pv_status pv_evaluate(pv_context *ctx, const double *x, const double *y,
                      const double *circulation, size_t n, double *u, double *v);
/* VelocityKernel::hamiltonian (src/compute.h:29): computed on the GPU. */
pv_status pv_hamiltonian(pv_context *ctx, const double *x, const double *y,
                         const double *circulation, size_t n, double *hamiltonian);
/* computeInvariants(vortices, kernel) (src/compute.cpp:157-163):
 * out[0..4] = circulation, linear impulse x, linear impulse y, angular impulse, Hamiltonian. */
pv_status pv_invariants(pv_context *ctx, const double *x, const double *y,
                        const double *circulation, size_t n, double out[5]);

/* ---- device-resident state (the VelocityKernel device-stepping hooks) --------------------- */

/* uploadDeviceState (src/compute.h:31). Validates like the reference (finite data; periodic
 * zero total circulation; disk positions inside). Invalidates the DOPRI5 FSAL derivative. */
pv_status pv_upload_state(pv_context *ctx, const double *x, const double *y,
                          const double *circulation, size_t n);
/* downloadDeviceState (src/compute.h:32): n must equal the uploaded population. */
pv_status pv_download_state(pv_context *ctx, double *x, double *y, size_t n);
/* evaluateDeviceState (src/compute.h:33): velocities of the device state. */
pv_status pv_evaluate_state(pv_context *ctx, double *u, double *v, size_t n);
/* deviceRk4Step (src/compute.h:34); semantics of RungeKuttaIntegrator::rk4Step
 * (src/timestep.cpp:31-61). The state is unchanged when the step fails. */
pv_status pv_rk4_step(pv_context *ctx, double dt);
/* deviceDopri5Step (src/compute.h:35); semantics of RungeKuttaIntegrator::dopri5Step
 * (src/timestep.cpp:62-120): FSAL, max-norm error, step-size control and rejections all run
 * on the GPU; one host synchronisation per attempt. */
pv_status pv_dopri5_step(pv_context *ctx, double dt, double absolute_tolerance,
                         double relative_tolerance, double minimum_time_step,
                         double maximum_time_step, pv_step_result *result);
/* invalidateDeviceDerivative (src/compute.h:36). */
pv_status pv_invalidate_derivative(pv_context *ctx);
/* computeInvariants of the device state (src/compute.cpp:157-163), out as pv_invariants. */
pv_status pv_state_invariants(pv_context *ctx, double out[5]);
/* The candidate scan of DipoleManager::process (src/dipole.cpp:49-78) on the device state:
 * opposite-sign pairs closer than threshold (minimum image in the periodic box) and, in a disk,
 * wall-image candidates. Writes min(count, capacity) candidates in no particular order;
 * *count is the full number. count == 0 means process() would return 0 without touching its
 * random generator (src/dipole.cpp:101-102), so a driver may skip the download. */
pv_status pv_dipole_scan(pv_context *ctx, double threshold, pv_dipole_candidate *out,
                         size_t capacity, size_t *count);

/* ---- dipole events on the device state (DipoleManager, src/dipole.h:19-40) ----------------- */

/* SimParams::dipoleReinjection (src/params.h:10). */
#define PV_REINJECT_NONE 0
#define PV_REINJECT_INDEPENDENT 1
#define PV_REINJECT_PAIRED 2

typedef struct pv_dipole_config {
    int removal;          /* SimParams::dipoleRemoval */
    double distance;      /* SimParams::dipoleRemovalDistance */
    int reinjection;      /* SimParams::dipoleReinjection, PV_REINJECT_* */
    uint64_t random_seed; /* SimParams::randomSeed */
} pv_dipole_config;

/* DipoleManager::DipoleManager(params) (src/dipole.cpp:29-30): the event settings, zero counts
 * and the reinjection generator seeded as the reference seeds it. The box length / disk radius
 * are the context's. */
pv_status pv_dipole_configure(pv_context *ctx, const pv_dipole_config *config);
/* DipoleManager::process (src/dipole.cpp:42-127) applied to the device state in place: the
 * candidate scan runs on the device, only the candidate list crosses to the host, where the
 * closest-first disjoint selection and the reinjection draws are made; survivors are compacted
 * in order on the device and reinjected vortices appended. The population, order, positions and
 * generator state afterwards equal the reference's. *events = pairs processed (wall events
 * count one). Any event invalidates the cached derivative. Errors as the reference throws them
 * (a failed paired placement is PV_ERROR_RUNTIME; the state is then unspecified). */
pv_status pv_dipole_process(pv_context *ctx, size_t *events);
/* DipoleManager::state() (src/dipole.cpp:182-186): the removed/reinjected counts and the
 * generator's text state (std::mt19937_64 stream format, as written into checkpoints).
 * *length = bytes of the state text without a terminator; written only when capacity suffices
 * (capacity > *length, NUL-terminated); PV_ERROR_CAPACITY otherwise. */
pv_status pv_dipole_state(const pv_context *ctx, uint64_t *removed, uint64_t *reinjected,
                          char *engine_state, size_t capacity, size_t *length);
/* DipoleManager::DipoleManager(params, state) (src/dipole.cpp:32-40): restores counts and, when
 * engine_state is non-empty, the generator ("invalid random-generator state in checkpoint"
 * otherwise). pv_dipole_configure must have been called first. */
pv_status pv_dipole_restore(pv_context *ctx, uint64_t removed, uint64_t reinjected,
                            const char *engine_state);

/* ---- text output at GPU rates (the reference formats on the host with
 *      std::ostream << std::setprecision(17)) ------------------------------------------------
 * Rows are formatted on the GPU, one thread per vortex, with every double printed exactly as the
 * reference's stream prints it (17 significant digits, correctly rounded, %g layout), packed on
 * the GPU and copied to `out` in one transfer. *length = the frame's bytes; when capacity is
 * smaller nothing is copied and PV_ERROR_CAPACITY is returned. n * PV_TRAJECTORY_ROW_MAX
 * (n * PV_CHECKPOINT_ROW_MAX) bytes always suffice. No terminator is written. */
#define PV_TRAJECTORY_ROW_MAX 192
#define PV_CHECKPOINT_ROW_MAX 80

/* The rows TrajectoryWriter::write (src/print.cpp:29-40) appends for one frame of the device
 * state, "time,frame,index,x,y,circulation,u,v\n" per vortex, with the velocity evaluated on the
 * device (evaluateDeviceState, as the driver's writeTrajectory does, src/main.cpp:251-258);
 * fails like evaluateDeviceState on a non-finite velocity. */
pv_status pv_format_trajectory(pv_context *ctx, double time, uint64_t frame, char *out,
                               size_t capacity, size_t *length);
/* The same rows for host arrays (TrajectoryWriter::write's own arguments). */
pv_status pv_format_trajectory_host(pv_context *ctx, double time, uint64_t frame, const double *x,
                                    const double *y, const double *circulation, const double *u,
                                    const double *v, size_t n, char *out, size_t capacity,
                                    size_t *length);
/* The vortex block of writeCheckpoint (src/checkpoint.cpp:86-88) for the device state:
 * "x y circulation\n" per vortex. */
pv_status pv_format_checkpoint_vortices(pv_context *ctx, char *out, size_t capacity,
                                        size_t *length);

/* Circulations of the device state (they change only through pv_upload_state and
 * pv_dipole_process); n must equal the device population. No counterpart: the reference's
 * driver keeps the population on the host and processes dipoles there. */
pv_status pv_download_circulation(pv_context *ctx, double *circulation, size_t n);

/* How the context evaluates its device state (no reference counterpart; for benchmarks and
 * profiles). symmetric = 1: the periodic box is evaluated once per unordered pair (each pair's
 * series serves both vortices); rows = partial-sum rows the stage reduction adds. */
typedef struct pv_plan_info {
    int symmetric;
    int rows;
    int targets_per_thread; /* ordered kernel */
    int chunk;              /* ordered kernel: sources per work item */
    int symmetric_min_ctas; /* symmetric form: the kernel built for this many CTAs per SM (0: default) */
    int symmetric_targets;  /* symmetric form: targets per lane off the diagonal */
    int symmetric_grid_ctas; /* symmetric form: persistent CTAs per SM of its grid */
} pv_plan_info;
pv_status pv_state_plan(const pv_context *ctx, pv_plan_info *info);

/* Population of the device state. */
pv_status pv_state_size(const pv_context *ctx, size_t *n);
/* Velocity evaluations made so far by the stepping hooks (the reference's CountingKernel,
 * tests/tests.cpp:281-296, counts the same events). */
pv_status pv_evaluation_count(const pv_context *ctx, uint64_t *count);

/* ---- multi-step device loops (no reference counterpart: the reference's driver calls one
 *      step at a time, src/main.cpp:292-308) ------------------------------------------------- */

/* `steps` RK4 steps of size dt, enqueued back to back with one synchronisation at the end. */
pv_status pv_rk4_advance(pv_context *ctx, double dt, uint64_t steps);

/* ---- batched ensembles (no reference counterpart: the reference runs one simulation per
 *      process) ------------------------------------------------------------------------------
 * Many independent simulations of uneven population and mixed geometry share one device arena
 * and advance together in lock-step DOPRI5 attempts, each with its own step size, tolerances,
 * end time, step budget and failure status. Each velocity stage of an attempt is one persistent
 * launch draining a (simulation, target block, source chunk) work queue. A simulation's result
 * does not depend on which other simulations share the batch. */

typedef struct pv_batch pv_batch;

typedef struct pv_batch_config {
    size_t capacity_vortices;              /* arena room (vortices over all simulations) */
    uint32_t max_simulations;              /* simulation slots */
    int device;                            /* CUDA ordinal */
    uint64_t max_steps_per_simulation;     /* default accepted-step budget (0: unlimited) */
    size_t partial_chunks_per_vortex_slot; /* partial-sum room per arena vortex (0: 16) */
} pv_batch_config;

/* One solve: integrate to t_end with DOPRI5 (the reference driver's integrator dopri5). */
typedef struct pv_batch_solve {
    double t_end;
    double dt;                  /* first step (timeStep), clamped to [dtmin, dtmax] */
    double absolute_tolerance;
    double relative_tolerance;
    double minimum_time_step;
    double maximum_time_step;
    uint64_t max_steps;         /* accepted-step budget (0: the batch default) */
} pv_batch_solve;

#define PV_SIM_RUNNING 1
#define PV_SIM_DONE 2    /* reached t_end */
#define PV_SIM_FAILED 3  /* stopped with an error: see status (device status code) */
#define PV_SIM_BUDGET 4  /* stopped at its step budget before t_end */

/* Which condition stopped a simulation whose status is the adaptive integrator's failure (the
 * reference throws the same runtime_error for each: src/timestep.cpp:116-117, src/main.cpp:314). */
#define PV_FAILURE_NONE 0
#define PV_FAILURE_REJECTION_CAP 1   /* more than 32 rejections in one step */
#define PV_FAILURE_DT_FLOOR 2        /* rejected at dt <= minimum time step */
#define PV_FAILURE_NO_TIME_ADVANCE 3 /* t + dt == t: the step cannot advance the time */

typedef struct pv_batch_sim_info {
    int state;                  /* PV_SIM_* */
    int status;                 /* device status code when failed, 0 otherwise */
    double time;
    double suggested_time_step;
    uint64_t accepted_steps;
    uint64_t rejected_steps;
    uint32_t population;
    int failure;                /* PV_FAILURE_* when status is the integrator's failure */
    int targets_per_thread;     /* of its ordered work items (pv_set_batch_tuning); 0 when it takes
                                   the once-per-unordered-pair items */
} pv_batch_sim_info;

typedef struct pv_batch_totals {
    uint64_t attempts;
    uint32_t work_items;        /* velocity work items per stage (running simulations) */
    size_t free_vortices;
    uint32_t running;
    uint32_t occupied_slots;
} pv_batch_totals;

pv_status pv_batch_create(const pv_batch_config *config, pv_batch **out);
void pv_batch_destroy(pv_batch *batch);
const char *pv_batch_last_error(const pv_batch *batch);
/* Admits one simulation (validated like uploadDeviceState); PV_ERROR_CAPACITY when the batch has
 * no free slot or arena room. *id identifies it until pv_batch_release. */
pv_status pv_batch_add(pv_batch *batch, const pv_params *params, const double *x, const double *y,
                       const double *circulation, size_t n, const pv_batch_solve *solve,
                       uint32_t *id);
/* Runs up to `attempts` lock-step DOPRI5 attempts of every running simulation, then
 * synchronises; *running receives the number still running. */
pv_status pv_batch_advance(pv_batch *batch, uint32_t attempts, uint32_t *running);
pv_status pv_batch_info(pv_batch *batch, uint32_t id, pv_batch_sim_info *info);
/* Current positions of simulation id (n must equal its population). */
pv_status pv_batch_result(pv_batch *batch, uint32_t id, double *x, double *y, size_t n);
/* Frees the slot and arena room of simulation id (stopping it first if it is still running). */
pv_status pv_batch_release(pv_batch *batch, uint32_t id);
pv_status pv_batch_status(pv_batch *batch, pv_batch_totals *totals);
pv_status pv_batch_stream(const pv_batch *batch, void **stream);
/* Autotuner table of the batch's ordered work items: targets per thread (1, 2 or 4; 4 not for the
 * periodic box; 0 restores the default of 4 for the plane, 1 for the box and 2 for the disk) for a
 * geometry, a precision and populations with floor(log2 N) == log2_n. Process-wide; read when a
 * simulation is admitted (pv_batch_add), so a simulation's work items, like its results, depend
 * only on its own geometry, precision and N. pv_get_batch_tuning returns the value in effect. */
pv_status pv_set_batch_tuning(int geometry, int precision, int log2_n, int per_thread);
pv_status pv_get_batch_tuning(int geometry, int precision, int log2_n, int *per_thread);

/* ---- allocation-free evaluation (no counterpart in the reference) ------------------------ */

/* Largest population pv_evaluate_device_noalloc accepts. */
#define PV_NOALLOC_MAX_VORTICES 349440

/* VelocityKernel::evaluate semantics for n vortices whose arrays are already in GPU memory, for
 * callers that cannot allocate device memory or let a library allocate it: hosts that own all GPU
 * memory through their own pool, and time-stepping loops that cannot pay for the device-wide
 * synchronisation of cudaMalloc/cudaFree. x, y, circulation (16-byte aligned) and u, v are DEVICE
 * pointers of the current device; stream is a cudaStream_t (NULL: the legacy default stream).
 * Creates no context and calls no allocator: its scratch (8 MiB: scaled circulations, chunk partial
 * sums, status word) is one fixed device array inside the library, held by every GPU that loads
 * the library until the process exits. n above PV_NOALLOC_MAX_VORTICES is rejected with
 * PV_ERROR_INVALID_ARGUMENT. The call synchronises `stream`; the message of a failure is returned
 * by pv_last_error(NULL). The first call on a device looks up the array's device address (do it
 * before any stream capture). All calls on a device share the array, so calls whose GPU work
 * overlaps in time race and must be ordered by the caller. FP64 only. */
pv_status pv_evaluate_device_noalloc(const pv_params *params, const double *x, const double *y,
                                     const double *circulation, size_t n, double *u, double *v,
                                     void *stream);

/* ---- diagnostics (no reference counterpart) --------------------------------------------- */

/* Kernel kinds counted by pv_get_kernel_stats. */
#define PV_KERNEL_VELOCITY 0   /* tiled pair-sum kernel */
#define PV_KERNEL_STAGE 1      /* chunk reduction + stage position / combine / error + control */
#define PV_KERNEL_ACCEPT 2     /* state update of an accepted step */
#define PV_KERNEL_INVARIANTS 3 /* moments, Hamiltonian tiles, final sum */
#define PV_KERNEL_DIPOLE 4     /* close-dipole candidate scan and survivor compaction */
#define PV_KERNEL_OUTPUT 5     /* text formatting of trajectory / checkpoint rows */
#define PV_KERNEL_NEAR 6       /* FP32C: the FP64 pass over the near-field pairs */
#define PV_KERNEL_KINDS 7

typedef struct pv_kernel_stats {
    uint64_t launches[PV_KERNEL_KINDS];       /* kernels launched by this context */
    uint64_t timed_launches[PV_KERNEL_KINDS]; /* launches bracketed by CUDA events */
    double milliseconds[PV_KERNEL_KINDS];     /* summed event time of the timed launches */
} pv_kernel_stats;

/* The context's CUDA stream (a cudaStream_t) through *stream, so that a caller can order its own
 * work or events after the context's kernels. */
pv_status pv_context_stream(const pv_context *ctx, void **stream);
/* Autotuner table of the velocity plan: targets held in registers per thread (1, 2 or 4; 0 restores
 * the built-in heuristic) for a geometry, a precision and populations N with floor(log2 N) ==
 * log2_n. Process-wide; read when a context plans an evaluation (pv_upload_state,
 * pv_evaluate_range). pointvortex_b200/autotune.py fills it by timing the candidates. */
pv_status pv_set_tuning(int geometry, int precision, int log2_n, int per_thread);
pv_status pv_get_tuning(int geometry, int precision, int log2_n, int *per_thread);
/* Autotuner table of the once-per-unordered-pair form (periodic box and plane), by geometry,
 * precision and floor(log2 N): mode 0 restores the built-in plan, 1 selects the ordered kernel,
 * 2 the symmetric form; min_ctas (periodic FP64: 7 or 8, else 0) selects the kernel built for that
 * many resident CTAs per SM; targets (plane: 4 or 8; periodic FP64: 2, with min_ctas 0; else 0)
 * the targets per lane off the diagonal. Process-wide;
 * read when a context plans its device state (pv_upload_state). No reference counterpart. */
pv_status pv_set_symmetric_tuning(int geometry, int precision, int log2_n, int mode, int min_ctas,
                                  int targets);
pv_status pv_get_symmetric_tuning(int geometry, int precision, int log2_n, int *mode,
                                  int *min_ctas, int *targets);
/* Autotuner table of the symmetric form's persistent grid: CTAs per SM for a geometry (0 plane,
 * 1 periodic), a precision and populations N with floor(log2 N) == log2_n (0 restores as many as
 * fit, the default; a value above what fits is clamped to it). Fewer CTAs than fit can finish
 * sooner: the work queue's last round of items is then fuller. Process-wide; read when a context
 * plans its device state (pv_upload_state). No reference counterpart. */
pv_status pv_set_symmetric_grid(int geometry, int precision, int log2_n, int ctas_per_sm);
pv_status pv_get_symmetric_grid(int geometry, int precision, int log2_n, int *ctas_per_sm);
/* Near-field radius of the FP32-compensated form (precision PV_PRECISION_FP32C): periodic pairs
 * closer than it (minimum image), disk pairs closer than it and disk wall images closer than it to
 * their target are left out of the FP32 sums and evaluated in FP64. radius < 0 selects the default for the population (twice
 * the mean spacing of N uniform vortices in the periodic box, once in the disk), 0 turns the near
 * field off. Applies to the device state
 * at once and to later evaluations; the plane and FP64 contexts ignore it. No reference
 * counterpart (the reference evaluates in FP64 only). */
pv_status pv_set_near_field(pv_context *ctx, double radius);
/* The near-field radius in use for the device state (0 when there is none). */
pv_status pv_get_near_field(const pv_context *ctx, double *radius);
/* Polls of the context's bounded device waits before they give up with the runtime error "a bounded
 * device wait timed out": copy_polls for a velocity tile's bulk copies (default 2^22), barrier_polls
 * for a grid barrier of the cooperative RK4 steps (default 2^24); a negative value restores the
 * default, 0 gives up without polling. A wait that gives up leaves the device state at the last
 * completed step (a velocity tile first waits, with the default bound, for its copies in flight; a
 * grid barrier is broken for every CTA at once). Only the tests of these exits shorten them. No
 * reference counterpart (the reference CUDA backend has no device-side waits). */
pv_status pv_set_wait_limits(pv_context *ctx, int64_t copy_polls, int64_t barrier_polls);
/* Bracket every launch of the context with CUDA events recorded on its own stream. */
pv_status pv_set_profiling(pv_context *ctx, int enabled);
/* Synchronises the context stream and returns the counters accumulated since the last reset. */
pv_status pv_get_kernel_stats(pv_context *ctx, pv_kernel_stats *out);
pv_status pv_reset_kernel_stats(pv_context *ctx);

/* Arithmetic peak of `device` at its current clocks, measured with independent FMA chains on
 * every SM: kind 0 = FP64 FMA, 1 = FP32 FMA. *flops_per_second = 2 x FMAs / elapsed time. */
pv_status pv_probe_peak(int device, int kind, double *flops_per_second);

#ifdef __cplusplus
}
#endif
#endif
