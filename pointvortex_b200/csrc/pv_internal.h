// pv_internal.h — host-side declarations shared by the translation units of libpvb200.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <string>

#include "pv_geometry.cuh"
#include "pv_pair32.cuh"

namespace pvb {

// Launches a kernel that may be scheduled while the previous kernel of the stream drains
// (programmatic stream serialization); the kernel calls pdl_enter() before touching memory, which
// waits for that kernel to complete. In a stream capture the launch becomes a programmatic edge.
template <typename... Params, typename... Args>
cudaError_t launch_pdl(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem,
                       cudaStream_t stream, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<Params>(args)...);
}

// ---- velocity evaluation ---------------------------------------------------------------------
// One launch evaluates targets [t_begin, t_end) against sources [0, n_src). The source range is
// cut into `num_chunks` chunks; work item (target block, chunk) writes its partial sums to
// pu/pv[chunk * stride + (t - t_begin)]. A reduction pass (stage kernel) sums the chunks in
// fixed order, so results do not depend on scheduling.
struct EvalArgs {
    const double *tx, *ty;          // target positions (indexed by global vortex index)
    const double *sx, *sy, *sg;     // source positions and scaled circulation
    size_t t_begin, t_end;
    size_t n_src;
    double *pu, *pv;
    size_t stride;
    int chunk;                      // sources per chunk (even)
    int num_chunks;
    int *status;
    GeometryConsts g;
    uint32_t wait_limit = kWaitLimit;  // polls of a bounded tile wait (pv_set_wait_limits)
    f32::NearLists near = {nullptr, nullptr};  // FP32C near-field lists (indexed by target)
};

struct EvalPlan {
    int block;         // threads per CTA
    int per_thread;    // targets held in registers per thread
    int chunk;         // sources per work item
    int num_chunks;
    int target_blocks;
    size_t items() const { return static_cast<size_t>(num_chunks) * target_blocks; }
};

EvalPlan plan_evaluation(int geometry, size_t n_targets, size_t n_sources, int sm_count,
                         int per_thread_override = 0, int precision = 0);
// The autotuner's table of targets per thread (pv_set_tuning / pv_get_tuning).
int tuning_lookup(int geometry, int precision, size_t n);
bool tuning_store(int geometry, int precision, int log2_n, int per_thread);
cudaError_t launch_velocity(const EvalArgs &a, const EvalPlan &p, cudaStream_t stream);
// The FP32-compensated precision form (pv_velocity32.cu): same arguments, same partial layout.
cudaError_t launch_velocity_fp32c(const EvalArgs &a, const EvalPlan &p, cudaStream_t stream);
// Resident CTAs per SM of the FP32-compensated ordered kernel (the planner's wave arithmetic).
int resident_fp32c(int geometry, int per_thread);

// The periodic box and the infinite plane (FP64, FP32C) evaluated once per unordered pair
// (pv_symmetric.cu) for a whole population (targets = sources). Partial rows: `blocks` rows of
// `stride` (u, v) pairs, row r of vortex i at rows[r * stride + i].
struct SymmetricPlan {
    int a = 0;           // 32-vortex sub-blocks per block; 0: not used
    int blocks = 0;      // partial rows
    unsigned items = 0;  // block pairs (I <= J)
    int grid = 0;        // persistent CTAs
    int precision = 0;   // PV_PRECISION_FP64 or PV_PRECISION_FP32C
    int geometry = 0;    // GEO_PERIODIC or GEO_INFINITE
    int targets = 1;     // targets per lane off the diagonal (the plane: 4 or 8)
    int min_ctas = 0;    // periodic FP64: the kernel built for 7 or 8 CTAs per SM (0: default)
    int grid_ctas = 0;   // persistent CTAs per SM (grid / SMs)
    bool enabled() const { return a > 0; }
};
constexpr size_t kSymmetricMinN = 2048;       // periodic box below: the ordered kernel
constexpr size_t kSymmetricPlaneMinN = 16384;   // infinite plane below: the ordered kernel
constexpr size_t kSymmetricPlane32MinN = 16384; // the same for the FP32-compensated plane
constexpr size_t kSymmetricPlaneWideN = 32768;  // the plane from here: 8 targets per lane
constexpr size_t kSymmetricPartialBytes = static_cast<size_t>(256) << 20;  // a grows past this
constexpr size_t kSymmetricPartialBytesMax = static_cast<size_t>(4) << 30;  // beyond: ordered kernel
SymmetricPlan plan_symmetric(size_t n, int sm_count, int precision, int geometry);
// The autotuner's table of the symmetric form (pv_set_symmetric_tuning); 0 = the built-in plan.
int symmetric_tuning_lookup(int geometry, int precision, size_t n);
// Autotuner table of the symmetric form's persistent grid: CTAs per SM (0: as many as fit), by
// geometry, precision and floor(log2 N) (pv_set_symmetric_grid).
int symmetric_grid_lookup(int geometry, int precision, size_t n);
bool symmetric_grid_store(int geometry, int precision, int log2_n, int ctas_per_sm);
bool symmetric_tuning_store(int geometry, int precision, int log2_n, int mode, int min_ctas,
                            int targets);
// p.items packed (I << 16) | J: the diagonal items first, then I < J row by row.
void symmetric_items(const SymmetricPlan &p, unsigned *out);
// counter: two words, zero before the first launch; each launch leaves them zero again.
// near: the near-field lists of the FP32C periodic kernel (pv_pair32.cuh; count == nullptr:
// none); the other kernels ignore it.
cudaError_t launch_symmetric(const double *x, const double *y, const double *gs, size_t n,
                             const SymmetricPlan &p, const unsigned *items, unsigned *counter,
                             double2 *rows, size_t stride, const GeometryConsts &g,
                             const f32::NearLists &near, cudaStream_t stream);

// ---- FP32C near field (pv_near.cu) -----------------------------------------------------------
// The FP64 pass over the pairs an FP32 evaluation listed (f32::NearLists): their exact terms are
// added into the last partial row, and every list count is reset. Targets [t_begin, t_end) of n
// sources; the partial entry of target i in row r is r * stride + (i - t_begin), in pr
// (interleaved rows of the symmetric kernels) or pu/pv (chunk partials).
struct NearPass {
    f32::NearLists lists;
    const double *x, *y, *gs;  // the evaluated positions and the scaled circulations
    size_t n;
    size_t t_begin, t_end;
    double *pu, *pv;
    double2 *pr;
    size_t stride;
    int rows;
    GeometryConsts g;
};
cudaError_t launch_near_field(const NearPass &a, cudaStream_t stream);
// The default near-field radius of the FP32C form for n vortices (0: the geometry has none).
double default_near_radius(const GeometryConsts &g, size_t n);

// ---- stage kernels (reduction, stage positions, RK4 combine, DOPRI5 error and control) ------
enum StageMode : int {
    STAGE_REDUCE_ONLY = 0,  // k = sum of partials
    STAGE_POSITION = 1,     // ... then xt = x0 + dt * sum_j coef_j k_j, validated
    STAGE_RK4_COMBINE = 2,  // ... then xt = x0 + dt * (k0 + 2 k1 + 2 k2 + k3) / 6, validated
    STAGE_DOPRI_ERROR = 3,  // ... then scaled error, max-reduced, step control by the last block
};

struct StageArgs {
    size_t n;
    int mode;
    int reduce;                     // 1: reduce partials into k_s; 0: k_s already final
    int num_chunks;
    size_t stride;
    const double *pu, *pv;          // chunk partials, u and v apart
    const double2 *pr;              // or (non-null) interleaved (u, v) rows of the symmetric kernels
    int s;                          // index of the stage being produced (k_s)
    double *kx[7], *ky[7];          // stage velocity fields
    const double *ex, *ey;          // positions the stage was evaluated at (slow path)
    const double *gamma;            // raw circulations (slow path)
    size_t n_src;                   // population of ex/ey/gamma (slow path)
    size_t t_offset;                // global index of element 0 (host-array target ranges)
    int nonfinite_ok;               // evaluateRange: a finite-free result is returned, not an error
    const double *x0, *y0;          // step-start state
    double *xt, *yt;                // next stage position / combined state
    double coef[7];                 // a_{s+1, j}
    int ncoef;
    double dt;                      // used when dt_from_control == 0
    int dt_from_control;            // DOPRI5: read dt from the control block
    double w[7];                    // DOPRI5: b5 - b4
    DeviceControl *ctl;
    GeometryConsts g;
    // FP32C: the near-field pass of the evaluation whose partial rows this stage reduces, fused
    // into it (near.lists.count == nullptr: none; reduce must be 1). The stage's target i is the
    // lists' target near.t_begin + i.
    NearPass near;
};

cudaError_t launch_stage(const StageArgs &a, cudaStream_t stream, int sm_count);

// Polls a grid barrier of the cooperative RK4 steps waits before it gives up (ST_TIMEOUT).
constexpr uint32_t kGridSpinLimit = 1u << 24;

// RK4 steps of a small FP64 population in one cooperative launch (pv_stepping.cu): the four
// stages as enqueue_rk4 sets them up (stage[3].xt/yt: the combined state), bit for bit the same
// results as launching them. barrier: the grid barrier's arrival counter, zero at every
// launch. Eligible up to kRk4StepsMaxN vortices with fewer than 32 chunks.
struct Rk4Steps {
    StageArgs stage[4];
    double *x, *y;          // the state, updated after every step
    const double *gs;       // scaled circulations
    size_t n;
    int chunk, num_chunks;  // the ordered kernel's source chunks
    uint64_t steps;
    unsigned long long *barrier;
    uint32_t spin_limit = kGridSpinLimit;  // polls of a grid-barrier wait (pv_set_wait_limits)
};
constexpr size_t kRk4StepsMaxN = 2048;
bool rk4_steps_eligible(size_t n, int num_chunks);
cudaError_t launch_rk4_steps(const Rk4Steps &p, int sm_count, cudaStream_t stream);

// Accept kernel: state <- xt (and, for DOPRI5, k0 <- k6 when the attempt was accepted).
cudaError_t launch_accept(double *x, double *y, const double *xt, const double *yt, double *k0x,
                          double *k0y, const double *k6x, const double *k6y, size_t n, int dopri,
                          DeviceControl *ctl, cudaStream_t stream);

// ---- invariants ------------------------------------------------------------------------------
// Moments (circulation, Ix, Iy, angular impulse) and the Hamiltonian of n vortices. Block
// partials go to `scratch` (>= invariants_scratch_doubles(n, sm) doubles); a final single-block
// pass sums them in fixed order. out[0..4] (device) as computeInvariants. Moment errors go to
// *status, Hamiltonian errors to *status_h.
size_t invariants_scratch_doubles(size_t n, int sm_count);
cudaError_t launch_invariants(const double *x, const double *y, const double *gamma, size_t n,
                              const GeometryConsts &g, double *scratch, double *out, int *status,
                              int *status_h, cudaStream_t stream);

// ---- close-dipole candidate scan --------------------------------------------------------------
struct DipoleCandidateDev {
    unsigned long long first, second;
    double distance_squared;
};
cudaError_t launch_dipole_scan(const double *x, const double *y, const double *gamma, size_t n,
                               const GeometryConsts &g, double threshold,
                               DipoleCandidateDev *out, size_t capacity,
                               unsigned long long *count, cudaStream_t stream,
                               const DeviceControl *gate = nullptr);  // gate: scan iff accepted

// Order-preserving removal of the sorted indices removed[0, m) from (x, y, g, gs)[0, n) into
// (ox, oy, og, ogs)[0, n - m).
cudaError_t launch_compact_survivors(const double *x, const double *y, const double *g,
                                     const double *gs, size_t n, const unsigned long long *removed,
                                     size_t m, double *ox, double *oy, double *og, double *ogs,
                                     cudaStream_t stream);

// ---- text output (pv_output.cu) -----------------------------------------------------------------
enum RowKind { ROWS_TRAJECTORY = 0, ROWS_CHECKPOINT = 1 };
constexpr int kTrajectoryRowStride = 192;  // time(24),frame(20),index(20) and five doubles(5 x 25)
constexpr int kCheckpointRowStride = 80;   // three doubles (3 x 25)

struct RowFormat {
    const double *x, *y, *g, *u, *v;
    size_t n;
    int kind;        // RowKind
    int stride;      // staging bytes per row
    int prefix_len;  // trajectory rows: "time,frame," formatted once
    char prefix[48];
};
// "time,frame," as the trajectory rows begin; returns its length (at most 46).
int format_prefix(double time, uint64_t frame, char *out);
// Formats rows [0, f.n) into staging (f.stride bytes each), then packs them into out;
// block_sums needs ceil(n / 256) + 1 entries and receives the frame's byte count at
// block_sums[ceil(n / 256)].
cudaError_t launch_format_rows(const RowFormat &f, char *staging, uint32_t *lengths,
                               unsigned long long *block_sums, char *out, cudaStream_t stream);

// ---- shared host helpers (pv_context.cu) -------------------------------------------------------
// Kernel-constructor validation and fast-path constants of a parameter set.
int make_geometry_consts(const struct pv_params &p, GeometryConsts &g, std::string &message);
// Sets the calling thread's message returned by pv_last_error(NULL).
void set_thread_error(const std::string &message);

// ---- diagnostics --------------------------------------------------------------------------------
cudaError_t launch_peak_probe(int kind, int blocks, int threads, int iterations, double *sink,
                              cudaStream_t stream);

} // namespace pvb
