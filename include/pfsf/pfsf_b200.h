/*
 * pfsf_b200.h -- additive exports of the B200 build (ABI MINOR additions:
 * no existing struct, enum value or signature changes).
 *
 * The reference tick runs a fixed 16-step schedule and never iterates to a
 * tolerance.  These entry points add a solve of the symmetric per-link
 * 26-point operator
 *     sum_j w_ij (phi_i - phi_j) = s_i     (solid voxels i)
 *     w_ij = {1, 0.5, 1/6}[face/edge/corner] * 2 k_i k_j / (k_i + k_j)
 * (anchors Dirichlet phi = 0, air and out-of-box links dropped) to a relative
 * residual ||s - A phi||_2 / ||s||_2 <= rel_tol, for all listed islands,
 * either island by island (plain FP32) or batched in one persistent launch
 * with reduced-precision coefficient storage and FP32 residual refinement.
 */
#ifndef PFSF_B200_H
#define PFSF_B200_H
#include "pfsf_types.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PFSF_PREC_FP32 = 0, /* kappa and coarse levels stored FP32 */
    PFSF_PREC_BF16 = 1, /* kappa and coarse levels stored BF16 */
    PFSF_PREC_FP16 = 2, /* kappa and coarse levels stored FP16 */
} pfsf_precision;

typedef enum {
    PFSF_SOLVE_PER_ISLAND = 0, /* one island at a time, one kernel per step */
    PFSF_SOLVE_BATCHED = 1,    /* all islands in one persistent launch */
} pfsf_solve_mode;

/* flags of pfsf_solve_to_tolerance */
#define PFSF_SOLVE_NO_UPLOAD 0x1u   /* inputs already resident on the device */
#define PFSF_SOLVE_NO_READBACK 0x2u /* leave phi on the device */
#define PFSF_SOLVE_COLD_START 0x4u  /* start from phi = 0 instead of the registered phi */

/* Caller-owned host arrays of one island for the tolerance solve. */
typedef struct pfsf_island_kappa_buffers {
    void* phi_addr; /* float32 x N: initial guess in, solution out */
    int64_t phi_bytes;
    void* source_addr; /* float32 x N */
    int64_t source_bytes;
    void* kappa_addr; /* float32 x N, per-voxel conductivity (> 0 on non-air) */
    int64_t kappa_bytes;
    void* voxel_type_addr; /* uint8 x N */
    int64_t voxel_type_bytes;
} pfsf_island_kappa_buffers;

typedef struct pfsf_solve_stats {
    int32_t struct_bytes;
    int32_t islands_solved;
    int32_t islands_converged;
    int32_t max_iterations;  /* largest outer iteration count over islands */
    double max_rel_residual; /* largest final ||s - A phi|| / ||s|| (FP64) */
    float device_ms;         /* solve time on the engine stream (CUDA events); in batched mode it
                                includes the teams' reads of mapped inputs and writes of phi */
    float upload_ms;         /* input copies and preparation before the solve */
    float readback_ms;       /* phi conversion and copies after the solve */
    int32_t kernel_launches; /* kernels launched by the solve */
    int64_t inner_iterations_total; /* sum over islands of inner PCG iterations */
    double algorithmic_bytes;       /* compulsory bytes of every pass the solve made:
                                       each array a pass touches counted once per pass */
    int64_t active_voxels;          /* solid voxels over all solved islands */
    double island_ms_sum;           /* batched mode: sum over islands of solve time */
    double island_ms_max;           /* batched mode: longest single island solve */
    double span_ms;                 /* batched mode: first island start to last island end */
    double setup_ms_sum;            /* batched mode: sum over islands of the hierarchy build */
    double precond_ms_sum;          /* batched mode: sum over islands of the time in V-cycles */
    double vcycle_fine_ms_sum;      /* ... of which fine-level passes */
    double vcycle_coarse_ms_sum;    /* ... coarse levels smoothed by the whole team */
    double vcycle_tail_ms_sum;      /* ... the coarsest levels (single warp or team) */
    int32_t persistent_ctas;        /* batched mode: CTAs of the persistent launch(es) */
    int32_t reserved;
} pfsf_solve_stats;

/* Registers the kappa-form inputs of an island created by pfsf_add_island.
 * NULL pointers or undersized arrays -> PFSF_ERROR_INVALID_ARG. */
PFSF_API pfsf_result pfsf_register_island_kappa(pfsf_engine engine, int32_t island_id,
                                                const pfsf_island_kappa_buffers* bufs);
PFSF_API void pfsf_set_precision_mode(pfsf_engine engine, pfsf_precision mode);
PFSF_API void pfsf_set_solve_mode(pfsf_engine engine, pfsf_solve_mode mode);

/* No counterpart in the reference ABI (its native V-cycle takes two W legs
 * on the coarse levels, dispatcher_vcycle.cpp:315-340, 373-374).  Multigrid
 * cycle of the batched tolerance solve's preconditioner: PFSF_MG_V (default)
 * or PFSF_MG_W, which visits every level below the first coarse level twice.
 * The per-island plain solve always runs V-cycles. */
typedef enum { PFSF_MG_V = 0, PFSF_MG_W = 1 } pfsf_mg_cycle;
PFSF_API void pfsf_set_mg_cycle(pfsf_engine engine, pfsf_mg_cycle cycle);

/* Replaces the reference's unexported aggregation correction
 * (NP/src/solver/dispatcher_amg.cpp:83 recordAMGCorrection with the
 * aggregates of NP/src/solver/amg_builder.cpp:9 buildAMG), which its native
 * tick declares but never records.  enable != 0: every PCG start of the
 * reference tick (pfsf_tick_dbb / pfsf_tick) first applies
 * phi += P D_c^-1 P^T r to the start's residual r, then starts again from the
 * corrected phi.  Aggregates are rebuilt on the device whenever an island's
 * inputs are uploaded.  Off by default (the reference tick as recorded). */
PFSF_API void pfsf_set_amg(pfsf_engine engine, int32_t enable);

/* Solves every listed island to rel_tol (max_iter outer iterations at most)
 * and writes phi back to its registered phi array.  Returns PFSF_OK even if
 * some island did not converge (see out->islands_converged). */
PFSF_API pfsf_result pfsf_solve_to_tolerance(pfsf_engine engine, const int32_t* island_ids, int32_t count,
                                             double rel_tol, int32_t max_iter, uint32_t flags,
                                             pfsf_solve_stats* out);

/* pfsf_tick_dbb with the fixed 16-step schedule (pfsf_engine.cpp:484)
 * replaced by the tolerance solve: every listed island must have both the
 * reference buffers (pfsf_register_island_buffers: face conductivity,
 * rcomp, rtens, max_phi, type ...) and the kappa-form buffers
 * (pfsf_register_island_kappa); all of them are solved to rel_tol in one
 * batched solve (phi written back to the kappa phi array, which is also the
 * next tick's starting guess), then on that phi: the history update
 * H = max(H, psi_e) (rbgs_smooth.comp.glsl:177-191), the phase field, the
 * failure scan and the failure compaction of the reference tick, with the
 * {count}{x,y,z,type} tuples appended to failure_addr exactly as
 * pfsf_tick_dbb does (count pre-zeroed) and phi copied to the stress
 * readback buffer when one is registered.  Listed islands are processed
 * whether or not they are marked dirty; the reference-layout buffers are
 * re-uploaded for dirty islands (as pfsf_tick_dbb does), the kappa-form
 * buffers on every call.  out may be NULL. */
PFSF_API pfsf_result pfsf_tick_tolerance(pfsf_engine engine, const int32_t* island_ids, int32_t count,
                                         int64_t epoch, void* failure_addr, int64_t failure_bytes, double rel_tol,
                                         int32_t max_iter, pfsf_solve_stats* out);

/* No counterpart in the reference ABI.  Convergence record of one island in
 * the last forward tolerance solve of the current island set (an adjoint
 * solve leaves it in place).  INVALID_ARG before any solve of the set. */
typedef enum pfsf_island_team {
    PFSF_TEAM_PLAIN = 0,   /* plain mode: one kernel per operation */
    PFSF_TEAM_GRID = 1,    /* the whole GPU (cooperative launch) */
    PFSF_TEAM_CLUSTER = 2, /* one thread-block cluster */
    PFSF_TEAM_CTA = 3,     /* one CTA */
    PFSF_TEAM_WARP = 4     /* one warp */
} pfsf_island_team;

typedef struct pfsf_island_report {
    int32_t struct_bytes;
    int32_t lx, ly, lz;
    int32_t levels;            /* hierarchy levels including the fine level */
    int32_t inner_iterations;  /* inner PCG iterations over all outer steps */
    int32_t outer_iterations;  /* FP64 residual refinements */
    int32_t converged;         /* 1 when rel_residual <= the requested tolerance */
    int32_t team;              /* pfsf_island_team */
    int32_t team_ctas;         /* CTAs of the team (0 for a warp or plain mode) */
    double rel_residual;       /* final ||s - A phi|| / ||s|| (FP64) */
    double solve_ms;           /* batched mode: the island's solve time */
    double setup_ms;           /* batched mode: hierarchy build */
    double precond_ms;         /* batched mode: time in V-cycles */
    double start_ms;           /* batched mode: solve start after the first island's start */
} pfsf_island_report;

PFSF_API pfsf_result pfsf_island_solve_report(pfsf_engine engine, int32_t island_id, pfsf_island_report* out);

/* No counterpart in the reference ABI.  Launch-shape parameters of the
 * batched tolerance solve.  pfsf_init takes them from the tuning file the
 * autotuner writes (pfsf_b200/autotune.py: timed trials on a size-bucketed
 * island set, one section per GPU model and SM count) -- the file named by
 * PFSF_TUNE_FILE, else tune/pfsf_tune.txt beside the library's lib/
 * directory -- then from the PFSF_CLUSTER, PFSF_CLUSTER_MIN_VOXELS,
 * PFSF_GRID_MIN_VOXELS, PFSF_WARP_MAX_VOXELS, PFSF_CHEB_K, PFSF_CHEB_LOWER,
 * PFSF_COARSE_WEIGHT, PFSF_TAIL_CELLS, PFSF_COARSE_SWEEPS, PFSF_INNER_ETA variables when
 * set; built-in defaults otherwise. */
typedef enum pfsf_tuning_source {
    PFSF_TUNING_DEFAULT = 0,  /* built-in defaults */
    PFSF_TUNING_FILE = 1,     /* the tuning file's section for this GPU */
    PFSF_TUNING_ENV = 2,      /* at least one environment override */
    PFSF_TUNING_CALLER = 3    /* pfsf_set_tuning */
} pfsf_tuning_source;

typedef struct pfsf_tuning {
    int32_t struct_bytes;
    int32_t cluster;              /* CTAs per thread-block cluster for big islands: 1 (none), 4 or 8 */
    int64_t cluster_min_voxels;   /* islands of at least this many voxels go to clusters */
    int64_t grid_min_voxels;      /* ... to the whole GPU, one at a time */
    int64_t warp_max_voxels;      /* islands below this many voxels go to single warps (0: none) */
    int32_t cheb_k;               /* Chebyshev smoothing degree, 1..4 */
    int32_t source;               /* pfsf_tuning_source (read only) */
    /* solver parameters (read and written only when struct_bytes covers them) */
    float cheb_lower;             /* Chebyshev interval [cheb_lower * lmax, lmax], 0 < cheb_lower < 1 */
    float coarse_weight;          /* coarse-correction weight of the V-cycle, 0 < w < 2 (keeps it SPD) */
    int32_t tail_cells;           /* coarse levels of at most this many cells run on one warp, 0..1048576 */
    int32_t coarse_sweeps;        /* smoothing steps on the coarsest level, 1..16 */
    float inner_eta;              /* inner PCG stops at max(inner_eta, 0.3 tol / relres) of the outer residual,
                                     1e-6 < inner_eta < 1 */
    int32_t reserved;
} pfsf_tuning;

/* out->struct_bytes: the caller's sizeof(pfsf_tuning) (an older, shorter struct gets the fields
 * it has; 0 or less: the whole current struct is written). */
PFSF_API pfsf_result pfsf_get_tuning(pfsf_engine engine, pfsf_tuning* out);
/* INVALID_ARG for out-of-range values (nothing changes then). */
PFSF_API pfsf_result pfsf_set_tuning(pfsf_engine engine, const pfsf_tuning* in);

/* No counterpart in the reference ABI.  Shape of the last reference tick
 * (pfsf_tick_dbb / pfsf_tick) or tolerance-tick tail: the dispatched islands
 * run as groups of equal schedule, each schedule step one kernel launch over
 * its group, the whole launch sequence replayed from a CUDA graph while the
 * group structure is unchanged.  INVALID_ARG before the first tick. */
typedef struct pfsf_tick_report {
    int32_t struct_bytes;
    int32_t islands;           /* islands dispatched */
    int32_t groups;            /* schedule groups */
    int32_t graph_replayed;    /* 1: the captured launch sequence was reused; 2: captured again and the
                                  instantiated graph updated in place; 0: captured and instantiated */
    int64_t kernel_launches;   /* kernels the tick launched */
    double algorithmic_bytes;  /* device-memory bytes of the tick's passes: every
                                  array a pass touches counted once per pass */
    double grid_voxels;        /* voxels of the dispatched islands' boxes */
    float device_ms;           /* engine-stream time from the table upload to the
                                  result copy (CUDA events) */
    int32_t host_us;           /* host time from the call's planning to the graph launch (planning,
                                  table, and any capture, update or instantiation), microseconds */
} pfsf_tick_report;

PFSF_API pfsf_result pfsf_last_tick_report(pfsf_engine engine, pfsf_tick_report* out);

/* No counterpart in the reference's native ABI; the Java path reduces it on
 * the GPU with phi_reduce_max.comp.glsl and feeds PFSFScheduler.checkDivergence.
 * Largest phi of the island at the end of its last tick (reference or
 * tolerance tick), reduced on the device in the same pass as the failure
 * scan; 0 before the island's first tick. */
PFSF_API pfsf_result pfsf_island_phi_max(pfsf_engine engine, int32_t island_id, float* out);

/* Copies the FP64 solution accumulator of the last tolerance solve of an
 * island (count = min(N, capacity) values).  The FP32 phi written back by
 * pfsf_solve_to_tolerance is this vector rounded to float32. */
PFSF_API pfsf_result pfsf_read_solution64(pfsf_engine engine, int32_t island_id, double* out, int64_t capacity,
                                          int64_t* out_count);

/* No counterpart in the reference ABI (which has no gradient code).
 * Caller-owned host arrays of one island for the adjoint of the tolerance
 * solve: grad_phi = dL/dphi in, grad_source = dL/ds and grad_kappa = dL/dkappa
 * out (float32 x N each). */
typedef struct pfsf_island_adjoint_buffers {
    const void* grad_phi_addr;
    int64_t grad_phi_bytes;
    void* grad_source_addr;
    int64_t grad_source_bytes;
    void* grad_kappa_addr;
    int64_t grad_kappa_bytes;
} pfsf_island_adjoint_buffers;

PFSF_API pfsf_result pfsf_register_island_adjoint(pfsf_engine engine, int32_t island_id,
                                                  const pfsf_island_adjoint_buffers* bufs);

/* Gradient of a loss L(phi) through the last pfsf_solve_to_tolerance of the
 * same island set (same ids, same order): one solve A lambda = dL/dphi with
 * the same symmetric operator, solver and precision mode (to rel_tol), then
 * an edge-product pass
 *     dL/ds_i     = lambda_i                                     (solid i)
 *     dL/dkappa_i = - sum_j dw_ij/dk_i (lambda_i - lambda_j)(phi_i - phi_j)
 * in FP64 from the FP64 forward solution, written to the registered
 * grad_source / grad_kappa arrays (0 on air; dL/ds 0 on anchors).  The
 * forward solution stays readable through pfsf_read_solution64.  Returns
 * PFSF_ERROR_INVALID_ARG if an island has no adjoint buffers or the arena
 * does not hold a forward solution of exactly this island set.  flags:
 * PFSF_SOLVE_NO_READBACK leaves the gradients on the device. */
PFSF_API pfsf_result pfsf_adjoint_to_tolerance(pfsf_engine engine, const int32_t* island_ids, int32_t count,
                                               double rel_tol, int32_t max_iter, uint32_t flags,
                                               pfsf_solve_stats* out);

/* Island labelling (no counterpart in the reference C ABI: the reference
 * labels through its Java/Vulkan label-propagation dispatch,
 * SH/label_prop_*.comp.glsl, PFSFLabelPropRecorder.java).  One record per
 * 26-connected component of the non-air voxels -- the reference's 12-uint
 * component layout (label_prop_summarise_alloc.comp.glsl:57-69). */
typedef struct pfsf_label_component {
    uint32_t root_label;  /* 1 + smallest flat index of the component */
    uint32_t block_count; /* voxels in the component */
    uint32_t anchored;    /* 1 if any voxel is PFSF_VOXEL_ANCHOR */
    uint32_t _pad0;
    uint32_t aabb_min[3]; /* x, y, z */
    uint32_t _pad1;
    uint32_t aabb_max[3];
    uint32_t _pad2;
} pfsf_label_component;

/* Labels the non-air voxels (uint8 type x lx*ly*lz, host) into 26-connected
 * components on the GPU.  out_labels (uint32 x N, host, may be NULL): every
 * voxel's component label = 1 + the smallest flat index in its component
 * (the fixed point of the reference's hook/jump label propagation),
 * 0xFFFFFFFF on air.  out_components: the first min(count, capacity)
 * components in ascending root_label order; *out_count = that number;
 * *out_overflow = 1 when there were more than capacity components.
 * Synchronous: returns after the outputs are written. */
PFSF_API pfsf_result pfsf_label_components(pfsf_engine engine, const uint8_t* voxel_type, int32_t lx, int32_t ly,
                                           int32_t lz, uint32_t* out_labels, pfsf_label_component* out_components,
                                           int32_t capacity, int32_t* out_count, int32_t* out_overflow);

/* Diagnostic read of the per-island tick state (not part of the reference
 * ABI; used by parity tests and tooling).  field: 0 phi (float32 x N),
 * 1 history H (float32 x N), 2 damage d (float32 x N), 3 failure flags
 * (uint8 x N), 4 macro-block residual bits (uint32 x blocks), 5 schedule state
 * {int32 chebyshev_iter, pcg_allocated, mg_allocated, float prev, last macro
 * residual} (20 bytes), and the device copies of the inputs: 6 source
 * (float32 x N), 7 face conductivity (float32 x 6N, SoA), 8 voxel type
 * (uint8 x N), 9 max_phi, 10 rcomp, 11 rtens (float32 x N), 12 aggregate of each voxel
 * (int32 x N, -1 left out), 13 prolongation weights (float32 x N), 14 coarse diagonal
 * (float32 per aggregate); 12-14 are empty until pfsf_set_amg's correction first runs.  Copies min(bytes, field size); *out_bytes gets the
 * field size. */
PFSF_API pfsf_result pfsf_debug_read_field(pfsf_engine engine, int32_t island_id, int32_t field, void* out,
                                           int64_t bytes, int64_t* out_bytes);

/* No counterpart in the reference ABI.  Failure-flag compaction that
 * allocates nothing, for callers that cannot call cudaMalloc / cudaFree (a
 * physics thread whose tick budget cannot absorb the device-wide
 * synchronisation those calls may cause, or code that only borrows device
 * buffers it does not own).  It runs the compaction pfsf_tick_dbb uses --
 * failure flags (uint8 x lx*ly*lz, on the device) to {x, y, z, type} int32
 * tuples in voxel order, world coordinates = origin + local -- with its
 * per-chunk scratch in a fixed array inside the library (128 KiB per GPU,
 * held until the process exits) instead of engine-allocated memory.
 *   dev_fail_flags, dev_tuples (capacity x 4 int32), dev_count (1 int32):
 *   device memory owned by the caller.  *dev_count receives the number of
 *   failed voxels, which may exceed capacity; tuples past capacity are
 *   dropped.
 *   stream: a cudaStream_t (NULL = legacy default stream); the call only
 *   enqueues work, the caller synchronises before reading the outputs.
 * Limits and rules: islands above 67,108,864 voxels are rejected with
 * PFSF_ERROR_INVALID_ARG.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) and caches it together with
 * the CUDA context current at the time; make that first call before any
 * stream capture.  After cudaDeviceReset (a new primary context) the next
 * call looks the address up again, so make that call outside a capture too.
 * An error already pending in the CUDA runtime when the call starts (from the
 * caller's own earlier work) is left pending and the call returns
 * PFSF_ERROR_VULKAN without launching anything.  All calls on a device share
 * the one array, so calls whose GPU work overlaps (different streams, no
 * ordering) race and corrupt each other's results; serialise them. */
PFSF_API pfsf_result pfsf_compact_failures_noalloc(const uint8_t* dev_fail_flags, int32_t lx, int32_t ly,
                                                   int32_t lz, pfsf_pos origin, int32_t* dev_tuples,
                                                   int32_t capacity, int32_t* dev_count, void* stream);

/* Test access (no counterpart in the reference ABI): evaluates on the current
 * device, for n host doubles s, the FP64 link reciprocal the tolerance solve
 * uses (hardware reciprocal + two Newton steps; IEEE division outside
 * [2^-1022, 2^1020]) into out_rcp64 and the IEEE quotient 1.0 / s into
 * out_ieee.  Allocates its own device memory; n <= 2^26. */
PFSF_API pfsf_result pfsf_debug_rcp64(const double* in, double* out_rcp64, double* out_ieee, int64_t n);

/* Test access (no counterpart in the reference ABI): one fine-level pass of
 * the whole-GPU tier on an island of the last batched solve (pass 0: a
 * Chebyshev smoothing step, 1: the FP32 matvec), repeated `reps` times on
 * the engine stream; *ms = mean time per pass (CUDA events), *bytes = the
 * pass's algorithmic bytes (the staged input vector and kappa of every box
 * cell, the per-solid-voxel arrays once). */
PFSF_API pfsf_result pfsf_debug_time_pass(pfsf_engine engine, int32_t island_id, int32_t pass, int32_t reps,
                                          float* ms, double* bytes);

/* The cudaStream_t the engine launches on (for event timing by callers). */
PFSF_API void* pfsf_get_stream(pfsf_engine engine);

/* Number of kernels this engine has launched since creation. */
PFSF_API int64_t pfsf_kernel_launch_count(pfsf_engine engine);

#ifdef __cplusplus
}
#endif
#endif
