/*
 * b2p_pdhg.h -- C ABI of the B200 (sm_100a) restarted-Halpern PDHG engine.
 *
 * This is the drop-in boundary for PRAMANA's PDHG engine.  The reference
 * exposes the path as C++ (src/pdhg/pdhg.h:73-80):
 *
 *   PdhgResult solvePdhg(const Model&, const PdhgOptions&, const Deadline*);
 *   std::vector<PdhgResult> solvePdhgBatch(const Model&, const std::vector<LpCase>&,
 *                                          const PdhgOptions&, const Deadline*, PdhgStats*);
 *   bool gpuAvailable();
 *   Json gpuInfoJson();
 *
 * and drives its GPU through gpu::CudaContext (src/gpu/cuda_driver.h:43-81)
 * and the GpuBackend class (src/pdhg/pdhg.cpp:219-389).  The entry points
 * below replace those: plain pointers and sizes, int return codes, no C++
 * types and no exceptions across the boundary.  Results are in the original
 * space of the (minimisation) model, exactly like PdhgResult.
 *
 * Errors: every function returns B2P_OK (0) or a B2P_ERR_* code, and
 * b2p_last_error() gives a message for the calling thread.  There is no CPU
 * fallback: without a usable sm_100 device the solve entry points return
 * B2P_ERR_NO_DEVICE.
 *
 * Threading: one solve per calling thread; an engine object must not be used
 * from two threads at once.
 */
#ifndef B2P_PDHG_H
#define B2P_PDHG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Return codes. */
enum {
  B2P_OK = 0,
  B2P_ERR_INVALID = 1,   /* bad argument or inconsistent model */
  B2P_ERR_CUDA = 2,      /* a CUDA runtime call failed */
  B2P_ERR_NO_DEVICE = 3, /* no usable sm_100 GPU (or disabled by PRAMANA_DISABLE_GPU) */
  B2P_ERR_OOM = 4,       /* device allocation failed */
  B2P_ERR_TOO_LARGE = 5  /* size beyond a documented maximum */
};

/* Termination status; the numbering is pramana::Status (src/util/common.h:27-39). */
enum {
  B2P_STATUS_NOT_SOLVED = 0,
  B2P_STATUS_OPTIMAL = 1,
  B2P_STATUS_TIME_LIMIT = 5,
  B2P_STATUS_ITERATION_LIMIT = 6
};

/* Kernel form of a single-LP solve. */
enum {
  B2P_KERNELS_AUTO = 0,
  B2P_KERNELS_FUSED = 1,    /* two fused SpMV kernels per iteration, CUDA graph per check interval */
  B2P_KERNELS_RESIDENT = 2  /* one persistent cooperative kernel per check interval, operators in shared memory */
};

/* Arithmetic of the iterates. */
enum {
  B2P_PRECISION_FP64 = 0, /* plain form: FP64 everywhere, iterate parity with the reference */
  /* mixed form: operator values and iterates stored in FP32, row sums of
   * exact FP32 products in FP64; check sums, termination, restarts and
   * primal weight in FP64.  A single LP (resident form) whose FP32 point meets
   * the tolerance is re-measured in FP64 before it is returned; when that
   * fails, or the FP32 run stalls, the solve continues in FP64 from the FP32
   * point (the FP64 polish).  A batch (num_cases > 1) runs in FP32 until
   * every case has met the tolerance there or stalled, then re-measures all
   * cases in FP64: those that pass terminate, the rest continue in FP64.  A
   * single LP too large for the resident form runs in FP64.  Many LPs
   * (b2p_solve_pdhg_multi) in the CTA form: every LP runs in FP32 until its
   * FP32 point meets the tolerance or stalls, then in FP64 from that point,
   * measured first; the block-diagonal form runs FP64 (stats.precision_used
   * says which ran). */
  B2P_PRECISION_MIXED = 1
};

/* A minimisation LP  min c'x + offset, L <= Ax <= U, l <= x <= u, with A in
 * CSC form.  Replaces pramana::Model + SparseMatrix (src/core/model.h:24-64,
 * src/core/sparse.h:11-16).  Bounds with |v| >= 1e20 are infinite. */
typedef struct b2p_lp {
  int32_t num_rows;
  int32_t num_cols;
  const int32_t* start; /* num_cols + 1 column pointers */
  const int32_t* index; /* row index of each nonzero */
  const double* value;
  const double* col_cost;
  const double* col_lower;
  const double* col_upper;
  const double* row_lower;
  const double* row_upper;
  double obj_offset;
} b2p_lp;

/* One case of a family sharing A; NULL means "same as the base model".
 * Replaces pramana::LpCase (src/pdhg/pdhg.h:67-70). */
typedef struct b2p_case {
  const double* cost;
  const double* col_lower;
  const double* col_upper;
  const double* row_lower;
  const double* row_upper;
} b2p_case;

/* Replaces pramana::PdhgOptions (src/pdhg/pdhg.h:32-42) plus the Deadline
 * (src/util/timer.h:22-42) and the device choice (PRAMANA_GPU_DEVICE,
 * src/gpu/cuda_driver.cpp:223). */
typedef struct b2p_options {
  double tolerance;         /* relative KKT tolerance (default 1e-6) */
  int64_t max_iterations;   /* default 1,000,000 */
  int32_t check_every;      /* iterations between convergence checks (default 64) */
  int32_t ruiz_iterations;  /* default 10 */
  int32_t pock_chambolle;   /* default 1 */
  int32_t rescale_objective_and_bounds; /* default 1 */
  double reflection;        /* rho in [0,1] (default 1) */
  int32_t log_interval;     /* progress line every N checks on stderr (0 = off) */
  int32_t device;           /* CUDA ordinal; -1 = PRAMANA_GPU_DEVICE or 0 */
  double time_limit;        /* seconds; <= 0 = none */
  const volatile int32_t* cancel_flag; /* polled at every check when non-NULL; nonzero = stop */
  int32_t precision;        /* B2P_PRECISION_* */
  int32_t use_graphs;       /* capture each check interval as one CUDA graph (default 1) */
  /* SpMV schedule of the single-LP kernels (0 = automatic): lanes per short
   * row of A and of A^T (a power of two, 1..32), and how many rounds of 4
   * entries per lane a short row may take before it moves to the one-warp-
   * per-row path. */
  int32_t lanes_per_row_a;
  int32_t lanes_per_row_at;
  int32_t short_row_rounds;
  /* Single-LP kernel form: B2P_KERNELS_AUTO picks the resident form when the
   * LP's operators fit in the SMs' shared memory. */
  int32_t kernel_mode;
  /* SpMV schedule of the multi-LP engine's fused kernels, per operator:
   * B2P_SCHEDULE_BINNED (rows binned by length, lanes per short row),
   * B2P_SCHEDULE_TILED (warp tiles of up to 32 short rows whose entries one
   * warp loads coalesced), B2P_SCHEDULE_TUNED (the autotuner times every
   * binned lane count and the tiles on the device and keeps the fastest), or
   * B2P_SCHEDULE_AUTO (TUNED from 2^20 nonzeros on, BINNED below). */
  int32_t spmv_schedule;
  /* Multi-LP engine form (B2P_MULTI_*): the block-diagonal form (every LP's
   * rows in the same fused kernels, host decisions at each check, one CUDA
   * graph per check interval) or the CTA form (one thread block runs one LP's
   * whole loop, decisions included, in a single launch).  B2P_MULTI_AUTO
   * picks the CTA form when every LP fits one block's shared memory. */
  int32_t multi_form;
  /* CTA form: bytes of shared memory one LP may use (0 = the device's
   * per-block maximum); an LP that does not fit keeps its operators, or all
   * of its data, in global memory. */
  int32_t cta_smem_limit;
  /* CTA form: threads per block (128, 256, 512 or 1024; 0 = autotuned with
   * the kernel variant). */
  int32_t cta_threads;
  /* CTA form: kernel variant (B2P_CTA_*; 0 = autotuned): the general kernel
   * (any LP size, three storage tiers) or the owner kernel, whose threads
   * each own 1 or 2 rows and columns and keep their state in registers (LPs
   * with max(m, n) <= 2 x threads whose data fit in shared memory). */
  int32_t cta_kernel;
  /* FP64 batches (k > 1 cases sharing A): variant of the two per-iteration
   * kernels -- 0 = timed on the device when the batch's vectors far exceed L2
   * (plain otherwise); 1..4 force (cases per thread, evict-first streamed
   * vectors) = (1, no), (2, no), (1, yes), (2, yes); 5..8 the same with whole
   * warps per row (row entries loaded once per warp and shared by shuffle)
   * where k / cases per thread is a multiple of 32; 9..16, 17..24 and 25..32
   * are 1..8 in the row-tiled layouts of 4, 8 and 16 rows per block (each
   * warp one row, the warps of a block on consecutive rows of one chunk of 32
   * cases, the blocks chunk by chunk). */
  int32_t batch_variant;
  /* Batches (k > 1 cases sharing A), FP64 phase: 0 = whenever half of the
   * live cases have terminated, pack the others into a narrower interleave
   * (each case's state moves unchanged, so its iterates do not change; the
   * kernels stop streaming the finished cases' vectors); 1 = never. */
  int32_t batch_no_compaction;
  /* CTA form: layout of the operators its general kernel reads from global
   * memory -- B2P_CTA_LAYOUT_AUTO (sliced ELL: the entries of 32 consecutive
   * rows interleaved so that a warp's loads are coalesced) or
   * B2P_CTA_LAYOUT_CSR (the CSR arrays as they are).  The row sums are the
   * same in both (left to right per row), so are the iterates. */
  int32_t cta_layout;
  int32_t pad_options;
} b2p_options;
enum { B2P_CTA_LAYOUT_AUTO = 0, B2P_CTA_LAYOUT_CSR = 1 };
enum { B2P_MULTI_AUTO = 0, B2P_MULTI_GRID = 1, B2P_MULTI_CTA = 2 };
enum { B2P_CTA_AUTO = 0, B2P_CTA_GENERAL = 1, B2P_CTA_OWNER1 = 2, B2P_CTA_OWNER2 = 3 };

enum { B2P_SCHEDULE_AUTO = 0, B2P_SCHEDULE_BINNED = 1, B2P_SCHEDULE_TILED = 2, B2P_SCHEDULE_TUNED = 3 };

/* Replaces pramana::PdhgStats (src/pdhg/pdhg.h:44-56). */
typedef struct b2p_stats {
  int64_t iterations;
  int32_t restarts;
  int32_t pad0;
  double primal_residual, dual_residual, gap;
  double primal_weight;
  double setup_seconds, solve_seconds;
  double kernel_seconds;   /* device time of the iteration loop (CUDA events) */
  double transfer_seconds; /* host<->device copies */
  int64_t bytes_uploaded, bytes_downloaded, kernel_launches;
  double spectral_norm;
  /* setup breakdown: prepare = the CSR of A on host threads, then the upload
   * of A and A^T, the scaling and the ||A|| estimate on the device; upload =
   * everything after the host structure (uploads, device scaling, case
   * vectors; overlaps prepare); graph = kernel set-up (schedules,
   * resident-form set-up, capture and instantiation of the CUDA graphs) */
  double prepare_seconds, upload_seconds, graph_seconds;
  int32_t lanes_per_row_a, lanes_per_row_at; /* schedule used */
  int32_t kernel_mode;                        /* B2P_KERNELS_FUSED or B2P_KERNELS_RESIDENT (batches: FUSED) */
  int32_t resident_blocks;                    /* cooperative grid size in resident form */
  int64_t resident_smem_bytes;                /* largest block's shared memory in resident form */
  int32_t precision_used;                     /* B2P_PRECISION_* actually run */
  int32_t batch_compactions;                  /* batches: times the live cases were packed narrower */
  int64_t fp32_iterations;                    /* mixed form: iterations run in FP32 */
  int32_t schedule_a, schedule_at;            /* multi-LP: B2P_SCHEDULE_BINNED or _TILED per operator */
  double autotune_seconds;                    /* multi-LP: time the autotuner took (part of setup) */
  int32_t streaming_a, streaming_at;          /* multi-LP binned schedules, FP64 batches: evict-first streaming loads */
  int32_t multi_form;                         /* multi-LP: B2P_MULTI_GRID or B2P_MULTI_CTA */
  int32_t cta_threads;                        /* CTA form: threads per block (autotuned) */
  int64_t cta_smem_bytes;                     /* CTA form: dynamic shared memory per block */
  int32_t cta_lps_smem;                       /* CTA form: LPs held wholly in shared memory */
  int32_t cta_lps_vectors;                    /* CTA form: LPs with only their iterates in shared memory */
  int32_t cta_owned_per_thread;               /* CTA form: rows and columns each thread owns (0 = general kernel) */
  int32_t tile_rows_at;                       /* FP64 batches: rows per block of the A^T kernel's row-tiled layout (0 = none) */
  int32_t cases_per_thread_at, cases_per_thread_a; /* FP64 batches: cases per thread of the A^T / A kernels */
  int32_t warp_rows_at, warp_rows_a;          /* FP64 batches: whole warps per row, entries shared by shuffle */
  int32_t tile_rows_a;                        /* FP64 batches: the same for the A kernel */
  int32_t cta_sliced;                         /* CTA form: 1 if the sliced-ELL operators were built and used */
} b2p_stats;

/* Replaces pramana::PdhgResult (src/pdhg/pdhg.h:58-65) minus the vectors,
 * which go to caller-provided arrays. */
typedef struct b2p_result {
  int32_t status; /* B2P_STATUS_* */
  int32_t pad0;
  int64_t iterations;
  double objective, dual_objective;
  double relative_kkt;
} b2p_result;

/* Fills the reference defaults (src/pdhg/pdhg.h:32-42). */
void b2p_default_options(b2p_options* opts);

/* solvePdhg (src/pdhg/pdhg.cpp:712-717): x[num_cols], row_dual[num_rows]
 * receive the solution in the original space; either may be NULL. */
int b2p_solve_pdhg(const b2p_lp* lp, const b2p_options* opts, double* x, double* row_dual, b2p_result* result,
                   b2p_stats* stats);

/* solvePdhgBatch (src/pdhg/pdhg.cpp:719-728): num_cases LPs sharing A.
 * x is num_cases x num_cols and row_dual num_cases x num_rows (row-major by
 * case); results has num_cases entries. */
int b2p_solve_pdhg_batch(const b2p_lp* base, const b2p_case* cases, int32_t num_cases, const b2p_options* opts,
                         double* x, double* row_dual, b2p_result* results, b2p_stats* batch_stats);

/* Many independent LPs of different sizes (each with its own A) in one
 * solve.  No counterpart in the reference, which batches only cases sharing
 * one A (solvePdhgBatch); each LP here gets exactly the reference's algorithm
 * (its own scaling, steps, primal weight, restarts and termination), and all
 * of them advance together as one block-diagonal operator on the GPU.
 * x_start[b] / row_dual_start[b], when given (either array or entry may be
 * NULL), warm-start LP b (original space; x is projected onto the bounds).
 * x[b] (num_cols of LP b) and row_dual[b] (num_rows) receive LP b's
 * solution (either array, or any entry, may be NULL); results has num_lps
 * entries.  stats: kernel_seconds is the device time of the loop;
 * iterations the global iteration count. */
int b2p_solve_pdhg_multi(const b2p_lp* lps, int32_t num_lps, const b2p_options* opts, const double* const* x_start,
                         const double* const* row_dual_start, double* const* x, double* const* row_dual,
                         b2p_result* results, b2p_stats* stats);

/* b2p_solve_pdhg_multi with primal weights in and out (no counterpart in the
 * reference, whose primal weight starts at ||c|| / ||b|| of the scaled LP,
 * src/pdhg/pdhg.cpp:497-500).  Weights are in the original space's units:
 * w = omega gamma / beta, omega the scaled LP's primal weight and beta /
 * gamma its bound and objective rescalings, so that LPs of one family with
 * different rescalings exchange them.  primal_weight_start[b] (the array may
 * be NULL; entries that are not finite and positive keep the default) sets
 * LP b's initial weight; primal_weight[b] (may be NULL) receives its weight
 * at termination.  b2p_solve_pdhg_multi is this call with both NULL. */
int b2p_solve_pdhg_multi_warm(const b2p_lp* lps, int32_t num_lps, const b2p_options* opts,
                              const double* const* x_start, const double* const* row_dual_start,
                              const double* primal_weight_start, double* const* x, double* const* row_dual,
                              double* primal_weight, b2p_result* results, b2p_stats* stats);

/* gpuAvailable (src/pdhg/pdhg.cpp:730): 1 if an sm_100 device is usable. */
int b2p_gpu_available(void);

/* gpuInfoJson (src/pdhg/pdhg.cpp:732-746): writes a NUL-terminated JSON
 * object into buf (cap bytes) and returns the full length needed. */
int b2p_gpu_info_json(char* buf, size_t cap);

/* Message of the last error on this thread ("" if none). */
const char* b2p_last_error(void);

/* ---- Two-phase form of the same solve --------------------------------------
 * b2p_engine_create does the work of runPdhg before its loop (prepare,
 * GpuBackend::init uploads, case vectors; src/pdhg/pdhg.cpp:485-558);
 * b2p_engine_solve runs the loop (pdhg.cpp:560-687) from the initial point,
 * and may be called again to repeat the identical solve; b2p_engine_fetch
 * copies the last solution back.  num_cases <= 0 means a single solve of the
 * base model. */
typedef struct b2p_engine b2p_engine;

int b2p_engine_create(const b2p_lp* lp, const b2p_case* cases, int32_t num_cases, const b2p_options* opts,
                      b2p_engine** out);
int b2p_engine_solve(b2p_engine* e, b2p_result* results, b2p_stats* stats);
int b2p_engine_fetch(b2p_engine* e, double* x, double* row_dual);
int b2p_engine_destroy(b2p_engine* e);
/* Warm start: the starting point of the following b2p_engine_solve calls, in
 * the original space -- x is num_cases x num_cols, row_dual num_cases x
 * num_rows (case-major; num_cases = 1 for a single solve); x is projected
 * onto the bounds; primal_weight > 0 replaces the initial primal weight of
 * every case.  NULL x and NULL row_dual restore the cold start.  No
 * counterpart in the reference, whose PDHG always starts from x = projection
 * of 0, y = 0 (src/pdhg/pdhg.cpp:509, 519, 536-539). */
int b2p_engine_set_start(b2p_engine* e, const double* x, const double* row_dual, double primal_weight);
/* When on, every fused SpMV kernel launch (and, in resident form, every
 * interval launch) of the next solve is bracketed by CUDA events;
 * b2p_engine_kernel_times then returns, per kernel class (0 = A^T y + primal
 * step, 1 = A x+ + dual step, 2 = resident interval kernel, 3 / 4 = the FP32
 * primal / dual kernels of a mixed-precision batch), the count and the summed
 * device milliseconds; for class 2 the count is in iterations. */
int b2p_engine_set_profiling(b2p_engine* e, int32_t on);
int b2p_engine_kernel_times(b2p_engine* e, int32_t kernel_class, int64_t* launches, double* total_ms);
/* Algorithmic bytes of one launch of a kernel class (CSR values, indices and
 * row pointers read once, gathered vector read once, every streamed vector
 * read or written once; classes 3 and 4 with 4-byte values and vectors);
 * class 2: bytes of one iteration (classes 0 + 1). */
int b2p_engine_kernel_bytes(b2p_engine* e, int32_t kernel_class, double* bytes);

/* ---- KKT evaluation ---------------------------------------------------------
 * Relative KKT error of caller-given points, as runPdhg measures it at every
 * check (src/pdhg/pdhg.cpp:166-197, 608-615), in the original space: for case
 * b, out[4b..4b+3] = relative primal residual, relative dual residual,
 * relative gap, and their maximum.  x is num_cases x num_cols, row_dual
 * num_cases x num_rows (case-major); num_cases <= 0 means one point of the
 * base model.  Host arrays in and out.  (The reference computes this only
 * inside its loop; this entry judges points from elsewhere, e.g. warm
 * starts.) */
int b2p_kkt_residual(const b2p_lp* lp, const b2p_case* cases, int32_t num_cases, const double* x,
                     const double* row_dual, double* out);

/* ---- Certification ----------------------------------------------------------
 * Rigorous outward-rounded Neumaier-Shcherbina lower bound on
 * min { c'x : L <= Ax <= U, l <= x <= u } (objective offset excluded) that is
 * valid for ANY row dual y, for num_cases cases of a shared A at once
 * (num_cases <= 0: one case, the base model).  Replaces safeDualBound /
 * SafeBoundResult (src/cert/certifier.h:79-96, certifier.cpp:58-118) and gives
 * bit-identical results: same projection of y, same outward-rounded interval
 * reduced costs in column order, same in-order downward sum.  row_dual is
 * num_cases x num_rows (case-major); out has num_cases entries. */
typedef struct b2p_safe_bound {
  double bound;                  /* -inf when a wrong-signed reduced cost sits on an infinite bound */
  int32_t infinite_terms;        /* columns that forced -inf */
  int32_t pad0;
  double max_dual_infeasibility; /* largest clipped wrong-signed reduced cost */
  double row_projection;         /* largest change of y by the sign-cone projection */
  double cost_perturbation;      /* relative cost change the clipped bound is rigorous for */
} b2p_safe_bound;

int b2p_safe_dual_bound(const b2p_lp* lp, const b2p_case* cases, int32_t num_cases, const double* row_dual,
                        b2p_safe_bound* out);

/* Constraint-implied column bounds, for num_cases cases of a shared A at once
 * (num_cases <= 0: one case, the base model): what the certifier of the
 * reference falls back on for first-order duals (src/cert/certifier.cpp:340-356
 * over Propagator::propagate, src/mip/propagate.cpp:23-138), computed on the
 * GPU by activity-based bound tightening in Jacobi rounds -- every row's
 * activity range from the previous round's bounds, then every column's
 * bounds intersected with what its rows imply -- with every operation rounded
 * in the safe direction, so the bounds contain every feasible point of the
 * exact LP.  Rounds run until no bound moves by more than 1e-9 relative (at
 * most 1,024).  Untightened bounds are returned as given; a case proved
 * infeasible keeps the bounds it had when that was found.  Outputs are
 * num_cases x num_cols (case-major).  The reference relaxes each tightened
 * bound by 1e-6 (1 + |bound|) instead of rounding outward, so its bounds are
 * looser by about that much; both are valid. */
int b2p_implied_bounds(const b2p_lp* lp, const b2p_case* cases, int32_t num_cases, double* col_lower_out,
                       double* col_upper_out);

/* The certifier's verdict on an OPTIMAL claim (x, row_dual) of an LP
 * (certify, src/cert/certifier.cpp:208-380, LP branch), for num_cases cases
 * of a shared A at once, on the GPU: relative column and row violations
 * against primal_feasibility (row activities as compensated dot products),
 * the objective c'x + offset (compensated), the outward-rounded safe dual
 * bound of b2p_safe_dual_bound -- retried over the constraint-implied column
 * bounds of b2p_implied_bounds when it is -inf -- rounded down with the
 * offset, and the relative gap (pobj - LB) / max(1, |pobj|) against
 * relative_gap; without a finite bound the largest wrong-signed reduced cost
 * is held against dual_feasibility.  The safe bound over the given column
 * bounds is bit-identical to the reference's; the primal figures agree with
 * the reference's to rounding (the sums are compensated differently).  x is
 * num_cases x num_cols, row_dual num_cases x num_rows (case-major). */
typedef struct b2p_cert_tolerances {
  double primal_feasibility; /* CertTolerances::primalFeas, 1e-6 */
  double dual_feasibility;   /* CertTolerances::dualFeas, 1e-6 */
  double relative_gap;       /* CertTolerances::relGap, 1e-6 */
} b2p_cert_tolerances;

typedef struct b2p_certificate {
  int32_t accepted;              /* Certificate::accepted */
  int32_t used_implied_bounds;   /* the bound came from constraint-implied column bounds */
  double primal_objective;       /* c'x + offset */
  double safe_dual_bound;        /* rigorous lower bound incl. offset, -inf if none */
  double certified_gap;          /* relative gap, +inf without a bound */
  double max_primal_violation;   /* max of the two below */
  double max_col_violation;      /* relative column-bound violation */
  double max_row_violation;      /* relative row violation */
  double max_dual_violation;     /* SafeBoundResult::maxDualInfeasibility */
  double cost_perturbation;      /* SafeBoundResult::costPerturbation */
  int32_t infinite_terms;
  int32_t worst_row;             /* row of max_row_violation, -1 if none */
} b2p_certificate;

int b2p_certify_lp(const b2p_lp* lp, const b2p_case* cases, int32_t num_cases, const double* x,
                   const double* row_dual, const b2p_cert_tolerances* tol, b2p_certificate* out);

/* Allocation-free form of b2p_kkt_residual.  No counterpart in the
 * reference.  For callers that cannot allocate device memory (a host
 * framework that owns all device memory through its own pool, or a path where
 * allocation is forbidden): every array is a caller-owned DEVICE pointer of
 * the current device, and the call itself allocates nothing.  Inputs: A as
 * CSR (a_ptr[num_rows+1], a_idx, a_val) and as CSC read as the CSR of A^T
 * (at_ptr[num_cols+1], at_idx, at_val), and per point b (case-major) cost,
 * col_lower, col_upper (num_points x num_cols), row_lower, row_upper
 * (num_points x num_rows), x and row_dual.  Output: out[4b..4b+3] as in
 * b2p_kkt_residual, written on `stream` (a cudaStream_t; NULL = the legacy
 * default stream) -- the call only enqueues; synchronize the stream before
 * reading out.
 * Checks before any launch: each array the kernels may read or write must be
 * memory of the current device (host memory, unregistered addresses and other
 * GPUs' memory give B2P_ERR_INVALID naming the argument; a_idx, a_val, at_idx
 * and at_val may be NULL only when num_rows or num_cols is 0).  A CUDA error
 * left pending on the calling thread by earlier work is neither cleared nor
 * charged to this call: the call returns B2P_ERR_CUDA without launching.  A
 * failure of its own launches is returned as B2P_ERR_CUDA and cleared.
 * Scratch: the reductions' block partials live in one file-scope device array
 * of 458,752 bytes, which every GPU that loads this library holds until the
 * process exits.  num_points above 32 is rejected with B2P_ERR_TOO_LARGE.
 * Every call shares that array and it keeps the last call's contents (the
 * kernels write every partial before reading it, so nothing has to start at
 * zero); calls that overlap on the GPU -- on different streams or from
 * different threads without ordering -- race on it.  The first call on a
 * device looks the array's device address up (cudaGetSymbolAddress, once per
 * device, with that device current); make that first call before any stream
 * capture. */
int b2p_kkt_residual_noalloc(int32_t num_rows, int32_t num_cols, int32_t num_points, const int32_t* a_ptr,
                             const int32_t* a_idx, const double* a_val, const int32_t* at_ptr, const int32_t* at_idx,
                             const double* at_val, const double* cost, const double* col_lower,
                             const double* col_upper, const double* row_lower, const double* row_upper,
                             const double* x, const double* row_dual, double* out, void* stream);

/* ---- Kernel-level entry -------------------------------------------------
 * y(i,b) = sum_p val[p] * x(idx[p], b) for a CSR matrix (rows x cols) and k
 * interleaved right-hand sides (element (i,b) at i*k+b), summed left to right
 * like CpuBackend::mult (src/pdhg/pdhg.cpp:93-103).  Host arrays in and out. */
int b2p_csr_spmv(int32_t rows, int32_t cols, int32_t k, const int32_t* ptr, const int32_t* idx, const double* val,
                 const double* x, double* y);

#ifdef __cplusplus
}
#endif

#endif /* B2P_PDHG_H */
