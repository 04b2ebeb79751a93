/*
 * pdlp_b200 -- C ABI of the B200-native PDLP engine.
 *
 * This library replaces, for the `--method pdlp` path of sovopt
 * (manabsen006-a11y/Sovereign-MOE), two reference interfaces:
 *
 *   1. the solver entry point  solve_pdlp(prob, params) -> Solution
 *      (src/sovopt/lp/pdlp.py:238-494, parameters pdlp.py:79-116,
 *      info pdlp.py:119-132), and
 *   2. the kernel-level Backend the solver is written against
 *      (src/sovopt/core/backend.py:317-493: spmv, primal_step, dual_step,
 *      pdhg_primal, pdhg_dual, pdhg_accum, dot, nrm2, nrm_inf).
 *
 * Conventions
 *   - Every call returns int: 0 on success, a negative PDLP_ERR_* code on
 *     failure; pdlp_last_error() gives a thread-local message.
 *   - Pointers are plain device pointers unless a `memory` argument says
 *     PDLP_MEM_HOST.  The library never frees memory it did not allocate; it
 *     owns only its handles' scratch.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *   - A handle (pdlp_batch) is used from one host thread at a time.
 *   - Sparse matrices use the reference's storage (src/sovopt/core/sparse.py:
 *     263-298): int64 pointers, int32 indices, float64 values, held in both
 *     CSR (rows) and CSC (columns).
 */
#ifndef PDLP_B200_H
#define PDLP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PDLP_ABI_VERSION 5

/* ---- error codes ------------------------------------------------------- */
#define PDLP_OK                   0
#define PDLP_ERR_ARG             -1   /* invalid argument / malformed input   */
#define PDLP_ERR_OOM             -2   /* device memory does not fit           */
#define PDLP_ERR_CUDA            -3   /* a CUDA runtime call failed           */
#define PDLP_ERR_BARRIER_TIMEOUT -4   /* a bounded device wait gave up        */
#define PDLP_ERR_NUMERICAL       -5   /* non-finite input data                */
#define PDLP_ERR_STATE           -6   /* call not valid in the handle's state */
#define PDLP_ERR_BOUNDS          -7   /* an index check failed (bounds-checked
                                         builds only, -DPDLP_BOUNDS_CHECK)    */

/* ---- statuses: same integers as sovopt Status (src/sovopt/core/problem.py:58-69) */
#define PDLP_STATUS_OPTIMAL          0
#define PDLP_STATUS_INFEASIBLE       1
#define PDLP_STATUS_INFEASIBLE_OR_UNBOUNDED 3
#define PDLP_STATUS_ITERATION_LIMIT  4
#define PDLP_STATUS_TIME_LIMIT       5
#define PDLP_STATUS_NUMERICAL        8
#define PDLP_STATUS_INTERRUPTED      9
#define PDLP_STATUS_RUNNING         -1

#define PDLP_MEM_DEVICE 0
#define PDLP_MEM_HOST   1

/* scaling methods (params.scaling of pdlp.py:113; scaling.py:312-318) */
#define PDLP_SCALING_PDLP            0   /* Ruiz (10) then Pock-Chambolle, pow2 */
#define PDLP_SCALING_NONE            1
#define PDLP_SCALING_RUIZ            2   /* Ruiz (20), pow2                     */
#define PDLP_SCALING_POCK_CHAMBOLLE  3

/* arithmetic of the iteration's sparse products (the reference: float64) */
#define PDLP_PRECISION_FP64          0   /* everything float64                  */
#define PDLP_PRECISION_FP32_SPMV     1   /* A x / A'y of the iteration in float32
                                            (values, gathered directions and the
                                            row sums); iterates, running sums,
                                            KKT, restarts and objective float64 */

/* One LP in the reference's row-bounds form rl <= Ax <= ru, l <= x <= u
 * (src/sovopt/core/problem.py:81-128).  Infinite bounds are +-1e30. */
typedef struct pdlp_problem_desc {
    int32_t m, n;
    int64_t nnz;
    const int64_t* rp; const int32_t* ri; const double* rx;   /* CSR of A */
    const int64_t* cp; const int32_t* ci; const double* cx;   /* CSC of A */
    const double* c;
    const double* row_lb; const double* row_ub;
    const double* col_lb; const double* col_ub;
    const uint8_t* kind;        /* optional (NULL): VarKind per column; non-zero
                                   columns keep a scale factor of 1         */
    double obj_offset;
    int32_t sense;              /* 1 minimise, -1 maximise (ObjSense)       */
    int32_t memory;             /* PDLP_MEM_DEVICE or PDLP_MEM_HOST          */
} pdlp_problem_desc;

/* PDLPParams (src/sovopt/lp/pdlp.py:79-116), same names and defaults. */
typedef struct pdlp_params {
    double eps_abs, eps_rel, feas_cap;
    int64_t max_iter;
    double time_limit;                  /* seconds, measured from admission  */
    int32_t check_every, stepsize_every;
    double beta_sufficient, beta_necessary, beta_artificial;
    double primal_weight_smoothing;
    int32_t scaling;                    /* PDLP_SCALING_*                    */
    const double* power_start;          /* optional n-vector (memory as the
                                           problem) starting the power
                                           iteration for ||A||_2 (pdlp.py:
                                           140-159 uses default_rng(0)); NULL:
                                           a fixed device-generated vector   */
    double time_used;                   /* seconds already spent by the caller
                                           (counts against time_limit)       */
    int32_t history_capacity;           /* checks recorded (0 = none)        */
    int32_t precision;                  /* PDLP_PRECISION_*                  */
    /* Infeasibility detection (no counterpart in the reference, whose PDLP
     * runs an infeasible LP to its iteration or time limit).  When nonzero,
     * the change of the iterates between checks of at least 256 iterations is
     * tested as a Farkas ray: a dual ray certifying primal infeasibility ends
     * the solve as PDLP_STATUS_INFEASIBLE, and a primal ray certifying dual
     * infeasibility ends it as PDLP_STATUS_INFEASIBLE_OR_UNBOUNDED; either
     * must hold at two checks in a row, with a violation at most
     * eps_infeasible times the ray's objective.  Off by default. */
    int32_t detect_infeasibility;
    double eps_infeasible;              /* default 1e-8                      */
    /* Scheduling hint (no counterpart in the reference): the caller's
     * estimate of the PDHG iterations this LP needs, 0 = none.  When every
     * running LP of a batch has one, the engine sizes their block teams by
     * expected remaining work (work per iteration times the square root of
     * the iterations left) instead of work per iteration, so that the LPs
     * expected to run longest get more blocks.  Results do not depend on it:
     * an LP's bits are the same whichever warps run its tiles. */
    double expected_iterations;
} pdlp_params;

void pdlp_params_default(pdlp_params* p);

/* Result of one solve: PDLPInfo (pdlp.py:119-132) plus the Solution scalars. */
typedef struct pdlp_result {
    int32_t status;
    int64_t iterations, restarts, rejected_steps;
    double primal_res, dual_res, gap, primal_obj, dual_obj;  /* NaN unless OPTIMAL */
    double step_size, primal_weight;
    double objective;              /* c'x + offset of the returned point       */
    double scale_obj;              /* objective scale of the preconditioner    */
    int32_t history_len;           /* checks recorded in the history buffer    */
    double device_seconds;         /* engine time for this LP on the device    */
    int64_t device_start_ns;       /* device clock (%globaltimer, ns) at the
                                      LP's first engine pass, and at its end
                                      (0 while running); comparable between
                                      the LPs of one device                  */
    int64_t device_end_ns;
} pdlp_result;

/* ---- library ---------------------------------------------------------- */
int pdlp_abi_version(void);
const char* pdlp_last_error(void);
/* Number of kernels this library has launched in the process so far (all
 * entry points); lets a caller count the GPU launches inside a timed region.
 * No counterpart in the reference (its kernels are CuPy RawModule calls). */
int64_t pdlp_launch_count(void);

/* ---- whole solve: solve_pdlp (pdlp.py:238-494) ------------------------- *
 * Solves one LP: scaling, PDHG, restarts and termination all run on the
 * device.  x (n), y (m), reduced_costs (n) receive the unscaled solution with
 * the reference's conventions (y textbook sign, d = c - A'y, x clipped to its
 * bounds); any of them may be NULL.  history (optional, 5*capacity doubles)
 * receives (k, primal_res, dual_res, gap, primal_obj) per check.  All output
 * pointers live in `out_memory`. */
int pdlp_solve(const pdlp_problem_desc* prob, const pdlp_params* params,
               void* stream, pdlp_result* result,
               double* x, double* y, double* reduced_costs, double* history,
               int32_t out_memory);

/* ---- batched / served engine ------------------------------------------- *
 * A batch holds device-resident LPs ("slots") that one persistent kernel
 * advances together, each with its own step size, primal weight, restart
 * state and termination.  LPs may be admitted and retired between steps. */
typedef struct pdlp_batch pdlp_batch;

typedef struct pdlp_batch_config {
    int32_t max_slots;          /* capacity of the slot table               */
    int32_t persistent;         /* 1: one cooperative launch per call to
                                   pdlp_batch_step; 0: one launch per phase
                                   (replayed from a CUDA graph)             */
    int32_t block_threads;      /* 0 = default (128); no other value is
                                   accepted                                 */
    int32_t tile_rows;          /* 0 = default                              */
    int32_t tile_nnz;           /* 0 = default                              */
    int32_t lanes_override;     /* 0 = per-LP choice; else lanes per row    */
    int64_t memory_budget;      /* bytes the batch may hold; 0 = free HBM   */
    int64_t barrier_timeout_us; /* wall-clock limit of every device-side wait
                                   (team barriers, staging copies); 0 = 4 s.
                                   A wait that runs out ends the step with
                                   PDLP_ERR_BARRIER_TIMEOUT and the batch
                                   refuses later calls (PDLP_ERR_STATE)     */
    int32_t autotune;           /* 1: an admitted LP whose nnz profile has an
                                   entry in the process's tuning cache
                                   (pdlp_tune_lp) takes its lanes per row and
                                   tile shape from it; 0: the engine's fixed
                                   rules (lanes from the mean row length,
                                   tiles tile_rows x tile_nnz)             */
    int32_t test_withhold_arrival; /* test hook, 0 = off.  1: the last block
                                   of the first team of two or more blocks
                                   leaves the kernel at its first barrier
                                   without arriving, so the team's bounded
                                   wait runs out (a flag nothing sets); it
                                   exercises the timeout path without any
                                   device fault                             */
} pdlp_batch_config;

void pdlp_batch_config_default(pdlp_batch_config* cfg);
int pdlp_batch_create(const pdlp_batch_config* cfg, void* stream, pdlp_batch** out);
int pdlp_batch_destroy(pdlp_batch* b);
/* Copies (host or device) and preconditions one LP into a free slot.
 * Returns PDLP_ERR_OOM when it does not fit the memory budget, leaving the
 * batch unchanged. */
int pdlp_batch_admit(pdlp_batch* b, const pdlp_problem_desc* prob,
                     const pdlp_params* params, int32_t* slot_out);
/* Admits `count` LPs (arrays of descriptors and parameters; params NULL for
 * the defaults) with three host synchronisations in all instead of two per
 * LP: one for the device pointer arrays (only when an LP is in device
 * memory), one for the device checks' verdicts and one at the end.  The
 * device work of the whole call is two launches: one kernel copies every
 * device-resident input into the slots (an array declared PDLP_MEM_DEVICE
 * must be device or managed memory, else PDLP_ERR_ARG), one validates every
 * LP's arrays.
 * slots_out[i] and codes_out[i] (each optional) receive each LP's slot (-1
 * when refused) and code; a refused LP leaves the others admitted.  Returns
 * the first refusal's code (its message in pdlp_last_error) or PDLP_OK.
 * No counterpart in the reference, which solves one LP per call. */
int pdlp_batch_admit_many(pdlp_batch* b, int32_t count, const pdlp_problem_desc* probs,
                          const pdlp_params* params, int32_t* slots_out, int32_t* codes_out);
/* Advances every running slot by `max_steps` engine steps (a step is one
 * half-iteration pair: the A pass and the A^T pass), or until it finishes.
 * The call returns once every slot that was running has done its max_steps
 * steps or finished; *active_out receives the number still running.  With
 * 256 or fewer slots running, each slot steps at its own pace on its own team
 * of blocks, in one or more launches. */
int pdlp_batch_step(pdlp_batch* b, int64_t max_steps, int32_t* active_out);
/* Status and info of a slot (status PDLP_STATUS_RUNNING while running). */
int pdlp_batch_poll(pdlp_batch* b, int32_t slot, pdlp_result* result);
/* Copies a finished slot's solution out (pointers in `memory`; NULL skips). */
int pdlp_batch_fetch(pdlp_batch* b, int32_t slot, double* x, double* y,
                     double* reduced_costs, double* history, int32_t memory);
/* Status of every slot as of the last pdlp_batch_step (no device access):
 * status_out[s] for s < n is PDLP_STATUS_RUNNING, a final status, or
 * PDLP_SLOT_FREE for an unused slot. */
#define PDLP_SLOT_FREE -2
int pdlp_batch_statuses(pdlp_batch* b, int32_t* status_out, int32_t n);
/* Releases a slot.  Its device arena is kept for later admissions (best
 * fit, at most twice the size needed); kept arenas count against the memory
 * budget, are freed before an admission would be refused, and are freed by
 * pdlp_batch_destroy. */
int pdlp_batch_retire(pdlp_batch* b, int32_t slot);
/* Poll, fetch and (when retire != 0) retire n finished slots at once: their
 * results into results[0..n) (optional), x[i], y[i], d[i] and history[i] as
 * pdlp_batch_fetch writes them (each pointer array optional, each entry may be
 * NULL), with one synchronisation of the batch's stream for the whole set
 * (two when histories are fetched) instead of three per slot.  A running, free or repeated slot is refused
 * (PDLP_ERR_STATE / PDLP_ERR_ARG) before anything is copied.  No counterpart
 * in the reference, which solves one LP per call; it is the collecting side
 * of pdlp_batch_admit_many. */
int pdlp_batch_collect_many(pdlp_batch* b, int32_t n, const int32_t* slots, pdlp_result* results,
                            double* const* x, double* const* y, double* const* d,
                            double* const* history, int32_t memory, int32_t retire);
/* Requests the slot to stop at its next check (status INTERRUPTED). */
int pdlp_batch_cancel(pdlp_batch* b, int32_t slot);
/* The slot's preconditioner, the reference's Scaling (src/sovopt/numerics/
 * scaling.py:60-108, built by scale_problem(method="pdlp"), scaling.py:374-478):
 * row factors r (m), column factors c (n), both powers of two, with the scaled
 * problem A' = diag(r) A diag(c), and the objective scale.  Pointers in
 * `memory`; NULL skips.  Valid once the slot has left its preconditioning
 * passes (it has iterated, or finished); PDLP_ERR_STATE before that. */
int pdlp_batch_scaling(pdlp_batch* b, int32_t slot, double* row_scale, double* col_scale,
                       double* obj_scale, int32_t memory);
/* Device bytes a slot for this problem would take (admission planning). */
int64_t pdlp_slot_bytes(int32_t m, int32_t n, int64_t nnz);
/* Per-kernel timing of the last pdlp_batch_step: total device milliseconds
 * and algorithmic bytes moved by the PDHG iterations. */
int pdlp_batch_last_timing(pdlp_batch* b, double* ms, double* iter_bytes,
                           int64_t* iterations);

/* ---- engine autotuner --------------------------------------------------- *
 * No counterpart in the reference, whose kernels have one fixed launch shape
 * (backend.py:379-384).  The tuner picks, per nnz profile, the lanes that sum
 * each row of the A pass and of the A^T pass and the tile shape (rows and
 * entries per warp tile), by timing short solo runs of an LP with each
 * candidate: lanes 1, 2, 4 for either pass with the default tiles, then tiles
 * of 64 or 32 rows and 512 or 256 entries with the best lanes.  Each run
 * admits the LP into a private one-slot batch on `stream`, runs it past its
 * preconditioning, then times 2 x 64 engine steps (the faster counts), so a
 * tuning costs about a dozen short solves.  Every candidate runs on the same
 * number of blocks, about eight default tiles per warp: the load a warp
 * carries in a full batch (alone on all the blocks it can use, an LP would
 * favour small tiles, which lose in a loaded batch).  Results go to a process-wide
 * cache (guarded by a mutex) keyed by the LP's profile: batches created with
 * pdlp_batch_config.autotune = 1 use it at admission.  Tuning changes only
 * how an LP's rows are split across lanes and warps, so a tuned LP's result
 * equals the untuned one up to the summation order. */
typedef struct pdlp_tune_key {
    int32_t rows_bucket;        /* floor(log2(m + 1))                       */
    int32_t row_len_bucket;     /* floor(2 log2(nnz / m + 1)): half octaves  */
    int32_t col_len_bucket;     /* floor(2 log2(nnz / n + 1))               */
} pdlp_tune_key;

typedef struct pdlp_tuning {
    int32_t lanes_rows, lanes_cols;     /* lanes per row: A pass, A^T pass   */
    int32_t tile_rows, tile_nnz;        /* warp tile: rows and entries       */
    double us_per_iteration;            /* the choice's time per PDHG
                                           iteration of the tuned LP, on the
                                           tuner's fixed block count        */
    double default_us_per_iteration;    /* the same with the fixed rules     */
} pdlp_tuning;

void pdlp_tune_key_of(int32_t m, int32_t n, int64_t nnz, pdlp_tune_key* key);
/* Tunes the engine for this LP (host or device arrays, as for admission) and
 * stores the result under its profile; *out (optional) receives it. */
int pdlp_tune_lp(const pdlp_problem_desc* prob, const pdlp_params* params, void* stream,
                 pdlp_tuning* out);
int pdlp_tune_cache_size(void);
/* Entry i (0 <= i < size) of the cache, in key order. */
int pdlp_tune_cache_get(int32_t i, pdlp_tune_key* key, pdlp_tuning* tuning);
/* Stores an entry (e.g. one saved by an earlier process); the choice is
 * checked: lanes 1, 2, 4, 8, 16 or 32, 1 <= tile_rows <= 64,
 * 1 <= tile_nnz <= 512. */
int pdlp_tune_cache_put(const pdlp_tune_key* key, const pdlp_tuning* tuning);
void pdlp_tune_cache_clear(void);

/* ---- kernel-level Backend (backend.py:317-493) -------------------------- *
 * Device pointers; `stream` as above.  FP64 unless named _f32. */

/* y = A x, A in CSR with int64 pointers (backend.py:373-384).  Asynchronous
 * on `stream`; a fixed summation order, so repeated calls give the same bits.
 * Rows longer than 256 entries are summed by a second launch from a per-
 * (device, stream) list that the library keeps between calls.  It is
 * allocated on the first call with a given stream and grown when a larger m
 * comes; those calls synchronise the stream. */
int pdlp_spmv_f64(int32_t m, const int64_t* rp, const int32_t* ri, const double* rx,
                  const double* x, double* y, void* stream);
int pdlp_spmv_f32(int32_t m, const int64_t* rp, const int32_t* ri, const float* rx,
                  const float* x, float* y, void* stream);
/* The same with an explicit variant of the row-block pass (the plain calls
 * use PDLP_SPMV_STREAMED).  STREAMED: every row of at most 256 entries is
 * streamed, in runs of consecutive rows whose entries fit a warp's 256-entry
 * buffer: independent coalesced loads, products staged in shared memory,
 * each row summed in storage order.  ROW_GROUPS: every row takes the row-group path
 * (L lanes per row from the block's mean row length, strided sums then a
 * xor butterfly).  BANDED: as STREAMED, but a block of 256 rows whose
 * streamed entries' column indices span at most 3072 columns first loads x
 * over that span into shared memory, and gathers from it (banded matrices,
 * e.g. multi-period plans).  All give the same results up to the summation
 * order; STREAMED and BANDED sum each streamed row in storage order. */
#define PDLP_SPMV_AUTO        0
#define PDLP_SPMV_STREAMED    1
#define PDLP_SPMV_ROW_GROUPS  2
#define PDLP_SPMV_BANDED      3
int pdlp_spmv_ex_f64(int32_t variant, int32_t m, const int64_t* rp, const int32_t* ri,
                     const double* rx, const double* x, double* y, void* stream);
int pdlp_spmv_ex_f32(int32_t variant, int32_t m, const int64_t* rp, const int32_t* ri,
                     const float* rx, const float* x, float* y, void* stream);
/* The SpMV autotuner: times each variant on this matrix and these vectors
 * (one warm call, then three interleaved rounds of `reps` calls, 0 = 10, with
 * CUDA events on `stream`, each variant's fastest round counting),
 * writes y = A x, and returns the fastest variant in *best_variant and each
 * variant's milliseconds per call in ms_per_variant[3] (STREAMED, ROW_GROUPS,
 * BANDED; optional).  Synchronises the stream.  The reference has a fixed launch
 * shape (backend.py:379-384); the caller keeps the choice per matrix. */
int pdlp_spmv_tune_f64(int32_t m, const int64_t* rp, const int32_t* ri, const double* rx,
                       const double* x, double* y, void* stream, int32_t reps,
                       int32_t* best_variant, double* ms_per_variant);
int pdlp_spmv_tune_f32(int32_t m, const int64_t* rp, const int32_t* ri, const float* rx,
                       const float* x, float* y, void* stream, int32_t reps,
                       int32_t* best_variant, double* ms_per_variant);
/* Planned SpMV: y = A x on a fixed sparsity pattern, analysed once
 * (backend.py:373-384 on the matrix the PDHG loop multiplies at every
 * iteration).  pdlp_spmv_plan_create copies rp and ri to the host (it
 * synchronises `stream`), checks them (non-decreasing pointers, 0 <= index <
 * n_cols), cuts the rows into tiles of at most 512 rows and 2048 entries, and
 * gives each tile a window of at most 3072 columns holding most of its indices
 * plus a halo of up to 32 further columns (its most used outside the window).
 * The plan keeps its own copy of the pattern on the device (rp and ri may be
 * freed after the call); the values rx are passed to each run and may change.
 * pdlp_spmv_plan_run_* launches one persistent kernel: per SM a copy warp
 * streams tiles (row pointers, indices, values and the x window) into a ring
 * of shared-memory stages with bulk asynchronous copies, a halo warp gathers
 * the halo into the stage, and sixteen consumer warps sum the rows from shared
 * memory; an entry in neither window nor halo gathers x from global memory.
 * Rows of at most 64 entries are summed by one lane in storage order
 * (bit-identical to the reference's CPU kernel); longer rows by a warp,
 * lane-strided then a xor butterfly.  rx and x must be 16-byte aligned (as
 * cudaMalloc and torch allocations are).  When fewer than half the entries
 * fall in a window or halo, a run is the row-block kernel instead
 * (pdlp_spmv_ex_* with PDLP_SPMV_STREAMED on the plan's copy; no alignment
 * rule).  The tile kernel is launched as a programmatic dependent of the
 * kernel before it in `stream`: it may start staging the plan's own arrays
 * while that kernel drains, but reads rx and x and writes y only after it
 * has completed, so stream order holds as for any launch.
 * Asynchronous; repeated runs give the same bits.  A wait inside the
 * kernel that runs out (1 s) records PDLP_ERR_BARRIER_TIMEOUT, which
 * pdlp_spmv_plan_status returns (and clears) after synchronising `stream`. */
typedef struct pdlp_spmv_plan pdlp_spmv_plan;
#define PDLP_SPMV_PLAN_TILES     0
#define PDLP_SPMV_PLAN_STREAMED  1
typedef struct {
  int32_t tiles;             /* tiles of rows */
  int32_t banded_tiles;      /* tiles that stage an x window */
  int32_t huge_rows;         /* rows over 2048 entries (read from global memory) */
  int32_t ctas;              /* CTAs of a run (one per SM at most) */
  int32_t kernel;            /* PDLP_SPMV_PLAN_TILES, or PDLP_SPMV_PLAN_STREAMED when fewer
                                than half the entries are staged: a run is then
                                pdlp_spmv_ex_* with PDLP_SPMV_STREAMED */
  int32_t reserved;
  int64_t entries;           /* nnz */
  int64_t entries_in_band;   /* entries whose x is staged (window or halo) */
  double seconds;            /* host time of pdlp_spmv_plan_create */
} pdlp_spmv_plan_info;
int pdlp_spmv_plan_create(int32_t m, int32_t n_cols, const int64_t* rp, const int32_t* ri,
                          void* stream, pdlp_spmv_plan** out);
int pdlp_spmv_plan_run_f64(pdlp_spmv_plan* plan, const double* rx, const double* x, double* y,
                           void* stream);
int pdlp_spmv_plan_run_f32(pdlp_spmv_plan* plan, const float* rx, const float* x, float* y,
                           void* stream);
int pdlp_spmv_plan_get_info(const pdlp_spmv_plan* plan, pdlp_spmv_plan_info* out);
int pdlp_spmv_plan_status(pdlp_spmv_plan* plan, void* stream);
void pdlp_spmv_plan_destroy(pdlp_spmv_plan* plan);
/* Y = A X, X dense (ncols, k) row-major, batch index fastest (backend.py:386-400) */
int pdlp_spmm_f64(int32_t m, int32_t k, const int64_t* rp, const int32_t* ri,
                  const double* rx, const double* X, double* Y, void* stream);
/* xnew = clamp(x - tau (c + aty), lo, hi) (backend.py:404-415) */
int pdlp_primal_step(int32_t n, double* xnew, const double* x, const double* c,
                     const double* aty, const double* lo, const double* hi,
                     double tau, void* stream);
/* ynew = w - sigma clamp(w / sigma, rl, ru), w = y + sigma ax (backend.py:417-434) */
int pdlp_dual_step(int32_t m, double* ynew, const double* y, const double* ax,
                   const double* rl, const double* ru, double sigma, void* stream);
/* x <- clamp(x - tau (c + aty), lo, hi), dx = xnew - xold (backend.py:441-452) */
int pdlp_pdhg_primal(int32_t n, double* x, double* dx, const double* c,
                     const double* aty, const double* lo, const double* hi,
                     double tau, void* stream);
/* ax += adx; w = y + sigma (ax + adx); y <- prox; dy (backend.py:454-467) */
int pdlp_pdhg_dual(int32_t m, double* y, double* dy, double* ax, const double* adx,
                   const double* rl, const double* ru, double sigma, void* stream);
/* acc += inc; sum += eta v (backend.py:469-479) */
int pdlp_pdhg_accum(int32_t n, double* acc, const double* inc, double* run_sum,
                    const double* v, double eta, void* stream);
/* Reductions to a host double (synchronising, like the reference's float()
 * conversions, backend.py:483-490).  Deterministic: a fixed reduction tree. */
int pdlp_dot(int64_t n, const double* a, const double* b, double* out, void* stream);
int pdlp_nrm2(int64_t n, const double* a, double* out, void* stream);
int pdlp_nrm_inf(int64_t n, const double* a, double* out, void* stream);
/* ---- batched node relaxation (mip/bnr.py:176-301) ----------------------- *
 * K node LPs that share one pdlp-scaled problem (matrix, costs, row bounds)
 * and differ only in column bounds, advanced together by a fixed number of
 * PDHG iterations with a step size per node, then bounded by each node's safe
 * dual bound (mip/safebound.py:194-235).  Node blocks are (rows, K) with the
 * node index fastest, so each sparse product reads A once for all K nodes. */
typedef struct pdlp_bnr pdlp_bnr;
/* BNREngine.__init__ (bnr.py:128-151): the scaled problem (CSR and CSC of A,
 * c, row bounds, obj_offset; col bounds and kind unused) and the objective
 * scale; node buffers for max_batch nodes, grown on demand. */
int pdlp_bnr_create(const pdlp_problem_desc* scaled, double obj_scale, int32_t max_batch,
                    void* stream, pdlp_bnr** out);
int pdlp_bnr_destroy(pdlp_bnr* b);
/* BNREngine.solve_batch: col_lb / col_ub (n, K); warm_x (n, K) and warm_y
 * (m, K) or both NULL (start at 0); iters iterations with step exponents
 * step_growth / step_damp (BNRConfig: 0.3 / 0.6).  Outputs, each optional:
 * bounds[K] in the original objective scale (+inf for an empty box, -inf
 * when the duals certify nothing), x (n, K), y (m, K), infeasible[K] (1 for
 * an empty box).  Pointers in `memory`.  The step sizes persist in the
 * engine between calls, as in the reference. */
int pdlp_bnr_solve_batch(pdlp_bnr* b, int32_t K, const double* col_lb, const double* col_ub,
                         const double* warm_x, const double* warm_y, int32_t iters,
                         double step_growth, double step_damp, double* bounds, double* x,
                         double* y, uint8_t* infeasible, int32_t memory);
/* The engine's current step sizes of the first K nodes (host arrays). */
int pdlp_bnr_step_sizes(pdlp_bnr* b, int32_t K, double* eta, double* omega);

/* a . b to a host double, like pdlp_dot, but without allocating any device
 * memory.  No counterpart in the reference.  It is for callers that must not
 * allocate: a serving loop that has given the free device memory to resident
 * problems (an allocation there could fail with out-of-memory in the middle
 * of a step), or any caller whose device footprint must stay fixed and known
 * before it starts.  The scratch is one fixed 128 KiB array per device, so n
 * is limited to 2^28 = 268435456 elements; a larger n returns PDLP_ERR_ARG
 * (use pdlp_dot then).  The first call on a device (n = 0 is enough) looks up
 * that array's address with the device current: make it before any stream
 * capture.  Every call on a device shares the array and leaves the last
 * call's partial sums in it, so calls whose execution overlaps (other
 * streams, other host threads) race and must be serialised by the caller.
 * The result equals pdlp_dot's up to rounding (a different, but fixed,
 * summation tree). */
int pdlp_dot_noalloc(int64_t n, const double* a, const double* b, double* out, void* stream);

/* ---- crossover to a basis (host) ---------------------------------------
 * Turns a PDLP point into an optimal basic solution, for ranging and warm
 * starts: sovopt's src/sovopt/lp/crossover.py (basis_from_point, crossover).
 * Both calls run on the host cores and take a problem with memory
 * PDLP_MEM_HOST; c is minimised and `sense` is ignored (the caller negates c
 * and y for a maximisation, as crossover.py:206-211 does).  Statuses over
 * [x ; s] (n structurals, then one logical per row, bounded by the row's
 * bounds), with the values of src/sovopt/lp/basis.py:75-79: */
#define PDLP_BASIC     0
#define PDLP_AT_LOWER  1
#define PDLP_AT_UPPER  2
#define PDLP_FREE      3
#define PDLP_FIXED     4
#define PDLP_STATUS_UNBOUNDED 2

typedef struct pdlp_crossover_info {
    int32_t placed;          /* structurals pushed into the basis             */
    int32_t candidates;      /* structurals offered (free, then by score)     */
    int32_t rejected;        /* offered but dependent on those already in     */
    int32_t factorizations;
    int32_t repairs;         /* dependent columns swapped for logicals at a
                                refactorisation (0 by construction)           */
    int32_t reserved;
    double seconds;
} pdlp_crossover_info;

/* basis_from_point (crossover.py:80-187): scores every variable of [x ; s]
 * by its distance to the nearest bound relative to its range (less 1e-9
 * |d_j| with d = c - A'y, or nothing when y is NULL), offers the free
 * structurals and then those scoring above 1e-9 by decreasing score, and
 * pushes each into the basis (starting from the all-logical one) on the
 * largest |B^-1 M_j| entry in a row still holding its logical, skipping it
 * when that entry is at most pivot_tol.  status_out (n + m) gets exactly m
 * PDLP_BASIC entries; the rest rest on their nearest bound (PDLP_FIXED when
 * the bounds are within tol_fixed * max(1, |lb|)).  The reference passes
 * tol_fixed = 1e-12 and pivot_tol = max(SimplexParams.pivot_tol, 1e-7). */
int pdlp_basis_from_point(const pdlp_problem_desc* prob, const double* x, const double* y,
                          double tol_fixed, double pivot_tol, uint8_t* status_out,
                          pdlp_crossover_info* info);

/* SimplexParams (src/sovopt/lp/simplex.py:94-196): the fields this simplex
 * uses, with the same defaults. */
typedef struct pdlp_simplex_params {
    double feas_tol, opt_tol, pivot_tol;     /* 1e-7 each                     */
    int64_t max_iter;                        /* 1,000,000                     */
    double time_limit;                       /* 300 s                         */
    int32_t refactor_freq;                   /* 150 pivots between LUs        */
    int32_t reserved;
} pdlp_simplex_params;

typedef struct pdlp_simplex_info {
    int32_t status;          /* PDLP_STATUS_*                                 */
    int32_t phase;           /* the phase it ended in (1 or 2)                */
    int64_t iterations;      /* pivots plus bound flips                       */
    int64_t phase1_iterations, bound_flips, degenerate_pivots;
    int64_t dual_iterations;   /* pivots of the dual simplex                 */
    int64_t cost_shifts;       /* costs shifted to make a start dual feasible */
    int32_t factorizations, repairs;
    double objective;        /* c'x of the returned point                     */
    double primal_infeasibility, dual_infeasibility;
    int64_t lu_nnz;
    double seconds;
} pdlp_simplex_info;

int pdlp_simplex_default_params(pdlp_simplex_params* params);

/* The revised simplex that finishes a crossover (the role of
 * src/sovopt/lp/simplex.py:1181-1374 in crossover.py:213), on a copy of the
 * LP scaled by powers of two.  From warm_status when it has exactly m
 * PDLP_BASIC entries, else from the all-logical basis: a primal feasible
 * start goes to the primal simplex; any other start is made dual feasible
 * (boxed nonbasics moved to the bound their reduced cost wants, the other
 * costs shifted) and runs the bounded dual simplex to primal feasibility,
 * then, with the true costs, the primal simplex (Dantzig pricing, Harris
 * ratio test with bound flips, Bland's rule after 50 degenerate pivots in a
 * row).  A dual ray is confirmed by a composite primal phase 1 before
 * INFEASIBLE is returned.  It returns OPTIMAL only once fresh factors show
 * the basis primal feasible to feas_tol and dual feasible to opt_tol.  Writes x
 * (n), y (m, B^-T c_B), d (n, c - A'y, 0 on basic columns) and the final
 * basis_status (n + m).  params NULL: defaults. */
int pdlp_simplex_solve(const pdlp_problem_desc* prob, const pdlp_simplex_params* params,
                       const uint8_t* warm_status, double* x, double* y, double* d,
                       uint8_t* basis_status, pdlp_simplex_info* info);

#ifdef __cplusplus
}
#endif

#endif /* PDLP_B200_H */
