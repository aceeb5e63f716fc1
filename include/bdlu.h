/*
 * bdlu.h - C ABI of the B200 numeric engine for BlockDAGLU's hot path.
 *
 * The reference exposes its numeric factor and solve through the C++ class
 * blockdaglu::Solver (blockdaglu/include/blockdaglu/solver.h:43-126) and, for
 * DLL callers, through CreateAlgorithm/DestroyAlgorithm
 * (blockdaglu/src/exports.cpp:16-23).  This header is the plain-C boundary
 * under an equivalent Solver: an opaque handle, plain pointers and sizes,
 * integer status codes mirroring blockdaglu::SolverError, and no exceptions
 * across the boundary.  The C++ class in include/blockdaglu/solver.h wraps it.
 *
 * Memory: the handle owns every device allocation.  Host-pointer arguments are
 * read or written before the call returns.  Functions whose name ends in
 * _device take device pointers and a CUDA stream (cudaStream_t passed as void*;
 * NULL means the legacy default stream) and return once the work is enqueued.
 *
 * Threading: one handle must not be used from two threads at once.  Distinct
 * handles may be used concurrently (solver.h:43-126 gives the same rule).
 */
#ifndef BDLU_H_
#define BDLU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes, one for one with blockdaglu::SolverError (solver.h:19-31). */
enum bdlu_status {
  BDLU_OK = 0,
  BDLU_NOT_PREPARED = 1,
  BDLU_INVALID_DIMENSION = 2,
  BDLU_INVALID_INDEX = 3,
  BDLU_NON_FINITE_VALUE = 4,
  BDLU_INVALID_RHS = 5,
  BDLU_BACKEND_UNAVAILABLE = 6,
  BDLU_ANALYSIS_FAILED = 7,
  BDLU_FACTORIZATION_FAILED = 8,
  BDLU_SOLVE_FAILED = 9,
  BDLU_EXPORT_FAILED = 10
};

/* Route, as selected by analyze (solver.h:72-76 Mode). */
enum bdlu_mode { BDLU_MODE_AUTO = 0, BDLU_MODE_KLU = 1, BDLU_MODE_BLOCK = 2 };

typedef struct bdlu_solver bdlu_solver;

/* Solver::Solver / ~Solver (solver.h:45-46). */
bdlu_solver* bdlu_create(void);
void bdlu_destroy(bdlu_solver* h);

/* Solver::set_matrix(CooMatrix m, int32_t dimension) (solver.h:48-49,
 * solver.cpp:749-800).  Storage only: the triplets are copied and nothing is
 * validated until analyze.  dimension = -1 infers n from the largest index. */
int bdlu_set_coo(bdlu_solver* h, const int32_t* rows, const int32_t* cols, const double* vals,
                 int64_t nnz, int32_t dimension);

/* Solver::analyze (solver.h:50, solver.cpp:802-1182): validation and
 * canonicalisation, DM/BTF, block merge, UBTF split, block DAG and levels,
 * upload of the per-pattern device structure. */
int bdlu_analyze(bdlu_solver* h);

/* Solver::factor (solver.h:51, solver.cpp:1184-1350): numeric factorisation of
 * every diagonal block on the GPU. */
int bdlu_factor(bdlu_solver* h);

/* Value-only refactor (no counterpart API in the reference; there a value
 * change is set_matrix + analyze + factor, solver.cpp:749-1350).  `vals` holds
 * nnz values in canonical order: sorted by (row, col) with duplicates summed
 * and exact zeros dropped, i.e. the order bdlu_canonical_pattern returns.  The
 * pattern, permutations, blocks and pivot-free structure are reused. */
int bdlu_refactor_values(bdlu_solver* h, const double* vals, int64_t nnz);
int bdlu_refactor_values_device(bdlu_solver* h, const double* d_vals, int64_t nnz, void* stream);

/* Solver::solve_in_place (solver.h:52, solver.cpp:1352-1539), generalised to
 * nrhs right-hand sides stored column-major with leading dimension ldb >= n.
 * B is overwritten by X. */
int bdlu_solve(bdlu_solver* h, double* B, int32_t ldb, int32_t nrhs);
int bdlu_solve_device(bdlu_solver* h, double* d_B, int32_t ldb, int32_t nrhs, void* stream);

/* Refactor + solve in one call (the serving unit of work); values in
 * canonical order, B column-major, overwritten by X. */
int bdlu_refactor_solve(bdlu_solver* h, const double* vals, int64_t nnz, double* B, int32_t ldb,
                        int32_t nrhs);

/* Solver::last_error / last_error_message (solver.h:54-55).  Copies the
 * message (NUL-terminated, truncated to len) and returns the status code. */
int bdlu_last_error(const bdlu_solver* h, char* buf, int64_t len);

/* Solver::n / selected_mode (solver.h:64-65): "KLU" or "BLOCK". */
int32_t bdlu_n(const bdlu_solver* h);
const char* bdlu_selected_mode(const bdlu_solver* h);

/* Canonical pattern after analyze: nnz, and rows/cols if non-NULL. */
int64_t bdlu_canonical_pattern(const bdlu_solver* h, int32_t* rows, int32_t* cols);

/* Lazy exports, Solver::getP/getQ/getL/getU/get_rearranged_matrix
 * (solver.h:58-62, solver.cpp:1665-1725).  COO triplets; call with cap = 0 to
 * get the count, then again with buffers of that size.  Returns the entry
 * count, or -(status) on failure.  The identity dense(rearranged) =
 * dense(L) * dense(U) holds (apps/tests/main.cpp:170-195). */
int64_t bdlu_export_p(bdlu_solver* h, int32_t* rows, int32_t* cols, double* vals, int64_t cap);
int64_t bdlu_export_q(bdlu_solver* h, int32_t* rows, int32_t* cols, double* vals, int64_t cap);
int64_t bdlu_export_l(bdlu_solver* h, int32_t* rows, int32_t* cols, double* vals, int64_t cap);
int64_t bdlu_export_u(bdlu_solver* h, int32_t* rows, int32_t* cols, double* vals, int64_t cap);
int64_t bdlu_export_rearranged(bdlu_solver* h, int32_t* rows, int32_t* cols, double* vals,
                               int64_t cap);

/* Per-result statistics (the reference prints these as USERALGO_PROFILE lines,
 * solver.cpp:1510-1517). */
typedef struct bdlu_stats {
  int32_t n;
  int32_t nblocks;
  int32_t nblocks_raw;
  int32_t max_block;
  int32_t max_level;
  int32_t refine_iters;      /* refinement steps taken by the last solve */
  int32_t nunits;            /* raw BTF blocks: the device's factor/solve units */
  int32_t unit_levels;       /* depth of the unit DAG: sequential steps of the solve */
  int32_t max_unit;          /* largest raw BTF block */
  int32_t factor_launches;   /* kernels launched by the last factor */
  int32_t solve_launches;    /* kernels launched by the last solve */
  int64_t nnz;
  int64_t nnz_offdiag;
  int64_t dense_entries;     /* sum of m^2 over dense-factored blocks */
  double factor_flops;       /* algorithmic flops of one factor */
  double residual_inf;       /* |Ax-b|_inf / (|A|_inf |x|_inf + |b|_inf), last solve, worst rhs */
  double last_factor_ms;     /* device time of the last factor */
  double last_solve_ms;      /* device time of the last solve */
  int32_t precision;         /* trailing-update arithmetic of the last factor: 0 FP64, 1 TF32, 2 3xTF32 */
} bdlu_stats;
int bdlu_get_stats(const bdlu_solver* h, bdlu_stats* out);

/* Device time in ms of the phases of the last factor and solve, from CUDA
 * events on the stream they ran on: [0] value gather, [1] shared-memory LU of
 * small blocks, [2] blocked LU of large blocks, [3] first solve sweep
 * (permute, level-scheduled block solve, unpermute), [4] refinement steps and
 * residual.  Writes min(cap, 5) values; returns 5.  Synchronises. */
int bdlu_phase_times(bdlu_solver* h, double* ms, int32_t cap);

/* Engine options.
 *   "refine_iters": number of FP64 iterative-refinement steps (r = b - Ax,
 *     solve, x += d) after each solve; default is the reference's REFINE_ITERS
 *     environment value, else 0 (solver.cpp:1449-1465).
 *   "refactor_pivoting": 0 (default) lets a value-only refactor keep the pivot
 *     order of the last full factorisation for blocks factored across CTAs
 *     (KLU's klu_refactor reuses the pivot order the same way); a zero pivot,
 *     or a host-buffer solve whose residual exceeds 1e-12, triggers a
 *     factorisation with partial pivoting.  1 pivots on every refactor.
 *   "sparse_lu": sparse LU of diagonal blocks (the reference's opt-in
 *     Gilbert-Peierls route, gp_lu.cpp:84-306), from the next analyze.  0 off
 *     (default unless USERALGO_SPARSE_LU_KERNEL=gp), 1 the reference's route:
 *     every block of USERALGO_DENSE_BLOCK_MAX (64) < m <= USERALGO_GP_MAX_N
 *     (4096) rows is factored without pivoting over its fill pattern and kept
 *     if the reference's gate would accept it (no row swap under the
 *     diagonal preference USERALGO_GP_DIAG_TOL, no pivot below
 *     USERALGO_GP_PIVOT_TOL or USERALGO_GP_MIN_ABS_DIAG); accepted factors
 *     are bit-identical to the reference's.  A rejected block is factored
 *     dense, for this factor and later ones of the handle.  2 the same for
 *     blocks whose fill is at most "sparse_fill_max" (default 0.01) of m^2.
 *     Environment settings that relax the gate, scale rows or drop entries
 *     turn the route off.  "sparse_max_n" overrides USERALGO_GP_MAX_N.  A
 *     device-pointer refactor does not wait for the factor's status: a block
 *     that fails the test there is found, like a zero pivot, by the next
 *     host-buffer solve, which factors again with the block dense.
 *   "analysis_only": 1 makes analyze stop after the host analysis (no device
 *     upload); factor then reports BDLU_BACKEND_UNAVAILABLE.  For structure
 *     inspection on machines without a GPU.
 *   "precision": 0 (default) FP64 throughout.  1 selects the mixed route: the
 *     trailing updates of blocks above the shared-memory size run on tensor
 *     cores with TF32 operands and FP32 accumulation (panels, pivoting and
 *     storage stay FP64), and host-buffer solves refine in FP64 until the
 *     relative residual is <= 1e-12.  A level whose refinement stagnates is
 *     replaced for this and later factorisations: TF32, then 3xTF32 (about
 *     FP32 accuracy), then FP64.  stats.precision and stats.refine_iters
 *     report the level and the refinement steps.  Device-pointer solves run
 *     "refine_iters" steps only.  2 is the mixed route starting at 3xTF32.
 *     The tensor-core updates are tcgen05.mma (kind::tf32) with the
 *     accumulator in tensor memory.
 *   "refactor_schedule": order of the FP64 value-only refactor of blocks
 *     above the shared-memory size.  0: a chain of per-step launches (panel,
 *     then trailing update, one step of lookahead).  1: one persistent kernel
 *     works through the block's tile task graph (diagonal LU, strip solves,
 *     trailing updates; each task starts when its input tiles are ready).
 *     Both give bit-identical factors.  Unset, the autotuner picks per
 *     pattern (see bdlu_tuner_report).
 *   "lu_small_threads": launch width of the small-unit LU: 0 (default) the
 *     autotuner's, 1 one thread per row with the rows in registers (units up
 *     to 96 rows), 32 one warp per unit (units up to 64 rows), 64 / 128 / 256
 *     threads per unit (units up to that many rows).  Same factors.
 *   "programmatic_launch": 1 (default) launches each solve level from the
 *     second on as a programmatic dependent of the previous one (its factor
 *     staging and launch overlap the previous level); 0 keeps plain stream
 *     order, for processes that run many solves on many streams at once
 *     (the serving loop does).  Same results.
 *   "small_launch": -1 (default) the autotuner's, 0 one launch per size
 *     bucket, 1 one persistent launch over a task queue.  Same factors.
 *   "wait_limit": polls a bounded wait between tiles (large-unit solve
 *     sweeps, tile task graph refactor) makes before it gives up with an
 *     error status; 0 (default) about half a second.  Short limits make the
 *     waits run out on purpose (tests of that error path).
 * Returns BDLU_OK, or BDLU_INVALID_DIMENSION for an unknown key or value. */
int bdlu_set_option(bdlu_solver* h, const char* key, double value);

/* ---- Batches of independent systems ---------------------------------------
 * The reference solves one system per Solver; its callers loop over systems
 * (one Solver each, apps/benchmark/main.cpp:271-297).  A batch replaces that
 * loop: the systems are analysed together as one block-diagonal system (the
 * BTF blocks of each system, DAG levels aligned), so every block of every
 * system is factored by the same launches and every level of every system is
 * solved by one launch.  Each system keeps the reference's per-system
 * semantics: its own validation (errors name the system), canonicalisation
 * (duplicates summed, zeros dropped) and block decomposition; the block route
 * is always used.
 *   bdlu_batch_add: storage only; n > 0 is required; returns the system's
 *     index, or -(status).
 *   bdlu_batch_analyze: validates every system and analyses the batch.
 *   Right-hand sides and solutions: rows row_offset(k) .. row_offset(k+1)-1 of
 *     each column of B belong to system k (ldb >= row_offset(count)).
 *   Value-only refactor: the systems' values in their canonical order, back
 *     to back; system k's start at nnz_offset(k).
 *   row_offset / nnz_offset take k in 0..count and return -1 before analyze.
 * Stats, phase times and errors are those of the whole batch; the residual in
 * the stats is taken over the block-diagonal system. */
typedef struct bdlu_batch bdlu_batch;
bdlu_batch* bdlu_batch_create(void);
void bdlu_batch_destroy(bdlu_batch* b);
int32_t bdlu_batch_add(bdlu_batch* b, const int32_t* rows, const int32_t* cols, const double* vals, int64_t nnz,
                       int32_t n);
int bdlu_batch_analyze(bdlu_batch* b);
int bdlu_batch_factor(bdlu_batch* b);
int bdlu_batch_refactor_values(bdlu_batch* b, const double* vals, int64_t nnz);
int bdlu_batch_refactor_values_device(bdlu_batch* b, const double* d_vals, int64_t nnz, void* stream);
int bdlu_batch_solve(bdlu_batch* b, double* B, int32_t ldb, int32_t nrhs);
int bdlu_batch_solve_device(bdlu_batch* b, double* d_B, int32_t ldb, int32_t nrhs, void* stream);
int32_t bdlu_batch_count(const bdlu_batch* b);
int64_t bdlu_batch_row_offset(const bdlu_batch* b, int32_t k);
int64_t bdlu_batch_nnz_offset(const bdlu_batch* b, int32_t k);
int bdlu_batch_last_error(const bdlu_batch* b, char* buf, int64_t len);
int bdlu_batch_get_stats(const bdlu_batch* b, bdlu_stats* out);
int bdlu_batch_phase_times(bdlu_batch* b, double* ms, int32_t cap);

/* ---- Serving: refactor + solve requests over resident patterns -------------
 * The reference serves one request at a time per Solver.  A server keeps many
 * patterns (each analysed once on the host when added; plan, factors and work
 * space on the device while resident) and runs value-only refactor + solve
 * requests with continuous batching: `slots` workers, each with its own CUDA
 * stream, take the oldest queued request whose pattern is not being served,
 * so requests for different patterns overlap on the device and requests for
 * one pattern run in arrival order.  A pattern is uploaded when a request for
 * it is admitted; if the device-memory budget would be exceeded, idle
 * resident patterns are released, least recently used first, and a request
 * waits while busy patterns hold the memory.  A pattern that cannot fit even
 * alone fails its requests with BDLU_BACKEND_UNAVAILABLE.  Each request runs
 * exactly what bdlu_refactor_solve runs (same checks, pivot-order reuse and
 * fallback, residual), so its result does not depend on what else is served.
 *   add_pattern: COO + n (>= 0, or -1 to infer); host analysis; returns the
 *     pattern id or -(status).  Values per request: pattern_nnz(id), in the
 *     canonical order.
 *   submit: vals (pattern_nnz values) and B (ldb >= n, nrhs columns) are
 *     read and B overwritten with X by a worker; both must stay valid until
 *     bdlu_server_wait returns for the request.  Returns a request id or
 *     -(status).
 *   wait: blocks until the request is done; returns its status and, if the
 *     pointers are not NULL, its relative residual and latency (submit to
 *     result in B, ms).
 *   get_stats: latency percentiles and throughput over completed requests
 *     since creation or the last reset_stats.
 *   destroy: finishes queued requests first. */
typedef struct bdlu_server bdlu_server;
typedef struct bdlu_server_stats {
  int64_t completed;
  int64_t failed;
  double p50_ms;
  double p99_ms;
  double mean_ms;
  double max_ms;
  double throughput;        /* completed requests per second, first submit to last completion */
  int64_t resident_bytes;   /* device bytes of resident patterns (estimates for ones being uploaded) */
  int64_t evictions;        /* patterns released to admit others */
  int32_t peak_concurrency; /* most requests running at once */
  int64_t kernel_launches;  /* engine kernels launched by the completed requests (graph nodes counted) */
  double factor_flops;      /* dense-block LU flops of the completed requests (one factor each) */
  double mean_stage_ms;     /* per request, worker wall time: device upload, input staging and checks */
  double mean_factor_ms;    /*   value-only refactor, up to its status */
  double mean_solve_ms;     /*   solve, residual, result copy-out */
} bdlu_server_stats;
bdlu_server* bdlu_server_create(int64_t memory_budget_bytes, int32_t slots);
void bdlu_server_destroy(bdlu_server* s);
int32_t bdlu_server_add_pattern(bdlu_server* s, const int32_t* rows, const int32_t* cols, const double* vals,
                                int64_t nnz, int32_t n);
int64_t bdlu_server_pattern_nnz(bdlu_server* s, int32_t pattern);
/* Device bytes the pattern takes: measured once it has been resident, an
 * estimate from its plan before. */
int64_t bdlu_server_pattern_bytes(bdlu_server* s, int32_t pattern);
int64_t bdlu_server_submit(bdlu_server* s, int32_t pattern, const double* vals, int64_t nnz, double* B, int32_t ldb,
                           int32_t nrhs);
/* Device-resident request: d_vals and d_B are device pointers (the current
 * device's memory); the values and right-hand sides never cross to the host
 * (no host finiteness check), X overwrites d_B. */
int64_t bdlu_server_submit_device(bdlu_server* s, int32_t pattern, const double* d_vals, int64_t nnz, double* d_B,
                                  int32_t ldb, int32_t nrhs);
int bdlu_server_wait(bdlu_server* s, int64_t request, double* residual, double* latency_ms);
int bdlu_server_drain(bdlu_server* s);
int bdlu_server_get_stats(bdlu_server* s, bdlu_server_stats* out);
int bdlu_server_reset_stats(bdlu_server* s);
int bdlu_server_last_error(const bdlu_server* s, char* buf, int64_t len);
/* Server-wide option, applied to every pattern (present and added later)
 * with bdlu_set_option's meaning: "precision" (0 FP64, 1 mixed with FP64
 * refinement, 2 mixed starting at 3xTF32).  Only while no request is queued
 * or running (else BDLU_NOT_PREPARED). */
int bdlu_server_set_option(bdlu_server* s, const char* key, double value);

/* ---- Dense batch solve without allocation -----------------------------------
 * No counterpart in the reference.  For callers that must not allocate
 * device memory where they solve (an allocator or memory budget closed after
 * start-up, real-time loops that cannot absorb cudaMalloc's latency and
 * implicit synchronisation, code called back inside another framework's step):
 * solves A_i X_i = B_i for `batch` dense m x m matrices with the engine's
 * dense-block partial-pivoting LU, using only the caller's buffers and a
 * static device scratch built into the library (about 8.5 MiB, held on every
 * GPU that loads the library until exit).  No cudaMalloc, cudaFree or other
 * allocating call is made.
 *   d_A: batch matrices, each m*m column-major, contiguous (not modified).
 *   d_B, d_X: batch blocks of m x nrhs, column-major (ld m), contiguous; X may
 *   be the same buffer as B.
 * Limits: m <= 128, batch*m*m <= 1048576, batch*m <= 65536; larger sizes
 * return BDLU_INVALID_DIMENSION with a message.  A singular matrix returns
 * BDLU_FACTORIZATION_FAILED (a zero or NaN pivot); the X block of every
 * matrix that failed is left unwritten (with X the same buffer as B it still
 * holds B) and the other matrices are solved.  Uses the calling
 * thread's current device; the call waits for `stream` before returning
 * (it reads the per-matrix status back), so it can never be called while a
 * stream capture is active on that stream or in relaxed-capture mode on
 * the thread.  Every call on a
 * device shares the one scratch, so calls whose work overlaps on the GPU (other
 * streams, other host threads) race and must be serialised by the caller.
 * msg (may be NULL) receives an error message of at most msg_len bytes. */
int bdlu_dense_batch_solve_noalloc(const double* d_A, int32_t m, int32_t batch, const double* d_B,
                                   double* d_X, int32_t nrhs, void* stream, char* msg, int64_t msg_len);

/* ---- Host analysis, exposed for parity testing ----------------------------
 * Same calling convention as SuiteSparse btf_order as bound by the reference
 * (blockdaglu/src/btf_dynamic.h:19-28, called at ubtf_block_solver.cpp:661-670):
 * returns nblocks; Q holds BTF_FLIP(-j-2) marks for unmatched columns. */
int32_t bdlu_btf_order(int32_t n, const int32_t* Ap, const int32_t* Ai, int32_t* P, int32_t* Q,
                       int32_t* R, int32_t* nmatch);

/* merge_block_boundaries (ubtf_block_solver.cpp:393-476); returns new count
 * of boundaries (nblocks'+1) written to Rout (capacity nR). */
int32_t bdlu_merge_block_boundaries(const int32_t* R, int32_t nR, int32_t n, int32_t merge_max,
                                    int32_t* Rout);

/* Analysis products after analyze, for parity checks: copies whichever
 * pointers are non-NULL.  Sizes: P,Q: n; R: nblocks+1; off_ptr: n+1;
 * off_col/off_src: nnz_offdiag; level: nblocks. */
int bdlu_get_decomposition(const bdlu_solver* h, int32_t* P, int32_t* Q, int32_t* R,
                           int32_t* off_ptr, int32_t* off_col, int32_t* off_src, int32_t* level);

/* Dense factor of block b after factor (for parity with the reference's dense
 * micro-kernel, ubtf_block_solver.cpp:1450-1498): m*m values row-major and m
 * LAPACK-style pivots.  Returns m, or -(status). */
int32_t bdlu_get_block_lu(bdlu_solver* h, int32_t b, double* lu_rowmajor, int32_t* piv);

/* Factor route of every unit (raw BTF block, the device's factor and solve
 * unit) after analyze: start[u] its first permuted row, route[u] 0 scalar,
 * 1 dense LU in shared memory, 2 dense blocked LU, 3 sparse LU;
 * reason[u] -1 when the sparse-LU route did not try the unit, 0 when it
 * factors it, 1-4 when a factor's pivot test rejected it (the reference's
 * gp_gate_eval reasons, ubtf_block_solver.cpp:197-235: 1 zero pivot, 2 a row
 * swap, 3 a tiny pivot, 4 smallest pivot below USERALGO_GP_MIN_ABS_DIAG) and
 * it was factored dense since, 5 when its pattern kept it dense (no
 * structural diagonal after fill, or fill above "sparse_fill_max");
 * lu_nnz[u] the entries its factor stores (m*m for a dense unit, those of
 * L + U over the fill pattern for a sparse one, 1 for a scalar).  Writes
 * min(cap, nunits) entries of each non-NULL array; returns nunits, or
 * -(status).  The reference's counterpart is its per-block diagnostics
 * (BlockFactor::gp_tried / gp_reject_reason, ubtf_block_solver.h:74-84). */
int32_t bdlu_get_unit_routes(const bdlu_solver* h, int32_t* start, int32_t* route, int32_t* reason, int64_t* lu_nnz,
                             int32_t cap);

/* Pattern and value signatures of the canonical matrix after analyze
 * (compute_matrix_sig, compute_matrix_sig2, compute_matrix_value_sig,
 * blockdaglu/src/solver.cpp:96-136): sigs[0..2].  The serving loop keys its
 * resident patterns by them. */
int bdlu_matrix_signatures(const bdlu_solver* h, uint64_t* sigs);

/* ---- Autotuner --------------------------------------------------------------
 * No counterpart in the reference (it tunes by environment knobs,
 * blockdaglu/src/ubtf_block_solver.cpp:35-568).  The engine times its
 * launch-shape and schedule candidates on the GPU it runs on and keeps the
 * faster (every candidate computes bit-identical results): the width of the
 * shared-memory LU per size bucket (one warp per unit, or 64 / 128 / 256
 * threads per unit), per pattern signature the small units as per-bucket
 * launches or as one persistent launch over a task queue, and per pattern
 * signature the value-only refactor schedule of large units (step chain or
 * tile task graph,
 * decided over the pattern's first six refactors that wait for their
 * status: the faster of two steady trials each, after one capture trial
 * each; the tile task graph replaces the chain only if it is more than 2 %
 * faster).  Choices persist in $BDLU_TUNE_CACHE, else
 * $HOME/.cache/bdlu/tune-<gpu>.json; BDLU_AUTOTUNE=0 disables tuning.
 * bdlu_tuner_report writes the choices as JSON (NUL-terminated, at most len
 * bytes) and returns the bytes needed including the NUL. */
int64_t bdlu_tuner_report(char* buf, int64_t len);

/* ---- Seeded synthetic systems --------------------------------------------- */
enum bdlu_synth_family { BDLU_SYNTH_BLOCK = 0, BDLU_SYNTH_CIRCUIT = 1, BDLU_SYNTH_PRECISION = 3 };
typedef struct bdlu_synth bdlu_synth;
/* family BLOCK: n rows, param = number of blocks (0: n/50).
 * family CIRCUIT: n rows, param = number of Pareto blocks (0: 1000*n/200000).
 * family PRECISION: n = number of large blocks, param = log10(kappa). */
bdlu_synth* bdlu_synth_create(int32_t family, uint64_t seed, int32_t n, int32_t param, int32_t nrhs);
void bdlu_synth_destroy(bdlu_synth* s);
int32_t bdlu_synth_n(const bdlu_synth* s);
int64_t bdlu_synth_nnz(const bdlu_synth* s);
int32_t bdlu_synth_nrhs(const bdlu_synth* s);
int32_t bdlu_synth_nblocks(const bdlu_synth* s);
void bdlu_synth_copy(const bdlu_synth* s, int32_t* rows, int32_t* cols, double* vals, double* x_true,
                     double* b);
void bdlu_synth_block_sizes(const bdlu_synth* s, int32_t* sizes);
void bdlu_synth_perturb(const bdlu_synth* s, uint64_t seed, double* vals_out);

#ifdef __cplusplus
}
#endif

#endif /* BDLU_H_ */
