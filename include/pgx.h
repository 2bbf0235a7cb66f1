/*
 * pgx.h — C ABI of the B200-native GeMSLR-FGMRES solve phase.
 *
 * The library takes over the SOLVE phase of the reference ParGeMSLR
 * (Hitenze/pargemslr): FlexGmresClass::Solve driven by the GeMSLR multilevel
 * preconditioner (GemslrClass::Solve / SolveLevel / SolveB /
 * SolveApplyLowRankLevel and the level-0 Schur-complement inner FGMRES).
 * The reference's SETUP phase (partitioning, ILUT, low-rank bases) produces
 * the structures that the pgx_gemslr_* calls below import; from then on every
 * solve runs on one GPU with hand-written sm_100a kernels.
 *
 * Conventions
 *   - Every call returns an int status: 0 on success, otherwise one of the
 *     PGX_ERROR_* codes.  The values 100-107 are the reference's own error
 *     codes (ParGeMSLR INC/pargemslr.hpp:9-21); 200+ are GPU-side codes.
 *     pgx_last_error() gives a message for the calling thread's last failure.
 *   - Matrices are CSR with 32-bit row pointers and column indices
 *     (the reference's CsrMatrixClass layout, SRC/matrices/csr_matrix.hpp:27)
 *     and FP64 values.  Dense matrices are column-major with leading
 *     dimension = rows (DenseMatrixClass, SRC/matrices/dense_matrix.cpp:114).
 *   - Import calls COPY their inputs; the handle owns its device copies,
 *     like the hypre plugin's matrix import
 *     (TESTS/hypre/pargemslr_hypre_interface.cpp:119-129).
 *   - Solve calls BORROW x and b (host or device pointers, see `location`),
 *     like hypre_PargemslrParallelGEMSLRDSolve (…interface.cpp:344-369).
 *   - A handle is used by one host thread at a time; distinct handles may be
 *     used concurrently (each owns its own CUDA stream).
 */
#ifndef PGX_H
#define PGX_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PGX_SUCCESS                0
#define PGX_ERROR_INVALID_OPTION   100 /* PARGEMSLR_ERROR_INVALED_OPTION */
#define PGX_ERROR_INVALID_PARAM    101 /* PARGEMSLR_ERROR_INVALED_PARAM */
#define PGX_ERROR_IO               102 /* PARGEMSLR_ERROR_IO_ERROR */
#define PGX_ERROR_ILU_EMPTY_ROW    103 /* PARGEMSLR_ERROR_ILU_EMPTY_ROW */
#define PGX_ERROR_DOUBLE_INIT_FREE 104 /* PARGEMSLR_ERROR_DOUBLE_INIT_FREE */
#define PGX_ERROR_FUNCTION_CALL    106 /* PARGEMSLR_ERROR_FUNCTION_CALL_ERR */
#define PGX_ERROR_MEMORY_LOCATION  107 /* PARGEMSLR_ERROR_MEMORY_LOCATION */
#define PGX_ERROR_CUDA             200 /* a CUDA runtime call failed */
#define PGX_ERROR_OOM              201 /* device memory could not be reserved */
#define PGX_ERROR_TIMEOUT          202 /* a bounded device-side wait expired */
#define PGX_ERROR_NOT_FINITE       203 /* NaN/Inf met in the right-hand side or iterate */
#define PGX_ERROR_NO_DEVICE        204 /* no usable CUDA device */

/* ---- precision of the preconditioner apply -------------------------------
 * PGX_PRECISION_FP64: everything in FP64 (the reference's arithmetic).
 * PGX_PRECISION_MIXED: factors, coupling blocks, low-rank bases and the
 *   whole preconditioner apply (including the level-0 inner FGMRES) stored
 *   and accumulated in FP32; the outer FGMRES (residual SpMV, Arnoldi
 *   orthogonalisation, Givens rotations, least squares, true residual)
 *   stays FP64. */
#define PGX_PRECISION_FP64  0
#define PGX_PRECISION_MIXED 1
/* Complex systems (the reference's complexd instantiation: FlexGmresClass,
 * GemslrClass and ParallelGemslrClass over ComplexValueClass<double>,
 * SRC/utils/complex.hpp; TESTS/parallel/driver_laplacian_gemslrz_par.cpp).
 * Every value array of such a handle (pgx_csr values, dinv, W, WH, x, b,
 * X, B) holds n values as 2n doubles {re, im} interleaved, the layout of
 * ComplexValueClass and of C99 double complex; strides (ldx, ldb) count
 * values.  PGX_PRECISION_COMPLEX_FP64 keeps everything in complex128;
 * PGX_PRECISION_COMPLEX_MIXED stores and applies the preconditioner in
 * complex64 with the outer FGMRES in complex128.  A complex handle is
 * imported through pgx_gemslr_set_*; pgx_gemslr_setup is real only. */
#define PGX_PRECISION_COMPLEX_FP64  2
#define PGX_PRECISION_COMPLEX_MIXED 3

/* ---- memory location of borrowed vectors (reference kMemoryHost/Device) */
#define PGX_LOCATION_HOST   0
#define PGX_LOCATION_DEVICE 1

typedef struct pgx_gemslr_s *pgx_handle;

/* A CSR matrix view: rows x cols, nnz entries.  rowptr has rows+1 entries
 * (rowptr[0] == 0); colidx/values have nnz entries.  An absent matrix is
 * {0, 0, 0, NULL, NULL, NULL}. */
typedef struct {
   int32_t rows;
   int32_t cols;
   int64_t nnz;
   const int32_t *rowptr;
   const int32_t *colidx;
   const double *values;
} pgx_csr;

/* One level l of the GeMSLR hierarchy after setup, in the permuted ordering
 * (rows lev_ptr[l] .. lev_ptr[l+1]-1 of P A P^T form the block-diagonal B_l).
 *   ncomp, dom_ptr: subdomains of the level, dom_ptr[0..ncomp] relative to
 *       the level start (GemslrClass::_dom_ptr_v2, gemslr.hpp:1630).
 *   L, U, dinv: the level's ILU factors with all subdomains concatenated
 *       block-diagonally, column indices relative to the level start.
 *       L strictly lower (unit diagonal implied), U strictly upper, dinv the
 *       INVERSE diagonal (IluClass::_L/_U/_D, ilu.cpp:3677-3790).
 *   B:  the unfactored block-diagonal B_l (GemslrLevelClass::_B_mat_v), used
 *       by the Schur-complement operator of the level-0 inner solve.
 *   E, F: coupling blocks, E is m_l x n_l, F is n_l x m_l with
 *       m_l = n - lev_ptr[l+1] (GemslrLevelClass::_E_mat/_F_mat).  Absent on
 *       the last level.
 *   rank, W, WH: low-rank correction, W and WH are m_l x rank column-major,
 *       WH = W ((I - H)^-1 - I) (GemslrLevelClass::_Wk/_WHk, applied by
 *       SolveApplyLowRankLevel, gemslr.cpp:3681-3722).  rank 0: none. */
typedef struct {
   int32_t ncomp;
   const int32_t *dom_ptr;
   pgx_csr L;
   pgx_csr U;
   const double *dinv;
   pgx_csr B;
   pgx_csr E;
   pgx_csr F;
   int32_t rank;
   const double *W;
   const double *WH;
} pgx_level;

/* Per-solve outcome. */
typedef struct {
   int32_t status;        /* PGX_SUCCESS or an error code */
   int32_t iters;         /* FlexGmresClass::GetNumberIterations */
   double rel_res;        /* FlexGmresClass::GetFinalRelativeResidual: the
                             Givens estimate |rs|/||b|| (fgmres.hpp:542) */
   double true_rel_res;   /* ||b - A x||_2 / ||b||_2 computed in FP64 on the GPU */
   double solve_ms;       /* device time of the solve (CUDA events) */
   int32_t launches;      /* kernels this library launched for the solve */
} pgx_result;

/* ---- library ----------------------------------------------------------- */

/* Select the CUDA device for handles created afterwards by this thread
 * (replaces the device part of PargemslrInit, SRC/utils/parallel.cpp:304). */
int pgx_init(int device);
/* Release library-wide state (PargemslrFinalize, parallel.cpp:554). */
int pgx_finalize(void);
/* Message describing the calling thread's most recent error. */
const char *pgx_last_error(void);
/* Library version as major*10000 + minor*100 + patch (0.2.0 = 200 adds the
 * parameter and Matrix Market vector readers, pgx_gemslr_nnz and the hypre
 * interface of pgx_hypre.h). */
int pgx_version(void);

/* ---- GeMSLR solve handle (replaces GemslrClass + FlexGmresClass solve) ---
 *
 * Import sequence, mirroring what GemslrClass::Setup leaves behind
 * (gemslr.cpp:1602-1711):
 *   pgx_gemslr_create      n, precision
 *   pgx_gemslr_set_matrix  A (the unpermuted system matrix, FlexGmres's A)
 *   pgx_gemslr_set_perm    pperm (and qperm for unsymmetric reorderings)
 *   pgx_gemslr_set_levels  nlev, lev_ptr[nlev+1]
 *   pgx_gemslr_set_level   once per level
 *   pgx_gemslr_set_inner   the level-0 Schur FGMRES settings
 *   pgx_gemslr_commit      build schedules, upload, allocate work space
 */
int pgx_gemslr_create(pgx_handle *handle, int32_t n, int32_t precision);
int pgx_gemslr_set_matrix(pgx_handle handle, const pgx_csr *A);
int pgx_gemslr_set_perm(pgx_handle handle, const int32_t *pperm, const int32_t *qperm);
int pgx_gemslr_set_levels(pgx_handle handle, int32_t nlev, const int32_t *lev_ptr);
int pgx_gemslr_set_level(pgx_handle handle, int32_t level, const pgx_level *desc);
int pgx_gemslr_set_inner(pgx_handle handle, int32_t enable, int32_t maxits, double tol);
/* The solve option (PARGEMSLR_IO_ADVANCED_GLOBAL_SOLVE, params[141];
 * GemslrSolveOptionEnum, gemslr.hpp:120-128), set before commit:
 *   0 the additive LU solve (default);
 *   1 the U solve: every level of the solve phase skips its block-L part and
 *     starts from z = rhs (GemslrClass::SolveLevel, gemslr.cpp:3527-3532);
 *   2 the multiplicative solve of ParallelGemslrClass (SolveLevelGemslrMul,
 *     parallel_gemslr.cpp:5816-6050) with the level-0 inner FGMRES on the RAP
 *     operator (RAPMatVec, :7194); it needs every level's B blocks
 *     (pgx_level.B), the reference's setup run with the same option, and runs
 *     one right-hand side per slot (no multi-lane slots, no systems solve).
 * GemslrClass itself solves options 2 and 3 as 0; option 3 (the modified-ILU
 * multiplicative solve) is refused with PGX_ERROR_INVALID_OPTION.
 * pgx_gemslr_setup reads options 0 and 1 from its params. */
int pgx_gemslr_set_solve_option(pgx_handle handle, int32_t option);
int pgx_gemslr_commit(pgx_handle handle);
int pgx_gemslr_destroy(pgx_handle handle);

/* Build a committed handle from A alone: the host-side GeMSLR setup of this
 * library (nested-dissection levels, RCM inside subdomains, dual-threshold
 * ILUT per subdomain, coupling blocks) followed by the low-rank corrections
 * computed on the GPU by subspace iteration (the reference's option
 * kGemslrLowrankSubspaceIteration, gemslr.cpp:2592-2656).  params is the
 * reference's double[180] array; the slots read are NLEV_GLOBAL (20),
 * ILU_DROPTOL_B/C_GLOBAL (40, 44), ILU_ROWNNZ_B/C_GLOBAL (48, 50),
 * ILU_PERM_OPTION_GLOBAL (58: 0 = none, PGX_REORDER_MULTICOLOR, otherwise RCM), LR_RANK1/2_GLOBAL
 * (74, 75), LR_RANK_FACTOR1/2_GLOBAL (78, 79), LR_MAXITS1_GLOBAL (90) and
 * SCHUR_ENABLE / SCHUR_ITER_TOL / SCHUR_MAXITS (130-132).  Replaces
 * GemslrClass::Setup (gemslr.cpp:1602-1711) when no reference library is
 * linked; partitions come from this library's own bisection, not METIS. */
/* Slot 58 value for a greedy multicolor order inside every subdomain (red-black
 * on a grid stencil), an option beyond the reference's orderings
 * (kIluReorderingNo..Input = 0..5, ilu.hpp:92-100).  The rows of one color are
 * uncoupled.  On the 3D 7-point Laplacian (ILUT 1e-3 / 200) the ILU factors
 * then have about a quarter of the dependency levels of the RCM order; the
 * level-0 triangular passes of a one-lane solve at 128^3 ran 1.35x shorter on
 * a B200, at 26 FGMRES iterations against 24.  On the 2D 5-point Laplacian
 * (ILUT 1e-2 / 20) the level counts are about equal. */
#define PGX_REORDER_MULTICOLOR 6
int pgx_gemslr_setup(pgx_handle *handle, const pgx_csr *A, const double *params, int32_t precision);

/* Bytes of device memory the committed handle holds (factors, matrices,
 * Krylov basis for kdim, work vectors), every solve slot and the multi-lane
 * factor layouts included; used for admission control. */
int pgx_gemslr_device_bytes(pgx_handle handle, int32_t kdim, int64_t *bytes);

/* Nonzeros of the preconditioner, counted as ParallelGemslrClass::GetNumNonzeros
 * counts them (parallel_gemslr.cpp:7609-7632 over 1022-1056): nnz_bsolver sums
 * the ILU factors of every level's B blocks, n_l + nnz(L_l) + nnz(U_l)
 * (IluClass, ilu.cpp:2149); nnz_lr sums W_l and WH_l, m_l x r_l entries each.
 * Host-side, valid once every level is set; either pointer may be NULL. */
int pgx_gemslr_nnz(pgx_handle handle, int64_t *nnz_bsolver, int64_t *nnz_lr);

/* FGMRES(kdim) solve of A x = b right-preconditioned by GeMSLR
 * (FlexGmresClass::Solve, fgmres.hpp:263-558).  params is the reference's
 * double[180] parameter array (PARGEMSLR_IO_*, utils.hpp:77-297) from which
 * SOLVER_KDIM (11), SOLVER_MAXITS (12), SOLVER_TOL (13) and SOLVER_ATOL (14)
 * are read; NULL keeps kdim 50, maxits 100, tol 1e-6 relative.  x holds the
 * initial guess on entry and the solution on return. */
int pgx_gemslr_solve(pgx_handle handle, double *x, const double *b, int32_t location,
                     const double *params, pgx_result *result);

/* FlexGmresClass::GetRelativeResidual (fgmres.hpp:683): the Givens
 * relative residual estimates of the handle's last pgx_gemslr_solve or
 * pgx_gemslr_solve_static: entry 0 is ||r0||/||b||, entry j the estimate
 * after iteration j (fgmres.hpp:362-364, 450-452), and 0 for an iteration
 * that broke down.  *count receives iterations + 1 (the reference's vector
 * is maxits + 1 long and zero past the last iteration); a zero right-hand
 * side, or an x0 that already solves the system, gives one entry, 0.  At most
 * `capacity` entries are written to hist; hist may be NULL to ask for the
 * count.  Solves of the other slots (batch, server) keep no history. */
int pgx_gemslr_residual_history(pgx_handle handle, int32_t capacity, double *hist, int32_t *count);

/* ---- solve without device allocation -------------------------------------
 * No counterpart in the reference: it exists for callers of this library
 * that must not allocate device memory at solve time.  pgx_gemslr_solve
 * allocates a slot's Krylov basis on its first solve (and again when kdim
 * grows) and instantiates a CUDA graph of the restart cycle.  Some callers
 * cannot let that happen: an application whose device memory is owned by
 * its own pool (a framework's caching allocator or a fixed arena sized at
 * start-up) can see cudaMalloc fail although the pool has room; a
 * latency-bound loop cannot take the device-wide synchronisation that
 * cudaMalloc and cudaFree may cause; a service with a fixed memory budget
 * must not grow after start-up.
 *
 * pgx_gemslr_solve_static is pgx_gemslr_solve (same arguments, results and
 * errors) with the Krylov basis taken from a fixed pool of
 * PGX_STATIC_BASIS_BYTES in the library's static device memory, and with the
 * restart cycles enqueued kernel by kernel; it calls no cudaMalloc, cudaFree
 * or allocating library routine.  The pool must hold the basis:
 * 8*n*(kdim+1) bytes (rounded up to 256) plus n*(kdim+1) entries of the
 * preconditioner precision (8 bytes FP64, 4 bytes mixed); e.g. kdim = 50
 * allows n up to 41,120 in FP64 and 54,827 in the mixed precision.  Larger
 * problems are refused with PGX_ERROR_INVALID_PARAM and a message giving
 * both sizes.  The handle's own work space (allocated by commit) is used
 * as by pgx_gemslr_solve.
 *
 * Every GPU on which the library is loaded holds the pool until the process
 * exits.  The first call on a device looks up the pool's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture
 * begins.  The address is kept for the life of the device's primary
 * context: after cudaDeviceReset (or any teardown of that context) the
 * library must not be used on that device again in the same process, as the
 * kept address no longer belongs to the new context.  All calls on one
 * device share the pool and each clears the part
 * it uses before the solve, but calls that overlap on the GPU (from several
 * host threads, on one or several handles of the same device) race on it:
 * the caller must serialise them.  result->launches is 0: the kernels are
 * not counted by this variant. */
#define PGX_STATIC_BASIS_BYTES (32u << 20)
int pgx_gemslr_solve_static(pgx_handle handle, double *x, const double *b, int32_t location,
                            const double *params, pgx_result *result);

/* ---- concurrent solves and serving --------------------------------------
 * A committed handle holds the preconditioner (factors, coupling blocks,
 * low-rank bases) once; each solve slot adds its own work space (CUDA
 * stream, work vectors, Krylov basis, FGMRES state, captured restart cycle).
 * Solves in different slots run concurrently on the GPU and read the factors
 * in common.  A result does not depend on the slot that computed it or on
 * what ran beside it: every reduction has a fixed order.  The reference
 * solves one right-hand side at a time per process; slots have no
 * counterpart there. */
typedef struct pgx_server_s *pgx_server;

/* Number of solve slots (1..256; slot 0 is the handle itself).  Refused while
 * a server created on the handle is live. */
int pgx_gemslr_set_slots(pgx_handle handle, int32_t nslots);
/* Right-hand sides each additional slot (slots 1..) advances together: 1, 2
 * or 4.  A multi-lane slot keeps one FGMRES state per lane and runs the
 * triangular passes of all its lanes in one kernel, so each factor entry is
 * read once for all of them; every other step runs per lane with the
 * single-solve arithmetic, so results do not change with the lane count.
 * The slots are rebuilt; refused while a server is live. */
int pgx_gemslr_set_lanes(pgx_handle handle, int32_t lanes);
/* Device bytes one additional slot needs for FGMRES(kdim). */
int pgx_gemslr_slot_bytes(pgx_handle handle, int32_t kdim, int64_t *bytes);

/* Solve nrhs systems A X(:,r) = B(:,r) (columns with leading dimensions ldx
 * and ldb, x0 = the incoming X), spreading them over the slots; results[r]
 * receives each outcome.  Returns the first error met, PGX_SUCCESS
 * otherwise. */
int pgx_gemslr_solve_batch(pgx_handle handle, int32_t nrhs, double *X, int64_t ldx, const double *B,
                           int64_t ldb, int32_t location, const double *params, pgx_result *results);

/* Serving loop over one resident preconditioned matrix.  Requests queue in
 * submission order; pgx_server_step admits the oldest waiting request into
 * every free slot and advances each in-flight solve by at most one restart
 * cycle, without blocking; pgx_server_collect hands back finished requests
 * with their ids (request_id >= 0).  x and b stay borrowed until their
 * request is collected.  While a server is live, the handle's slots belong
 * to it: set_slots, solve, solve_batch, commit and destroy are refused.
 * pgx_server_destroy finishes the in-flight solves first. */
int pgx_server_create(pgx_handle handle, const double *params, pgx_server *server);
int pgx_server_submit(pgx_server server, double *x, const double *b, int32_t location, int64_t request_id);
int pgx_server_step(pgx_server server, int32_t *n_active, int32_t *n_queued);
int pgx_server_collect(pgx_server server, int32_t max, int64_t *ids, pgx_result *results, int32_t *n);
int pgx_server_destroy(pgx_server server);

/* Serve on a thread of the library's own: pgx_server_start runs the step
 * loop above on a background thread until pgx_server_stop (or destroy).
 * While it runs, pgx_server_submit and pgx_server_collect may be called from
 * any thread, and pgx_server_step is refused.  An error met by the thread is
 * returned by pgx_server_stop; the affected requests are collected with it
 * in their status. */
int pgx_server_start(pgx_server server);
int pgx_server_stop(pgx_server server);

/* Serving pool: many resident preconditioned matrices behind one request
 * queue and one device-memory budget.  No counterpart in the reference,
 * which serves one matrix per process.  pgx_pool_add makes a committed
 * handle a member (its factors, its own slot and that slot's Krylov basis
 * count against the budget at once; refused with PGX_ERROR_OOM when they do
 * not fit); while a handle is a member its slots belong to the pool and
 * solve, set_slots, commit and destroy are refused.  pgx_pool_submit queues
 * a request for member `index`.  pgx_pool_step advances every request in
 * flight by at most one restart cycle, then admits waiting requests first
 * fit in arrival order: a request runs in an idle slot of its member, or in
 * a new slot (work space and FGMRES(kdim) basis, pgx_gemslr_slot_bytes) if
 * the budget has room, if need be after releasing idle slots of other
 * members, least recently used first; otherwise it waits.  The pool's FGMRES
 * options come from `params` at creation (SOLVER_KDIM, MAXITS, TOL, ATOL).
 * pgx_pool_start / stop run the step loop on a thread of the library's own
 * (as pgx_server_start); pgx_pool_collect returns finished requests;
 * pgx_pool_stats the bytes counted now and at most so far, and the number of
 * slots; pgx_pool_destroy finishes the requests in flight and returns the
 * handles to their owners. */
typedef struct pgx_pool_s *pgx_pool;
int pgx_pool_create(int64_t budget_bytes, const double *params, pgx_pool *pool);
int pgx_pool_add(pgx_pool pool, pgx_handle handle, int32_t *index);
int pgx_pool_submit(pgx_pool pool, int32_t index, double *x, const double *b, int32_t location,
                    int64_t request_id);
int pgx_pool_step(pgx_pool pool, int32_t *n_active, int32_t *n_queued);
int pgx_pool_start(pgx_pool pool);
int pgx_pool_stop(pgx_pool pool);
int pgx_pool_collect(pgx_pool pool, int32_t max, int64_t *ids, pgx_result *results, int32_t *n);
int pgx_pool_stats(pgx_pool pool, int64_t *bytes_in_use, int64_t *peak_bytes, int32_t *slots);
int pgx_pool_destroy(pgx_pool pool);

/* ---- many systems in one launch -----------------------------------------
 * No counterpart in the reference, which solves one system per
 * FlexGmresClass::Solve call (fgmres.hpp:263-558).  A systems object packs
 * the preconditioners of `count` committed real handles (each its own
 * matrix, levels, factors and low-rank bases; sizes may differ) and solves
 * all of them with ONE persistent kernel launch: each CTA takes the next
 * system of a work list ordered by estimated cost, largest first, and runs
 * that system's whole FGMRES(kdim) with its GeMSLR preconditioner (level
 * recursion, low-rank corrections, the level-0 inner Schur FGMRES) before it
 * takes the next.  The arithmetic is that of pgx_gemslr_solve with the same
 * handle and precision; sums are formed in another order, so iterates agree
 * to rounding, not bit for bit.  The handles stay usable and unchanged; the
 * object keeps its own copies and may outlive them.
 *   pgx_systems_solve: x[i] (initial guess in, solution out) and b[i] of
 *     system i, all on the host or all on the device; params as for
 *     pgx_gemslr_solve (one set for every system); results[i] receives system
 *     i's outcome, its solve_ms being the span of that system inside the
 *     launch and launches 1.
 *   pgx_systems_tune: the schedule autotuner.  It solves a sample of the
 *     batch (every stride-th system of the work list past its largest
 *     sixteenth; stride 1 is the whole batch) from x0 = 0 into the object's
 *     own vectors, by coordinate descent over the CTA shape (256 threads x 2
 *     per SM, 512 x 1, 512 x 2, 1024 x 1), then the SpMV lanes per row (2, 4,
 *     8), then the levels the triangular passes fetch ahead (2, 3); it keeps
 *     the fastest and returns its device time.  pgx_systems_tune_table returns
 *     the candidates tried, five doubles each (threads, CTAs per SM, lanes,
 *     depth, ms).
 *   pgx_systems_set_schedule / get_schedule: the schedule in use (default 256
 *     threads, 2 CTAs per SM, 2 lanes, depth 2).
 *   pgx_systems_timing: per system, the start and end of its solve in the last
 *     launch, in ms from the first system's start, and the time it spent in
 *     its triangular (B-block) solves (device clock; any array may be NULL);
 *     pgx_systems_last_ms: the device time of the last solve's launch (CUDA
 *     events around the kernel). */
typedef struct pgx_systems_s *pgx_systems;
int pgx_systems_create(pgx_systems *out, const pgx_handle *handles, int32_t count);
int pgx_systems_solve(pgx_systems systems, double *const *x, const double *const *b, int32_t location,
                      const double *params, pgx_result *results);
int pgx_systems_tune(pgx_systems systems, const double *const *b, int32_t location, const double *params,
                     int32_t stride, double *best_ms);
int pgx_systems_tune_table(pgx_systems systems, int32_t capacity, double *table, int32_t *rows);
int pgx_systems_set_schedule(pgx_systems systems, int32_t threads, int32_t ctas_per_sm, int32_t lanes,
                             int32_t depth);
int pgx_systems_get_schedule(pgx_systems systems, int32_t *threads, int32_t *ctas_per_sm, int32_t *lanes,
                             int32_t *depth);
int pgx_systems_timing(pgx_systems systems, int32_t capacity, double *start_ms, double *end_ms, double *tri_ms);
int pgx_systems_last_ms(pgx_systems systems, double *ms);
int pgx_systems_device_bytes(pgx_systems systems, int64_t *bytes);
int pgx_systems_destroy(pgx_systems systems);

/* Apply the preconditioner once, z = M^-1 v (GemslrClass::Solve,
 * gemslr.cpp:3431-3472), on host or device vectors. */
int pgx_gemslr_precond_apply(pgx_handle handle, double *z, const double *v, int32_t location);

/* Measurement: average device time (CUDA events on the handle's stream,
 * over `reps` launches) and algorithmic bytes per launch of one building
 * block of the solve: which 0 = lower triangular pass of `level`, 1 = upper
 * triangular pass of `level`, 2 = outer CSR SpMV, 3 / 4 = the lower / upper
 * pass of `level` merged over the lanes of a multi-lane slot (vectors counted
 * once per lane, the factor once).  Algorithmic bytes count
 * every operand once: nnz*(value+index) + row pointers + schedule + vectors
 * in and out. */
int pgx_gemslr_kernel_stats(pgx_handle handle, int32_t which, int32_t level, int32_t reps, double *avg_ms,
                            double *bytes);

/* A text description of slot `slot` of a committed handle (0 = the handle's
 * own slot), one line per structure: for every level the kernel and layout
 * of the L and U passes (per-subdomain pipeline, segmented or level-set;
 * lanes per row, dependency levels, chunks) and the SpMV variant of A, E_l,
 * F_l and C_0 (lanes per row or merge path); for a multi-lane slot its
 * merged layouts.  Plays the part of the reference's setup report
 * (GemslrClass print level).  *length receives the text's length; at most
 * capacity - 1 characters and a terminating zero are written to buf, which
 * may be NULL to ask for the length. */
int pgx_gemslr_describe(pgx_handle handle, int32_t slot, char *buf, int32_t capacity, int32_t *length);

/* Bounded waits.  No counterpart in the reference, whose triangular solves
 * run on one host thread.  The triangular solves that cross subdomains
 * (factors that are not block diagonal, or subdomains too large for one CTA)
 * let a row wait on values other CTAs publish; every such wait gives up
 * after `polls` polls of about 20 ns each (default 2^21), records the
 * expiry, and the kernel finishes, so the solve returns PGX_ERROR_TIMEOUT
 * instead of hanging and the CUDA context stays usable.
 * pgx_gemslr_set_wait_limit sets the bound for every slot of a handle
 * (captured restart cycles are rebuilt).  pgx_wait_selfcheck runs that
 * triangular kernel, on the current device, over two rows of which the
 * second waits on the first and only the second is scheduled: nothing ever
 * publishes the value, so the wait can only end by its bound.  *status
 * receives what a solve would report (PGX_ERROR_TIMEOUT when the bound
 * worked) and *wait_ms the kernel's device time. */
int pgx_gemslr_set_wait_limit(pgx_handle handle, int64_t polls);
int pgx_wait_selfcheck(int64_t polls, int32_t *status, double *wait_ms);

/* ---- building blocks (each is also used inside the solve) ---------------
 * The level-set schedule of a unit-lower (uplo 'L') or upper (uplo 'U')
 * triangular CSR factor, by the rule of IluClass::BuildLevels
 * (ilu.cpp:832-1062): level(i) = 1 + max level over the row's dependencies,
 * rows ordered by level then by index.  level_ptr needs n+1 entries,
 * order n entries; *nlevels receives the number of levels. */
int pgx_build_levels(char uplo, int32_t n, const int32_t *rowptr, const int32_t *colidx,
                     int32_t *nlevels, int32_t *level_ptr, int32_t *order);

/* Read a coordinate Matrix Market file with real or integer values, general
 * or symmetric (the files CooMatrixClass::ReadFromMMFile /
 * CooMatrixReadFromFile accept, matrixops.cpp:11134), into 0-based CSR with
 * columns sorted within each row and duplicates summed; a symmetric file's
 * off-diagonal entries are mirrored.  The arrays are allocated by the
 * library: release them with pgx_csr_free.  Errors: PGX_ERROR_IO. */
int pgx_csr_read_mm(const char *path, pgx_csr *A);
int pgx_csr_free(pgx_csr *A);

/* Read a vector stored as a coordinate Matrix Market file of M rows (the
 * right-hand sides of the reference's matrix lists, e.g. gr_30_30_b.mtx), as
 * SequentialVectorClass::ReadFromMMFile reads it (vectorops.cpp:1116-1180):
 * M entries, zero except x[I - idxin] = value for each listed entry "I J
 * value", a later entry replacing an earlier one, J not used.  *n receives M;
 * x may be NULL to ask for M only, otherwise it needs capacity >= M entries.
 * Errors: PGX_ERROR_IO (unreadable file or entry, index out of range);
 * PGX_ERROR_INVALID_PARAM (capacity below M). */
int pgx_vector_read_mm(const char *path, int32_t idxin, int32_t capacity, double *x, int32_t *n);

/* ---- parameter arrays ----------------------------------------------------
 * The double[PGX_PARAMS_SIZE] array every entry point above takes is the one
 * SetWithParameterArray reads (index names in SRC/utils/utils.hpp:77-297).
 * pgx_params_default fills it as PargemslrSetDefaultParameterArray does
 * (SRC/utils/utils.cpp:30-126).  pgx_params_read_file then overwrites the
 * slots a driver's parameter file names, as that driver's
 * read_inputs_from_file does, line k of the file setting its fixed slots:
 *   PGX_INPUTS_SEQUENTIAL  TESTS/sequential/inputs (io.cpp:336-725)
 *   PGX_INPUTS_PARALLEL    TESTS/parallel/inputs (io_par.cpp:359-819)
 *   PGX_INPUTS_HYPRE       TESTS/hypre/inputs (pargemslr_hypre_interface.cpp:391-820)
 * Errors: PGX_ERROR_IO for a file that cannot be opened or an unknown keyword
 * (the line is named in pgx_last_error; the lines before it stay applied, as
 * in the reference); PGX_ERROR_INVALID_PARAM for an unknown format. */
#define PGX_PARAMS_SIZE 180
#define PGX_INPUTS_SEQUENTIAL 0
#define PGX_INPUTS_PARALLEL   1
#define PGX_INPUTS_HYPRE      2
int pgx_params_default(double *params);
int pgx_params_read_file(const char *path, int32_t format, double *params);
/* The command-line overrides the drivers' read_inputs applies
 * (TESTS/sequential/io.cpp:729-748): "-tol V", "-kdim N", "-maxits N" among
 * argv[0..argc-1], each taking the first occurrence whose next argument does
 * not start with '-', read with atof / atoi (PargemslrReadInputArg,
 * SRC/utils/utils.cpp:389-416). */
int pgx_params_read_args(int32_t argc, const char *const *argv, double *params);

/* CSR SpMV, y = alpha * A x + beta * y (CsrMatrixClass::MatVec,
 * matrixops.cpp:5139-5330), with the kernel every solve uses for A, E_l,
 * F_l and C_0.  The variant is picked per matrix from its row-length
 * histogram (pgx_csr_spmv_plan, host arrays): S lanes per row, with S the
 * smallest power of two (2..32) for which the 90th-percentile row fits one
 * batch of S * 4 unrolled loads; or the merge-path SpMV (every thread the
 * same number of row ends plus nonzeros) when rows are skewed: the longest
 * row is longer than 16 batches and rows longer than 4 batches hold more
 * than a tenth of the nonzeros.  pgx_csr_spmv_device runs the plan's choice
 * on device arrays; pgx_csr_spmv_device_variant forces one: 0 the plan's,
 * 1 lanes per row, 2 merge path.  The two variants sum a row in different
 * orders, so their results agree to rounding, not bit for bit. */
int pgx_csr_spmv_plan(const pgx_csr *A, int32_t *lanes, int32_t *merge_path);
int pgx_csr_spmv_device(const pgx_csr *A_device, double alpha, const double *x, double beta, double *y);
int pgx_csr_spmv_device_variant(const pgx_csr *A_device, int32_t variant, double alpha, const double *x,
                                double beta, double *y);

/* Block low-rank correction of complex64 vectors on the tensor cores, the
 * kernel pair a complex mixed-precision slot of 8 or 16 lanes applies at
 * every level (GemslrClass::SolveApplyLowRankLevel, gemslr.cpp:3681-3722,
 * followed by the Axpy of gemslr.cpp:3585-3590, for all lanes at once):
 *   x_q <- x_q + WH (W^H x_q),  q = 0 .. nrhs-1
 * W and WH are m x r column-major, X holds nrhs vectors ldx values apart;
 * every array is complex64 ({re, im} floats) in device memory.  nrhs is 8 or
 * 16 and r at most 64.  The two GEMMs run as tcgen05.mma kind::tf32 with each
 * FP32 operand split into a high and a low tf32 part (three MMAs per product),
 * which keeps them to about FP32 accuracy.  This call allocates its scratch
 * and synchronises the device; the slots keep theirs. */
int pgx_lowrank_block_apply_c64(int32_t m, int32_t r, int32_t nrhs, const void *W, const void *WH, void *X,
                                int64_t ldx);

#ifdef __cplusplus
}
#endif

#endif /* PGX_H */
