/* tensors_b200 -- C-ABI of the B200 supernodal sparse Cholesky.
 *
 * A drop-in for the Sparse::CholeskyDecomposition<Scal,Int,LInt,parQ> path of
 * HenrikSchumacher/Tensors (src/Sparse/CholeskyDecomposition.hpp).  The
 * reference is a header-only C++ class with no C interface; every function
 * here replaces one of its members, cited as file:line of the reference.
 * Integer types follow the reference's driver (Example_SparseCholesky/
 * main.cpp:31-32): Int = int32_t for rows/columns, LInt = int64_t for
 * nonzero positions.  Scal = double.
 *
 * Conventions
 *  - Every function returns an int status: TB_OK (0) on success, a positive
 *    TB_NOT_SPD from the numeric factorization when a pivot is not positive
 *    (the reference returns 1, CholeskyDecomposition/Numeric.hpp:99), and a
 *    negative TB_ERR_* on misuse or a CUDA failure.  tb_last_error() gives a
 *    message for the last failure on the calling thread.
 *  - Matrices are CSR with the full symmetric pattern and a structurally
 *    present diagonal (CholeskyDecomposition.hpp:63-65, :404-423).
 *  - Right-hand sides and solutions are row-major n x nrhs blocks with leading
 *    dimensions, as in CholeskyDecomposition/Solve.hpp:22-80.
 *  - Functions without a _device suffix take HOST pointers and copy through
 *    pinned staging buffers; _device variants take device pointers on the
 *    handle's GPU and stream.
 *  - A handle is not re-entrant (neither is the reference object): use one
 *    handle per host thread / stream.
 */
#ifndef TENSORS_B200_H
#define TENSORS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum tb_status {
    TB_OK                      = 0,
    TB_NOT_SPD                 = 1,
    TB_ERR_INVALID_ARGUMENT    = -1,
    TB_ERR_INVALID_PATTERN     = -2,
    TB_ERR_INVALID_PERMUTATION = -3,
    TB_ERR_MISSING_DIAGONAL    = -4,
    TB_ERR_NOT_FACTORIZED      = -5,
    TB_ERR_CUDA                = -6,
    TB_ERR_OUT_OF_MEMORY       = -7,
    TB_ERR_NO_DEVICE           = -8,
    TB_ERR_TIMEOUT             = -9,
    TB_ERR_NOT_CONVERGED       = -10,
    TB_ERR_IO                  = -11,
    TB_ERR_FORMAT              = -12
};

/* Supernode strategies (CholeskyDecomposition.hpp:119-124). */
enum tb_supernode_strategy { TB_SN_MAXIMAL = 0, TB_SN_FUNDAMENTAL = 1, TB_SN_AMALGAMATED = 2 };

/* Factorization methods (CholeskyDecomposition.hpp:126-130).  Both compute
 * the same factor; on the GPU both run the level-scheduled supernodal kernels. */
enum tb_factorization_method { TB_MULTIFRONTAL = 0, TB_LEFT_LOOKING = 1 };

/* Arrays of the symbolic structure, for tb_chol_array_size/_copy
 * (getters of CholeskyDecomposition/InputOutput.hpp:304-367 and the trees). */
enum tb_array {
    TB_ARRAY_PERM = 0,            /* GetPermutation().GetPermutation()        */
    TB_ARRAY_PERM_INV = 1,        /* GetPermutation().GetInversePermutation() */
    TB_ARRAY_VALUE_PERM = 2,      /* GetValuePermutation()                    */
    TB_ARRAY_SN_RP = 3,           /* SN_RowPointers()                         */
    TB_ARRAY_SN_OUTER = 4,        /* SN_Outer()                               */
    TB_ARRAY_SN_INNER = 5,        /* SN_Inner()                               */
    TB_ARRAY_ROW_TO_SN = 6,       /* RowToSN()                                */
    TB_ARRAY_SN_TRI_PTR = 7,      /* SN_TrianglePointers()                    */
    TB_ARRAY_SN_REC_PTR = 8,      /* SN_RectanglePointers()                   */
    TB_ARRAY_ATREE_PARENTS = 9,   /* AssemblyTree().Parents()                 */
    TB_ARRAY_ETREE_PARENTS = 10,  /* EliminationTree().Parents()              */
    TB_ARRAY_OUTER = 11,          /* GetA().Outer()  (permuted pattern)       */
    TB_ARRAY_INNER = 12,          /* GetA().Inner()                           */
    TB_ARRAY_ATREE_CHILD_PTR = 13,/* AssemblyTree().ChildPointers()           */
    TB_ARRAY_ATREE_CHILD_IDX = 14 /* AssemblyTree().ChildIndices()            */
};

/* Scalar types of values, right-hand sides and solutions at the boundary
 * (the reference's ExtScal and B_T / X_T template arguments). */
enum tb_dtype { TB_F64 = 0, TB_F32 = 1 };

typedef struct tb_chol tb_chol;
typedef struct tb_factor tb_factor;

/* Message of the last failing call on this thread (never NULL). */
const char * tb_last_error( void );

/* Phase ranges.  Every phase of the path (symbolic analysis and its steps,
 * numeric factorization, ReadNonzeroValues, ClearFactors, solves and their
 * sweeps) is an NVTX range named with the reference's TOOLS_PTIMER tag of
 * that phase (e.g. "CholeskyDecomposition::NumericFactorization",
 * Numeric.hpp:34), visible in timeline tools.  tb_trace_record(1) clears and
 * starts a host-side list of the ranges entered (0 stops it);
 * tb_trace_names copies it, one name per line, into buf (at most cap bytes,
 * NUL-terminated) and returns the bytes the whole list needs.
 * tb_trace_times writes the host wall time of each recorded range, in the
 * same order, in milliseconds (-1 for a range still open), into ms (at most
 * cap entries) and returns the number of recorded ranges: the durations the
 * reference's TOOLS_PTIMER logs for the same phases. */
int tb_trace_record( int32_t enabled );
int64_t tb_trace_names( char * buf, int64_t cap );
int64_t tb_trace_times( double * ms, int64_t cap );

/* Library / device information: CUDA device ordinal used by new handles. */
int tb_set_device( int device );

/* Constructors, CholeskyDecomposition.hpp:313-371.  The pattern is copied.
 * perm == NULL: the matrix is already permuted (ctor :350).  Otherwise
 * perm[i] is the original index placed at position i (ctor :336,
 * Inverse::False).  thread_count is the host thread count of the symbolic
 * phase and the device plan (the reference's thread_count); 0 or less: every
 * hardware thread.  The result does not depend on it. */
int tb_chol_create( tb_chol ** out, int32_t n, const int64_t * outer, const int32_t * inner,
                    const int32_t * perm, int32_t thread_count );
int tb_chol_destroy( tb_chol * h );

/* Setters, CholeskyDecomposition/InputOutput.hpp:369-409. */
int tb_chol_set_supernode_strategy( tb_chol * h, int32_t strategy );
int tb_chol_set_amalgamation_threshold( tb_chol * h, int32_t threshold );
int tb_chol_set_factorization_method( tb_chol * h, int32_t method );

/* SymbolicFactorization(), CholeskyDecomposition/Symbolic.hpp:3-66.  Lazy and
 * idempotent; also builds and uploads the device execution plan. */
int tb_chol_symbolic( tb_chol * h );

/* NumericFactorization(A_val, reg), CholeskyDecomposition/Numeric.hpp:3-24:
 * values in the caller's original CSR order; reg is added to every diagonal
 * entry.  Returns TB_OK, TB_NOT_SPD (the handle is still marked factorized,
 * Numeric.hpp:95) or an error. */
int tb_chol_numeric( tb_chol * h, const double * values, double reg );
int tb_chol_numeric_device( tb_chol * h, const double * d_values, double reg );
/* NumericFactorization<ExtScal>(cptr<ExtScal> A_val, ExtScal reg),
 * Numeric.hpp:3-8: values of type dtype (TB_F64 or TB_F32), converted to
 * FP64 on copy (ReadNonzeroValues casts, Numeric.hpp:165-180). */
int tb_chol_numeric_ex( tb_chol * h, const void * values, int32_t dtype, double reg );
int tb_chol_numeric_device_ex( tb_chol * h, const void * d_values, int32_t dtype, double reg );

/* Solve: X = alpha * A^{-1} B + beta * X (Solve.hpp:22-80).  B and X are
 * row-major n x nrhs with leading dimensions ldB, ldX >= nrhs; they may
 * alias.  When beta == 0 the old X is not read. */
int tb_chol_solve( tb_chol * h, double alpha, const double * B, int32_t ldB,
                   double beta, double * X, int32_t ldX, int32_t nrhs );
int tb_chol_solve_device( tb_chol * h, double alpha, const double * d_B, int32_t ldB,
                          double beta, double * d_X, int32_t ldX, int32_t nrhs );
/* Solve<NRHS,parQ,op,a_T,B_T,b_T,X_T> (Solve.hpp:20-27): B of type b_dtype
 * and X of type x_dtype (TB_F64 or TB_F32), each cast on copy; the solve
 * itself runs as tb_chol_solve / tb_chol_solve_device. */
int tb_chol_solve_ex( tb_chol * h, double alpha, const void * B, int32_t ldB, int32_t b_dtype,
                      double beta, void * X, int32_t ldX, int32_t x_dtype, int32_t nrhs );
int tb_chol_solve_device_ex( tb_chol * h, double alpha, const void * d_B, int32_t ldB, int32_t b_dtype,
                             double beta, void * d_X, int32_t ldX, int32_t x_dtype, int32_t nrhs );

/* NumericalFactorization_T (CholeskyDecomposition.hpp:132-201): a numeric
 * factor held apart from any handle (device memory: the factor storage, the
 * inverse diagonal blocks and the values it was computed from).  A new one is
 * empty (not factorized).  tb_factor_state: NumericallyFactorizedQ,
 * NumericallyGoodQ, AllocatedByteCount and the precision of the stored factor
 * (-1 when it never held one). */
int tb_factor_create( tb_factor ** out );
int tb_factor_destroy( tb_factor * f );
int tb_factor_state( tb_factor * f, int32_t * factorized, int32_t * good, int64_t * bytes, int32_t * precision );
/* SwapNumericalFactorization (Numeric.hpp:228-254): exchanges the handle's
 * numeric factor with f.  A factor that says factorized but not good, or
 * whose storage is smaller than the handle's symbolic analysis requires, is
 * then treated as unfactorized.  The handle takes the incoming factor's
 * precision; its captured factor and solve graphs are dropped (they hold the
 * outgoing storage's addresses).  f must be empty or live on the handle's
 * device. */
int tb_chol_swap_factor( tb_chol * h, tb_factor * f );

/* Half solves (Solve.hpp:182-310) with the documented meaning:
 * upper: X = alpha * P^T U^{-1} P B + beta X;  lower: X = alpha * P^T U^{-T} P B + beta X. */
int tb_chol_upper_solve( tb_chol * h, double alpha, const double * B, int32_t ldB,
                         double beta, double * X, int32_t ldX, int32_t nrhs );
int tb_chol_lower_solve( tb_chol * h, double alpha, const double * B, int32_t ldB,
                         double beta, double * X, int32_t ldX, int32_t nrhs );

/* Residual helper: R = B - A X for the matrix passed to the last numeric
 * factorization (values in caller order), on device buffers (row-major,
 * leading dimension nrhs).  Used for iterative refinement and tests. */
int tb_chol_residual_device( tb_chol * h, const double * d_B, const double * d_X,
                             double * d_R, int32_t nrhs );

/* Queries. */
int tb_chol_sn_count( tb_chol * h, int32_t * out );
int tb_chol_row_count( tb_chol * h, int32_t * out );
int tb_chol_nonzero_count( tb_chol * h, int64_t * out );
int tb_chol_array_size( tb_chol * h, int32_t which, int64_t * out );
int tb_chol_array_copy( tb_chol * h, int32_t which, int64_t * out );
int tb_chol_factorized( tb_chol * h, int32_t * factorized, int32_t * good );
/* First supernode whose pivot failed, or -1. */
int tb_chol_failed_supernode( tb_chol * h, int32_t * out );
/* RequiredTriangularSize / RequiredRectangularSize (Numeric.hpp:193-215). */
int tb_chol_factor_sizes( tb_chol * h, int64_t * tri_size, int64_t * rec_size );
/* Copy the factor back in the reference's layout: SN_TriangleValues and
 * SN_RectangleValues (InputOutput.hpp:339-352), row-major U0 / U1 blocks. */
int tb_chol_factor_values( tb_chol * h, double * tri, double * rec );
/* U as a CSR matrix in the permuted ordering, as the reference's GetU
 * (InputOutput.hpp:116-217): row i of supernode s holds the triangle's
 * columns i .. end of s, then the supernode's column set; rows sorted.
 * tb_chol_u_nonzero_count (host-only, after the symbolic phase) sizes
 * inner / values; outer has n + 1 entries. */
int tb_chol_u_nonzero_count( tb_chol * h, int64_t * out );
int tb_chol_get_u( tb_chol * h, int64_t * outer, int32_t * inner, double * values );
/* LogDeterminant (InputOutput.hpp:294-297) and WriteFactorDiagonal (:238-257). */
int tb_chol_log_det( tb_chol * h, double * out );
int tb_chol_factor_diagonal( tb_chol * h, double * diag );
/* Factor flops Sum_s [n0^3/3 + n0^2 n1 + n0 n1^2] and nnz(U). */
int tb_chol_flop_count( tb_chol * h, double * factor_flops, double * nnz_u );
/* Plan statistics (host-only, after the symbolic phase): out[0] arena
 * doubles (triangles + rectangles + update matrices), out[1] update-matrix
 * doubles, out[2] levels, out[3] factorization launches, out[4] GEMM tile
 * tasks, out[5] panel tasks, out[6] extend-add tasks, out[7] forward-solve
 * launches, out[8] back-solve launches, out[9] supernodes, out[10] fronts
 * (runs of supernodes merged for computation), out[11] flops of the front
 * factorization (explicit zeros of merged fronts included), out[12] simulated
 * microseconds of the scheduled task graph (0 before the first numeric
 * factorization on a device), out[13] tasks of the graph, out[14] tasks of
 * the solve's task graph, out[15] its first level, out[16] CTAs of the
 * persistent factorization launch (0 before the device plan exists),
 * out[17] / out[18] host microseconds of the last symbolic analysis / plan
 * build, out[19] tensor-core tiles of the mixed-precision path, out[20]
 * blocks of its operand image (8 KB each), out[21] useful flops of the
 * 64 x 64 GEMM tiles, out[22] the flops those tiles execute (full tiles),
 * out[23] super-panels of the large fronts' solves, out[24] / out[25] the
 * forward / back sweep launches with them.  Returns the number of entries
 * written (at most cap). */
int tb_chol_plan_stats( tb_chol * h, int64_t * out, int32_t cap );
/* Host-side bounds check of every device task of the plan (also run before
 * the plan is first uploaded).  TB_OK or TB_ERR_INVALID_ARGUMENT with the
 * first violation in tb_last_error(). */
int tb_chol_check_plan( tb_chol * h );
/* Device bytes held by the handle. */
int tb_chol_device_bytes( tb_chol * h, int64_t * out );

/* Stream of the handle (a cudaStream_t; NULL = a stream the handle owns). */
int tb_chol_set_stream( tb_chol * h, void * stream );
/* Capture the numeric factorization into a CUDA graph on first use (default
 * on); off runs the same kernels as individual launches. */
int tb_chol_set_graph( tb_chol * h, int32_t enabled );
/* Arithmetic of the factorization.  TB_PRECISION_FP64 (default): FP64 factor,
 * FP64 arithmetic.  TB_PRECISION_MIXED: the factor is stored in FP32, the
 * Schur-complement updates (the bulk of the flops) run as split-precision
 * 3xTF32 tensor-core products with FP32 accumulation, the diagonal-block
 * Cholesky and the triangular solves with the panels run in FP64 on FP32
 * data, and tb_chol_solve / tb_chol_solve_device refine in FP64: conjugate
 * gradients on (A + reg I) x = b with the FP64 matrix, preconditioned by the
 * FP32 factor, until max_c |b_c - (A + reg I) x_c| / |b_c| <= tol.  Half
 * solves are not refined.  Changing the precision discards the factor. */
enum tb_precision { TB_PRECISION_FP64 = 0, TB_PRECISION_MIXED = 1 };
int tb_chol_set_precision( tb_chol * h, int32_t precision );
/* Refinement target and iteration cap of mixed-precision solves (defaults
 * 1e-12, 30). */
int tb_chol_set_refinement( tb_chol * h, double tol, int32_t max_iterations );
/* Refinement steps and final relative residual of the last mixed solve. */
int tb_chol_refinement_info( tb_chol * h, int32_t * iterations, double * relres );
/* When the refinement of a mixed solve breaks down (its residual becomes
 * non-finite, grows a million-fold, or misses the target within the cap:
 * FP32 is too coarse for the matrix, kappa far beyond 1 / eps_fp32), the
 * solve refactors the same matrix in FP64 from the values the handle holds
 * on the device and runs the same refinement with the FP64 factor as the
 * preconditioner; the handle then stays in FP64 (its solves still refined to
 * the target) until tb_chol_set_precision is called again.  This reports the precision in use
 * (TB_PRECISION_FP64 after such a fallback) and whether the fallback
 * happened (no counterpart in the reference, which has no mixed precision). */
int tb_chol_precision_in_use( tb_chol * h, int32_t * precision, int32_t * fell_back );
/* Mixed precision only: pivots of the last factorization that came out at or
 * below tau = 1e-5 x |assembled diagonal entry of the row| and were raised to
 * tau instead of failing (static pivoting: for ill-conditioned matrices FP32
 * rounding of the Schur complements can wipe out small pivots, and the FP64
 * refinement corrects the perturbation).  In this mode a matrix that is not
 * positive definite is reported by the solve, whose refinement then does not
 * reach its target (TB_ERR_NOT_CONVERGED), not by the factorization. */
int tb_chol_perturbed_pivots( tb_chol * h, int32_t * out );
/* Schedule of the numeric factorization.  TB_SCHEDULE_LEVELS (default): one
 * launch per task kind, level and panel step (also used while profiling).
 * TB_SCHEDULE_TASK_GRAPH: the levels below the first level with 8
 * or more panel steps run as level launches; the levels from there up run as
 * one persistent launch whose CTAs take the tasks (extend-adds, panel potrf /
 * trsm, GEMM tiles, inverse diagonal blocks) from a dependency-ordered list,
 * so the next panel of a front and independent fronts overlap.
 * TB_SCHEDULE_TASK_GRAPH_ALL: every level in the persistent launch (changing
 * to or from it redoes the symbolic phase).  All compute the same factor,
 * bit for bit. */
enum tb_schedule { TB_SCHEDULE_LEVELS = 0, TB_SCHEDULE_TASK_GRAPH = 1, TB_SCHEDULE_TASK_GRAPH_ALL = 2 };
int tb_chol_set_schedule( tb_chol * h, int32_t schedule );
/* Schedule of the solve sweeps.  TB_SCHEDULE_LEVELS (default): one launch per
 * level and panel step in each sweep.  TB_SCHEDULE_TASK_GRAPH: the levels
 * below the first level with 4 or more panel steps as level launches, the
 * levels from there up as one persistent launch per sweep whose CTAs take the
 * solve tasks in dependency order (a panel's tasks start once every update of
 * its rows is in).  TB_SCHEDULE_TASK_GRAPH_ALL: every level in the persistent
 * launch.  The schedules agree to rounding (updates of shared rows are
 * atomic additions in any order).  A wait of the persistent launch that runs
 * out of time is reported (TB_ERR_TIMEOUT) by the next call that
 * synchronizes with the solve. */
int tb_chol_set_solve_schedule( tb_chol * h, int32_t schedule );
/* Autotuner (no counterpart in the reference): after a numeric
 * factorization, times the factorization of the same values under
 * TB_SCHEDULE_LEVELS and TB_SCHEDULE_TASK_GRAPH and one solve with nrhs
 * right-hand sides under both solve schedules (best of two runs each, after
 * one that captures the graphs), and keeps the fastest of each.  The factor
 * is the same bit for bit under both factor schedules, so it stays valid.
 * choice (2 entries, may be NULL): the factor and the solve schedule chosen;
 * times_ms (4 entries, may be NULL): factor levels, factor task graph, solve
 * levels, solve task graph. */
int tb_chol_autotune( tb_chol * h, int32_t nrhs, int32_t * choice, double * times_ms );
/* Plan options (no counterpart in the reference): defer_steps (1-4) panel
 * steps over which a front's trailing update is deferred (default 3); relax,
 * the fronts' amalgamation relaxation: 0 tight, 1 default, 2 loose; tc_width,
 * the widest tensor-core tile of the mixed-precision path (128 or 256).  A
 * change rebuilds the device plan (the symbolic analysis stands) and leaves
 * the handle unfactorized.  tb_chol_autotune_plan: after a factorization,
 * factors the same values under each candidate set (deferral 2-4 x the three
 * relaxations, x both tile widths in mixed precision), timed, keeps the
 * fastest and refactors under it; choice[0..2] the kept options, times_ms[i]
 * (at most cap) each candidate's ms.  Returns the number of candidates. */
int tb_chol_set_plan_options( tb_chol * h, int32_t defer_steps, int32_t relax, int32_t tc_width );
int tb_chol_plan_options( tb_chol * h, int32_t * defer_steps, int32_t * relax, int32_t * tc_width );
int tb_chol_autotune_plan( tb_chol * h, int32_t * choice, double * times_ms, int32_t cap );
/* Execution trace of the persistent factorization launch: when enabled,
 * each task records when it was taken, when its inputs were ready, when it
 * was done (%globaltimer ns) and which CTA ran it.  tb_chol_trace writes 6
 * entries per task in list order (kind, index, taken, ready, done, CTA;
 * cap >= 6 x tasks) for the last factorization and returns the task count. */
int tb_chol_set_trace( tb_chol * h, int32_t enabled );
int tb_chol_trace( tb_chol * h, int64_t * out, int64_t cap );
/* Execution trace of the persistent solve launches of the last solve with
 * the trace enabled (tb_chol_set_trace), first 64 right-hand sides: per task
 * of the forward then the back sweep, 6 int64 (sweep 0/1, solve task index,
 * taken_ns, ready_ns, done_ns, cta), in list order.  Returns the number of
 * rows; cap must hold 12 x the graph's task count. */
int tb_chol_solve_trace( tb_chol * h, int64_t * out, int64_t cap );
/* Per-kernel timing: when enabled, factorizations run as direct launches
 * bracketed by CUDA events and tb_chol_kernel_profile reports, per launch
 * kind (0 zero, 1 extend-add, 2 panel trsm, 3 GEMM tiles, 4 inversion of
 * the diagonal blocks for the solves, 6 panel potrf, 7 clear + assembly),
 * the milliseconds and launches of the last factorization and the
 * algorithmic flops of the GEMM tiles (8 entries each). */
int tb_chol_set_profiling( tb_chol * h, int32_t enabled );
int tb_chol_kernel_profile( tb_chol * h, double * ms, int64_t * launches, double * flops );
/* Per launch of the last profiled factorization (at most cap entries):
 * info[4i..4i+3] = kind, level, panel step (or child rank), task count and
 * ms[i] its duration; entry 0 is the clear + assembly.  Returns the count. */
int tb_chol_launch_profile( tb_chol * h, int64_t * info, double * ms, int32_t cap );
/* Direct solve with the FP64 factor (tb_chol_solve_device's result on an FP64
 * handle) that allocates no device memory: its two permuted work blocks live
 * in a fixed device array of 2 x 4,194,304 doubles (64 MiB) per device, so
 * n * nrhs must not exceed 4,194,304 (else TB_ERR_INVALID_ARGUMENT, nothing
 * launched).  For callers that may not allocate at solve time.  Handles that
 * solve by refinement (mixed precision, or FP64 after a failed refinement) are
 * rejected with TB_ERR_INVALID_ARGUMENT.  The sweeps run as level launches
 * (no waits, no timeout).  The first call on a device looks the array up
 * (make it outside stream capture; the caller's current device is kept);
 * calls that can overlap on one device share the array and must be
 * serialised.  No counterpart in the reference. */
int tb_chol_solve_device_noalloc( tb_chol * h, double alpha, const double * d_B, int32_t ldB,
                                  double beta, double * d_X, int32_t ldX, int32_t nrhs );
/* Per launch of the last solve run with profiling enabled (at most cap
 * entries): info[4i..4i+3] = sweep (0 forward, 1 back), level, panel step,
 * task count and ms[i] its duration.  Returns the count. */
int tb_chol_solve_profile( tb_chol * h, int64_t * info, double * ms, int32_t cap );
/* Conjugate gradients preconditioned by the factor: the reference's
 * ConjugateGradient::operator() (ConjugateGradient.hpp:109-356) with the
 * operator X -> (A' + reg I) X and the preconditioner P = the handle's factor
 * (any precision).  A' has the handle's pattern and the given values (caller
 * CSR order; NULL: the values of the last factorization), so a factor can
 * precondition a nearby matrix.  X = alpha x + beta X, with x the iterate,
 * started from 0 or, with use_initial_guess, from X.  Stops when every column
 * meets |r.P r| <= rel_tol^2 |b.P b| (the reference's CheckResiduals,
 * :470-480) or after max_iter steps; iterations and, when non-NULL,
 * relres[nrhs] = sqrt(|r.P r| / |b.P b|) report the end state.
 * TB_ERR_NOT_CONVERGED (X still written) when a column misses the tolerance.
 * _device: device pointers on the handle's stream. */
int tb_chol_cg( tb_chol * h, const double * values, double reg, double alpha, const double * B, int32_t ldB,
                double beta, double * X, int32_t ldX, int32_t nrhs, double rel_tol, int32_t max_iter,
                int32_t use_initial_guess, int32_t * iterations, double * relres );
int tb_chol_cg_device( tb_chol * h, const double * values, double reg, double alpha, const double * B, int32_t ldB,
                       double beta, double * X, int32_t ldX, int32_t nrhs, double rel_tol, int32_t max_iter,
                       int32_t use_initial_guess, int32_t * iterations, double * relres );
/* Number of kernel launches the last numeric factorization / solve issued. */
int tb_chol_launch_counts( tb_chol * h, int64_t * factor_launches, int64_t * solve_launches );
/* GMRES preconditioned by the factor: the reference's GMRES::operator()
 * (GMRES.hpp:124-330), left preconditioning, restarted after max_iter Arnoldi
 * steps (two Gram-Schmidt passes each, Givens rotations), one Krylov space
 * per column, with the operator (A' + reg I) (values: A' in the caller's CSR
 * order, NULL = the factored values) and P = this factor's solve.
 * X = alpha x + beta X; with use_initial_guess the iteration starts from X.
 * Converged when every column's |P (b - A x)| <= rel_tol |P b| (its
 * CheckResiduals); relres[c] reports that ratio.  TB_ERR_NOT_CONVERGED after
 * max_restarts restarts without it (X still written). */
int tb_chol_gmres( tb_chol * h, const double * values, double reg, double alpha, const double * B, int32_t ldB,
                   double beta, double * X, int32_t ldX, int32_t nrhs, double rel_tol, int32_t max_iter,
                   int32_t max_restarts, int32_t use_initial_guess, int32_t * iterations, int32_t * restarts, double * relres );
int tb_chol_gmres_device( tb_chol * h, const double * d_values, double reg, double alpha, const double * d_B, int32_t ldB,
                          double beta, double * d_X, int32_t ldX, int32_t nrhs, double rel_tol, int32_t max_iter,
                          int32_t max_restarts, int32_t use_initial_guess, int32_t * iterations, int32_t * restarts,
                          double * relres );
/* Mixed precision: when the conjugate-gradient refinement of a solve breaks
 * down or stalls, the solve runs GMRES-IR (GMRES on the FP64 system,
 * preconditioned by the FP32 factor) before refactoring in FP64.  The GMRES
 * steps of the last solve, or -1 when it was not needed. */
int tb_chol_gmres_ir_iterations( tb_chol * h, int32_t * out );

/* ------------------------------------------------------------------------
 * Batches of independent systems (no counterpart in the reference, which
 * factors one matrix per object).  The systems become the diagonal blocks of
 * one matrix handled by a tb_chol (tb_batch_handle gives it, for setters such
 * as the precision and for statistics); its schedule defaults to level
 * launches over the merged task lists (TB_SCHEDULE_LEVELS; one persistent
 * launch for the whole batch is TB_SCHEDULE_TASK_GRAPH_ALL).  Each
 * system keeps its own pattern, permutation (NULL: identity) and values;
 * right-hand sides and solutions are per system (host calls) or the systems'
 * row-major n_s x nrhs blocks stacked in system order (device calls, row
 * offsets from tb_batch_offsets). */
typedef struct tb_batch tb_batch;
int tb_batch_create( tb_batch ** out, int32_t count, const int32_t * n, const int64_t * const * outer,
                     const int32_t * const * inner, const int32_t * const * perm, int32_t thread_count );
int tb_batch_destroy( tb_batch * b );
int tb_batch_handle( tb_batch * b, tb_chol ** out );
int tb_batch_count( tb_batch * b, int32_t * out );
/* count + 1 entries each: first row and first value of every system. */
int tb_batch_offsets( tb_batch * b, int64_t * row_offsets, int64_t * value_offsets );
int tb_batch_numeric( tb_batch * b, const double * const * values, double reg );
int tb_batch_numeric_device( tb_batch * b, const double * d_values, double reg );
/* First system whose factorization failed (-1: none). */
int tb_batch_failed_system( tb_batch * b, int32_t * out );
int tb_batch_solve( tb_batch * b, const double * const * B, double * const * X, int32_t nrhs );
int tb_batch_solve_device( tb_batch * b, const double * d_B, double * d_X, int32_t nrhs );

/* ------------------------------------------------------------------------
 * Request serving (no counterpart in the reference).  A server owns `slots`
 * worker threads on one GPU and a queue of requests over registered
 * matrices (sparsity pattern + permutation; footprint_bytes = the caller's
 * estimate of a handle's device memory, replaced by the measured size after
 * its first factorization).  Continuous batching: a free slot takes the
 * oldest queued request whose matrix is idle and whose footprint fits under
 * the HBM cap (idle resident factors are evicted least recently used first),
 * so requests arriving while others run start as soon as a slot and memory
 * are free, and requests on different matrices overlap on the device (each
 * matrix has its own stream).  A request factors (values != NULL, caller
 * order, copied at submission), solves (B, X host row-major n x nrhs, used
 * until tb_server_wait returns; refined to tol in the mixed mode), or both;
 * a solve-only request uses the resident factor, refactoring from the last
 * values if it was evicted.  precision: TB_PRECISION_MIXED or _FP64. */
typedef struct tb_server tb_server;
int tb_server_create( tb_server ** out, int device, int64_t hbm_cap_bytes, int32_t slots, int32_t precision );
int tb_server_destroy( tb_server * s );
int tb_server_add_matrix( tb_server * s, int32_t n, const int64_t * outer, const int32_t * inner, const int32_t * perm,
                          int64_t footprint_bytes, int64_t * matrix_id );
int tb_server_submit( tb_server * s, int64_t matrix_id, const double * values, double reg, const double * B, double * X,
                      int32_t nrhs, double tol, int64_t * request_id );
/* Blocks until the request is done; returns its status.  latency_ms: from
 * submission to completion; run_ms: on a slot; refinement steps / residual. */
int tb_server_wait( tb_server * s, int64_t request_id, int32_t * status, double * latency_ms, double * run_ms,
                    int32_t * iterations, double * relres );
int tb_server_stats( tb_server * s, int64_t * resident_bytes, int64_t * peak_resident_bytes, int64_t * evictions,
                     int64_t * refactors );

/* ------------------------------------------------------------------------
 * Fill-reducing ordering from the pattern alone (host only, no device
 * needed), for the constructor's permutation argument where the reference
 * calls METIS or AMD (src/Sparse/Metis.hpp:81,
 * src/Sparse/ApproximateMinimumDegree.hpp:58): George's automatic nested
 * dissection on the node graph (dofs_per_node consecutive rows form a node
 * and stay together): components split apart, rooted level structures from
 * pseudo-peripheral nodes, median-level separators ordered last, subgraphs
 * of at most leaf_size rows emitted in breadth-first order.  perm[i] is the
 * original row placed at position i (Inverse::False, as the constructor
 * takes it).  The pattern is symmetrized; a diagonal is not required.  The
 * sides of the top splits are ordered on up to thread_count threads (<= 0:
 * all host threads); the result does not depend on the thread count. */
int tb_nested_dissection( int32_t n, const int64_t * outer, const int32_t * inner, int32_t dofs_per_node,
                          int32_t leaf_size, int32_t thread_count, int32_t * perm );

/* ------------------------------------------------------------------------
 * MatrixMarket files (host only, no device needed).
 *
 * tb_matrix_market_read replaces MatrixCSR::LoadFromMatrixMarket
 * (src/Sparse/MatrixCSR/MatrixMarket.hpp:3-202) with the triple assembly it
 * calls (MatrixCSR::FromTriples, src/Sparse/MatrixCSR/FromTriples.hpp:4-209,
 * compressed and symmetrized): a coordinate file with field real, integer
 * or pattern (entries 1) and symmetry general or symmetric (the stored
 * triangle is mirrored, the diagonal kept once) becomes CSR with sorted
 * columns and repeated (i, j) entries summed in file order.  The arrays are
 * allocated by the library (rows + 1 int64 row pointers, nnz int32 columns,
 * nnz doubles) and released with tb_matrix_market_free.  thread_count <= 0:
 * all host threads.  TB_ERR_IO: unreadable file; TB_ERR_FORMAT: not a
 * supported MatrixMarket file (complex, skew-symmetric, hermitian and array
 * files included, as in the reference), an index outside the stated size,
 * or an entry count other than the size line's.
 *
 * tb_matrix_market_write replaces MatrixCSR::WriteToMatrixMarket
 * (MatrixMarket.hpp:205-306): "real general", one "%d %d %.17E" line per
 * stored entry in CSR order (a written file reads back bit-exact). */
int tb_matrix_market_read( const char * path, int32_t thread_count, int32_t * rows, int32_t * cols,
                           int64_t ** outer, int32_t ** inner, double ** values );
int tb_matrix_market_free( void * p );
int tb_matrix_market_write( const char * path, int32_t rows, int32_t cols, const int64_t * outer,
                            const int32_t * inner, const double * values );

#ifdef __cplusplus
}
#endif

#endif /* TENSORS_B200_H */
