// Kernel entry points of the FP64 supernodal factorization and solves.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "plan.hpp"

namespace tb
{

constexpr int kSolveMaxRhs = 64;   // right-hand sides per solve launch

// status[0]: bit 0 set when a pivot was not positive; status[1]: smallest
// failing (permuted) row index (initialised to INT_MAX); status[2]: pivots
// raised to their floor (mixed precision).
// T: factor storage, double (FP64 path) or float (mixed precision: FP32
// storage, 3xTF32 Schur updates, FP64 panel factorization and solves).
template<typename T>
void launch_assemble( const double * values, const std::int64_t * src, const std::int64_t * dst,
                      std::int64_t count, const double * reg, T * arena, cudaStream_t st );
template<typename T> void launch_zero( const ZeroTask * tasks, int count, T * arena, cudaStream_t st );
template<typename T>
void launch_export( const ExportTask * tasks, int count, const std::int32_t * colmap, const T * arena,
                    double * tri, double * rec, cudaStream_t st );
template<typename T> void launch_extend( const ExtendTask * tasks, int count, const std::int32_t * lut, T * arena, cudaStream_t st );
// Extend-add by parent rows (plan.hpp, ExtendPullTask): one launch per level.
template<typename T>
void launch_extend_pull( const ExtendPullTask * tasks, int count, const ExtendTask * segs, const std::int32_t * lut, T * arena,
                         cudaStream_t st );
// pivot_floor (mixed precision only, else null): element 0 the largest |a_ii|,
// element 1 + i the value a non-positive or lost pivot of permuted row i is
// raised to instead of failing; status[2] counts them.
// tinv: per panel (PanelTask::panel) the 64 x 64 inverse of its diagonal block, written here.
template<typename T> void launch_potrf( const PanelTask * tasks, int count, T * arena, int * status,
                                        const double * pivot_floor, double * tinv, cudaStream_t st );
// out (n + 1 doubles): the pivot floors in the layout of launch_potrf's pivot_floor.
void launch_pivot_floor( const std::int64_t * offsets, const float * arena, double rel, double * out, int n, cudaStream_t st );
// Uses the inverse diagonal blocks the panels' potrf wrote to tinv.  img
// (FP32 path, else null): the operand image the trsm also writes its panel
// rows into, split into TF32 hi and lo (tasks with PanelTask::img >= 0).
template<typename T> void launch_trsm( const PanelTask * tasks, int count, T * arena, const double * tinv, cudaStream_t st,
                                       float * img = nullptr );
// status[0] gets kStatusTcTimeout (2) when a tensor-core completion wait of
// the FP32 path ran out (its tile is then not updated).
template<typename T> void launch_gemm( const GemmTask * tasks, int count, T * arena, int * status, cudaStream_t st );

// The tensor map (CUtensorMap, 128 bytes) of the operand image, held by the
// host and passed to the tile kernel by value.
struct alignas(64) ImageMap { unsigned char bytes[128]; };
// Encodes the map of an operand image of `blocks` blocks at img; 0 on success.
int encode_image_map( ImageMap * out, const float * img, std::int64_t blocks );
// The FP32 path's tensor-core tiles (TcTask) of one launch: persistent CTAs,
// one per SM.  status[0] gets bit 2 when a wait of the kernel ran out.
void launch_gemm_tc_tiles( const TcTask * tasks, int count, float * arena, const ImageMap & map, int * status,
                           cudaStream_t st );
cudaError_t configure_tc_tiles();

// The numeric factorization as one persistent launch over the plan's task
// graph (Plan::dag).  counters (dag_counters ints), next and error must be
// zero before the launch; afterwards error != 0 names the task (index + 1)
// whose wait ran out of time.
struct DagArgs
{
    const DagTask * tasks;
    int ntasks;
    int * counters;
    int * next;
    int * error;
    void * arena;                 // factor storage (double or float, the launch's type)
    int * status;
    const double * pivot_floor;   // see launch_potrf
    const ZeroTask * zero;
    const ExtendTask * extend;
    const std::int32_t * lut;
    const PanelTask * potrf;
    const PanelTask * panel;
    const GemmTask * gemm;
    const SolveDiagTask * sdiag;
    double * tinv;
    unsigned long long timeout_ns;
    // optional execution trace, 4 entries per task in list order: time the
    // task was taken, its inputs were ready and it was done (%globaltimer
    // ns), and the CTA (block index) that ran it; nullptr: no trace
    unsigned long long * trace;
};
constexpr unsigned kDagMaxSpins = 1u << 26;    // bound on polls of one wait, besides the time limit
template<typename T> void launch_factor_dag( const DagArgs & args, int grid, cudaStream_t st );
// Resident CTAs per SM of the persistent kernel (0 on error).
int factor_dag_blocks_per_sm();

// One forward (upper = false) or backward solve step over `count` tasks;
// in / out row-major with leading dimension ld, k <= kSolveMaxRhs columns.
template<typename T>
void launch_solve_step( const SolveRestTask * tasks, int count, bool upper, const T * arena, const double * tinv,
                        const std::int32_t * sn_inner, double * in, double * out, int ld, int k, cudaStream_t st );

// The levels of the solve task graph as one persistent launch per sweep
// (Plan::solve_*): counters (one per graph panel), next and error zero
// before the launch; afterwards error != 0 names the list position (+ 1)
// whose wait ran out of time.
struct SolveDagArgs
{
    const SolveRestTask * tasks;          // all srest tasks
    const std::int32_t * order;           // srest indices in the sweep's order
    int ntasks;
    int upper;
    std::int64_t first_task;
    int first_panel;
    const std::int64_t * target_ptr;
    const std::int32_t * targets;
    const std::int32_t * fwd_expected;
    const std::int32_t * panel_tasks;
    int * counters;
    int * next;
    int * error;
    const double * tinv;
    const std::int32_t * sn_inner;
    unsigned long long timeout_ns;
    // optional execution trace, 4 entries per list position (as DagArgs::trace); nullptr: none
    unsigned long long * trace;
};
template<typename T>
void launch_solve_dag( const SolveDagArgs & args, int grid, const T * arena, double * in, double * out, int ld, int k,
                       cudaStream_t st );
// Resident CTAs per SM of the persistent solve kernel for k right-hand sides (0 on error).
int solve_dag_blocks_per_sm( int k );

// Super-panel solve (plan.hpp, SuperPanel): the inverses' round launches
// (after the factorization; tbuf: Plan::super_inv_size doubles), and the diag
// and rest steps of the sweeps (zbuf: n x ld doubles, zero before the back
// sweep; in / out as launch_solve_step's).
template<typename T>
void launch_super_inv( const SuperInvTask * tasks, int count, const SuperPanel * sps, const T * arena, const double * tinv,
                       double * tbuf, cudaStream_t st );
void launch_super_diag( const SuperSolveTask * tasks, int count, const SuperPanel * sps, const double * tbuf, bool upper,
                        const double * in, const double * zbuf, double * out, int ld, int k, cudaStream_t st );
template<typename T>
void launch_super_rest( const SuperSolveTask * tasks, int count, const SuperPanel * sps, const T * arena,
                        const std::int32_t * sn_inner, bool upper, double * in, double * zbuf, const double * out, int ld, int k,
                        cudaStream_t st );

// W (ldw) <- rows p[i] of B (ldB), k columns; columns k..kw-1 of W are zeroed.
void launch_gather_rows( const double * B, int ldB, const std::int32_t * p, double * W, int ldw,
                         int n, int k, cudaStream_t st, int kw = 0 );
void launch_scatter_rows( const double * W, int ldw, const std::int32_t * p_inv, double alpha, double beta,
                          double * Y, int ldY, int n, int k, cudaStream_t st );
void launch_residual( int n, const std::int64_t * outer, const std::int32_t * inner, const double * vals,
                      const double * X, const double * B, double * R, int k, cudaStream_t st );
void launch_init_status( int * status, cudaStream_t st );
// dst (n x k, leading dimension ldd) = src (leading dimension lds), converted.
void launch_widen( const float * src, int lds, double * dst, int ldd, std::int64_t n, int k, cudaStream_t st );
void launch_narrow( const double * src, int lds, float * dst, int ldd, std::int64_t n, int k, cudaStream_t st );
// R = B - (A + shift I) X, or (A + shift I) X when B is null;
// out[c] += X(:, c) . Y(:, c); the two CG updates with per-column scalars on
// the device; y += a x; Y = alpha X + beta Y.
void launch_apply_shifted( int n, const std::int64_t * outer, const std::int32_t * inner, const double * vals,
                           double shift, const double * X, int ldx, const double * B, int ldb, double * R, int ldr,
                           int k, cudaStream_t st );
void launch_column_dots( const double * X, int ldx, const double * Y, int ldy, int n, int k, double * out, cudaStream_t st );
void launch_cg_update_xr( int n, int k, const double * rz, const double * pq, const double * p, const double * q,
                          double * x, double * r, cudaStream_t st );
void launch_cg_update_p( int n, int k, const double * rz_new, const double * rz_old, const double * z, double * p,
                         cudaStream_t st );
void launch_axpy( std::int64_t n, double a, const double * x, double * y, cudaStream_t st );
// GMRES: out[i k + c] += Q_i(:, c) . q(:, c) for the nq vectors Q_i = Q + i nk;
// q += sign sum_i coef[i k + c] Q_i(:, c); x(:, c) /= sqrt(sq[c]) where sq[c] > 0.
void launch_multi_dots( const double * Q, std::int64_t nk, int nq, const double * q, int n, int k, double * out, cudaStream_t st );
void launch_multi_axpy( const double * Q, std::int64_t nk, int nq, const double * coef, double sign, double * q, int n, int k,
                        cudaStream_t st );
void launch_col_normalize( double * x, int n, int k, const double * sq, cudaStream_t st );
void launch_combine( int n, int k, double alpha, const double * X, int ldx, double beta, double * Y, int ldy, cudaStream_t st );
template<typename T>
void launch_gather_diag( const std::int64_t * offsets, const T * arena, double * out, int n, cudaStream_t st );

// Raises the dynamic shared-memory limits of the solve kernels on the
// current device; call once per device before the first launch.
cudaError_t configure_kernels();

} // namespace tb
