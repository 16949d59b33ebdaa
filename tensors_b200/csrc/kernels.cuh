// Kernel entry points of the FP64 supernodal factorization and solves.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "plan.hpp"

namespace tb
{

constexpr int kSolveMaxRhs = 64;   // right-hand sides per solve launch

// status[0]: bit 0 set when a pivot was not positive; status[1]: smallest
// failing (permuted) row index (initialised to INT_MAX).
void launch_assemble( const double * values, const std::int64_t * src, const std::int64_t * dst,
                      std::int64_t count, const double * reg, double * arena, cudaStream_t st );
void launch_zero( const ZeroTask * tasks, int count, double * arena, cudaStream_t st );
void launch_export( const ExportTask * tasks, int count, const std::int32_t * colmap, const double * arena,
                    double * tri, double * rec, cudaStream_t st );
void launch_extend( const ExtendTask * tasks, int count, const std::int32_t * lut, double * arena, cudaStream_t st );
void launch_potrf( const PanelTask * tasks, int count, double * arena, int * status, cudaStream_t st );
void launch_trsm( const PanelTask * tasks, int count, double * arena, cudaStream_t st );
void launch_gemm( const GemmTask * tasks, int count, double * arena, cudaStream_t st );

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
    double * arena;
    int * status;
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
void launch_factor_dag( const DagArgs & args, int grid, cudaStream_t st );
// Resident CTAs per SM of the persistent kernel (0 on error).
int factor_dag_blocks_per_sm();

// Inverse of every panel's diagonal block into tinv (count x 64 x 64).
void launch_invert_diag( const SolveDiagTask * tasks, int count, const double * arena, double * tinv, cudaStream_t st );
// One forward (upper = false) or backward solve step over `count` tasks;
// in / out row-major with leading dimension ld, k <= kSolveMaxRhs columns.
void launch_solve_step( const SolveRestTask * tasks, int count, bool upper, const double * arena, const double * tinv,
                        const std::int32_t * sn_inner, double * in, double * out, int ld, int k, cudaStream_t st );

void launch_gather_rows( const double * B, int ldB, const std::int32_t * p, double * W, int ldw,
                         int n, int k, cudaStream_t st );
void launch_scatter_rows( const double * W, int ldw, const std::int32_t * p_inv, double alpha, double beta,
                          double * Y, int ldY, int n, int k, cudaStream_t st );
void launch_residual( int n, const std::int64_t * outer, const std::int32_t * inner, const double * vals,
                      const double * X, const double * B, double * R, int k, cudaStream_t st );
void launch_init_status( int * status, cudaStream_t st );
void launch_gather_diag( const std::int64_t * offsets, const double * arena, double * out, int n, cudaStream_t st );

// Raises the dynamic shared-memory limits of the solve kernels on the
// current device; call once per device before the first launch.
cudaError_t configure_kernels();

} // namespace tb
