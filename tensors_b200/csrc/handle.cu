// C-ABI of the library (include/tensors_b200.h): handle lifetime, device
// memory, launch sequencing and CUDA-graph capture of the factorization.

#include "common.hpp"
#include "kernels.cuh"
#include "parallel.hpp"
#include "plan.hpp"
#include "plan_check.hpp"
#include "schedule.hpp"
#include "symbolic.hpp"
#include "trace.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <utility>
#include <climits>
#include <limits>
#include <map>
#include <mutex>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace
{

thread_local std::string g_error = "no error";
int g_device = 0;
// Bound on one dependency wait of the persistent factorization kernel.
constexpr unsigned long long kDagTimeoutNs = 2000000000ull;
// Mixed precision: a pivot is raised to this fraction of its row's assembled diagonal entry.
constexpr double kPivotFloorRel = 1e-5;

int fail( int code, const std::string & msg )
{
    g_error = msg;
    return code;
}

} // namespace

void tb::set_last_error( const std::string & msg ) { g_error = msg; }

namespace
{

#define TB_CUDA( call )                                                                              \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if( e_ != cudaSuccess )                                                                      \
        {                                                                                            \
            return fail( e_ == cudaErrorMemoryAllocation ? TB_ERR_OUT_OF_MEMORY : TB_ERR_CUDA,        \
                         std::string( #call ) + ": " + cudaGetErrorString( e_ ) );                   \
        }                                                                                            \
    } while( 0 )

#define TB_TRY( call )                         \
    do {                                       \
        const int s_ = (call);                 \
        if( s_ != TB_OK ) { return s_; }       \
    } while( 0 )

template<typename T>
struct DeviceArray
{
    T * ptr = nullptr;
    std::int64_t size = 0;
    ~DeviceArray() { release(); }
    void release() { if( ptr ) { cudaFree( ptr ); ptr = nullptr; } size = 0; }
    int reserve( std::int64_t n )
    {
        if( n <= size && ptr ) { return TB_OK; }
        release();
        TB_CUDA( cudaMalloc( &ptr, sizeof(T) * static_cast<size_t>( std::max<std::int64_t>( n, 1 ) ) ) );
        size = n;
        return TB_OK;
    }
    int upload( const std::vector<T> & v, cudaStream_t st )
    {
        TB_TRY( reserve( static_cast<std::int64_t>( v.size() ) ) );
        if( !v.empty() ) { TB_CUDA( cudaMemcpyAsync( ptr, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st ) ); }
        return TB_OK;
    }
};

struct PinnedBuffer
{
    void * ptr = nullptr;
    size_t bytes = 0;
    ~PinnedBuffer() { if( ptr ) { cudaFreeHost( ptr ); } }
    int reserve( size_t n )
    {
        if( n <= bytes && ptr ) { return TB_OK; }
        if( ptr ) { cudaFreeHost( ptr ); ptr = nullptr; }
        TB_CUDA( cudaMallocHost( &ptr, std::max<size_t>( n, 64 ) ) );
        bytes = n;
        return TB_OK;
    }
    template<typename T> T * as() { return static_cast<T*>( ptr ); }
};

} // namespace

struct tb_chol
{
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // second stream of the level schedule: the GEMM tiles of a panel step that
    // do not touch the next panel run there, overlapping the next potrf / trsm
    cudaStream_t side = nullptr;
    cudaEvent_t ev_trsm = nullptr, ev_rest = nullptr;

    // input pattern (copied, CholeskyDecomposition.hpp:313-371)
    std::int32_t n = 0;
    std::vector<std::int64_t> outer;
    std::vector<std::int32_t> inner;
    std::vector<std::int32_t> perm;
    bool has_perm = false;
    std::int32_t threads = 1;

    tb::SupernodeStrategy strategy = tb::SupernodeStrategy::Maximal;
    std::int32_t amalgamation_threshold = 4;
    std::int32_t method = TB_MULTIFRONTAL;

    bool symbolic_done = false;
    // plan options (tb_chol_set_plan_options): trailing-update deferral, front
    // relaxation preset, widest tensor-core tile; plan_dirty: rebuild the plan
    std::int32_t opt_defer = tb::kDeferSteps, opt_relax = 1, opt_tc_width = tb::kTcNMax;
    bool plan_dirty = false;
    std::int64_t analyze_us = 0, plan_us = 0;   // host time of the last symbolic analysis and plan build
    bool device_ready = false;
    bool kernels_configured = false;
    tb::Symbolic sym;
    tb::Plan plan;

    // device state
    DeviceArray<double>             arena;       // factor storage: doubles, or floats in the mixed-precision mode
    DeviceArray<std::int64_t>       asm_src, asm_dst, diag_off;
    DeviceArray<std::int32_t>       lut, sn_inner, p, p_inv, colmap;
    DeviceArray<tb::ZeroTask>       zero;
    DeviceArray<tb::ExportTask>     exports;
    DeviceArray<double>             exported;    // reference-layout factor (tri then rec)
    DeviceArray<tb::GemmTask>       gemm;
    DeviceArray<tb::TcTask>         tc;          // mixed precision: the GEMM updates as tensor-core tiles
    DeviceArray<float>              img;         // mixed precision: the tiles' operand image (TF32 hi / lo)
    tb::ImageMap                    img_map{};   // its tensor map
    DeviceArray<tb::PanelTask>      potrf, panel;
    DeviceArray<tb::ExtendTask>     extend;
    DeviceArray<tb::ExtendPullTask> extend_pull;
    DeviceArray<tb::ExtendTask>     extend_segs;
    DeviceArray<tb::SolveDiagTask>  sdiag;
    DeviceArray<tb::SolveRestTask>  srest;
    DeviceArray<tb::SuperPanel>     spanels;     // super-panel solve of the large fronts (Plan::spanels)
    DeviceArray<tb::SuperInvTask>   sinv;
    DeviceArray<tb::SuperSolveTask> ssolve;
    DeviceArray<double>             tsuper;      // their 512 x 512 inverses
    DeviceArray<std::int64_t>       a_outer;     // caller-order pattern, for residuals
    DeviceArray<std::int32_t>       a_inner;
    DeviceArray<double>             values;      // caller-order values of the last factorization
    DeviceArray<double>             reg;
    DeviceArray<int>                status;
    DeviceArray<double>             work, work2, work3, in, out, diag_vals;   // work3: the super-panel back sweep's sums
    DeviceArray<double>             tinv;        // inverse diagonal block of every panel (64 x 64 each)
    DeviceArray<tb::DagTask>        dag;         // the factorization as one dependency-ordered task list
    DeviceArray<int>                dag_state;   // task-graph counters, then the ticket and the error word
    // the solve's task graph (Plan::solve_*): orders, targets, expected counts,
    // and per-panel counters followed by the ticket and the error word
    DeviceArray<std::int32_t>       solve_fwd_order, solve_bwd_order, solve_targets, solve_fwd_expected, solve_panel_tasks;
    DeviceArray<std::int64_t>       solve_target_ptr;
    DeviceArray<int>                solve_state;
    PinnedBuffer                    pin_solve_err;   // error word of the last sweeps (list position + 1)
    std::map<int, int>              solve_grid;      // CTAs of the persistent solve launch per right-hand-side count
    DeviceArray<unsigned long long> solve_trace_buf; // with `trace`: forward then back sweep of the first RHS chunk
    int solve_schedule = TB_SCHEDULE_LEVELS;
    int dag_grid = 0;                            // CTAs of the persistent factorization launch
    bool use_dag = false;                        // persistent task-graph launch (else one launch per step)
    int schedule = TB_SCHEDULE_LEVELS;
    int precision = TB_PRECISION_FP64;
    double last_reg = 0.0;
    // iterative refinement of the mixed-precision solves
    double ir_tol = 1e-12;
    std::int32_t ir_max = 30;
    std::int32_t ir_iters = 0;
    double ir_relres = 0.0;
    std::int32_t gmres_iters = -1;               // GMRES-IR steps of the last refined solve (-1: not used)
    DeviceArray<double> ir_x, ir_r, ir_norms;
    DeviceArray<double> cg_buf, cg_scal, cg_host;   // tb_chol_cg: vectors, per-column scalars, host-call copies
    DeviceArray<double> gm_buf, gm_scal;            // GMRES: Krylov basis and work vectors, per-column scalars
    PinnedBuffer pin_gm;
    DeviceArray<double> pivot_floor;             // mixed precision: static-pivot floor per row
    std::int32_t perturbed_pivots = 0;
    bool fell_back = false;                      // a mixed solve's refinement failed: refactored in FP64
    PinnedBuffer pin_norms;
    bool trace = false;                          // record the persistent launch's execution trace
    DeviceArray<unsigned long long> trace_buf;
    PinnedBuffer                    pin_in, pin_out, pin_small;

    cudaGraphExec_t factor_graph = nullptr;
    bool use_graph = true;
    // captured solve sweeps on the work buffers, keyed by (which, nrhs)
    std::map<std::pair<int,int>, cudaGraphExec_t> solve_graphs;
    double * solve_graph_work = nullptr;
    double * solve_graph_work2 = nullptr;
    double * solve_graph_work3 = nullptr;

    // optional per-kernel timing of direct (non-graph) factorizations
    bool profiling = false;
    double kind_ms[8] = {};
    std::int64_t kind_launches[8] = {};
    std::vector<cudaEvent_t> events;
    std::vector<cudaEvent_t> chunk_events;   // host solves: completion of each chunk copied back
    std::vector<float> launch_ms;          // per factor launch of the last profiled run (0 = clear + assembly)
    std::vector<cudaEvent_t> solve_events;
    std::vector<std::int64_t> solve_info;  // per solve launch of the last profiled solve: upper, level, step, tasks
    std::vector<float> solve_ms;

    bool factorized = false;
    bool good = false;
    std::int32_t failed_sn = -1;
    std::int64_t factor_launch_count = 0;
    std::int64_t solve_launch_count = 0;
    std::int64_t solve_sweep_launches = 0;

    void drop_solve_graphs()
    {
        for( auto & kv : solve_graphs ) { cudaGraphExecDestroy( kv.second ); }
        solve_graphs.clear();
        solve_graph_work = nullptr;
        solve_graph_work2 = nullptr;
        solve_graph_work3 = nullptr;
    }

    ~tb_chol()
    {
        for( cudaEvent_t e : events ) { cudaEventDestroy( e ); }
        for( cudaEvent_t e : chunk_events ) { cudaEventDestroy( e ); }
        for( cudaEvent_t e : solve_events ) { cudaEventDestroy( e ); }
        drop_solve_graphs();
        if( factor_graph ) { cudaGraphExecDestroy( factor_graph ); }
        if( own_stream && stream ) { cudaStreamDestroy( stream ); }
        if( side ) { cudaStreamDestroy( side ); }
        if( ev_trsm ) { cudaEventDestroy( ev_trsm ); }
        if( ev_rest ) { cudaEventDestroy( ev_rest ); }
    }

    void invalidate_symbolic()
    {
        symbolic_done = false;
        device_ready = false;
        factorized = false;
        good = false;
        if( factor_graph ) { cudaGraphExecDestroy( factor_graph ); factor_graph = nullptr; }
        drop_solve_graphs();
    }
};

namespace
{

int check_handle( tb_chol * h )
{
    if( h == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null handle" ); }
    return TB_OK;
}

// The plan options' relaxation presets: tight, default (CHOLMOD-like), loose.
tb::Relaxation relaxation_preset( std::int32_t which )
{
    tb::Relaxation r;
    if( which == 0 ) { r.nrelax[0] = 4;  r.nrelax[1] = 16; r.nrelax[2] = 32;  r.zrelax[0] = 0.8; r.zrelax[1] = 0.1; r.zrelax[2] = 0.05; }
    if( which == 2 ) { r.nrelax[0] = 16; r.nrelax[1] = 48; r.nrelax[2] = 128; r.zrelax[0] = 0.9; r.zrelax[1] = 0.3; r.zrelax[2] = 0.15; }
    return r;
}

// Builds the device plan of the symbolic analysis with the handle's plan options.
void build_plan( tb_chol * h )
{
    tb::TraceRange plan_range( "tensors_b200::DevicePlan" );
    h->plan.dag_min_steps = h->schedule == TB_SCHEDULE_TASK_GRAPH_ALL ? 0 : tb::kDagMinSteps;
    h->plan.defer_steps = h->opt_defer;
    h->plan.tc_nmax = h->opt_tc_width;
    h->plan.relax = relaxation_preset( h->opt_relax );
    h->plan.threads = h->threads;
    h->plan.build( h->sym );
    if( h->solve_schedule == TB_SCHEDULE_LEVELS ) { h->plan.build_solve_graph( h->sym, h->plan.levels ); }
    else if( h->solve_schedule == TB_SCHEDULE_TASK_GRAPH_ALL ) { h->plan.build_solve_graph( h->sym, 0 ); }
    h->plan_dirty = false;
}

int ensure_symbolic( tb_chol * h )
{
    if( h->symbolic_done && h->plan_dirty )
    {
        // new plan options: the symbolic analysis stands, the device plan is rebuilt
        const auto t1 = std::chrono::steady_clock::now();
        build_plan( h );
        h->plan_us = std::chrono::duration_cast<std::chrono::microseconds>( std::chrono::steady_clock::now() - t1 ).count();
        h->device_ready = false;
        h->factorized = false;
        h->good = false;
        return TB_OK;
    }
    if( h->symbolic_done ) { return TB_OK; }
    tb::SymbolicInput in;
    in.n = h->n;
    in.outer = h->outer.data();
    in.inner = h->inner.data();
    in.perm = h->has_perm ? h->perm.data() : nullptr;
    in.strategy = h->strategy;
    in.amalgamation_threshold = h->amalgamation_threshold;
    in.threads = h->threads;
    tb::TraceRange range( "Sparse::CholeskyDecomposition::SymbolicFactorization" );
    const auto t0 = std::chrono::steady_clock::now();
    const int st = h->sym.analyze( in );
    const auto t1 = std::chrono::steady_clock::now();
    if( st != TB_OK )
    {
        const char * what = st == TB_ERR_INVALID_PERMUTATION ? "input is not a permutation"
                          : st == TB_ERR_MISSING_DIAGONAL    ? "diagonal of input matrix is not marked as nonzero"
                          : "invalid CSR pattern";
        return fail( st, std::string( "SymbolicFactorization: " ) + what );
    }
    build_plan( h );
    const auto t2 = std::chrono::steady_clock::now();
    h->analyze_us = std::chrono::duration_cast<std::chrono::microseconds>( t1 - t0 ).count();
    h->plan_us = std::chrono::duration_cast<std::chrono::microseconds>( t2 - t1 ).count();
    h->symbolic_done = true;
    h->device_ready = false;
    h->factorized = false;
    h->good = false;
    return TB_OK;
}

// Binds the handle's device and stream and uploads the plan (once per
// symbolic analysis).  Everything before this point is host-only, so the
// symbolic phase and its getters work without a GPU.
int ensure_device( tb_chol * h )
{
    TB_TRY( ensure_symbolic( h ) );
    TB_CUDA( cudaSetDevice( h->device ) );
    if( h->stream == nullptr )
    {
        TB_CUDA( cudaStreamCreateWithFlags( &h->stream, cudaStreamNonBlocking ) );
        h->own_stream = true;
    }
    if( h->side == nullptr )
    {
        TB_CUDA( cudaStreamCreateWithFlags( &h->side, cudaStreamNonBlocking ) );
        TB_CUDA( cudaEventCreateWithFlags( &h->ev_trsm, cudaEventDisableTiming ) );
        TB_CUDA( cudaEventCreateWithFlags( &h->ev_rest, cudaEventDisableTiming ) );
    }
    if( !h->kernels_configured )
    {
        TB_CUDA( tb::configure_kernels() );
        TB_CUDA( tb::configure_tc_tiles() );
        h->kernels_configured = true;
    }
    if( h->device_ready ) { return TB_OK; }
    {
        // the persistent launch's CTA count, and the task order for it
        int sms = 0;
        TB_CUDA( cudaDeviceGetAttribute( &sms, cudaDevAttrMultiProcessorCount, h->device ) );
        const int per_sm = tb::factor_dag_blocks_per_sm();
        if( per_sm <= 0 ) { return fail( TB_ERR_CUDA, "persistent factorization kernel cannot be resident" ); }
        h->dag_grid = static_cast<int>( std::min<std::int64_t>( static_cast<std::int64_t>( per_sm ) * sms,
                                                                static_cast<std::int64_t>( h->plan.dag.size() ) ) );
        tb::schedule_task_graph( h->plan, h->dag_grid );
    }
    {
        const std::string msg = tb::check_plan( h->sym, h->plan );
        if( !msg.empty() ) { return fail( TB_ERR_INVALID_ARGUMENT, "plan check: " + msg ); }
    }

    const tb::Symbolic & s = h->sym;
    const tb::Plan & pl = h->plan;
    cudaStream_t st_ = h->stream;
    TB_TRY( h->arena.reserve( h->precision == TB_PRECISION_MIXED ? (pl.arena_size() + 1) / 2 : pl.arena_size() ) );
    TB_TRY( h->asm_src.upload( pl.asm_src, st_ ) );
    TB_TRY( h->asm_dst.upload( pl.asm_dst, st_ ) );
    TB_TRY( h->lut.upload( pl.lut, st_ ) );
    TB_TRY( h->sn_inner.upload( s.sn_inner, st_ ) );
    TB_TRY( h->p.upload( s.p, st_ ) );
    TB_TRY( h->p_inv.upload( s.p_inv, st_ ) );
    TB_TRY( h->gemm.upload( pl.gemm, st_ ) );
    TB_TRY( h->potrf.upload( pl.potrf, st_ ) );
    TB_TRY( h->panel.upload( pl.panel, st_ ) );
    TB_TRY( h->extend.upload( pl.extend, st_ ) );
    TB_TRY( h->extend_pull.upload( pl.extend_pull, st_ ) );
    TB_TRY( h->extend_segs.upload( pl.extend_segs, st_ ) );
    TB_TRY( h->sdiag.upload( pl.sdiag, st_ ) );
    TB_TRY( h->srest.upload( pl.srest, st_ ) );
    TB_TRY( h->spanels.upload( pl.spanels, st_ ) );
    TB_TRY( h->sinv.upload( pl.sinv, st_ ) );
    TB_TRY( h->ssolve.upload( pl.ssolve, st_ ) );
    if( pl.super_inv_size > 0 ) { TB_TRY( h->tsuper.reserve( pl.super_inv_size ) ); }
    TB_TRY( h->zero.upload( pl.zero, st_ ) );
    TB_TRY( h->exports.upload( pl.exports, st_ ) );
    TB_TRY( h->colmap.upload( pl.colmap, st_ ) );
    TB_TRY( h->a_outer.upload( h->outer, st_ ) );
    TB_TRY( h->a_inner.upload( h->inner, st_ ) );
    TB_TRY( h->values.reserve( s.nnz ) );
    TB_TRY( h->reg.reserve( 1 ) );
    TB_TRY( h->status.reserve( 3 ) );
    TB_TRY( h->diag_off.upload( pl.diag_offset, st_ ) );
    TB_TRY( h->diag_vals.reserve( s.n ) );
    if( h->precision == TB_PRECISION_MIXED )
    {
        TB_TRY( h->pivot_floor.reserve( static_cast<std::int64_t>( s.n ) + 1 ) );
        TB_TRY( h->tc.upload( pl.tc, st_ ) );
        if( pl.img_blocks > 0 )
        {
            TB_TRY( h->img.reserve( pl.img_blocks * tb::kImgRows * tb::kImgK ) );
            const int e = tb::encode_image_map( &h->img_map, h->img.ptr, pl.img_blocks );
            if( e != 0 ) { return fail( TB_ERR_CUDA, "encoding the operand image's tensor map failed (" + std::to_string( e ) + ")" ); }
        }
    }
    TB_TRY( h->tinv.reserve( static_cast<std::int64_t>( pl.sdiag.size() ) * tb::kPanel * tb::kPanel ) );
    TB_TRY( h->dag.upload( pl.dag, st_ ) );
    TB_TRY( h->dag_state.reserve( static_cast<std::int64_t>( pl.dag_counters ) + 2 ) );
    TB_TRY( h->solve_fwd_order.upload( pl.solve_fwd_order, st_ ) );
    TB_TRY( h->solve_bwd_order.upload( pl.solve_bwd_order, st_ ) );
    TB_TRY( h->solve_targets.upload( pl.solve_targets, st_ ) );
    TB_TRY( h->solve_fwd_expected.upload( pl.solve_fwd_expected, st_ ) );
    TB_TRY( h->solve_panel_tasks.upload( pl.solve_panel_tasks, st_ ) );
    TB_TRY( h->solve_target_ptr.upload( pl.solve_target_ptr, st_ ) );
    TB_TRY( h->solve_state.reserve( static_cast<std::int64_t>( pl.solve_panel_tasks.size() ) + 2 ) );
    TB_TRY( h->pin_solve_err.reserve( 64 ) );
    *h->pin_solve_err.as<int>() = 0;
    h->solve_grid.clear();
    TB_CUDA( cudaStreamSynchronize( st_ ) );
    if( h->factor_graph ) { cudaGraphExecDestroy( h->factor_graph ); h->factor_graph = nullptr; }
    h->drop_solve_graphs();
    h->device_ready = true;
    return TB_OK;
}

template<typename T> T * arena_as( tb_chol * h ) { return reinterpret_cast<T *>( h->arena.ptr ); }

// One GEMM launch of the level schedule.  FP64: its 64 x 64 DMMA tiles.
// FP32: the 64 x 64 tiles of the fronts without an operand image (the launch's
// first small_count tiles), then the tensor-core tiles of the others.
template<typename T>
void issue_gemm( tb_chol * h, const tb::Launch & L, T * A, cudaStream_t s )
{
    if constexpr ( sizeof(T) == 8 )
    {
        tb::launch_gemm( h->gemm.ptr + L.first, L.count, A, h->status.ptr, s );
    }
    else
    {
        tb::launch_gemm( h->gemm.ptr + L.first, L.small_count, A, h->status.ptr, s );
        tb::launch_gemm_tc_tiles( h->tc.ptr + L.tc_first, L.tc_count, A, h->img_map, h->status.ptr, s );
    }
}

// Issues the numeric factorization on h->stream (capturable).  With
// `timed`, every launch is bracketed by events (kind index in `kinds`).
template<typename T>
std::int64_t issue_factor_t( tb_chol * h, bool timed, std::vector<int> * kinds )
{
    const tb::Plan & pl = h->plan;
    cudaStream_t st = h->stream;
    T * A = arena_as<T>( h );
    float * img = (sizeof(T) == 4 && h->img.ptr != nullptr) ? h->img.ptr : nullptr;
    std::int64_t launches = 0;
    std::size_t ev = 0;
    auto mark = [&]( int kind )
    {
        if( !timed ) { return; }
        cudaEventRecord( h->events[ev++], st );
        if( kind >= 0 ) { kinds->push_back( kind ); }
    };
    mark( -1 );
    {
        // ClearFactors (Numeric.hpp:256-268); update matrices are zeroed per level
        tb::TraceRange range( "Sparse::CholeskyDecomposition::ClearFactors" );
        cudaMemsetAsync( A, 0, sizeof(T) * static_cast<size_t>( pl.u0_size + pl.u1_size ), st );
        tb::launch_init_status( h->status.ptr, st );
    }
    {
        tb::TraceRange range( "Sparse::CholeskyDecomposition::ReadNonzeroValues" );
        tb::launch_assemble( h->values.ptr, h->asm_src.ptr, h->asm_dst.ptr,
                             static_cast<std::int64_t>( pl.asm_src.size() ), h->reg.ptr, A, st );
    }
    const double * floor = nullptr;
    if constexpr ( sizeof(T) == 4 )
    {
        tb::launch_pivot_floor( h->diag_off.ptr, A, kPivotFloorRel, h->pivot_floor.ptr, h->n, st );
        floor = h->pivot_floor.ptr;
        ++launches;
    }
    mark( 7 );
    launches += 2;
    if( h->use_dag && !timed )
    {
        for( const tb::Launch & L : pl.pre_dag_launches )
        {
            switch( L.kind )
            {
                case tb::LaunchKind::Zero:   tb::launch_zero( h->zero.ptr + L.first, L.count, A, st ); break;
                case tb::LaunchKind::Extend: tb::launch_extend( h->extend.ptr + L.first, L.count, h->lut.ptr, A, st ); break;
                case tb::LaunchKind::ExtendPull:
                    tb::launch_extend_pull( h->extend_pull.ptr + L.first, L.count, h->extend_segs.ptr, h->lut.ptr, A, st );
                    break;
                case tb::LaunchKind::Potrf:  tb::launch_potrf( h->potrf.ptr + L.first, L.count, A, h->status.ptr, floor, h->tinv.ptr, st ); break;
                case tb::LaunchKind::Trsm:   tb::launch_trsm( h->panel.ptr + L.first, L.count, A, h->tinv.ptr, st, img ); break;
                case tb::LaunchKind::Gemm:   issue_gemm( h, L, A, st ); break;
                default: break;
            }
            ++launches;
        }
        const int nc = pl.dag_counters;
        cudaMemsetAsync( h->dag_state.ptr, 0, sizeof(int) * (static_cast<size_t>( nc ) + 2), st );
        tb::DagArgs a{};
        a.tasks = h->dag.ptr; a.ntasks = static_cast<int>( pl.dag.size() );
        a.counters = h->dag_state.ptr; a.next = h->dag_state.ptr + nc; a.error = h->dag_state.ptr + nc + 1;
        a.arena = A; a.status = h->status.ptr; a.pivot_floor = floor;
        a.zero = h->zero.ptr; a.extend = h->extend.ptr; a.lut = h->lut.ptr;
        a.potrf = h->potrf.ptr; a.panel = h->panel.ptr; a.gemm = h->gemm.ptr;
        a.sdiag = h->sdiag.ptr; a.tinv = h->tinv.ptr;
        a.timeout_ns = kDagTimeoutNs;
        a.trace = h->trace ? h->trace_buf.ptr : nullptr;
        tb::launch_factor_dag<T>( a, h->dag_grid, st );
        launches += pl.dag.empty() ? 0 : 1;
        for( const tb::Launch & L : pl.sinv_launches )
        {
            tb::launch_super_inv( h->sinv.ptr + L.first, L.count, h->spanels.ptr, A, h->tinv.ptr, h->tsuper.ptr, st );
            ++launches;
        }
        return launches;
    }
    // One panel of look-ahead over two streams (the profiled path keeps one,
    // so that every launch is timed alone).  Main stream: potrf(q), trsm(q),
    // the tiles of step q that update panel q+1's rows (part 0).  Side
    // stream: the other tiles of step q (part 1), after trsm(q); they run
    // while potrf(q+1) and trsm(q+1) do.  Part 0 of step q waits for part 1
    // of step q-1 (both update panel q+1's rows), which also orders
    // potrf(q+1) after every update of its block; each C tile keeps the order
    // of its updates, so the factor is the same bit for bit.
    // Levels join the side stream at their boundaries (the next extend-adds
    // read the update matrices the part-1 tiles write).
    const bool overlap = !timed && h->side != nullptr;
    bool side_busy = false;
    std::int32_t level = -1;
    auto join = [&]()
    {
        if( !side_busy ) { return; }
        cudaEventRecord( h->ev_rest, h->side );
        cudaStreamWaitEvent( st, h->ev_rest, 0 );
        side_busy = false;
    };
    for( const tb::Launch & L : pl.factor_launches )
    {
        cudaStream_t s = st;
        if( overlap )
        {
            if( L.level != level ) { join(); level = L.level; }
            if( L.kind == tb::LaunchKind::Gemm )
            {
                if( L.part == 0 ) { join(); }
                else
                {
                    cudaStreamWaitEvent( h->side, h->ev_trsm, 0 );
                    s = h->side;
                    side_busy = true;
                }
            }
        }
        switch( L.kind )
        {
            case tb::LaunchKind::Zero:   tb::launch_zero( h->zero.ptr + L.first, L.count, A, s ); break;
            case tb::LaunchKind::Extend: tb::launch_extend( h->extend.ptr + L.first, L.count, h->lut.ptr, A, s ); break;
            case tb::LaunchKind::ExtendPull:
                tb::launch_extend_pull( h->extend_pull.ptr + L.first, L.count, h->extend_segs.ptr, h->lut.ptr, A, s );
                break;
            case tb::LaunchKind::Potrf:  tb::launch_potrf( h->potrf.ptr + L.first, L.count, A, h->status.ptr, floor, h->tinv.ptr, s ); break;
            case tb::LaunchKind::Trsm:   tb::launch_trsm( h->panel.ptr + L.first, L.count, A, h->tinv.ptr, s, img ); break;
            case tb::LaunchKind::Gemm:   issue_gemm( h, L, A, s ); break;
            default: break;
        }
        if( overlap && L.kind == tb::LaunchKind::Trsm ) { cudaEventRecord( h->ev_trsm, st ); }
        mark( static_cast<int>( L.kind == tb::LaunchKind::ExtendPull ? tb::LaunchKind::Extend : L.kind ) );
        ++launches;
    }
    if( overlap ) { join(); }
    // the large fronts' super-panel inverses for the solves (after every panel inverse exists)
    for( const tb::Launch & L : pl.sinv_launches )
    {
        tb::launch_super_inv( h->sinv.ptr + L.first, L.count, h->spanels.ptr, A, h->tinv.ptr, h->tsuper.ptr, st );
        mark( static_cast<int>( tb::LaunchKind::Invert ) );
        ++launches;
    }
    return launches;
}

std::int64_t issue_factor( tb_chol * h, bool timed = false, std::vector<int> * kinds = nullptr )
{
    return h->precision == TB_PRECISION_MIXED ? issue_factor_t<float>( h, timed, kinds )
                                              : issue_factor_t<double>( h, timed, kinds );
}

int run_factor( tb_chol * h, double reg )
{
    tb::TraceRange range( "Sparse::CholeskyDecomposition::NumericFactorization_Multifrontal" );
    cudaStream_t st = h->stream;
    TB_TRY( h->pin_small.reserve( 64 ) );
    double * pr = h->pin_small.as<double>();
    pr[0] = reg;
    h->last_reg = reg;
    TB_CUDA( cudaMemcpyAsync( h->reg.ptr, pr, sizeof(double), cudaMemcpyHostToDevice, st ) );
    if( h->profiling )
    {
        const std::size_t need = h->plan.factor_launches.size() + h->plan.sinv_launches.size() + 2;
        while( h->events.size() < need )
        {
            cudaEvent_t e;
            TB_CUDA( cudaEventCreate( &e ) );
            h->events.push_back( e );
        }
        std::vector<int> kinds;
        h->factor_launch_count = issue_factor( h, true, &kinds );
        TB_CUDA( cudaGetLastError() );
        TB_CUDA( cudaStreamSynchronize( st ) );
        for( int k = 0; k < 8; ++k ) { h->kind_ms[k] = 0.0; h->kind_launches[k] = 0; }
        h->launch_ms.assign( kinds.size(), 0.0f );
        for( std::size_t i = 0; i < kinds.size(); ++i )
        {
            float ms = 0.0f;
            TB_CUDA( cudaEventElapsedTime( &ms, h->events[i], h->events[i + 1] ) );
            h->kind_ms[kinds[i]] += ms;
            h->kind_launches[kinds[i]] += 1;
            h->launch_ms[i] = ms;
        }
    }
    else if( h->use_graph )
    {
        if( h->factor_graph == nullptr )
        {
            cudaGraph_t g = nullptr;
            TB_CUDA( cudaStreamBeginCapture( st, cudaStreamCaptureModeThreadLocal ) );
            h->factor_launch_count = issue_factor( h );
            const cudaError_t ce = cudaStreamEndCapture( st, &g );
            if( ce != cudaSuccess ) { return fail( TB_ERR_CUDA, std::string( "graph capture: " ) + cudaGetErrorString( ce ) ); }
            const cudaError_t ie = cudaGraphInstantiate( &h->factor_graph, g, 0 );
            cudaGraphDestroy( g );
            if( ie != cudaSuccess ) { h->factor_graph = nullptr; return fail( TB_ERR_CUDA, std::string( "graph instantiate: " ) + cudaGetErrorString( ie ) ); }
        }
        TB_CUDA( cudaGraphLaunch( h->factor_graph, st ) );
    }
    else
    {
        h->factor_launch_count = issue_factor( h );
        TB_CUDA( cudaGetLastError() );
    }
    int * ps = reinterpret_cast<int*>( pr + 1 );
    ps[3] = 0;
    TB_CUDA( cudaMemcpyAsync( ps, h->status.ptr, 3 * sizeof(int), cudaMemcpyDeviceToHost, st ) );
    if( h->use_dag && !h->profiling )
    {
        TB_CUDA( cudaMemcpyAsync( ps + 3, h->dag_state.ptr + h->plan.dag_counters + 1, sizeof(int), cudaMemcpyDeviceToHost, st ) );
    }
    TB_CUDA( cudaStreamSynchronize( st ) );
    h->perturbed_pivots = ps[2];
    if( ps[0] & 2 )
    {
        h->factorized = false;
        h->good = false;
        return fail( TB_ERR_TIMEOUT, "NumericFactorization: a tensor-core completion wait ran out of time" );
    }
    if( ps[3] != 0 )
    {
        h->factorized = false;
        h->good = false;
        return fail( TB_ERR_TIMEOUT, "NumericFactorization: persistent launch stopped, the wait of task "
                     + std::to_string( ps[3] - 1 ) + " ran out of time" );
    }
    h->factorized = true;                       // marked in any case, Numeric.hpp:94-95
    h->good = (ps[0] & 1) == 0;
    h->failed_sn = h->good ? -1 : h->sym.row_to_sn[std::min( std::max( ps[1], 0 ), h->n - 1 )];
    if( !h->good )
    {
        g_error = "NumericFactorization: matrix is not (sufficiently) positive-definite; first failing supernode "
                  + std::to_string( h->failed_sn );
        return TB_NOT_SPD;
    }
    return TB_OK;
}

int require_factor( tb_chol * h )
{
    if( h->factorized ) { TB_CUDA( cudaSetDevice( h->device ) ); }
    if( !h->factorized ) { return fail( TB_ERR_NOT_FACTORIZED, "Solve: nonzero values of matrix have not been passed, yet" ); }
    if( !h->good ) { return fail( TB_ERR_NOT_FACTORIZED, "Solve: numerical factorization was not successful" ); }
    return TB_OK;
}

// Issues the forward (which != 1) and back (which != 0) sweeps over two
// permuted n x k blocks (leading dimension k); capturable.  The right-hand
// side is expected in W for which 0 and 2 and in Y for which 1; the result
// is left in sweep_result( which, W, Y ).  The back sweep accumulates into W,
// which it clears first.
// With `timed`, every launch is bracketed by the handle's solve events and
// described in solve_info (the events must exist).
// levels_only: every level as a step launch, whatever the solve schedule (no
// persistent launch, so no wait that can run out of time).
std::int64_t issue_sweeps( tb_chol * h, int which, double * W, double * Y, std::int32_t k, bool timed = false,
                           bool levels_only = false )
{
    const tb::Plan & pl = h->plan;
    cudaStream_t st = h->stream;
    std::int64_t launches = 0;
    std::size_t ev = 0;
    auto begin = [&]() { if( timed ) { cudaEventRecord( h->solve_events[ev++], st ); } };
    auto end = [&]( std::int32_t level, std::int32_t step, std::int32_t count, int upper )
    {
        if( !timed ) { return; }
        cudaEventRecord( h->solve_events[ev++], st );
        h->solve_info.insert( h->solve_info.end(), { upper, level, step, count } );
    };
    if( timed ) { h->solve_info.clear(); }
    const bool mixed = h->precision == TB_PRECISION_MIXED;
    // the levels from solve_split_level up: one persistent launch per sweep
    bool graph = !levels_only && !pl.solve_fwd_order.empty();
    for( std::int32_t c0 = 0; c0 < k && graph; c0 += tb::kSolveMaxRhs )
    {
        const auto it = h->solve_grid.find( std::min( tb::kSolveMaxRhs, k - c0 ) );
        graph = it != h->solve_grid.end() && it->second > 0;
    }
    const std::int32_t split = graph ? pl.solve_split_level : pl.levels;
    // the large fronts step by super-panels when every level runs as launches
    const bool super = !graph && !levels_only && !pl.spanels.empty() && h->work3.ptr != nullptr;
    const std::vector<tb::Launch> & lower = super ? pl.lower_launches_sp : pl.lower_launches;
    const std::vector<tb::Launch> & upper_list = super ? pl.upper_launches_sp : pl.upper_launches;
    double * Z = h->work3.ptr;
    const std::int32_t np = static_cast<std::int32_t>( pl.solve_panel_tasks.size() );
    int * err = h->solve_state.ptr + np + 1;
    if( graph ) { cudaMemsetAsync( err, 0, sizeof(int), st ); }
    auto step = [&]( const tb::Launch & L, bool upper, double * in, double * out, std::int32_t kc, std::int32_t c0 )
    {
        begin();
        if( L.kind == tb::LaunchKind::SuperDiag )
        {
            tb::launch_super_diag( h->ssolve.ptr + L.first, L.count, h->spanels.ptr, h->tsuper.ptr, upper, in, Z + c0, out, k, kc, st );
        }
        else if( L.kind == tb::LaunchKind::SuperRest )
        {
            if( mixed ) { tb::launch_super_rest( h->ssolve.ptr + L.first, L.count, h->spanels.ptr, arena_as<float>( h ), h->sn_inner.ptr,
                                                 upper, in, Z + c0, out, k, kc, st ); }
            else        { tb::launch_super_rest( h->ssolve.ptr + L.first, L.count, h->spanels.ptr, arena_as<double>( h ), h->sn_inner.ptr,
                                                 upper, in, Z + c0, out, k, kc, st ); }
        }
        else if( mixed )
        {
            tb::launch_solve_step( h->srest.ptr + L.first, L.count, upper, arena_as<float>( h ), h->tinv.ptr,
                                   h->sn_inner.ptr, in, out, k, kc, st );
        }
        else
        {
            tb::launch_solve_step( h->srest.ptr + L.first, L.count, upper, arena_as<double>( h ), h->tinv.ptr,
                                   h->sn_inner.ptr, in, out, k, kc, st );
        }
        end( L.level, L.step, L.count, upper ? 1 : 0 );
        ++launches;
    };
    auto persistent = [&]( bool upper, double * in, double * out, std::int32_t kc, std::int32_t c0 )
    {
        cudaMemsetAsync( h->solve_state.ptr, 0, sizeof(int) * (static_cast<size_t>( np ) + 1), st );
        tb::SolveDagArgs a{};
        a.tasks = h->srest.ptr;
        a.order = upper ? h->solve_bwd_order.ptr : h->solve_fwd_order.ptr;
        a.ntasks = static_cast<int>( pl.solve_fwd_order.size() );
        a.upper = upper ? 1 : 0;
        a.first_task = pl.solve_first_task;
        a.first_panel = pl.solve_first_panel;
        a.target_ptr = h->solve_target_ptr.ptr;
        a.targets = h->solve_targets.ptr;
        a.fwd_expected = h->solve_fwd_expected.ptr;
        a.panel_tasks = h->solve_panel_tasks.ptr;
        a.counters = h->solve_state.ptr;
        a.next = h->solve_state.ptr + np;
        a.error = err;
        a.tinv = h->tinv.ptr;
        a.sn_inner = h->sn_inner.ptr;
        a.timeout_ns = kDagTimeoutNs;
        a.trace = (h->trace && h->solve_trace_buf.ptr && c0 == 0)
                ? h->solve_trace_buf.ptr + (upper ? 4 * static_cast<std::int64_t>( a.ntasks ) : 0) : nullptr;
        const int grid = h->solve_grid.at( kc );
        begin();
        if( mixed ) { tb::launch_solve_dag( a, grid, arena_as<float>( h ), in, out, k, kc, st ); }
        else        { tb::launch_solve_dag( a, grid, arena_as<double>( h ), in, out, k, kc, st ); }
        end( split, -1, a.ntasks, upper ? 1 : 0 );
        ++launches;
    };
    if( which != 1 )
    {
        tb::TraceRange range( "Sparse::CholeskyDecomposition::SN_LowerSolve" );
        // the super-panels' diag steps add their block pairs into zeroed rows
        if( super ) { cudaMemsetAsync( Y, 0, sizeof(double) * static_cast<size_t>( h->n ) * k, st ); }
        for( std::int32_t c0 = 0; c0 < k; c0 += tb::kSolveMaxRhs )
        {
            const std::int32_t kc = std::min( tb::kSolveMaxRhs, k - c0 );
            for( const tb::Launch & L : lower ) { if( L.level < split ) { step( L, false, W + c0, Y + c0, kc, c0 ); } }
            if( graph ) { persistent( false, W + c0, Y + c0, kc, c0 ); }
        }
    }
    if( which != 0 )
    {
        tb::TraceRange range( "Sparse::CholeskyDecomposition::SN_UpperSolve" );
        cudaMemsetAsync( W, 0, sizeof(double) * static_cast<size_t>( h->n ) * k, st );
        if( super ) { cudaMemsetAsync( Z, 0, sizeof(double) * static_cast<size_t>( h->n ) * k, st ); }
        for( std::int32_t c0 = 0; c0 < k; c0 += tb::kSolveMaxRhs )
        {
            const std::int32_t kc = std::min( tb::kSolveMaxRhs, k - c0 );
            if( graph ) { persistent( true, Y + c0, W + c0, kc, c0 ); }
            for( const tb::Launch & L : upper_list ) { if( L.level < split ) { step( L, true, Y + c0, W + c0, kc, c0 ); } }
        }
    }
    if( graph ) { cudaMemcpyAsync( h->pin_solve_err.ptr, err, sizeof(int), cudaMemcpyDeviceToHost, st ); }
    return launches;
}

// CTAs of the persistent solve launch for every right-hand-side chunk width
// of k (before the sweeps are issued or captured).
int prepare_solve_grid( tb_chol * h, std::int32_t k )
{
    if( h->plan.solve_fwd_order.empty() ) { return TB_OK; }
    int sms = 0;
    TB_CUDA( cudaDeviceGetAttribute( &sms, cudaDevAttrMultiProcessorCount, h->device ) );
    for( std::int32_t c0 = 0; c0 < k; c0 += tb::kSolveMaxRhs )
    {
        const std::int32_t kc = std::min( tb::kSolveMaxRhs, k - c0 );
        if( h->solve_grid.count( kc ) ) { continue; }
        const int per_sm = tb::solve_dag_blocks_per_sm( kc );
        if( per_sm <= 0 ) { return fail( TB_ERR_CUDA, "persistent solve kernel cannot be resident" ); }
        h->solve_grid[kc] = static_cast<int>( std::min<std::int64_t>( static_cast<std::int64_t>( per_sm ) * sms,
                                                                       static_cast<std::int64_t>( h->plan.solve_fwd_order.size() ) ) );
    }
    return TB_OK;
}

// After a synchronization: a wait of the persistent solve launch that ran out
// of time (the result is then wrong).
int check_solve_error( tb_chol * h )
{
    if( h->pin_solve_err.ptr == nullptr ) { return TB_OK; }
    int & e = *h->pin_solve_err.as<int>();
    if( e == 0 ) { return TB_OK; }
    const int pos = e - 1;
    e = 0;
    return fail( TB_ERR_TIMEOUT, "Solve: persistent solve launch stopped, the wait of list position " + std::to_string( pos )
                 + " ran out of time" );
}

// Right-hand-side columns a buffer is reserved for when nrhs are needed: the
// width class (8, 16, 32, 64; wider: as given), so that calls with varying
// nrhs regrow (free and reallocate, which waits for the whole device) at most
// once per class.
std::int64_t rhs_capacity( std::int32_t nrhs )
{
    return nrhs <= 8 ? 8 : nrhs <= 16 ? 16 : nrhs <= 32 ? 32 : nrhs <= tb::kSolveMaxRhs ? tb::kSolveMaxRhs : nrhs;
}

double * sweep_input( int which, double * W, double * Y ) { return which == 1 ? Y : W; }
double * sweep_result( int which, double * W, double * Y ) { return which == 0 ? Y : W; }

// which: 0 lower only, 1 upper only, 2 both.  d_B (ldB) -> d_X (ldX), device.
// The gather (ReadRightHandSide) and scatter (WriteSolution) run as direct
// launches; the sweeps are captured once per (which, nrhs) into a CUDA graph
// over the handle's work buffers.
int run_solve_core( tb_chol * h, int which, double alpha, const double * d_B, std::int32_t ldB,
                    double beta, double * d_X, std::int32_t ldX, std::int32_t nrhs )
{
    cudaStream_t st = h->stream;
    const std::int32_t n = h->n;
    const std::int32_t kb = std::max( 1, nrhs );
    if( ldB < kb || ldX < kb ) { return fail( TB_ERR_INVALID_ARGUMENT, "Solve: leading dimension smaller than nrhs" ); }
    // The sweeps run on the width class of nrhs (8, 16, 32 or 64 columns; wider: as given), the
    // extra columns zero: the kernels compute that many columns in any case, every column's
    // result depends on that column alone, and one captured graph and one set of work buffers
    // then serve every nrhs of the class instead of one per nrhs.
    const std::int32_t k = static_cast<std::int32_t>( rhs_capacity( kb ) );
    TB_TRY( h->work.reserve( static_cast<std::int64_t>(n) * k ) );
    TB_TRY( h->work2.reserve( static_cast<std::int64_t>(n) * k ) );
    if( !h->plan.spanels.empty() ) { TB_TRY( h->work3.reserve( static_cast<std::int64_t>(n) * k ) ); }
    double * W = h->work.ptr;
    double * Y = h->work2.ptr;
    if( h->solve_graph_work != W || h->solve_graph_work2 != Y || h->solve_graph_work3 != h->work3.ptr )
    {
        h->drop_solve_graphs();
        h->solve_graph_work = W;
        h->solve_graph_work2 = Y;
        h->solve_graph_work3 = h->work3.ptr;
    }
    TB_TRY( prepare_solve_grid( h, k ) );
    std::int64_t launches = 0;
    tb::launch_gather_rows( d_B, ldB, h->p.ptr, sweep_input( which, W, Y ), k, n, kb, st, k );   // ReadRightHandSide
    ++launches;
    if( h->use_graph && !h->profiling )
    {
        cudaGraphExec_t & g = h->solve_graphs[{ which, k }];
        if( g == nullptr )
        {
            cudaGraph_t graph = nullptr;
            TB_CUDA( cudaStreamBeginCapture( st, cudaStreamCaptureModeThreadLocal ) );
            h->solve_sweep_launches = issue_sweeps( h, which, W, Y, k );
            const cudaError_t ce = cudaStreamEndCapture( st, &graph );
            if( ce != cudaSuccess ) { h->solve_graphs.erase( { which, k } ); return fail( TB_ERR_CUDA, std::string( "graph capture: " ) + cudaGetErrorString( ce ) ); }
            const cudaError_t ie = cudaGraphInstantiate( &g, graph, 0 );
            cudaGraphDestroy( graph );
            if( ie != cudaSuccess ) { h->solve_graphs.erase( { which, k } ); return fail( TB_ERR_CUDA, std::string( "graph instantiate: " ) + cudaGetErrorString( ie ) ); }
        }
        TB_CUDA( cudaGraphLaunch( g, st ) );
        launches += h->solve_sweep_launches;
    }
    else if( h->profiling )
    {
        const std::int32_t chunks = (k + tb::kSolveMaxRhs - 1) / tb::kSolveMaxRhs;
        const std::size_t need = 2 * static_cast<std::size_t>( chunks )
                               * std::max( h->plan.lower_launches.size() + h->plan.upper_launches.size(),
                                           h->plan.lower_launches_sp.size() + h->plan.upper_launches_sp.size() );
        while( h->solve_events.size() < need )
        {
            cudaEvent_t e;
            TB_CUDA( cudaEventCreate( &e ) );
            h->solve_events.push_back( e );
        }
        launches += issue_sweeps( h, which, W, Y, k, true );
        TB_CUDA( cudaStreamSynchronize( st ) );
        h->solve_ms.clear();
        for( std::size_t i = 0; i < h->solve_info.size() / 4; ++i )
        {
            float ms = 0.0f;
            TB_CUDA( cudaEventElapsedTime( &ms, h->solve_events[2 * i], h->solve_events[2 * i + 1] ) );
            h->solve_ms.push_back( ms );
        }
    }
    else
    {
        launches += issue_sweeps( h, which, W, Y, k );
    }
    tb::launch_scatter_rows( sweep_result( which, W, Y ), k, h->p_inv.ptr, alpha, beta, d_X, ldX, n, kb, st );   // WriteSolution
    ++launches;
    h->solve_launch_count = launches;
    TB_CUDA( cudaGetLastError() );
    return TB_OK;
}

// Mixed-precision solve: conjugate gradients in FP64 on (A + reg I) x = b
// (the matrix of the last factorization), preconditioned by the FP32 factor
// F ~ A + reg I, one independent recurrence per right-hand side, started
// from x0 = F^{-1} b.  With an accurate factor this is iterative refinement
// that converges in a few steps; unlike plain refinement it still converges
// when cond(A) * eps_fp32 is not small.  Stops when
// max_c |r_c| / |b_c| <= tol or after the iteration cap.  Per-column scalars
// stay on the device; the residual norms are read back once per iteration.
int run_solve_refined( tb_chol * h, double alpha, const double * d_B, std::int32_t ldB,
                       double beta, double * d_X, std::int32_t ldX, std::int32_t nrhs );

// The refinement of a mixed solve failed (FP32 rounding is too coarse for
// the matrix: kappa far above 1 / eps_fp32): refactor the same matrix in FP64
// from the values the handle holds on the device and run the same conjugate
// gradients with the FP64 factor as the preconditioner.  The handle stays in
// FP64 until the precision is set again (tb_chol_precision_in_use tells).
int solve_fp64_fallback( tb_chol * h, double alpha, const double * d_B, std::int32_t ldB,
                         double beta, double * d_X, std::int32_t ldX, std::int32_t nrhs )
{
    h->precision = TB_PRECISION_FP64;
    h->fell_back = true;
    h->device_ready = false;
    if( h->factor_graph ) { cudaGraphExecDestroy( h->factor_graph ); h->factor_graph = nullptr; }
    h->drop_solve_graphs();
    TB_TRY( ensure_device( h ) );
    const int fs = run_factor( h, h->last_reg );
    if( fs != TB_OK )
    {
        return fail( fs < 0 ? fs : TB_ERR_NOT_CONVERGED, "Solve: mixed-precision refinement failed and the FP64 "
                     "refactorization did not succeed: " + g_error );
    }
    return run_solve_refined( h, alpha, d_B, ldB, beta, d_X, ldX, nrhs );
}

// Restarted GMRES preconditioned from the left by the handle's factor: the
// reference's GMRES::operator() (GMRES.hpp:124-330, Solve :333-485,
// ArnoldiStep :529-590 with two Gram-Schmidt passes, Givens rotations
// :592-655, CheckResiduals :802-818), one Krylov space per right-hand side
// column, vectors on the device, the small Hessenberg systems on the host.
// Operator: (A' + shift I) with values `vals` (caller order).  sol (n x k,
// packed) holds the initial guess when use_x0 and receives the solution.
// Stops when every column's preconditioned residual |P (b - A x)| is at most
// rel_tol |P b| (the reference's TOL) or after max_restarts restarts of m
// Arnoldi steps.  relres (k entries) gets |P r| / |P b| per column.
struct GmresOutcome
{
    std::int32_t iterations = 0, restarts = 0;
    bool converged = false;
};

int run_gmres( tb_chol * h, const double * vals, double shift, const double * d_B, std::int32_t ldB, std::int32_t k,
               double * sol, bool use_x0, double rel_tol, std::int32_t m, std::int32_t max_restarts, double * relres,
               GmresOutcome & out )
{
    tb::TraceRange range( "GMRES::operator()" );
    const std::int32_t n = h->n;
    cudaStream_t st = h->stream;
    m = std::max<std::int32_t>( 1, std::min<std::int32_t>( m, n ) );
    const std::int64_t nk = static_cast<std::int64_t>( n ) * k;
    TB_TRY( h->gm_buf.reserve( (static_cast<std::int64_t>( m ) + 2) * nk ) );        // Q_0..Q_m, z
    TB_TRY( h->gm_scal.reserve( (2 * (static_cast<std::int64_t>( m ) + 1) + 2) * k ) ); // two dot passes, |q|^2, |Pb|^2
    const size_t hcount = static_cast<size_t>( 2 * (m + 1) + 2 ) * static_cast<size_t>( k );
    TB_TRY( h->pin_gm.reserve( sizeof(double) * hcount ) );
    double * Q = h->gm_buf.ptr;
    double * z = Q + (static_cast<std::int64_t>( m ) + 1) * nk;
    double * hd = h->gm_scal.ptr;                                   // [2][m+1][k]
    double * qsq = hd + 2 * (static_cast<std::int64_t>( m ) + 1) * k;
    double * bsq = qsq + k;
    double * hp = h->pin_gm.as<double>();
    auto precondition = [&]( const double * in, std::int32_t ld, double * o ) -> int {
        return run_solve_core( h, 2, 1.0, in, ld, 0.0, o, k, k );
    };
    auto sqnorms = [&]( const double * x, double * o ) -> int {
        TB_CUDA( cudaMemsetAsync( o, 0, sizeof(double) * static_cast<size_t>( k ), st ) );
        tb::launch_column_dots( x, k, x, k, n, k, o, st );
        return TB_OK;
    };
    auto fetch = [&]( const double * d, size_t count ) -> int {
        TB_CUDA( cudaMemcpyAsync( hp, d, sizeof(double) * count, cudaMemcpyDeviceToHost, st ) );
        TB_CUDA( cudaStreamSynchronize( st ) );
        return check_solve_error( h );
    };

    // |P b| per column: the tolerance reference (GMRES.hpp:174-186)
    TB_TRY( precondition( d_B, ldB, z ) );
    TB_TRY( sqnorms( z, bsq ) );
    TB_TRY( fetch( bsq, static_cast<size_t>( k ) ) );
    std::vector<double> tol( static_cast<size_t>( k ) ), bn( static_cast<size_t>( k ) );
    double bmax = 0.0;
    for( std::int32_t c = 0; c < k; ++c )
    {
        if( std::isnan( hp[c] ) ) { return fail( TB_ERR_INVALID_ARGUMENT, "GMRES: right-hand side contains NaNs" ); }
        bn[static_cast<size_t>( c )] = std::sqrt( hp[c] );
        tol[static_cast<size_t>( c )] = rel_tol * bn[static_cast<size_t>( c )];
        bmax = std::max( bmax, bn[static_cast<size_t>( c )] );
    }
    if( !(bmax > 0.0) )
    {
        TB_CUDA( cudaMemsetAsync( sol, 0, sizeof(double) * static_cast<size_t>( nk ), st ) );
        for( std::int32_t c = 0; c < k; ++c ) { relres[c] = 0.0; }
        out.converged = true;
        return TB_OK;
    }
    const size_t mk = static_cast<size_t>( m );
    std::vector<double> H( (mk + 1) * mk * static_cast<size_t>( k ) ), cs( mk * k ), sn( mk * k ), beta( (mk + 1) * k );
    auto Hat = [&]( size_t i, size_t j, std::int32_t c ) -> double & { return H[(i * mk + j) * k + static_cast<size_t>( c )]; };
    bool first = true;
    for( std::int32_t restart = 0; restart <= max_restarts; ++restart )
    {
        // r = b - A x (x = 0 at a start without a guess); Q_0 = P r / |P r|
        if( first && !use_x0 )
        {
            // x = 0: P r = P b, which z still holds
            TB_CUDA( cudaMemsetAsync( sol, 0, sizeof(double) * static_cast<size_t>( nk ), st ) );
            TB_CUDA( cudaMemcpyAsync( Q, z, sizeof(double) * static_cast<size_t>( nk ), cudaMemcpyDeviceToDevice, st ) );
        }
        else
        {
            tb::launch_apply_shifted( n, h->a_outer.ptr, h->a_inner.ptr, vals, shift, sol, k, d_B, ldB, z, k, k, st );
            TB_TRY( precondition( z, k, Q ) );
        }
        first = false;
        TB_TRY( sqnorms( Q, qsq ) );
        tb::launch_col_normalize( Q, n, k, qsq, st );
        TB_TRY( fetch( qsq, static_cast<size_t>( k ) ) );
        std::fill( H.begin(), H.end(), 0.0 );
        std::fill( beta.begin(), beta.end(), 0.0 );
        bool succ = true;
        for( std::int32_t c = 0; c < k; ++c )
        {
            beta[static_cast<size_t>( c )] = std::sqrt( hp[c] );
            succ = succ && beta[static_cast<size_t>( c )] <= tol[static_cast<size_t>( c )];
        }
        std::int32_t iter = 0;
        while( !succ && iter < m )
        {
            double * qn = Q + (static_cast<std::int64_t>( iter ) + 1) * nk;
            tb::launch_apply_shifted( n, h->a_outer.ptr, h->a_inner.ptr, vals, shift, Q + static_cast<std::int64_t>( iter ) * nk,
                                      k, nullptr, k, z, k, k, st );                      // z = A Q_iter
            TB_TRY( precondition( z, k, qn ) );                                          // Q_iter+1 = P A Q_iter
            for( int g = 0; g < 2; ++g )
            {
                // classical Gram-Schmidt against Q_0..Q_iter, twice
                double * hg = hd + static_cast<std::int64_t>( g ) * (static_cast<std::int64_t>( m ) + 1) * k;
                TB_CUDA( cudaMemsetAsync( hg, 0, sizeof(double) * static_cast<size_t>( iter + 1 ) * k, st ) );
                tb::launch_multi_dots( Q, nk, iter + 1, qn, n, k, hg, st );
                tb::launch_multi_axpy( Q, nk, iter + 1, hg, -1.0, qn, n, k, st );
            }
            TB_TRY( sqnorms( qn, qsq ) );
            tb::launch_col_normalize( qn, n, k, qsq, st );
            // both passes' coefficients and |q|^2 to the host: hp = [pass 0][pass 1][|q|^2]
            const size_t it = static_cast<size_t>( iter );
            TB_CUDA( cudaMemcpyAsync( hp, hd, sizeof(double) * (it + 1) * k, cudaMemcpyDeviceToHost, st ) );
            TB_CUDA( cudaMemcpyAsync( hp + (it + 1) * k, hd + (static_cast<std::int64_t>( m ) + 1) * k,
                                      sizeof(double) * (it + 1) * k, cudaMemcpyDeviceToHost, st ) );
            TB_CUDA( cudaMemcpyAsync( hp + 2 * (it + 1) * k, qsq, sizeof(double) * static_cast<size_t>( k ), cudaMemcpyDeviceToHost, st ) );
            TB_CUDA( cudaStreamSynchronize( st ) );
            TB_TRY( check_solve_error( h ) );
            for( std::int32_t c = 0; c < k; ++c )
            {
                const size_t cc = static_cast<size_t>( c );
                for( size_t i = 0; i <= it; ++i ) { Hat( i, it, c ) = hp[i * k + cc] + hp[(it + 1 + i) * k + cc]; }
                Hat( it + 1, it, c ) = std::sqrt( std::max( hp[2 * (it + 1) * k + cc], 0.0 ) );
                // Givens rotations (GMRES.hpp:592-655)
                for( size_t i = 0; i < it; ++i )
                {
                    const double xi = Hat( i, it, c ), eta = Hat( i + 1, it, c );
                    const double co = cs[i * k + cc], si = sn[i * k + cc];
                    Hat( i, it, c ) = co * xi + si * eta;
                    Hat( i + 1, it, c ) = -si * xi + co * eta;
                }
                const double xi = Hat( it, it, c ), eta = Hat( it + 1, it, c );
                const double r = std::sqrt( xi * xi + eta * eta );
                double co, si;
                if( std::abs( xi ) <= std::numeric_limits<double>::epsilon() * r ) { co = 0.0; si = 1.0; }
                else { co = std::abs( xi ) / r; si = (xi / std::abs( xi )) * eta / r; }
                cs[it * k + cc] = co;
                sn[it * k + cc] = si;
                Hat( it, it, c ) = co * xi + si * eta;
                Hat( it + 1, it, c ) = 0.0;
                beta[(it + 1) * k + cc] = -si * beta[it * k + cc];
                beta[it * k + cc] = co * beta[it * k + cc];
            }
            ++iter;
            succ = true;
            for( std::int32_t c = 0; c < k; ++c )
            {
                succ = succ && std::abs( beta[static_cast<size_t>( iter ) * k + static_cast<size_t>( c )] ) <= tol[static_cast<size_t>( c )];
            }
        }
        // least squares: H y = beta (upper triangular, iter x iter), then x += Q y
        if( iter > 0 )
        {
            std::vector<double> y( static_cast<size_t>( iter ) * k );
            for( std::int32_t c = 0; c < k; ++c )
            {
                const size_t cc = static_cast<size_t>( c );
                for( std::int32_t i = iter - 1; i >= 0; --i )
                {
                    double v = beta[static_cast<size_t>( i ) * k + cc];
                    for( std::int32_t j = i + 1; j < iter; ++j ) { v -= Hat( static_cast<size_t>( i ), static_cast<size_t>( j ), c ) * y[static_cast<size_t>( j ) * k + cc]; }
                    const double d = Hat( static_cast<size_t>( i ), static_cast<size_t>( i ), c );
                    y[static_cast<size_t>( i ) * k + cc] = d != 0.0 ? v / d : 0.0;
                }
            }
            std::copy( y.begin(), y.end(), hp );
            TB_CUDA( cudaMemcpyAsync( hd, hp, sizeof(double) * y.size(), cudaMemcpyHostToDevice, st ) );
            tb::launch_multi_axpy( Q, nk, iter, hd, 1.0, sol, n, k, st );
            TB_CUDA( cudaStreamSynchronize( st ) );          // hp is reused by the next restart
        }
        out.iterations += iter;
        out.restarts = restart;
        for( std::int32_t c = 0; c < k; ++c )
        {
            const size_t cc = static_cast<size_t>( c );
            relres[c] = bn[cc] > 0.0 ? std::abs( beta[static_cast<size_t>( iter ) * k + cc] ) / bn[cc] : 0.0;
        }
        if( succ ) { out.converged = true; break; }
    }
    TB_CUDA( cudaGetLastError() );
    return TB_OK;
}

int run_solve_refined( tb_chol * h, double alpha, const double * d_B, std::int32_t ldB,
                       double beta, double * d_X, std::int32_t ldX, std::int32_t nrhs )
{
    tb::TraceRange range( "tensors_b200::Refinement" );
    cudaStream_t st = h->stream;
    const std::int32_t n = h->n;
    const std::int32_t k = std::max( 1, nrhs );
    if( ldB < k || ldX < k ) { return fail( TB_ERR_INVALID_ARGUMENT, "Solve: leading dimension smaller than nrhs" ); }
    const std::int64_t nk = static_cast<std::int64_t>( n ) * k;
    const std::int64_t kcap = rhs_capacity( k );
    TB_TRY( h->ir_x.reserve( 4 * n * kcap ) );         // x, r, z (and q), p
    TB_TRY( h->ir_r.reserve( n * kcap ) );
    TB_TRY( h->ir_norms.reserve( 5 * kcap ) );         // |r|^2, |b|^2, rz, rz_new, pq
    TB_TRY( h->pin_norms.reserve( sizeof(double) * 2 * static_cast<size_t>( kcap ) ) );
    double * hn = h->pin_norms.as<double>();
    double * X = h->ir_x.ptr;
    double * P = X + nk;
    double * Z = X + 2 * nk;
    double * Q = X + 3 * nk;
    double * R = h->ir_r.ptr;
    double * rr = h->ir_norms.ptr;
    double * bb = rr + k;
    double * rz = rr + 2 * k;
    double * rz_new = rr + 3 * k;
    double * pq = rr + 4 * k;
    const double shift = h->last_reg;
    std::int64_t launches = 0;
    auto apply = [&]( const double * x, const double * b, double * out ) {
        tb::launch_apply_shifted( n, h->a_outer.ptr, h->a_inner.ptr, h->values.ptr, shift, x, k, b, b == d_B ? ldB : k, out, k, k, st );
        ++launches;
    };
    auto dots = [&]( const double * x, int ldx, const double * y, int ldy, double * out ) -> int {
        TB_CUDA( cudaMemsetAsync( out, 0, sizeof(double) * static_cast<size_t>( k ), st ) );
        tb::launch_column_dots( x, ldx, y, ldy, n, k, out, st );
        ++launches;
        return TB_OK;
    };
    auto precondition = [&]( const double * in, double * out ) -> int {
        TB_TRY( run_solve_core( h, 2, 1.0, in, k, 0.0, out, k, k ) );
        launches += h->solve_launch_count;
        return TB_OK;
    };

    h->gmres_iters = -1;
    TB_TRY( dots( d_B, ldB, d_B, ldB, bb ) );
    TB_TRY( run_solve_core( h, 2, 1.0, d_B, ldB, 0.0, X, k, k ) );   // x0 = F^{-1} b
    launches += h->solve_launch_count;
    apply( X, d_B, R );                                             // r = b - A x
    h->ir_iters = 0;
    bool restart = true, verified = true, broke_down = false;
    double rel0 = 0.0;
    for( std::int32_t it = 0;; ++it )
    {
        TB_TRY( dots( R, k, R, k, rr ) );
        TB_CUDA( cudaMemcpyAsync( hn, rr, sizeof(double) * 2 * static_cast<size_t>( k ), cudaMemcpyDeviceToHost, st ) );
        TB_CUDA( cudaStreamSynchronize( st ) );
        TB_TRY( check_solve_error( h ) );
        double rel = 0.0;
        for( std::int32_t c = 0; c < k; ++c )
        {
            const double bn = std::sqrt( hn[k + c] ), rn = std::sqrt( hn[c] );
            const double v = bn > 0.0 ? rn / bn : rn;
            if( !(v <= rel) ) { rel = v; }              // a NaN residual propagates (std::max would drop it)
        }
        h->ir_relres = rel;
        if( it == 0 ) { rel0 = rel; }
        // breakdown: a non-finite residual, or one grown far beyond the first
        // (the FP32 factor is no preconditioner for this matrix)
        if( !std::isfinite( rel ) || rel > 1e6 * rel0 ) { broke_down = true; break; }
        if( it >= h->ir_max ) { break; }
        if( rel <= h->ir_tol )
        {
            // the recurrence r -= a q drifts from b - A x in finite precision:
            // accept only when the true residual meets the target as well
            if( verified ) { break; }
            apply( X, d_B, R );
            verified = true;
            restart = true;
            continue;
        }
        verified = false;
        TB_TRY( precondition( R, Z ) );                             // z = F^{-1} r
        if( restart )
        {
            TB_TRY( dots( R, k, Z, k, rz ) );
            TB_CUDA( cudaMemcpyAsync( P, Z, sizeof(double) * static_cast<size_t>( nk ), cudaMemcpyDeviceToDevice, st ) );
            restart = false;
        }
        else
        {
            TB_TRY( dots( R, k, Z, k, rz_new ) );
            tb::launch_cg_update_p( n, k, rz_new, rz, Z, P, st );   // p = z + (rz_new / rz) p
            TB_CUDA( cudaMemcpyAsync( rz, rz_new, sizeof(double) * static_cast<size_t>( k ), cudaMemcpyDeviceToDevice, st ) );
            ++launches;
        }
        apply( P, nullptr, Q );                                     // q = A p
        TB_TRY( dots( P, k, Q, k, pq ) );
        tb::launch_cg_update_xr( n, k, rz, pq, P, Q, X, R, st );    // x += a p, r -= a q
        ++launches;
        ++h->ir_iters;
    }
    if( (broke_down || !(h->ir_relres <= h->ir_tol)) && h->precision == TB_PRECISION_MIXED )
    {
        // GMRES-IR (Carson & Higham 2018): GMRES on the FP64 system, preconditioned by the same
        // FP32 factor, from the refinement's iterate (from zero if that broke down); accepted when
        // the true residual meets the target, else the matrix is refactored in FP64
        std::vector<double> rel( static_cast<size_t>( k ) );
        GmresOutcome go;
        // (its stopping rule bounds the preconditioned residual: a tenth of the target leaves room for the true one)
        const int gst = run_gmres( h, h->values.ptr, shift, d_B, ldB, k, X, !broke_down, 0.1 * h->ir_tol, 30, 3, rel.data(), go );
        if( gst == TB_OK )
        {
            apply( X, d_B, R );
            TB_TRY( dots( R, k, R, k, rr ) );
            TB_CUDA( cudaMemcpyAsync( hn, rr, sizeof(double) * 2 * static_cast<size_t>( k ), cudaMemcpyDeviceToHost, st ) );
            TB_CUDA( cudaStreamSynchronize( st ) );
            double rel_true = 0.0;
            for( std::int32_t c = 0; c < k; ++c )
            {
                const double bn = std::sqrt( hn[k + c] ), rn = std::sqrt( hn[c] );
                const double v = bn > 0.0 ? rn / bn : rn;
                if( !(v <= rel_true) ) { rel_true = v; }
            }
            h->gmres_iters = go.iterations;
            if( rel_true <= h->ir_tol )
            {
                h->ir_relres = rel_true;
                tb::launch_combine( n, k, alpha, X, k, beta, d_X, ldX, st );
                h->solve_launch_count = launches + 1;
                TB_CUDA( cudaGetLastError() );
                return TB_OK;
            }
        }
        return solve_fp64_fallback( h, alpha, d_B, ldB, beta, d_X, ldX, nrhs );
    }
    if( broke_down )
    {
        return fail( TB_ERR_NOT_CONVERGED, "Solve: refinement broke down (non-finite or diverging residual)" );
    }
    tb::launch_combine( n, k, alpha, X, k, beta, d_X, ldX, st );
    h->solve_launch_count = launches + 1;
    TB_CUDA( cudaGetLastError() );
    if( !(h->ir_relres <= h->ir_tol) )
    {
        char msg[160];
        std::snprintf( msg, sizeof(msg), "Solve: refinement stopped at relative residual %.3e after %d steps (target %.3e)",
                       h->ir_relres, static_cast<int>( h->ir_iters ), h->ir_tol );
        return fail( TB_ERR_NOT_CONVERGED, msg );
    }
    return TB_OK;
}

int run_solve_device( tb_chol * h, int which, double alpha, const double * d_B, std::int32_t ldB,
                      double beta, double * d_X, std::int32_t ldX, std::int32_t nrhs )
{
    tb::TraceRange range( which == 2 ? "Sparse::CholeskyDecomposition::Solve"
                        : which == 1 ? "Sparse::CholeskyDecomposition::UpperSolve" : "Sparse::CholeskyDecomposition::LowerSolve" );
    // refined: mixed precision, and a handle that fell back to FP64 from it (its target still holds)
    if( (h->precision == TB_PRECISION_MIXED || h->fell_back) && which == 2 )
    {
        return run_solve_refined( h, alpha, d_B, ldB, beta, d_X, ldX, nrhs );
    }
    return run_solve_core( h, which, alpha, d_B, ldB, beta, d_X, ldX, nrhs );
}

// Host-buffer solve through pinned staging buffers.
// Host buffers of either scalar type (the reference casts on copy,
// Solve.hpp:20-27, ReadNonzeroValues Numeric.hpp:165-180).
int dtype_size( std::int32_t dtype ) { return dtype == TB_F32 ? 4 : dtype == TB_F64 ? 8 : 0; }

// body(b, e) over rows [0, n) on up to 16 host threads, one per MB of copy.
template<typename Body>
void host_rows( std::int64_t n, std::int64_t row_bytes, Body && body )
{
    const std::int64_t total = n * std::max<std::int64_t>( row_bytes, 1 );
    const unsigned hw = std::max( 1u, std::thread::hardware_concurrency() );
    const std::int64_t threads = std::min<std::int64_t>( std::min<std::int64_t>( hw, 16 ), std::max<std::int64_t>( 1, total >> 20 ) );
    if( threads <= 1 || n < 2 ) { body( std::int64_t( 0 ), n ); return; }
    std::vector<std::thread> pool;
    for( std::int64_t t = 0; t < threads; ++t )
    {
        const std::int64_t b = n * t / threads, e = n * (t + 1) / threads;
        pool.emplace_back( [&body, b, e]() { body( b, e ); } );
    }
    for( auto & th : pool ) { th.join(); }
}

// Packed n x k doubles <- caller rows of type dtype (leading dimension ld).
void stage_rows_in( double * dst, const void * src, std::int32_t dtype, std::int64_t n, std::int32_t k, std::int32_t ld )
{
    host_rows( n, static_cast<std::int64_t>( k ) * 8, [&]( std::int64_t b, std::int64_t e )
    {
        if( dtype == TB_F64 )
        {
            const double * s = static_cast<const double *>( src );
            if( ld == k ) { std::memcpy( dst + b * k, s + b * k, sizeof(double) * static_cast<size_t>( (e - b) * k ) ); return; }
            for( std::int64_t i = b; i < e; ++i ) { std::memcpy( dst + i * k, s + i * ld, sizeof(double) * static_cast<size_t>( k ) ); }
        }
        else
        {
            const float * s = static_cast<const float *>( src );
            for( std::int64_t i = b; i < e; ++i )
            {
                for( std::int32_t c = 0; c < k; ++c ) { dst[i * k + c] = static_cast<double>( s[i * ld + c] ); }
            }
        }
    } );
}

// Caller rows of type dtype (leading dimension ld) <- packed n x k doubles.
void stage_rows_out( void * dst, std::int32_t dtype, std::int32_t ld, const double * src, std::int64_t n, std::int32_t k )
{
    host_rows( n, static_cast<std::int64_t>( k ) * 8, [&]( std::int64_t b, std::int64_t e )
    {
        if( dtype == TB_F64 )
        {
            double * d = static_cast<double *>( dst );
            if( ld == k ) { std::memcpy( d + b * k, src + b * k, sizeof(double) * static_cast<size_t>( (e - b) * k ) ); return; }
            for( std::int64_t i = b; i < e; ++i ) { std::memcpy( d + i * ld, src + i * k, sizeof(double) * static_cast<size_t>( k ) ); }
        }
        else
        {
            float * d = static_cast<float *>( dst );
            for( std::int64_t i = b; i < e; ++i )
            {
                for( std::int32_t c = 0; c < k; ++c ) { d[i * ld + c] = static_cast<float>( src[i * k + c] ); }
            }
        }
    } );
}

// Host buffers of either type: staged through pinned memory on all host
// threads (cast on copy), solved on the device, copied back.
int run_solve_host( tb_chol * h, int which, double alpha, const void * B, std::int32_t ldB, std::int32_t b_dtype,
                    double beta, void * X, std::int32_t ldX, std::int32_t x_dtype, std::int32_t nrhs )
{
    if( B == nullptr || X == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "Solve: null buffer" ); }
    if( dtype_size( b_dtype ) == 0 || dtype_size( x_dtype ) == 0 ) { return fail( TB_ERR_INVALID_ARGUMENT, "Solve: unknown scalar type" ); }
    const std::int32_t n = h->n;
    const std::int32_t k = std::max( 1, nrhs );
    if( ldB < k || ldX < k ) { return fail( TB_ERR_INVALID_ARGUMENT, "Solve: leading dimension smaller than nrhs" ); }
    const std::int64_t kcap = rhs_capacity( k );
    cudaStream_t st = h->stream;
    TB_TRY( h->pin_in.reserve( sizeof(double) * static_cast<size_t>(n) * kcap ) );
    TB_TRY( h->pin_out.reserve( sizeof(double) * static_cast<size_t>(n) * kcap ) );
    TB_TRY( h->in.reserve( static_cast<std::int64_t>(n) * kcap ) );
    TB_TRY( h->out.reserve( static_cast<std::int64_t>(n) * kcap ) );
    double * pi = h->pin_in.as<double>();
    double * po = h->pin_out.as<double>();
    // in chunks of rows: the copy of chunk c to the device runs while the host stages chunk c + 1
    const std::int64_t rows_per_chunk = std::max<std::int64_t>( 1, (std::int64_t( 16 ) << 20) / (8 * std::int64_t( k )) );
    const int esz = dtype_size( b_dtype ), xsz = dtype_size( x_dtype );
    for( std::int64_t r0 = 0; r0 < n; r0 += rows_per_chunk )
    {
        const std::int64_t rc = std::min<std::int64_t>( rows_per_chunk, n - r0 );
        stage_rows_in( pi + r0 * k, static_cast<const char *>( B ) + r0 * ldB * esz, b_dtype, rc, k, ldB );
        TB_CUDA( cudaMemcpyAsync( h->in.ptr + r0 * k, pi + r0 * k, sizeof(double) * static_cast<size_t>( rc * k ),
                                  cudaMemcpyHostToDevice, st ) );
        if( beta != 0.0 )
        {
            stage_rows_in( po + r0 * k, static_cast<const char *>( X ) + r0 * ldX * xsz, x_dtype, rc, k, ldX );
            TB_CUDA( cudaMemcpyAsync( h->out.ptr + r0 * k, po + r0 * k, sizeof(double) * static_cast<size_t>( rc * k ),
                                      cudaMemcpyHostToDevice, st ) );
        }
    }
    TB_TRY( run_solve_device( h, which, alpha, h->in.ptr, k, beta, h->out.ptr, k, k ) );
    // back in chunks: the host unstages chunk c while chunk c + 1 is copied
    std::vector<cudaEvent_t> done;
    for( std::int64_t r0 = 0; r0 < n; r0 += rows_per_chunk )
    {
        const std::int64_t rc = std::min<std::int64_t>( rows_per_chunk, n - r0 );
        TB_CUDA( cudaMemcpyAsync( po + r0 * k, h->out.ptr + r0 * k, sizeof(double) * static_cast<size_t>( rc * k ),
                                  cudaMemcpyDeviceToHost, st ) );
        if( h->chunk_events.size() <= done.size() )
        {
            cudaEvent_t e;
            TB_CUDA( cudaEventCreateWithFlags( &e, cudaEventDisableTiming ) );
            h->chunk_events.push_back( e );
        }
        TB_CUDA( cudaEventRecord( h->chunk_events[done.size()], st ) );
        done.push_back( h->chunk_events[done.size()] );
    }
    size_t c = 0;
    for( std::int64_t r0 = 0; r0 < n; r0 += rows_per_chunk, ++c )
    {
        const std::int64_t rc = std::min<std::int64_t>( rows_per_chunk, n - r0 );
        TB_CUDA( cudaEventSynchronize( done[c] ) );
        if( c == 0 ) { TB_TRY( check_solve_error( h ) ); }
        stage_rows_out( static_cast<char *>( X ) + r0 * ldX * xsz, x_dtype, ldX, po + r0 * k, rc, k );
    }
    TB_CUDA( cudaStreamSynchronize( st ) );
    return TB_OK;
}

int run_solve_host( tb_chol * h, int which, double alpha, const double * B, std::int32_t ldB,
                    double beta, double * X, std::int32_t ldX, std::int32_t nrhs )
{
    return run_solve_host( h, which, alpha, B, ldB, TB_F64, beta, X, ldX, TB_F64, nrhs );
}

int fetch_diagonal( tb_chol * h, std::vector<double> & d )
{
    TB_TRY( require_factor( h ) );
    if( h->precision == TB_PRECISION_MIXED ) { tb::launch_gather_diag( h->diag_off.ptr, arena_as<float>( h ), h->diag_vals.ptr, h->n, h->stream ); }
    else { tb::launch_gather_diag( h->diag_off.ptr, arena_as<double>( h ), h->diag_vals.ptr, h->n, h->stream ); }
    d.resize( static_cast<size_t>(h->n) );
    TB_CUDA( cudaMemcpyAsync( d.data(), h->diag_vals.ptr, sizeof(double) * d.size(), cudaMemcpyDeviceToHost, h->stream ) );
    TB_CUDA( cudaStreamSynchronize( h->stream ) );
    return TB_OK;
}

} // namespace

namespace
{
template<typename T>
std::int64_t copy_array( const std::vector<T> & v, std::int64_t * out )
{
    if( out ) { for( size_t i = 0; i < v.size(); ++i ) { out[i] = static_cast<std::int64_t>( v[i] ); } }
    return static_cast<std::int64_t>( v.size() );
}

int array_op( tb_chol * h, std::int32_t which, std::int64_t * size, std::int64_t * out )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( ensure_symbolic( h ) );
    const tb::Symbolic & s = h->sym;
    std::int64_t n = -1;
    switch( which )
    {
        case TB_ARRAY_PERM:            n = copy_array( s.p, out ); break;
        case TB_ARRAY_PERM_INV:        n = copy_array( s.p_inv, out ); break;
        case TB_ARRAY_VALUE_PERM:      n = copy_array( s.value_perm, out ); break;
        case TB_ARRAY_SN_RP:           n = copy_array( s.sn_rp, out ); break;
        case TB_ARRAY_SN_OUTER:        n = copy_array( s.sn_outer, out ); break;
        case TB_ARRAY_SN_INNER:        n = copy_array( s.sn_inner, out ); break;
        case TB_ARRAY_ROW_TO_SN:       n = copy_array( s.row_to_sn, out ); break;
        case TB_ARRAY_SN_TRI_PTR:      n = copy_array( s.sn_tri_ptr, out ); break;
        case TB_ARRAY_SN_REC_PTR:      n = copy_array( s.sn_rec_ptr, out ); break;
        case TB_ARRAY_ATREE_PARENTS:   n = copy_array( s.atree_parent, out ); break;
        case TB_ARRAY_ETREE_PARENTS:   n = copy_array( s.etree_parent, out ); break;
        case TB_ARRAY_OUTER:           n = copy_array( s.outer, out ); break;
        case TB_ARRAY_INNER:           n = copy_array( s.inner, out ); break;
        case TB_ARRAY_ATREE_CHILD_PTR: n = copy_array( s.atree_child_ptr, out ); break;
        case TB_ARRAY_ATREE_CHILD_IDX: n = copy_array( s.atree_child_idx, out ); break;
        default: return fail( TB_ERR_INVALID_ARGUMENT, "unknown array selector" );
    }
    if( size ) { *size = n; }
    return TB_OK;
}
} // namespace

extern "C" {

const char * tb_last_error( void ) { return g_error.c_str(); }

int tb_set_device( int device )
{
    int count = 0;
    if( cudaGetDeviceCount( &count ) != cudaSuccess || count == 0 ) { return fail( TB_ERR_NO_DEVICE, "no CUDA device" ); }
    if( device < 0 || device >= count ) { return fail( TB_ERR_INVALID_ARGUMENT, "device ordinal out of range" ); }
    g_device = device;
    return TB_OK;
}

int tb_chol_create( tb_chol ** out, std::int32_t n, const std::int64_t * outer, const std::int32_t * inner,
                    const std::int32_t * perm, std::int32_t thread_count )
{
    if( out == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null output handle" ); }
    *out = nullptr;
    if( n <= 0 ) { return fail( TB_ERR_INVALID_ARGUMENT, "Size n of matrix is <= 0" ); }
    if( outer == nullptr || inner == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null pattern" ); }
    if( outer[0] != 0 || outer[n] < n ) { return fail( TB_ERR_INVALID_PATTERN, "invalid row pointers" ); }
    auto * h = new tb_chol();
    h->device = g_device;
    h->n = n;
    h->outer.assign( outer, outer + n + 1 );
    h->inner.assign( inner, inner + outer[n] );
    if( perm != nullptr ) { h->perm.assign( perm, perm + n ); h->has_perm = true; }
    h->threads = thread_count;                 // <= 0: every hardware thread
    *out = h;
    return TB_OK;
}

int tb_chol_destroy( tb_chol * h )
{
    if( h == nullptr ) { return TB_OK; }
    if( h->stream ) { cudaSetDevice( h->device ); cudaStreamSynchronize( h->stream ); }
    delete h;
    return TB_OK;
}

int tb_chol_set_supernode_strategy( tb_chol * h, std::int32_t strategy )
{
    if( h == nullptr || strategy < 0 || strategy > 2 ) { return fail( TB_ERR_INVALID_ARGUMENT, "invalid supernode strategy" ); }
    const auto s = static_cast<tb::SupernodeStrategy>( strategy );
    if( s != h->strategy ) { h->strategy = s; h->invalidate_symbolic(); }
    return TB_OK;
}

int tb_chol_set_amalgamation_threshold( tb_chol * h, std::int32_t threshold )
{
    if( h == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null handle" ); }
    if( threshold != h->amalgamation_threshold ) { h->amalgamation_threshold = threshold; h->invalidate_symbolic(); }
    return TB_OK;
}

int tb_chol_set_factorization_method( tb_chol * h, std::int32_t method )
{
    if( h == nullptr || (method != TB_MULTIFRONTAL && method != TB_LEFT_LOOKING) ) { return fail( TB_ERR_INVALID_ARGUMENT, "invalid factorization method" ); }
    h->method = method;
    return TB_OK;
}

int tb_chol_symbolic( tb_chol * h )
{
    TB_TRY( check_handle( h ) );
    return ensure_symbolic( h );
}

int tb_chol_numeric( tb_chol * h, const double * values, double reg )
{
    return tb_chol_numeric_ex( h, values, TB_F64, reg );
}

int tb_chol_numeric_ex( tb_chol * h, const void * values, std::int32_t dtype, double reg )
{
    TB_TRY( check_handle( h ) );
    if( values == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "NumericFactorization: null values" ); }
    if( dtype_size( dtype ) == 0 ) { return fail( TB_ERR_INVALID_ARGUMENT, "NumericFactorization: unknown scalar type" ); }
    TB_TRY( ensure_device( h ) );
    const size_t bytes = sizeof(double) * static_cast<size_t>( h->sym.nnz );
    TB_TRY( h->pin_in.reserve( bytes ) );
    // in chunks: the copy of chunk c to the device runs while the host stages chunk c + 1
    const std::int64_t chunk = std::int64_t( 2 ) << 20;          // values per chunk (16 MB of FP64)
    const int esz = dtype_size( dtype );
    double * pin = h->pin_in.as<double>();
    for( std::int64_t i0 = 0; i0 < h->sym.nnz; i0 += chunk )
    {
        const std::int64_t c = std::min<std::int64_t>( chunk, h->sym.nnz - i0 );
        stage_rows_in( pin + i0, static_cast<const char *>( values ) + i0 * esz, dtype, c, 1, 1 );
        TB_CUDA( cudaMemcpyAsync( h->values.ptr + i0, pin + i0, sizeof(double) * static_cast<size_t>( c ), cudaMemcpyHostToDevice, h->stream ) );
    }
    return run_factor( h, reg );
}

int tb_chol_numeric_device_ex( tb_chol * h, const void * d_values, std::int32_t dtype, double reg )
{
    TB_TRY( check_handle( h ) );
    if( d_values == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "NumericFactorization: null values" ); }
    if( dtype == TB_F64 ) { return tb_chol_numeric_device( h, static_cast<const double *>( d_values ), reg ); }
    if( dtype != TB_F32 ) { return fail( TB_ERR_INVALID_ARGUMENT, "NumericFactorization: unknown scalar type" ); }
    TB_TRY( ensure_device( h ) );
    tb::launch_widen( static_cast<const float *>( d_values ), 1, h->values.ptr, 1, h->sym.nnz, 1, h->stream );
    TB_CUDA( cudaGetLastError() );
    return run_factor( h, reg );
}

int tb_chol_numeric_device( tb_chol * h, const double * d_values, double reg )
{
    TB_TRY( check_handle( h ) );
    if( d_values == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "NumericFactorization: null values" ); }
    TB_TRY( ensure_device( h ) );
    if( d_values != h->values.ptr )
    {
        TB_CUDA( cudaMemcpyAsync( h->values.ptr, d_values, sizeof(double) * static_cast<size_t>( h->sym.nnz ),
                                  cudaMemcpyDeviceToDevice, h->stream ) );
    }
    return run_factor( h, reg );
}

int tb_chol_solve( tb_chol * h, double alpha, const double * B, std::int32_t ldB,
                   double beta, double * X, std::int32_t ldX, std::int32_t nrhs )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( require_factor( h ) );
    return run_solve_host( h, 2, alpha, B, ldB, beta, X, ldX, nrhs );
}

int tb_chol_solve_device( tb_chol * h, double alpha, const double * d_B, std::int32_t ldB,
                          double beta, double * d_X, std::int32_t ldX, std::int32_t nrhs )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( require_factor( h ) );
    if( d_B == nullptr || d_X == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "Solve: null buffer" ); }
    return run_solve_device( h, 2, alpha, d_B, ldB, beta, d_X, ldX, nrhs );
}

int tb_chol_upper_solve( tb_chol * h, double alpha, const double * B, std::int32_t ldB,
                         double beta, double * X, std::int32_t ldX, std::int32_t nrhs )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( require_factor( h ) );
    return run_solve_host( h, 1, alpha, B, ldB, beta, X, ldX, nrhs );
}

int tb_chol_lower_solve( tb_chol * h, double alpha, const double * B, std::int32_t ldB,
                         double beta, double * X, std::int32_t ldX, std::int32_t nrhs )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( require_factor( h ) );
    return run_solve_host( h, 0, alpha, B, ldB, beta, X, ldX, nrhs );
}

int tb_chol_residual_device( tb_chol * h, const double * d_B, const double * d_X, double * d_R, std::int32_t nrhs )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( require_factor( h ) );
    tb::launch_residual( h->n, h->a_outer.ptr, h->a_inner.ptr, h->values.ptr, d_X, d_B, d_R, std::max( 1, nrhs ), h->stream );
    TB_CUDA( cudaGetLastError() );
    return TB_OK;
}

// Preconditioned conjugate gradients with the factor as the preconditioner,
// step for step the reference's ConjugateGradient::operator()
// (ConjugateGradient.hpp:109-356): r = b (- A x0), z = P r, p = z,
// rho = r.z; then u = A p, alpha = rho / p.u, x += alpha p, r -= alpha u,
// z = P r, beta = rho_new / rho, p = z + beta p, until |rho_c| <= tol^2 |b_c.P b_c|
// for every column (CheckResiduals, :470-480) or max_iter steps; then
// X = alpha_out x + beta_out X.  One recurrence per column, scalars on the device.
int tb_chol_cg_device( tb_chol * h, const double * d_values, double reg, double alpha, const double * d_B, std::int32_t ldB,
                       double beta, double * d_X, std::int32_t ldX, std::int32_t nrhs, double rel_tol, std::int32_t max_iter,
                       std::int32_t use_initial_guess, std::int32_t * iterations, double * relres )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( require_factor( h ) );
    const std::int32_t n = h->n;
    const std::int32_t k = std::max( 1, nrhs );
    if( d_B == nullptr || d_X == nullptr || ldB < k || ldX < k || max_iter < 0 || !(rel_tol >= 0.0) )
    {
        return fail( TB_ERR_INVALID_ARGUMENT, "ConjugateGradient: bad argument" );
    }
    cudaStream_t st = h->stream;
    const std::int64_t nk = static_cast<std::int64_t>( n ) * k;
    TB_TRY( h->cg_buf.reserve( 5 * nk ) );             // x, r, z, p, u
    TB_TRY( h->cg_scal.reserve( 4 * k ) );             // b.Pb, rho, rho_old, p.u
    TB_TRY( h->pin_norms.reserve( sizeof(double) * 2 * static_cast<size_t>( k ) ) );
    double * x = h->cg_buf.ptr;
    double * r = x + nk;
    double * z = x + 2 * nk;
    double * p = x + 3 * nk;
    double * u = x + 4 * nk;
    double * bsq = h->cg_scal.ptr;
    double * rho = bsq + k;
    double * rho_old = bsq + 2 * k;
    double * pu = bsq + 3 * k;
    double * hn = h->pin_norms.as<double>();
    const double * vals = d_values != nullptr ? d_values : h->values.ptr;
    auto dots = [&]( const double * a, const double * b, double * out ) -> int {
        TB_CUDA( cudaMemsetAsync( out, 0, sizeof(double) * static_cast<size_t>( k ), st ) );
        tb::launch_column_dots( a, k, b, k, n, k, out, st );
        return TB_OK;
    };
    auto precondition = [&]( const double * in, double * out ) -> int {
        return run_solve_core( h, 2, 1.0, in, k, 0.0, out, k, k );
    };
    // host copy of rho and b.Pb; true when every column meets its tolerance
    std::vector<double> tol2( static_cast<size_t>( k ) );
    auto converged = [&]( bool * done ) -> int {
        TB_CUDA( cudaMemcpyAsync( hn, bsq, sizeof(double) * 2 * static_cast<size_t>( k ), cudaMemcpyDeviceToHost, st ) );
        TB_CUDA( cudaStreamSynchronize( st ) );
        TB_TRY( check_solve_error( h ) );
        *done = true;
        for( std::int32_t c = 0; c < k; ++c ) { *done = *done && std::abs( hn[k + c] ) <= tol2[static_cast<size_t>( c )]; }
        return TB_OK;
    };
    std::int32_t iter = 0;
    bool done = false;
    if( alpha != 0.0 )
    {
        tb::launch_combine( n, k, 1.0, d_B, ldB, 0.0, r, k, st );              // r = b
        TB_TRY( precondition( r, z ) );                                          // z = P b
        TB_TRY( dots( r, z, bsq ) );
        TB_CUDA( cudaMemcpyAsync( hn, bsq, sizeof(double) * static_cast<size_t>( k ), cudaMemcpyDeviceToHost, st ) );
        TB_CUDA( cudaStreamSynchronize( st ) );
        TB_TRY( check_solve_error( h ) );
        double bmax = 0.0;
        for( std::int32_t c = 0; c < k; ++c )
        {
            if( std::isnan( hn[c] ) ) { return fail( TB_ERR_INVALID_ARGUMENT, "ConjugateGradient: right-hand side contains NaNs" ); }
            tol2[static_cast<size_t>( c )] = std::abs( hn[c] ) * rel_tol * rel_tol;
            bmax = std::max( bmax, std::abs( hn[c] ) );
        }
        if( bmax > 0.0 )
        {
            if( use_initial_guess )
            {
                tb::launch_combine( n, k, 1.0, d_X, ldX, 0.0, x, k, st );      // x = x0
                tb::launch_apply_shifted( n, h->a_outer.ptr, h->a_inner.ptr, vals, reg, x, k, r, k, u, k, k, st );   // b - A x0
                std::swap( r, u );                                               // r = b - A x0 (u is scratch)
                TB_TRY( precondition( r, z ) );
            }
            else
            {
                TB_CUDA( cudaMemsetAsync( x, 0, sizeof(double) * static_cast<size_t>( nk ), st ) );
            }
            TB_CUDA( cudaMemcpyAsync( p, z, sizeof(double) * static_cast<size_t>( nk ), cudaMemcpyDeviceToDevice, st ) );
            TB_TRY( dots( r, z, rho ) );
            TB_TRY( converged( &done ) );
            while( !done && iter < max_iter )
            {
                tb::launch_apply_shifted( n, h->a_outer.ptr, h->a_inner.ptr, vals, reg, p, k, nullptr, k, u, k, k, st );   // u = A p
                TB_TRY( dots( p, u, pu ) );
                tb::launch_cg_update_xr( n, k, rho, pu, p, u, x, r, st );       // x += alpha p, r -= alpha u
                TB_TRY( precondition( r, z ) );                                  // z = P r
                TB_CUDA( cudaMemcpyAsync( rho_old, rho, sizeof(double) * static_cast<size_t>( k ), cudaMemcpyDeviceToDevice, st ) );
                TB_TRY( dots( r, z, rho ) );
                tb::launch_cg_update_p( n, k, rho, rho_old, z, p, st );         // p = z + beta p
                TB_TRY( converged( &done ) );
                ++iter;
            }
            tb::launch_combine( n, k, alpha, x, k, beta, d_X, ldX, st );         // X = alpha x + beta X
        }
        else
        {
            done = true;                                                         // b = 0: X = beta X
            tb::launch_combine( n, k, beta, d_X, ldX, 0.0, d_X, ldX, st );
        }
    }
    else
    {
        done = true;                                                             // alpha = 0: X = beta X
        tb::launch_combine( n, k, beta, d_X, ldX, 0.0, d_X, ldX, st );
    }
    TB_CUDA( cudaGetLastError() );
    TB_CUDA( cudaStreamSynchronize( st ) );
    if( iterations != nullptr ) { *iterations = iter; }
    if( relres != nullptr )
    {
        for( std::int32_t c = 0; c < k; ++c )
        {
            const double b2 = std::abs( hn[c] );
            relres[c] = alpha == 0.0 || b2 <= 0.0 ? 0.0 : std::sqrt( std::abs( hn[k + c] ) / b2 );
        }
    }
    if( !done )
    {
        return fail( TB_ERR_NOT_CONVERGED, "ConjugateGradient: not converged after " + std::to_string( iter ) + " iterations" );
    }
    return TB_OK;
}

// Host-buffer form of tb_chol_cg_device: values (caller order, NULL = those
// of the last factorization), B and X are copied through device scratch.
int tb_chol_cg( tb_chol * h, const double * values, double reg, double alpha, const double * B, std::int32_t ldB,
                double beta, double * X, std::int32_t ldX, std::int32_t nrhs, double rel_tol, std::int32_t max_iter,
                std::int32_t use_initial_guess, std::int32_t * iterations, double * relres )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( require_factor( h ) );
    const std::int32_t k = std::max( 1, nrhs );
    if( B == nullptr || X == nullptr || ldB < k || ldX < k ) { return fail( TB_ERR_INVALID_ARGUMENT, "ConjugateGradient: bad argument" ); }
    const std::int64_t nnz = h->outer[h->n];
    const std::int64_t nk = static_cast<std::int64_t>( h->n ) * k;
    cudaStream_t st = h->stream;
    TB_TRY( h->cg_host.reserve( (values != nullptr ? nnz : 0) + 2 * nk ) );
    double * dB = h->cg_host.ptr;
    double * dX = dB + nk;
    double * dv = values != nullptr ? dX + nk : nullptr;
    TB_CUDA( cudaMemcpy2DAsync( dB, sizeof(double) * k, B, sizeof(double) * ldB, sizeof(double) * k, h->n, cudaMemcpyHostToDevice, st ) );
    if( use_initial_guess || beta != 0.0 )
    {
        TB_CUDA( cudaMemcpy2DAsync( dX, sizeof(double) * k, X, sizeof(double) * ldX, sizeof(double) * k, h->n, cudaMemcpyHostToDevice, st ) );
    }
    else
    {
        TB_CUDA( cudaMemsetAsync( dX, 0, sizeof(double) * static_cast<size_t>( nk ), st ) );
    }
    if( dv != nullptr ) { TB_CUDA( cudaMemcpyAsync( dv, values, sizeof(double) * static_cast<size_t>( nnz ), cudaMemcpyHostToDevice, st ) ); }
    const int status = tb_chol_cg_device( h, dv, reg, alpha, dB, k, beta, dX, k, nrhs, rel_tol, max_iter, use_initial_guess,
                                          iterations, relres );
    if( status < 0 && status != TB_ERR_NOT_CONVERGED ) { return status; }
    const std::string msg = g_error;
    TB_CUDA( cudaMemcpy2DAsync( X, sizeof(double) * ldX, dX, sizeof(double) * k, sizeof(double) * k, h->n, cudaMemcpyDeviceToHost, st ) );
    TB_CUDA( cudaStreamSynchronize( st ) );
    if( status != TB_OK ) { g_error = msg; }
    return status;
}

// GMRES preconditioned by the factor: the reference's GMRES::operator()
// (GMRES.hpp:124-330) with the operator (A' + reg I) and P = the factor's
// solve; X = alpha x + beta X.  Device buffers.
int tb_chol_gmres_device( tb_chol * h, const double * d_values, double reg, double alpha, const double * d_B, std::int32_t ldB,
                          double beta, double * d_X, std::int32_t ldX, std::int32_t nrhs, double rel_tol, std::int32_t max_iter,
                          std::int32_t max_restarts, std::int32_t use_initial_guess, std::int32_t * iterations,
                          std::int32_t * restarts, double * relres )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( require_factor( h ) );
    const std::int32_t n = h->n;
    const std::int32_t k = std::max( 1, nrhs );
    if( d_B == nullptr || d_X == nullptr || ldB < k || ldX < k || max_iter < 1 || max_restarts < 0 || !(rel_tol >= 0.0) )
    {
        return fail( TB_ERR_INVALID_ARGUMENT, "GMRES: bad argument" );
    }
    cudaStream_t st = h->stream;
    const std::int64_t nk = static_cast<std::int64_t>( n ) * k;
    TB_TRY( h->cg_buf.reserve( nk ) );
    double * x = h->cg_buf.ptr;
    std::vector<double> rel( static_cast<size_t>( k ), 0.0 );
    GmresOutcome go;
    if( alpha != 0.0 )
    {
        if( use_initial_guess ) { tb::launch_combine( n, k, 1.0, d_X, ldX, 0.0, x, k, st ); }
        const double * vals = d_values != nullptr ? d_values : h->values.ptr;
        TB_TRY( run_gmres( h, vals, reg, d_B, ldB, k, x, use_initial_guess != 0, rel_tol, max_iter, max_restarts, rel.data(), go ) );
        tb::launch_combine( n, k, alpha, x, k, beta, d_X, ldX, st );          // X = alpha x + beta X
    }
    else
    {
        go.converged = true;
        tb::launch_combine( n, k, beta, d_X, ldX, 0.0, d_X, ldX, st );
    }
    TB_CUDA( cudaGetLastError() );
    TB_CUDA( cudaStreamSynchronize( st ) );
    if( iterations ) { *iterations = go.iterations; }
    if( restarts ) { *restarts = go.restarts; }
    if( relres ) { for( std::int32_t c = 0; c < k; ++c ) { relres[c] = rel[static_cast<size_t>( c )]; } }
    if( !go.converged )
    {
        return fail( TB_ERR_NOT_CONVERGED, "GMRES: not converged after " + std::to_string( go.restarts ) + " restarts ("
                     + std::to_string( go.iterations ) + " steps)" );
    }
    return TB_OK;
}

// Host-buffer form of tb_chol_gmres_device (values NULL: those of the last factorization).
int tb_chol_gmres( tb_chol * h, const double * values, double reg, double alpha, const double * B, std::int32_t ldB,
                   double beta, double * X, std::int32_t ldX, std::int32_t nrhs, double rel_tol, std::int32_t max_iter,
                   std::int32_t max_restarts, std::int32_t use_initial_guess, std::int32_t * iterations,
                   std::int32_t * restarts, double * relres )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( require_factor( h ) );
    const std::int32_t k = std::max( 1, nrhs );
    if( B == nullptr || X == nullptr || ldB < k || ldX < k ) { return fail( TB_ERR_INVALID_ARGUMENT, "GMRES: bad argument" ); }
    const std::int64_t nnz = h->outer[h->n];
    const std::int64_t nk = static_cast<std::int64_t>( h->n ) * k;
    cudaStream_t st = h->stream;
    TB_TRY( h->cg_host.reserve( (values != nullptr ? nnz : 0) + 2 * nk ) );
    double * dB = h->cg_host.ptr;
    double * dX = dB + nk;
    double * dv = values != nullptr ? dX + nk : nullptr;
    TB_CUDA( cudaMemcpy2DAsync( dB, sizeof(double) * k, B, sizeof(double) * ldB, sizeof(double) * k, h->n, cudaMemcpyHostToDevice, st ) );
    if( use_initial_guess || beta != 0.0 )
    {
        TB_CUDA( cudaMemcpy2DAsync( dX, sizeof(double) * k, X, sizeof(double) * ldX, sizeof(double) * k, h->n, cudaMemcpyHostToDevice, st ) );
    }
    else
    {
        TB_CUDA( cudaMemsetAsync( dX, 0, sizeof(double) * static_cast<size_t>( nk ), st ) );
    }
    if( dv != nullptr ) { TB_CUDA( cudaMemcpyAsync( dv, values, sizeof(double) * static_cast<size_t>( nnz ), cudaMemcpyHostToDevice, st ) ); }
    const int status = tb_chol_gmres_device( h, dv, reg, alpha, dB, k, beta, dX, k, nrhs, rel_tol, max_iter, max_restarts,
                                             use_initial_guess, iterations, restarts, relres );
    if( status < 0 && status != TB_ERR_NOT_CONVERGED ) { return status; }
    const std::string msg = g_error;
    TB_CUDA( cudaMemcpy2DAsync( X, sizeof(double) * ldX, dX, sizeof(double) * k, sizeof(double) * k, h->n, cudaMemcpyDeviceToHost, st ) );
    TB_CUDA( cudaStreamSynchronize( st ) );
    if( status != TB_OK ) { g_error = msg; }
    return status;
}

int tb_chol_gmres_ir_iterations( tb_chol * h, std::int32_t * out )
{
    TB_TRY( check_handle( h ) );
    if( out ) { *out = h->gmres_iters; }
    return TB_OK;
}

int tb_chol_sn_count( tb_chol * h, std::int32_t * out )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( ensure_symbolic( h ) );
    *out = h->sym.sn_count;
    return TB_OK;
}

int tb_chol_row_count( tb_chol * h, std::int32_t * out )
{
    if( h == nullptr || out == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null argument" ); }
    *out = h->n;
    return TB_OK;
}

int tb_chol_nonzero_count( tb_chol * h, std::int64_t * out )
{
    if( h == nullptr || out == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null argument" ); }
    *out = h->outer[h->n];
    return TB_OK;
}


int tb_chol_array_size( tb_chol * h, std::int32_t which, std::int64_t * out )
{
    if( out == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null output" ); }
    return array_op( h, which, out, nullptr );
}

int tb_chol_array_copy( tb_chol * h, std::int32_t which, std::int64_t * out )
{
    if( out == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null output" ); }
    return array_op( h, which, nullptr, out );
}

int tb_chol_factorized( tb_chol * h, std::int32_t * factorized, std::int32_t * good )
{
    if( h == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null handle" ); }
    if( factorized ) { *factorized = h->factorized ? 1 : 0; }
    if( good ) { *good = h->good ? 1 : 0; }
    return TB_OK;
}

int tb_chol_failed_supernode( tb_chol * h, std::int32_t * out )
{
    if( h == nullptr || out == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null argument" ); }
    *out = h->failed_sn;
    return TB_OK;
}

int tb_chol_factor_sizes( tb_chol * h, std::int64_t * tri_size, std::int64_t * rec_size )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( ensure_symbolic( h ) );
    if( tri_size ) { *tri_size = h->sym.sn_tri_ptr[h->sym.sn_count]; }
    if( rec_size ) { *rec_size = h->sym.sn_rec_ptr[h->sym.sn_count]; }
    return TB_OK;
}

int tb_chol_factor_values( tb_chol * h, double * tri, double * rec )
{
    TB_TRY( check_handle( h ) );
    if( !h->factorized ) { return fail( TB_ERR_NOT_FACTORIZED, "factor values requested before NumericFactorization" ); }
    TB_CUDA( cudaSetDevice( h->device ) );
    const std::int64_t ts = h->sym.sn_tri_ptr[h->sym.sn_count];
    const std::int64_t rs = h->sym.sn_rec_ptr[h->sym.sn_count];
    TB_TRY( h->exported.reserve( ts + rs ) );
    if( h->precision == TB_PRECISION_MIXED )
    {
        tb::launch_export( h->exports.ptr, static_cast<int>( h->plan.exports.size() ), h->colmap.ptr, arena_as<float>( h ),
                           h->exported.ptr, h->exported.ptr + ts, h->stream );
    }
    else
    {
        tb::launch_export( h->exports.ptr, static_cast<int>( h->plan.exports.size() ), h->colmap.ptr, arena_as<double>( h ),
                           h->exported.ptr, h->exported.ptr + ts, h->stream );
    }
    TB_CUDA( cudaGetLastError() );
    if( tri && ts ) { TB_CUDA( cudaMemcpyAsync( tri, h->exported.ptr, sizeof(double) * ts, cudaMemcpyDeviceToHost, h->stream ) ); }
    if( rec && rs ) { TB_CUDA( cudaMemcpyAsync( rec, h->exported.ptr + ts, sizeof(double) * rs, cudaMemcpyDeviceToHost, h->stream ) ); }
    TB_CUDA( cudaStreamSynchronize( h->stream ) );
    return TB_OK;
}

// Nonzeros of U (InputOutput.hpp:124-137): per supernode row i, the
// triangle's columns i .. i_end - 1 and the supernode's n1 columns.
int tb_chol_u_nonzero_count( tb_chol * h, std::int64_t * out )
{
    TB_TRY( check_handle( h ) );
    if( out == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null output" ); }
    TB_TRY( ensure_symbolic( h ) );
    const tb::Symbolic & s = h->sym;
    std::int64_t nnz = 0;
    for( std::int32_t k = 0; k < s.sn_count; ++k )
    {
        const std::int64_t n0 = s.sn_rp[k + 1] - s.sn_rp[k], n1 = s.sn_outer[k + 1] - s.sn_outer[k];
        nnz += n0 * (n0 + 1) / 2 + n0 * n1;
    }
    *out = nnz;
    return TB_OK;
}

// U as CSR in the permuted ordering, rows sorted, as the reference's GetU
// (InputOutput.hpp:116-217) lays it out: row i of supernode s holds U0's row
// from the diagonal on (columns i .. i_end - 1), then U1's row (columns
// SN_inner[SN_outer[s] ..]).
int tb_chol_get_u( tb_chol * h, std::int64_t * outer, std::int32_t * inner, double * values )
{
    TB_TRY( check_handle( h ) );
    if( outer == nullptr || inner == nullptr || values == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null output" ); }
    const tb::Symbolic & s = h->sym;
    if( !h->factorized ) { return fail( TB_ERR_NOT_FACTORIZED, "GetU requested before NumericFactorization" ); }
    std::vector<double> tri( static_cast<size_t>( s.sn_tri_ptr[s.sn_count] ) ), rec( static_cast<size_t>( s.sn_rec_ptr[s.sn_count] ) );
    TB_TRY( tb_chol_factor_values( h, tri.data(), rec.data() ) );
    outer[0] = 0;
    for( std::int32_t k = 0; k < s.sn_count; ++k )
    {
        const std::int32_t i0 = s.sn_rp[k], i1 = s.sn_rp[k + 1];
        const std::int32_t n0 = i1 - i0;
        const std::int64_t l0 = s.sn_outer[k];
        const std::int32_t n1 = static_cast<std::int32_t>( s.sn_outer[k + 1] - l0 );
        const double * U0 = tri.data() + s.sn_tri_ptr[k];
        const double * U1 = rec.data() + s.sn_rec_ptr[k];
        for( std::int32_t r = 0; r < n0; ++r )
        {
            std::int64_t e = outer[i0 + r];
            for( std::int32_t c = r; c < n0; ++c, ++e ) { inner[e] = i0 + c; values[e] = U0[static_cast<std::int64_t>( r ) * n0 + c]; }
            for( std::int32_t c = 0; c < n1; ++c, ++e ) { inner[e] = s.sn_inner[static_cast<size_t>( l0 + c )]; values[e] = U1[static_cast<std::int64_t>( r ) * n1 + c]; }
            outer[i0 + r + 1] = e;
        }
    }
    return TB_OK;
}

int tb_chol_log_det( tb_chol * h, double * out )
{
    TB_TRY( check_handle( h ) );
    if( out == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null output" ); }
    std::vector<double> d;
    TB_TRY( fetch_diagonal( h, d ) );
    double s = 0.0;
    for( double v : d ) { s += std::log( v ); }
    *out = 2.0 * s;
    return TB_OK;
}

int tb_chol_factor_diagonal( tb_chol * h, double * diag )
{
    TB_TRY( check_handle( h ) );
    if( diag == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null output" ); }
    std::vector<double> d;
    TB_TRY( fetch_diagonal( h, d ) );
    std::copy( d.begin(), d.end(), diag );
    return TB_OK;
}

int tb_chol_flop_count( tb_chol * h, double * factor_flops, double * nnz_u )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( ensure_symbolic( h ) );
    if( factor_flops ) { *factor_flops = h->plan.factor_flops; }
    if( nnz_u ) { *nnz_u = h->plan.nnz_u; }
    return TB_OK;
}

int tb_chol_plan_stats( tb_chol * h, std::int64_t * out, std::int32_t cap )
{
    TB_TRY( check_handle( h ) );
    if( out == nullptr || cap < 0 ) { return fail( TB_ERR_INVALID_ARGUMENT, "null output" ); }
    TB_TRY( ensure_symbolic( h ) );
    const tb::Plan & pl = h->plan;
    const std::int64_t v[] = {
        pl.arena_size(), pl.v_size, pl.levels, static_cast<std::int64_t>( pl.factor_launches.size() ) + 2,
        static_cast<std::int64_t>( pl.gemm.size() ), static_cast<std::int64_t>( pl.panel.size() ),
        static_cast<std::int64_t>( pl.extend.size() ), static_cast<std::int64_t>( pl.lower_launches.size() ),
        static_cast<std::int64_t>( pl.upper_launches.size() ), h->sym.sn_count, pl.front_count,
        static_cast<std::int64_t>( pl.front_flops ), static_cast<std::int64_t>( pl.dag_makespan_us ),
        static_cast<std::int64_t>( pl.dag.size() ), static_cast<std::int64_t>( pl.solve_fwd_order.size() ),
        pl.solve_split_level, h->dag_grid, h->analyze_us, h->plan_us,
        static_cast<std::int64_t>( pl.tc.size() ), pl.img_blocks, static_cast<std::int64_t>( pl.gemm_flops ),
        static_cast<std::int64_t>( pl.gemm_tile_flops ), static_cast<std::int64_t>( pl.spanels.size() ),
        static_cast<std::int64_t>( pl.lower_launches_sp.size() ), static_cast<std::int64_t>( pl.upper_launches_sp.size() ) };
    const std::int32_t m = std::min<std::int32_t>( cap, static_cast<std::int32_t>( sizeof(v) / sizeof(v[0]) ) );
    for( std::int32_t i = 0; i < m; ++i ) { out[i] = v[i]; }
    return m;
}

int tb_chol_check_plan( tb_chol * h )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( ensure_symbolic( h ) );
    const std::string msg = tb::check_plan( h->sym, h->plan );
    if( !msg.empty() ) { return fail( TB_ERR_INVALID_ARGUMENT, "plan check: " + msg ); }
    return TB_OK;
}

int tb_chol_device_bytes( tb_chol * h, std::int64_t * out )
{
    if( h == nullptr || out == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null argument" ); }
    std::int64_t b = 0;
    b += h->arena.size * 8 + h->asm_src.size * 8 + h->asm_dst.size * 8 + h->diag_off.size * 8;
    b += (h->lut.size + h->sn_inner.size + h->p.size + h->p_inv.size + h->a_inner.size) * 4;
    b += h->gemm.size * (std::int64_t)sizeof(tb::GemmTask) + (h->panel.size + h->potrf.size) * (std::int64_t)sizeof(tb::PanelTask);
    b += (h->extend.size + h->extend_segs.size) * (std::int64_t)sizeof(tb::ExtendTask) + h->sdiag.size * (std::int64_t)sizeof(tb::SolveDiagTask);
    b += h->extend_pull.size * (std::int64_t)sizeof(tb::ExtendPullTask);
    b += h->srest.size * (std::int64_t)sizeof(tb::SolveRestTask) + h->a_outer.size * 8;
    b += h->zero.size * (std::int64_t)sizeof(tb::ZeroTask) + h->exports.size * (std::int64_t)sizeof(tb::ExportTask);
    b += h->colmap.size * 4 + h->exported.size * 8;
    b += (h->values.size + h->work.size + h->work2.size + h->in.size + h->out.size + h->diag_vals.size + h->tinv.size) * 8;
    *out = b;
    return TB_OK;
}

int tb_chol_set_stream( tb_chol * h, void * stream )
{
    TB_TRY( check_handle( h ) );
    TB_CUDA( cudaSetDevice( h->device ) );
    if( h->stream ) { TB_CUDA( cudaStreamSynchronize( h->stream ) ); }
    if( h->factor_graph ) { cudaGraphExecDestroy( h->factor_graph ); h->factor_graph = nullptr; }
    h->drop_solve_graphs();
    if( h->own_stream && h->stream ) { cudaStreamDestroy( h->stream ); }
    if( stream == nullptr )
    {
        TB_CUDA( cudaStreamCreateWithFlags( &h->stream, cudaStreamNonBlocking ) );
        h->own_stream = true;
    }
    else
    {
        h->stream = static_cast<cudaStream_t>( stream );
        h->own_stream = false;
    }
    return TB_OK;
}

int tb_chol_set_graph( tb_chol * h, std::int32_t enabled )
{
    if( h == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null handle" ); }
    h->use_graph = (enabled != 0);
    return TB_OK;
}

int tb_chol_set_schedule( tb_chol * h, std::int32_t schedule )
{
    TB_TRY( check_handle( h ) );
    if( schedule != TB_SCHEDULE_LEVELS && schedule != TB_SCHEDULE_TASK_GRAPH && schedule != TB_SCHEDULE_TASK_GRAPH_ALL )
    {
        return fail( TB_ERR_INVALID_ARGUMENT, "unknown schedule" );
    }
    if( schedule == h->schedule ) { return TB_OK; }
    const bool split_changes = (schedule == TB_SCHEDULE_TASK_GRAPH_ALL) != (h->schedule == TB_SCHEDULE_TASK_GRAPH_ALL);
    h->schedule = schedule;
    h->use_dag = schedule != TB_SCHEDULE_LEVELS;
    if( split_changes ) { h->invalidate_symbolic(); }
    if( h->factor_graph ) { cudaGraphExecDestroy( h->factor_graph ); h->factor_graph = nullptr; }
    return TB_OK;
}

int tb_chol_set_solve_schedule( tb_chol * h, std::int32_t schedule )
{
    TB_TRY( check_handle( h ) );
    if( schedule != TB_SCHEDULE_LEVELS && schedule != TB_SCHEDULE_TASK_GRAPH && schedule != TB_SCHEDULE_TASK_GRAPH_ALL )
    {
        return fail( TB_ERR_INVALID_ARGUMENT, "unknown schedule" );
    }
    if( schedule == h->solve_schedule ) { return TB_OK; }
    h->solve_schedule = schedule;
    if( h->symbolic_done )
    {
        if( h->stream ) { TB_CUDA( cudaStreamSynchronize( h->stream ) ); }
        tb::Plan & pl = h->plan;
        if( schedule == TB_SCHEDULE_LEVELS ) { pl.build_solve_graph( h->sym, pl.levels ); }
        else if( schedule == TB_SCHEDULE_TASK_GRAPH_ALL ) { pl.build_solve_graph( h->sym, 0 ); }
        else { pl.build_solve_graph( h->sym, pl.solve_default_split ); }
        if( h->device_ready )
        {
            cudaStream_t st_ = h->stream;
            TB_TRY( h->solve_fwd_order.upload( pl.solve_fwd_order, st_ ) );
            TB_TRY( h->solve_bwd_order.upload( pl.solve_bwd_order, st_ ) );
            TB_TRY( h->solve_targets.upload( pl.solve_targets, st_ ) );
            TB_TRY( h->solve_fwd_expected.upload( pl.solve_fwd_expected, st_ ) );
            TB_TRY( h->solve_panel_tasks.upload( pl.solve_panel_tasks, st_ ) );
            TB_TRY( h->solve_target_ptr.upload( pl.solve_target_ptr, st_ ) );
            TB_TRY( h->solve_state.reserve( static_cast<std::int64_t>( pl.solve_panel_tasks.size() ) + 2 ) );
            TB_CUDA( cudaStreamSynchronize( st_ ) );
            h->solve_grid.clear();
        }
    }
    h->drop_solve_graphs();
    return TB_OK;
}

int tb_chol_autotune( tb_chol * h, std::int32_t nrhs, std::int32_t * choice, double * times_ms )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( require_factor( h ) );
    cudaStream_t st = h->stream;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    TB_CUDA( cudaEventCreate( &e0 ) );
    TB_CUDA( cudaEventCreate( &e1 ) );
    auto elapsed = [&]() -> double {
        float ms = 0.0f;
        cudaEventSynchronize( e1 );
        cudaEventElapsedTime( &ms, e0, e1 );
        return ms;
    };
    const double inf = std::numeric_limits<double>::infinity();
    const std::int32_t sched[2] = { TB_SCHEDULE_LEVELS, TB_SCHEDULE_TASK_GRAPH };
    double t[4] = { inf, inf, inf, inf };
    int status = TB_OK;
    // factorization: the same values and shift as the last one; the factor is
    // the same bit for bit under both schedules, so the handle's stays valid
    for( int s = 0; s < 2 && status == TB_OK; ++s )
    {
        status = tb_chol_set_schedule( h, sched[s] );
        for( int rep = 0; rep < 3 && status == TB_OK; ++rep )       // the first run captures the graph
        {
            cudaEventRecord( e0, st );
            status = run_factor( h, h->last_reg );
            cudaEventRecord( e1, st );
            if( rep > 0 ) { t[s] = std::min( t[s], elapsed() ); }
        }
    }
    const std::int32_t k = std::max( 1, nrhs );
    if( status == TB_OK )
    {
        status = tb_chol_set_schedule( h, t[1] < t[0] ? sched[1] : sched[0] );
    }
    if( status == TB_OK )
    {
        // one solve's sweeps on zero right-hand sides (the work does not depend on the values)
        const std::int64_t nk = static_cast<std::int64_t>( h->n ) * k;
        status = h->ir_x.reserve( 2 * nk );
        if( status == TB_OK ) { cudaMemsetAsync( h->ir_x.ptr, 0, sizeof(double) * static_cast<size_t>( nk ), st ); }
        for( int s = 0; s < 2 && status == TB_OK; ++s )
        {
            status = tb_chol_set_solve_schedule( h, sched[s] );
            for( int rep = 0; rep < 3 && status == TB_OK; ++rep )
            {
                cudaEventRecord( e0, st );
                status = run_solve_core( h, 2, 1.0, h->ir_x.ptr, k, 0.0, h->ir_x.ptr + nk, k, k );
                cudaEventRecord( e1, st );
                if( rep > 0 && status == TB_OK ) { t[2 + s] = std::min( t[2 + s], elapsed() ); }
            }
        }
        if( status == TB_OK ) { status = tb_chol_set_solve_schedule( h, t[3] < t[2] ? sched[1] : sched[0] ); }
    }
    cudaEventDestroy( e0 );
    cudaEventDestroy( e1 );
    if( status != TB_OK ) { return status; }
    if( choice ) { choice[0] = t[1] < t[0] ? sched[1] : sched[0]; choice[1] = t[3] < t[2] ? sched[1] : sched[0]; }
    if( times_ms ) { for( int i = 0; i < 4; ++i ) { times_ms[i] = t[i]; } }
    return TB_OK;
}

int tb_chol_set_plan_options( tb_chol * h, std::int32_t defer_steps, std::int32_t relax, std::int32_t tc_width )
{
    TB_TRY( check_handle( h ) );
    if( defer_steps < 1 || defer_steps > 4 || relax < 0 || relax > 2 || (tc_width != 128 && tc_width != 256) )
    {
        return fail( TB_ERR_INVALID_ARGUMENT, "plan options: defer_steps 1-4, relax 0-2, tc_width 128 or 256" );
    }
    if( defer_steps == h->opt_defer && relax == h->opt_relax && tc_width == h->opt_tc_width ) { return TB_OK; }
    h->opt_defer = defer_steps;
    h->opt_relax = relax;
    h->opt_tc_width = tc_width;
    if( h->symbolic_done ) { h->plan_dirty = true; }
    h->device_ready = false;
    h->factorized = false;
    h->good = false;
    if( h->factor_graph ) { cudaGraphExecDestroy( h->factor_graph ); h->factor_graph = nullptr; }
    h->drop_solve_graphs();
    return TB_OK;
}

int tb_chol_plan_options( tb_chol * h, std::int32_t * defer_steps, std::int32_t * relax, std::int32_t * tc_width )
{
    TB_TRY( check_handle( h ) );
    if( defer_steps ) { *defer_steps = h->opt_defer; }
    if( relax ) { *relax = h->opt_relax; }
    if( tc_width ) { *tc_width = h->opt_tc_width; }
    return TB_OK;
}

// Times the factorization of the last values under every candidate plan
// option set (two runs each, the second timed) and keeps the fastest; the
// handle ends factored under it.
int tb_chol_autotune_plan( tb_chol * h, std::int32_t * choice, double * times_ms, std::int32_t cap )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( require_factor( h ) );
    std::vector<std::array<std::int32_t, 3>> cand;
    for( std::int32_t d : { 2, 3, 4 } )
    {
        for( std::int32_t r : { 0, 1, 2 } )
        {
            if( h->precision == TB_PRECISION_MIXED ) { for( std::int32_t w : { 128, 256 } ) { cand.push_back( { d, r, w } ); } }
            else { cand.push_back( { d, r, h->opt_tc_width } ); }
        }
    }
    const double reg = h->last_reg;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    TB_CUDA( cudaEventCreate( &e0 ) );
    TB_CUDA( cudaEventCreate( &e1 ) );
    double best = std::numeric_limits<double>::infinity();
    size_t pick = 0;
    int status = TB_OK;
    for( size_t c = 0; c < cand.size() && status == TB_OK; ++c )
    {
        status = tb_chol_set_plan_options( h, cand[c][0], cand[c][1], cand[c][2] );
        if( status == TB_OK ) { status = ensure_device( h ); }
        double t = std::numeric_limits<double>::infinity();
        for( int rep = 0; rep < 2 && status == TB_OK; ++rep )
        {
            cudaEventRecord( e0, h->stream );
            status = run_factor( h, reg );
            cudaEventRecord( e1, h->stream );
            cudaEventSynchronize( e1 );
            float ms = 0.0f;
            cudaEventElapsedTime( &ms, e0, e1 );
            if( rep == 1 ) { t = ms; }
        }
        if( times_ms && static_cast<std::int32_t>( c ) < cap ) { times_ms[c] = t; }
        if( status == TB_OK && t < best ) { best = t; pick = c; }
    }
    cudaEventDestroy( e0 );
    cudaEventDestroy( e1 );
    if( status != TB_OK ) { return status; }
    TB_TRY( tb_chol_set_plan_options( h, cand[pick][0], cand[pick][1], cand[pick][2] ) );
    TB_TRY( ensure_device( h ) );
    const int st = run_factor( h, reg );
    if( st < 0 ) { return st; }
    if( choice ) { choice[0] = cand[pick][0]; choice[1] = cand[pick][1]; choice[2] = cand[pick][2]; }
    return static_cast<int>( cand.size() );
}

int tb_chol_set_precision( tb_chol * h, std::int32_t precision )
{
    TB_TRY( check_handle( h ) );
    if( precision != TB_PRECISION_FP64 && precision != TB_PRECISION_MIXED ) { return fail( TB_ERR_INVALID_ARGUMENT, "unknown precision" ); }
    h->fell_back = false;
    if( precision == h->precision ) { return TB_OK; }
    h->precision = precision;
    h->device_ready = false;        // storage of the other width; the next factorization re-creates the device plan
    h->factorized = false;
    h->good = false;
    if( h->factor_graph ) { cudaGraphExecDestroy( h->factor_graph ); h->factor_graph = nullptr; }
    h->drop_solve_graphs();
    return TB_OK;
}

int tb_chol_set_refinement( tb_chol * h, double tol, std::int32_t max_iterations )
{
    TB_TRY( check_handle( h ) );
    if( !(tol >= 0.0) || max_iterations < 0 ) { return fail( TB_ERR_INVALID_ARGUMENT, "refinement: tol >= 0 and max_iterations >= 0" ); }
    h->ir_tol = tol;
    h->ir_max = max_iterations;
    return TB_OK;
}

int tb_chol_refinement_info( tb_chol * h, std::int32_t * iterations, double * relres )
{
    TB_TRY( check_handle( h ) );
    if( iterations ) { *iterations = h->ir_iters; }
    if( relres ) { *relres = h->ir_relres; }
    return TB_OK;
}

int tb_chol_precision_in_use( tb_chol * h, std::int32_t * precision, std::int32_t * fell_back )
{
    TB_TRY( check_handle( h ) );
    if( precision ) { *precision = h->precision; }
    if( fell_back ) { *fell_back = h->fell_back ? 1 : 0; }
    return TB_OK;
}

int tb_chol_perturbed_pivots( tb_chol * h, std::int32_t * out )
{
    TB_TRY( check_handle( h ) );
    if( out ) { *out = h->perturbed_pivots; }
    return TB_OK;
}

int tb_chol_set_trace( tb_chol * h, std::int32_t enabled )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( ensure_device( h ) );
    if( enabled )
    {
        TB_TRY( h->trace_buf.reserve( 4 * static_cast<std::int64_t>( h->plan.dag.size() ) ) );
        TB_TRY( h->solve_trace_buf.reserve( 8 * static_cast<std::int64_t>( h->plan.srest.size() ) ) );
    }
    if( (enabled != 0) != h->trace )
    {
        h->trace = enabled != 0;
        if( h->factor_graph ) { cudaGraphExecDestroy( h->factor_graph ); h->factor_graph = nullptr; }
        h->drop_solve_graphs();
    }
    return TB_OK;
}

int tb_chol_trace( tb_chol * h, std::int64_t * out, std::int64_t cap )
{
    TB_TRY( check_handle( h ) );
    if( !h->trace || h->trace_buf.ptr == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "trace not enabled" ); }
    const std::int64_t n = static_cast<std::int64_t>( h->plan.dag.size() );
    if( out == nullptr || cap < 6 * n ) { return fail( TB_ERR_INVALID_ARGUMENT, "trace buffer too small" ); }
    std::vector<unsigned long long> raw( static_cast<size_t>( 4 * n ) );
    TB_CUDA( cudaMemcpyAsync( raw.data(), h->trace_buf.ptr, sizeof(unsigned long long) * raw.size(), cudaMemcpyDeviceToHost, h->stream ) );
    TB_CUDA( cudaStreamSynchronize( h->stream ) );
    for( std::int64_t k = 0; k < n; ++k )
    {
        const tb::DagTask & t = h->plan.dag[static_cast<size_t>( k )];
        out[6 * k + 0] = t.kind;
        out[6 * k + 1] = t.index;
        for( int j = 0; j < 4; ++j ) { out[6 * k + 2 + j] = static_cast<std::int64_t>( raw[static_cast<size_t>( 4 * k + j )] ); }
    }
    return static_cast<int>( std::min<std::int64_t>( n, INT_MAX ) );
}

int tb_chol_solve_trace( tb_chol * h, std::int64_t * out, std::int64_t cap )
{
    TB_TRY( check_handle( h ) );
    if( !h->trace || h->solve_trace_buf.ptr == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "trace not enabled" ); }
    const std::int64_t n = static_cast<std::int64_t>( h->plan.solve_fwd_order.size() );
    if( out == nullptr || cap < 12 * n ) { return fail( TB_ERR_INVALID_ARGUMENT, "trace buffer too small" ); }
    std::vector<unsigned long long> raw( static_cast<size_t>( 8 * n ) );
    if( n > 0 )
    {
        TB_CUDA( cudaMemcpyAsync( raw.data(), h->solve_trace_buf.ptr, sizeof(unsigned long long) * raw.size(),
                                  cudaMemcpyDeviceToHost, h->stream ) );
        TB_CUDA( cudaStreamSynchronize( h->stream ) );
    }
    for( std::int64_t k = 0; k < 2 * n; ++k )
    {
        const int upper = k >= n ? 1 : 0;
        const std::int64_t pos = k - upper * n;
        out[6 * k + 0] = upper;
        out[6 * k + 1] = upper ? h->plan.solve_bwd_order[static_cast<size_t>( pos )] : h->plan.solve_fwd_order[static_cast<size_t>( pos )];
        for( int j = 0; j < 4; ++j ) { out[6 * k + 2 + j] = static_cast<std::int64_t>( raw[static_cast<size_t>( 4 * k + j )] ); }
    }
    return static_cast<int>( std::min<std::int64_t>( 2 * n, INT_MAX ) );
}

int tb_chol_set_profiling( tb_chol * h, std::int32_t enabled )
{
    if( h == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null handle" ); }
    h->profiling = (enabled != 0);
    return TB_OK;
}

int tb_chol_kernel_profile( tb_chol * h, double * ms, std::int64_t * launches, double * flops )
{
    if( h == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null handle" ); }
    for( int k = 0; k < 8; ++k )
    {
        if( ms ) { ms[k] = h->kind_ms[k]; }
        if( launches ) { launches[k] = h->kind_launches[k]; }
        if( flops ) { flops[k] = 0.0; }
    }
    if( flops && h->symbolic_done ) { flops[static_cast<int>( tb::LaunchKind::Gemm )] = h->plan.gemm_flops; }
    return TB_OK;
}

int tb_chol_launch_profile( tb_chol * h, std::int64_t * info, double * ms, std::int32_t cap )
{
    if( h == nullptr || cap < 0 ) { return fail( TB_ERR_INVALID_ARGUMENT, "null handle" ); }
    const std::int32_t m = std::min<std::int32_t>( cap, static_cast<std::int32_t>( h->launch_ms.size() ) );
    for( std::int32_t i = 0; i < m; ++i )
    {
        if( i == 0 )
        {
            if( info ) { info[0] = 7; info[1] = -1; info[2] = -1; info[3] = 1; }
        }
        else if( info )
        {
            // the factor launches, then the super-panel inverse rounds (reported as Invert)
            const std::size_t nf = h->plan.factor_launches.size();
            const std::size_t j = static_cast<std::size_t>( i - 1 );
            const tb::Launch * L = j < nf ? &h->plan.factor_launches[j]
                                          : (j - nf < h->plan.sinv_launches.size() ? &h->plan.sinv_launches[j - nf] : nullptr);
            if( L == nullptr ) { info[4 * i] = -1; info[4 * i + 1] = -1; info[4 * i + 2] = -1; info[4 * i + 3] = 0; }
            else
            {
                const tb::LaunchKind kind = L->kind == tb::LaunchKind::ExtendPull ? tb::LaunchKind::Extend
                                          : L->kind == tb::LaunchKind::SuperInv ? tb::LaunchKind::Invert : L->kind;
                info[4 * i + 0] = static_cast<std::int64_t>( kind );
                info[4 * i + 1] = L->level;
                info[4 * i + 2] = L->step;
                info[4 * i + 3] = L->count;
            }
        }
        if( ms ) { ms[i] = h->launch_ms[static_cast<size_t>( i )]; }
    }
    return m;
}

int tb_chol_solve_profile( tb_chol * h, std::int64_t * info, double * ms, std::int32_t cap )
{
    if( h == nullptr || cap < 0 ) { return fail( TB_ERR_INVALID_ARGUMENT, "null handle" ); }
    const std::int32_t m = std::min<std::int32_t>( cap, static_cast<std::int32_t>( h->solve_ms.size() ) );
    for( std::int32_t i = 0; i < m; ++i )
    {
        if( info ) { for( int j = 0; j < 4; ++j ) { info[4 * i + j] = h->solve_info[static_cast<size_t>( 4 * i + j )]; } }
        if( ms ) { ms[i] = h->solve_ms[static_cast<size_t>( i )]; }
    }
    return m;
}

int tb_chol_launch_counts( tb_chol * h, std::int64_t * factor_launches, std::int64_t * solve_launches )
{
    if( h == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null handle" ); }
    if( factor_launches ) { *factor_launches = h->factor_launch_count; }
    if( solve_launches ) { *solve_launches = h->solve_launch_count; }
    return TB_OK;
}

} // extern "C"

// ---------------------------------------------------------------------------
// Scalar types at the boundary and the numeric-factor container.
// ---------------------------------------------------------------------------

// NumericalFactorization_T (CholeskyDecomposition.hpp:132-201): a numeric
// factor held apart from any handle.  Here it is the device state a
// factorization leaves behind: the front storage (FP64, or FP32 in the
// mixed-precision mode), the inverse diagonal blocks the solves use, the
// matrix values and shift the mixed mode's refinement needs, and the
// factorized / good flags.
struct tb_factor
{
    int device = -1;
    DeviceArray<double> arena, tinv, values;
    int precision = -1;                          // of the stored factor; -1: never held one
    double last_reg = 0.0;
    bool factorized = false, good = false, fell_back = false;
    std::int32_t failed_sn = -1, perturbed_pivots = 0;
};

namespace
{

template<typename T> void swap_arrays( DeviceArray<T> & a, DeviceArray<T> & b )
{
    std::swap( a.ptr, b.ptr );
    std::swap( a.size, b.size );
}

// Device sizes a factor of the handle's symbolic analysis needs, for a precision.
std::int64_t required_arena( const tb_chol * h, int precision )
{
    return precision == TB_PRECISION_MIXED ? (h->plan.arena_size() + 1) / 2 : h->plan.arena_size();
}

} // namespace

extern "C" {

int tb_factor_create( tb_factor ** out )
{
    if( out == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null output" ); }
    *out = new tb_factor();
    return TB_OK;
}

int tb_factor_destroy( tb_factor * f )
{
    int caller = -1;
    if( f != nullptr && f->device >= 0 && cudaGetDevice( &caller ) == cudaSuccess ) { cudaSetDevice( f->device ); }
    delete f;
    if( caller >= 0 ) { cudaSetDevice( caller ); }
    return TB_OK;
}

int tb_factor_state( tb_factor * f, std::int32_t * factorized, std::int32_t * good, std::int64_t * bytes,
                     std::int32_t * precision )
{
    if( f == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "null factor" ); }
    if( factorized ) { *factorized = f->factorized ? 1 : 0; }
    if( good ) { *good = f->good ? 1 : 0; }
    if( bytes ) { *bytes = 8 * (f->arena.size + f->tinv.size + f->values.size); }
    if( precision ) { *precision = f->precision; }
    return TB_OK;
}

int tb_chol_swap_factor( tb_chol * h, tb_factor * f )
{
    TB_TRY( check_handle( h ) );
    if( f == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "SwapNumericalFactorization: null factor" ); }
    if( f->device >= 0 && f->device != h->device )
    {
        return fail( TB_ERR_INVALID_ARGUMENT, "SwapNumericalFactorization: the factor lives on another device" );
    }
    TB_TRY( ensure_symbolic( h ) );
    // captured factor and solve graphs hold the outgoing storage's addresses
    if( h->factor_graph ) { cudaGraphExecDestroy( h->factor_graph ); h->factor_graph = nullptr; }
    h->drop_solve_graphs();
    if( h->device_ready ) { TB_CUDA( cudaSetDevice( h->device ) ); TB_CUDA( cudaStreamSynchronize( h->stream ) ); }
    const int incoming = f->precision;
    swap_arrays( h->arena, f->arena );
    swap_arrays( h->tinv, f->tinv );
    swap_arrays( h->values, f->values );
    std::swap( h->last_reg, f->last_reg );
    std::swap( h->factorized, f->factorized );
    std::swap( h->good, f->good );
    std::swap( h->fell_back, f->fell_back );
    std::swap( h->failed_sn, f->failed_sn );
    std::swap( h->perturbed_pivots, f->perturbed_pivots );
    f->precision = h->precision;
    f->device = h->device;
    if( incoming >= 0 && incoming != h->precision )
    {
        // the factor's storage width: the next factorization re-creates the device plan for it
        h->precision = incoming;
        h->device_ready = false;
    }
    // Numeric.hpp:232-253: a factor marked factorized but not good, or too
    // small for this symbolic analysis, is treated as unfactorized
    if( h->factorized && !h->good ) { h->factorized = false; }
    const std::int64_t need_tinv = static_cast<std::int64_t>( h->plan.sdiag.size() ) * tb::kPanel * tb::kPanel;
    if( h->factorized && (h->arena.size < required_arena( h, h->precision ) || h->tinv.size < need_tinv
                          || h->values.size < h->sym.nnz || h->arena.ptr == nullptr) )
    {
        h->factorized = false;
        h->good = false;
    }
    // a factor to solve with needs the device plan (built here for a handle that never factored);
    // its storage is large enough for it and is kept
    if( h->factorized ) { TB_TRY( ensure_device( h ) ); }
    if( h->device_ready )
    {
        // the device plan stays: storage too small for it is grown (its contents are then moot)
        TB_TRY( h->arena.reserve( required_arena( h, h->precision ) ) );
        TB_TRY( h->tinv.reserve( need_tinv ) );
        TB_TRY( h->values.reserve( h->sym.nnz ) );
    }
    return TB_OK;
}

int tb_chol_solve_ex( tb_chol * h, double alpha, const void * B, std::int32_t ldB, std::int32_t b_dtype,
                      double beta, void * X, std::int32_t ldX, std::int32_t x_dtype, std::int32_t nrhs )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( require_factor( h ) );
    return run_solve_host( h, 2, alpha, B, ldB, b_dtype, beta, X, ldX, x_dtype, nrhs );
}

int tb_chol_solve_device_ex( tb_chol * h, double alpha, const void * d_B, std::int32_t ldB, std::int32_t b_dtype,
                             double beta, void * d_X, std::int32_t ldX, std::int32_t x_dtype, std::int32_t nrhs )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( require_factor( h ) );
    if( d_B == nullptr || d_X == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "Solve: null buffer" ); }
    if( dtype_size( b_dtype ) == 0 || dtype_size( x_dtype ) == 0 ) { return fail( TB_ERR_INVALID_ARGUMENT, "Solve: unknown scalar type" ); }
    const std::int32_t n = h->n;
    const std::int32_t k = std::max( 1, nrhs );
    if( ldB < k || ldX < k ) { return fail( TB_ERR_INVALID_ARGUMENT, "Solve: leading dimension smaller than nrhs" ); }
    if( b_dtype == TB_F64 && x_dtype == TB_F64 )
    {
        return run_solve_device( h, 2, alpha, static_cast<const double *>( d_B ), ldB, beta, static_cast<double *>( d_X ), ldX, nrhs );
    }
    cudaStream_t st = h->stream;
    const double * B = static_cast<const double *>( d_B );
    std::int32_t ldb = ldB;
    if( b_dtype == TB_F32 )
    {
        TB_TRY( h->in.reserve( static_cast<std::int64_t>( n ) * k ) );
        tb::launch_widen( static_cast<const float *>( d_B ), ldB, h->in.ptr, k, n, k, st );
        B = h->in.ptr;
        ldb = k;
    }
    if( x_dtype == TB_F64 ) { return run_solve_device( h, 2, alpha, B, ldb, beta, static_cast<double *>( d_X ), ldX, nrhs ); }
    TB_TRY( h->out.reserve( static_cast<std::int64_t>( n ) * k ) );
    if( beta != 0.0 ) { tb::launch_widen( static_cast<const float *>( d_X ), ldX, h->out.ptr, k, n, k, st ); }
    TB_TRY( run_solve_device( h, 2, alpha, B, ldb, beta, h->out.ptr, k, nrhs ) );
    tb::launch_narrow( h->out.ptr, k, static_cast<float *>( d_X ), ldX, n, k, st );
    TB_CUDA( cudaGetLastError() );
    return TB_OK;
}

} // extern "C"

// ---------------------------------------------------------------------------
// Solve without any device allocation.
//
// Some callers cannot allocate device memory at solve time: a real-time loop
// that has reserved everything up front and must not stall in the allocator,
// a memory-capped serving process that admits work only against a fixed
// budget, or code running while another component owns the allocator.
// tb_chol_solve_device grows a per-handle work block on first use (and when
// nrhs grows), which such callers cannot allow.  tb_chol_solve_device_noalloc
// runs the same gather, forward/back sweeps and scatter, but its permuted
// two work blocks are one fixed, file-scope device array instead.
//
//  - Capacity: n * nrhs <= kNoAllocScratchEntries (4,194,304 doubles per
//    block, 64 MiB for both); larger requests are rejected with
//    TB_ERR_INVALID_ARGUMENT before anything is launched.
//  - Set-up: the first call on a device looks up the array's device address
//    with cudaGetSymbolAddress (that device current) and caches it; make
//    that first call outside any stream capture.
//  - Nothing in the array has to start at zero: the gather writes every
//    entry the forward sweep reads, and the back sweep clears the block it
//    accumulates into.
//  - There is one array per device, shared by every handle: calls whose
//    solves can overlap on the device (other streams, other host threads)
//    race on it and must be serialised by the caller.
//  - It applies the FP64 factor once (the direct solve).  A mixed-precision
//    handle, or one that fell back to FP64 after a failed refinement, is
//    solved by refinement with more work vectors than this array holds, so
//    such handles are rejected with TB_ERR_INVALID_ARGUMENT.
//  - The sweeps always run as level launches, whatever the handle's solve
//    schedule: they contain no waits, so this path cannot time out.
//  - The array is part of the library's device code: with lazy module
//    loading (the CUDA default) it takes device memory once the first call
//    looks it up; with CUDA_MODULE_LOADING=EAGER every context that loads the
//    library holds the 64 MiB from the start.
// ---------------------------------------------------------------------------
namespace
{

constexpr std::int64_t kNoAllocScratchEntries = std::int64_t( 1 ) << 22;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__( 256 ) double g_noalloc_scratch[2 * kNoAllocScratchEntries];

std::mutex g_noalloc_mutex;
double * g_noalloc_ptr[kNoAllocMaxDevices] = {};

int noalloc_scratch( int device, double ** out )
{
    if( device < 0 || device >= kNoAllocMaxDevices ) { return fail( TB_ERR_INVALID_ARGUMENT, "device ordinal out of range" ); }
    std::lock_guard<std::mutex> lock( g_noalloc_mutex );
    if( g_noalloc_ptr[device] == nullptr )
    {
        // the symbol resolves on the current device: make it the handle's,
        // then give the caller back the device it had current
        int caller = 0;
        TB_CUDA( cudaGetDevice( &caller ) );
        void * p = nullptr;
        cudaError_t e = cudaSetDevice( device );
        if( e == cudaSuccess ) { e = cudaGetSymbolAddress( &p, g_noalloc_scratch ); }
        const cudaError_t back = cudaSetDevice( caller );
        if( e != cudaSuccess )
        {
            return fail( TB_ERR_CUDA, std::string( "solve_device_noalloc: looking up the fixed scratch: " ) + cudaGetErrorString( e ) );
        }
        if( back != cudaSuccess )
        {
            return fail( TB_ERR_CUDA, std::string( "solve_device_noalloc: restoring the current device: " ) + cudaGetErrorString( back ) );
        }
        g_noalloc_ptr[device] = static_cast<double *>( p );
    }
    *out = g_noalloc_ptr[device];
    return TB_OK;
}

} // namespace

extern "C" {

int tb_chol_solve_device_noalloc( tb_chol * h, double alpha, const double * d_B, std::int32_t ldB,
                                  double beta, double * d_X, std::int32_t ldX, std::int32_t nrhs )
{
    TB_TRY( check_handle( h ) );
    TB_TRY( require_factor( h ) );
    if( d_B == nullptr || d_X == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "Solve: null buffer" ); }
    if( h->precision == TB_PRECISION_MIXED || h->fell_back )
    {
        return fail( TB_ERR_INVALID_ARGUMENT, "solve_device_noalloc: the handle solves by refinement (mixed precision, "
                     "or FP64 after a failed refinement), which needs work vectors beyond the fixed scratch; "
                     "use tb_chol_solve_device" );
    }
    const std::int32_t n = h->n;
    const std::int32_t k = std::max( 1, nrhs );
    if( ldB < k || ldX < k ) { return fail( TB_ERR_INVALID_ARGUMENT, "Solve: leading dimension smaller than nrhs" ); }
    if( static_cast<std::int64_t>( n ) * k > kNoAllocScratchEntries )
    {
        return fail( TB_ERR_INVALID_ARGUMENT, "solve_device_noalloc: n * nrhs = " +
                     std::to_string( static_cast<std::int64_t>( n ) * k ) + " exceeds the fixed scratch of " +
                     std::to_string( kNoAllocScratchEntries ) + " doubles per block" );
    }
    double * W = nullptr;
    TB_TRY( noalloc_scratch( h->device, &W ) );
    double * Y = W + kNoAllocScratchEntries;
    cudaStream_t st = h->stream;
    std::int64_t launches = 2;
    tb::launch_gather_rows( d_B, ldB, h->p.ptr, W, k, n, k, st );
    launches += issue_sweeps( h, 2, W, Y, k, false, true );
    tb::launch_scatter_rows( W, k, h->p_inv.ptr, alpha, beta, d_X, ldX, n, k, st );
    h->solve_launch_count = launches;
    TB_CUDA( cudaGetLastError() );
    return TB_OK;
}

} // extern "C"
