// FP64 kernels of the supernodal factorization and solves (sm_100a).
//
// Every kernel consumes a flat task array built by Plan::build (plan.cpp):
// one CTA per task, no inter-CTA dependencies inside a launch, so a level's
// work for all of its supernodes is a handful of launches regardless of how
// many supernodes it has.  FP64 has no tcgen05 MMA kind, so the FP64 tile
// products use DMMA (mma.sync.m8n8k4.f64), the only FP64 tensor-core path on
// Blackwell.

#include "kernels.cuh"

#include <climits>

namespace tb
{
namespace
{

constexpr int kGemmThreads  = 128;
constexpr int kGemmK        = 16;
constexpr int kGemmLd       = kTile + 4;   // padded smem row (2 wavefronts per fragment load)
constexpr int kPanelThreads = kRestChunk;
constexpr int kSolveThreads = 256;
constexpr int kMaxRhs       = kSolveMaxRhs;   // columns per solve launch

__device__ __forceinline__ void dmma_8x8x4( double (&d)[2], double a, double b )
{
    asm volatile( "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                  : "+d"(d[0]), "+d"(d[1]) : "d"(a), "d"(b) );
}

// ---------------------------------------------------------------- assembly
// arena[dst] = values[src] (+ reg on the diagonal): ReadNonzeroValues
// (Numeric.hpp:165-180) fused with FetchFromA (Multifrontal.hpp:249-321).
__global__ void assemble_kernel( const double * __restrict__ values, const std::int64_t * __restrict__ src,
                                 const std::int64_t * __restrict__ dst, std::int64_t count,
                                 const double * __restrict__ reg, double * __restrict__ arena )
{
    const double r = *reg;
    for( std::int64_t e = blockIdx.x * (std::int64_t)blockDim.x + threadIdx.x; e < count;
         e += (std::int64_t)gridDim.x * blockDim.x )
    {
        const std::uint64_t d = static_cast<std::uint64_t>( dst[e] );
        double v = values[src[e]];
        if( d & kDiagFlag ) { v += r; }
        arena[d & (kDiagFlag - 1)] = v;
    }
}

// ------------------------------------------------------------------ zeroing
__global__ void zero_kernel( const ZeroTask * __restrict__ tasks, double * __restrict__ arena )
{
    const ZeroTask t = tasks[blockIdx.x];
    double * p = arena + t.offset;
    std::int64_t i = threadIdx.x;
    // align to 16 bytes, then store double2
    const int head = static_cast<int>( (reinterpret_cast<std::uintptr_t>( p ) >> 3) & 1 );
    if( head && threadIdx.x == 0 && t.count > 0 ) { p[0] = 0.0; }
    const std::int64_t body = (t.count - head) / 2;
    double2 * q = reinterpret_cast<double2 *>( p + head );
    for( ; i < body; i += blockDim.x ) { q[i] = make_double2( 0.0, 0.0 ); }
    const std::int64_t tail = head + 2 * body;
    if( threadIdx.x == 0 && tail < t.count ) { p[tail] = 0.0; }
}

// ---------------------------------------------------------------- export
// Reference layout from the fronts: U0 of supernode s is the diagonal block
// of its front at row offset roff; column l of its U1 is front U0 column
// colmap[l] (>= 0) or front U1 column -colmap[l]-1.
__global__ void export_kernel( const ExportTask * __restrict__ tasks, const std::int32_t * __restrict__ colmap_all,
                               const double * __restrict__ arena, double * __restrict__ tri, double * __restrict__ rec )
{
    const ExportTask t = tasks[blockIdx.x];
    const std::int32_t * colmap = colmap_all + t.colmap;
    for( int r = t.r_begin; r < t.r_end; ++r )
    {
        const std::int64_t fr = t.roff + r;
        const double * f0 = arena + t.fu0 + fr * t.fld0;
        const double * f1 = arena + t.fu1 + fr * t.fld1;
        double * d0 = tri + t.tri + (std::int64_t)r * t.n0s;
        for( int c = threadIdx.x; c < t.n0s; c += blockDim.x ) { d0[c] = (c >= r) ? f0[t.roff + c] : 0.0; }
        double * d1 = rec + t.rec + (std::int64_t)r * t.n1s;
        for( int l = threadIdx.x; l < t.n1s; l += blockDim.x )
        {
            const int cm = colmap[l];
            d1[l] = (cm >= 0) ? f0[cm] : f1[-cm - 1];
        }
    }
}

// ------------------------------------------------------------- extend-add
// One warp per row of the child's update W; lanes walk the row's upper part
// (coalesced reads of W, lut-indexed adds into the parent front).
__global__ __launch_bounds__(256) void extend_kernel( const ExtendTask * __restrict__ tasks,
                                                      const std::int32_t * __restrict__ lut_all,
                                                      double * __restrict__ arena )
{
    const ExtendTask t = tasks[blockIdx.x];
    const std::int32_t * lut = lut_all + t.lut;
    const double * W = arena + t.w;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    for( int i = t.row_begin + warp; i < t.row_end; i += 8 )
    {
        const std::int64_t li = lut[i];
        const double * Wi = W + (std::int64_t)i * t.ldw;
        if( i < t.mid )
        {
            double * row0 = arena + t.u0 + li * t.ld0p;
            double * row1 = arena + t.u1 + li * t.ld1p;
            for( int j = i + lane; j < t.m1; j += 32 )
            {
                const int lj = lut[j];
                const double v = Wi[j];
                if( j < t.mid ) { row0[lj] += v; } else { row1[lj] += v; }
            }
        }
        else
        {
            double * rowv = arena + t.v + li * t.ldvp;
            for( int j = i + lane; j < t.m1; j += 32 ) { rowv[lut[j]] += Wi[j]; }
        }
    }
}

// ------------------------------------------------------------------ panel
// Cholesky of a panel's nb x nb diagonal block, in shared memory and then
// in place (LAPACK potrf of FactorizeSupernode, Multifrontal.hpp:438-449).
// A row that forms a 1 x 1 reference supernode takes sqrt(|a|) as the
// reference does (:471) and never reports failure.
// Panel kernels work on the 64 x 64 diagonal block in 8 x 8 sub-blocks:
// sequential 8-step recurrences run in registers (unrolled 8 x 8), and every
// update between sub-blocks is an 8 x 8 x 8 product on the FP64 tensor cores
// (two DMMA m8n8k4).  The outer loops over sub-blocks stay rolled so the code
// fits the instruction cache.
constexpr int kPotrfThreads = 256;
constexpr int kTrsmThreads  = 256;
constexpr int kSub          = 8;                     // sub-block edge
constexpr int kSubs         = kPanel / kSub;         // 8 sub-blocks per panel edge
constexpr int kXld          = kRestChunk + 4;        // padded row of the staged rest columns
constexpr size_t kTrsmSmemBytes = sizeof(double) * (kPanel * (kPanel + 1) + kPanel * kXld);

// C(8x8) += A(8x8) * B(8x8) with A read through a(i, k), B through b(k, j)
// and C through c(i, j) (warp-wide; fragment layouts of mma.m8n8k4.f64).
template<typename FA, typename FB>
__device__ __forceinline__ void dmma_8x8x8( double (&acc)[2], FA a, FB b )
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for( int s = 0; s < 2; ++s )
    {
        dmma_8x8x4( acc, a( lane >> 2, (lane & 3) + 4 * s ), b( (lane & 3) + 4 * s, lane >> 2 ) );
    }
}

__global__ __launch_bounds__(kPotrfThreads) void potrf_kernel( const PanelTask * __restrict__ tasks,
                                                               double * __restrict__ arena, int * __restrict__ status )
{
    const PanelTask t = tasks[blockIdx.x];
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int nb = min( kPanel, t.n0 - t.r0 );
    __shared__ double D[kPanel][kPanel + 1];
    __shared__ double inv_d[kPanel];
    __shared__ int fail;

    double * U0 = arena + t.u0 + (std::int64_t)t.r0 * t.ld0 + t.r0;
    for( int idx = tid; idx < kPanel * kPanel; idx += kPotrfThreads )
    {
        const int r = idx / kPanel, c = idx % kPanel;
        double v = (r == c) ? 1.0 : 0.0;                 // identity padding beyond nb
        if( r < nb && c < nb && r <= c ) { v = U0[(std::int64_t)r * t.ld0 + c]; }
        D[r][c] = v;
    }
    if( tid == 0 ) { fail = -1; }
    __syncthreads();

    const int nsub = (nb + kSub - 1) / kSub;
    for( int b = 0; b < nsub; ++b )
    {
        const int o = b * kSub;
        // (a) Cholesky of the 8 x 8 diagonal sub-block: lane c < 8 holds column c
        if( warp == 0 )
        {
            double a[kSub];
#pragma unroll
            for( int r = 0; r < kSub; ++r ) { a[r] = (lane < kSub && r <= lane) ? D[o + r][o + lane] : 0.0; }
#pragma unroll
            for( int r = 0; r < kSub; ++r )
            {
                double d = __shfl_sync( 0xffffffffu, a[r], r );
                if( lane == 0 )
                {
                    if( (t.single_rows >> (o + r)) & 1 ) { }
                    else if( o + r < nb && !(d > 0.0) && fail < 0 ) { fail = o + r; }
                }
                if( (t.single_rows >> (o + r)) & 1 ) { d = fabs( d ); }
                // reciprocal square root and one product instead of sqrt and a
                // division: both are long dependent sequences on the FP64 pipe
                const double inv = rsqrt( d );
                const double piv = d * inv;
                if( lane == r ) { a[r] = piv; inv_d[o + r] = inv; }
                if( lane > r ) { a[r] *= inv; }                     // U(r, lane)
#pragma unroll
                for( int r2 = r + 1; r2 < kSub; ++r2 )
                {
                    const double urr2 = __shfl_sync( 0xffffffffu, a[r], r2 );   // U(r, r2)
                    if( lane >= r2 ) { a[r2] -= urr2 * a[r]; }
                }
            }
            if( lane < kSub )
            {
#pragma unroll
                for( int r = 0; r < kSub; ++r ) { if( r <= lane ) { D[o + r][o + lane] = a[r]; } }
            }
        }
        __syncthreads();
        // (b) rows o..o+7 of the columns right of the sub-block: U_b,c = L_bb^{-1} A_b,c
        {
            const int col = o + kSub + tid;
            if( col < kPanel )
            {
                double x[kSub];
#pragma unroll
                for( int r = 0; r < kSub; ++r ) { x[r] = D[o + r][col]; }
#pragma unroll
                for( int r = 0; r < kSub; ++r )
                {
                    x[r] *= inv_d[o + r];
#pragma unroll
                    for( int r2 = r + 1; r2 < kSub; ++r2 ) { x[r2] -= D[o + r][o + r2] * x[r]; }
                }
#pragma unroll
                for( int r = 0; r < kSub; ++r ) { D[o + r][col] = x[r]; }
            }
        }
        __syncthreads();
        // (c) trailing sub-blocks (b2, b3), b < b2 <= b3: D -= U_b,b2^T U_b,b3
        {
            const int rem = kSubs - 1 - b;
            const int tiles = rem * (rem + 1) / 2;
            for( int tile = warp; tile < tiles; tile += kPotrfThreads / 32 )
            {
                int b2 = 0, acc_t = tile;
                while( acc_t >= rem - b2 ) { acc_t -= rem - b2; ++b2; }
                const int b3 = b2 + acc_t;
                const int o2 = o + kSub + b2 * kSub, o3 = o + kSub + b3 * kSub;
                double acc[2] = { 0.0, 0.0 };
                dmma_8x8x8( acc, [&]( int i, int k ) { return D[o + k][o2 + i]; },
                                 [&]( int k, int j ) { return D[o + k][o3 + j]; } );
                const int i = lane >> 2, j = 2 * (lane & 3);
                D[o2 + i][o3 + j]     -= acc[0];
                D[o2 + i][o3 + j + 1] -= acc[1];
            }
        }
        __syncthreads();
    }
    for( int idx = tid; idx < nb * nb; idx += kPotrfThreads )
    {
        const int r = idx / nb, c = idx % nb;
        if( r <= c ) { U0[(std::int64_t)r * t.ld0 + c] = D[r][c]; }
    }
    if( tid == 0 && fail >= 0 )
    {
        atomicOr( status, 1 );
        atomicMin( status + 1, t.row0 + t.r0 + fail );
    }
}

// Solve D^T x = u against the factored diagonal block for the rest columns
// [c0, c0 + kRestChunk) (trsm of FactorizeSupernode, Multifrontal.hpp:
// 452-466): the columns are staged in shared memory; per 8-row sub-block,
// one thread per column solves the 8 x 8 triangle in registers, then the
// warps update the rows below with DMMA (warp w owns columns 8w..8w+7).
__global__ __launch_bounds__(kTrsmThreads) void trsm_kernel( const PanelTask * __restrict__ tasks,
                                                             double * __restrict__ arena )
{
    extern __shared__ double tsm[];
    double (*D)[kPanel + 1] = reinterpret_cast<double (*)[kPanel + 1]>( tsm );
    double (*X)[kXld] = reinterpret_cast<double (*)[kXld]>( tsm + kPanel * (kPanel + 1) );
    __shared__ double inv_d[kPanel];
    const PanelTask t = tasks[blockIdx.x];
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int nb = min( kPanel, t.n0 - t.r0 );
    const int r1 = t.r0 + nb;
    const int m = t.n0 - r1;
    const int rest = m + t.n1;
    const int cw = min( kRestChunk, rest - t.c0 );
    double * U0 = arena + t.u0;
    double * U1 = arena + t.u1;
    for( int idx = tid; idx < kPanel * kPanel; idx += kTrsmThreads )
    {
        const int r = idx / kPanel, c = idx % kPanel;
        double v = (r == c) ? 1.0 : 0.0;
        if( r < nb && c < nb && r <= c ) { v = U0[(std::int64_t)(t.r0 + r) * t.ld0 + t.r0 + c]; }
        D[r][c] = v;
    }
    for( int idx = tid; idx < kPanel * kRestChunk; idx += kTrsmThreads )
    {
        const int r = idx / kRestChunk, cc = idx % kRestChunk;
        const int col = t.c0 + cc;
        double v = 0.0;
        if( r < nb && cc < cw )
        {
            v = (col < m) ? U0[(std::int64_t)(t.r0 + r) * t.ld0 + r1 + col]
                          : U1[(std::int64_t)(t.r0 + r) * t.ld1 + (col - m)];
        }
        X[r][cc] = v;
    }
    __syncthreads();
    if( tid < kPanel ) { inv_d[tid] = 1.0 / D[tid][tid]; }
    __syncthreads();
    const int nsub = (nb + kSub - 1) / kSub;
    for( int b = 0; b < nsub; ++b )
    {
        const int o = b * kSub;
        if( tid < kRestChunk )
        {
            double x[kSub];
#pragma unroll
            for( int r = 0; r < kSub; ++r ) { x[r] = X[o + r][tid]; }
#pragma unroll
            for( int r = 0; r < kSub; ++r )
            {
                x[r] *= inv_d[o + r];
#pragma unroll
                for( int r2 = r + 1; r2 < kSub; ++r2 ) { x[r2] -= D[o + r][o + r2] * x[r]; }
            }
#pragma unroll
            for( int r = 0; r < kSub; ++r ) { X[o + r][tid] = x[r]; }
        }
        __syncthreads();
        for( int b2 = b + 1; b2 < nsub; ++b2 )
        {
            const int o2 = b2 * kSub;
            for( int ct = warp; ct < kRestChunk / kSub; ct += kTrsmThreads / 32 )
            {
                const int cb = ct * kSub;
                double acc[2] = { 0.0, 0.0 };
                dmma_8x8x8( acc, [&]( int i, int k ) { return D[o + k][o2 + i]; },
                                 [&]( int k, int j ) { return X[o + k][cb + j]; } );
                const int i = lane >> 2, j = 2 * (lane & 3);
                X[o2 + i][cb + j]     -= acc[0];
                X[o2 + i][cb + j + 1] -= acc[1];
            }
        }
        __syncthreads();
    }
    for( int idx = tid; idx < nb * kRestChunk; idx += kTrsmThreads )
    {
        const int r = idx / kRestChunk, cc = idx % kRestChunk;
        const int col = t.c0 + cc;
        if( cc < cw )
        {
            if( col < m ) { U0[(std::int64_t)(t.r0 + r) * t.ld0 + r1 + col] = X[r][cc]; }
            else          { U1[(std::int64_t)(t.r0 + r) * t.ld1 + (col - m)] = X[r][cc]; }
        }
    }
}

// ------------------------------------------------------------------- gemm
// C[m0:m0+64, c0:c0+64] -= A[:, m0:]^T B[:, c0:] for row-major K x M / K x N
// panels: 4 warps in a 2 x 2 arrangement, each a 32 x 32 block of 8 x 8
// DMMA tiles.  K is streamed through a kGemmStages-deep ring of shared-memory
// stages filled by 16-byte cp.async copies (every operand row starts on a
// 16-byte boundary: the plan pads leading dimensions to kLdAlign), so the
// copies of the next chunks overlap the MMAs of the current one.
constexpr int kGemmStages = 3;
constexpr int kGemmStageDoubles = 2 * kGemmK * kGemmLd;          // A and B of one stage
constexpr size_t kGemmSmemBytes = sizeof(double) * kGemmStages * kGemmStageDoubles;

__device__ __forceinline__ void cp_async_16( double * smem_dst, const double * gmem_src, int src_bytes )
{
    const unsigned saddr = static_cast<unsigned>( __cvta_generic_to_shared( smem_dst ) );
    asm volatile( "cp.async.cg.shared.global [%0], [%1], 16, %2;\n" :: "r"(saddr), "l"(gmem_src), "r"(src_bytes) );
}
__device__ __forceinline__ void cp_async_commit() { asm volatile( "cp.async.commit_group;\n" ::: "memory" ); }
template<int N> __device__ __forceinline__ void cp_async_wait() { asm volatile( "cp.async.wait_group %0;\n" :: "n"(N) : "memory" ); }

__global__ __launch_bounds__(kGemmThreads) void gemm_tn_kernel( const GemmTask * __restrict__ tasks,
                                                                double * __restrict__ arena )
{
    extern __shared__ __align__(16) double gsm[];
    const GemmTask t = tasks[blockIdx.x];
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int wm = warp >> 1, wn = warp & 1;
    const double * A = arena + t.a;
    const double * B = arena + t.b;

    double acc[4][4][2];
#pragma unroll
    for( int i = 0; i < 4; ++i )
#pragma unroll
        for( int j = 0; j < 4; ++j ) { acc[i][j][0] = 0.0; acc[i][j][1] = 0.0; }

    // Each stage holds kGemmK rows of 64 doubles for A and for B = 512
    // 16-byte chunks per operand; thread tid copies chunks tid + 128 * l.
    constexpr int kChunks = kGemmK * kTile / 2 / kGemmThreads;       // 4 per operand
    auto issue = [&]( int stage, int k0 )
    {
        double * As = gsm + stage * kGemmStageDoubles;
        double * Bs = As + kGemmK * kGemmLd;
#pragma unroll
        for( int l = 0; l < kChunks; ++l )
        {
            const int idx = tid + kGemmThreads * l;
            const int r = idx / (kTile / 2), c = 2 * (idx % (kTile / 2));
            const int k = k0 + r;
            const int am = t.M - (t.m0 + c), bn = t.N - (t.c0 + c);
            const int abytes = (k < t.K) ? (am >= 2 ? 16 : (am == 1 ? 8 : 0)) : 0;
            const int bbytes = (k < t.K) ? (bn >= 2 ? 16 : (bn == 1 ? 8 : 0)) : 0;
            cp_async_16( As + r * kGemmLd + c, abytes ? A + (std::int64_t)k * t.lda + t.m0 + c : A, abytes );
            cp_async_16( Bs + r * kGemmLd + c, bbytes ? B + (std::int64_t)k * t.ldb + t.c0 + c : B, bbytes );
        }
    };

    const int nk = (t.K + kGemmK - 1) / kGemmK;
#pragma unroll
    for( int s = 0; s < kGemmStages - 1; ++s )
    {
        if( s < nk ) { issue( s, s * kGemmK ); }
        cp_async_commit();
    }
    for( int kc = 0; kc < nk; ++kc )
    {
        cp_async_wait<kGemmStages - 2>();
        __syncthreads();
        {
            const int nxt = kc + kGemmStages - 1;
            if( nxt < nk ) { issue( nxt % kGemmStages, nxt * kGemmK ); }
            cp_async_commit();
        }
        const double * As = gsm + (kc % kGemmStages) * kGemmStageDoubles;
        const double * Bs = As + kGemmK * kGemmLd;
#pragma unroll
        for( int kk = 0; kk < kGemmK; kk += 4 )
        {
            double af[4], bf[4];
#pragma unroll
            for( int i = 0; i < 4; ++i ) { af[i] = As[(kk + (lane & 3)) * kGemmLd + wm * 32 + i * 8 + (lane >> 2)]; }
#pragma unroll
            for( int j = 0; j < 4; ++j ) { bf[j] = Bs[(kk + (lane & 3)) * kGemmLd + wn * 32 + j * 8 + (lane >> 2)]; }
#pragma unroll
            for( int i = 0; i < 4; ++i )
#pragma unroll
                for( int j = 0; j < 4; ++j ) { dmma_8x8x4( acc[i][j], af[i], bf[j] ); }
        }
    }
    cp_async_wait<0>();

    double * C = arena + t.c;
#pragma unroll
    for( int i = 0; i < 4; ++i )
    {
        const int row = t.m0 + wm * 32 + i * 8 + (lane >> 2);
        if( row >= t.M ) { continue; }
        double * Crow = C + (std::int64_t)row * t.ldc;
#pragma unroll
        for( int j = 0; j < 4; ++j )
        {
            const int col = t.c0 + wn * 32 + j * 8 + (lane & 3) * 2;
            const bool ok0 = col < t.N && (!t.upper || row <= col);
            const bool ok1 = col + 1 < t.N && (!t.upper || row <= col + 1);
            if( ok0 && ok1 )
            {
                double2 v = *reinterpret_cast<const double2 *>( Crow + col );
                v.x -= acc[i][j][0];
                v.y -= acc[i][j][1];
                *reinterpret_cast<double2 *>( Crow + col ) = v;
            }
            else
            {
                if( ok0 ) { Crow[col] -= acc[i][j][0]; }
                if( ok1 ) { Crow[col + 1] -= acc[i][j][1]; }
            }
        }
    }
}

// ------------------------------------------------------------------ solves
// Triangular solve with a panel's diagonal block for the panel's rows of X
// (k <= 64 columns): D^T x = b forward (LowerSolver.hpp:183-197) or
// D x = b backward (UpperSolver.hpp:190-200).
__global__ __launch_bounds__(kSolveThreads) void solve_diag_kernel( const SolveDiagTask * __restrict__ tasks, int upper,
                                                                    const double * __restrict__ arena,
                                                                    double * __restrict__ X, int ldx, int k )
{
    extern __shared__ double smem[];
    double (*D)[kPanel + 1] = reinterpret_cast<double (*)[kPanel + 1]>( smem );
    double * Xs = smem + kPanel * (kPanel + 1);        // [kPanel][k]
    const SolveDiagTask t = tasks[blockIdx.x];
    const int tid = threadIdx.x;
    const int nb = min( kPanel, t.n0 - t.r0 );
    // thread -> (row group g, column c); groups cover rows g, g+G, g+2G, ...
    const int c = tid % k;
    const int g = tid / k;
    const int G = kSolveThreads / k;
    const double * U0 = arena + t.u0 + (std::int64_t)t.r0 * t.ld0 + t.r0;
    for( int r = tid / kPanel; r < nb; r += kSolveThreads / kPanel )
    {
        const int cc = tid % kPanel;
        if( cc < nb ) { D[r][cc] = (cc >= r) ? U0[(std::int64_t)r * t.ld0 + cc] : 0.0; }
    }
    const std::int64_t row_base = (std::int64_t)t.row0 + t.r0;
    if( g < G )
    {
        for( int r = g; r < nb; r += G ) { Xs[r * k + c] = X[(row_base + r) * ldx + c]; }
    }
    __syncthreads();
    if( !upper )
    {
        for( int r = 0; r < nb; ++r )
        {
            if( tid < k ) { Xs[r * k + tid] /= D[r][r]; }
            __syncthreads();
            if( g < G )
            {
                const double xr = Xs[r * k + c];
                for( int r2 = r + 1 + g; r2 < nb; r2 += G ) { Xs[r2 * k + c] -= D[r][r2] * xr; }
            }
            __syncthreads();
        }
    }
    else
    {
        for( int r = nb - 1; r >= 0; --r )
        {
            if( tid < k ) { Xs[r * k + tid] /= D[r][r]; }
            __syncthreads();
            if( g < G )
            {
                const double xr = Xs[r * k + c];
                for( int r2 = g; r2 < r; r2 += G ) { Xs[r2 * k + c] -= D[r2][r] * xr; }
            }
            __syncthreads();
        }
    }
    if( g < G )
    {
        for( int r = g; r < nb; r += G ) { X[(row_base + r) * ldx + c] = Xs[r * k + c]; }
    }
}

// The rest of a panel in the solves.  Forward: X[rest] -= P^T X_panel, with
// rows of the supernode itself updated in place and ancestor rows (through
// SN_inner) by atomic adds, since other supernodes of the level may target
// them (LowerSolver.hpp:199-231).  Backward: X_panel -= P X[rest] gathered
// from final rows (UpperSolver.hpp:151-188), reduced over rest chunks by
// atomic adds.
__global__ __launch_bounds__(kSolveThreads) void solve_rest_kernel( const SolveRestTask * __restrict__ tasks, int upper,
                                                                    const double * __restrict__ arena,
                                                                    const std::int32_t * __restrict__ sn_inner,
                                                                    double * __restrict__ X, int ldx, int k )
{
    extern __shared__ double smem[];
    double (*P)[kSolveRest + 1] = reinterpret_cast<double (*)[kSolveRest + 1]>( smem );   // [kPanel][kSolveRest+1]
    double * Xs = smem + kPanel * (kSolveRest + 1);
    __shared__ std::int64_t trow[kSolveRest];
    const SolveRestTask t = tasks[blockIdx.x];
    const int tid = threadIdx.x;
    const int nb = min( kPanel, t.n0 - t.r0 );
    const int r1 = t.r0 + nb;
    const int m = t.n0 - r1;
    const int cw = t.c1 - t.c0;
    const int c = tid % k;
    const int g = tid / k;
    const int G = kSolveThreads / k;
    const double * U0 = arena + t.u0;
    const double * U1 = arena + t.u1;
    {
        const int jj = tid % kSolveRest;
        const int j = t.c0 + jj;
        if( jj < cw )
        {
            const double * src = (j < m) ? U0 + (std::int64_t)t.r0 * t.ld0 + r1 + j
                                         : U1 + (std::int64_t)t.r0 * t.ld1 + (j - m);
            const std::int64_t ld = (j < m) ? t.ld0 : t.ld1;
            for( int i = tid / kSolveRest; i < nb; i += kSolveThreads / kSolveRest ) { P[i][jj] = src[i * ld]; }
            if( tid < kSolveRest )
            {
                trow[jj] = (j < m) ? (std::int64_t)t.row0 + r1 + j : (std::int64_t)sn_inner[t.inner + (j - m)];
            }
        }
    }
    const std::int64_t panel_row = (std::int64_t)t.row0 + t.r0;
    if( !upper )
    {
        if( g < G )
        {
            for( int i = g; i < nb; i += G ) { Xs[i * k + c] = X[(panel_row + i) * ldx + c]; }
        }
        __syncthreads();
        if( g < G )
        {
            for( int jj = g; jj < cw; jj += G )
            {
                double acc = 0.0;
                for( int i = 0; i < nb; ++i ) { acc += P[i][jj] * Xs[i * k + c]; }
                double * dst = X + trow[jj] * ldx + c;
                if( t.c0 + jj < m ) { *dst -= acc; } else { atomicAdd( dst, -acc ); }
            }
        }
    }
    else
    {
        __syncthreads();
        if( g < G )
        {
            for( int jj = g; jj < cw; jj += G ) { Xs[jj * k + c] = X[trow[jj] * ldx + c]; }
        }
        __syncthreads();
        if( g < G )
        {
            for( int i = g; i < nb; i += G )
            {
                double acc = 0.0;
                for( int jj = 0; jj < cw; ++jj ) { acc += P[i][jj] * Xs[jj * k + c]; }
                atomicAdd( X + (panel_row + i) * ldx + c, -acc );
            }
        }
    }
}

// ------------------------------------------------------ permutations, SpMV
__global__ void gather_rows_kernel( const double * __restrict__ B, int ldB, const std::int32_t * __restrict__ p,
                                    double * __restrict__ W, int ldw, int n, int k )
{
    const std::int64_t total = (std::int64_t)n * k;
    for( std::int64_t e = blockIdx.x * (std::int64_t)blockDim.x + threadIdx.x; e < total;
         e += (std::int64_t)gridDim.x * blockDim.x )
    {
        const std::int64_t i = e / k;
        const int c = static_cast<int>( e % k );
        W[i * ldw + c] = B[(std::int64_t)p[i] * ldB + c];
    }
}

__global__ void scatter_rows_kernel( const double * __restrict__ W, int ldw, const std::int32_t * __restrict__ p_inv,
                                     double alpha, double beta, double * __restrict__ Y, int ldY, int n, int k )
{
    const std::int64_t total = (std::int64_t)n * k;
    for( std::int64_t e = blockIdx.x * (std::int64_t)blockDim.x + threadIdx.x; e < total;
         e += (std::int64_t)gridDim.x * blockDim.x )
    {
        const std::int64_t i = e / k;
        const int c = static_cast<int>( e % k );
        double y = (alpha == 0.0) ? 0.0 : alpha * W[(std::int64_t)p_inv[i] * ldw + c];
        if( beta != 0.0 ) { y += beta * Y[i * ldY + c]; }
        Y[i * ldY + c] = y;
    }
}

// R = B - A X, one warp per row, lanes over the row's entries.
__global__ void residual_kernel( int n, const std::int64_t * __restrict__ outer, const std::int32_t * __restrict__ inner,
                                 const double * __restrict__ vals, const double * __restrict__ X,
                                 const double * __restrict__ B, double * __restrict__ R, int k )
{
    const int lane = threadIdx.x & 31;
    const std::int64_t warp = (blockIdx.x * (std::int64_t)blockDim.x + threadIdx.x) >> 5;
    const std::int64_t warps = ((std::int64_t)gridDim.x * blockDim.x) >> 5;
    for( std::int64_t i = warp; i < n; i += warps )
    {
        for( int c = 0; c < k; ++c )
        {
            double s = 0.0;
            for( std::int64_t e = outer[i] + lane; e < outer[i+1]; e += 32 ) { s += vals[e] * X[(std::int64_t)inner[e] * k + c]; }
#pragma unroll
            for( int o = 16; o > 0; o >>= 1 ) { s += __shfl_xor_sync( 0xffffffffu, s, o ); }
            if( lane == 0 ) { R[i * k + c] = B[i * k + c] - s; }
        }
    }
}

__global__ void gather_diag_kernel( const std::int64_t * __restrict__ offsets, const double * __restrict__ arena,
                                    double * __restrict__ out, int n )
{
    for( std::int64_t i = blockIdx.x * (std::int64_t)blockDim.x + threadIdx.x; i < n; i += (std::int64_t)gridDim.x * blockDim.x )
    {
        out[i] = arena[offsets[i]];
    }
}

__global__ void init_status_kernel( int * status )
{
    status[0] = 0;
    status[1] = INT_MAX;
}

int grid_for( std::int64_t work, int threads )
{
    const std::int64_t blocks = (work + threads - 1) / threads;
    return static_cast<int>( blocks < 1 ? 1 : (blocks > 148 * 32 ? 148 * 32 : blocks) );
}

} // namespace

void launch_assemble( const double * values, const std::int64_t * src, const std::int64_t * dst,
                      std::int64_t count, const double * reg, double * arena, cudaStream_t st )
{
    if( count <= 0 ) { return; }
    assemble_kernel<<<grid_for( count, 256 ), 256, 0, st>>>( values, src, dst, count, reg, arena );
}

void launch_zero( const ZeroTask * tasks, int count, double * arena, cudaStream_t st )
{
    if( count > 0 ) { zero_kernel<<<count, 256, 0, st>>>( tasks, arena ); }
}

void launch_export( const ExportTask * tasks, int count, const std::int32_t * colmap, const double * arena,
                    double * tri, double * rec, cudaStream_t st )
{
    if( count > 0 ) { export_kernel<<<count, 128, 0, st>>>( tasks, colmap, arena, tri, rec ); }
}

void launch_extend( const ExtendTask * tasks, int count, const std::int32_t * lut, double * arena, cudaStream_t st )
{
    if( count > 0 ) { extend_kernel<<<count, 256, 0, st>>>( tasks, lut, arena ); }
}

void launch_potrf( const PanelTask * tasks, int count, double * arena, int * status, cudaStream_t st )
{
    if( count > 0 ) { potrf_kernel<<<count, kPotrfThreads, 0, st>>>( tasks, arena, status ); }
}

void launch_trsm( const PanelTask * tasks, int count, double * arena, cudaStream_t st )
{
    if( count > 0 ) { trsm_kernel<<<count, kTrsmThreads, kTrsmSmemBytes, st>>>( tasks, arena ); }
}

void launch_gemm( const GemmTask * tasks, int count, double * arena, cudaStream_t st )
{
    if( count > 0 ) { gemm_tn_kernel<<<count, kGemmThreads, kGemmSmemBytes, st>>>( tasks, arena ); }
}

void launch_solve_diag( const SolveDiagTask * tasks, int count, bool upper, const double * arena,
                        double * X, int ldx, int k, cudaStream_t st )
{
    if( count <= 0 ) { return; }
    const size_t smem = sizeof(double) * (kPanel * (kPanel + 1) + kPanel * kMaxRhs);
    solve_diag_kernel<<<count, kSolveThreads, smem, st>>>( tasks, upper ? 1 : 0, arena, X, ldx, k );
}

void launch_solve_rest( const SolveRestTask * tasks, int count, bool upper, const double * arena,
                        const std::int32_t * sn_inner, double * X, int ldx, int k, cudaStream_t st )
{
    if( count <= 0 ) { return; }
    const size_t smem = sizeof(double) * (kPanel * (kSolveRest + 1) + kSolveRest * kMaxRhs);
    solve_rest_kernel<<<count, kSolveThreads, smem, st>>>( tasks, upper ? 1 : 0, arena, sn_inner, X, ldx, k );
}

void launch_gather_rows( const double * B, int ldB, const std::int32_t * p, double * W, int ldw,
                         int n, int k, cudaStream_t st )
{
    gather_rows_kernel<<<grid_for( (std::int64_t)n * k, 256 ), 256, 0, st>>>( B, ldB, p, W, ldw, n, k );
}

void launch_scatter_rows( const double * W, int ldw, const std::int32_t * p_inv, double alpha, double beta,
                          double * Y, int ldY, int n, int k, cudaStream_t st )
{
    scatter_rows_kernel<<<grid_for( (std::int64_t)n * k, 256 ), 256, 0, st>>>( W, ldw, p_inv, alpha, beta, Y, ldY, n, k );
}

void launch_residual( int n, const std::int64_t * outer, const std::int32_t * inner, const double * vals,
                      const double * X, const double * B, double * R, int k, cudaStream_t st )
{
    residual_kernel<<<grid_for( (std::int64_t)n * 32, 256 ), 256, 0, st>>>( n, outer, inner, vals, X, B, R, k );
}

cudaError_t configure_kernels()
{
    {
        const cudaError_t g = cudaFuncSetAttribute( trsm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                    (int)kTrsmSmemBytes );
        if( g != cudaSuccess ) { return g; }
    }
    {
        const cudaError_t g = cudaFuncSetAttribute( gemm_tn_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                    (int)kGemmSmemBytes );
        if( g != cudaSuccess ) { return g; }
    }
    cudaError_t e = cudaFuncSetAttribute( solve_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)( sizeof(double) * (kPanel * (kPanel + 1) + kPanel * kMaxRhs) ) );
    if( e != cudaSuccess ) { return e; }
    return cudaFuncSetAttribute( solve_rest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)( sizeof(double) * (kPanel * (kSolveRest + 1) + kSolveRest * kMaxRhs) ) );
}

void launch_gather_diag( const std::int64_t * offsets, const double * arena, double * out, int n, cudaStream_t st )
{
    gather_diag_kernel<<<grid_for( n, 256 ), 256, 0, st>>>( offsets, arena, out, n );
}

void launch_init_status( int * status, cudaStream_t st )
{
    init_status_kernel<<<1, 1, 0, st>>>( status );
}

} // namespace tb
