// FP64 kernels of the supernodal factorization and solves (sm_100a).
//
// Every kernel consumes a flat task array built by Plan::build (plan.cpp):
// one CTA per task, no inter-CTA dependencies inside a launch, so a level's
// work for all of its supernodes is a handful of launches regardless of how
// many supernodes it has.  FP64 has no tcgen05 MMA kind, so the FP64 tile
// products use DMMA (mma.sync.m8n8k4.f64), the only FP64 tensor-core path on
// Blackwell.

#include "kernels.cuh"

#include <algorithm>
#include <climits>
#include <type_traits>

namespace tb
{
namespace
{

constexpr int kGemmThreads  = 256;
constexpr int kGemmK        = 16;
constexpr int kGemmLd       = kTile + 4;   // padded smem row (2 wavefronts per fragment load)
constexpr int kSolveThreads = 256;

__device__ __forceinline__ void dmma_8x8x4( double (&d)[2], double a, double b )
{
    asm volatile( "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                  : "+d"(d[0]), "+d"(d[1]) : "d"(a), "d"(b) );
}

__device__ __forceinline__ void cp_async_16( void * smem_dst, const void * gmem_src, int src_bytes )
{
    const unsigned saddr = static_cast<unsigned>( __cvta_generic_to_shared( smem_dst ) );
    asm volatile( "cp.async.cg.shared.global [%0], [%1], 16, %2;\n" :: "r"(saddr), "l"(gmem_src), "r"(src_bytes) );
}
__device__ __forceinline__ void cp_async_commit() { asm volatile( "cp.async.commit_group;\n" ::: "memory" ); }
template<int N> __device__ __forceinline__ void cp_async_wait() { asm volatile( "cp.async.wait_group %0;\n" :: "n"(N) : "memory" ); }

// 8-byte asynchronous copy global -> shared, zero-filled when !valid (the
// source address is then not read, but must still be a mapped address).
// Tile loads are issued this way so that all of a thread's copies are in
// flight at once instead of one load-then-store round trip per element.
__device__ __forceinline__ void cp_async_8( double * smem_dst, const double * gmem_src, bool valid )
{
    const unsigned saddr = static_cast<unsigned>( __cvta_generic_to_shared( smem_dst ) );
    asm volatile( "cp.async.ca.shared.global [%0], [%1], 8, %2;\n" :: "r"(saddr), "l"(gmem_src), "r"(valid ? 8 : 0) );
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile( "cp.async.wait_all;\n" ::: "memory" ); }

__device__ __forceinline__ void cp_async_4( void * smem_dst, const void * gmem_src, bool valid )
{
    const unsigned saddr = static_cast<unsigned>( __cvta_generic_to_shared( smem_dst ) );
    asm volatile( "cp.async.ca.shared.global [%0], [%1], 4, %2;\n" :: "r"(saddr), "l"(gmem_src), "r"(valid ? 4 : 0) );
}

// Stages kIters elements per thread (element idx = threadIdx.x + u * kThreads)
// of a factor block into double shared-memory cells with asynchronous copies,
// so that all of a thread's copies are in flight together.  src( idx, fill )
// returns the element's address, or nullptr with `fill` set to the value of a
// cell outside the block; dst( idx ) is the cell.  FP32 storage: the float is
// copied into the cell's first 4 bytes and widened in place by stage_finish,
// which every thread calls for its own cells after cp_async_wait_all and
// before the block is shared (__syncthreads).
template<typename T, int kIters, int kThreads, typename Src, typename Dst>
__device__ __forceinline__ void stage_block( const T * base, Src src, Dst dst )
{
#pragma unroll 4
    for( int u = 0; u < kIters; ++u )
    {
        const int idx = threadIdx.x + u * kThreads;
        double fill = 0.0;
        const T * s = src( idx, fill );
        if( s != nullptr || fill == 0.0 )
        {
            if constexpr ( sizeof(T) == 8 ) { cp_async_8( dst( idx ), s ? s : base, s != nullptr ); }
            else { cp_async_4( dst( idx ), s ? s : base, s != nullptr ); }
        }
        else { *dst( idx ) = fill; }
    }
}

template<typename T, int kIters, int kThreads, typename Src, typename Dst>
__device__ __forceinline__ void stage_finish( Src src, Dst dst )
{
    if constexpr ( sizeof(T) == 4 )
    {
#pragma unroll 4
        for( int u = 0; u < kIters; ++u )
        {
            const int idx = threadIdx.x + u * kThreads;
            double fill = 0.0;
            const T * s = src( idx, fill );
            if( s != nullptr || fill == 0.0 )
            {
                double * d = dst( idx );
                *d = static_cast<double>( *reinterpret_cast<const float *>( d ) );
            }
        }
    }
}

// Programmatic dependent launch (sm_90+).  Kernels of the level schedule are
// launched with programmatic stream serialization: a kernel lets the next one
// in its stream launch as soon as all of its own CTAs are running
// (pdl_allow_next), and the next one's CTAs do the work that does not read
// the previous kernel's results (their own task records, factor blocks) and
// then wait for that kernel to complete with its memory visible (pdl_wait),
// so launch latency and independent loads overlap the previous kernel.
// Launched without the attribute, both are no-ops.
__device__ __forceinline__ void pdl_allow_next() { asm volatile( "griddepcontrol.launch_dependents;\n" ::: "memory" ); }
__device__ __forceinline__ void pdl_wait() { asm volatile( "griddepcontrol.wait;\n" ::: "memory" ); }

// Fire-and-forget additions into global memory: the read-modify-write runs in
// the L2 cache and the thread does not wait for it.
__device__ __forceinline__ void red_add_f64( double * p, double a )
{
    asm volatile( "red.global.add.f64 [%0], %1;\n" :: "l"(p), "d"(a) : "memory" );
}

__device__ __forceinline__ void red_add_f32( float * p, float a )
{
    asm volatile( "red.global.add.f32 [%0], %1;\n" :: "l"(p), "f"(a) : "memory" );
}

__device__ __forceinline__ void red_add_v4f32( float * p, float a, float b, float c, float d )
{
    asm volatile( "red.global.add.v4.f32 [%0], {%1, %2, %3, %4};\n" :: "l"(p), "f"(a), "f"(b), "f"(c), "f"(d) : "memory" );
}

__device__ __forceinline__ void red_add_any( double * p, double a ) { red_add_f64( p, a ); }
__device__ __forceinline__ void red_add_any( float * p, float a ) { red_add_f32( p, a ); }

// ---------------------------------------------------------------- assembly
// arena[dst] = values[src] (+ reg on the diagonal): ReadNonzeroValues
// (Numeric.hpp:165-180) fused with FetchFromA (Multifrontal.hpp:249-321).
template<typename T>
__global__ void assemble_kernel( const double * __restrict__ values, const std::int64_t * __restrict__ src,
                                 const std::int64_t * __restrict__ dst, std::int64_t count,
                                 const double * __restrict__ reg, T * __restrict__ arena )
{
    const double r = *reg;
    for( std::int64_t e = blockIdx.x * (std::int64_t)blockDim.x + threadIdx.x; e < count;
         e += (std::int64_t)gridDim.x * blockDim.x )
    {
        const std::uint64_t d = static_cast<std::uint64_t>( dst[e] );
        double v = values[src[e]];
        if( d & kDiagFlag ) { v += r; }
        arena[d & (kDiagFlag - 1)] = static_cast<T>( v );
    }
}

// ------------------------------------------------------------------ zeroing
// One warp per row of the task's rows, lanes over its columns [r, n).
template<typename T>
__device__ __forceinline__ void zero_body( const ZeroTask & t, T * __restrict__ arena )
{
    // a row's upper part [r, n): the entries up to the first 16-byte boundary, then 16-byte
    // stores, then the tail
    constexpr int kV = 16 / static_cast<int>( sizeof(T) );
    const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    for( int r = t.row_begin + static_cast<int>( threadIdx.x >> 5 ); r < t.row_end; r += warps )
    {
        T * p = arena + t.offset + static_cast<std::int64_t>( r ) * t.ld + r;
        const int len = t.n - r;
        int head = static_cast<int>( ((16u - (reinterpret_cast<std::uintptr_t>( p ) & 15u)) & 15u) / sizeof(T) );
        head = min( head, len );
        if( lane < head ) { p[lane] = T( 0 ); }
        T * q = p + head;
        const int nv = (len - head) / kV;
        float4 * qv = reinterpret_cast<float4 *>( q );
        for( int v = lane; v < nv; v += 32 ) { qv[v] = make_float4( 0.f, 0.f, 0.f, 0.f ); }
        for( int c = nv * kV + lane; c < len - head; c += 32 ) { q[c] = T( 0 ); }
    }
}

template<typename T>
__global__ void zero_kernel( const ZeroTask * __restrict__ tasks, T * __restrict__ arena )
{
    pdl_allow_next();
    pdl_wait();
    zero_body( tasks[blockIdx.x], arena );
}

// ---------------------------------------------------------------- export
// Reference layout from the fronts: U0 of supernode s is the diagonal block
// of its front at row offset roff; column l of its U1 is front U0 column
// colmap[l] (>= 0) or front U1 column -colmap[l]-1.
template<typename T>
__global__ void export_kernel( const ExportTask * __restrict__ tasks, const std::int32_t * __restrict__ colmap_all,
                               const T * __restrict__ arena, double * __restrict__ tri, double * __restrict__ rec )
{
    const ExportTask t = tasks[blockIdx.x];
    const std::int32_t * colmap = colmap_all + t.colmap;
    for( int r = t.r_begin; r < t.r_end; ++r )
    {
        const std::int64_t fr = t.roff + r;
        const T * f0 = arena + t.fu0 + fr * t.fld0;
        const T * f1 = arena + t.fu1 + fr * t.fld1;
        double * d0 = tri + t.tri + (std::int64_t)r * t.n0s;
        for( int c = threadIdx.x; c < t.n0s; c += blockDim.x ) { d0[c] = (c >= r) ? static_cast<double>( f0[t.roff + c] ) : 0.0; }
        double * d1 = rec + t.rec + (std::int64_t)r * t.n1s;
        for( int l = threadIdx.x; l < t.n1s; l += blockDim.x )
        {
            const int cm = colmap[l];
            d1[l] = static_cast<double>( (cm >= 0) ? f0[cm] : f1[-cm - 1] );
        }
    }
}

// ------------------------------------------------------------- extend-add
// One warp per row of the child's update W; lanes walk the row's upper part
// (coalesced reads of W, lut-indexed adds into the parent front).
template<typename T>
__device__ __forceinline__ void extend_body( const ExtendTask & t, const std::int32_t * __restrict__ lut_all,
                                             T * __restrict__ arena )
{
    const std::int32_t * lut = lut_all + t.lut;
    const T * W = arena + t.w;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    constexpr int kU = 4;     // entries per lane in flight: the lut entries and W values of a group are
                              // loaded before any target is added to.  The targets get their additions
                              // as reductions in the memory system (no load round trip): a launch adds
                              // at most one child into any parent entry (one child rank per pass), so
                              // the sum is the plain target + W in the passes' order.
    for( int i = t.row_begin + warp; i < t.row_end; i += 8 )
    {
        const std::int64_t li = lut[i];
        const T * Wi = W + (std::int64_t)i * t.ldw;
        T * row0 = arena + t.u0 + li * t.ld0p;
        T * row1 = arena + t.u1 + li * t.ld1p;
        T * rowv = arena + t.v + li * t.ldvp;
        const bool upper_part = i < t.mid;
        for( int j0 = i + lane; j0 < t.m1; j0 += 32 * kU )
        {
            T v[kU];
            T * dst[kU];
#pragma unroll
            for( int u = 0; u < kU; ++u )
            {
                const int j = j0 + 32 * u;
                dst[u] = nullptr;
                v[u] = T( 0 );
                if( j < t.m1 )
                {
                    const int lj = lut[j];
                    v[u] = Wi[j];
                    dst[u] = upper_part ? ((j < t.mid) ? row0 + lj : row1 + lj) : rowv + lj;
                }
            }
#pragma unroll
            for( int u = 0; u < kU; ++u ) { if( dst[u] ) { red_add_any( dst[u], v[u] ); } }
        }
    }
}

template<typename T>
__global__ __launch_bounds__(256) void extend_kernel( const ExtendTask * __restrict__ tasks,
                                                      const std::int32_t * __restrict__ lut_all,
                                                      T * __restrict__ arena )
{
    pdl_allow_next();
    const ExtendTask t = tasks[blockIdx.x];
    pdl_wait();
    extend_body( t, lut_all, arena );
}

// Extend-add by parent rows (ExtendPullTask): the CTA adds its segments one
// child after the other, as reductions in the memory system; a fence and a
// barrier between two children make every reduction of the first performed
// before any of the next is issued, so every entry gets the sum of the passes
// by child rank, in the same order (the CTA owns its parent rows for the
// launch).  Inside a segment the (row, 128 columns) chunks go round-robin to
// the warps, so long rows of large update matrices spread over the CTA.
template<typename T>
__global__ __launch_bounds__(256) void extend_pull_kernel( const ExtendPullTask * __restrict__ tasks, const ExtendTask * __restrict__ segs,
                                                           const std::int32_t * __restrict__ lut_all, T * __restrict__ arena )
{
    constexpr int kU = 4, kChunk = 32 * kU, kWarps = 8;
    pdl_allow_next();
    const ExtendPullTask t = tasks[blockIdx.x];
    pdl_wait();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for( std::int64_t g = t.seg_first; g < t.seg_first + t.seg_count; ++g )
    {
        if( g > t.seg_first )
        {
            __threadfence();
            __syncthreads();
        }
        const ExtendTask e = segs[g];
        const std::int32_t * lut = lut_all + e.lut;
        const T * W = arena + e.w;
        int unit = 0;                                   // chunks before row i, over the segment
        for( int i = e.row_begin; i < e.row_end; ++i )
        {
            const int nch = (e.m1 - i + kChunk - 1) / kChunk;
            int k = (warp - unit % kWarps + kWarps) % kWarps;
            unit += nch;
            if( k >= nch ) { continue; }
            const std::int64_t li = lut[i];
            const T * Wi = W + (std::int64_t)i * e.ldw;
            T * row0 = arena + e.u0 + li * e.ld0p;
            T * row1 = arena + e.u1 + li * e.ld1p;
            T * rowv = arena + e.v + li * e.ldvp;
            const bool upper_part = i < e.mid;
            for( ; k < nch; k += kWarps )
            {
                if constexpr ( sizeof(T) == 4 )
                {
                    // FP32: lane quads of consecutive columns; a quad whose targets are four
                    // consecutive, 16-byte aligned entries goes out as one vector reduction
                    const int j0 = i + k * kChunk + 4 * lane;
                    T v[4];
                    T * dst[4];
#pragma unroll
                    for( int u = 0; u < 4; ++u )
                    {
                        const int j = j0 + u;
                        dst[u] = nullptr;
                        v[u] = T( 0 );
                        if( j < e.m1 )
                        {
                            const int lj = lut[j];
                            v[u] = Wi[j];
                            dst[u] = upper_part ? ((j < e.mid) ? row0 + lj : row1 + lj) : rowv + lj;
                        }
                    }
                    const bool quad = dst[3] != nullptr && dst[1] == dst[0] + 1 && dst[2] == dst[0] + 2 && dst[3] == dst[0] + 3
                                      && (reinterpret_cast<std::uintptr_t>( dst[0] ) & 15u) == 0;
                    if( quad ) { red_add_v4f32( reinterpret_cast<float *>( dst[0] ), v[0], v[1], v[2], v[3] ); }
                    else
                    {
#pragma unroll
                        for( int u = 0; u < 4; ++u ) { if( dst[u] ) { red_add_any( dst[u], v[u] ); } }
                    }
                }
                else
                {
                    const int j0 = i + k * kChunk + lane;
                    T v[kU];
                    T * dst[kU];
#pragma unroll
                    for( int u = 0; u < kU; ++u )
                    {
                        const int j = j0 + 32 * u;
                        dst[u] = nullptr;
                        v[u] = T( 0 );
                        if( j < e.m1 )
                        {
                            const int lj = lut[j];
                            v[u] = Wi[j];
                            dst[u] = upper_part ? ((j < e.mid) ? row0 + lj : row1 + lj) : rowv + lj;
                        }
                    }
#pragma unroll
                    for( int u = 0; u < kU; ++u ) { if( dst[u] ) { red_add_any( dst[u], v[u] ); } }
                }
            }
        }
    }
}

// TF32 rounding (round to nearest, ties away) of an FP32 value, as bits.
__device__ __forceinline__ unsigned to_tf32( float x )
{
    unsigned r;
    asm( "cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x) );
    return r;
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
constexpr size_t kTrsmSmemBytes = sizeof(double) * (2 * kPanel * kXld);

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

constexpr size_t kPotrfSmemBytes = sizeof(double) * (2 * kPanel * (kPanel + 1) + 2 * kPanel + 1);

template<typename T> __device__ __forceinline__ double round_to( double v ) { return static_cast<double>( static_cast<T>( v ) ); }

// Panel factorization state in shared memory.  D: the 64 x 64 block, upper
// triangle (A, overwritten by U row block by row block); Ti: the inverse
// T = U^{-1} (upper tiles; diagonal tiles zero below the diagonal; its
// strictly lower tiles serve as per-warp scratch); inv_d: the reciprocal
// pivots the row-block solves use.
struct PotrfShared
{
    double (*D)[kPanel + 1];
    double (*Ti)[kPanel + 1];
    double * inv_d;
    double * floor_s;
    int * fail;
    int * redo;
};

// The scratch tile of warp w = 1..7: the strictly lower tile (7, w - 1) of Ti.
__device__ __forceinline__ double (*potrf_scratch( const PotrfShared & sh ))[kPanel + 1]
{
    return reinterpret_cast<double (*)[kPanel + 1]>( &sh.Ti[kPanel - kSub][kSub * ((threadIdx.x >> 5) - 1)] );
}

// Stores a factored diagonal tile: U_qq, rounded to the storage type, over
// the tile's upper triangle and its reciprocal pivots (of the unrounded
// pivots) into inv_d.
template<typename T>
__device__ __forceinline__ void potrf_store_tile( const PotrfShared & sh, int o, const double (&a)[kSub][kSub], const double (&iv)[kSub] )
{
    if( (threadIdx.x & 31) == 0 )
    {
#pragma unroll
        for( int r = 0; r < kSub; ++r )
        {
#pragma unroll
            for( int c = r; c < kSub; ++c ) { sh.D[o + r][o + c] = round_to<T>( a[r][c] ); }
            sh.inv_d[o + r] = iv[r];
        }
    }
    __syncwarp();
}

// The diagonal tile's Cholesky with pivot floors (mixed precision): a pivot
// lost to FP32 rounding (for a 1 x 1 supernode too: |a| can cancel to 0) is
// raised to its floor (static pivoting); the FP64 refinement corrects it.
// The raised pivot also bounds the row's entries in the block by beta =
// sqrt(max |a_ii|), the growth bound of the modified Cholesky of Gill, Murray
// and Wright: a small pivot under a large row would otherwise make the next
// pivots of the block hugely negative, floored in turn, until FP32
// overflows.  Runs only for tiles with a pivot at or below its floor, after
// the tile's row block is complete.
template<typename T>
__device__ __noinline__ void potrf_tile_floored( const PotrfShared & sh, const PanelTask & t, int q, int nb, const T * __restrict__ arena,
                                                 int * __restrict__ status, const double * __restrict__ pivot_floor )
{
    const int lane = threadIdx.x & 31;
    const int o = kSub * q;
    double a[kSub][kSub], iv[kSub];
#pragma unroll
    for( int r = 0; r < kSub; ++r )
    {
#pragma unroll
        for( int c = r; c < kSub; ++c ) { a[r][c] = sh.D[o + r][o + c]; }
    }
#pragma unroll
    for( int r = 0; r < kSub; ++r )
    {
        double d = a[r][r];
        const bool single = (t.single_rows >> (o + r)) & 1;
        if( single ) { d = fabs( d ); }                     // 1 x 1 reference supernodes: sqrt(|a|)
        const double tau = sh.floor_s[o + r];
        if( o + r < nb && !(d > tau) )
        {
            // the row's largest entry: this tile's columns, the rest of the
            // block and the row's rest columns in U0 and U1, which the trsm
            // divides by the pivot
            double m = 0.0;
#pragma unroll
            for( int c = r + 1; c < kSub; ++c ) { m = fmax( m, fabs( a[r][c] ) ); }
            for( int c = o + kSub + lane; c < kPanel; c += 32 ) { m = fmax( m, fabs( sh.D[o + r][c] ) ); }
            const std::int64_t grow = t.r0 + o + r;
            for( int c = t.r0 + nb + lane; c < t.n0; c += 32 ) { m = fmax( m, fabs( static_cast<double>( arena[t.u0 + grow * t.ld0 + c] ) ) ); }
            for( int c = lane; c < t.n1; c += 32 ) { m = fmax( m, fabs( static_cast<double>( arena[t.u1 + grow * t.ld1 + c] ) ) ); }
#pragma unroll
            for( int s2 = 16; s2 > 0; s2 >>= 1 ) { m = fmax( m, __shfl_xor_sync( 0xffffffffu, m, s2 ) ); }
            if( lane == 0 ) { atomicAdd( status + 2, 1 ); }
            const double beta2 = pivot_floor[0];
            d = fmax( tau, beta2 > 0.0 ? m * m / beta2 : 0.0 );
        }
        iv[r] = rsqrt( d );
        a[r][r] = d * iv[r];
#pragma unroll
        for( int c = r + 1; c < kSub; ++c ) { a[r][c] *= iv[r]; }
#pragma unroll
        for( int r2 = r + 1; r2 < kSub; ++r2 )
        {
#pragma unroll
            for( int c = r2; c < kSub; ++c ) { a[r2][c] -= a[r][r2] * a[r][c]; }
        }
    }
    potrf_store_tile<T>( sh, o, a, iv );
}

// Cholesky of the diagonal tile q of D by one warp.  Every lane holds the
// whole tile in registers and runs the same branch-free recurrence, so that
// a pivot's chain is one reciprocal square root, one product and one fused
// multiply-add; pivot checks come after the tile.  A non-positive pivot (FP64)
// records the first failing row and lets NaNs run on, as before.  With pivot
// floors (mixed precision), a tile that has a pivot at or below its floor is
// factored again by potrf_tile_floored, whose raised pivots depend on the
// whole row: speculative (the tile's row block right of it may still be
// changing) returns false instead, with nothing written.
template<typename T>
__device__ bool potrf_diag_tile( const PotrfShared & sh, const PanelTask & t, int q, int nb, const T * __restrict__ arena,
                                 int * __restrict__ status, const double * __restrict__ pivot_floor, bool speculative )
{
    const int lane = threadIdx.x & 31;
    const int o = kSub * q;
    const unsigned singles = static_cast<unsigned>( (t.single_rows >> o) & 0xff );
    double a[kSub][kSub], iv[kSub], piv[kSub], fl[kSub];
#pragma unroll
    for( int r = 0; r < kSub; ++r )
    {
#pragma unroll
        for( int c = r; c < kSub; ++c ) { a[r][c] = sh.D[o + r][o + c]; }
        // the pivot floors are read with the tile, off the pivot chain
        if constexpr ( sizeof(T) == 4 ) { fl[r] = sh.floor_s[o + r]; }
    }
#pragma unroll
    for( int r = 0; r < kSub; ++r )
    {
        const double d = ((singles >> r) & 1) ? fabs( a[r][r] ) : a[r][r];   // 1 x 1 reference supernodes: sqrt(|a|)
        piv[r] = d;
        iv[r] = rsqrt( d );
        a[r][r] = d * iv[r];
#pragma unroll
        for( int c = r + 1; c < kSub; ++c ) { a[r][c] *= iv[r]; }
#pragma unroll
        for( int r2 = r + 1; r2 < kSub; ++r2 )
        {
#pragma unroll
            for( int c = r2; c < kSub; ++c ) { a[r2][c] -= a[r][r2] * a[r][c]; }
        }
    }
    if constexpr ( sizeof(T) == 4 )
    {
        bool low = false;
#pragma unroll
        for( int r = 0; r < kSub; ++r ) { low |= o + r < nb && !(piv[r] > fl[r]); }
        if( low && pivot_floor != nullptr )
        {
            if( speculative ) { return false; }
            potrf_tile_floored<T>( sh, t, q, nb, arena, status, pivot_floor );
            return true;
        }
    }
    if( lane == 0 )
    {
#pragma unroll
        for( int r = 0; r < kSub; ++r )
        {
            if( !((singles >> r) & 1) && o + r < nb && !(piv[r] > 0.0) && *sh.fail < 0 ) { *sh.fail = o + r; }
        }
    }
    potrf_store_tile<T>( sh, o, a, iv );
    return true;
}

// Cholesky of one panel's 64 x 64 diagonal block D (identity beyond nb) and
// the inverse T = D^{-1} of its factor (LAPACK potrf of FactorizeSupernode,
// Multifrontal.hpp:438-449, plus the inverse the panel's trsm and the solves
// use), right-looking by 8 x 8 tiles, two barriers per tile step b:
//   1. U_bc = U_bb^{-T} A_bc for the columns right of tile b, one column per
//      thread; one warp forms W_b = U_bb^{-1} (tile (b, b) of T).
//   2. warp 0 applies row block b's update to tile (b+1, b+1) and factors
//      that tile ahead; the other warps update the other trailing tiles and
//      form column block b of T, T_ib = -(sum_{k=i..b-1} T_ik U_kb) W_b.
// Tile products run on the FP64 tensor cores (two DMMA m8n8k4 each).  A row
// that forms a 1 x 1 reference supernode takes sqrt(|a|) as the reference
// does (:471) and never reports failure.  With FP32 storage every U value is
// rounded to FP32 as it is formed, so the in-panel updates, W and T use the
// stored factor (T inverts it), as the updates of later panels do.
template<typename T>
__device__ __forceinline__ void potrf_body( const PanelTask & t, T * __restrict__ arena, int * __restrict__ status,
                                            double * smem, const double * __restrict__ pivot_floor, double * __restrict__ tinv )
{
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int nb = min( kPanel, t.n0 - t.r0 );
    PotrfShared sh;
    sh.D = reinterpret_cast<double (*)[kPanel + 1]>( smem );
    sh.Ti = reinterpret_cast<double (*)[kPanel + 1]>( smem + kPanel * (kPanel + 1) );
    sh.inv_d = smem + 2 * kPanel * (kPanel + 1);
    sh.floor_s = sh.inv_d + kPanel;                     // the panel's pivot floors (mixed precision)
    sh.fail = reinterpret_cast<int *>( sh.floor_s + kPanel );
    sh.redo = sh.fail + 1;

    T * U0 = arena + t.u0 + (std::int64_t)t.r0 * t.ld0 + t.r0;
    auto stage_src = [&]( int idx, double & fill ) -> const T *
    {
        const int r = idx / kPanel, c = idx % kPanel;
        fill = (r >= nb && r == c) ? 1.0 : 0.0;      // identity padding beyond nb
        return (r < nb && c < nb && r <= c) ? U0 + (std::int64_t)r * t.ld0 + c : nullptr;
    };
    auto stage_dst = [&]( int idx ) { return &sh.D[idx / kPanel][idx % kPanel]; };
    stage_block<T, kPanel * kPanel / kPotrfThreads, kPotrfThreads>( U0, stage_src, stage_dst );
    // the pivot floors after the block's copies are in flight (their loads overlap)
    if( pivot_floor != nullptr && tid < nb ) { sh.floor_s[tid] = pivot_floor[1 + t.row0 + t.r0 + tid]; }
    if( tid == 0 ) { *sh.fail = -1; *sh.redo = 0; }
    cp_async_wait_all();
    stage_finish<T, kPanel * kPanel / kPotrfThreads, kPotrfThreads>( stage_src, stage_dst );
    __syncthreads();

    const int nsub = (nb + kSub - 1) / kSub;
    if( warp == 0 ) { potrf_diag_tile<T>( sh, t, 0, nb, arena, status, pivot_floor, false ); }
    __syncthreads();
    const int i8 = lane >> 2, j8 = 2 * (lane & 3);        // this lane's entries of an 8 x 8 DMMA result
    for( int b = 0; b < nsub; ++b )
    {
        const int o = kSub * b;
        const int rem = nsub - 1 - b;                   // trailing tile rows / columns
        // 1. row block b right of its diagonal tile; W_b
        if( tid < kSub * rem )
        {
            const int col = o + kSub + tid;
            double x[kSub];
#pragma unroll
            for( int r = 0; r < kSub; ++r ) { x[r] = sh.D[o + r][col]; }
#pragma unroll
            for( int r = 0; r < kSub; ++r )
            {
                x[r] *= sh.inv_d[o + r];
#pragma unroll
                for( int r2 = r + 1; r2 < kSub; ++r2 ) { x[r2] -= sh.D[o + r][o + r2] * x[r]; }
            }
#pragma unroll
            for( int r = 0; r < kSub; ++r ) { sh.D[o + r][col] = round_to<T>( x[r] ); }
        }
        else if( warp == 7 )
        {
            // column j = lane of W_b = U_bb^{-1} (lanes 8-31 repeat lanes 0-7 and store nothing):
            // w_jj = 1 / u_jj, then for k = j-1, .., 0 w_k = -(sum_{i>k} u_ki w_i) / u_kk, as one
            // branch-free recurrence over k = 7..0.  The reciprocals of the stored pivots come from
            // one Newton step on the tile's reciprocal square roots, r = v (2 - u v).
            const int j = lane & (kSub - 1);
            double rec[kSub], w[kSub], sum[kSub];
#pragma unroll
            for( int k = 0; k < kSub; ++k )
            {
                const double v = sh.inv_d[o + k];
                rec[k] = v * fma( -sh.D[o + k][o + k], v, 2.0 );
                sum[k] = 0.0;
            }
#pragma unroll
            for( int k = kSub - 1; k >= 0; --k )
            {
                w[k] = j == k ? rec[k] : (j > k ? -rec[k] * sum[k] : 0.0);
#pragma unroll
                for( int i = 0; i < k; ++i ) { sum[i] = fma( sh.D[o + i][o + k], w[k], sum[i] ); }
            }
            if( lane < kSub )
            {
#pragma unroll
                for( int i = 0; i < kSub; ++i ) { sh.Ti[o + i][o + j] = w[i]; }
            }
        }
        __syncthreads();
        // 2. trailing tiles and T's column block b
        if( warp == 0 )
        {
            if( rem > 0 )
            {
                const int o1 = o + kSub;
                double acc[2] = { 0.0, 0.0 };
                dmma_8x8x8( acc, [&]( int ii, int k ) { return sh.D[o + k][o1 + ii]; }, [&]( int k, int jj ) { return sh.D[o + k][o1 + jj]; } );
                sh.D[o1 + i8][o1 + j8] -= acc[0];
                sh.D[o1 + i8][o1 + j8 + 1] -= acc[1];
                __syncwarp();
                if( !potrf_diag_tile<T>( sh, t, b + 1, nb, arena, status, pivot_floor, true ) && lane == 0 ) { *sh.redo = 1; }
            }
        }
        else
        {
            const int tiles = rem * (rem + 1) / 2 - (rem > 0 ? 1 : 0);     // all but (b+1, b+1)
            // warp 4 shares warp 0's SM sub-partition (warp index mod 4) and
            // stays idle, so that the tile factorization's FP64 chain does not
            // wait behind tile products
            for( int job = warp - (warp < 4 ? 1 : 2); warp != 4 && job < tiles + b; job += kPotrfThreads / 32 - 2 )
            {
                if( job < tiles )
                {
                    // job -> (b2, c), column by column of the trailing triangle after (b+1, b+1)
                    int c = b + 2, left = job;
                    while( left >= c - b ) { left -= c - b; ++c; }
                    const int o2 = kSub * (b + 1 + left), oc = kSub * c;
                    double acc[2] = { 0.0, 0.0 };
                    dmma_8x8x8( acc, [&]( int ii, int k ) { return sh.D[o + k][o2 + ii]; }, [&]( int k, int jj ) { return sh.D[o + k][oc + jj]; } );
                    sh.D[o2 + i8][oc + j8] -= acc[0];
                    sh.D[o2 + i8][oc + j8 + 1] -= acc[1];
                }
                else
                {
                    // T_ib, i = job - tiles < b
                    const int oi = kSub * (job - tiles);
                    double acc[2] = { 0.0, 0.0 };
                    for( int ok = oi; ok < o; ok += kSub )
                    {
                        dmma_8x8x8( acc, [&]( int ii, int kk ) { return sh.Ti[oi + ii][ok + kk]; },
                                         [&]( int kk, int jj ) { return sh.D[ok + kk][o + jj]; } );
                    }
                    double (*S)[kPanel + 1] = potrf_scratch( sh );
                    S[i8][j8] = acc[0];
                    S[i8][j8 + 1] = acc[1];
                    __syncwarp();
                    double acc2[2] = { 0.0, 0.0 };
                    dmma_8x8x8( acc2, [&]( int ii, int k ) { return S[ii][k]; }, [&]( int k, int jj ) { return sh.Ti[o + k][o + jj]; } );
                    sh.Ti[oi + i8][o + j8] = -acc2[0];
                    sh.Ti[oi + i8][o + j8 + 1] = -acc2[1];
                    __syncwarp();
                }
            }
        }
        __syncthreads();
        if( *sh.redo )
        {
            // a pivot of tile (b+1, b+1) needed its floor: factor the tile again
            // now that its row block is complete
            if( warp == 0 ) { potrf_diag_tile<T>( sh, t, b + 1, nb, arena, status, pivot_floor, false ); }
            __syncthreads();
            if( tid == 0 ) { *sh.redo = 0; }
            __syncthreads();
        }
    }
    for( int idx = tid; idx < kPanel * kPanel; idx += kPotrfThreads )
    {
        const int r = idx >> 6, c = idx & 63;
        if( r <= c && c < nb ) { U0[(std::int64_t)r * t.ld0 + c] = static_cast<T>( sh.D[r][c] ); }
    }
    if( tid == 0 && *sh.fail >= 0 )
    {
        atomicOr( status, 1 );
        atomicMin( status + 1, t.row0 + t.r0 + *sh.fail );
    }
    // only the leading nsub x nsub tiles of T are formed (the trsm and the
    // solves read no more)
    const int nbp = kSub * nsub;
    double * out = tinv + (std::int64_t)t.panel * (kPanel * kPanel);
    for( int idx = tid; idx < nbp * kPanel; idx += kPotrfThreads )
    {
        const int r = idx >> 6, c = idx & 63;
        if( c < nbp ) { out[idx] = (r <= c) ? sh.Ti[r][c] : 0.0; }
    }
}

template<typename T>
__global__ __launch_bounds__(kPotrfThreads, 1) void potrf_kernel( const PanelTask * __restrict__ tasks,
                                                               T * __restrict__ arena, int * __restrict__ status,
                                                               const double * __restrict__ pivot_floor,
                                                               double * __restrict__ tinv )
{
    extern __shared__ __align__(16) double psm[];
    pdl_allow_next();
    const PanelTask t = tasks[blockIdx.x];
    pdl_wait();
    potrf_body( t, arena, status, psm, pivot_floor, tinv );
}

// X = D^{-T} U for the rest columns [c0, c0 + kRestChunk) of a panel (trsm of
// FactorizeSupernode, Multifrontal.hpp:452-466) as the product X = T^T U with
// the inverse T = D^{-1} that the panel's potrf left in tinv: X row block rb
// takes the K blocks 0..rb.  Warp w computes the output tiles (rb, ct) with
// rb = (w + ct) mod 8, one of every block row, so every warp does the same
// 36 8 x 8 x 8 DMMA steps (when nb = 64); no step waits on another.
// Operand-image entry of U row k, rest column `col` of a panel whose rest
// columns start at U0 column r1 (m of them in U0, the rest U1 columns).
__device__ __forceinline__ std::int64_t img_offset( const PanelTask & t, int k, int col, int r1, int m )
{
    const int ucol = col < m ? r1 + col : col - m;
    const int ct = col < m ? ucol / kImgRows : t.img_t0 + ucol / kImgRows;
    const std::int64_t blk = t.img + static_cast<std::int64_t>( k / kImgK ) * 2 * t.img_tf + ct;
    return blk * (kImgRows * kImgK) + (ucol % kImgRows) * kImgK + (k % kImgK);
}

template<typename T>
__device__ __forceinline__ void trsm_body( const PanelTask & t, T * __restrict__ arena, const double * __restrict__ tinv,
                                           double * tsm, float * __restrict__ img = nullptr )
{
    double (*Ti)[kXld] = reinterpret_cast<double (*)[kXld]>( tsm );
    double (*X)[kXld] = reinterpret_cast<double (*)[kXld]>( tsm + kPanel * kXld );
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int nb = min( kPanel, t.n0 - t.r0 );
    const int nbb = (nb + kSub - 1) / kSub;
    const int r1 = t.r0 + nb;
    const int m = t.n0 - r1;
    const int rest = m + t.n1;
    const int cw = min( kRestChunk, rest - t.c0 );
    T * U0 = arena + t.u0;
    T * U1 = arena + t.u1;
    static_assert( kRestChunk == kPanel, "trsm assumes square blocks" );
    {
        // only the leading (nb rounded up to 8)^2 block of T is read
        const double * Tg = tinv + (std::int64_t)t.panel * (kPanel * kPanel);
        const int nbp = kSub * nbb;
#pragma unroll
        for( int u = 0; u < kPanel * kPanel / (2 * kTrsmThreads); ++u )
        {
            const int idx = 2 * (tid + u * kTrsmThreads);
            const bool used = (idx >> 6) < nbp && (idx & 63) < nbp;
            cp_async_16( &Ti[idx >> 6][idx & 63], used ? Tg + idx : Tg, used ? 16 : 0 );
        }
    }
    auto stage_src = [&]( int idx, double & ) -> const T *
    {
        const int r = idx / kPanel, c = idx % kPanel;
        const int col = t.c0 + c;
        if( r >= nb || c >= cw ) { return nullptr; }
        return (col < m) ? U0 + (std::int64_t)(t.r0 + r) * t.ld0 + r1 + col
                         : U1 + (std::int64_t)(t.r0 + r) * t.ld1 + (col - m);
    };
    auto stage_dst = [&]( int idx ) { return &X[idx / kPanel][idx % kPanel]; };
    stage_block<T, kPanel * kRestChunk / kTrsmThreads, kTrsmThreads>( U0, stage_src, stage_dst );
    cp_async_wait_all();
    stage_finish<T, kPanel * kRestChunk / kTrsmThreads, kTrsmThreads>( stage_src, stage_dst );
    __syncthreads();
    const int nct = (cw + kSub - 1) / kSub;
    double res[kRestChunk / kSub][2];
#pragma unroll
    for( int ct = 0; ct < kRestChunk / kSub; ++ct )
    {
        res[ct][0] = 0.0; res[ct][1] = 0.0;
        const int rb = (warp + ct) & (kSubs - 1);
        if( rb >= nbb || ct >= nct ) { continue; }
        for( int kb = 0; kb <= rb; ++kb )
        {
            dmma_8x8x8( res[ct], [&]( int i, int k ) { return Ti[kSub * kb + k][kSub * rb + i]; },
                                 [&]( int k, int j ) { return X[kSub * kb + k][kSub * ct + j]; } );
        }
    }
    // the products are done: the results replace the staged block, then go out coalesced
    __syncthreads();
#pragma unroll
    for( int ct = 0; ct < kRestChunk / kSub; ++ct )
    {
        const int rb = (warp + ct) & (kSubs - 1);
        if( rb >= nbb || ct >= nct ) { continue; }
        const int r = kSub * rb + (lane >> 2), cc = kSub * ct + 2 * (lane & 3);
        X[r][cc] = static_cast<double>( static_cast<T>( res[ct][0] ) );
        X[r][cc + 1] = static_cast<double>( static_cast<T>( res[ct][1] ) );
    }
    __syncthreads();
    // U rows: consecutive threads, consecutive columns
    for( int idx = tid; idx < kPanel * kRestChunk; idx += kTrsmThreads )
    {
        const int r = idx >> 6, cc = idx & 63;
        if( r >= nb || cc >= cw ) { continue; }
        const int col = t.c0 + cc;
        const T v = static_cast<T>( X[r][cc] );
        if( col < m ) { U0[(std::int64_t)(t.r0 + r) * t.ld0 + r1 + col] = v; }
        else          { U1[(std::int64_t)(t.r0 + r) * t.ld1 + (col - m)] = v; }
    }
    if constexpr ( sizeof(T) == 4 )
    {
        if( img != nullptr && t.img >= 0 )
        {
            // the stored FP32 values split into TF32 hi + lo, for the tensor-core tiles: the
            // image is K-major, so a warp writes one column's 32 k values of a k-chunk at once
            // (128 contiguous bytes per part)
            const std::int64_t lo_off = static_cast<std::int64_t>( t.img_tf ) * (kImgRows * kImgK);
            for( int pair = warp; pair < 2 * cw; pair += kTrsmThreads / 32 )
            {
                const int cc = pair >> 1, r = 32 * (pair & 1) + lane;
                if( r >= nb ) { continue; }
                const float v = static_cast<float>( X[r][cc] );
                const unsigned hi = to_tf32( v );
                const std::int64_t o = img_offset( t, t.r0 + r, t.c0 + cc, r1, m );
                img[o] = __uint_as_float( hi );
                img[o + lo_off] = __uint_as_float( to_tf32( v - __uint_as_float( hi ) ) );
            }
        }
    }
    if constexpr ( sizeof(T) == 4 )
    {
        // the last panel: image rows n0 .. (n0 rounded up to the 32-row k-chunk) are zero, so
        // that the update matrix's tiles (K = n0) can read whole chunks
        if( img != nullptr && t.img >= 0 && t.r0 + nb == t.n0 )
        {
            const int pad = (kImgK - t.n0 % kImgK) % kImgK;
            for( int idx = threadIdx.x; idx < pad * cw; idx += kTrsmThreads )
            {
                const int k = t.n0 + idx / cw, col = t.c0 + idx % cw;
                const std::int64_t o = img_offset( t, k, col, r1, m );
                img[o] = 0.0f;
                img[o + static_cast<std::int64_t>( t.img_tf ) * (kImgRows * kImgK)] = 0.0f;
            }
        }
    }
}

template<typename T>
__global__ __launch_bounds__(kTrsmThreads) void trsm_kernel( const PanelTask * __restrict__ tasks,
                                                             T * __restrict__ arena, const double * __restrict__ tinv,
                                                             float * __restrict__ img )
{
    extern __shared__ __align__(16) double tsm[];
    pdl_allow_next();
    const PanelTask t = tasks[blockIdx.x];
    pdl_wait();
    trsm_body( t, arena, tinv, tsm, img );
}

// ------------------------------------------------------------------- gemm
// C[m0:m0+64, c0:c0+64] -= A[:, m0:]^T B[:, c0:] for row-major K x M / K x N
// panels: 8 warps in a 2 x 4 arrangement, each a 32 x 16 block of 8 x 8
// DMMA tiles.  K is streamed through a kGemmStages-deep ring of shared-memory
// stages filled by 16-byte cp.async copies (every operand row starts on a
// 16-byte boundary: the plan pads leading dimensions to kLdAlign), so the
// copies of the next chunks overlap the MMAs of the current one.
constexpr int kGemmStages = 3;
constexpr int kGemmStageDoubles = 2 * kGemmK * kGemmLd;          // A and B of one stage
constexpr size_t kGemmSmemBytes = sizeof(double) * kGemmStages * kGemmStageDoubles;

__device__ __forceinline__ void gemm_body( const GemmTask & t, double * __restrict__ arena, double * gsm )
{
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int wm = warp & 1, wn = warp >> 1;
    const double * A = arena + t.a;
    const double * B = arena + t.b;

    double acc[4][2][2];
#pragma unroll
    for( int i = 0; i < 4; ++i )
#pragma unroll
        for( int j = 0; j < 2; ++j ) { acc[i][j][0] = 0.0; acc[i][j][1] = 0.0; }

    // Each stage holds kGemmK rows of 64 doubles for A and for B = 512
    // 16-byte chunks per operand; thread tid copies chunks tid + 256 * l.
    constexpr int kChunks = kGemmK * kTile / 2 / kGemmThreads;       // 2 per operand
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
            double af[4], bf[2];
#pragma unroll
            for( int i = 0; i < 4; ++i ) { af[i] = As[(kk + (lane & 3)) * kGemmLd + wm * 32 + i * 8 + (lane >> 2)]; }
#pragma unroll
            for( int j = 0; j < 2; ++j ) { bf[j] = Bs[(kk + (lane & 3)) * kGemmLd + wn * 16 + j * 8 + (lane >> 2)]; }
#pragma unroll
            for( int i = 0; i < 4; ++i )
#pragma unroll
                for( int j = 0; j < 2; ++j ) { dmma_8x8x4( acc[i][j], af[i], bf[j] ); }
        }
    }
    cp_async_wait<0>();
    // the ring is reused by the next task of a persistent CTA
    __syncthreads();

    // C -= acc as reductions in the memory system (no load round trip); every C
    // entry gets one contribution per launch, so the result is the plain C - acc
    double * C = arena + t.c;
#pragma unroll
    for( int i = 0; i < 4; ++i )
    {
        const int row = t.m0 + wm * 32 + i * 8 + (lane >> 2);
        if( row >= t.M ) { continue; }
        double * Crow = C + (std::int64_t)row * t.ldc;
#pragma unroll
        for( int j = 0; j < 2; ++j )
        {
            const int col = t.c0 + wn * 16 + j * 8 + (lane & 3) * 2;
            if( col < t.N && (!t.upper || row <= col) ) { red_add_f64( Crow + col, -acc[i][j][0] ); }
            if( col + 1 < t.N && (!t.upper || row <= col + 1) ) { red_add_f64( Crow + col + 1, -acc[i][j][1] ); }
        }
    }
}

// FP32 storage: the same tiles as split-precision 3xTF32 products on the
// 5th-generation tensor cores (x = hi + lo with hi, lo TF32; a b ~ a_lo b_hi +
// a_hi b_lo + a_hi b_hi, FP32 accumulation in tensor memory).  K is streamed
// in chunks of 32 rows through two shared-memory stages; every chunk is read
// from global memory into registers one chunk ahead (a warp reads 4 rows of
// 8 consecutive floats), split, and stored in the canonical K-major
// no-swizzle layout of tcgen05 operands: core matrices of 8 (m or n) rows x
// 4 k (16 B per row, 128 B per core matrix), the 8 row groups 128 B apart
// (stride byte offset) and the k groups of 4 1024 B apart (leading byte
// offset).  One thread issues the 12 tcgen05.mma (M = N = 64, K = 8) of a
// chunk and commits them to the stage's mbarrier; the stage is refilled once
// that barrier has completed.  The 64 x 64 accumulator is read back with
// tcgen05.ld, staged in shared memory and subtracted from C with coalesced
// 16-byte accesses (the plan keeps C offsets and leading dimensions
// multiples of 4 floats).
constexpr int kTcK = 32;                               // k rows per chunk
constexpr int kTcPart = kTcK * kTile * 4;              // one operand part (64 x 32 TF32): 8 KB
constexpr int kTcStage = 4 * kTcPart;                  // A_hi, A_lo, B_hi, B_lo
constexpr size_t kGemmSmemBytesF = 2 * kTcStage;       // 64 KB
constexpr int kTcSld = kTile + 4;                      // staged result row (floats)
constexpr int kTcCols = 64;                            // tensor-memory columns per CTA (FP32 accumulator 64 x 64)
constexpr unsigned kTcMaxPolls = 1u << 24;             // bound on the polls of one mbarrier wait
constexpr unsigned long long kTcTimeoutNs = 1000000000ull;
constexpr int kStatusTcTimeout = 2;                    // status[0] bit: a tensor-core completion wait ran out
static_assert( kGemmSmemBytesF >= sizeof(float) * kTile * kTcSld, "result staging does not fit" );

__device__ __forceinline__ std::uint32_t smem_u32( const void * p )
{
    return static_cast<std::uint32_t>( __cvta_generic_to_shared( p ) );
}

__device__ __forceinline__ unsigned long long tc_now()
{
    unsigned long long t;
    asm volatile( "mov.u64 %0, %%globaltimer;\n" : "=l"(t) );
    return t;
}

__device__ __forceinline__ int ld_acquire_i32( const int * p )
{
    int v;
    asm volatile( "ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory" );
    return v;
}

// Waits until the mbarrier phase of the given parity has completed; false
// when the wait ran out (polls or time).
__device__ __forceinline__ bool tc_wait( std::uint32_t bar, std::uint32_t parity )
{
    const unsigned long long start = tc_now();
    for( unsigned i = 0; i < kTcMaxPolls; ++i )
    {
        std::uint32_t done;
        asm volatile( "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
                      : "=r"(done) : "r"(bar), "r"(parity) : "memory" );
        if( done ) { return true; }
        if( (i & 1023u) == 1023u && tc_now() - start > kTcTimeoutNs ) { return false; }
    }
    return false;
}

// Per-CTA tensor-core state: the accumulator's tensor-memory address, the two
// stage mbarriers and the number of commits made to each (the parity of the
// next completion to wait for), carried across the tasks of a persistent CTA.
struct TcState
{
    std::uint32_t tmem;
    std::uint32_t bar;            // shared address of bar[0]; bar[1] = bar + 8
    unsigned commits0, commits1;  // commits made to bar[0] / bar[1]
    __device__ unsigned commits( int s ) const { return s ? commits1 : commits0; }
};

// All threads of the CTA; warp 0 allocates the accumulator columns.
__device__ __forceinline__ TcState tc_setup( std::uint64_t * bars, std::uint32_t * s_tmem )
{
    if( threadIdx.x == 0 )
    {
        asm volatile( "mbarrier.init.shared::cta.b64 [%0], 1;\n" :: "r"(smem_u32( bars )) );
        asm volatile( "mbarrier.init.shared::cta.b64 [%0], 1;\n" :: "r"(smem_u32( bars + 1 )) );
        asm volatile( "fence.mbarrier_init.release.cluster;\n" ::: "memory" );
    }
    if( (threadIdx.x >> 5) == 0 )
    {
        asm volatile( "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" :: "r"(smem_u32( s_tmem )), "r"(kTcCols) );
        asm volatile( "tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" );
    }
    asm volatile( "tcgen05.fence::before_thread_sync;\n" ::: "memory" );
    __syncthreads();
    asm volatile( "tcgen05.fence::after_thread_sync;\n" ::: "memory" );
    TcState tc;
    tc.tmem = *s_tmem;
    tc.bar = smem_u32( bars );
    tc.commits0 = 0;
    tc.commits1 = 0;
    return tc;
}

// All threads of the CTA, after its last task: frees the accumulator columns.
__device__ __forceinline__ void tc_teardown( const TcState & tc )
{
    asm volatile( "tcgen05.fence::before_thread_sync;\n" ::: "memory" );
    __syncthreads();
    if( (threadIdx.x >> 5) == 0 )
    {
        asm volatile( "tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" :: "r"(tc.tmem), "r"(kTcCols) );
    }
}

// Shared-memory matrix descriptor of one K-major no-swizzle operand part:
// start address, leading byte offset 1024 (next 4 k), stride byte offset 128
// (next 8 rows), descriptor version 1 (sm_100), no swizzle.
__device__ __forceinline__ std::uint64_t tc_desc( std::uint32_t addr )
{
    return static_cast<std::uint64_t>( (addr >> 4) & 0x3FFFu ) | (static_cast<std::uint64_t>( 1024 >> 4 ) << 16)
         | (static_cast<std::uint64_t>( 128 >> 4 ) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B, both
// K-major, N = 64 (bits 17-22: N / 8), M = 64 (bits 24-28: M / 16).
constexpr std::uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((64u >> 4) << 24);

__device__ __forceinline__ void gemm_body( const GemmTask & t, float * __restrict__ arena, double * smem, TcState & tc,
                                           int * status )
{
    unsigned char * sm = reinterpret_cast<unsigned char *>( smem );
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // this thread's elements of every chunk: k = 4 i + kl (i = 0..7), row mn of A and of B
    const int mn = 8 * warp + (lane & 7), kl = lane >> 3;
    const bool a_ok = t.m0 + mn < t.M, b_ok = t.c0 + mn < t.N;
    const float * A = arena + t.a;
    const float * B = arena + t.b;
    const std::int64_t acol = t.m0 + mn, bcol = t.c0 + mn;
    const int soff = warp * 128 + (lane & 7) * 16 + kl * 4;   // K-major offset of (mn, kl) in a part
    const int nk = (t.K + kTcK - 1) / kTcK;
    float ra[8], rb[8];
    auto load = [&]( int c )
    {
#pragma unroll
        for( int i = 0; i < 8; ++i )
        {
            const int k = c * kTcK + 4 * i + kl;
            ra[i] = (k < t.K && a_ok) ? A[(std::int64_t)k * t.lda + acol] : 0.0f;
            rb[i] = (k < t.K && b_ok) ? B[(std::int64_t)k * t.ldb + bcol] : 0.0f;
        }
    };
    if( nk > 0 ) { load( 0 ); }
    bool ok = true;
    for( int c = 0; c < nk; ++c )
    {
        const int s = c & 1;
        unsigned char * st = sm + s * kTcStage;
        float ca[8], cb[8];
#pragma unroll
        for( int i = 0; i < 8; ++i ) { ca[i] = ra[i]; cb[i] = rb[i]; }
        if( c + 1 < nk ) { load( c + 1 ); }
        // the stage is free once the MMAs of its previous chunk have completed
        const bool mine = (tc.commits( s ) == 0) || tc_wait( tc.bar + 8 * s, (tc.commits( s ) & 1u) ^ 1u );
#pragma unroll
        for( int i = 0; i < 8; ++i )
        {
            const unsigned ha = to_tf32( ca[i] ), hb = to_tf32( cb[i] );
            const int o = i * 1024 + soff;
            *reinterpret_cast<unsigned *>( st + o ) = ha;
            *reinterpret_cast<unsigned *>( st + kTcPart + o ) = to_tf32( ca[i] - __uint_as_float( ha ) );
            *reinterpret_cast<unsigned *>( st + 2 * kTcPart + o ) = hb;
            *reinterpret_cast<unsigned *>( st + 3 * kTcPart + o ) = to_tf32( cb[i] - __uint_as_float( hb ) );
        }
        asm volatile( "fence.proxy.async.shared::cta;\n" ::: "memory" );
        if( __syncthreads_or( mine ? 0 : 1 ) ) { ok = false; break; }
        if( tid == 0 )
        {
            asm volatile( "tcgen05.fence::after_thread_sync;\n" ::: "memory" );
            const std::uint32_t base = smem_u32( st );
#pragma unroll
            for( int ks = 0; ks < kTcK / 8; ++ks )
            {
                const std::uint32_t off = ks * 2048;
                const std::uint64_t ahi = tc_desc( base + off ), alo = tc_desc( base + kTcPart + off );
                const std::uint64_t bhi = tc_desc( base + 2 * kTcPart + off ), blo = tc_desc( base + 3 * kTcPart + off );
                const std::uint64_t ad[3] = { alo, ahi, ahi }, bd[3] = { bhi, blo, bhi };
#pragma unroll
                for( int u = 0; u < 3; ++u )
                {
                    const std::uint32_t accumulate = (c > 0 || ks > 0 || u > 0) ? 1u : 0u;
                    asm volatile( "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                                  "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
                                  :: "r"(tc.tmem), "l"(ad[u]), "l"(bd[u]), "r"(kTcIdesc), "r"(accumulate) );
                }
            }
            asm volatile( "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                          :: "r"(tc.bar + 8 * s) : "memory" );
        }
        if( s ) { ++tc.commits1; } else { ++tc.commits0; }
    }
    // every commit of both stages complete: the accumulator is final and the
    // stages are free for the next task
    bool fine = ok;
#pragma unroll
    for( int s = 0; s < 2; ++s )
    {
        if( fine && tc.commits( s ) > 0 ) { fine = tc_wait( tc.bar + 8 * s, (tc.commits( s ) & 1u) ^ 1u ); }
    }
    if( __syncthreads_or( fine ? 0 : 1 ) )
    {
        if( tid == 0 )
        {
            atomicOr( status, kStatusTcTimeout );
            // one more bounded wait for the MMAs in flight before the memory is reused
            for( int s = 0; s < 2; ++s ) { if( tc.commits( s ) > 0 ) { tc_wait( tc.bar + 8 * s, (tc.commits( s ) & 1u) ^ 1u ); } }
        }
        __syncthreads();
        return;
    }
    if( nk == 0 ) { return; }
    asm volatile( "tcgen05.fence::after_thread_sync;\n" ::: "memory" );
    float * S = reinterpret_cast<float *>( sm );
    {
        // warp w reads accumulator rows 16 (w % 4) .. +15 (tensor-memory lanes 32 (w % 4) .. +15 for
        // M = 64), columns 32 (w / 4) .. +31
        const int q = warp & 3, h = warp >> 2;
        std::uint32_t v[32];
        asm volatile( "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
                      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
                        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                      : "r"(tc.tmem + ((std::uint32_t)(32 * q) << 16) + 32 * h) );
        asm volatile( "tcgen05.wait::ld.sync.aligned;\n" ::: "memory" );
        asm volatile( "tcgen05.fence::before_thread_sync;\n" ::: "memory" );
        if( lane < 16 )
        {
            float4 * dst = reinterpret_cast<float4 *>( S + (16 * q + lane) * kTcSld + 32 * h );
#pragma unroll
            for( int j = 0; j < 8; ++j )
            {
                dst[j] = make_float4( __uint_as_float( v[4 * j] ), __uint_as_float( v[4 * j + 1] ),
                                      __uint_as_float( v[4 * j + 2] ), __uint_as_float( v[4 * j + 3] ) );
            }
        }
    }
    __syncthreads();
    float * C = arena + t.c;
    const int cq = 4 * (tid & 15);
    const int col = t.c0 + cq;
#pragma unroll
    for( int i = 0; i < 4; ++i )
    {
        const int r = (tid >> 4) + 16 * i;
        const int row = t.m0 + r;
        if( row >= t.M || col >= t.N ) { continue; }
        const float4 d = *reinterpret_cast<const float4 *>( S + r * kTcSld + cq );
        float * Cp = C + (std::int64_t)row * t.ldc + col;
        if( col + 3 < t.N && (!t.upper || row <= col) )
        {
            red_add_v4f32( Cp, -d.x, -d.y, -d.z, -d.w );
        }
        else
        {
            const float dv[4] = { d.x, d.y, d.z, d.w };
#pragma unroll
            for( int j = 0; j < 4; ++j )
            {
                if( col + j < t.N && (!t.upper || row <= col + j) ) { atomicAdd( Cp + j, -dv[j] ); }
            }
        }
    }
    // the staged result and the accumulator are reused by the next task
    __syncthreads();
}

// One CTA per SM slot, looping over the launch's tiles with its tensor memory
// held throughout.
__global__ __launch_bounds__(kGemmThreads, 3) void gemm_tc_kernel( const GemmTask * __restrict__ tasks, int count,
                                                                  float * __restrict__ arena, int * status )
{
    extern __shared__ __align__(16) double gsm[];
    __shared__ std::uint64_t bars[2];
    __shared__ std::uint32_t s_tmem;
    pdl_allow_next();
    pdl_wait();
    TcState tc = tc_setup( bars, &s_tmem );
    for( int i = blockIdx.x; i < count; i += gridDim.x ) { gemm_body( tasks[i], arena, gsm, tc, status ); }
    tc_teardown( tc );
}

__global__ __launch_bounds__(kGemmThreads) void gemm_tn_kernel( const GemmTask * __restrict__ tasks,
                                                                double * __restrict__ arena )
{
    extern __shared__ __align__(16) double gsm[];
    pdl_allow_next();
    const GemmTask t = tasks[blockIdx.x];
    pdl_wait();
    gemm_body( t, arena, gsm );
}

// ------------------------------------------------------------------ solves
// The supernodal solves (LowerSolver.hpp:143-305, UpperSolver.hpp:127-255)
// run as one launch per (level, panel step) and sweep.  The triangular solves
// with the 64 x 64 diagonal blocks become products with their inverses
// (computed by the panel potrf), so every CTA of a step can form the panel's
// solution itself and no CTA waits for another.

constexpr int kTld = kPanel + 4;   // padded shared-memory row of 64-wide blocks (conflict-free DMMA fragments)
// Doubles of shared memory the solve step's staged rest block takes (64 x kTld of T, rounded up).

// acc[ct] (8 x 8 tile ct of this warp's 8 output rows, NCT tiles) += sum over
// the K blocks [kb0, kb1) of A(i, kk) * B(kk, ct * 8 + j).
template<int NCT, typename FA, typename FB>
__device__ __forceinline__ void warp_rows_product( double (&acc)[NCT][2], int kb0, int kb1, FA a, FB b )
{
    for( int kb = kb0; kb < kb1; ++kb )
    {
#pragma unroll
        for( int ct = 0; ct < NCT; ++ct )
        {
            dmma_8x8x8( acc[ct], [&]( int i, int kk ) { return a( i, kb * 8 + kk ); },
                                 [&]( int kk, int j ) { return b( kb * 8 + kk, ct * 8 + j ); } );
        }
    }
}

// One solve step.  Forward (U^T y = b): every task forms x_q = T_q^T y_q for
// the panel's rows of `in`; the owner writes x_q to `out`, and a task with
// rest rows subtracts P^T x_q from its (up to) 64 rest rows of `in` (rows of
// the front in place, ancestor rows by atomic adds: other fronts of the level
// may target them).  Backward (U x = y): `out` starts at zero on the panel's
// rows; a task adds T_q (y_q - P x_r) (owner) or -T_q P x_r, with x_r its rest
// rows of `out`, already final.  The owner is the task with c0 <= 0: the
// first rest chunk, or a rest-less task for a front's last panel without
// rest.  Warp w owns rows 8w..8w+7 of every 64 x KP product (KP = k rounded
// up to a power of two >= 8) as 8 x 8 DMMA tiles and skips row and K blocks
// beyond the panel's nb rows and the task's cw rest rows; only the used
// block of T is copied.  The body is instantiated per KP: with the tile
// counts known at compile time the tile loops unroll and the accumulators
// take only the registers they need (a task ran 11.6 us with KP a run-time
// value and 7 us with it fixed, 64^3 Laplacian with 16 RHS).
//
// atomic_own: rows of the task's own front are updated with atomics too (the
// task-graph solve, where panels of one front can run concurrently).
//
// kPdl: launched with programmatic stream serialization; the factor blocks (T,
// the rest block) and the rest rows' indices are loaded before pdl_wait, the
// vectors the previous step writes only after it.
template<typename T, int KP, bool kPdl = false>
__device__ __forceinline__ void solve_step_body( const SolveRestTask & t, int upper, const T * __restrict__ arena,
                                                 const double * __restrict__ tinv,
                                                 const std::int32_t * __restrict__ sn_inner,
                                                 double * in, double * out, int ld, int k, bool atomic_own, double * ssm )
{
    constexpr int kp = KP;
    constexpr int lkp = KP == 8 ? 3 : KP == 16 ? 4 : KP == 32 ? 5 : 6;
    constexpr int ldv = kp + 4;
    double (*sT)[kTld] = reinterpret_cast<double (*)[kTld]>( ssm );
    double * sX = ssm + kPanel * kTld;              // [64][ldv]: x_q (forward) / x_r (backward)
    double * sY = sX + kPanel * ldv;                // [64][ldv]: y_q
    __shared__ std::int64_t trow[kSolveRest];
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    constexpr int nct = kp >> 3;
    const int nb = min( kPanel, t.n0 - t.r0 );
    const int nbb = (nb + 7) >> 3;
    const int r1 = t.r0 + nb;
    const int m = t.n0 - r1;
    const bool owner = t.c0 <= 0;
    const bool has_rest = t.c0 >= 0;
    const int cw = has_rest ? t.c1 - t.c0 : 0;
    const std::int64_t prow = (std::int64_t)t.row0 + t.r0;

    {
        // only the leading (nb rounded up to 8)^2 block of T is read below
        const double * Tg = tinv + (std::int64_t)t.panel * (kPanel * kPanel);
        const int nbp = 8 * nbb;
#pragma unroll
        for( int u = 0; u < kPanel * kPanel / (2 * kSolveThreads); ++u )
        {
            const int idx = 2 * (tid + u * kSolveThreads);
            const bool used = (idx >> 6) < nbp && (idx & 63) < nbp;
            cp_async_16( &sT[idx >> 6][idx & 63], used ? Tg + idx : Tg, used ? 16 : 0 );
        }
    }
    if( tid < kSolveRest )
    {
        const int col = t.c0 + tid;
        trow[tid] = (tid < cw) ? ((col < m) ? (std::int64_t)t.row0 + r1 + col
                                            : (std::int64_t)sn_inner[t.inner + (col - m)]) : -1;
    }
    // The panel's rest block P (factor data: final before any solve step) goes straight into
    // registers as this warp's DMMA A fragments (lane: row lane / 4 of the 8-row tile, K index
    // lane % 4 + 4 s of each 8-wide K block kb), loaded before the wait on the previous launch.
    // Forward: A(i, K) = P[K][o + i] (K over the panel's rows); back: A(i, K) = P[o + i][K]
    // (K over the rest columns).  Without a staged copy of P a CTA needs 35 KB (FP64) or
    // 17 KB (FP32) less shared memory, so more CTAs share an SM.
    const T * U0 = arena + t.u0 + (std::int64_t)t.r0 * t.ld0;
    const T * U1 = arena + t.u1 + (std::int64_t)t.r0 * t.ld1;
    const int o = warp * 8;
    T pf[kPanel / 8][2];
    {
        auto rest_at = [&]( int i, int cc ) -> T
        {
            const int col = t.c0 + cc;
            return (col < m) ? U0[(std::int64_t)i * t.ld0 + r1 + col] : U1[(std::int64_t)i * t.ld1 + (col - m)];
        };
#pragma unroll
        for( int kb = 0; kb < kPanel / 8; ++kb )
        {
#pragma unroll
            for( int s = 0; s < 2; ++s )
            {
                const int kk = 8 * kb + (lane & 3) + 4 * s;
                const int i = upper ? o + (lane >> 2) : kk;          // panel row
                const int cc = upper ? kk : o + (lane >> 2);         // rest column
                pf[kb][s] = (has_rest && i < nb && cc < cw) ? rest_at( i, cc ) : T( 0 );
            }
        }
    }
    if constexpr ( kPdl ) { pdl_wait(); }
    // y_q: the panel's rows of `in` (forward: every task; backward: the owner)
    const bool need_y = !upper || owner;
#pragma unroll 4
    for( int idx = tid; idx < (kPanel << lkp); idx += kSolveThreads )
    {
        const int i = idx >> lkp, c = idx & (kp - 1);
        const bool valid = need_y && i < nb && c < k;
        cp_async_8( &sY[i * ldv + c], valid ? in + (prow + i) * ld + c : in, valid );
    }
    __syncthreads();
    if( upper )
    {
        // x_r: the rest rows of `out`, final
#pragma unroll 4
        for( int idx = tid; idx < (kPanel << lkp); idx += kSolveThreads )
        {
            const int i = idx >> lkp, c = idx & (kp - 1);
            const bool valid = i < cw && c < k;
            cp_async_8( &sX[i * ldv + c], valid ? out + trow[i] * ld + c : out, valid );
        }
    }
    cp_async_wait_all();
    __syncthreads();

    const int fi = lane >> 2, fj = 2 * (lane & 3);     // accumulator fragment: row fi, columns fj, fj + 1
    double acc[nct][2];
    // acc += P-part (A fragments in pf) times rows of sX, K blocks [0, kbn)
    auto rest_product = [&]( int kbn )
    {
#pragma unroll
        for( int kb = 0; kb < kPanel / 8; ++kb )
        {
            if( kb >= kbn ) { break; }
#pragma unroll
            for( int ct = 0; ct < nct; ++ct )
            {
#pragma unroll
                for( int s = 0; s < 2; ++s )
                {
                    dmma_8x8x4( acc[ct], static_cast<double>( pf[kb][s] ),
                                sX[(8 * kb + (lane & 3) + 4 * s) * ldv + ct * 8 + (lane >> 2)] );
                }
            }
        }
    };
#pragma unroll
    for( int ct = 0; ct < nct; ++ct ) { acc[ct][0] = 0.0; acc[ct][1] = 0.0; }
    if( !upper )
    {
        // x_q = T^T y_q (T^T lower triangular: K blocks 0..warp)
        if( o < nb )
        {
            warp_rows_product<nct>( acc, 0, warp + 1, [&]( int i, int kk ) { return sT[kk][o + i]; },
                                                      [&]( int kk, int c ) { return sY[kk * ldv + c]; } );
#pragma unroll
            for( int ct = 0; ct < nct; ++ct )
            {
                sX[(o + fi) * ldv + ct * 8 + fj]     = acc[ct][0];
                sX[(o + fi) * ldv + ct * 8 + fj + 1] = acc[ct][1];
            }
        }
        __syncthreads();
        if( owner )
        {
            for( int idx = tid; idx < (kPanel << lkp); idx += kSolveThreads )
            {
                const int i = idx >> lkp, c = idx & (kp - 1);
                if( i < nb && c < k ) { out[(prow + i) * ld + c] = sX[i * ldv + c]; }
            }
        }
        if( !has_rest || o >= cw ) { return; }
        // rest rows: y_r -= P^T x_q
#pragma unroll
        for( int ct = 0; ct < nct; ++ct ) { acc[ct][0] = 0.0; acc[ct][1] = 0.0; }
        rest_product( nbb );
        const int jj = o + fi;
        if( jj < cw )
        {
            double * dst = in + trow[jj] * ld;
            const bool own_row = t.c0 + jj < m;
#pragma unroll
            for( int ct = 0; ct < nct; ++ct )
            {
#pragma unroll
                for( int e = 0; e < 2; ++e )
                {
                    const int c = ct * 8 + fj + e;
                    if( c < k )
                    {
                        if( own_row && !atomic_own ) { dst[c] -= acc[ct][e]; } else { atomicAdd( dst + c, -acc[ct][e] ); }
                    }
                }
            }
        }
    }
    else
    {
        // sY rows of this warp <- (owner ? y_q : 0) - P x_r
        if( has_rest && o < nb )
        {
            rest_product( (cw + 7) >> 3 );
#pragma unroll
            for( int ct = 0; ct < nct; ++ct )
            {
#pragma unroll
                for( int e = 0; e < 2; ++e )
                {
                    double & v = sY[(o + fi) * ldv + ct * 8 + fj + e];
                    v = (owner ? v : 0.0) - acc[ct][e];
                }
            }
        }
        __syncthreads();
        if( o >= nb ) { return; }
        // z = T (.) (T upper triangular: K blocks warp..nbb-1)
#pragma unroll
        for( int ct = 0; ct < nct; ++ct ) { acc[ct][0] = 0.0; acc[ct][1] = 0.0; }
        warp_rows_product<nct>( acc, warp, nbb, [&]( int i, int kk ) { return sT[o + i][kk]; },
                                                [&]( int kk, int c ) { return sY[kk * ldv + c]; } );
        const int i = o + fi;
        if( i < nb )
        {
            double * dst = out + (prow + i) * ld;
#pragma unroll
            for( int ct = 0; ct < nct; ++ct )
            {
#pragma unroll
                for( int e = 0; e < 2; ++e )
                {
                    const int c = ct * 8 + fj + e;
                    if( c < k ) { atomicAdd( dst + c, acc[ct][e] ); }
                }
            }
        }
    }
}

// One kernel per right-hand-side width KP, so that each gets the registers it needs.
template<typename T, int KP>
__global__ __launch_bounds__(kSolveThreads) void solve_step_kernel( const SolveRestTask * __restrict__ tasks, int upper,
                                                                    const T * __restrict__ arena,
                                                                    const double * __restrict__ tinv,
                                                                    const std::int32_t * __restrict__ sn_inner,
                                                                    double * in, double * out, int ld, int k )
{
    extern __shared__ __align__(16) double ssm[];
    pdl_allow_next();
    solve_step_body<T, KP, true>( tasks[blockIdx.x], upper, arena, tinv, sn_inner, in, out, ld, k, false, ssm );
}

// The solve's task graph (Plan::solve_*) as one persistent launch per sweep:
// CTAs take tasks in list order, thread 0 waits (bounded) until the task's
// inputs are final, the CTA runs the step body with atomic updates of every
// row, and thread 0 signals after a fence.  Forward: wait for the panel's
// expected contributions, signal every target panel.  Back: wait until every
// target panel has all of its tasks done, signal the task's own panel.
template<typename T, int KP>
__global__ __launch_bounds__(kSolveThreads) void solve_dag_kernel( const SolveDagArgs a, const T * __restrict__ arena,
                                                                   double * in, double * out, int ld, int k )
{
    extern __shared__ __align__(16) double ssm[];
    __shared__ int s_idx, s_ok;
    const int tid = threadIdx.x;
    for( ;; )
    {
        if( tid == 0 )
        {
            int idx = a.ntasks, ok = 0;
            if( *reinterpret_cast<volatile int *>( a.error ) == 0 ) { idx = atomicAdd( a.next, 1 ); }
            if( idx < a.ntasks )
            {
                const int ti = a.order[idx];
                const int g = ti - a.first_task;
                const unsigned long long start = tc_now();
                if( a.trace ) { a.trace[4 * (std::int64_t)idx] = start; a.trace[4 * (std::int64_t)idx + 3] = blockIdx.x; }
                ok = 1;
                // forward: one wait (the task's panel); back: one per target panel
                const int nw = a.upper ? static_cast<int>( a.target_ptr[g + 1] - a.target_ptr[g] ) : 1;
                for( int w = 0; w < nw && ok; ++w )
                {
                    const int pnl = a.upper ? a.targets[a.target_ptr[g] + w] : a.tasks[ti].panel - a.first_panel;
                    const int need = a.upper ? a.panel_tasks[pnl] : a.fwd_expected[pnl];
                    unsigned spins = 0;
                    while( ld_acquire_i32( a.counters + pnl ) < need )
                    {
                        ++spins;
                        if( (spins & 31u) == 0 )
                        {
                            if( *reinterpret_cast<volatile int *>( a.error ) != 0 ) { ok = 0; break; }
                            if( tc_now() - start > a.timeout_ns || spins > kDagMaxSpins )
                            {
                                atomicCAS( a.error, 0, idx + 1 );
                                ok = 0;
                                break;
                            }
                        }
                        __nanosleep( 64 );
                    }
                }
                if( a.trace ) { a.trace[4 * (std::int64_t)idx + 1] = tc_now(); }
            }
            s_idx = idx;
            s_ok = ok;
        }
        __syncthreads();
        const int idx = s_idx;
        if( idx >= a.ntasks || !s_ok ) { break; }
        const int ti = a.order[idx];
        solve_step_body<T, KP>( a.tasks[ti], a.upper, arena, a.tinv, a.sn_inner, in, out, ld, k, true, ssm );
        __threadfence();
        __syncthreads();
        if( tid == 0 )
        {
            if( a.trace ) { a.trace[4 * (std::int64_t)idx + 2] = tc_now(); }
            const int g = ti - a.first_task;
            if( a.upper ) { atomicAdd( a.counters + (a.tasks[ti].panel - a.first_panel), 1 ); }
            else
            {
                for( std::int64_t e = a.target_ptr[g]; e < a.target_ptr[g + 1]; ++e ) { atomicAdd( a.counters + a.targets[e], 1 ); }
            }
        }
    }
}

// ------------------------------------------------- persistent factorization
// The whole numeric factorization as one launch: each CTA repeatedly takes
// the next task of the plan's dependency-ordered list (an atomic ticket),
// waits until the task's counters reach their targets, runs the task body
// and increments its counters.  Tasks are taken in list order and every wait
// is satisfied by tasks earlier in the list, so the earliest unfinished task
// can always proceed; waits are nevertheless bounded in time, and a wait that
// runs out records the task in `error` and makes every CTA stop.
//
// Counter protocol: every thread fences its own writes of the task, the CTA
// synchronises, and thread 0 increments the counters (release); a waiting
// thread 0 reads counters with ld.acquire.gpu and the CTA synchronises
// before any thread touches the task's data.
constexpr int kDagThreads = 256;
constexpr size_t kDagSmemBytes = kTrsmSmemBytes > kGemmSmemBytes ? kTrsmSmemBytes : kGemmSmemBytes;
static_assert( kDagSmemBytes >= kPotrfSmemBytes && kDagSmemBytes >= kGemmSmemBytesF, "persistent kernel shared memory too small" );

__device__ __forceinline__ int ld_acquire( const int * p )
{
    int v;
    asm volatile( "ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory" );
    return v;
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile( "mov.u64 %0, %%globaltimer;\n" : "=l"(t) );
    return t;
}

// Thread 0 only: 1 when all waits of the task are met, 0 on timeout or when
// another CTA has reported an error.
__device__ int dag_wait( const DagTask & t, const DagArgs & a, int idx )
{
    const unsigned long long start = global_ns();
    for( int i = 0; i < kDagWaits; ++i )
    {
        if( t.wait[i] < 0 ) { continue; }
        const int * c = a.counters + t.wait[i];
        unsigned spins = 0;
        while( ld_acquire( c ) < t.target[i] )
        {
            ++spins;
            if( (spins & 31u) == 0 )
            {
                if( *reinterpret_cast<volatile int *>( a.error ) != 0 ) { return 0; }
                if( global_ns() - start > a.timeout_ns || spins > kDagMaxSpins )
                {
                    atomicCAS( a.error, 0, idx + 1 );
                    return 0;
                }
            }
            __nanosleep( 100 );
        }
    }
    return 1;
}

template<typename T>
__global__ __launch_bounds__(kDagThreads, 3) void factor_dag_kernel( const DagArgs a )
{
    T * arena = static_cast<T *>( a.arena );
    extern __shared__ __align__(16) double dsm[];
    __shared__ int s_idx, s_ok;
    __shared__ std::uint64_t tc_bars[2];
    __shared__ std::uint32_t tc_tmem;
    const int tid = threadIdx.x;
    TcState tc{};
    if constexpr ( sizeof(T) == 4 ) { tc = tc_setup( tc_bars, &tc_tmem ); }
    for( ;; )
    {
        if( tid == 0 )
        {
            int idx = a.ntasks, ok = 0;
            if( *reinterpret_cast<volatile int *>( a.error ) == 0 ) { idx = atomicAdd( a.next, 1 ); }
            if( idx < a.ntasks )
            {
                const unsigned long long taken = a.trace ? global_ns() : 0ull;
                ok = dag_wait( a.tasks[idx], a, idx );
                if( a.trace )
                {
                    a.trace[4 * (std::int64_t)idx]     = taken;
                    a.trace[4 * (std::int64_t)idx + 1] = global_ns();
                    a.trace[4 * (std::int64_t)idx + 3] = blockIdx.x;
                }
            }
            s_idx = idx;
            s_ok = ok;
        }
        __syncthreads();
        const int idx = s_idx;
        if( idx >= a.ntasks || !s_ok ) { break; }
        const DagTask t = a.tasks[idx];
        switch( static_cast<LaunchKind>( t.kind ) )
        {
            case LaunchKind::Zero:   zero_body( a.zero[t.index], arena ); break;
            case LaunchKind::Extend: extend_body( a.extend[t.index], a.lut, arena ); break;
            case LaunchKind::Potrf:  potrf_body( a.potrf[t.index], arena, a.status, dsm, a.pivot_floor, a.tinv ); break;
            case LaunchKind::Trsm:   trsm_body( a.panel[t.index], arena, a.tinv, dsm ); break;
            case LaunchKind::Gemm:
                if constexpr ( sizeof(T) == 4 ) { gemm_body( a.gemm[t.index], arena, dsm, tc, a.status ); }
                else { gemm_body( a.gemm[t.index], arena, dsm ); }
                break;
            default: break;
        }
        __threadfence();
        __syncthreads();
        if( tid == 0 )
        {
            if( a.trace ) { a.trace[4 * (std::int64_t)idx + 2] = global_ns(); }
            if( t.signal[0] >= 0 ) { atomicAdd( a.counters + t.signal[0], 1 ); }
            if( t.signal[1] >= 0 ) { atomicAdd( a.counters + t.signal[1], 1 ); }
        }
    }
    if constexpr ( sizeof(T) == 4 ) { tc_teardown( tc ); }
}

// ------------------------------------------------------ permutations, SpMV
// W rows (kw columns) <- rows p[i] of B (k columns), columns k..kw-1 zero.
__global__ void gather_rows_kernel( const double * __restrict__ B, int ldB, const std::int32_t * __restrict__ p,
                                    double * __restrict__ W, int ldw, int n, int k, int kw )
{
    const std::int64_t total = (std::int64_t)n * kw;
    for( std::int64_t e = blockIdx.x * (std::int64_t)blockDim.x + threadIdx.x; e < total;
         e += (std::int64_t)gridDim.x * blockDim.x )
    {
        const std::int64_t i = e / kw;
        const int c = static_cast<int>( e % kw );
        W[i * ldw + c] = c < k ? B[(std::int64_t)p[i] * ldB + c] : 0.0;
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
// R = B - (A + shift I) X (B != nullptr) or R = (A + shift I) X (B == nullptr)
// for row-major blocks with leading dimensions.  One warp per row: the lanes
// form 32 / KP groups of KP columns (KP = k rounded up to a power of two, at
// most 32); group g takes the row's entries g, g + G, ... (one broadcast load
// of the entry, one contiguous load of KP values of x's row), the groups'
// sums meet by log2(G) shuffles, and group 0 writes the row.  Blocks of 32
// columns when k > 32.
template<int KP>
__global__ __launch_bounds__(256) void spmv_rows_kernel( int n, const std::int64_t * __restrict__ outer, const std::int32_t * __restrict__ inner,
                                                         const double * __restrict__ vals, double shift,
                                                         const double * __restrict__ X, int ldx, const double * __restrict__ B, int ldb,
                                                         double * __restrict__ R, int ldr, int k )
{
    constexpr int G = 32 / KP;
    const int lane = threadIdx.x & 31;
    const int g = lane / KP, c = lane % KP;
    const std::int64_t warp = (blockIdx.x * (std::int64_t)blockDim.x + threadIdx.x) >> 5;
    const std::int64_t warps = ((std::int64_t)gridDim.x * blockDim.x) >> 5;
    for( std::int64_t i = warp; i < n; i += warps )
    {
        const std::int64_t e0 = outer[i], e1 = outer[i + 1];
        for( int c0 = 0; c0 < k; c0 += KP )
        {
            const int col = c0 + c;
            const bool live = col < k;
            double s = 0.0;
#pragma unroll 4
            for( std::int64_t e = e0 + g; e < e1; e += G )
            {
                const double v = vals[e];
                const std::int64_t j = inner[e];
                if( live ) { s = fma( v, X[j * ldx + col], s ); }
            }
#pragma unroll
            for( int o = KP; o < 32; o <<= 1 ) { s += __shfl_xor_sync( 0xffffffffu, s, o ); }
            if( g == 0 && live )
            {
                const double ax = s + shift * X[i * ldx + col];
                R[i * ldr + col] = B ? B[i * ldb + col] - ax : ax;
            }
        }
    }
}

// The same product for k >= 3: a group of KP lanes takes a whole row (KP
// columns of it, blocks of 32 when k > 32), 32 / KP rows per warp, with no
// cross-lane sum; the rows a warp holds together are consecutive, so rows
// with the same pattern (the dofs of one node) share their x loads in L1.
template<int KP>
__global__ __launch_bounds__(256) void spmv_group_kernel( int n, const std::int64_t * __restrict__ outer, const std::int32_t * __restrict__ inner,
                                                          const double * __restrict__ vals, double shift,
                                                          const double * __restrict__ X, int ldx, const double * __restrict__ B, int ldb,
                                                          double * __restrict__ R, int ldr, int k )
{
    constexpr int G = 32 / KP;
    const int lane = threadIdx.x & 31;
    const int g = lane / KP, c = lane % KP;
    const std::int64_t grp = ((blockIdx.x * (std::int64_t)blockDim.x + threadIdx.x) >> 5) * G + g;
    const std::int64_t groups = (((std::int64_t)gridDim.x * blockDim.x) >> 5) * G;
    for( std::int64_t i = grp; i < n; i += groups )
    {
        const std::int64_t e0 = outer[i], e1 = outer[i + 1];
        for( int c0 = 0; c0 < k; c0 += KP )
        {
            const int col = c0 + c;
            if( col >= k ) { continue; }
            // four independent sums keep four gathers of x in flight per lane
            double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
            std::int64_t e = e0;
            for( ; e + 4 <= e1; e += 4 )
            {
                const double v0 = vals[e], v1 = vals[e + 1], v2 = vals[e + 2], v3 = vals[e + 3];
                const std::int64_t j0 = inner[e], j1 = inner[e + 1], j2 = inner[e + 2], j3 = inner[e + 3];
                s0 = fma( v0, X[j0 * ldx + col], s0 );
                s1 = fma( v1, X[j1 * ldx + col], s1 );
                s2 = fma( v2, X[j2 * ldx + col], s2 );
                s3 = fma( v3, X[j3 * ldx + col], s3 );
            }
            for( ; e < e1; ++e ) { s0 = fma( vals[e], X[(std::int64_t)inner[e] * ldx + col], s0 ); }
            const double ax = ((s0 + s1) + (s2 + s3)) + shift * X[i * ldx + col];
            R[i * ldr + col] = B ? B[i * ldb + col] - ax : ax;
        }
    }
}

// out[c] += sum_i X[i][c] Y[i][c] (out zeroed by the caller).  The lanes form
// groups of KP columns as in spmv_rows_kernel, so that a warp reads whole
// rows; per block the columns' sums meet in shared memory and go out with one
// atomic addition per column.
template<int KP>
__global__ __launch_bounds__(256) void column_dots_kernel( const double * __restrict__ X, int ldx, const double * __restrict__ Y, int ldy,
                                                           int n, int k, double * __restrict__ out )
{
    constexpr int G = 32 / KP;
    __shared__ double part[8][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane / KP, c = lane % KP;
    const std::int64_t gw = (blockIdx.x * (std::int64_t)blockDim.x + threadIdx.x) >> 5;
    const std::int64_t warps = ((std::int64_t)gridDim.x * blockDim.x) >> 5;
    for( int c0 = 0; c0 < k; c0 += KP )
    {
        const int col = c0 + c;
        double s = 0.0;
        if( col < k )
        {
#pragma unroll 4
            for( std::int64_t i = gw * G + g; i < n; i += warps * G ) { s = fma( X[i * ldx + col], Y[i * ldy + col], s ); }
        }
#pragma unroll
        for( int o = KP; o < 32; o <<= 1 ) { s += __shfl_xor_sync( 0xffffffffu, s, o ); }
        if( g == 0 ) { part[warp][c] = s; }
        __syncthreads();
        if( threadIdx.x < KP && c0 + threadIdx.x < k )
        {
            double t = 0.0;
#pragma unroll
            for( int w = 0; w < 8; ++w ) { t += part[w][threadIdx.x]; }
            if( t != 0.0 ) { atomicAdd( out + c0 + threadIdx.x, t ); }
        }
        __syncthreads();
    }
}

// Conjugate-gradient updates with per-column scalars kept on the device:
// alpha_c = rz[c] / pq[c];  x += alpha p;  r -= alpha q.
__global__ void cg_update_xr_kernel( int n, int k, const double * __restrict__ rz, const double * __restrict__ pq,
                                     const double * __restrict__ p, const double * __restrict__ q,
                                     double * __restrict__ x, double * __restrict__ r )
{
    const std::int64_t total = (std::int64_t)n * k;
    for( std::int64_t e = blockIdx.x * (std::int64_t)blockDim.x + threadIdx.x; e < total; e += (std::int64_t)gridDim.x * blockDim.x )
    {
        const int c = static_cast<int>( e % k );
        const double a = pq[c] != 0.0 ? rz[c] / pq[c] : 0.0;
        x[e] += a * p[e];
        r[e] -= a * q[e];
    }
}

// beta_c = rz_new[c] / rz_old[c];  p = z + beta p.
__global__ void cg_update_p_kernel( int n, int k, const double * __restrict__ rz_new, const double * __restrict__ rz_old,
                                    const double * __restrict__ z, double * __restrict__ p )
{
    const std::int64_t total = (std::int64_t)n * k;
    for( std::int64_t e = blockIdx.x * (std::int64_t)blockDim.x + threadIdx.x; e < total; e += (std::int64_t)gridDim.x * blockDim.x )
    {
        const int c = static_cast<int>( e % k );
        const double b = rz_old[c] != 0.0 ? rz_new[c] / rz_old[c] : 0.0;
        p[e] = z[e] + b * p[e];
    }
}

// GMRES (GMRES.hpp): out[i k + c] += Q_i(:, c) . q(:, c) for the nq Krylov
// vectors Q_i (n x k each, nk apart); blockIdx.y = i.
__global__ void multi_dots_kernel( const double * __restrict__ Q, std::int64_t nk, const double * __restrict__ q,
                                   int n, int k, double * __restrict__ out )
{
    const double * Qi = Q + blockIdx.y * nk;
    for( int c = 0; c < k; ++c )
    {
        double s = 0.0;
        for( std::int64_t i = blockIdx.x * (std::int64_t)blockDim.x + threadIdx.x; i < n; i += (std::int64_t)gridDim.x * blockDim.x )
        {
            s += Qi[i * k + c] * q[i * k + c];
        }
#pragma unroll
        for( int o = 16; o > 0; o >>= 1 ) { s += __shfl_xor_sync( 0xffffffffu, s, o ); }
        if( (threadIdx.x & 31) == 0 && s != 0.0 ) { atomicAdd( out + blockIdx.y * k + c, s ); }
    }
}

// q += sign * sum_{i < nq} coef[i k + c] Q_i(:, c).
__global__ void multi_axpy_kernel( const double * __restrict__ Q, std::int64_t nk, int nq, const double * __restrict__ coef,
                                   double sign, double * __restrict__ q, int n, int k )
{
    const std::int64_t total = (std::int64_t)n * k;
    for( std::int64_t e = blockIdx.x * (std::int64_t)blockDim.x + threadIdx.x; e < total; e += (std::int64_t)gridDim.x * blockDim.x )
    {
        const int c = static_cast<int>( e % k );
        double s = 0.0;
        for( int i = 0; i < nq; ++i ) { s += coef[i * k + c] * Q[i * nk + e]; }
        q[e] += sign * s;
    }
}

// x(:, c) /= sqrt(sq[c]) where sq[c] > 0 (normalises by squared column norms).
__global__ void col_normalize_kernel( double * __restrict__ x, int n, int k, const double * __restrict__ sq )
{
    const std::int64_t total = (std::int64_t)n * k;
    for( std::int64_t e = blockIdx.x * (std::int64_t)blockDim.x + threadIdx.x; e < total; e += (std::int64_t)gridDim.x * blockDim.x )
    {
        const int c = static_cast<int>( e % k );
        if( sq[c] > 0.0 ) { x[e] /= sqrt( sq[c] ); }
    }
}

__global__ void axpy_kernel( std::int64_t n, double a, const double * __restrict__ x, double * __restrict__ y )
{
    for( std::int64_t i = blockIdx.x * (std::int64_t)blockDim.x + threadIdx.x; i < n; i += (std::int64_t)gridDim.x * blockDim.x )
    {
        y[i] += a * x[i];
    }
}

// Y = alpha X + beta Y (beta == 0: Y is not read).
__global__ void combine_kernel( int n, int k, double alpha, const double * __restrict__ X, int ldx,
                                double beta, double * __restrict__ Y, int ldy )
{
    const std::int64_t total = (std::int64_t)n * k;
    for( std::int64_t e = blockIdx.x * (std::int64_t)blockDim.x + threadIdx.x; e < total; e += (std::int64_t)gridDim.x * blockDim.x )
    {
        const std::int64_t i = e / k;
        const int c = static_cast<int>( e % k );
        double y = alpha * X[i * ldx + c];
        if( beta != 0.0 ) { y += beta * Y[i * ldy + c]; }
        Y[i * ldy + c] = y;
    }
}

template<typename T>
__global__ void gather_diag_kernel( const std::int64_t * __restrict__ offsets, const T * __restrict__ arena,
                                    double * __restrict__ out, int n )
{
    for( std::int64_t i = blockIdx.x * (std::int64_t)blockDim.x + threadIdx.x; i < n; i += (std::int64_t)gridDim.x * blockDim.x )
    {
        out[i] = static_cast<double>( arena[offsets[i]] );
    }
}

__global__ void init_status_kernel( int * status )
{
    status[0] = 0;
    status[1] = INT_MAX;
    status[2] = 0;
}

// Launch with programmatic stream serialization (see pdl_allow_next).
template<typename... KArgs, typename... Args>
void launch_pdl( void (*kernel)( KArgs... ), unsigned grid, unsigned block, size_t smem, cudaStream_t st, Args... args )
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3( grid );
    cfg.blockDim = dim3( block );
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx( &cfg, kernel, static_cast<KArgs>( args )... );
}

int grid_for( std::int64_t work, int threads )
{
    const std::int64_t blocks = (work + threads - 1) / threads;
    return static_cast<int>( blocks < 1 ? 1 : (blocks > 148 * 32 ? 148 * 32 : blocks) );
}

// ------------------------------------------------------ super-panel solve
// Large fronts solve 512 pivot rows per step (SuperPanel, plan.hpp): the
// inverse T of the 512 x 512 diagonal block, formed after the factorization
// from the 64-row panel inverses, replaces eight sequential panel steps by
// one product with T.  64 x 64 blocks throughout; warp w owns output rows
// 8w..8w+7 as 8 x 8 DMMA tiles.
constexpr int kSld = kPanel + 1;                        // padded smem row of a 64 x 64 block
// Doubles of shared memory a 64 x kSld block of T takes (rounded up to 16 bytes).
template<typename T> __host__ __device__ constexpr int super_block_doubles() { return ((kPanel * kSld * static_cast<int>( sizeof(T) ) + 15) / 16) * 2; }
constexpr size_t kSuperInvSmem = sizeof(double) * 2 * kPanel * kSld;

__device__ __forceinline__ int super_block_rows( const SuperPanel & sp, int b ) { return min( kPanel, sp.rows - b * kPanel ); }

// acc[ct] (this warp's rows of 8 x 8 tile ct) += A(64 x 64) B(64 x 64) with A through a(i, k), B through b(k, j).
template<typename FA, typename FB>
__device__ __forceinline__ void block_product_64( double (&acc)[8][2], FA a, FB b )
{
    const int warp = threadIdx.x >> 5;
    for( int kb = 0; kb < kSubs; ++kb )
    {
#pragma unroll
        for( int ct = 0; ct < 8; ++ct )
        {
            dmma_8x8x8( acc[ct], [&]( int i, int k ) { return a( 8 * warp + i, 8 * kb + k ); },
                                 [&]( int k, int j ) { return b( 8 * kb + k, 8 * ct + j ); } );
        }
    }
}

// One block (i, j) of a super-panel's inverse (round j - i; rounds run in
// order, so the blocks T_kj with k > i are complete): T_ii is panel i's
// inverse (its nb x nb part), T_ij = -T_ii sum_{k=i+1..j} U_ik T_kj.
template<typename T>
__global__ __launch_bounds__(256) void super_inv_kernel( const SuperInvTask * __restrict__ tasks, const SuperPanel * __restrict__ sps,
                                                         const T * __restrict__ arena, const double * __restrict__ tinv,
                                                         double * __restrict__ tbuf )
{
    extern __shared__ __align__(16) double ism[];
    pdl_allow_next();
    const SuperInvTask task = tasks[blockIdx.x];
    const SuperPanel sp = sps[task.sp];
    pdl_wait();
    // two 64 x 64 blocks: the products' operands, then S (in A's place) and T_ii (in Bm's)
    double (*A)[kSld] = reinterpret_cast<double (*)[kSld]>( ism );
    double (*Bm)[kSld] = A + kPanel;
    double (*S)[kSld] = A;
    double (*Tii)[kSld] = Bm;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int i = task.i, j = task.j;
    const int nbi = super_block_rows( sp, i );
    double * out = tbuf + sp.t + (std::int64_t)(kPanel * i) * sp.ldt + kPanel * j;
    auto load_tinv = [&]( double (*D)[kSld], int b, int nbb )
    {
        const double * src = tinv + (std::int64_t)sp.panel[b] * (kPanel * kPanel);
#pragma unroll 4
        for( int idx = tid; idx < kPanel * kPanel; idx += 256 )
        {
            const int r = idx >> 6, c = idx & 63;
            const bool valid = r < nbb && c < nbb;
            cp_async_8( &D[r][c], valid ? src + idx : src, valid );
        }
        cp_async_wait_all();
    };
    if( i == j )
    {
        load_tinv( Tii, i, nbi );
        __syncthreads();
        for( int idx = tid; idx < kPanel * kPanel; idx += 256 ) { out[(idx >> 6) * sp.ldt + (idx & 63)] = Tii[idx >> 6][idx & 63]; }
        return;
    }
    double acc[8][2];
#pragma unroll
    for( int ct = 0; ct < 8; ++ct ) { acc[ct][0] = 0.0; acc[ct][1] = 0.0; }
    const T * U0 = arena + sp.u0;
    for( int k = i + 1; k <= j; ++k )
    {
        const int nbk = super_block_rows( sp, k );
        const double * tk = tbuf + sp.t + (std::int64_t)(kPanel * k) * sp.ldt + kPanel * j;
        auto src = [&]( int idx, double & fill ) -> const T *
        {
            fill = 0.0;
            const int r = idx >> 6, c = idx & 63;
            return (r < nbi && c < nbk) ? U0 + (std::int64_t)(sp.r0 + kPanel * i + r) * sp.ld0 + sp.r0 + kPanel * k + c : nullptr;
        };
        auto dst = [&]( int idx ) { return &A[idx >> 6][idx & 63]; };
        stage_block<T, kPanel * kPanel / 256, 256>( U0, src, dst );
        // T_kj is zero outside its valid rows and columns
#pragma unroll 4
        for( int idx = tid; idx < kPanel * kPanel; idx += 256 ) { cp_async_8( &Bm[idx >> 6][idx & 63], tk + (idx >> 6) * sp.ldt + (idx & 63), true ); }
        cp_async_wait_all();
        stage_finish<T, kPanel * kPanel / 256, 256>( src, dst );
        __syncthreads();
        block_product_64( acc, [&]( int r, int c ) { return A[r][c]; }, [&]( int r, int c ) { return Bm[r][c]; } );
        __syncthreads();
    }
#pragma unroll
    for( int ct = 0; ct < 8; ++ct )
    {
        S[8 * warp + (lane >> 2)][8 * ct + 2 * (lane & 3)] = acc[ct][0];
        S[8 * warp + (lane >> 2)][8 * ct + 2 * (lane & 3) + 1] = acc[ct][1];
        acc[ct][0] = 0.0; acc[ct][1] = 0.0;
    }
    load_tinv( Tii, i, nbi );
    __syncthreads();
    block_product_64( acc, [&]( int r, int c ) { return Tii[r][c]; }, [&]( int r, int c ) { return S[r][c]; } );
#pragma unroll
    for( int ct = 0; ct < 8; ++ct )
    {
        const int r = 8 * warp + (lane >> 2), c = 8 * ct + 2 * (lane & 3);
        out[r * sp.ldt + c] = -acc[ct][0];
        out[r * sp.ldt + c + 1] = -acc[ct][1];
    }
}

// Stages x rows [row, row + nr) (leading dimension ld, k columns) of a sweep
// vector into V (64 x KP, leading dimension KP + 4) with 8-byte asynchronous
// copies; cells outside nr x k are zero.
template<int KP>
__device__ __forceinline__ void stage_rows( double * V, const double * x, std::int64_t row, int nr, int ld, int k )
{
    constexpr int ldv = KP + 4;
#pragma unroll 4
    for( int idx = threadIdx.x; idx < kPanel * KP; idx += 256 )
    {
        const int r = idx / KP, c = idx % KP;
        const bool ok = r < nr && c < k;
        cp_async_8( V + r * ldv + c, ok ? x + (row + r) * ld + c : x, ok );
    }
}

// One block pair of a super-panel's diag step.  Forward (task (o, b), b <= o):
// x_o += T_bo^T y_b; back (b >= o): x_o += T_ob (y_b + z_b).  y: `in`, z: the
// rest steps' sums in `zbuf`, x: `out`, whose block rows are zero before the
// step (the pairs of one block row add into it).  KP = k rounded up to a power
// of two >= 8.  One 64 x 64 block of T and one 64 x k block of vectors per
// CTA, all copies in flight together.
template<int KP>
__global__ __launch_bounds__(256) void super_diag_kernel( const SuperSolveTask * __restrict__ tasks, const SuperPanel * __restrict__ sps,
                                                          const double * __restrict__ tbuf, int upper, const double * in,
                                                          const double * zbuf, double * out, int ld, int k )
{
    extern __shared__ __align__(16) double dsm[];
    pdl_allow_next();
    const SuperSolveTask task = tasks[blockIdx.x];
    const SuperPanel sp = sps[task.sp];
    constexpr int nct = KP / 8;
    constexpr int ldv = KP + 4;
    double (*Tb)[kSld] = reinterpret_cast<double (*)[kSld]>( dsm );
    double * V = dsm + kPanel * kSld;                  // [64][ldv]
    double * Z = V + kPanel * ldv;                     // [64][ldv], back sweep only
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int o = task.blk, b = task.c0;
    const int nbb = super_block_rows( sp, b );
    const std::int64_t brow = (std::int64_t)sp.row0 + sp.r0;
    // forward: block (b, o) of T, read transposed; back: block (o, b).  The
    // blocks are zero outside their valid rows and columns.
    const double * tb = upper ? tbuf + sp.t + (std::int64_t)(kPanel * o) * sp.ldt + kPanel * b
                              : tbuf + sp.t + (std::int64_t)(kPanel * b) * sp.ldt + kPanel * o;
#pragma unroll 4
    for( int idx = tid; idx < kPanel * kPanel; idx += 256 ) { cp_async_8( &Tb[idx >> 6][idx & 63], tb + (idx >> 6) * sp.ldt + (idx & 63), true ); }
    pdl_wait();
    stage_rows<KP>( V, in, brow + kPanel * b, nbb, ld, k );
    if( upper ) { stage_rows<KP>( Z, zbuf, brow + kPanel * b, nbb, ld, k ); }
    cp_async_wait_all();
    if( upper )
    {
        for( int idx = tid; idx < kPanel * KP; idx += 256 ) { V[(idx / KP) * ldv + idx % KP] += Z[(idx / KP) * ldv + idx % KP]; }
    }
    __syncthreads();
    double acc[nct][2];
#pragma unroll
    for( int ct = 0; ct < nct; ++ct ) { acc[ct][0] = 0.0; acc[ct][1] = 0.0; }
    for( int kb = 0; kb < kSubs; ++kb )
    {
#pragma unroll
        for( int ct = 0; ct < nct; ++ct )
        {
            if( upper ) { dmma_8x8x8( acc[ct], [&]( int i, int kk ) { return Tb[8 * warp + i][8 * kb + kk]; },
                                               [&]( int kk, int j ) { return V[(8 * kb + kk) * ldv + 8 * ct + j]; } ); }
            else        { dmma_8x8x8( acc[ct], [&]( int i, int kk ) { return Tb[8 * kb + kk][8 * warp + i]; },
                                               [&]( int kk, int j ) { return V[(8 * kb + kk) * ldv + 8 * ct + j]; } ); }
        }
    }
    const int nbo = super_block_rows( sp, o );
    const int r = 8 * warp + (lane >> 2);
    if( r < nbo )
    {
        double * dst = out + (brow + kPanel * o + r) * ld;
#pragma unroll
        for( int ct = 0; ct < nct; ++ct )
        {
            const int c = 8 * ct + 2 * (lane & 3);
            if( c < k ) { red_add_f64( dst + c, acc[ct][0] ); }
            if( c + 1 < k ) { red_add_f64( dst + c + 1, acc[ct][1] ); }
        }
    }
}

// One (block, rest chunk) pair of a super-panel's rest step, rest columns
// [c0, c1) of block b.  Forward: y_rest -= U_{b,rest}^T x_b (x_b: `out`, final
// after the diag step; y: `in`, every row by reductions, as the eight blocks
// add into the same rows).  Back: z_b -= U_{b,rest} x_rest (x_rest: `out`,
// final; z: reductions into `zbuf`).
template<typename T, int KP>
__global__ __launch_bounds__(256) void super_rest_kernel( const SuperSolveTask * __restrict__ tasks, const SuperPanel * __restrict__ sps,
                                                          const T * __restrict__ arena, const std::int32_t * __restrict__ sn_inner,
                                                          int upper, double * in, double * zbuf, const double * out, int ld, int k )
{
    extern __shared__ __align__(16) double rsm[];
    pdl_allow_next();
    const SuperSolveTask task = tasks[blockIdx.x];
    const SuperPanel sp = sps[task.sp];
    constexpr int nct = KP / 8;
    constexpr int ldv = KP + 4;
    __shared__ std::int64_t trow[kSolveRest];
    // the factor block in the factor's type (FP32 storage: half the shared memory), widened as read
    T (*P)[kSld] = reinterpret_cast<T (*)[kSld]>( rsm );
    double * V = rsm + super_block_doubles<T>();        // [64][ldv]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int r1 = sp.r0 + sp.rows;
    const int m = sp.n0 - r1;
    const int cw = task.c1 - task.c0;
    const int b = task.blk;
    const int nbb = super_block_rows( sp, b );
    const std::int64_t brow = (std::int64_t)sp.row0 + sp.r0;
    if( tid < kSolveRest )
    {
        const int col = task.c0 + tid;
        trow[tid] = (tid < cw) ? ((col < m) ? (std::int64_t)sp.row0 + r1 + col : (std::int64_t)sn_inner[sp.inner + (col - m)]) : -1;
    }
    // P: rows of block b (U rows r0 + 64 b + rr), the chunk's rest columns
    const T * U0 = arena + sp.u0;
    const T * U1 = arena + sp.u1;
#pragma unroll 4
    for( int idx = tid; idx < kPanel * kPanel; idx += 256 )
    {
        const int rr = idx >> 6, jj = idx & 63;
        const bool valid = rr < nbb && jj < cw;
        const int col = task.c0 + jj;
        const std::int64_t urow = sp.r0 + kPanel * b + rr;
        const T * src = !valid ? U0 : col < m ? U0 + urow * sp.ld0 + r1 + col : U1 + urow * sp.ld1 + (col - m);
        if constexpr ( sizeof(T) == 8 ) { cp_async_8( reinterpret_cast<double *>( &P[rr][jj] ), reinterpret_cast<const double *>( src ), valid ); }
        else { cp_async_4( &P[rr][jj], src, valid ); }
    }
    pdl_wait();
    __syncthreads();                                    // trow
    if( upper )
    {
        // x_rest: the chunk's rows of `out`
#pragma unroll 4
        for( int idx = tid; idx < kPanel * KP; idx += 256 )
        {
            const int r = idx / KP, c = idx % KP;
            const bool ok = r < cw && c < k;
            cp_async_8( V + r * ldv + c, ok ? out + trow[r] * ld + c : out, ok );
        }
    }
    else { stage_rows<KP>( V, out, brow + kPanel * b, nbb, ld, k ); }
    cp_async_wait_all();
    __syncthreads();
    double acc[nct][2];
#pragma unroll
    for( int ct = 0; ct < nct; ++ct ) { acc[ct][0] = 0.0; acc[ct][1] = 0.0; }
    for( int kb = 0; kb < kSubs; ++kb )
    {
#pragma unroll
        for( int ct = 0; ct < nct; ++ct )
        {
            // forward: acc(jj, c) = sum_rr P[rr][jj] x_b[rr][c]; back: acc(rr, c) = sum_jj P[rr][jj] x_rest[jj][c]
            if( upper ) { dmma_8x8x8( acc[ct], [&]( int i, int kk ) { return static_cast<double>( P[8 * warp + i][8 * kb + kk] ); },
                                               [&]( int kk, int j ) { return V[(8 * kb + kk) * ldv + 8 * ct + j]; } ); }
            else        { dmma_8x8x8( acc[ct], [&]( int i, int kk ) { return static_cast<double>( P[8 * kb + kk][8 * warp + i] ); },
                                               [&]( int kk, int j ) { return V[(8 * kb + kk) * ldv + 8 * ct + j]; } ); }
        }
    }
    const int r = 8 * warp + (lane >> 2);
    if( upper ? r < nbb : r < cw )
    {
        double * row = upper ? zbuf + (brow + kPanel * b + r) * ld : in + trow[r] * ld;
#pragma unroll
        for( int ct = 0; ct < nct; ++ct )
        {
            const int c = 8 * ct + 2 * (lane & 3);
            if( c < k ) { red_add_f64( row + c, -acc[ct][0] ); }
            if( c + 1 < k ) { red_add_f64( row + c + 1, -acc[ct][1] ); }
        }
    }
}

} // namespace

template<typename T>
void launch_assemble( const double * values, const std::int64_t * src, const std::int64_t * dst,
                      std::int64_t count, const double * reg, T * arena, cudaStream_t st )
{
    if( count <= 0 ) { return; }
    assemble_kernel<<<grid_for( count, 256 ), 256, 0, st>>>( values, src, dst, count, reg, arena );
}

template<typename T>
void launch_zero( const ZeroTask * tasks, int count, T * arena, cudaStream_t st )
{
    if( count > 0 ) { launch_pdl( zero_kernel<T>, count, 256, 0, st, tasks, arena ); }
}

template<typename T>
void launch_export( const ExportTask * tasks, int count, const std::int32_t * colmap, const T * arena,
                    double * tri, double * rec, cudaStream_t st )
{
    if( count > 0 ) { export_kernel<<<count, 128, 0, st>>>( tasks, colmap, arena, tri, rec ); }
}

template<typename T>
void launch_extend( const ExtendTask * tasks, int count, const std::int32_t * lut, T * arena, cudaStream_t st )
{
    if( count > 0 ) { launch_pdl( extend_kernel<T>, count, 256, 0, st, tasks, lut, arena ); }
}

template<typename T>
void launch_extend_pull( const ExtendPullTask * tasks, int count, const ExtendTask * segs, const std::int32_t * lut, T * arena,
                         cudaStream_t st )
{
    if( count > 0 ) { launch_pdl( extend_pull_kernel<T>, count, 256, 0, st, tasks, segs, lut, arena ); }
}

template<typename T>
void launch_potrf( const PanelTask * tasks, int count, T * arena, int * status, const double * pivot_floor, double * tinv,
                   cudaStream_t st )
{
    if( count > 0 ) { launch_pdl( potrf_kernel<T>, count, kPotrfThreads, kPotrfSmemBytes, st, tasks, arena, status, pivot_floor, tinv ); }
}

// floor[i] = rel * |diagonal entry of row i| after assembly (FP32 storage).
// out[1 + i] = rel * |a_ii|; out[0] = max_i |a_ii| (cleared by the caller),
// by an integer maximum over the bit patterns of non-negative doubles.
__global__ void pivot_floor_kernel( const std::int64_t * __restrict__ offsets, const float * __restrict__ arena, double rel,
                                    double * __restrict__ out, int n )
{
    unsigned long long mx = 0ull;
    for( std::int64_t i = blockIdx.x * (std::int64_t)blockDim.x + threadIdx.x; i < n; i += (std::int64_t)gridDim.x * blockDim.x )
    {
        const double a = fabs( static_cast<double>( arena[offsets[i]] ) );
        out[1 + i] = rel * a;
        const unsigned long long bits = static_cast<unsigned long long>( __double_as_longlong( a ) );
        mx = bits > mx ? bits : mx;
    }
#pragma unroll
    for( int o = 16; o > 0; o >>= 1 )
    {
        const unsigned long long v = __shfl_xor_sync( 0xffffffffu, mx, o );
        mx = v > mx ? v : mx;
    }
    if( (threadIdx.x & 31) == 0 && mx != 0ull ) { atomicMax( reinterpret_cast<unsigned long long *>( out ), mx ); }
}

void launch_pivot_floor( const std::int64_t * offsets, const float * arena, double rel, double * out, int n, cudaStream_t st )
{
    cudaMemsetAsync( out, 0, sizeof(double), st );
    pivot_floor_kernel<<<grid_for( n, 256 ), 256, 0, st>>>( offsets, arena, rel, out, n );
}

template<typename T>
void launch_trsm( const PanelTask * tasks, int count, T * arena, const double * tinv, cudaStream_t st, float * img )
{
    if( count > 0 ) { launch_pdl( trsm_kernel<T>, count, kTrsmThreads, kTrsmSmemBytes, st, tasks, arena, tinv, img ); }
}

template<typename T>
void launch_gemm( const GemmTask * tasks, int count, T * arena, int * status, cudaStream_t st )
{
    if( count <= 0 ) { return; }
    if constexpr ( sizeof(T) == 8 )
    {
        (void)status;
        launch_pdl( gemm_tn_kernel, count, kGemmThreads, kGemmSmemBytes, st, tasks, arena );
    }
    else
    {
        int dev = 0, sms = 0;
        cudaGetDevice( &dev );
        cudaDeviceGetAttribute( &sms, cudaDevAttrMultiProcessorCount, dev );
        const int grid = std::min( count, 3 * std::max( sms, 1 ) );
        launch_pdl( gemm_tc_kernel, grid, kGemmThreads, kGemmSmemBytesF, st, tasks, count, arena, status );
    }
}

template<typename T>
void launch_factor_dag( const DagArgs & args, int grid, cudaStream_t st )
{
    if( args.ntasks > 0 && grid > 0 ) { factor_dag_kernel<T><<<grid, kDagThreads, kDagSmemBytes, st>>>( args ); }
}

// The occupancy query answers 1 for the FP32 instance, which allocates tensor
// memory, although 3 such CTAs (64 KB of shared memory and 64 TMEM columns
// each) were measured co-resident on one SM; both instances have the same
// shared memory and launch bounds, so the FP64 instance's answer is used for
// both.  Correctness does not depend on residency: tasks are taken by running
// CTAs in a topological order.
int factor_dag_blocks_per_sm()
{
    int b = 0;
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor( &b, factor_dag_kernel<double>, kDagThreads, kDagSmemBytes );
    return e == cudaSuccess ? b : 0;
}


static int solve_lkp( int k )
{
    int l = 3;
    while( (1 << l) < k ) { ++l; }
    return l;
}

template<typename T>
static size_t solve_smem_bytes( int k )
{
    return sizeof(double) * (kPanel * kTld + 2 * kPanel * ((1 << solve_lkp( k )) + 4));
}

template<typename T>
void launch_solve_dag( const SolveDagArgs & args, int grid, const T * arena, double * in, double * out, int ld, int k,
                       cudaStream_t st )
{
    if( args.ntasks <= 0 || grid <= 0 ) { return; }
    const size_t sm = solve_smem_bytes<T>( k );
    switch( solve_lkp( k ) )
    {
        case 3:  solve_dag_kernel<T, 8><<<grid, kSolveThreads, sm, st>>>( args, arena, in, out, ld, k ); break;
        case 4:  solve_dag_kernel<T, 16><<<grid, kSolveThreads, sm, st>>>( args, arena, in, out, ld, k ); break;
        case 5:  solve_dag_kernel<T, 32><<<grid, kSolveThreads, sm, st>>>( args, arena, in, out, ld, k ); break;
        default: solve_dag_kernel<T, 64><<<grid, kSolveThreads, sm, st>>>( args, arena, in, out, ld, k ); break;
    }
}

template<typename T>
int solve_dag_occupancy( int k )
{
    const size_t sm = solve_smem_bytes<T>( k );
    int n = 0;
    cudaError_t e = cudaSuccess;
    switch( solve_lkp( k ) )
    {
        case 3:  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor( &n, solve_dag_kernel<T, 8>, kSolveThreads, sm ); break;
        case 4:  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor( &n, solve_dag_kernel<T, 16>, kSolveThreads, sm ); break;
        case 5:  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor( &n, solve_dag_kernel<T, 32>, kSolveThreads, sm ); break;
        default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor( &n, solve_dag_kernel<T, 64>, kSolveThreads, sm ); break;
    }
    return e == cudaSuccess ? n : 0;
}

int solve_dag_blocks_per_sm( int k )
{
    return std::min( solve_dag_occupancy<double>( k ), solve_dag_occupancy<float>( k ) );
}

template<typename T>
void launch_solve_step( const SolveRestTask * tasks, int count, bool upper, const T * arena, const double * tinv,
                        const std::int32_t * sn_inner, double * in, double * out, int ld, int k, cudaStream_t st )
{
    if( count <= 0 ) { return; }
    const size_t sm = solve_smem_bytes<T>( k );
    const int u = upper ? 1 : 0;
    switch( solve_lkp( k ) )
    {
        case 3:  launch_pdl( solve_step_kernel<T, 8>, count, kSolveThreads, sm, st, tasks, u, arena, tinv, sn_inner, in, out, ld, k ); break;
        case 4:  launch_pdl( solve_step_kernel<T, 16>, count, kSolveThreads, sm, st, tasks, u, arena, tinv, sn_inner, in, out, ld, k ); break;
        case 5:  launch_pdl( solve_step_kernel<T, 32>, count, kSolveThreads, sm, st, tasks, u, arena, tinv, sn_inner, in, out, ld, k ); break;
        default: launch_pdl( solve_step_kernel<T, 64>, count, kSolveThreads, sm, st, tasks, u, arena, tinv, sn_inner, in, out, ld, k ); break;
    }
}

template<typename T>
void launch_super_inv( const SuperInvTask * tasks, int count, const SuperPanel * sps, const T * arena, const double * tinv,
                       double * tbuf, cudaStream_t st )
{
    if( count > 0 ) { launch_pdl( super_inv_kernel<T>, count, 256, kSuperInvSmem, st, tasks, sps, arena, tinv, tbuf ); }
}

static size_t super_solve_smem( int k )
{
    return sizeof(double) * (kPanel * kSld + 2 * kPanel * ((1 << solve_lkp( k )) + 4));
}

template<typename T>
static size_t super_rest_smem( int k )
{
    return sizeof(double) * (super_block_doubles<T>() + kPanel * ((1 << solve_lkp( k )) + 4));
}

void launch_super_diag( const SuperSolveTask * tasks, int count, const SuperPanel * sps, const double * tbuf, bool upper,
                        const double * in, const double * zbuf, double * out, int ld, int k, cudaStream_t st )
{
    if( count <= 0 ) { return; }
    const size_t sm = super_solve_smem( k );
    const int u = upper ? 1 : 0;
    switch( solve_lkp( k ) )
    {
        case 3:  launch_pdl( super_diag_kernel<8>, count, 256, sm, st, tasks, sps, tbuf, u, in, zbuf, out, ld, k ); break;
        case 4:  launch_pdl( super_diag_kernel<16>, count, 256, sm, st, tasks, sps, tbuf, u, in, zbuf, out, ld, k ); break;
        case 5:  launch_pdl( super_diag_kernel<32>, count, 256, sm, st, tasks, sps, tbuf, u, in, zbuf, out, ld, k ); break;
        default: launch_pdl( super_diag_kernel<64>, count, 256, sm, st, tasks, sps, tbuf, u, in, zbuf, out, ld, k ); break;
    }
}

template<typename T>
void launch_super_rest( const SuperSolveTask * tasks, int count, const SuperPanel * sps, const T * arena,
                        const std::int32_t * sn_inner, bool upper, double * in, double * zbuf, const double * out, int ld, int k,
                        cudaStream_t st )
{
    if( count <= 0 ) { return; }
    const size_t sm = super_rest_smem<T>( k );
    const int u = upper ? 1 : 0;
    switch( solve_lkp( k ) )
    {
        case 3:  launch_pdl( super_rest_kernel<T, 8>, count, 256, sm, st, tasks, sps, arena, sn_inner, u, in, zbuf, out, ld, k ); break;
        case 4:  launch_pdl( super_rest_kernel<T, 16>, count, 256, sm, st, tasks, sps, arena, sn_inner, u, in, zbuf, out, ld, k ); break;
        case 5:  launch_pdl( super_rest_kernel<T, 32>, count, 256, sm, st, tasks, sps, arena, sn_inner, u, in, zbuf, out, ld, k ); break;
        default: launch_pdl( super_rest_kernel<T, 64>, count, 256, sm, st, tasks, sps, arena, sn_inner, u, in, zbuf, out, ld, k ); break;
    }
}

template<typename T>
void launch_gather_diag( const std::int64_t * offsets, const T * arena, double * out, int n, cudaStream_t st )
{
    gather_diag_kernel<<<grid_for( n, 256 ), 256, 0, st>>>( offsets, arena, out, n );
}

#define TB_INSTANTIATE( T )                                                                                          \
    template void launch_assemble<T>( const double *, const std::int64_t *, const std::int64_t *, std::int64_t,      \
                                      const double *, T *, cudaStream_t );                                         \
    template void launch_zero<T>( const ZeroTask *, int, T *, cudaStream_t );                                        \
    template void launch_export<T>( const ExportTask *, int, const std::int32_t *, const T *, double *, double *,    \
                                    cudaStream_t );                                                                \
    template void launch_extend<T>( const ExtendTask *, int, const std::int32_t *, T *, cudaStream_t );             \
    template void launch_extend_pull<T>( const ExtendPullTask *, int, const ExtendTask *, const std::int32_t *, T *, cudaStream_t ); \
    template void launch_potrf<T>( const PanelTask *, int, T *, int *, const double *, double *, cudaStream_t );     \
    template void launch_trsm<T>( const PanelTask *, int, T *, const double *, cudaStream_t, float * );              \
    template void launch_gemm<T>( const GemmTask *, int, T *, int *, cudaStream_t );                                 \
    template void launch_solve_dag<T>( const SolveDagArgs &, int, const T *, double *, double *, int, int, cudaStream_t );                                        \
    template void launch_factor_dag<T>( const DagArgs &, int, cudaStream_t );                                        \
    template void launch_solve_step<T>( const SolveRestTask *, int, bool, const T *, const double *,                \
                                        const std::int32_t *, double *, double *, int, int, cudaStream_t );         \
    template void launch_gather_diag<T>( const std::int64_t *, const T *, double *, int, cudaStream_t );          \
    template void launch_super_inv<T>( const SuperInvTask *, int, const SuperPanel *, const T *, const double *,      \
                                       double *, cudaStream_t );                                                    \
    template void launch_super_rest<T>( const SuperSolveTask *, int, const SuperPanel *, const T *,                 \
                                        const std::int32_t *, bool, double *, double *, const double *, int, int,   \
                                        cudaStream_t );
TB_INSTANTIATE( double )
TB_INSTANTIATE( float )
#undef TB_INSTANTIATE

void launch_gather_rows( const double * B, int ldB, const std::int32_t * p, double * W, int ldw,
                         int n, int k, cudaStream_t st, int kw )
{
    kw = std::max( kw, k );
    gather_rows_kernel<<<grid_for( (std::int64_t)n * kw, 256 ), 256, 0, st>>>( B, ldB, p, W, ldw, n, k, kw );
}

void launch_scatter_rows( const double * W, int ldw, const std::int32_t * p_inv, double alpha, double beta,
                          double * Y, int ldY, int n, int k, cudaStream_t st )
{
    scatter_rows_kernel<<<grid_for( (std::int64_t)n * k, 256 ), 256, 0, st>>>( W, ldw, p_inv, alpha, beta, Y, ldY, n, k );
}

template<typename Launch>
static void by_column_width( int k, Launch launch )
{
    if( k <= 1 ) { launch( std::integral_constant<int, 1>{} ); }
    else if( k <= 2 ) { launch( std::integral_constant<int, 2>{} ); }
    else if( k <= 4 ) { launch( std::integral_constant<int, 4>{} ); }
    else if( k <= 8 ) { launch( std::integral_constant<int, 8>{} ); }
    else if( k <= 16 ) { launch( std::integral_constant<int, 16>{} ); }
    else { launch( std::integral_constant<int, 32>{} ); }
}

void launch_residual( int n, const std::int64_t * outer, const std::int32_t * inner, const double * vals,
                      const double * X, const double * B, double * R, int k, cudaStream_t st )
{
    launch_apply_shifted( n, outer, inner, vals, 0.0, X, k, B, k, R, k, k, st );
}

cudaError_t configure_kernels()
{
    const struct { const void * fn; size_t bytes; } attrs[] = {
        { reinterpret_cast<const void *>( potrf_kernel<double> ), kPotrfSmemBytes },
        { reinterpret_cast<const void *>( potrf_kernel<float> ), kPotrfSmemBytes },
        { reinterpret_cast<const void *>( trsm_kernel<double> ), kTrsmSmemBytes },
        { reinterpret_cast<const void *>( trsm_kernel<float> ), kTrsmSmemBytes },
        { reinterpret_cast<const void *>( gemm_tn_kernel ), kGemmSmemBytes },
        { reinterpret_cast<const void *>( gemm_tc_kernel ), kGemmSmemBytesF },
        { reinterpret_cast<const void *>( factor_dag_kernel<double> ), kDagSmemBytes },
        { reinterpret_cast<const void *>( factor_dag_kernel<float> ), kDagSmemBytes },
        { reinterpret_cast<const void *>( solve_step_kernel<double, 8> ), solve_smem_bytes<double>( 8 ) },
        { reinterpret_cast<const void *>( solve_step_kernel<double, 16> ), solve_smem_bytes<double>( 16 ) },
        { reinterpret_cast<const void *>( solve_step_kernel<double, 32> ), solve_smem_bytes<double>( 32 ) },
        { reinterpret_cast<const void *>( solve_step_kernel<double, 64> ), solve_smem_bytes<double>( 64 ) },
        { reinterpret_cast<const void *>( solve_step_kernel<float, 8> ), solve_smem_bytes<float>( 8 ) },
        { reinterpret_cast<const void *>( solve_step_kernel<float, 16> ), solve_smem_bytes<float>( 16 ) },
        { reinterpret_cast<const void *>( solve_step_kernel<float, 32> ), solve_smem_bytes<float>( 32 ) },
        { reinterpret_cast<const void *>( solve_step_kernel<float, 64> ), solve_smem_bytes<float>( 64 ) },
        { reinterpret_cast<const void *>( solve_dag_kernel<double, 8> ), solve_smem_bytes<double>( 8 ) },
        { reinterpret_cast<const void *>( solve_dag_kernel<double, 16> ), solve_smem_bytes<double>( 16 ) },
        { reinterpret_cast<const void *>( solve_dag_kernel<double, 32> ), solve_smem_bytes<double>( 32 ) },
        { reinterpret_cast<const void *>( solve_dag_kernel<double, 64> ), solve_smem_bytes<double>( 64 ) },
        { reinterpret_cast<const void *>( solve_dag_kernel<float, 8> ), solve_smem_bytes<float>( 8 ) },
        { reinterpret_cast<const void *>( solve_dag_kernel<float, 16> ), solve_smem_bytes<float>( 16 ) },
        { reinterpret_cast<const void *>( solve_dag_kernel<float, 32> ), solve_smem_bytes<float>( 32 ) },
        { reinterpret_cast<const void *>( solve_dag_kernel<float, 64> ), solve_smem_bytes<float>( 64 ) },
        { reinterpret_cast<const void *>( super_inv_kernel<double> ), kSuperInvSmem },
        { reinterpret_cast<const void *>( super_inv_kernel<float> ), kSuperInvSmem },
        { reinterpret_cast<const void *>( super_diag_kernel<8> ), super_solve_smem( 8 ) },
        { reinterpret_cast<const void *>( super_diag_kernel<16> ), super_solve_smem( 16 ) },
        { reinterpret_cast<const void *>( super_diag_kernel<32> ), super_solve_smem( 32 ) },
        { reinterpret_cast<const void *>( super_diag_kernel<64> ), super_solve_smem( 64 ) },
        { reinterpret_cast<const void *>( super_rest_kernel<double, 8> ), super_rest_smem<double>( 8 ) },
        { reinterpret_cast<const void *>( super_rest_kernel<double, 16> ), super_rest_smem<double>( 16 ) },
        { reinterpret_cast<const void *>( super_rest_kernel<double, 32> ), super_rest_smem<double>( 32 ) },
        { reinterpret_cast<const void *>( super_rest_kernel<double, 64> ), super_rest_smem<double>( 64 ) },
        { reinterpret_cast<const void *>( super_rest_kernel<float, 8> ), super_rest_smem<float>( 8 ) },
        { reinterpret_cast<const void *>( super_rest_kernel<float, 16> ), super_rest_smem<float>( 16 ) },
        { reinterpret_cast<const void *>( super_rest_kernel<float, 32> ), super_rest_smem<float>( 32 ) },
        { reinterpret_cast<const void *>( super_rest_kernel<float, 64> ), super_rest_smem<float>( 64 ) },
    };
    for( const auto & a : attrs )
    {
        const cudaError_t e = cudaFuncSetAttribute( a.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)a.bytes );
        if( e != cudaSuccess ) { return e; }
    }
    return cudaSuccess;
}

void launch_apply_shifted( int n, const std::int64_t * outer, const std::int32_t * inner, const double * vals,
                           double shift, const double * X, int ldx, const double * B, int ldb, double * R, int ldr,
                           int k, cudaStream_t st )
{
    if( n <= 0 ) { return; }
    if( k >= 3 )
    {
        // one warp per 32 / KP rows, up to 32 blocks per SM (measured best on a 3-dof 27-point stencil)
        const int grid = grid_for( (std::int64_t)n * 32, 256 );
        by_column_width( k, [&]( auto kp ) {
            if constexpr ( decltype( kp )::value >= 4 )
            {
                spmv_group_kernel<decltype( kp )::value><<<grid, 256, 0, st>>>( n, outer, inner, vals, shift, X, ldx, B, ldb, R, ldr, k );
            }
        } );
        return;
    }
    const int grid = grid_for( (std::int64_t)n * 32, 256 );
    by_column_width( k, [&]( auto kp ) {
        spmv_rows_kernel<decltype( kp )::value><<<grid, 256, 0, st>>>( n, outer, inner, vals, shift, X, ldx, B, ldb, R, ldr, k );
    } );
}

void launch_column_dots( const double * X, int ldx, const double * Y, int ldy, int n, int k, double * out, cudaStream_t st )
{
    if( n <= 0 ) { return; }
    // two blocks per SM: few atomics per column, every row read once
    const int grid = static_cast<int>( std::min<std::int64_t>( 296, ((std::int64_t)n + 255) / 256 ) );
    by_column_width( k, [&]( auto kp ) {
        column_dots_kernel<decltype( kp )::value><<<grid, 256, 0, st>>>( X, ldx, Y, ldy, n, k, out );
    } );
}

void launch_cg_update_xr( int n, int k, const double * rz, const double * pq, const double * p, const double * q,
                          double * x, double * r, cudaStream_t st )
{
    cg_update_xr_kernel<<<grid_for( (std::int64_t)n * k, 256 ), 256, 0, st>>>( n, k, rz, pq, p, q, x, r );
}

void launch_cg_update_p( int n, int k, const double * rz_new, const double * rz_old, const double * z, double * p,
                         cudaStream_t st )
{
    cg_update_p_kernel<<<grid_for( (std::int64_t)n * k, 256 ), 256, 0, st>>>( n, k, rz_new, rz_old, z, p );
}

void launch_multi_dots( const double * Q, std::int64_t nk, int nq, const double * q, int n, int k, double * out, cudaStream_t st )
{
    if( nq <= 0 ) { return; }
    multi_dots_kernel<<<dim3( static_cast<unsigned>( grid_for( n, 256 ) ), static_cast<unsigned>( nq ) ), 256, 0, st>>>( Q, nk, q, n, k, out );
}

void launch_multi_axpy( const double * Q, std::int64_t nk, int nq, const double * coef, double sign, double * q, int n, int k,
                        cudaStream_t st )
{
    if( nq <= 0 ) { return; }
    multi_axpy_kernel<<<grid_for( (std::int64_t)n * k, 256 ), 256, 0, st>>>( Q, nk, nq, coef, sign, q, n, k );
}

void launch_col_normalize( double * x, int n, int k, const double * sq, cudaStream_t st )
{
    col_normalize_kernel<<<grid_for( (std::int64_t)n * k, 256 ), 256, 0, st>>>( x, n, k, sq );
}

void launch_axpy( std::int64_t n, double a, const double * x, double * y, cudaStream_t st )
{
    axpy_kernel<<<grid_for( n, 256 ), 256, 0, st>>>( n, a, x, y );
}

void launch_combine( int n, int k, double alpha, const double * X, int ldx, double beta, double * Y, int ldy, cudaStream_t st )
{
    combine_kernel<<<grid_for( (std::int64_t)n * k, 256 ), 256, 0, st>>>( n, k, alpha, X, ldx, beta, Y, ldy );
}

// Row-major n x k blocks between the two scalar types (the reference casts
// right-hand sides and solutions on copy, Solve.hpp:20-27).
template<typename S, typename D>
__global__ void convert_rows_kernel( const S * __restrict__ src, int lds, D * __restrict__ dst, int ldd, std::int64_t n, int k )
{
    const std::int64_t total = n * k;
    for( std::int64_t i = blockIdx.x * static_cast<std::int64_t>( blockDim.x ) + threadIdx.x; i < total;
         i += static_cast<std::int64_t>( gridDim.x ) * blockDim.x )
    {
        const std::int64_t r = i / k;
        const int c = static_cast<int>( i - r * k );
        dst[r * ldd + c] = static_cast<D>( src[r * lds + c] );
    }
}

void launch_widen( const float * src, int lds, double * dst, int ldd, std::int64_t n, int k, cudaStream_t st )
{
    if( n * k > 0 ) { convert_rows_kernel<float, double><<<grid_for( std::min<std::int64_t>( n * k, std::int64_t( 1 ) << 24 ), 256 ), 256, 0, st>>>( src, lds, dst, ldd, n, k ); }
}

void launch_narrow( const double * src, int lds, float * dst, int ldd, std::int64_t n, int k, cudaStream_t st )
{
    if( n * k > 0 ) { convert_rows_kernel<double, float><<<grid_for( std::min<std::int64_t>( n * k, std::int64_t( 1 ) << 24 ), 256 ), 256, 0, st>>>( src, lds, dst, ldd, n, k ); }
}

void launch_init_status( int * status, cudaStream_t st )
{
    init_status_kernel<<<1, 1, 0, st>>>( status );
}

} // namespace tb
