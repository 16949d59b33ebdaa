// Schur-complement tiles of the FP32 path on the 5th-generation tensor cores
// (sm_100a): C -= A^T B as split-precision 3xTF32 products.
//
// Operands come from the operand image (plan.hpp, TcTask): every panel row,
// once its trsm is done, is stored split into TF32 hi and lo parts, transposed
// into K-major blocks of 64 U columns x 32 k.  One 3D tensor map covers the
// whole image (x: 32 k, y: 64 columns, z: block), with a box of 2 blocks and
// the 128-byte swizzle, so one TMA copy (cp.async.bulk.tensor) brings a
// 128-row x 32-k operand tile into shared memory already in the canonical
// K-major SWIZZLE_128B layout of tcgen05 operands.  The product of one 32-k
// chunk is 4 k-steps x 3 tcgen05.mma (a_lo b_hi, a_hi b_lo, a_hi b_hi: the
// small terms first; the lo x lo term is dropped, Ootomo & Yokota 2022) of
// M = 128, N = nt (<= 256), K = 8, accumulated in FP32 in tensor memory.
//
// Persistent, warp-specialised CTAs (one per SM: 192 KB of shared memory):
//   warp 0    TMA producer: fills a 2-stage ring (A hi/lo, B hi/lo per stage)
//   warp 1    MMA issuer (one thread) and tensor-memory owner
//   warps 2-5 epilogue: tensor memory -> registers, C -= acc by reductions in L2
// Two 256-column accumulators (all 512 tensor-memory columns) alternate
// between tiles, so the epilogue of one tile overlaps the MMAs of the next.
// Every mbarrier wait is bounded (polls and time); a wait that runs out sets
// bit 2 of status[0], stops every role of the CTA, waits (bounded) for the
// copies and products in flight, frees the tensor memory and returns, and the
// factorization then reports TB_ERR_TIMEOUT.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>

#include "kernels.cuh"

namespace tb
{
namespace
{

constexpr int kTcThreads = 192;                    // 6 warps
constexpr int kTcStages = 2;
constexpr int kTcPartA = kTcM * 128;               // one A part: 128 rows x 128 B = 16 KB
constexpr int kTcPartB = kTcNMax * 128;            // one B part: 256 rows x 128 B = 32 KB
constexpr int kTcStageBytes = 2 * kTcPartA + 2 * kTcPartB;   // A hi, A lo, B hi, B lo: 96 KB
constexpr int kTcBoxBytes = 2 * kImgRows * kImgK * 4;        // one tensor-map box (2 blocks): 16 KB
constexpr size_t kTcSmemBytes = static_cast<size_t>( kTcStages ) * kTcStageBytes + 1024;   // + alignment slack
constexpr int kTcAccCols = 256;                    // FP32 accumulator columns per buffer
constexpr unsigned kTcPollLimit = 1u << 26;        // polls of one wait
constexpr unsigned long long kTcWaitNs = 1000000000ull;
constexpr int kStatusTcTimeout = 2;                // status[0] bit (shared with the 64 x 64 tensor-core tiles)
static_assert( kTcSmemBytes <= 232448, "shared memory of the tensor-core tile kernel" );

__device__ __forceinline__ std::uint32_t smem_addr( const void * p )
{
    return static_cast<std::uint32_t>( __cvta_generic_to_shared( p ) );
}

__device__ __forceinline__ unsigned long long now_ns()
{
    unsigned long long t;
    asm volatile( "mov.u64 %0, %%globaltimer;\n" : "=l"(t) );
    return t;
}

__device__ __forceinline__ void bar_init( std::uint32_t bar, unsigned count )
{
    asm volatile( "mbarrier.init.shared::cta.b64 [%0], %1;\n" :: "r"(bar), "r"(count) : "memory" );
}

__device__ __forceinline__ void bar_arrive( std::uint32_t bar )
{
    asm volatile( "mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];\n" :: "r"(bar) : "memory" );
}

__device__ __forceinline__ void bar_expect_tx( std::uint32_t bar, unsigned bytes )
{
    asm volatile( "mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;\n" :: "r"(bar), "r"(bytes) : "memory" );
}

__device__ __forceinline__ bool bar_try( std::uint32_t bar, std::uint32_t parity )
{
    std::uint32_t done;
    asm volatile( "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
                  : "=r"(done) : "r"(bar), "r"(parity) : "memory" );
    return done != 0;
}

// Waits for the completion of the barrier phase with the given parity; false
// when the CTA is aborting or the wait ran out (which starts the abort).
__device__ __forceinline__ bool bar_wait( std::uint32_t bar, std::uint32_t parity, volatile int * abort, int * status )
{
    const unsigned long long start = now_ns();
    for( unsigned i = 0; i < kTcPollLimit; ++i )
    {
        if( bar_try( bar, parity ) ) { return true; }
        if( (i & 255u) == 255u )
        {
            if( *abort ) { return false; }
            if( now_ns() - start > kTcWaitNs ) { break; }
        }
    }
    *abort = 1;
    atomicOr( status, kStatusTcTimeout );
    return false;
}

// A bounded wait used while shutting down (no abort check).
__device__ __forceinline__ void bar_drain( std::uint32_t bar, std::uint32_t parity )
{
    const unsigned long long start = now_ns();
    for( unsigned i = 0; i < kTcPollLimit; ++i )
    {
        if( bar_try( bar, parity ) ) { return; }
        if( (i & 255u) == 255u && now_ns() - start > kTcWaitNs ) { return; }
    }
}

// Shared-memory descriptor of a K-major SWIZZLE_128B operand: start address,
// stride byte offset 1024 (next group of 8 rows), version 1, layout type 2.
// Within a 128-byte row the k-step is selected by advancing the start address
// (32 B per 8 TF32), the swizzle being applied on the address bits.
__device__ __forceinline__ std::uint64_t sw128_desc( std::uint32_t addr )
{
    return static_cast<std::uint64_t>( (addr >> 4) & 0x3FFFu ) | (static_cast<std::uint64_t>( 1 ) << 16)
         | (static_cast<std::uint64_t>( 1024 >> 4 ) << 32) | (1ull << 46) | (2ull << 61);
}

// kind::tf32 instruction descriptor: FP32 accumulator, TF32 A and B, both
// K-major, M = 128, N = n.
__device__ __forceinline__ std::uint32_t tf32_idesc( int n )
{
    return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<std::uint32_t>( n >> 3 ) << 17)
         | (static_cast<std::uint32_t>( kTcM >> 4 ) << 24);
}

__device__ __forceinline__ void tma_load_box( std::uint32_t dst, const CUtensorMap * map, int z, std::uint32_t bar )
{
    asm volatile( "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n"
                  :: "r"(dst), "l"(reinterpret_cast<std::uint64_t>( map )), "r"(0), "r"(0), "r"(z), "r"(bar) : "memory" );
}

__device__ __forceinline__ void mma_tf32( std::uint32_t tmem, std::uint64_t ad, std::uint64_t bd, std::uint32_t idesc,
                                          std::uint32_t accumulate )
{
    asm volatile( "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                  "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
                  :: "r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(accumulate) : "memory" );
}

__device__ __forceinline__ void mma_commit( std::uint32_t bar )
{
    asm volatile( "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" :: "r"(bar) : "memory" );
}

__device__ __forceinline__ void tmem_ld32( std::uint32_t addr, std::uint32_t (&v)[32] )
{
    asm volatile( "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                  "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
                  : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                    "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
                    "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                    "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                  : "r"(addr) );
    asm volatile( "tcgen05.wait::ld.sync.aligned;\n" ::: "memory" );
}

// Fire-and-forget additions into global memory (the read-modify-write runs in
// the L2 cache; the thread does not wait for it).
__device__ __forceinline__ void red_add_v4( float * p, float a, float b, float c, float d )
{
    asm volatile( "red.global.add.v4.f32 [%0], {%1, %2, %3, %4};\n" :: "l"(p), "f"(a), "f"(b), "f"(c), "f"(d) : "memory" );
}

__device__ __forceinline__ void red_add( float * p, float a )
{
    asm volatile( "red.global.add.f32 [%0], %1;\n" :: "l"(p), "f"(a) : "memory" );
}

__device__ __forceinline__ int tc_chunks( const TcTask & t ) { return (t.K + kImgK - 1) / kImgK; }
__device__ __forceinline__ int tc_b_boxes( const TcTask & t ) { return (t.nt + 2 * kImgRows - 1) / (2 * kImgRows); }

__global__ __launch_bounds__(kTcThreads, 1) void gemm_tc_tile_kernel( const TcTask * __restrict__ tasks, int count,
                                                                     float * __restrict__ arena,
                                                                     const __grid_constant__ CUtensorMap img_map,
                                                                     int * status )
{
    extern __shared__ unsigned char tc_smem_raw[];
    __shared__ __align__(8) std::uint64_t full_bar[kTcStages], empty_bar[kTcStages];
    __shared__ __align__(8) std::uint64_t acc_full[2], acc_empty[2];
    __shared__ std::uint32_t s_tmem;
    __shared__ int s_abort;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // programmatic dependent launch: let the next kernel launch once every CTA
    // runs, and wait for the previous one (which wrote the operands and C)
    asm volatile( "griddepcontrol.launch_dependents;\n" ::: "memory" );
    asm volatile( "griddepcontrol.wait;\n" ::: "memory" );
    // the 128-byte swizzle repeats every 1024 bytes: operand parts start on 1024-byte boundaries
    const std::uint32_t base = (smem_addr( tc_smem_raw ) + 1023u) & ~1023u;
    volatile int * abort = &s_abort;

    if( threadIdx.x == 0 )
    {
        for( int s = 0; s < kTcStages; ++s ) { bar_init( smem_addr( &full_bar[s] ), 1 ); bar_init( smem_addr( &empty_bar[s] ), 1 ); }
        for( int b = 0; b < 2; ++b ) { bar_init( smem_addr( &acc_full[b] ), 1 ); bar_init( smem_addr( &acc_empty[b] ), 4 ); }
        s_abort = 0;
        asm volatile( "fence.mbarrier_init.release.cluster;\n" ::: "memory" );
    }
    if( warp == 1 )
    {
        asm volatile( "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" :: "r"(smem_addr( &s_tmem )), "r"(2 * kTcAccCols) );
        asm volatile( "tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" );
    }
    asm volatile( "tcgen05.fence::before_thread_sync;\n" ::: "memory" );
    __syncthreads();
    asm volatile( "tcgen05.fence::after_thread_sync;\n" ::: "memory" );
    const std::uint32_t tmem = s_tmem;

    if( warp == 0 )
    {
        // ---------------------------------------------------------- producer
        if( lane == 0 )
        {
            unsigned g = 0;   // chunks issued
            for( int i = blockIdx.x; i < count && !*abort; i += gridDim.x )
            {
                const TcTask t = tasks[i];
                const int nk = tc_chunks( t ), nbb = tc_b_boxes( t );
                const unsigned bytes = static_cast<unsigned>( 2 * kTcBoxBytes + 2 * nbb * kTcBoxBytes );
                for( int c = 0; c < nk; ++c, ++g )
                {
                    const int s = static_cast<int>( g % kTcStages );
                    const unsigned round = g / kTcStages;
                    if( round > 0 && !bar_wait( smem_addr( &empty_bar[s] ), (round - 1) & 1u, abort, status ) ) { break; }
                    const std::uint32_t fb = smem_addr( &full_bar[s] );
                    bar_expect_tx( fb, bytes );
                    const std::uint32_t st = base + static_cast<std::uint32_t>( s ) * kTcStageBytes;
                    const std::int64_t zc = t.blk + static_cast<std::int64_t>( c ) * 2 * t.tf;
                    tma_load_box( st, &img_map, static_cast<int>( zc + t.ta ), fb );                         // A hi
                    tma_load_box( st + kTcPartA, &img_map, static_cast<int>( zc + t.tf + t.ta ), fb );       // A lo
                    for( int j = 0; j < nbb; ++j )
                    {
                        tma_load_box( st + 2 * kTcPartA + j * kTcBoxBytes, &img_map,
                                      static_cast<int>( zc + t.tb + 2 * j ), fb );                            // B hi
                        tma_load_box( st + 2 * kTcPartA + kTcPartB + j * kTcBoxBytes, &img_map,
                                      static_cast<int>( zc + t.tf + t.tb + 2 * j ), fb );                     // B lo
                    }
                }
            }
            // shutting down: every copy issued has landed before the shared memory is released
            for( unsigned h = (g > kTcStages ? g - kTcStages : 0); h < g; ++h )
            {
                bar_drain( smem_addr( &full_bar[h % kTcStages] ), (h / kTcStages) & 1u );
            }
        }
    }
    else if( warp == 1 )
    {
        // ------------------------------------------------------- MMA issuer
        if( lane == 0 )
        {
            unsigned g = 0, tile = 0;
            bool ok = true;
            for( int i = blockIdx.x; i < count && ok; i += gridDim.x, ++tile )
            {
                const TcTask t = tasks[i];
                const int nk = tc_chunks( t );
                const int b = static_cast<int>( tile & 1u );
                const unsigned use = tile >> 1;
                // the epilogue has read this accumulator's previous tile
                if( use > 0 && !bar_wait( smem_addr( &acc_empty[b] ), (use - 1) & 1u, abort, status ) ) { ok = false; break; }
                asm volatile( "tcgen05.fence::after_thread_sync;\n" ::: "memory" );
                const std::uint32_t acc = tmem + static_cast<std::uint32_t>( b * kTcAccCols );
                const std::uint32_t idesc = tf32_idesc( t.nt );
                for( int c = 0; c < nk; ++c, ++g )
                {
                    const int s = static_cast<int>( g % kTcStages );
                    if( !bar_wait( smem_addr( &full_bar[s] ), (g / kTcStages) & 1u, abort, status ) ) { ok = false; break; }
                    asm volatile( "tcgen05.fence::after_thread_sync;\n" ::: "memory" );
                    const std::uint32_t st = base + static_cast<std::uint32_t>( s ) * kTcStageBytes;
#pragma unroll
                    for( int ks = 0; ks < kImgK / 8; ++ks )
                    {
                        const std::uint32_t o = static_cast<std::uint32_t>( ks * 32 );
                        const std::uint64_t ahi = sw128_desc( st + o ), alo = sw128_desc( st + kTcPartA + o );
                        const std::uint64_t bhi = sw128_desc( st + 2 * kTcPartA + o );
                        const std::uint64_t blo = sw128_desc( st + 2 * kTcPartA + kTcPartB + o );
                        const std::uint32_t first = (c == 0 && ks == 0) ? 0u : 1u;
                        mma_tf32( acc, alo, bhi, idesc, first );
                        mma_tf32( acc, ahi, blo, idesc, 1u );
                        mma_tf32( acc, ahi, bhi, idesc, 1u );
                    }
                    mma_commit( smem_addr( &empty_bar[s] ) );     // the stage is free once these products are done
                }
                if( !ok ) { break; }
                mma_commit( smem_addr( &acc_full[b] ) );          // the accumulator is final
            }
            // shutting down: the products in flight have finished with the stages
            if( g > 0 )
            {
                const unsigned last = g - 1;
                bar_drain( smem_addr( &empty_bar[last % kTcStages] ), (last / kTcStages) & 1u );
            }
        }
    }
    else
    {
        // --------------------------------------------------------- epilogue
        const int q = warp & 3;                  // tensor-memory lanes 32q .. 32q+31 = tile rows
        unsigned tile = 0;
        for( int i = blockIdx.x; i < count; i += gridDim.x, ++tile )
        {
            const TcTask t = tasks[i];
            const int b = static_cast<int>( tile & 1u );
            if( !bar_wait( smem_addr( &acc_full[b] ), (tile >> 1) & 1u, abort, status ) ) { break; }
            asm volatile( "tcgen05.fence::after_thread_sync;\n" ::: "memory" );
            const int row = t.m0 + 32 * q + lane;
            float * crow = arena + t.c + static_cast<std::int64_t>( row ) * t.ldc;
            const std::uint32_t acc = tmem + (static_cast<std::uint32_t>( 32 * q ) << 16) + static_cast<std::uint32_t>( b * kTcAccCols );
            for( int j = 0; j < t.nt; j += 32 )
            {
                std::uint32_t v[32];
                tmem_ld32( acc + static_cast<std::uint32_t>( j ), v );
                if( row >= t.M ) { continue; }
                const int col0 = t.c0 + j;
                // C -= acc as reductions in the memory system (no load round trip): every C entry
                // gets exactly one contribution per launch, so the result is the plain C - acc
#pragma unroll
                for( int u = 0; u < 8; ++u )
                {
                    const int col = col0 + 4 * u;
                    if( col >= t.N ) { break; }
                    float * p = crow + col;
                    if( col + 3 < t.N && (!t.upper || row <= col) )
                    {
                        red_add_v4( p, -__uint_as_float( v[4 * u] ), -__uint_as_float( v[4 * u + 1] ),
                                    -__uint_as_float( v[4 * u + 2] ), -__uint_as_float( v[4 * u + 3] ) );
                    }
                    else
                    {
#pragma unroll
                        for( int e = 0; e < 4; ++e )
                        {
                            if( col + e < t.N && (!t.upper || row <= col + e) ) { red_add( p + e, -__uint_as_float( v[4 * u + e] ) ); }
                        }
                    }
                }
            }
            // this warp has read its rows of the accumulator
            asm volatile( "tcgen05.fence::before_thread_sync;\n" ::: "memory" );
            __syncwarp();
            if( lane == 0 ) { bar_arrive( smem_addr( &acc_empty[b] ) ); }
        }
    }

    asm volatile( "tcgen05.fence::before_thread_sync;\n" ::: "memory" );
    __syncthreads();
    if( warp == 1 )
    {
        asm volatile( "tcgen05.fence::after_thread_sync;\n" ::: "memory" );
        asm volatile( "tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" :: "r"(tmem), "r"(2 * kTcAccCols) );
    }
}

} // namespace

void launch_gemm_tc_tiles( const TcTask * tasks, int count, float * arena, const ImageMap & map, int * status,
                           cudaStream_t st )
{
    if( count <= 0 ) { return; }
    int dev = 0, sms = 0;
    cudaGetDevice( &dev );
    cudaDeviceGetAttribute( &sms, cudaDevAttrMultiProcessorCount, dev );
    const int grid = std::min( count, std::max( sms, 1 ) );
    const CUtensorMap * m = reinterpret_cast<const CUtensorMap *>( map.bytes );
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3( static_cast<unsigned>( grid ) );
    cfg.blockDim = dim3( kTcThreads );
    cfg.dynamicSmemBytes = kTcSmemBytes;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx( &cfg, gemm_tc_tile_kernel, tasks, count, arena, *m, status );
}

cudaError_t configure_tc_tiles()
{
    return cudaFuncSetAttribute( reinterpret_cast<const void *>( gemm_tc_tile_kernel ),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>( kTcSmemBytes ) );
}

// The operand image's tensor map: 3D (32 k, 64 columns, blocks) FP32 with a
// box of 2 blocks and the 128-byte swizzle (its inner extent, 32 x 4 bytes, is
// the swizzle span).  cuTensorMapEncodeTiled comes from the driver through the
// runtime's entry-point query, so the library needs no link to libcuda.
int encode_image_map( ImageMap * out, const float * img, std::int64_t blocks )
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if( encode == nullptr )
    {
        void * fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if( cudaGetDriverEntryPoint( "cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q ) != cudaSuccess
            || q != cudaDriverEntryPointSuccess || fn == nullptr )
        {
            return -1;
        }
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>( fn );
    }
    static_assert( sizeof( CUtensorMap ) == sizeof( out->bytes ), "tensor map size" );
    if( blocks <= 0 || blocks > 0x7FFFFFFF || (reinterpret_cast<std::uintptr_t>( img ) & 15u) != 0 ) { return -2; }
    const cuuint64_t dims[3] = { static_cast<cuuint64_t>( kImgK ), static_cast<cuuint64_t>( kImgRows ),
                                 static_cast<cuuint64_t>( blocks ) };
    const cuuint64_t strides[2] = { static_cast<cuuint64_t>( kImgK ) * 4, static_cast<cuuint64_t>( kImgK ) * kImgRows * 4 };
    const cuuint32_t box[3] = { static_cast<cuuint32_t>( kImgK ), static_cast<cuuint32_t>( kImgRows ), 2u };
    const cuuint32_t elem[3] = { 1u, 1u, 1u };
    CUtensorMap * m = reinterpret_cast<CUtensorMap *>( out->bytes );
    const CUresult r = encode( m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>( img ), dims, strides, box, elem,
                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE );
    return r == CUDA_SUCCESS ? 0 : static_cast<int>( r );
}

} // namespace tb
