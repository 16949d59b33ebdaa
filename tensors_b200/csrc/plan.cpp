// Device execution plan; see plan.hpp.

#include "plan.hpp"
#include "parallel.hpp"

#include <stdexcept>
#include "common.hpp"

#include <algorithm>
#include <map>
#include <set>
#include <utility>

namespace tb
{
namespace
{
using I32 = std::int32_t;
using I64 = std::int64_t;

constexpr I64 kExtendEntries = 8192;   // target entries of W per extend-add task
constexpr I64 kExportEntries = 16384;  // target entries per export task
constexpr I64 kZeroChunk = 1 << 16;     // doubles per zeroing task

void push_tiles( std::vector<GemmTask> & out, I64 a, I32 lda, I64 b, I32 ldb, I64 c, I32 ldc,
                 I32 K, I32 M, I32 N, bool symmetric )
{
    for( I32 m0 = 0; m0 < M; m0 += kTile )
    {
        for( I32 c0 = symmetric ? m0 : 0; c0 < N; c0 += kTile )
        {
            GemmTask t{};
            t.a = a; t.b = b; t.c = c;
            t.lda = lda; t.ldb = ldb; t.ldc = ldc;
            t.K = K; t.M = M; t.N = N;
            t.m0 = m0; t.c0 = c0;
            t.upper = (symmetric && m0 == c0) ? 1 : 0;
            out.push_back( t );
        }
    }
}

// The tensor-core tiles of the fronts with an operand image (see TcTask):
// kTcM x nt tiles (nt up to nmax <= kTcNMax) over C's M x N entries (symmetric: the
// tiles on and right of the diagonal).  next_rows: the call updates the next
// panel's rows, which the tiles of the first tile row contain.
void push_tc( std::vector<TcTask> & out, std::vector<char> & next, bool next_rows, I64 blk, I32 tf,
              I32 ta0, I32 tb0, I32 K, I64 c, I32 ldc, I32 M, I32 N, bool symmetric, I32 nmax )
{
    for( I32 m0 = 0; m0 < M; m0 += kTcM )
    {
        for( I32 c0 = symmetric ? m0 : 0; c0 < N; c0 += nmax )
        {
            TcTask t{};
            t.c = c; t.blk = blk;
            t.ldc = ldc; t.M = M; t.N = N;
            t.m0 = m0; t.c0 = c0; t.K = K;
            t.ta = ta0 + m0 / kImgRows; t.tb = tb0 + c0 / kImgRows; t.tf = tf;
            t.nt = static_cast<I32>( std::min<I64>( nmax, ceil_div( N - c0, kImgRows ) * kImgRows ) );
            t.upper = symmetric ? 1 : 0;
            out.push_back( t );
            next.push_back( next_rows && m0 == 0 ? 1 : 0 );
        }
    }
}

// Best-fit allocator over [0, capacity) with a coalescing free list; grows
// the capacity when nothing fits.  Free blocks are indexed both by address
// (for coalescing) and by (size, address) (for the O(log n) best-fit lookup),
// so a merged plan over thousands of small fronts stays linear-logarithmic.
class RegionAllocator
{
public:
    I64 allocate( I64 size )
    {
        if( size <= 0 ) { return 0; }
        auto fit = by_size_.lower_bound( { size, I64(-1) } );
        if( fit != by_size_.end() )
        {
            const I64 off = fit->second;
            const I64 rest = fit->first - size;
            erase_block( off );
            if( rest > 0 ) { insert_block( off + size, rest ); }
            return off;
        }
        // extend: reuse a free block that ends at the top
        if( !free_.empty() )
        {
            auto last = std::prev( free_.end() );
            if( last->first + last->second == top_ )
            {
                const I64 off = last->first;
                erase_block( off );
                top_ = off + size;
                return off;
            }
        }
        const I64 off = top_;
        top_ += size;
        return off;
    }
    void release( I64 off, I64 size )
    {
        if( size <= 0 ) { return; }
        auto next = free_.lower_bound( off );
        if( next != free_.begin() )
        {
            auto prev = std::prev( next );
            if( prev->first + prev->second == off )
            {
                off = prev->first;
                size += prev->second;
                erase_block( off );
            }
        }
        next = free_.lower_bound( off + size );
        if( next != free_.end() && next->first == off + size )
        {
            size += next->second;
            erase_block( next->first );
        }
        insert_block( off, size );
    }
    I64 capacity() const { return top_; }

private:
    void insert_block( I64 off, I64 size )
    {
        free_.emplace( off, size );
        by_size_.emplace( size, off );
    }
    void erase_block( I64 off )
    {
        auto it = free_.find( off );
        by_size_.erase( { it->second, off } );
        free_.erase( it );
    }

    std::map<I64,I64> free_;              // address -> size
    std::set<std::pair<I64,I64>> by_size_; // (size, address)
    I64 top_ = 0;
};

} // namespace

void Plan::build( const Symbolic & sym )
{
    const I32 S = sym.sn_count;
    const I32 n = sym.n;

    factor_flops = 0.0;
    nnz_u = 0.0;
    for( I32 s = 0; s < S; ++s )
    {
        const double a = sym.n0(s), b = sym.n1(s);
        factor_flops += a * a * a / 3.0 + a * a * b + a * b * b;
        nnz_u += a * (a + 1.0) / 2.0 + a * b;
    }

    // ---------------------------------------------------------------- fronts
    // Walk supernodes in order; supernode s joins the front of s+1 when it is
    // the last child of s+1 (aTree parent == s+1, so rows are contiguous) and
    // the relaxation limits allow it.
    std::vector<I32> merged_into( static_cast<size_t>(S), -1 );
    {
        std::vector<I64> rows( static_cast<size_t>(S) );
        std::vector<double> zeros( static_cast<size_t>(S), 0.0 );
        for( I32 s = 0; s < S; ++s ) { rows[s] = sym.n0(s); }
        for( I32 s = 0; s + 1 < S; ++s )
        {
            const I32 p = sym.atree_parent[s];
            if( p != s + 1 ) { continue; }
            const double a0 = static_cast<double>(rows[s]), a1 = sym.n1(s);
            const double b0 = sym.n0(p), b1 = sym.n1(p);
            const double m0 = a0 + b0;
            const double z = zeros[s] + zeros[p] + a0 * (b0 + b1 - a1);
            const double total = m0 * (m0 + 1.0) / 2.0 + m0 * b1;
            bool take;
            if( m0 <= relax.nrelax[0] )      { take = true; }
            else if( m0 <= relax.nrelax[1] ) { take = z < relax.zrelax[0] * total; }
            else if( m0 <= relax.nrelax[2] ) { take = z < relax.zrelax[1] * total; }
            else                             { take = z < relax.zrelax[2] * total; }
            if( take )
            {
                merged_into[s] = p;
                rows[p] = static_cast<I64>(m0);
                zeros[p] = z;
            }
        }
    }
    front_of_sn.assign( static_cast<size_t>(S), -1 );
    front_sn_first.clear(); front_sn_last.clear();
    {
        I32 first = 0;
        for( I32 s = 0; s < S; ++s )
        {
            if( merged_into[s] >= 0 ) { continue; }
            front_sn_first.push_back( first );
            front_sn_last.push_back( s );
            first = s + 1;
        }
    }
    front_count = static_cast<I32>( front_sn_last.size() );
    const I32 F = front_count;
    front_row0.resize( static_cast<size_t>(F) );
    front_n0.resize( static_cast<size_t>(F) );
    front_n1.resize( static_cast<size_t>(F) );
    front_cols.resize( static_cast<size_t>(F) );
    front_parent.resize( static_cast<size_t>(F) );
    for( I32 f = 0; f < F; ++f )
    {
        for( I32 s = front_sn_first[f]; s <= front_sn_last[f]; ++s ) { front_of_sn[s] = f; }
        front_row0[f] = sym.sn_rp[front_sn_first[f]];
        front_n0[f] = sym.sn_rp[front_sn_last[f] + 1] - front_row0[f];
        front_n1[f] = sym.n1( front_sn_last[f] );
        front_cols[f] = sym.sn_outer[front_sn_last[f]];
    }
    front_flops = 0.0;
    front_entries = 0.0;
    for( I32 f = 0; f < F; ++f )
    {
        const I32 p = sym.atree_parent[front_sn_last[f]];
        front_parent[f] = (p < S) ? front_of_sn[p] : F;
        const double a = front_n0[f], b = front_n1[f];
        front_flops += a * a * a / 3.0 + a * a * b + a * b * b;
        front_entries += a * (a + 1.0) / 2.0 + a * b;
    }
    std::vector<I32> child_ptr( static_cast<size_t>(F) + 2, 0 ), child_idx( static_cast<size_t>(F) );
    for( I32 f = 0; f < F; ++f ) { ++child_ptr[front_parent[f] + 1]; }
    for( I32 f = 0; f <= F; ++f ) { child_ptr[f+1] += child_ptr[f]; }
    {
        std::vector<I32> next( child_ptr.begin(), child_ptr.end() - 1 );
        for( I32 f = 0; f < F; ++f ) { child_idx[next[front_parent[f]]++] = f; }
    }

    // levels by height
    level_of.assign( static_cast<size_t>(F), 0 );
    levels = F > 0 ? 1 : 0;
    for( I32 f = 0; f < F; ++f )
    {
        const I32 p = front_parent[f];
        if( p < F ) { level_of[p] = std::max( level_of[p], level_of[f] + 1 ); }
        levels = std::max( levels, level_of[f] + 1 );
    }
    std::vector<std::vector<I32>> by_level( static_cast<size_t>(levels) );
    for( I32 f = 0; f < F; ++f ) { by_level[level_of[f]].push_back( f ); }

    // ---------------------------------------------------------- arena layout
    front_u0.resize( static_cast<size_t>(F) );
    front_u1.resize( static_cast<size_t>(F) );
    front_ld0.resize( static_cast<size_t>(F) );
    front_ld1.resize( static_cast<size_t>(F) );
    front_v.assign( static_cast<size_t>(F), 0 );
    u0_size = u1_size = 0;
    for( I32 f = 0; f < F; ++f )
    {
        front_ld0[f] = static_cast<I32>( ceil_div( front_n0[f], kLdAlign ) * kLdAlign );
        front_ld1[f] = static_cast<I32>( ceil_div( front_n1[f], kLdAlign ) * kLdAlign );
    }
    for( I32 f = 0; f < F; ++f ) { front_u0[f] = u0_size; u0_size += static_cast<I64>(front_n0[f]) * front_ld0[f]; }
    for( I32 f = 0; f < F; ++f ) { front_u1[f] = u0_size + u1_size; u1_size += static_cast<I64>(front_n0[f]) * front_ld1[f]; }
    // update matrices: live from the front's level until its parent's level
    std::vector<std::vector<I32>> release_at( static_cast<size_t>(levels) + 1 );
    {
        RegionAllocator va;
        std::vector<I64> voff( static_cast<size_t>(F), 0 );
        for( I32 h = 0; h < levels; ++h )
        {
            for( I32 f : by_level[h] )
            {
                const I64 sz = static_cast<I64>(front_n1[f]) * front_ld1[f];
                voff[f] = va.allocate( sz );
                const I32 p = front_parent[f];
                release_at[p < F ? level_of[p] : h].push_back( f );
            }
            for( I32 f : release_at[h] ) { va.release( voff[f], static_cast<I64>(front_n1[f]) * front_ld1[f] ); }
        }
        v_size = va.capacity();
        for( I32 f = 0; f < F; ++f ) { front_v[f] = u0_size + u1_size + voff[f]; }
    }

    // ---------------------------------------------------- extend-add tables
    lut.assign( sym.sn_inner.size(), 0 );   // a front's columns are a slice of SN_inner
    front_lut.resize( static_cast<size_t>(F) );
    std::vector<I32> mid( static_cast<size_t>(F), 0 );
    {
        std::vector<I32> idx( static_cast<size_t>(n), 0 );
        for( I32 p = 0; p < F; ++p )
        {
            const I32 rb = front_row0[p], re = rb + front_n0[p];
            for( I32 r = rb; r < re; ++r ) { idx[r] = r - rb; }
            for( I32 j = 0; j < front_n1[p]; ++j ) { idx[sym.sn_inner[front_cols[p] + j]] = j; }
            for( I32 c = child_ptr[p]; c < child_ptr[p+1]; ++c )
            {
                const I32 t = child_idx[c];
                front_lut[t] = front_cols[t];
                I32 m = 0;
                for( I32 i = 0; i < front_n1[t]; ++i )
                {
                    const I32 col = sym.sn_inner[front_cols[t] + i];
                    lut[front_cols[t] + i] = idx[col];
                    if( col < re ) { ++m; }
                }
                mid[t] = m;
            }
        }
    }

    // ------------------------------------------------------- assembly map
    {
        // row i's upper entries occupy [first[i], first[i + 1]): rows fill in parallel
        std::vector<I64> first( static_cast<size_t>(n) + 1, 0 );
        for( I32 i = 0; i < n; ++i ) { first[static_cast<size_t>(i) + 1] = first[static_cast<size_t>(i)] + (sym.outer[i+1] - sym.diag[i]); }
        asm_src.assign( static_cast<size_t>( first[static_cast<size_t>(n)] ), 0 );
        asm_dst.assign( static_cast<size_t>( first[static_cast<size_t>(n)] ), 0 );
        parallel_rows( n, [&]( I64 b, I64 e )
        {
            for( I32 i = static_cast<I32>( b ); i < static_cast<I32>( e ); ++i )
            {
                const I32 f = front_of_sn[ sym.row_to_sn[i] ];
                const I32 rb = front_row0[f], re = rb + front_n0[f];
                const I32 * cols = sym.sn_inner.data() + front_cols[f];
                I32 l = 0;
                I64 out = first[static_cast<size_t>(i)];
                for( I64 k = sym.diag[i]; k < sym.outer[i+1]; ++k, ++out )
                {
                    const I32 j = sym.inner[k];
                    I64 dst;
                    if( j < re )
                    {
                        dst = front_u0[f] + static_cast<I64>(front_ld0[f]) * (i - rb) + (j - rb);
                    }
                    else
                    {
                        while( cols[l] < j ) { ++l; }
                        dst = front_u1[f] + static_cast<I64>(front_ld1[f]) * (i - rb) + l;
                    }
                    asm_src[static_cast<size_t>(out)] = sym.value_perm[k];
                    asm_dst[static_cast<size_t>(out)] = static_cast<I64>( static_cast<std::uint64_t>(dst) | (j == i ? kDiagFlag : 0ull) );
                }
            }
        }, threads );
    }

    // ------------------------------------------ export to reference layout
    colmap.assign( sym.sn_inner.size(), 0 );
    exports.clear();
    diag_offset.resize( static_cast<size_t>(n) );
    {
        std::vector<I32> pos( static_cast<size_t>(n), -1 );
        for( I32 f = 0; f < F; ++f )
        {
            const I32 rb = front_row0[f], re = rb + front_n0[f];
            for( I32 j = 0; j < front_n1[f]; ++j ) { pos[sym.sn_inner[front_cols[f] + j]] = j; }
            for( I32 r = rb; r < re; ++r ) { diag_offset[r] = front_u0[f] + static_cast<I64>(front_ld0[f] + 1) * (r - rb); }
            for( I32 s = front_sn_first[f]; s <= front_sn_last[f]; ++s )
            {
                const I64 cb = sym.sn_outer[s];
                for( I32 l = 0; l < sym.n1(s); ++l )
                {
                    const I32 j = sym.sn_inner[cb + l];
                    colmap[cb + l] = (j < re) ? (j - rb) : -(pos[j] + 1);
                }
                const I32 n0s = sym.n0(s), n1s = sym.n1(s);
                const I64 per_row = std::max<I64>( 1, n0s + n1s );
                const I32 rows_per_task = static_cast<I32>( std::max<I64>( 1, kExportEntries / per_row ) );
                for( I32 r = 0; r < n0s; r += rows_per_task )
                {
                    ExportTask e{};
                    e.fu0 = front_u0[f]; e.fu1 = front_u1[f];
                    e.tri = sym.sn_tri_ptr[s]; e.rec = sym.sn_rec_ptr[s];
                    e.colmap = cb;
                    e.fn0 = front_n0[f]; e.fn1 = front_n1[f];
                    e.fld0 = front_ld0[f]; e.fld1 = front_ld1[f];
                    e.roff = sym.sn_rp[s] - rb;
                    e.n0s = n0s; e.n1s = n1s;
                    e.r_begin = r; e.r_end = std::min( n0s, r + rows_per_task );
                    exports.push_back( e );
                }
            }
        }
    }

    // ------------------------------------------------ operand image
    // Fronts whose widest update has at least 128 columns (and >= 16 pivot
    // rows) get an operand image and tensor-core tiles on the FP32 path; the
    // updates of the smaller ones stay 64 x 64 tiles (an image block holds 32
    // rows of k and 64 columns, mostly empty for them).
    front_img.assign( static_cast<size_t>(F), -1 );
    img_blocks = 0;
    std::vector<I32> img_t0( static_cast<size_t>(F), 0 ), img_tf( static_cast<size_t>(F), 0 );
    for( I32 f = 0; f < F; ++f )
    {
        const I32 n0 = front_n0[f], n1 = front_n1[f];
        if( n0 < 16 || std::max<I32>( n0 - kPanel, 0 ) + n1 < 2 * kImgRows ) { continue; }
        img_t0[f] = static_cast<I32>( ceil_div( n0, kImgRows ) );
        img_tf[f] = img_t0[f] + static_cast<I32>( ceil_div( n1, kImgRows ) );
        front_img[f] = img_blocks;
        img_blocks += ceil_div( n0, kImgK ) * 2 * img_tf[f];
    }

    // -------------------------------------------------- launch sequences
    gemm.clear(); tc.clear(); potrf.clear(); panel.clear(); extend.clear(); zero.clear(); sdiag.clear(); srest.clear();
    extend_pull.clear(); extend_segs.clear();
    gemm_flops = 0.0;
    gemm_tile_flops = 0.0;
    factor_launches.clear(); lower_launches.clear(); upper_launches.clear();
    dag.clear();

    struct Range { I64 first; I32 count; };
    std::vector<std::vector<Range>> rest_ranges( static_cast<size_t>(levels) );
    std::vector<std::vector<I32>> front_panels( static_cast<size_t>(F) );   // sdiag index of each panel, in step order

    // Dependency counters of the task graph (see DagTask): per level the
    // finished extend-add tasks, per front the extend-adds received and
    // the zeroing chunks done, per panel the potrf, trsm chunks, GEMM tiles
    // of the panel's row block that feed the next panel, and all GEMM tiles.
    // Panel indices follow the potrf / sdiag arrays, so they are only known
    // while the arrays are built; counters are laid out once the panel count
    // is known, so their ids are assigned in a second pass (CounterRef).
    enum CounterKind : I32 { kExtLevel = 0, kExtIn, kZeroDone, kPotrfDone, kTrsmDone, kNextDone, kGemmDone };
    struct CounterRef { I32 kind = -1, idx = 0; };
    struct PendingTask { I32 kind, index, level; CounterRef signal[2]; CounterRef wait[kDagWaits]; I32 target[kDagWaits]; };
    I32 cur_level = 0;
    std::vector<PendingTask> pending;
    auto make = [&]( LaunchKind k, I64 index ) {
        PendingTask t{};
        t.kind = static_cast<I32>( k ); t.index = static_cast<I32>( index ); t.level = cur_level;
        for( int i = 0; i < kDagWaits; ++i ) { t.target[i] = 0; }
        return t;
    };
    auto add_wait = [&]( PendingTask & t, I32 kind, I32 idx, I32 target ) {
        if( target <= 0 ) { return; }
        for( int i = 0; i < kDagWaits; ++i )
        {
            if( t.wait[i].kind < 0 ) { t.wait[i] = { kind, idx }; t.target[i] = target; return; }
        }
        throw std::logic_error( "task with too many dependencies" );
    };

    std::vector<I32> ext_into( static_cast<size_t>(F), 0 );        // extend tasks into each front (so far)
    std::vector<I32> zero_of( static_cast<size_t>(F), 0 );         // zeroing chunks of each front's V
    std::vector<I32> last_panel( static_cast<size_t>(F), -1 );     // panel index of the front's latest panel
    std::vector<I32> panel_tiles, panel_next, panel_trsm;          // per panel: GEMM tiles, next-row tiles, trsm chunks
    // Update-matrix regions are reused across levels: a level's zeroing
    // waits until every extend-add of the earlier levels has read its child's
    // region.  Each level's extend-adds wait for all those of the previous
    // level that has any, so the count of that one level covers all before.
    I32 prev_ext_level = -1, prev_ext_count = 0;

    std::vector<I32> panel_level, level_steps( static_cast<size_t>(levels), 0 );
    for( I32 h = 0; h < levels; ++h )
    {
        const auto & L = by_level[h];
        cur_level = h;
        const size_t extend_before = extend.size();   // this level's extend-adds signal its counter

        // zero this level's update matrices before children add into them;
        // the regions may have been used by fronts consumed at earlier levels
        {
            const I64 first = static_cast<I64>(zero.size());
            for( I32 f : L )
            {
                // the upper triangle only, in groups of rows of about kZeroChunk entries
                const I32 nv = front_n1[f];
                for( I32 r = 0; r < nv; )
                {
                    I32 e = r;
                    I64 cnt = 0;
                    while( e < nv && cnt < kZeroChunk ) { cnt += nv - e; ++e; }
                    PendingTask t = make( LaunchKind::Zero, static_cast<I64>(zero.size()) );
                    if( prev_ext_level >= 0 ) { add_wait( t, kExtLevel, prev_ext_level, prev_ext_count ); }
                    t.signal[0] = { kZeroDone, f };
                    pending.push_back( t );
                    ++zero_of[f];
                    ZeroTask z{};
                    z.offset = front_v[f]; z.count = cnt;
                    z.n = nv; z.ld = front_ld1[f]; z.row_begin = r; z.row_end = e;
                    zero.push_back( z );
                    r = e;
                }
            }
            const I32 count = static_cast<I32>( static_cast<I64>(zero.size()) - first );
            if( count > 0 ) { factor_launches.push_back( { LaunchKind::Zero, count, first, h, 0 } ); }
        }

        // extend-add passes by child rank (one child per parent and pass, so
        // no two tasks of a pass touch the same parent entries)
        I32 max_children = 0;
        for( I32 f : L ) { max_children = std::max( max_children, child_ptr[f+1] - child_ptr[f] ); }
        const I64 level_ext_first = static_cast<I64>( extend.size() );
        for( I32 r = 0; r < max_children; ++r )
        {
            const I64 first = static_cast<I64>(extend.size());
            for( I32 p : L )
            {
                const I32 cb = child_ptr[p], ce = child_ptr[p+1];
                if( cb + r >= ce ) { continue; }
                const I32 t = child_idx[cb + r];
                const I32 m1 = front_n1[t];
                if( m1 == 0 ) { continue; }
                const I32 before = ext_into[p];
                I32 row = 0;
                while( row < m1 )
                {
                    I32 end = row;
                    I64 entries = 0;
                    while( end < m1 && (entries == 0 || entries + (m1 - end) <= kExtendEntries) )
                    {
                        entries += m1 - end;
                        ++end;
                    }
                    ExtendTask e{};
                    e.w = front_v[t];
                    e.u0 = front_u0[p]; e.u1 = front_u1[p]; e.v = front_v[p];
                    e.lut = front_lut[t];
                    e.m1 = m1; e.mid = mid[t];
                    e.n0p = front_n0[p]; e.n1p = front_n1[p];
                    e.ldw = front_ld1[t];
                    e.ld0p = front_ld0[p]; e.ld1p = front_ld1[p]; e.ldvp = front_ld1[p];
                    e.row_begin = row; e.row_end = end;
                    PendingTask d = make( LaunchKind::Extend, static_cast<I64>(extend.size()) );
                    add_wait( d, kGemmDone, last_panel[t], panel_tiles[static_cast<size_t>( last_panel[t] )] );
                    add_wait( d, kZeroDone, p, zero_of[p] );
                    add_wait( d, kExtIn, p, before );
                    if( prev_ext_level >= 0 ) { add_wait( d, kExtLevel, prev_ext_level, prev_ext_count ); }
                    d.signal[0] = { kExtIn, p };
                    d.signal[1] = { kExtLevel, h };
                    pending.push_back( d );
                    ++ext_into[p];
                    extend.push_back( e );
                    row = end;
                }
            }
            (void)first;
        }
        // the level launch: the same additions by blocks of parent rows (ExtendPullTask), a block
        // growing while its children's entries stay within kExtendPullEntries
        {
            const I64 pull_first = static_cast<I64>( extend_pull.size() );
            std::vector<I64> row_work;
            for( I32 p : L )
            {
                const I32 cb = child_ptr[p], ce = child_ptr[p+1];
                for( int space = 0; space < 2 && cb < ce; ++space )
                {
                    const I32 prow = space == 0 ? front_n0[p] : front_n1[p];
                    row_work.assign( static_cast<size_t>( prow ), 0 );
                    for( I32 c = cb; c < ce; ++c )
                    {
                        const I32 t = child_idx[c];
                        const I32 m1 = front_n1[t];
                        const I32 lo = space == 0 ? 0 : mid[t], hi = space == 0 ? mid[t] : m1;
                        for( I32 i = lo; i < hi; ++i ) { row_work[static_cast<size_t>( lut[front_lut[t] + i] )] += m1 - i; }
                    }
                    for( I32 b0 = 0; b0 < prow; )
                    {
                        I32 b1 = b0;
                        I64 work = 0;
                        while( b1 < prow && (b1 == b0 || work + row_work[static_cast<size_t>( b1 )] <= kExtendPullEntries) )
                        {
                            work += row_work[static_cast<size_t>( b1 )];
                            ++b1;
                        }
                        if( work > 0 )
                        {
                            const I64 seg_first = static_cast<I64>( extend_segs.size() );
                            for( I32 c = cb; c < ce; ++c )
                            {
                                const I32 t = child_idx[c];
                                const I32 m1 = front_n1[t];
                                if( m1 == 0 ) { continue; }
                                // the child's rows in this space map to increasing parent rows
                                const I32 * lt = lut.data() + front_lut[t];
                                const I32 lo = space == 0 ? 0 : mid[t], hi = space == 0 ? mid[t] : m1;
                                const I32 ia = static_cast<I32>( std::lower_bound( lt + lo, lt + hi, b0 ) - lt );
                                const I32 ib = static_cast<I32>( std::lower_bound( lt + lo, lt + hi, b1 ) - lt );
                                if( ia >= ib ) { continue; }
                                ExtendTask e{};
                                e.w = front_v[t];
                                e.u0 = front_u0[p]; e.u1 = front_u1[p]; e.v = front_v[p];
                                e.lut = front_lut[t];
                                e.m1 = m1; e.mid = mid[t];
                                e.n0p = front_n0[p]; e.n1p = front_n1[p];
                                e.ldw = front_ld1[t];
                                e.ld0p = front_ld0[p]; e.ld1p = front_ld1[p]; e.ldvp = front_ld1[p];
                                e.row_begin = ia; e.row_end = ib;
                                extend_segs.push_back( e );
                            }
                            const I32 nseg = static_cast<I32>( static_cast<I64>( extend_segs.size() ) - seg_first );
                            extend_pull.push_back( { seg_first, nseg, space, b0, b1 } );
                        }
                        b0 = b1;
                    }
                }
            }
            const I32 npull = static_cast<I32>( static_cast<I64>( extend_pull.size() ) - pull_first );
            if( npull > 0 )
            {
                Launch Lp{ LaunchKind::ExtendPull, npull, pull_first, h, 0 };
                Lp.tc_first = level_ext_first;
                Lp.tc_count = static_cast<I32>( static_cast<I64>( extend.size() ) - level_ext_first );
                factor_launches.push_back( Lp );
            }
        }

        // panel steps; in the task graph a step's GEMM tiles that update the
        // next panel's rows come first, then the next panel's potrf (which also
        // inverts its diagonal block) and trsm, then the rest of the step's
        // tiles (one step of look-ahead)
        I32 Q = 0;
        for( I32 f : L ) { Q = std::max<I32>( Q, static_cast<I32>( ceil_div( front_n0[f], kPanel ) ) ); }
        rest_ranges[h].resize( static_cast<size_t>(Q) );
        level_steps[static_cast<size_t>(h)] = Q;
        std::vector<std::vector<PendingTask>> step_potrf( static_cast<size_t>(Q) ), step_trsm( static_cast<size_t>(Q) ),
            next_tiles( static_cast<size_t>(Q) ), rest_tiles( static_cast<size_t>(Q) );
        for( I32 q = 0; q < Q; ++q )
        {
            const I64 ofirst = static_cast<I64>(potrf.size());
            const I64 pfirst = static_cast<I64>(panel.size());
            const I64 gfirst = static_cast<I64>(gemm.size());
            const I64 rfirst = static_cast<I64>(srest.size());
            std::vector<GemmTask> tiles;
            std::vector<I32> tile_panel, tile_prev;
            std::vector<char> tile_next, tile_small;
            std::vector<TcTask> tct;
            std::vector<char> tct_next;
            for( I32 f : L )
            {
                const I32 n0 = front_n0[f], n1 = front_n1[f];
                const I32 r0 = q * kPanel;
                if( r0 >= n0 ) { continue; }
                const I32 nb = std::min( kPanel, n0 - r0 );
                const I32 r1 = r0 + nb;
                const I32 rest = (n0 - r1) + n1;
                const I32 pi = static_cast<I32>( potrf.size() );
                const I32 prev = last_panel[f];
                last_panel[f] = pi;
                panel_tiles.push_back( 0 ); panel_next.push_back( 0 ); panel_trsm.push_back( 0 ); panel_level.push_back( h );
                std::int64_t singles = 0;
                for( I32 r = 0; r < nb; ++r )
                {
                    const I32 s = sym.row_to_sn[front_row0[f] + r0 + r];
                    if( sym.n0(s) == 1 ) { singles |= (std::int64_t(1) << r); }
                }
                const I32 ld0 = front_ld0[f], ld1 = front_ld1[f];
                PanelTask t{};
                t.u0 = front_u0[f]; t.u1 = front_u1[f];
                t.n0 = n0; t.n1 = n1; t.r0 = r0; t.c0 = 0;
                t.ld0 = ld0; t.ld1 = ld1;
                t.row0 = front_row0[f];
                t.single_rows = singles;
                t.panel = pi;                   // == sdiag.size(): one potrf task and one SolveDiagTask per panel
                t.img = front_img[f]; t.img_t0 = img_t0[f]; t.img_tf = img_tf[f];
                {
                    PendingTask d = make( LaunchKind::Potrf, static_cast<I64>(potrf.size()) );
                    // the first panel starts once the children's contributions are in and
                    // the front's own update matrix is cleared (its last step writes it)
                    if( q == 0 ) { add_wait( d, kExtIn, f, ext_into[f] ); add_wait( d, kZeroDone, f, zero_of[f] ); }
                    else { add_wait( d, kNextDone, prev, panel_next[static_cast<size_t>(prev)] ); }
                    d.signal[0] = { kPotrfDone, pi };
                    step_potrf[q].push_back( d );
                }
                potrf.push_back( t );
                for( I32 c0 = 0; c0 < rest; c0 += kRestChunk )
                {
                    t.c0 = c0;
                    PendingTask d = make( LaunchKind::Trsm, static_cast<I64>(panel.size()) );
                    add_wait( d, kPotrfDone, pi, 1 );
                    d.signal[0] = { kTrsmDone, pi };
                    step_trsm[q].push_back( d );
                    ++panel_trsm[static_cast<size_t>(pi)];
                    panel.push_back( t );
                }
                const I32 m = n0 - r1;
                const size_t tfirst = tiles.size();
                if( m > 0 )
                {
                    // Trailing updates are deferred over defer_steps panel steps: the
                    // next panel's rows [r1, r1 + 64) get every pending panel at once,
                    // and the whole trailing matrix is updated at every defer_steps-th
                    // step, with the rows of the panels since the last such update
                    // (contiguous in U0 / U1, K up to 64 defer_steps).  Each C entry is
                    // read and written defer_steps times less often and the tiles are
                    // that much deeper; the next panel still sees every update before
                    // its potrf, and every contribution is applied exactly once.
                    const I32 j = q % defer_steps;
                    const I32 k0 = r0 - j * kPanel;
                    const I32 K = r1 - k0;
                    const I32 rows = (j + 1 < defer_steps) ? std::min( kPanel, m ) : m;
                    const I64 pa = front_u0[f] + static_cast<I64>(k0) * ld0 + r1;        // U0[k0:r1, r1:n0]
                    push_tiles( tiles, pa, ld0, pa, ld0, front_u0[f] + static_cast<I64>(r1) * ld0 + r1, ld0, K, rows, m, true );
                    if( n1 > 0 )
                    {
                        push_tiles( tiles, pa, ld0, front_u1[f] + static_cast<I64>(k0) * ld1, ld1,
                                    front_u1[f] + static_cast<I64>(r1) * ld1, ld1, K, rows, n1, false );
                    }
                    // tiles of rows [r1, r1 + 64) feed the next panel
                    for( size_t i = tfirst; i < tiles.size(); ++i ) { tile_next.push_back( tiles[i].m0 == 0 ? 1 : 0 ); }
                    if( front_img[f] >= 0 )
                    {
                        // r1 and k0 are multiples of 64: whole image column tiles and k-chunks
                        const I64 blk = front_img[f] + static_cast<I64>( k0 / kImgK ) * 2 * img_tf[f];
                        const I32 ta = r1 / kImgRows;
                        push_tc( tct, tct_next, true, blk, img_tf[f], ta, ta, K,
                                 front_u0[f] + static_cast<I64>(r1) * ld0 + r1, ld0, rows, m, true, tc_nmax );
                        if( n1 > 0 )
                        {
                            push_tc( tct, tct_next, true, blk, img_tf[f], ta, img_t0[f], K,
                                     front_u1[f] + static_cast<I64>(r1) * ld1, ld1, rows, n1, false, tc_nmax );
                        }
                    }
                }
                else if( n1 > 0 && front_parent[f] < F )
                {
                    push_tiles( tiles, front_u1[f], ld1, front_u1[f], ld1, front_v[f], ld1, n0, n1, n1, true );
                    for( size_t i = tfirst; i < tiles.size(); ++i ) { tile_next.push_back( 0 ); }
                    if( front_img[f] >= 0 )
                    {
                        push_tc( tct, tct_next, false, front_img[f], img_tf[f], img_t0[f], img_t0[f], n0,
                                 front_v[f], ld1, n1, n1, true, tc_nmax );
                    }
                }
                for( size_t i = tfirst; i < tiles.size(); ++i ) { tile_small.push_back( front_img[f] < 0 ? 1 : 0 ); }
                for( size_t i = tfirst; i < tiles.size(); ++i ) { tile_panel.push_back( pi ); tile_prev.push_back( prev ); }
                {
                    SolveRestTask t{};
                    t.u0 = front_u0[f]; t.u1 = front_u1[f]; t.inner = front_cols[f];
                    t.n0 = n0; t.n1 = n1; t.r0 = r0; t.row0 = front_row0[f];
                    t.ld0 = ld0; t.ld1 = ld1;
                    t.panel = static_cast<I32>( sdiag.size() );
                    if( rest == 0 )
                    {
                        t.c0 = -1; t.c1 = 0;            // owner without rest rows
                        srest.push_back( t );
                    }
                    for( I32 c0 = 0; c0 < rest; c0 += kSolveRest )
                    {
                        t.c0 = c0; t.c1 = std::min( rest, c0 + kSolveRest );
                        srest.push_back( t );
                    }
                }
                front_panels[static_cast<size_t>( f )].push_back( static_cast<I32>( sdiag.size() ) );
                sdiag.push_back( { front_u0[f], n0, r0, front_row0[f], ld0 } );
            }
            // tiles of the step: next-row tiles first, each group by K descending
            std::vector<size_t> order( tiles.size() );
            for( size_t i = 0; i < order.size(); ++i ) { order[i] = i; }
            std::stable_sort( order.begin(), order.end(), [&]( size_t x, size_t y ) {
                if( tile_next[x] != tile_next[y] ) { return tile_next[x] > tile_next[y]; }
                if( tile_small[x] != tile_small[y] ) { return tile_small[x] > tile_small[y]; }
                return tiles[x].K > tiles[y].K;
            } );
            for( size_t i : order )
            {
                const GemmTask & t = tiles[i];
                const double rows = std::min( kTile, t.M - t.m0 ), cols = std::min( kTile, t.N - t.c0 );
                gemm_flops += 2.0 * t.K * (t.upper ? rows * (rows + 1.0) / 2.0 + rows * (cols - rows) : rows * cols);
                gemm_tile_flops += 2.0 * t.K * kTile * kTile;
                const I32 pi = tile_panel[i];
                const I32 prev = tile_prev[i];
                PendingTask d = make( LaunchKind::Gemm, static_cast<I64>(gemm.size()) );
                add_wait( d, kTrsmDone, pi, panel_trsm[static_cast<size_t>(pi)] );
                // the previous step's tiles of the front update the same C blocks
                if( prev >= 0 ) { add_wait( d, kGemmDone, prev, panel_tiles[static_cast<size_t>(prev)] ); }
                d.signal[0] = { kGemmDone, pi };
                if( tile_next[i] ) { d.signal[1] = { kNextDone, pi }; ++panel_next[static_cast<size_t>(pi)]; }
                (tile_next[i] ? next_tiles[q] : rest_tiles[q]).push_back( d );
                gemm.push_back( t );
            }
            for( size_t i : order ) { ++panel_tiles[static_cast<size_t>( tile_panel[i] )]; }

            const I32 oc = static_cast<I32>( static_cast<I64>(potrf.size()) - ofirst );
            const I32 pc = static_cast<I32>( static_cast<I64>(panel.size()) - pfirst );
            const I32 gc = static_cast<I32>( static_cast<I64>(gemm.size()) - gfirst );
            if( oc > 0 ) { factor_launches.push_back( { LaunchKind::Potrf, oc, ofirst, h, q } ); }
            if( pc > 0 ) { factor_launches.push_back( { LaunchKind::Trsm, pc, pfirst, h, q } ); }
            {
                // the step's tiles are in the order of `order`: the next panel's rows first,
                // within each part the tiles of fronts without an operand image first
                I32 gn = 0, sn0 = 0, sn1 = 0;
                for( size_t i : order )
                {
                    gn += tile_next[i] ? 1 : 0;
                    if( tile_small[i] ) { (tile_next[i] ? sn0 : sn1) += 1; }
                }
                // the same updates as tensor-core tiles: next-row tiles first, deepest first
                std::vector<size_t> tord( tct.size() );
                for( size_t i = 0; i < tord.size(); ++i ) { tord[i] = i; }
                std::stable_sort( tord.begin(), tord.end(), [&]( size_t x, size_t y ) {
                    if( tct_next[x] != tct_next[y] ) { return tct_next[x] > tct_next[y]; }
                    return tct[x].K > tct[y].K;
                } );
                const I64 tfirst = static_cast<I64>( tc.size() );
                I32 tn = 0;
                for( size_t i : tord ) { tc.push_back( tct[i] ); tn += tct_next[i] ? 1 : 0; }
                const I32 tcount = static_cast<I32>( tct.size() );
                if( gn > 0 )
                {
                    Launch L{ LaunchKind::Gemm, gn, gfirst, h, q, 0 };
                    L.small_count = sn0; L.tc_first = tfirst; L.tc_count = tn;
                    factor_launches.push_back( L );
                }
                if( gc > gn )
                {
                    Launch L{ LaunchKind::Gemm, gc - gn, gfirst + gn, h, q, 1 };
                    L.small_count = sn1; L.tc_first = tfirst + tn; L.tc_count = tcount - tn;
                    factor_launches.push_back( L );
                }
            }
            rest_ranges[h][q] = { rfirst, static_cast<I32>( static_cast<I64>(srest.size()) - rfirst ) };
        }
        // task order of the level: P0 T0, then per step q: the tiles that feed
        // panel q+1, panel q+1's potrf and trsm, the other tiles
        auto emit = [&]( const std::vector<PendingTask> & v ) { pending.insert( pending.end(), v.begin(), v.end() ); };
        if( Q > 0 ) { emit( step_potrf[0] ); emit( step_trsm[0] ); }
        for( I32 q = 0; q < Q; ++q )
        {
            emit( next_tiles[q] );
            if( q + 1 < Q ) { emit( step_potrf[q+1] ); emit( step_trsm[q+1] ); }
            emit( rest_tiles[q] );
        }
        {
            const I32 count = static_cast<I32>( extend.size() - extend_before );
            if( count > 0 ) { prev_ext_level = h; prev_ext_count = count; }
        }
    }

    // counter ids: [extend-adds per level][extend-in per front][zeroed per front]
    // [potrf, trsm, next-row tiles, all tiles per panel]
    {
        const I32 NP = static_cast<I32>( potrf.size() );
        const I32 Lv = levels;
        const I32 base[7] = { 0, Lv, Lv + F, Lv + 2 * F, Lv + 2 * F + NP, Lv + 2 * F + 2 * NP, Lv + 2 * F + 3 * NP };
        dag_counters = Lv + 2 * F + 4 * NP;
        auto id = [&]( const CounterRef & r ) { return r.kind < 0 ? -1 : base[r.kind] + r.idx; };
        // The levels below the first one whose fronts take kDagMinSteps or
        // more panel steps run as level launches (many small independent
        // fronts, where one launch per step keeps every SM full); the levels
        // from there up, where long chains of panel steps follow each other,
        // run as the task graph.  Waits on counters of the launched levels
        // are met before the persistent launch starts and are dropped.
        dag_split_level = levels;
        for( I32 h = 0; h < levels; ++h ) { if( level_steps[static_cast<size_t>(h)] >= dag_min_steps ) { dag_split_level = h; break; } }
        auto counter_level = [&]( const CounterRef & r ) -> I32 {
            switch( r.kind )
            {
                case kExtLevel: return r.idx;
                case kExtIn: case kZeroDone: return level_of[static_cast<size_t>( r.idx )];
                default: return panel_level[static_cast<size_t>( r.idx )];
            }
        };
        dag.reserve( pending.size() );
        for( const PendingTask & t : pending )
        {
            if( t.level < dag_split_level ) { continue; }
            DagTask d{};
            d.kind = t.kind; d.index = t.index;
            for( int i = 0; i < 2; ++i ) { d.signal[i] = id( t.signal[i] ); }
            int w = 0;
            for( int i = 0; i < kDagWaits; ++i ) { d.wait[i] = -1; d.target[i] = 0; }
            for( int i = 0; i < kDagWaits; ++i )
            {
                if( t.wait[i].kind < 0 || counter_level( t.wait[i] ) < dag_split_level ) { continue; }
                d.wait[w] = id( t.wait[i] ); d.target[w] = t.target[i]; ++w;
            }
            dag.push_back( d );
        }
        dag_first_panel = static_cast<I32>( std::find_if( panel_level.begin(), panel_level.end(),
                                                          [&]( I32 l ) { return l >= dag_split_level; } ) - panel_level.begin() );
    }

    // the launches that precede the persistent launch: the levels below the split
    pre_dag_launches.clear();
    for( const Launch & L : factor_launches ) { if( L.level < dag_split_level ) { pre_dag_launches.push_back( L ); } }
    for( I32 h = 0; h < levels; ++h )
    {
        for( size_t q = 0; q < rest_ranges[h].size(); ++q )
        {
            const Range r = rest_ranges[h][q];
            if( r.count > 0 ) { lower_launches.push_back( { LaunchKind::Solve, r.count, r.first, h, static_cast<I32>(q) } ); }
        }
    }
    for( I32 h = levels; h-- > 0; )
    {
        for( size_t q = rest_ranges[h].size(); q-- > 0; )
        {
            const Range r = rest_ranges[h][q];
            if( r.count > 0 ) { upper_launches.push_back( { LaunchKind::Solve, r.count, r.first, h, static_cast<I32>(q) } ); }
        }
    }
    I32 solve_split = levels;
    for( I32 h = 0; h < levels; ++h ) { if( level_steps[static_cast<size_t>(h)] >= kSolveDagMinSteps ) { solve_split = h; break; } }
    solve_default_split = solve_split;
    build_super( front_panels, [&]( I32 h, size_t q ) { return std::make_pair( rest_ranges[static_cast<size_t>(h)][q].first,
                                                                              rest_ranges[static_cast<size_t>(h)][q].count ); },
                 [&]( I32 h ) { return rest_ranges[static_cast<size_t>(h)].size(); }, by_level );
    build_solve_graph( sym, solve_split );
}

// The super-panel solve: super-panels of the large fronts, the rounds of their
// inverses, and the solve launch lists in which their panel steps are replaced.
// Within each (level, step) range of srest the tasks of the large fronts are
// moved behind the others (the order inside a range is free: its tasks are
// independent, and each panel keeps its own tasks' order), so the step
// launches of the super-panel lists cover the range's leading part.
template<typename RangeOf, typename RangeCount>
void Plan::build_super( const std::vector<std::vector<I32>> & front_panels, RangeOf range_of, RangeCount ranges,
                        const std::vector<std::vector<I32>> & by_level )
{
    spanels.clear(); sinv.clear(); sinv_launches.clear(); ssolve.clear();
    lower_launches_sp.clear(); upper_launches_sp.clear();
    super_inv_size = 0;
    const I32 F = front_count;
    std::vector<char> big( static_cast<size_t>(F), 0 );
    std::vector<std::vector<I32>> front_sp( static_cast<size_t>(F) );
    if( use_super )
    {
        for( I32 f = 0; f < F; ++f ) { big[static_cast<size_t>(f)] = front_n0[f] >= kSuperMinRows ? 1 : 0; }
    }
    for( I32 f = 0; f < F; ++f )
    {
        if( !big[static_cast<size_t>(f)] ) { continue; }
        const std::vector<I32> & pan = front_panels[static_cast<size_t>(f)];
        for( I32 r0 = 0; r0 < front_n0[f]; r0 += kSuperRows )
        {
            SuperPanel sp{};
            sp.u0 = front_u0[f]; sp.u1 = front_u1[f]; sp.inner = front_cols[f];
            sp.t = super_inv_size;
            sp.n0 = front_n0[f]; sp.n1 = front_n1[f]; sp.ld0 = front_ld0[f]; sp.ld1 = front_ld1[f];
            sp.r0 = r0; sp.rows = std::min( kSuperRows, front_n0[f] - r0 ); sp.row0 = front_row0[f];
            sp.ldt = kPanel * static_cast<I32>( ceil_div( sp.rows, kPanel ) );
            for( I32 b = 0; b < kSuperPanels; ++b )
            {
                const size_t q = static_cast<size_t>( r0 / kPanel + b );
                sp.panel[b] = (b * kPanel < sp.rows && q < pan.size()) ? pan[q] : -1;
            }
            front_sp[static_cast<size_t>(f)].push_back( static_cast<I32>( spanels.size() ) );
            spanels.push_back( sp );
            super_inv_size += static_cast<I64>( sp.ldt ) * sp.ldt;
        }
    }
    if( spanels.empty() ) { return; }
    // the inverses: round d forms the blocks at distance d from the diagonal
    for( I32 d = 0; d < kSuperPanels; ++d )
    {
        const I64 first = static_cast<I64>( sinv.size() );
        for( I32 p = 0; p < static_cast<I32>( spanels.size() ); ++p )
        {
            const I32 nblk = static_cast<I32>( ceil_div( spanels[static_cast<size_t>(p)].rows, kPanel ) );
            for( I32 i = 0; i + d < nblk; ++i ) { sinv.push_back( { p, i, i + d, 0 } ); }
        }
        const I32 count = static_cast<I32>( static_cast<I64>( sinv.size() ) - first );
        if( count > 0 ) { sinv_launches.push_back( { LaunchKind::SuperInv, count, first, levels, d } ); }
    }
    // srest ranges: the large fronts' tasks last
    // (a task's front is large exactly when its n0 is: the criterion is the front's pivot-row count)
    auto is_big_task = [&]( const SolveRestTask & t ) { return use_super && t.n0 >= kSuperMinRows; };
    std::vector<std::vector<I32>> regular( static_cast<size_t>(levels) );
    for( I32 h = 0; h < levels; ++h )
    {
        for( size_t q = 0; q < ranges( h ); ++q )
        {
            const auto r = range_of( h, q );
            auto b = srest.begin() + r.first, e = b + r.second;
            std::stable_partition( b, e, [&]( const SolveRestTask & t ) { return !is_big_task( t ); } );
            I32 nreg = 0;
            for( auto it = b; it != e; ++it ) { nreg += is_big_task( *it ) ? 0 : 1; }
            regular[static_cast<size_t>(h)].push_back( nreg );
        }
    }
    // per level: the step launches of the other fronts, then the super-panel steps
    auto super_steps = [&]( I32 h ) {
        size_t m = 0;
        for( I32 f : by_level[static_cast<size_t>(h)] ) { m = std::max( m, front_sp[static_cast<size_t>(f)].size() ); }
        return m;
    };
    auto push_super = [&]( std::vector<Launch> & list, I32 h, size_t s, bool diag, bool forward )
    {
        const I64 first = static_cast<I64>( ssolve.size() );
        for( I32 f : by_level[static_cast<size_t>(h)] )
        {
            const std::vector<I32> & v = front_sp[static_cast<size_t>(f)];
            if( s >= v.size() ) { continue; }
            const I32 p = v[s];
            const SuperPanel & sp = spanels[static_cast<size_t>(p)];
            const I32 nblk = static_cast<I32>( ceil_div( sp.rows, kPanel ) );
            if( diag )
            {
                // block pairs (o, b): forward b <= o, back b >= o
                for( I32 o = 0; o < nblk; ++o )
                {
                    for( I32 b = forward ? 0 : o; b < (forward ? o + 1 : nblk); ++b ) { ssolve.push_back( { p, o, b, 0 } ); }
                }
            }
            else
            {
                const I32 rest = (sp.n0 - sp.r0 - sp.rows) + sp.n1;
                for( I32 b = 0; b < nblk; ++b )
                {
                    for( I32 c0 = 0; c0 < rest; c0 += kSolveRest ) { ssolve.push_back( { p, b, c0, std::min( rest, c0 + kSolveRest ) } ); }
                }
            }
        }
        const I32 count = static_cast<I32>( static_cast<I64>( ssolve.size() ) - first );
        if( count > 0 )
        {
            Launch L{ diag ? LaunchKind::SuperDiag : LaunchKind::SuperRest, count, first, h, static_cast<I32>( s ) };
            L.part = forward ? 0 : 1;
            list.push_back( L );
        }
    };
    for( I32 h = 0; h < levels; ++h )
    {
        for( size_t q = 0; q < ranges( h ); ++q )
        {
            const auto r = range_of( h, q );
            const I32 nreg = regular[static_cast<size_t>(h)][q];
            if( nreg > 0 ) { lower_launches_sp.push_back( { LaunchKind::Solve, nreg, r.first, h, static_cast<I32>(q) } ); }
        }
        for( size_t st = 0; st < super_steps( h ); ++st )
        {
            push_super( lower_launches_sp, h, st, true, true );
            push_super( lower_launches_sp, h, st, false, true );
        }
    }
    for( I32 h = levels; h-- > 0; )
    {
        for( size_t st = super_steps( h ); st-- > 0; )
        {
            push_super( upper_launches_sp, h, st, false, false );
            push_super( upper_launches_sp, h, st, true, false );
        }
        for( size_t q = ranges( h ); q-- > 0; )
        {
            const auto r = range_of( h, q );
            const I32 nreg = regular[static_cast<size_t>(h)][q];
            if( nreg > 0 ) { upper_launches_sp.push_back( { LaunchKind::Solve, nreg, r.first, h, static_cast<I32>(q) } ); }
        }
    }
}

void Plan::build_solve_graph( const Symbolic & sym, I32 split )
{
    solve_split_level = std::min( std::max( split, 0 ), levels );
    solve_fwd_order.clear(); solve_bwd_order.clear(); solve_target_ptr.clear(); solve_targets.clear();
    solve_fwd_expected.clear(); solve_panel_tasks.clear();
    solve_first_task = static_cast<I64>( srest.size() );
    for( const Launch & L : lower_launches )
    {
        if( L.level >= solve_split_level ) { solve_first_task = std::min( solve_first_task, L.first ); }
    }
    // the lowest panel of the graph's tasks (the super-panel lists reorder the tasks inside a
    // (level, step) range, so the first task need not hold it)
    solve_first_panel = static_cast<I32>( sdiag.size() );
    for( I64 t = solve_first_task; t < static_cast<I64>( srest.size() ); ++t )
    {
        solve_first_panel = std::min( solve_first_panel, srest[static_cast<size_t>( t )].panel );
    }
    const I64 nt = static_cast<I64>( srest.size() ) - solve_first_task;
    const I32 np = static_cast<I32>( sdiag.size() ) - solve_first_panel;
    solve_target_ptr.assign( static_cast<size_t>( nt ) + 1, 0 );
    solve_fwd_expected.assign( static_cast<size_t>( np ), 0 );
    solve_panel_tasks.assign( static_cast<size_t>( np ), 0 );
    if( nt == 0 ) { return; }

    // panel id of (front, panel step)
    auto front_of_row = [&]( I32 row ) { return front_of_sn[static_cast<size_t>( sym.row_to_sn[static_cast<size_t>( row )] )]; };
    std::vector<std::vector<I32>> panel_of( static_cast<size_t>( front_count ) );
    for( I32 p = solve_first_panel; p < static_cast<I32>( sdiag.size() ); ++p )
    {
        const SolveDiagTask & d = sdiag[static_cast<size_t>(p)];
        std::vector<I32> & v = panel_of[static_cast<size_t>( front_of_row( d.row0 ) )];
        const size_t q = static_cast<size_t>( d.r0 / kPanel );
        if( v.size() <= q ) { v.resize( q + 1, -1 ); }
        v[q] = p;
    }
    auto panel_of_row = [&]( I32 f, I32 local ) -> I32 {
        const std::vector<I32> & v = panel_of[static_cast<size_t>(f)];
        const size_t q = static_cast<size_t>( local / kPanel );
        return q < v.size() ? v[q] : -1;
    };
    std::vector<I32> tg;
    for( I64 i = 0; i < nt; ++i )
    {
        const SolveRestTask & t = srest[static_cast<size_t>( solve_first_task + i )];
        ++solve_panel_tasks[static_cast<size_t>( t.panel - solve_first_panel )];
        tg.clear();
        if( t.c0 >= 0 )
        {
            const I32 f = front_of_row( t.row0 );
            const I32 nb = std::min( kPanel, t.n0 - t.r0 );
            const I32 r1 = t.r0 + nb, m = t.n0 - r1;
            for( I32 col = t.c0; col < t.c1; ++col )
            {
                I32 p = -1;
                if( col < m ) { p = panel_of_row( f, r1 + col ); }
                else
                {
                    const I32 g = sym.sn_inner[static_cast<size_t>( t.inner + (col - m) )];
                    const I32 fa = front_of_row( g );
                    p = panel_of_row( fa, g - front_row0[static_cast<size_t>(fa)] );
                }
                if( p >= solve_first_panel && (tg.empty() || tg.back() != p) ) { tg.push_back( p ); }
            }
            std::sort( tg.begin(), tg.end() );
            tg.erase( std::unique( tg.begin(), tg.end() ), tg.end() );
        }
        for( I32 p : tg )
        {
            solve_targets.push_back( p - solve_first_panel );
            ++solve_fwd_expected[static_cast<size_t>( p - solve_first_panel )];
        }
        solve_target_ptr[static_cast<size_t>( i ) + 1] = static_cast<I64>( solve_targets.size() );
        solve_fwd_order.push_back( static_cast<I32>( solve_first_task + i ) );
    }
    // back sweep: panels in reverse order, each panel's tasks in list order
    for( I64 e = static_cast<I64>( srest.size() ); e > solve_first_task; )
    {
        I64 b = e - 1;
        while( b > solve_first_task && srest[static_cast<size_t>( b - 1 )].panel == srest[static_cast<size_t>( e - 1 )].panel ) { --b; }
        for( I64 j = b; j < e; ++j ) { solve_bwd_order.push_back( static_cast<I32>( j ) ); }
        e = b;
    }
}

} // namespace tb
