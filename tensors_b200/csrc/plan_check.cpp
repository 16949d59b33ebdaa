// Host-side bounds check of a device plan.
//
// Every device kernel of the factorization and solves reads and writes the
// arena only through the offsets, sizes and leading dimensions in its task
// records.  This check recomputes, for every task, the extreme offsets the
// kernel can touch and verifies them against the buffers the kernel is given,
// so an indexing error is caught on the host before any launch.

#include "plan.hpp"
#include "plan_check.hpp"
#include "parallel.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <map>
#include <string>
#include <vector>

namespace tb
{
namespace
{
using I32 = std::int32_t;
using I64 = std::int64_t;

bool in_range( I64 first, I64 last_inclusive, I64 size )
{
    return first >= 0 && last_inclusive >= first && last_inclusive < size;
}

// The lowest index in [0, count) for which bad(i) holds, or -1; the range is
// split over `threads` host threads (<= 0: all) (the message is then rebuilt for that index, so
// the report does not depend on the threads).
template<typename Bad>
I64 first_bad( I64 threads, I64 count, Bad && bad )
{
    std::atomic<I64> first{ count };
    parallel_rows( count, [&]( I64 b, I64 e )
    {
        for( I64 i = b; i < e && i < first.load( std::memory_order_relaxed ); ++i )
        {
            if( !bad( i ) ) { continue; }
            I64 cur = first.load();
            while( i < cur && !first.compare_exchange_weak( cur, i ) ) {}
            break;
        }
    }, threads );
    const I64 f = first.load();
    return f < count ? f : -1;
}

} // namespace

std::string check_plan( const Symbolic & sym, const Plan & pl )
{
    const I64 arena = pl.arena_size();
    const I64 nnz = sym.nnz;
    const I64 inner_size = static_cast<I64>( sym.sn_inner.size() );
    const I64 tri_size = sym.sn_tri_ptr[sym.sn_count];
    const I64 rec_size = sym.sn_rec_ptr[sym.sn_count];

    if( pl.asm_src.size() != pl.asm_dst.size() ) { return "assembly map sizes differ"; }
    {
        auto entry = [&]( I64 e ) -> std::string
        {
            const I64 d = static_cast<I64>( static_cast<std::uint64_t>( pl.asm_dst[static_cast<size_t>( e )] ) & (kDiagFlag - 1) );
            const I64 src = pl.asm_src[static_cast<size_t>( e )];
            if( src < 0 || src >= nnz ) { return "assembly source out of range at " + std::to_string( e ); }
            if( d < 0 || d >= pl.u0_size + pl.u1_size ) { return "assembly target out of range at " + std::to_string( e ); }
            return std::string();
        };
        const I64 bad = first_bad( pl.threads, static_cast<I64>( pl.asm_src.size() ), [&]( I64 e ) { return !entry( e ).empty(); } );
        if( bad >= 0 ) { return entry( bad ); }
    }
    for( size_t i = 0; i < pl.diag_offset.size(); ++i )
    {
        if( pl.diag_offset[i] < 0 || pl.diag_offset[i] >= pl.u0_size ) { return "diagonal offset out of range"; }
    }
    for( const ZeroTask & z : pl.zero )
    {
        if( z.count <= 0 || z.row_begin < 0 || z.row_begin >= z.row_end || z.row_end > z.n || z.n > z.ld )
        {
            return "bad zero task";
        }
        if( !in_range( z.offset, z.offset + static_cast<I64>( z.row_end - 1 ) * z.ld + z.n - 1, arena ) ) { return "zero task out of range"; }
    }
    std::vector<I32> lut_seen( pl.lut.size() + 1, 0 );
    const size_t n_ext = pl.extend.size();
    for( size_t k = 0; k < n_ext + pl.extend_segs.size(); ++k )
    {
        const ExtendTask & t = k < n_ext ? pl.extend[k] : pl.extend_segs[k - n_ext];
        auto at = [&]() { return k < n_ext ? " (extend task " + std::to_string( k ) + ")"
                                           : " (extend segment " + std::to_string( k - n_ext ) + ")"; };   // built only on failure
        if( t.m1 <= 0 || t.mid < 0 || t.mid > t.m1 ) { return "bad extend dimensions" + at(); }
        if( t.row_begin < 0 || t.row_end > t.m1 || t.row_begin >= t.row_end ) { return "bad extend rows" + at(); }
        if( t.ldw < t.m1 || t.ld0p < t.n0p || t.ld1p < t.n1p || t.ldvp < t.n1p ) { return "extend leading dimension too small" + at(); }
        if( !in_range( t.w, t.w + static_cast<I64>(t.m1) * t.ldw - 1, arena ) ) { return "extend source out of range" + at(); }
        if( t.lut < 0 || t.lut + t.m1 > static_cast<I64>( pl.lut.size() ) ) { return "extend lut out of range" + at(); }
        const I64 u0n = static_cast<I64>(t.n0p) * t.ld0p, u1n = static_cast<I64>(t.n0p) * t.ld1p, vn = static_cast<I64>(t.n1p) * t.ldvp;
        if( u0n > 0 && !in_range( t.u0, t.u0 + u0n - 1, arena ) ) { return "extend U0 out of range" + at(); }
        if( u1n > 0 && !in_range( t.u1, t.u1 + u1n - 1, arena ) ) { return "extend U1 out of range" + at(); }
        if( t.mid < t.m1 && (vn == 0 || !in_range( t.v, t.v + vn - 1, arena )) ) { return "extend V out of range" + at(); }
        // the row groups of one child share its lookup table: check it once
        if( lut_seen[static_cast<size_t>( t.lut )] == t.m1 + 1 ) { continue; }
        lut_seen[static_cast<size_t>( t.lut )] = t.m1 + 1;
        for( I32 i = 0; i < t.m1; ++i )
        {
            const I32 l = pl.lut[t.lut + i];
            const I32 lim = (i < t.mid) ? t.n0p : t.n1p;
            if( l < 0 || l >= lim ) { return "extend lut value out of range" + at(); }
            if( i > 0 && i != t.mid && l <= pl.lut[t.lut + i - 1] ) { return "extend lut not increasing" + at(); }
        }
    }
    // extend-add by parent rows: per level launch, the segments cover every row of the level's
    // extend tasks once; a task's segments share one parent and one block of its pivot or update
    // rows, in child-rank order (the order of the children's first tasks in the passes)
    for( const Launch & L : pl.factor_launches )
    {
        if( L.kind != LaunchKind::ExtendPull ) { continue; }
        if( L.tc_first < 0 || L.tc_count < 0 || L.tc_first + L.tc_count > static_cast<I64>( pl.extend.size() ) ) { return "extend pull launch: task range"; }
        std::map<I64, std::pair<I64, std::vector<I32>>> rows;          // child W -> (rank, rows left to add)
        for( I64 k = L.tc_first; k < L.tc_first + L.tc_count; ++k )
        {
            const ExtendTask & t = pl.extend[static_cast<size_t>( k )];
            auto it = rows.find( t.w );
            if( it == rows.end() ) { it = rows.emplace( t.w, std::make_pair( k, std::vector<I32>( static_cast<size_t>( t.m1 ), 0 ) ) ).first; }
            for( I32 i = t.row_begin; i < t.row_end; ++i ) { ++it->second.second[static_cast<size_t>( i )]; }
        }
        for( I64 q = L.first; q < L.first + L.count; ++q )
        {
            const ExtendPullTask & u = pl.extend_pull[static_cast<size_t>( q )];
            if( u.seg_count <= 0 || u.seg_first < 0 || u.seg_first + u.seg_count > static_cast<I64>( pl.extend_segs.size() ) ) { return "extend pull task out of range"; }
            const ExtendTask & s0 = pl.extend_segs[static_cast<size_t>( u.seg_first )];
            const bool upper = u.space == 0;
            if( (u.space != 0 && u.space != 1) || u.b0 < 0 || u.b1 <= u.b0 || u.b1 > (upper ? s0.n0p : s0.n1p) ) { return "extend pull task rows out of range"; }
            I64 rank = -1;
            for( I64 g = u.seg_first; g < u.seg_first + u.seg_count; ++g )
            {
                const ExtendTask & t = pl.extend_segs[static_cast<size_t>( g )];
                if( t.u0 != s0.u0 || t.u1 != s0.u1 || t.v != s0.v ) { return "extend pull task spans parents"; }
                if( (t.row_end <= t.mid) != upper || (t.row_begin < t.mid) != upper ) { return "extend pull segment spans row spaces"; }
                if( pl.lut[t.lut + t.row_begin] < u.b0 || pl.lut[t.lut + t.row_end - 1] >= u.b1 ) { return "extend pull segment outside its row block"; }
                auto it = rows.find( t.w );
                if( it == rows.end() ) { return "extend pull segment of a child not in its level"; }
                if( it->second.first <= rank ) { return "extend pull segments not in child-rank order"; }
                rank = it->second.first;
                for( I32 i = t.row_begin; i < t.row_end; ++i ) { --it->second.second[static_cast<size_t>( i )]; }
            }
        }
        for( const auto & kv : rows )
        {
            for( I32 c : kv.second.second ) { if( c != 0 ) { return "extend pull launch does not add every child row once"; } }
        }
    }
    for( int which = 0; which < 2; ++which )
    {
        const std::vector<PanelTask> & list = which == 0 ? pl.potrf : pl.panel;
        for( size_t k = 0; k < list.size(); ++k )
        {
            const PanelTask & t = list[k];
            auto at = [&]() { return std::string( which == 0 ? " (potrf task " : " (trsm task " ) + std::to_string( k ) + ")"; };   // built only on failure
            if( t.n0 <= 0 || t.r0 < 0 || t.r0 >= t.n0 || t.n1 < 0 ) { return "bad panel dimensions" + at(); }
            if( t.ld0 < t.n0 || t.ld1 < t.n1 ) { return "panel leading dimension too small" + at(); }
            if( !in_range( t.u0, t.u0 + static_cast<I64>(t.n0) * t.ld0 - 1, arena ) ) { return "panel U0 out of range" + at(); }
            if( t.n1 > 0 && !in_range( t.u1, t.u1 + static_cast<I64>(t.n0) * t.ld1 - 1, arena ) ) { return "panel U1 out of range" + at(); }
            const I32 nb = std::min( kPanel, t.n0 - t.r0 );
            const I32 rest = (t.n0 - t.r0 - nb) + t.n1;
            if( which == 1 && (t.c0 < 0 || t.c0 >= rest) ) { return "panel chunk out of range" + at(); }
            if( t.row0 < 0 || t.row0 + t.n0 > sym.n ) { return "panel rows out of range" + at(); }
            // the inverse diagonal block: one per panel, written by the panel's potrf task
            if( t.panel < 0 || t.panel >= static_cast<I32>( pl.sdiag.size() ) ) { return "panel index out of range" + at(); }
            if( which == 0 && t.panel != static_cast<I32>( k ) ) { return "potrf task is not its panel's" + at(); }
            if( which == 1 && (pl.potrf[static_cast<size_t>( t.panel )].r0 != t.r0 || pl.potrf[static_cast<size_t>( t.panel )].u0 != t.u0) )
            {
                return "trsm task names another panel" + at();
            }
        }
    }
    {
        // every panel's contribution to every trailing entry is applied exactly
        // once, however the updates are grouped (deferral over panel steps):
        // the tiles' flops equal, front by front summed, 2 nb per upper entry of
        // each panel's trailing block and U1 rows, plus the update matrix V
        double expect = 0.0;
        const I32 F = pl.front_count;
        for( I32 f = 0; f < F; ++f )
        {
            const double n0 = pl.front_n0[static_cast<size_t>(f)], n1 = pl.front_n1[static_cast<size_t>(f)];
            for( I32 r0 = 0; r0 < pl.front_n0[static_cast<size_t>(f)]; r0 += kPanel )
            {
                const double nb = std::min<double>( kPanel, n0 - r0 ), m = n0 - r0 - nb;
                expect += 2.0 * nb * (m * (m + 1.0) / 2.0 + m * n1);
            }
            if( n1 > 0 && pl.front_parent[static_cast<size_t>(f)] < F ) { expect += 2.0 * n0 * n1 * (n1 + 1.0) / 2.0; }
        }
        if( std::abs( expect - pl.gemm_flops ) > 1e-12 * std::max( 1.0, expect ) )
        {
            return "GEMM tiles do not apply every panel update exactly once (flops " + std::to_string( pl.gemm_flops )
                   + ", expected " + std::to_string( expect ) + ")";
        }
    }
    {
        // update matrices: each lies in the update region, and two whose
        // lifetimes (the front's level to its parent's level, both inclusive)
        // intersect never share an entry
        const I32 F = pl.front_count;
        std::vector<std::vector<I32>> born( static_cast<size_t>( pl.levels ) ), dies( static_cast<size_t>( pl.levels ) );
        for( I32 f = 0; f < F; ++f )
        {
            const size_t fs = static_cast<size_t>( f );
            const I64 size = static_cast<I64>( pl.front_n1[fs] ) * pl.front_ld1[fs];
            if( size == 0 ) { continue; }
            if( pl.front_v[fs] < pl.u0_size + pl.u1_size || !in_range( pl.front_v[fs], pl.front_v[fs] + size - 1, arena ) )
            {
                return "update matrix outside the update region (front " + std::to_string( f ) + ")";
            }
            const I32 p = pl.front_parent[fs];
            const I32 last = p < F ? pl.level_of[static_cast<size_t>( p )] : pl.level_of[fs];
            if( pl.level_of[fs] < 0 || last < pl.level_of[fs] || last >= pl.levels ) { return "update matrix lifetime invalid (front " + std::to_string( f ) + ")"; }
            born[static_cast<size_t>( pl.level_of[fs] )].push_back( f );
            dies[static_cast<size_t>( last )].push_back( f );
        }
        std::map<I64,I32> live;   // offset -> front
        for( I32 h = 0; h < pl.levels; ++h )
        {
            for( I32 f : born[static_cast<size_t>( h )] )
            {
                const I64 off = pl.front_v[static_cast<size_t>( f )];
                const I64 end = off + static_cast<I64>( pl.front_n1[static_cast<size_t>( f )] ) * pl.front_ld1[static_cast<size_t>( f )];
                auto next = live.lower_bound( off );
                bool clash = next != live.end() && next->first < end;
                if( next != live.begin() )
                {
                    const I32 g = std::prev( next )->second;
                    clash = clash || pl.front_v[static_cast<size_t>( g )] + static_cast<I64>( pl.front_n1[static_cast<size_t>( g )] ) * pl.front_ld1[static_cast<size_t>( g )] > off;
                }
                if( clash ) { return "live update matrices overlap (front " + std::to_string( f ) + ", level " + std::to_string( h ) + ")"; }
                live.emplace( off, f );
            }
            for( I32 f : dies[static_cast<size_t>( h )] ) { live.erase( pl.front_v[static_cast<size_t>( f )] ); }
        }
    }
    {
        auto task = [&]( I64 k ) -> std::string
        {
            const GemmTask & t = pl.gemm[static_cast<size_t>( k )];
            auto at = [&]() { return " (gemm task " + std::to_string( k ) + ")"; };   // built only on failure
            if( t.K <= 0 || t.M <= 0 || t.N <= 0 || t.m0 < 0 || t.m0 >= t.M || t.c0 < 0 || t.c0 >= t.N ) { return "bad gemm dimensions" + at(); }
            if( t.M > t.lda || t.N > t.ldb || t.N > t.ldc ) { return "gemm leading dimension too small" + at(); }
            // 16-byte copies of FP64 (2 entries) and FP32 (4 entries) storage
            if( (t.a | t.b | t.c) % 4 != 0 || (t.lda | t.ldb | t.ldc) % 4 != 0 ) { return "gemm operand not 16-byte aligned" + at(); }
            if( !in_range( t.a, t.a + static_cast<I64>(t.K - 1) * t.lda + t.M - 1, arena ) ) { return "gemm A out of range" + at(); }
            if( !in_range( t.b, t.b + static_cast<I64>(t.K - 1) * t.ldb + t.N - 1, arena ) ) { return "gemm B out of range" + at(); }
            if( !in_range( t.c, t.c + static_cast<I64>(t.M - 1) * t.ldc + t.N - 1, arena ) ) { return "gemm C out of range" + at(); }
            return std::string();
        };
        const I64 bad = first_bad( pl.threads, static_cast<I64>( pl.gemm.size() ), [&]( I64 k ) { return !task( k ).empty(); } );
        if( bad >= 0 ) { return task( bad ); }
    }
    {
        // tensor-core tiles (FP32 path): C in the arena, 16-byte aligned rows;
        // the image blocks of their valid rows, columns and k-chunks inside the
        // image (the copies of the blocks past a front's end read other
        // fronts' data or zeros, used only for rows and columns not written)
        auto task = [&]( I64 k ) -> std::string
        {
            const TcTask & t = pl.tc[static_cast<size_t>( k )];
            auto at = [&]() { return " (tensor-core tile " + std::to_string( k ) + ")"; };   // built only on failure
            if( t.K <= 0 || t.M <= 0 || t.N <= 0 || t.m0 < 0 || t.m0 >= t.M || t.c0 < 0 || t.c0 >= t.N ) { return "bad tile dimensions" + at(); }
            if( t.nt < kImgRows || t.nt > kTcNMax || t.nt % kImgRows != 0 || t.m0 % kTcM != 0 || t.c0 % kImgRows != 0 ) { return "bad tile shape" + at(); }
            if( t.N > t.ldc || t.c % 4 != 0 || t.ldc % 4 != 0 ) { return "tile C leading dimension or alignment" + at(); }
            if( !in_range( t.c, t.c + static_cast<I64>(t.M - 1) * t.ldc + t.N - 1, arena ) ) { return "tile C out of range" + at(); }
            const I64 nk = (t.K + kImgK - 1) / kImgK;
            const I32 rows = std::min( kTcM, t.M - t.m0 ), cols = std::min( t.nt, t.N - t.c0 );
            if( t.tf <= 0 || t.ta < 0 || t.tb < 0 || t.ta + (rows - 1) / kImgRows >= t.tf || t.tb + (cols - 1) / kImgRows >= t.tf ) { return "tile column tiles out of range" + at(); }
            if( t.blk < 0 || t.blk + (nk - 1) * 2 * t.tf + 2 * t.tf > pl.img_blocks ) { return "tile k-chunks outside the operand image" + at(); }
            return std::string();
        };
        const I64 bad = first_bad( pl.threads, static_cast<I64>( pl.tc.size() ), [&]( I64 k ) { return !task( k ).empty(); } );
        if( bad >= 0 ) { return task( bad ); }
        // each panel step: its GEMM launches' small-front tiles and tensor-core tiles do the step's
        // updates (a tensor-core tile of the first tile row spans both launches' rows)
        for( const std::vector<Launch> * list : { &pl.factor_launches, &pl.pre_dag_launches } )
        {
            std::map<std::pair<I32, I32>, std::pair<double, double>> steps;   // (level, step) -> (want, got)
            for( const Launch & L : *list )
            {
                if( L.kind != LaunchKind::Gemm ) { continue; }
                if( L.small_count < 0 || L.small_count > L.count || L.tc_count < 0 || L.tc_first < 0
                    || L.tc_first + L.tc_count > static_cast<I64>( pl.tc.size() ) ) { return "tensor-core tile range out of bounds"; }
                double want = 0.0, got = 0.0;
                for( I64 i = L.first; i < L.first + L.count; ++i )
                {
                    const GemmTask & t = pl.gemm[static_cast<size_t>( i )];
                    const double r = std::min( kTile, t.M - t.m0 ), c = std::min( kTile, t.N - t.c0 );
                    const double f = 2.0 * t.K * (t.upper ? r * (r + 1.0) / 2.0 + r * (c - r) : r * c);
                    want += f;
                    if( i < L.first + L.small_count ) { got += f; }
                }
                for( I64 i = L.tc_first; i < L.tc_first + L.tc_count; ++i )
                {
                    const TcTask & t = pl.tc[static_cast<size_t>( i )];
                    const I64 r = std::min( kTcM, t.M - t.m0 ), c = std::min( t.nt, t.N - t.c0 );
                    double e = 0.0;
                    if( !t.upper ) { e = static_cast<double>( r ) * c; }
                    else
                    {
                        // entries (m0 + i, c0 + j) with m0 + i <= c0 + j
                        for( I64 i2 = 0; i2 < r; ++i2 ) { e += static_cast<double>( std::max<I64>( 0, c - std::max<I64>( 0, t.m0 + i2 - t.c0 ) ) ); }
                    }
                    got += 2.0 * t.K * e;
                }
                auto & acc = steps[{ L.level, L.step }];
                acc.first += want;
                acc.second += got;
            }
            for( const auto & kv : steps )
            {
                const double want = kv.second.first, got = kv.second.second;
                if( std::abs( want - got ) > 1e-12 * std::max( 1.0, want ) )
                {
                    return "tensor-core tiles do not do their step's updates (level " + std::to_string( kv.first.first ) + ", step "
                           + std::to_string( kv.first.second ) + ": " + std::to_string( got ) + " of " + std::to_string( want ) + " flops)";
                }
            }
        }
        // the trsm's image writes stay inside the front's image segments
        for( size_t k = 0; k < pl.panel.size(); ++k )
        {
            const PanelTask & t = pl.panel[k];
            if( t.img < 0 ) { continue; }
            const I64 t0 = (t.n0 + kImgRows - 1) / kImgRows, tf = t0 + (t.n1 + kImgRows - 1) / kImgRows;
            if( t.img_t0 != t0 || t.img_tf != tf || t.img + (t.n0 + kImgK - 1) / kImgK * 2 * tf > pl.img_blocks )
            {
                return "trsm image segment out of range (panel task " + std::to_string( k ) + ")";
            }
        }
    }
    for( size_t k = 0; k < pl.sdiag.size(); ++k )
    {
        const SolveDiagTask & t = pl.sdiag[k];
        if( t.n0 <= 0 || t.r0 < 0 || t.r0 >= t.n0 || t.ld0 < t.n0 ) { return "bad solve-diag dimensions"; }
        if( !in_range( t.u0, t.u0 + static_cast<I64>(t.n0) * t.ld0 - 1, arena ) ) { return "solve-diag U0 out of range"; }
        if( t.row0 < 0 || t.row0 + t.n0 > sym.n ) { return "solve-diag rows out of range"; }
    }
    for( size_t k = 0; k < pl.srest.size(); ++k )
    {
        const SolveRestTask & t = pl.srest[k];
        auto at = [&]() { return " (solve-rest task " + std::to_string( k ) + ")"; };   // built only on failure
        if( t.n0 <= 0 || t.r0 < 0 || t.r0 >= t.n0 || t.n1 < 0 ) { return "bad solve-rest dimensions" + at(); }
        const I32 nb = std::min( kPanel, t.n0 - t.r0 );
        const I32 rest = (t.n0 - t.r0 - nb) + t.n1;
        const bool owner = t.c0 < 0;
        if( owner ? (t.c0 != -1 || t.c1 != 0 || rest != 0)
                  : (t.c1 > rest || t.c0 >= t.c1 || t.c1 - t.c0 > kSolveRest) ) { return "solve-rest range out of bounds" + at(); }
        if( t.panel < 0 || static_cast<size_t>( t.panel ) >= pl.sdiag.size() ) { return "solve-rest panel out of range" + at(); }
        {
            const SolveDiagTask & d = pl.sdiag[static_cast<size_t>( t.panel )];
            if( d.u0 != t.u0 || d.r0 != t.r0 || d.n0 != t.n0 || d.row0 != t.row0 ) { return "solve-rest panel mismatch" + at(); }
        }
        if( t.ld0 < t.n0 || t.ld1 < t.n1 ) { return "solve-rest leading dimension too small" + at(); }
        if( !in_range( t.u0, t.u0 + static_cast<I64>(t.n0) * t.ld0 - 1, arena ) ) { return "solve-rest U0 out of range" + at(); }
        if( t.n1 > 0 && !in_range( t.u1, t.u1 + static_cast<I64>(t.n0) * t.ld1 - 1, arena ) ) { return "solve-rest U1 out of range" + at(); }
        if( t.n1 > 0 && (t.inner < 0 || t.inner + t.n1 > inner_size) ) { return "solve-rest columns out of range" + at(); }
        if( t.row0 < 0 || t.row0 + t.n0 > sym.n ) { return "solve-rest rows out of range" + at(); }
    }
    for( I32 v : sym.sn_inner ) { if( v < 0 || v >= sym.n ) { return "SN_inner value out of range"; } }
    {
        auto task = [&]( I64 k ) -> std::string
        {
            const ExportTask & t = pl.exports[static_cast<size_t>( k )];
            auto at = [&]() { return " (export task " + std::to_string( k ) + ")"; };   // built only on failure
            if( t.n0s <= 0 || t.r_begin < 0 || t.r_end > t.n0s || t.r_begin >= t.r_end ) { return "bad export rows" + at(); }
            if( t.roff < 0 || t.roff + t.n0s > t.fn0 ) { return "export rows outside the front" + at(); }
            if( !in_range( t.tri, t.tri + static_cast<I64>(t.n0s) * t.n0s - 1, tri_size ) ) { return "export tri out of range" + at(); }
            if( t.n1s > 0 && !in_range( t.rec, t.rec + static_cast<I64>(t.n0s) * t.n1s - 1, rec_size ) ) { return "export rec out of range" + at(); }
            if( t.fld0 < t.fn0 || t.fld1 < t.fn1 ) { return "export leading dimension too small" + at(); }
            if( !in_range( t.fu0, t.fu0 + static_cast<I64>(t.fn0) * t.fld0 - 1, arena ) ) { return "export front U0 out of range" + at(); }
            if( t.fn1 > 0 && !in_range( t.fu1, t.fu1 + static_cast<I64>(t.fn0) * t.fld1 - 1, arena ) ) { return "export front U1 out of range" + at(); }
            if( t.colmap < 0 || t.colmap + t.n1s > static_cast<I64>( pl.colmap.size() ) ) { return "export colmap out of range" + at(); }
            if( k > 0 )
            {
                // the row blocks of one supernode share its column map: the previous task
                // checked the same entries against the same limits (and failed first if any is bad)
                const ExportTask & p = pl.exports[static_cast<size_t>( k - 1 )];
                if( p.colmap == t.colmap && p.n1s == t.n1s && p.fn0 == t.fn0 && p.fn1 == t.fn1 ) { return std::string(); }
            }
            for( I32 l = 0; l < t.n1s; ++l )
            {
                const I32 cm = pl.colmap[t.colmap + l];
                if( cm >= 0 ? cm >= t.fn0 : (-cm - 1) >= t.fn1 ) { return "export colmap value out of range" + at(); }
            }
            return std::string();
        };
        // checked on all host threads, the first failing task reported
        const I64 bad = first_bad( pl.threads, static_cast<I64>( pl.exports.size() ), [&]( I64 k ) { return !task( k ).empty(); } );
        if( bad >= 0 ) { return task( bad ); }
    }
    auto size_of = [&]( LaunchKind kind ) -> I64
    {
        switch( kind )
        {
            case LaunchKind::Zero:   return static_cast<I64>( pl.zero.size() );
            case LaunchKind::Extend: return static_cast<I64>( pl.extend.size() );
            case LaunchKind::Trsm:   return static_cast<I64>( pl.panel.size() );
            case LaunchKind::Gemm:   return static_cast<I64>( pl.gemm.size() );
            case LaunchKind::Invert: return static_cast<I64>( pl.sdiag.size() );
            case LaunchKind::Solve:  return static_cast<I64>( pl.srest.size() );
            case LaunchKind::Potrf:  return static_cast<I64>( pl.potrf.size() );
            case LaunchKind::ExtendPull: return static_cast<I64>( pl.extend_pull.size() );
            default: break;
        }
        return -1;
    };
    for( const std::vector<Launch> * list : { &pl.factor_launches, &pl.pre_dag_launches, &pl.lower_launches, &pl.upper_launches } )
    {
        for( const Launch & L : *list )
        {
            if( L.count <= 0 || L.first < 0 || L.first + L.count > size_of( L.kind ) ) { return "launch task range out of bounds"; }
        }
    }
    // task graph: every task index in range, and every wait reached by
    // signals of tasks earlier in the list (so a first-come first-served
    // walk of the list never waits for a task that has not been taken)
    {
        std::vector<I64> cnt( static_cast<size_t>( std::max( 0, pl.dag_counters ) ), 0 );
        I64 work = 0;
        for( size_t k = 0; k < pl.dag.size(); ++k )
        {
            const DagTask & t = pl.dag[k];
            auto at = [&]() { return " (graph task " + std::to_string( k ) + ")"; };   // built only on failure
            const LaunchKind kind = static_cast<LaunchKind>( t.kind );
            if( kind == LaunchKind::Solve || t.index < 0 || t.index >= size_of( kind ) ) { return "task graph index out of range" + at(); }
            ++work;
            for( int i = 0; i < kDagWaits; ++i )
            {
                if( t.wait[i] < 0 ) { continue; }
                if( t.wait[i] >= pl.dag_counters ) { return "task graph counter out of range" + at(); }
                if( t.target[i] <= 0 || cnt[static_cast<size_t>( t.wait[i] )] < t.target[i] ) { return "task graph wait not reached by earlier tasks" + at(); }
            }
            for( int i = 0; i < 2; ++i )
            {
                if( t.signal[i] < 0 ) { continue; }
                if( t.signal[i] >= pl.dag_counters ) { return "task graph counter out of range" + at(); }
                ++cnt[static_cast<size_t>( t.signal[i] )];
            }
        }
        I64 expect = 0, pre = 0;
        // an ExtendPull launch stands for its level's extend tasks
        for( const Launch & L : pl.factor_launches ) { expect += L.kind == LaunchKind::ExtendPull ? L.tc_count : L.count; }
        for( const Launch & L : pl.pre_dag_launches ) { pre += L.kind == LaunchKind::ExtendPull ? L.tc_count : L.count; }
        if( work + pre != expect ) { return "task graph and preceding launches do not cover the factorization tasks"; }
    }
    for( const Launch & L : pl.lower_launches ) { if( L.kind != LaunchKind::Solve ) { return "unexpected launch kind in the forward solve"; } }
    for( const Launch & L : pl.upper_launches ) { if( L.kind != LaunchKind::Solve ) { return "unexpected launch kind in the back solve"; } }
    if( !pl.spanels.empty() )
    {
        // super-panels: blocks inside their fronts and the arena, inverses inside their buffer, the
        // panel inverses they start from belong to their rows
        const I64 nsp = static_cast<I64>( pl.spanels.size() );
        std::vector<I32> nblk( static_cast<size_t>( nsp ) ), nrest( static_cast<size_t>( nsp ) );
        for( I64 p = 0; p < nsp; ++p )
        {
            const SuperPanel & sp = pl.spanels[static_cast<size_t>( p )];
            const std::string at = " (super-panel " + std::to_string( p ) + ")";
            if( sp.rows <= 0 || sp.rows > kSuperRows || sp.r0 < 0 || sp.r0 % kSuperRows != 0 || sp.r0 + sp.rows > sp.n0 ) { return "bad super-panel rows" + at; }
            if( sp.ld0 < sp.n0 || sp.ld1 < sp.n1 || sp.n1 < 0 ) { return "bad super-panel dimensions" + at; }
            if( !in_range( sp.u0, sp.u0 + static_cast<I64>( sp.n0 ) * sp.ld0 - 1, arena ) ) { return "super-panel U0 out of range" + at; }
            if( sp.n1 > 0 && !in_range( sp.u1, sp.u1 + static_cast<I64>( sp.n0 ) * sp.ld1 - 1, arena ) ) { return "super-panel U1 out of range" + at; }
            if( sp.n1 > 0 && (sp.inner < 0 || sp.inner + sp.n1 > inner_size) ) { return "super-panel columns out of range" + at; }
            if( sp.row0 < 0 || sp.row0 + sp.n0 > sym.n ) { return "super-panel rows out of the matrix" + at; }
            if( sp.ldt != kPanel * ((sp.rows + kPanel - 1) / kPanel) ) { return "super-panel inverse edge" + at; }
            if( sp.t < 0 || sp.t + static_cast<I64>( sp.ldt ) * sp.ldt > pl.super_inv_size ) { return "super-panel inverse out of range" + at; }
            nblk[static_cast<size_t>( p )] = (sp.rows + kPanel - 1) / kPanel;
            nrest[static_cast<size_t>( p )] = (sp.n0 - sp.r0 - sp.rows) + sp.n1;
            for( I32 b = 0; b < kSuperPanels; ++b )
            {
                if( b < nblk[static_cast<size_t>( p )] )
                {
                    const I32 q = sp.panel[b];
                    if( q < 0 || q >= static_cast<I32>( pl.sdiag.size() ) ) { return "super-panel panel out of range" + at; }
                    const SolveDiagTask & d = pl.sdiag[static_cast<size_t>( q )];
                    if( d.u0 != sp.u0 || d.r0 != sp.r0 + b * kPanel || d.n0 != sp.n0 ) { return "super-panel panel mismatch" + at; }
                }
                else if( sp.panel[b] != -1 ) { return "super-panel panel beyond its rows" + at; }
            }
        }
        for( size_t t = 0; t < pl.sinv.size(); ++t )
        {
            const SuperInvTask & v = pl.sinv[t];
            if( v.sp < 0 || v.sp >= nsp || v.i < 0 || v.j < v.i || v.j >= nblk[static_cast<size_t>( v.sp )] ) { return "super-panel inverse task out of range"; }
        }
        for( const Launch & L : pl.sinv_launches )
        {
            if( L.kind != LaunchKind::SuperInv || L.count <= 0 || L.first < 0 || L.first + L.count > static_cast<I64>( pl.sinv.size() ) )
            {
                return "super-panel inverse launch out of bounds";
            }
            for( I64 t = L.first; t < L.first + L.count; ++t ) { if( pl.sinv[static_cast<size_t>( t )].j - pl.sinv[static_cast<size_t>( t )].i != L.step ) { return "super-panel inverse round mismatch"; } }
        }
        // each sweep: every other front's tasks once, every super-panel's diag blocks and rest rows once
        for( const std::vector<Launch> * list : { &pl.lower_launches_sp, &pl.upper_launches_sp } )
        {
            const bool forward = list == &pl.lower_launches_sp;
            I64 regular = 0;
            std::vector<I64> diag( static_cast<size_t>( nsp ), 0 ), rest( static_cast<size_t>( nsp ), 0 );
            for( const Launch & L : *list )
            {
                if( L.kind == LaunchKind::Solve )
                {
                    if( L.count <= 0 || L.first < 0 || L.first + L.count > static_cast<I64>( pl.srest.size() ) ) { return "super solve list: step launch out of bounds"; }
                    for( I64 t = L.first; t < L.first + L.count; ++t ) { if( pl.srest[static_cast<size_t>( t )].n0 >= kSuperMinRows ) { return "super solve list: a large front's panel step"; } }
                    regular += L.count;
                    continue;
                }
                if( (L.kind != LaunchKind::SuperDiag && L.kind != LaunchKind::SuperRest) || L.count <= 0 || L.first < 0
                    || L.first + L.count > static_cast<I64>( pl.ssolve.size() ) )
                {
                    return "super solve list: launch out of bounds";
                }
                for( I64 t = L.first; t < L.first + L.count; ++t )
                {
                    const SuperSolveTask & v = pl.ssolve[static_cast<size_t>( t )];
                    if( v.sp < 0 || v.sp >= nsp ) { return "super solve task out of range"; }
                    const size_t p = static_cast<size_t>( v.sp );
                    if( v.blk < 0 || v.blk >= nblk[p] ) { return "super solve block out of range"; }
                    if( L.kind == LaunchKind::SuperDiag )
                    {
                        // block pair (blk, c0): forward c0 <= blk, back c0 >= blk
                        if( v.c0 < 0 || v.c0 >= nblk[p] || (forward ? v.c0 > v.blk : v.c0 < v.blk) ) { return "super solve diag pair out of range"; }
                        ++diag[p];
                    }
                    else
                    {
                        if( v.c0 < 0 || v.c1 > nrest[p] || v.c0 >= v.c1 || v.c1 - v.c0 > kSolveRest ) { return "super solve rest rows out of range"; }
                        rest[p] += v.c1 - v.c0;
                    }
                }
            }
            I64 small = 0;
            for( const SolveRestTask & t : pl.srest ) { small += t.n0 >= kSuperMinRows ? 0 : 1; }
            if( regular != small ) { return "super solve list: the other fronts' steps are not covered once"; }
            for( I64 p = 0; p < nsp; ++p )
            {
                const I64 nb = nblk[static_cast<size_t>( p )];
                if( diag[static_cast<size_t>( p )] != nb * (nb + 1) / 2 || rest[static_cast<size_t>( p )] != nb * nrest[static_cast<size_t>( p )] )
                {
                    return "super solve list: super-panel " + std::to_string( p ) + " not covered once";
                }
            }
        }
    }
    {
        // solve task graph: sizes, ranges, and deadlock freedom: in the forward
        // list every task that updates a panel's rows comes before the panel's
        // first task; in the back list every task of a target panel comes
        // before the task that reads it
        const I64 nt = static_cast<I64>( pl.srest.size() ) - pl.solve_first_task;
        const I64 np = static_cast<I64>( pl.sdiag.size() ) - pl.solve_first_panel;
        if( static_cast<I64>( pl.solve_fwd_order.size() ) != (pl.solve_fwd_order.empty() ? 0 : nt)
            || pl.solve_bwd_order.size() != pl.solve_fwd_order.size() )
        {
            return "solve graph order sizes";
        }
        if( !pl.solve_fwd_order.empty() )
        {
            if( static_cast<I64>( pl.solve_target_ptr.size() ) != nt + 1 || static_cast<I64>( pl.solve_fwd_expected.size() ) != np
                || static_cast<I64>( pl.solve_panel_tasks.size() ) != np )
            {
                return "solve graph array sizes";
            }
            auto check_order = [&]( const std::vector<I32> & order, bool upper ) -> std::string
            {
                std::vector<I64> done( static_cast<size_t>( np ), 0 );       // forward: updates in; back: tasks done
                std::vector<char> seen( static_cast<size_t>( nt ), 0 );
                for( size_t pos = 0; pos < order.size(); ++pos )
                {
                    const I64 g = static_cast<I64>( order[pos] ) - pl.solve_first_task;
                    if( g < 0 || g >= nt || seen[static_cast<size_t>(g)] ) { return "solve graph order is not a permutation"; }
                    seen[static_cast<size_t>(g)] = 1;
                    const I64 p = pl.srest[static_cast<size_t>( order[pos] )].panel - pl.solve_first_panel;
                    if( p < 0 || p >= np ) { return "solve graph panel out of range"; }
                    for( I64 e = pl.solve_target_ptr[static_cast<size_t>(g)]; e < pl.solve_target_ptr[static_cast<size_t>(g) + 1]; ++e )
                    {
                        const I32 q = pl.solve_targets[static_cast<size_t>(e)];
                        if( q < 0 || q >= np ) { return "solve graph target out of range"; }
                        if( upper && done[static_cast<size_t>(q)] != pl.solve_panel_tasks[static_cast<size_t>(q)] )
                        {
                            return "back-solve task at list position " + std::to_string( pos ) + " reads an unfinished panel";
                        }
                    }
                    if( !upper && done[static_cast<size_t>(p)] != pl.solve_fwd_expected[static_cast<size_t>(p)] )
                    {
                        return "forward-solve task at list position " + std::to_string( pos ) + " starts before its updates";
                    }
                    if( upper ) { ++done[static_cast<size_t>(p)]; }
                    else
                    {
                        for( I64 e = pl.solve_target_ptr[static_cast<size_t>(g)]; e < pl.solve_target_ptr[static_cast<size_t>(g) + 1]; ++e )
                        {
                            ++done[static_cast<size_t>( pl.solve_targets[static_cast<size_t>(e)] )];
                        }
                    }
                }
                return std::string();
            };
            std::string m = check_order( pl.solve_fwd_order, false );
            if( !m.empty() ) { return m; }
            m = check_order( pl.solve_bwd_order, true );
            if( !m.empty() ) { return m; }
        }
    }
    return std::string();
}

} // namespace tb
