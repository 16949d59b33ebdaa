// Host-side symbolic analysis; see symbolic.hpp.
//
// Each step states the reference behaviour it reproduces (file:line in
// HenrikSchumacher/Tensors).  The data structures are this library's own:
// flat vectors, a per-row sort with a parallel row split, and a single
// supernode sweep parameterised by the merge rule.

#include "symbolic.hpp"
#include "trace.hpp"
#include "parallel.hpp"
#include "common.hpp"

#include <algorithm>
#include <atomic>
#include <numeric>
#include <thread>

namespace tb
{
namespace
{

using I32 = std::int32_t;
using I64 = std::int64_t;

// Sorted union of two strictly increasing runs (UniteSortedBuffers.hpp:6).
void sorted_union( const std::vector<I32> & a, const I32 * b, I64 nb, std::vector<I32> & out )
{
    out.clear();
    out.reserve( a.size() + static_cast<size_t>(nb) );
    std::set_union( a.begin(), a.end(), b, b + nb, std::back_inserter( out ) );
}

} // namespace

// Row i of the result is row rows[i] of the current pattern with every column
// c renamed cols_inv[c]; rows come out sorted and moved_from[k] names the old
// slot of new slot k (Permutation.hpp:828-930).
void Symbolic::permute_pattern( const std::vector<I32> & rows, const std::vector<I32> & cols_inv,
                                std::vector<I64> & moved_from )
{
    std::vector<I64> new_outer( static_cast<size_t>(n) + 1, 0 );
    for( I32 i = 0; i < n; ++i ) { new_outer[i+1] = new_outer[i] + (outer[rows[i]+1] - outer[rows[i]]); }
    std::vector<I32> new_inner( static_cast<size_t>(nnz) );
    moved_from.assign( static_cast<size_t>(nnz), 0 );
    parallel_rows( n, [&]( I64 b, I64 e )
    {
        // one 64-bit key per entry: new column (high word), slot within the old row (low word)
        std::vector<std::uint64_t> buf;
        for( I64 i = b; i < e; ++i )
        {
            const I64 src = outer[rows[i]];
            const I64 len = new_outer[i+1] - new_outer[i];
            buf.resize( static_cast<size_t>(len) );
            for( I64 k = 0; k < len; ++k )
            {
                buf[k] = (static_cast<std::uint64_t>( static_cast<std::uint32_t>( cols_inv[inner[src+k]] ) ) << 32) | static_cast<std::uint64_t>( k );
            }
            std::sort( buf.begin(), buf.end() );
            for( I64 k = 0; k < len; ++k )
            {
                new_inner [new_outer[i] + k] = static_cast<I32>( buf[k] >> 32 );
                moved_from[new_outer[i] + k] = src + static_cast<I64>( buf[k] & 0xffffffffu );
            }
        }
    }, threads_ );
    outer.swap( new_outer );
    inner.swap( new_inner );
}

// PatternCSR.hpp:408-445: position of the first entry of each row whose
// column is not left of the diagonal.
void Symbolic::locate_diagonal()
{
    diag.resize( static_cast<size_t>(n) );
    parallel_rows( n, [&]( I64 b, I64 e )
    {
        for( I64 i = b; i < e; ++i )
        {
            const I32 * first = inner.data() + outer[i];
            const I32 * last  = inner.data() + outer[i+1];
            diag[i] = outer[i] + ( std::lower_bound( first, last, static_cast<I32>(i) ) - first );
        }
    }, threads_ );
}

// Liu's elimination-tree algorithm with path compression over the full
// pattern (EliminationTreeParents.hpp:8-63); n marks a root.
//
// On several host threads the rows split into contiguous chunks.  Each chunk
// runs Liu's algorithm on its own rows and columns alone (its entries left of
// the chunk are set aside), which gives the elimination forest of the chunk's
// diagonal block.  A serial pass then runs Liu's algorithm once more over a
// smaller graph: every chunk forest's edges plus the set-aside entries.  For
// every k the vertices 0..k split into the same connected components in both
// graphs (the chunk forest restricted to a chunk's first rows spans the
// components of its diagonal block restricted to those rows), and the
// elimination tree depends on nothing else, so the tree is the same.
void Symbolic::elimination_tree()
{
    etree_parent.assign( static_cast<size_t>(n), n );
    std::vector<I32> ancestor( static_cast<size_t>(n), n );
    // row k's entries left of k, from column `from` on
    auto liu_rows = [&]( I32 kb, I32 ke, I32 from, std::vector<std::pair<I32,I32>> * aside )
    {
        for( I32 k = std::max( kb, 1 ); k < ke; ++k )
        {
            for( I64 l = outer[k]; l < outer[k+1]; ++l )
            {
                I32 i = inner[l];
                if( i >= k ) { break; }
                if( i < from ) { aside->emplace_back( k, i ); continue; }
                while( i != n && i < k )
                {
                    const I32 next = ancestor[i];
                    ancestor[i] = k;
                    if( next == n ) { etree_parent[i] = k; }
                    i = next;
                }
            }
        }
    };
    const I64 chunks = std::min<I64>( host_threads( threads_ ), std::max<I64>( 1, n / 65536 ) );
    if( chunks <= 1 ) { liu_rows( 0, n, 0, nullptr ); return; }

    std::vector<std::vector<std::pair<I32,I32>>> aside( static_cast<size_t>(chunks) );
    {
        std::vector<std::thread> pool;
        for( I64 t = 0; t < chunks; ++t )
        {
            const I32 b = static_cast<I32>( n * t / chunks ), e = static_cast<I32>( n * (t + 1) / chunks );
            pool.emplace_back( [&, t, b, e]() { liu_rows( b, e, b, &aside[static_cast<size_t>(t)] ); } );
        }
        for( auto & th : pool ) { th.join(); }
    }
    // the chunk forests' edges, by parent
    std::vector<I32> child_ptr( static_cast<size_t>(n) + 2, 0 ), child_idx;
    for( I32 i = 0; i < n; ++i ) { ++child_ptr[static_cast<size_t>( etree_parent[i] ) + 1]; }
    std::partial_sum( child_ptr.begin(), child_ptr.end(), child_ptr.begin() );
    child_idx.resize( static_cast<size_t>( child_ptr[static_cast<size_t>(n)] ) );
    {
        std::vector<I32> next( child_ptr.begin(), child_ptr.end() - 1 );
        for( I32 i = 0; i < n; ++i ) { if( etree_parent[i] < n ) { child_idx[static_cast<size_t>( next[etree_parent[i]]++ )] = i; } }
    }
    etree_parent.assign( static_cast<size_t>(n), n );
    ancestor.assign( static_cast<size_t>(n), n );
    auto climb = [&]( I32 i, I32 k )
    {
        while( i != n && i < k )
        {
            const I32 next = ancestor[i];
            ancestor[i] = k;
            if( next == n ) { etree_parent[i] = k; }
            i = next;
        }
    };
    for( I64 t = 0; t < chunks; ++t )
    {
        const I32 b = static_cast<I32>( n * t / chunks ), e = static_cast<I32>( n * (t + 1) / chunks );
        const auto & side = aside[static_cast<size_t>(t)];
        size_t q = 0;
        for( I32 k = b; k < e; ++k )
        {
            for( I32 c = child_ptr[k]; c < child_ptr[k+1]; ++c ) { climb( child_idx[static_cast<size_t>(c)], k ); }
            for( ; q < side.size() && side[q].first == k; ++q ) { climb( side[q].second, k ); }
        }
    }
}

// Child lists (ascending, as the reference's pair-assembled adjacency matrix,
// PatternCSR/FromPairs.hpp), descendant counts and -- optionally -- the
// postorder of the iterative DFS of Tree/Traverse_PostOrdered_Sequential.hpp
// (children pushed in reverse so the smallest is finished first), with the
// virtual root `parent.size()` omitted (Tree/Init.hpp:92-97).
void Symbolic::forest_of( const std::vector<I32> & parent, Forest & f, bool with_order )
{
    const I32 count = static_cast<I32>(parent.size());
    f.child_ptr.assign( static_cast<size_t>(count) + 2, 0 );
    for( I32 i = 0; i < count; ++i ) { ++f.child_ptr[parent[i]+1]; }
    std::partial_sum( f.child_ptr.begin(), f.child_ptr.end(), f.child_ptr.begin() );
    f.child_idx.resize( static_cast<size_t>(count) );
    {
        std::vector<I32> next( f.child_ptr.begin(), f.child_ptr.end() - 1 );
        for( I32 i = 0; i < count; ++i ) { f.child_idx[next[parent[i]]++] = i; }
    }
    // Children precede parents in every tree built here (parent > child), so
    // descendant counts accumulate in one ascending pass.
    f.desc.assign( static_cast<size_t>(count) + 1, 0 );
    for( I32 i = 0; i < count; ++i ) { f.desc[parent[i]] += f.desc[i] + 1; }
    f.postorder.clear();
    if( !with_order ) { return; }
    f.postorder.reserve( static_cast<size_t>(count) );
    struct Frame { I32 node; I32 next_child; };
    std::vector<Frame> stack;
    stack.push_back( { count, f.child_ptr[count] } );
    while( !stack.empty() )
    {
        Frame & fr = stack.back();
        if( fr.next_child < f.child_ptr[fr.node+1] )
        {
            const I32 c = f.child_idx[fr.next_child++];
            stack.push_back( { c, f.child_ptr[c] } );
        }
        else
        {
            if( fr.node != count ) { f.postorder.push_back( fr.node ); }
            stack.pop_back();
        }
    }
}

// Tree.hpp:264-286: every vertex precedes its parent and the parent's
// descendant block contains the vertex's.
bool Symbolic::postordered( const std::vector<I32> & parent, const std::vector<I32> & desc )
{
    const I32 count = static_cast<I32>(parent.size());
    for( I32 i = 0; i < count; ++i )
    {
        const I32 p_ = parent[i];
        if( !(i < p_) ) { return false; }
        if( static_cast<I64>(i) + desc[p_] < static_cast<I64>(p_) + desc[i] ) { return false; }
    }
    return true;
}

// One sweep over rows 1..n (Symbolic.hpp:71-588).  A row that starts a new
// fundamental supernode (FundamentalQ, Symbolic.hpp:590-622) closes the
// current one: its column set is the part of its first row's upper pattern at
// or beyond the closing row, united with the column sets of the first row's
// elimination-tree children (restricted to the same range).  The merge rule
// then decides whether the closed supernode joins its predecessor.
//
// Whether row i starts a supernode depends only on the pattern and the tree, so
// it is decided for all rows first, in parallel: row i (1 <= i < n) starts one
// if it has more than one child, or if some column j of its upper pattern was
// last seen, among the rows before i that record their columns (rows 1.. with
// at most one child; the sweep's early exit skips the others), before i's
// subtree.  The rows with column j in their upper pattern are the entries of
// row j's lower pattern (the pattern is symmetric), so one ascending pass over
// every row's lower pattern visits each (recording row, column) pair with the
// recording row before it; the flags it sets are only ever set to 1.
void Symbolic::supernode_starts( const Forest & et, std::vector<std::uint8_t> & fresh ) const
{
    fresh.assign( static_cast<size_t>(n) + 1, 0 );
    auto records = [&]( I32 r ) { return r >= 1 && et.child_ptr[r+1] - et.child_ptr[r] <= 1; };
    for( I32 i = 0; i < n; ++i ) { if( !records( i ) ) { fresh[static_cast<size_t>(i)] = 1; } }
    fresh[static_cast<size_t>(n)] = 1;
    std::uint8_t * flag = fresh.data();
    parallel_rows( n, [&]( I64 b, I64 e )
    {
        for( I64 j = b; j < e; ++j )
        {
            I32 last = -1;
            for( I64 k = outer[j]; k < diag[j]; ++k )
            {
                const I32 i = inner[k];
                if( !records( i ) ) { continue; }
                if( last < i - et.desc[i] + 1 ) { __atomic_store_n( flag + i, std::uint8_t(1), __ATOMIC_RELAXED ); }
                last = i;
            }
        }
    }, threads_ );
}

void Symbolic::supernodes( SupernodeStrategy strategy, I32 threshold, const Forest & et )
{
    std::vector<std::uint8_t> fresh;
    {
        TraceRange range( "tensors_b200::SupernodeStarts" );
        supernode_starts( et, fresh );
    }
    row_to_sn.assign( static_cast<size_t>(n), 0 );
    sn_rp.assign( 1, 0 );
    sn_outer.assign( 1, 0 );
    sn_inner.clear();

    std::vector<I32> cols, merged;
    I32 count = 0;        // closed supernodes so far
    I32 first = 0;        // first row of the open supernode
    I32 prev_rows = 0, prev_cols = 0;

    auto starts_supernode = [&]( I32 i ) -> bool { return fresh[static_cast<size_t>(i)] != 0; };

    // Trailing part (columns >= bound) of closed supernode k's column set.
    auto tail_of = [&]( I32 k, I32 bound ) -> std::pair<I64,I64>
    {
        const I64 b = sn_outer[k], e = sn_outer[k+1];
        const I64 a = std::lower_bound( sn_inner.begin() + b, sn_inner.begin() + e, bound ) - sn_inner.begin();
        return { a, e };
    };

    for( I32 i = 1; i <= n; ++i )
    {
        if( starts_supernode( i ) )
        {
            I32 rows = i - first;
            {
                const I64 kb = diag[first] + 1, ke = outer[first+1];
                const I64 a = std::lower_bound( inner.begin() + kb, inner.begin() + ke, i ) - inner.begin();
                cols.assign( inner.begin() + a, inner.begin() + ke );
            }
            for( I32 c = et.child_ptr[first]; c < et.child_ptr[first+1]; ++c )
            {
                const I32 k = row_to_sn[ et.child_idx[c] ];
                if( k == count ) { continue; }
                const auto [a, e] = tail_of( k, i );
                if( a < e ) { sorted_union( cols, sn_inner.data() + a, e - a, merged ); cols.swap( merged ); }
            }

            bool join = false;
            if( count > 0 && strategy == SupernodeStrategy::Maximal )
            {
                const auto [a, e] = tail_of( count - 1, i );
                join = !cols.empty() && ( e - a == static_cast<I64>(cols.size()) )
                       && std::equal( cols.begin(), cols.end(), sn_inner.begin() + a );
            }
            else if( count > 0 && strategy == SupernodeStrategy::Amalgamated && rows + prev_rows <= threshold )
            {
                const auto [a, e] = tail_of( count - 1, i );
                if( a < e ) { sorted_union( cols, sn_inner.data() + a, e - a, merged ); cols.swap( merged ); }
                join = true;
            }
            if( join )
            {
                --count;
                sn_rp.pop_back();
                sn_outer.pop_back();
                sn_inner.resize( sn_inner.size() - static_cast<size_t>(prev_cols) );
                for( I32 r = i - rows; r < i; ++r ) { row_to_sn[r] = count; }
                rows += prev_rows;
            }
            sn_inner.insert( sn_inner.end(), cols.begin(), cols.end() );
            ++count;
            sn_outer.push_back( static_cast<I64>(sn_inner.size()) );
            sn_rp.push_back( i );
            first = i;
            prev_rows = rows;
            prev_cols = static_cast<I32>(cols.size());
        }
        if( i < n ) { row_to_sn[i] = count; }
    }
    sn_count = count;
}

// Symbolic.hpp:36-60 and AssemblyTree.hpp:12-61: value pointers over full
// squares and rectangles; a supernode's parent owns the elimination-tree
// parent of its last row (the last supernode is always a root).
void Symbolic::assembly_tree()
{
    sn_tri_ptr.assign( static_cast<size_t>(sn_count) + 1, 0 );
    sn_rec_ptr.assign( static_cast<size_t>(sn_count) + 1, 0 );
    max_n0 = max_n1 = 0;
    for( I32 s = 0; s < sn_count; ++s )
    {
        max_n0 = std::max( max_n0, n0(s) );
        max_n1 = std::max( max_n1, n1(s) );
        sn_tri_ptr[s+1] = sn_tri_ptr[s] + static_cast<I64>(n0(s)) * n0(s);
        sn_rec_ptr[s+1] = sn_rec_ptr[s] + static_cast<I64>(n0(s)) * n1(s);
    }
    atree_parent.assign( static_cast<size_t>(sn_count), sn_count );
    for( I32 s = 0; s + 1 < sn_count; ++s )
    {
        const I32 up = etree_parent[ sn_rp[s+1] - 1 ];
        atree_parent[s] = up < n ? row_to_sn[up] : sn_count;
    }
    Forest f;
    forest_of( atree_parent, f, false );
    atree_child_ptr.assign( f.child_ptr.begin(), f.child_ptr.end() );
    atree_child_idx.swap( f.child_idx );
}

int Symbolic::analyze( const SymbolicInput & in )
{
    n = in.n;
    threads_ = in.threads;
    if( n <= 0 || in.outer == nullptr || in.inner == nullptr ) { return TB_ERR_INVALID_ARGUMENT; }
    nnz = in.outer[n];
    if( in.outer[0] != 0 || nnz < n ) { return TB_ERR_INVALID_PATTERN; }
    outer.assign( in.outer, in.outer + n + 1 );
    for( I32 i = 0; i < n; ++i ) { if( outer[i+1] < outer[i] ) { return TB_ERR_INVALID_PATTERN; } }
    inner.resize( static_cast<size_t>(nnz) );
    // Rows must be sorted unless a permutation is given, in which case the
    // permuted pattern is sorted here (as the reference's Permute does).
    std::atomic<bool> bad{ false };
    parallel_rows( n, [&]( I64 b, I64 e )
    {
        std::copy( in.inner + outer[b], in.inner + outer[e], inner.begin() + outer[b] );
        for( I64 i = b; i < e && !bad.load( std::memory_order_relaxed ); ++i )
        {
            for( I64 k = outer[i]; k < outer[i+1]; ++k )
            {
                if( inner[k] < 0 || inner[k] >= n || (in.perm == nullptr && k > outer[i] && inner[k] <= inner[k-1]) )
                {
                    bad.store( true );
                    break;
                }
            }
        }
    }, threads_ );
    if( bad.load() ) { return TB_ERR_INVALID_PATTERN; }

    p.resize( static_cast<size_t>(n) );
    p_inv.assign( static_cast<size_t>(n), -1 );
    if( in.perm != nullptr )
    {
        TraceRange range( "Sparse::CholeskyDecomposition::Init" );
        for( I32 i = 0; i < n; ++i )
        {
            const I32 v = in.perm[i];
            if( v < 0 || v >= n || p_inv[v] != -1 ) { return TB_ERR_INVALID_PERMUTATION; }
            p[i] = v;
            p_inv[v] = i;
        }
        permute_pattern( p, p_inv, value_perm );         // CholeskyDecomposition.hpp:313-331
        parallel_rows( n, [&]( I64 b, I64 e )             // duplicates are not a CSR pattern
        {
            for( I64 i = b; i < e && !bad.load( std::memory_order_relaxed ); ++i )
            {
                for( I64 k = outer[i] + 1; k < outer[i+1]; ++k )
                {
                    if( inner[k] == inner[k-1] ) { bad.store( true ); break; }
                }
            }
        }, threads_ );
        if( bad.load() ) { return TB_ERR_INVALID_PATTERN; }
    }
    else
    {
        std::iota( p.begin(), p.end(), 0 );               // CholeskyDecomposition.hpp:350-371
        std::iota( p_inv.begin(), p_inv.end(), 0 );
        value_perm.resize( static_cast<size_t>(nnz) );
        std::iota( value_perm.begin(), value_perm.end(), I64(0) );
    }
    locate_diagonal();
    for( I32 i = 0; i < n; ++i )                          // CholeskyDecomposition.hpp:404-423
    {
        if( diag[i] >= outer[i+1] || inner[diag[i]] != i ) { return TB_ERR_MISSING_DIAGONAL; }
    }

    // CholeskyDecomposition.hpp:427-472: make the elimination tree postordered.
    {
        TraceRange range( "Sparse::CholeskyDecomposition::EliminationTree" );
        elimination_tree();
    }
    Forest et;
    forest_of( etree_parent, et, true );
    if( !postordered( etree_parent, et.desc ) )
    {
        TraceRange range( "Sparse::CholeskyDecomposition::PostOrdering" );
        const std::vector<I32> & post = et.postorder;
        std::vector<I32> post_inv( static_cast<size_t>(n) );
        for( I32 i = 0; i < n; ++i ) { post_inv[post[i]] = i; }
        std::vector<I32> np( static_cast<size_t>(n) );
        for( I32 i = 0; i < n; ++i ) { np[i] = p[post[i]]; }
        p.swap( np );
        for( I32 i = 0; i < n; ++i ) { p_inv[p[i]] = i; }
        std::vector<I64> moved;
        permute_pattern( post, post_inv, moved );
        for( auto & m : moved ) { m = value_perm[m]; }
        value_perm.swap( moved );
        locate_diagonal();
        elimination_tree();
        forest_of( etree_parent, et, false );
    }

    {
        TraceRange range( in.strategy == SupernodeStrategy::Fundamental ? "Sparse::CholeskyDecomposition::FindFundamentalSupernodes"
                        : in.strategy == SupernodeStrategy::Amalgamated ? "Sparse::CholeskyDecomposition::FindAmalgamatedSupernodes"
                                                                        : "Sparse::CholeskyDecomposition::FindMaximalSupernodes" );
        supernodes( in.strategy, in.amalgamation_threshold, et );
    }
    {
        TraceRange range( "Sparse::CholeskyDecomposition::CreateAssemblyTree" );
        assembly_tree();
    }
    return TB_OK;
}

} // namespace tb
