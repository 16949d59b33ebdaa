// Coordinate-free nested dissection of a sparse symmetric pattern (host).
//
// The reference takes its fill-reducing permutation from METIS or AMD
// (src/Sparse/Metis.hpp:81, src/Sparse/ApproximateMinimumDegree.hpp:58);
// neither is available, and the project's geometric dissection needs node
// coordinates that a matrix read from a file does not carry.  This ordering
// needs the pattern only.  It is George's automatic nested dissection
// (A. George, J. Liu, "Computer Solution of Large Sparse Positive Definite
// Systems", 1981, ch. 8) on the node graph:
//  * a subgraph that is not connected is split into its components;
//  * a connected subgraph is given a rooted level structure (breadth-first
//    levels) from a pseudo-peripheral node (the George-Liu search: restart
//    from a minimum-degree node of the last level while the eccentricity
//    grows);
//  * the separator is taken at the median level k: either the nodes of level
//    k with a neighbour in level k + 1, or the nodes of level k + 1 with a
//    neighbour in level k, whichever is smaller; the two sides are ordered
//    recursively, the separator last;
//  * subgraphs of at most leaf_size nodes are emitted in breadth-first order.
// The dofs of a node (rows d*u .. d*u + d - 1) stay together.

#include "common.hpp"

#include <algorithm>
#include <atomic>
#include <future>
#include <thread>
#include <cstdint>
#include <string>
#include <vector>

namespace
{
using I32 = std::int32_t;
using I64 = std::int64_t;

int fail( int code, const std::string & msg )
{
    tb::set_last_error( msg );
    return code;
}

struct Graph
{
    I32 n = 0;
    std::vector<I64> ptr;
    std::vector<I32> adj;
    I32 degree( I32 v ) const { return static_cast<I32>( ptr[static_cast<size_t>( v ) + 1] - ptr[static_cast<size_t>( v )] ); }
};

// Node graph of the pattern: u ~ v when some row of node u holds a column of
// node v (u != v), symmetrized and without repeats.
Graph node_graph( I32 n, const I64 * outer, const I32 * inner, I32 d )
{
    Graph g;
    g.n = n / d;
    const size_t N = static_cast<size_t>( g.n );
    // distinct neighbours named by each node's rows
    std::vector<I64> optr( N + 1, 0 );
    std::vector<I32> oadj;
    std::vector<I32> mark( N, -1 );
    for( I32 u = 0; u < g.n; ++u )
    {
        for( I32 j = 0; j < d; ++j )
        {
            const I32 r = u * d + j;
            for( I64 k = outer[r]; k < outer[r + 1]; ++k )
            {
                const I32 v = inner[k] / d;
                if( v != u && mark[static_cast<size_t>( v )] != u ) { mark[static_cast<size_t>( v )] = u; oadj.push_back( v ); }
            }
        }
        optr[static_cast<size_t>( u ) + 1] = static_cast<I64>( oadj.size() );
    }
    // union with the transpose, sorted, without repeats
    std::vector<I64> cnt( N + 1, 0 );
    for( I32 u = 0; u < g.n; ++u )
    {
        cnt[static_cast<size_t>( u ) + 1] += optr[static_cast<size_t>( u ) + 1] - optr[static_cast<size_t>( u )];
        for( I64 k = optr[static_cast<size_t>( u )]; k < optr[static_cast<size_t>( u ) + 1]; ++k ) { ++cnt[static_cast<size_t>( oadj[static_cast<size_t>( k )] ) + 1]; }
    }
    for( size_t u = 0; u < N; ++u ) { cnt[u + 1] += cnt[u]; }
    std::vector<I32> raw( static_cast<size_t>( cnt[N] ) );
    std::vector<I64> pos( cnt.begin(), cnt.end() - 1 );
    for( I32 u = 0; u < g.n; ++u )
    {
        for( I64 k = optr[static_cast<size_t>( u )]; k < optr[static_cast<size_t>( u ) + 1]; ++k )
        {
            const I32 v = oadj[static_cast<size_t>( k )];
            raw[static_cast<size_t>( pos[static_cast<size_t>( u )]++ )] = v;
            raw[static_cast<size_t>( pos[static_cast<size_t>( v )]++ )] = u;
        }
    }
    g.ptr.assign( N + 1, 0 );
    g.adj.reserve( oadj.size() );
    for( I32 u = 0; u < g.n; ++u )
    {
        auto b = raw.begin() + cnt[static_cast<size_t>( u )], e = raw.begin() + cnt[static_cast<size_t>( u ) + 1];
        std::sort( b, e );
        e = std::unique( b, e );
        g.adj.insert( g.adj.end(), b, e );
        g.ptr[static_cast<size_t>( u ) + 1] = static_cast<I64>( g.adj.size() );
    }
    return g;
}

class Dissection
{
public:
    Dissection( const Graph & g, I32 leaf ) : g_( g ), leaf_( std::max( 1, leaf ) ),
        owner_( static_cast<size_t>( g.n ) ), level_( static_cast<size_t>( g.n ), -1 ), slot_( static_cast<size_t>( g.n ), -1 ),
        key1_( static_cast<size_t>( g.n ), 0 ), key2_( static_cast<size_t>( g.n ), 0 )
    {
        for( auto & o : owner_ ) { o.store( -1, std::memory_order_relaxed ); }
    }

    // The whole graph: the top levels of the dissection tree on up to
    // `threads` threads (the two sides of a split are independent), the rest
    // depth-first on each thread.  The order does not depend on the threads.
    std::vector<I32> run( int threads )
    {
        std::vector<I32> all( static_cast<size_t>( g_.n ) );
        for( I32 v = 0; v < g_.n; ++v ) { all[static_cast<size_t>( v )] = v; }
        int depth = 0;
        while( (1 << depth) < threads ) { ++depth; }
        return order_parallel( std::move( all ), depth );
    }

private:
    // One dissection step on a node set: emit it whole (small or not
    // separable), its components, or (left, right, separator).
    struct Step { int kind = 0; std::vector<std::vector<I32>> parts; };

    Step step( std::vector<I32> nodes )
    {
        const I32 id = stamp_.fetch_add( 1 ) + 1;
        for( I32 v : nodes ) { set_owner( v, id ); }
        // components, each in breadth-first order from its first node
        std::vector<std::vector<I32>> comps;
        for( I32 v : nodes )
        {
            if( owner( v ) != id ) { continue; }     // already reached
            comps.push_back( bfs( v, id, -id - 1 ) );
        }
        Step st;
        if( comps.size() > 1 ) { st.kind = 1; st.parts = std::move( comps ); return st; }
        std::vector<I32> & S = comps[0];            // connected; owner now -id - 1
        std::vector<I32> left, sep, right;
        if( static_cast<I32>( S.size() ) <= leaf_ || !split( S, -id - 1, left, sep, right ) )
        {
            st.parts.push_back( std::move( S ) );
            return st;
        }
        st.kind = 2;
        st.parts.push_back( std::move( left ) );
        st.parts.push_back( std::move( right ) );
        st.parts.push_back( std::move( sep ) );
        return st;
    }

    // Depth-first with an explicit stack: components in turn, and per split
    // the left side, the right side, then the separator.
    std::vector<I32> run_serial( std::vector<I32> nodes )
    {
        std::vector<I32> order;
        order.reserve( nodes.size() );
        struct Item { std::vector<I32> nodes; bool emit; };
        std::vector<Item> stack;
        stack.push_back( { std::move( nodes ), false } );
        while( !stack.empty() )
        {
            Item it = std::move( stack.back() );
            stack.pop_back();
            if( it.emit ) { order.insert( order.end(), it.nodes.begin(), it.nodes.end() ); continue; }
            Step st = step( std::move( it.nodes ) );
            if( st.kind == 0 ) { order.insert( order.end(), st.parts[0].begin(), st.parts[0].end() ); continue; }
            if( st.kind == 1 )
            {
                for( size_t c = st.parts.size(); c-- > 0; ) { stack.push_back( { std::move( st.parts[c] ), false } ); }
                continue;
            }
            stack.push_back( { std::move( st.parts[2] ), true } );
            stack.push_back( { std::move( st.parts[1] ), false } );
            stack.push_back( { std::move( st.parts[0] ), false } );
        }
        return order;
    }

    // The same order, with the sides of the top `depth` splits on two threads.
    std::vector<I32> order_parallel( std::vector<I32> nodes, int depth )
    {
        if( depth <= 0 || nodes.size() < kParallelMin ) { return run_serial( std::move( nodes ) ); }
        Step st = step( std::move( nodes ) );
        if( st.kind == 0 ) { return std::move( st.parts[0] ); }
        std::vector<I32> order;
        if( st.kind == 1 )
        {
            for( auto & c : st.parts )
            {
                std::vector<I32> o = order_parallel( std::move( c ), depth );
                order.insert( order.end(), o.begin(), o.end() );
            }
            return order;
        }
        auto left = std::async( std::launch::async, [this, &st, depth] { return order_parallel( std::move( st.parts[0] ), depth - 1 ); } );
        std::vector<I32> right = order_parallel( std::move( st.parts[1] ), depth - 1 );
        order = left.get();
        order.insert( order.end(), right.begin(), right.end() );
        order.insert( order.end(), st.parts[2].begin(), st.parts[2].end() );
        return order;
    }

    // Set membership labels: read across sets by concurrent searches (a
    // neighbour may belong to another thread's set), so accessed atomically.
    I32 owner( I32 v ) const { return owner_[static_cast<size_t>( v )].load( std::memory_order_relaxed ); }
    void set_owner( I32 v, I32 x ) { owner_[static_cast<size_t>( v )].store( x, std::memory_order_relaxed ); }

    // Breadth-first search over nodes with owner_ == from, relabelling them
    // to `to` and recording their levels; returns the nodes in visit order.
    std::vector<I32> bfs( I32 root, I32 from, I32 to )
    {
        std::vector<I32> q{ root };
        set_owner( root, to );
        level_[static_cast<size_t>( root )] = 0;
        for( size_t h = 0; h < q.size(); ++h )
        {
            const I32 u = q[h];
            for( I64 k = g_.ptr[static_cast<size_t>( u )]; k < g_.ptr[static_cast<size_t>( u ) + 1]; ++k )
            {
                const I32 v = g_.adj[static_cast<size_t>( k )];
                if( owner( v ) != from ) { continue; }
                set_owner( v, to );
                level_[static_cast<size_t>( v )] = level_[static_cast<size_t>( u )] + 1;
                q.push_back( v );
            }
        }
        return q;
    }

    // Level structure of the connected set S (owner sid) from `root`; the
    // owner marks are restored to sid afterwards.  Returns the depth.
    I32 levels_from( const std::vector<I32> & S, I32 sid, I32 root, std::vector<I32> & visit )
    {
        const I32 tmp = tmp_stamp_.fetch_sub( 1 ) - 1;
        visit = bfs( root, sid, tmp );
        for( I32 v : S ) { set_owner( v, sid ); }
        return level_[static_cast<size_t>( visit.back() )];
    }

    bool split( const std::vector<I32> & S, I32 sid, std::vector<I32> & left, std::vector<I32> & sep, std::vector<I32> & right )
    {
        // pseudo-peripheral root (George-Liu)
        std::vector<I32> visit;
        I32 root = S[0];
        I32 depth = levels_from( S, sid, root, visit );
        for( int tries = 0; tries < 8; ++tries )
        {
            const I32 best = far_node( visit, depth );
            std::vector<I32> visit2;
            const I32 depth2 = levels_from( S, sid, best, visit2 );
            if( depth2 <= depth ) { levels_from( S, sid, root, visit ); break; }
            root = best; depth = depth2; visit.swap( visit2 );
        }
        if( depth < 2 ) { return false; }
        // two keys per node: the level d1 from the root, and d1 - d2 with d2 the
        // level from a far node (cuts across the middle of the pseudo-diameter);
        // neighbours' keys differ by at most 1 and 2
        for( I32 v : S ) { key1_[static_cast<size_t>( v )] = level_[static_cast<size_t>( v )]; }
        std::vector<I32> visit2;
        levels_from( S, sid, far_node( visit, depth ), visit2 );
        for( I32 v : S ) { key2_[static_cast<size_t>( v )] = key1_[static_cast<size_t>( v )] - level_[static_cast<size_t>( v )] + depth; }
        // per key: buckets of nodes; candidate cuts (key <= c on the left) with
        // 40-60% of the nodes on each side, within 4 of the median cut
        struct Best { int which = -1; I32 c = 0; std::vector<I32> cover; };
        Best best;
        for( int which = 0; which < 2; ++which )
        {
            const std::vector<I32> & key = which == 0 ? key1_ : key2_;
            const I32 kmax = which == 0 ? depth : 2 * depth;
            std::vector<std::vector<I32>> bucket( static_cast<size_t>( kmax ) + 1 );
            for( I32 v : visit ) { bucket[static_cast<size_t>( key[static_cast<size_t>( v )] )].push_back( v ); }
            std::vector<I64> upto( static_cast<size_t>( kmax ) + 1, 0 );
            I64 acc = 0;
            for( I32 c = 0; c <= kmax; ++c ) { acc += static_cast<I64>( bucket[static_cast<size_t>( c )].size() ); upto[static_cast<size_t>( c )] = acc; }
            const I64 total = acc;
            I32 median = 0;
            while( median < kmax - 1 && 2 * upto[static_cast<size_t>( median )] < total ) { ++median; }
            for( I32 c = std::max( 0, median - 2 ); c <= std::min( kmax - 1, median + 2 ); ++c )
            {
                const I64 lo = upto[static_cast<size_t>( c )];
                if( lo == 0 || lo == total ) { continue; }
                if( c != median && !(5 * lo >= 2 * total && 5 * lo <= 3 * total) ) { continue; }
                std::vector<I32> cover = min_cover( bucket, key, c, sid );
                if( best.which < 0 || cover.size() < best.cover.size() ) { best.which = which; best.c = c; best.cover.swap( cover ); }
            }
        }
        if( best.which < 0 || best.cover.empty() ) { return false; }
        const std::vector<I32> & key = best.which == 0 ? key1_ : key2_;
        const I32 tag = tmp_stamp_.fetch_sub( 1 ) - 1;
        for( I32 v : best.cover ) { level_[static_cast<size_t>( v )] = tag; }    // level_ is free again: mark the cover
        for( I32 v : visit )                        // breadth-first order from the root
        {
            if( level_[static_cast<size_t>( v )] == tag ) { sep.push_back( v ); }
            else if( key[static_cast<size_t>( v )] <= best.c ) { left.push_back( v ); }
            else { right.push_back( v ); }
        }
        return !sep.empty() && !left.empty() && !right.empty();
    }

    // A minimum-degree node of the last level of a level structure.
    I32 far_node( const std::vector<I32> & visit, I32 depth ) const
    {
        I32 best = -1;
        for( size_t i = visit.size(); i-- > 0; )
        {
            const I32 v = visit[i];
            if( level_[static_cast<size_t>( v )] != depth ) { break; }
            if( best < 0 || g_.degree( v ) < g_.degree( best ) ) { best = v; }
        }
        return best;
    }

    // Minimum vertex cover of the edges that cross the cut key <= c | key > c
    // inside the set sid: a maximum matching of the bipartite cut graph by
    // augmenting paths, then Koenig's construction (the unmatched left ends
    // and what alternating paths reach from them; the cover is the left ends
    // not reached plus the right ends reached).  A vertex separator of the cut.
    std::vector<I32> min_cover( const std::vector<std::vector<I32>> & bucket, const std::vector<I32> & key, I32 c, I32 sid )
    {
        const I32 kmax = static_cast<I32>( bucket.size() ) - 1;
        auto crosses = [&]( I32 v, bool from_left ) {
            for( I64 e = g_.ptr[static_cast<size_t>( v )]; e < g_.ptr[static_cast<size_t>( v ) + 1]; ++e )
            {
                const I32 w = g_.adj[static_cast<size_t>( e )];
                if( owner( w ) != sid ) { continue; }
                if( from_left ? key[static_cast<size_t>( w )] > c : key[static_cast<size_t>( w )] <= c ) { return true; }
            }
            return false;
        };
        std::vector<I32> A, B;                        // left and right ends of cut edges
        for( I32 b = std::max( 0, c - 1 ); b <= c; ++b )
        {
            for( I32 v : bucket[static_cast<size_t>( b )] ) { if( crosses( v, true ) ) { A.push_back( v ); } }
        }
        for( I32 b = c + 1; b <= std::min( kmax, c + 2 ); ++b )
        {
            for( I32 v : bucket[static_cast<size_t>( b )] )
            {
                if( crosses( v, false ) ) { slot_[static_cast<size_t>( v )] = static_cast<I32>( B.size() ); B.push_back( v ); }
            }
        }
        const size_t na = A.size(), nb = B.size();
        std::vector<std::vector<I32>> nbr( na );       // A[i] -> indices into B
        for( size_t i = 0; i < na; ++i )
        {
            const I32 u = A[i];
            for( I64 e = g_.ptr[static_cast<size_t>( u )]; e < g_.ptr[static_cast<size_t>( u ) + 1]; ++e )
            {
                const I32 w = g_.adj[static_cast<size_t>( e )];
                if( owner( w ) == sid && key[static_cast<size_t>( w )] > c ) { nbr[i].push_back( slot_[static_cast<size_t>( w )] ); }
            }
        }
        std::vector<I32> match_a( na, -1 ), match_b( nb, -1 ), seen( nb, -1 );
        // augmenting paths (Kuhn), iterative depth-first search
        std::vector<std::pair<I32, size_t>> path;
        for( size_t i0 = 0; i0 < na; ++i0 )
        {
            path.assign( 1, { static_cast<I32>( i0 ), 0 } );
            bool found = false;
            while( !path.empty() && !found )
            {
                auto & top = path.back();
                const auto & adj = nbr[static_cast<size_t>( top.first )];
                if( top.second == adj.size() ) { path.pop_back(); continue; }
                const I32 j = adj[top.second++];
                if( seen[static_cast<size_t>( j )] == static_cast<I32>( i0 ) ) { continue; }
                seen[static_cast<size_t>( j )] = static_cast<I32>( i0 );
                if( match_b[static_cast<size_t>( j )] < 0 )
                {
                    // flip the path: each left node on it takes the right node it stepped to
                    I32 jj = j;
                    for( size_t p = path.size(); p-- > 0; )
                    {
                        const I32 ii = path[p].first;
                        const I32 prev = match_a[static_cast<size_t>( ii )];
                        match_a[static_cast<size_t>( ii )] = jj;
                        match_b[static_cast<size_t>( jj )] = ii;
                        jj = prev;
                    }
                    found = true;
                }
                else
                {
                    path.push_back( { match_b[static_cast<size_t>( j )], 0 } );
                }
            }
        }
        // Koenig: alternating reachability from the unmatched left ends
        std::vector<char> za( na, 0 ), zb( nb, 0 );
        std::vector<I32> q;
        for( size_t i = 0; i < na; ++i ) { if( match_a[i] < 0 ) { za[i] = 1; q.push_back( static_cast<I32>( i ) ); } }
        for( size_t h = 0; h < q.size(); ++h )
        {
            for( I32 j : nbr[static_cast<size_t>( q[h] )] )
            {
                if( zb[static_cast<size_t>( j )] ) { continue; }
                zb[static_cast<size_t>( j )] = 1;
                const I32 i = match_b[static_cast<size_t>( j )];
                if( i >= 0 && !za[static_cast<size_t>( i )] ) { za[static_cast<size_t>( i )] = 1; q.push_back( i ); }
            }
        }
        std::vector<I32> cover;
        for( size_t i = 0; i < na; ++i ) { if( !za[i] ) { cover.push_back( A[i] ); } }
        for( size_t j = 0; j < nb; ++j ) { if( zb[j] ) { cover.push_back( B[j] ); } }
        return cover;
    }

    const Graph & g_;
    I32 leaf_;
    static constexpr size_t kParallelMin = 20000;   // smaller sets are not worth a thread
    std::vector<std::atomic<I32>> owner_;
    std::vector<I32> level_, slot_, key1_, key2_;
    std::atomic<I32> stamp_{ 0 };
    std::atomic<I32> tmp_stamp_{ -(1 << 30) };
};

} // namespace

extern "C" int tb_nested_dissection( int32_t n, const int64_t * outer, const int32_t * inner, int32_t dofs_per_node,
                                     int32_t leaf_size, int32_t thread_count, int32_t * perm )
{
    if( n < 0 || (n > 0 && (outer == nullptr || inner == nullptr || perm == nullptr)) || dofs_per_node < 1 )
    {
        return fail( TB_ERR_INVALID_ARGUMENT, "tb_nested_dissection: bad argument" );
    }
    if( n % dofs_per_node != 0 ) { return fail( TB_ERR_INVALID_ARGUMENT, "tb_nested_dissection: n is not a multiple of dofs_per_node" ); }
    if( n == 0 ) { return TB_OK; }
    if( outer[0] != 0 ) { return fail( TB_ERR_INVALID_PATTERN, "tb_nested_dissection: outer[0] != 0" ); }
    for( I32 r = 0; r < n; ++r )
    {
        if( outer[r + 1] < outer[r] ) { return fail( TB_ERR_INVALID_PATTERN, "tb_nested_dissection: row pointers decrease" ); }
    }
    for( I64 k = 0; k < outer[n]; ++k )
    {
        if( inner[k] < 0 || inner[k] >= n ) { return fail( TB_ERR_INVALID_PATTERN, "tb_nested_dissection: column index out of range" ); }
    }
    const Graph g = node_graph( n, outer, inner, dofs_per_node );
    int threads = thread_count;
    if( threads <= 0 ) { const unsigned h = std::thread::hardware_concurrency(); threads = h == 0 ? 1 : static_cast<int>( std::min( h, 64u ) ); }
    const std::vector<I32> order = Dissection( g, std::max( 1, leaf_size / dofs_per_node ) ).run( threads );
    I64 i = 0;
    for( I32 u : order )
    {
        for( I32 j = 0; j < dofs_per_node; ++j ) { perm[i++] = u * dofs_per_node + j; }
    }
    return TB_OK;
}
