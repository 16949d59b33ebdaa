// Static list scheduling of the factorization's task graph.
//
// The persistent factorization kernel hands out tasks first come, first
// served in the order of Plan::dag, and a CTA that takes a task whose inputs
// are not ready yet waits for them.  The plan builds the list level by level
// (a valid but naive order), so CTAs would often wait behind long-running
// tasks.  This pass simulates the launch on the host: `workers` CTAs, task
// durations from a simple cost model, and whenever a CTA is free it starts
// the ready task with the longest remaining path to the end of the graph
// (its upward rank).  The simulated start order becomes the new list order:
// every task starts after the tasks it waits for have finished, so the order
// is again topological, and on the device the tasks a CTA takes are, as far
// as the cost model is right, ready when taken.
#include "plan.hpp"
#include "schedule.hpp"

#include <algorithm>
#include <queue>
#include <utility>
#include <vector>

namespace tb
{
namespace
{
using I32 = std::int32_t;
using I64 = std::int64_t;

// Microseconds of one task on one CTA (rough: a fixed latency plus work over
// a per-CTA rate).  Only relative sizes matter for the order.
double task_cost( const Plan & pl, const DagTask & t )
{
    switch( static_cast<LaunchKind>( t.kind ) )
    {
        case LaunchKind::Zero:   return 1.0 + static_cast<double>( pl.zero[t.index].count ) * 8.0 / 100e3;
        case LaunchKind::Extend:
        {
            const ExtendTask & e = pl.extend[t.index];
            double entries = 0.0;
            for( I32 r = e.row_begin; r < e.row_end; ++r ) { entries += e.m1 - r; }
            return 2.0 + entries * 24.0 / 50e3;
        }
        case LaunchKind::Potrf:  return 20.0;
        case LaunchKind::Trsm:   return 12.0;
        case LaunchKind::Invert: return 6.0;
        case LaunchKind::Gemm:
        {
            const GemmTask & g = pl.gemm[t.index];
            const double rows = std::min( kTile, g.M - g.m0 ), cols = std::min( kTile, g.N - g.c0 );
            return 3.0 + 2.0 * g.K * rows * cols / 120e3;
        }
        default: return 1.0;
    }
}

} // namespace

void schedule_task_graph( Plan & pl, int workers )
{
    const I64 n = static_cast<I64>( pl.dag.size() );
    const I32 nc = pl.dag_counters;
    if( n == 0 || workers <= 0 ) { return; }

    // waiters of every counter, sorted by target
    std::vector<I64> wptr( static_cast<size_t>(nc) + 1, 0 );
    for( const DagTask & t : pl.dag )
    {
        for( int i = 0; i < kDagWaits; ++i ) { if( t.wait[i] >= 0 ) { ++wptr[static_cast<size_t>( t.wait[i] ) + 1]; } }
    }
    for( I32 c = 0; c < nc; ++c ) { wptr[c + 1] += wptr[c]; }
    std::vector<std::pair<I32, I64>> waiters( static_cast<size_t>( wptr[nc] ) );     // (target, task)
    {
        std::vector<I64> fill( wptr.begin(), wptr.end() - 1 );
        for( I64 k = 0; k < n; ++k )
        {
            const DagTask & t = pl.dag[static_cast<size_t>(k)];
            for( int i = 0; i < kDagWaits; ++i )
            {
                if( t.wait[i] >= 0 ) { waiters[static_cast<size_t>( fill[t.wait[i]]++ )] = { t.target[i], k }; }
            }
        }
        for( I32 c = 0; c < nc; ++c ) { std::sort( waiters.begin() + wptr[c], waiters.begin() + wptr[c + 1] ); }
    }

    // upward ranks, in reverse list order: a task's successors are the
    // waiters, later in the list, of the counters it signals
    std::vector<double> cost( static_cast<size_t>(n) ), rank( static_cast<size_t>(n) );
    std::vector<double> later_max( static_cast<size_t>(nc), 0.0 );
    for( I64 k = n - 1; k >= 0; --k )
    {
        const DagTask & t = pl.dag[static_cast<size_t>(k)];
        cost[static_cast<size_t>(k)] = task_cost( pl, t );
        double succ = 0.0;
        for( int i = 0; i < 2; ++i ) { if( t.signal[i] >= 0 ) { succ = std::max( succ, later_max[t.signal[i]] ); } }
        rank[static_cast<size_t>(k)] = cost[static_cast<size_t>(k)] + succ;
        for( int i = 0; i < kDagWaits; ++i )
        {
            if( t.wait[i] >= 0 ) { later_max[t.wait[i]] = std::max( later_max[t.wait[i]], rank[static_cast<size_t>(k)] ); }
        }
    }

    // event simulation
    std::vector<I32> pending( static_cast<size_t>(n), 0 );
    std::vector<I32> count( static_cast<size_t>(nc), 0 );
    using Ready = std::pair<double, I64>;                    // (rank, -task) : highest rank, then list order
    std::priority_queue<std::pair<double, I64>> ready;
    for( I64 k = 0; k < n; ++k )
    {
        const DagTask & t = pl.dag[static_cast<size_t>(k)];
        for( int i = 0; i < kDagWaits; ++i ) { if( t.wait[i] >= 0 ) { ++pending[static_cast<size_t>(k)]; } }
        if( pending[static_cast<size_t>(k)] == 0 ) { ready.push( Ready{ rank[static_cast<size_t>(k)], -k } ); }
    }
    using Event = std::pair<double, I64>;                    // (finish time, task)
    std::priority_queue<Event, std::vector<Event>, std::greater<Event>> running;
    std::vector<DagTask> order;
    order.reserve( static_cast<size_t>(n) );
    double now = 0.0;
    int idle = workers;
    while( static_cast<I64>( order.size() ) < n || !running.empty() )
    {
        while( idle > 0 && !ready.empty() )
        {
            const I64 k = -ready.top().second;
            ready.pop();
            order.push_back( pl.dag[static_cast<size_t>(k)] );
            running.push( { now + cost[static_cast<size_t>(k)], k } );
            --idle;
        }
        if( running.empty() ) { break; }                     // nothing runnable: the graph is inconsistent
        const Event e = running.top();
        running.pop();
        now = e.first;
        ++idle;
        const DagTask & t = pl.dag[static_cast<size_t>( e.second )];
        for( int i = 0; i < 2; ++i )
        {
            const I32 c = t.signal[i];
            if( c < 0 ) { continue; }
            const I32 v = ++count[static_cast<size_t>(c)];
            auto lo = std::lower_bound( waiters.begin() + wptr[c], waiters.begin() + wptr[c + 1], std::make_pair( v, I64( -1 ) ) );
            for( auto it = lo; it != waiters.begin() + wptr[c + 1] && it->first == v; ++it )
            {
                if( --pending[static_cast<size_t>( it->second )] == 0 )
                {
                    ready.push( Ready{ rank[static_cast<size_t>( it->second )], -it->second } );
                }
            }
        }
    }
    if( static_cast<I64>( order.size() ) == n ) { pl.dag.swap( order ); }
    pl.dag_makespan_us = now;
}

} // namespace tb
