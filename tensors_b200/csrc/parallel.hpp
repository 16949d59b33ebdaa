// Host-side row parallelism shared by the symbolic analysis and the plan.
#pragma once

#include <algorithm>
#include <cstdint>
#include <thread>
#include <vector>

namespace tb
{

// body(b, e) over [0, count) split into contiguous ranges, one per host
// thread (one range below 65,536 items).
template<typename Body>
void parallel_rows( std::int64_t count, Body && body )
{
    const unsigned hw = std::max( 1u, std::thread::hardware_concurrency() );
    const std::int64_t threads = std::min<std::int64_t>( hw, std::max<std::int64_t>( 1, count / 65536 ) );
    if( threads <= 1 ) { body( std::int64_t(0), count ); return; }
    std::vector<std::thread> pool;
    for( std::int64_t t = 0; t < threads; ++t )
    {
        const std::int64_t b = count * t / threads, e = count * (t + 1) / threads;
        pool.emplace_back( [&body, b, e]() { body( b, e ); } );
    }
    for( auto & th : pool ) { th.join(); }
}

} // namespace tb
