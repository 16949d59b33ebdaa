// Host-side row parallelism shared by the symbolic analysis and the plan.
#pragma once

#include <algorithm>
#include <cstdint>
#include <thread>
#include <vector>

namespace tb
{

// Host threads for a requested count: <= 0 means every hardware thread.
inline std::int64_t host_threads( std::int64_t requested )
{
    const std::int64_t hw = std::max( 1u, std::thread::hardware_concurrency() );
    return requested > 0 ? requested : hw;
}

// body(b, e) over [0, count) split into contiguous ranges, one per host
// thread (at most max_threads, <= 0: every hardware thread; one range below
// 65,536 items).
template<typename Body>
void parallel_rows( std::int64_t count, Body && body, std::int64_t max_threads = 0 )
{
    const std::int64_t threads = std::min<std::int64_t>( host_threads( max_threads ), std::max<std::int64_t>( 1, count / 65536 ) );
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
