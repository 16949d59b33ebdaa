// Phase ranges: NVTX push/pop plus an optional host-side record (trace.hpp).
#include "trace.hpp"

#include <nvtx3/nvToolsExt.h>

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tensors_b200.h"

namespace tb
{
namespace
{
using Clock = std::chrono::steady_clock;

struct Record
{
    std::string name;
    Clock::time_point begin, end;
    bool closed = false;
};

std::atomic<bool> g_recording{ false };
std::atomic<std::uint64_t> g_epoch{ 0 };    // bumped by every tb_trace_record: stale open ranges are dropped
std::mutex g_mutex;
std::vector<Record> g_records;
constexpr size_t kMaxNames = 1 << 16;

// The open ranges of this thread: index into g_records (-1: not recorded) and
// the recording epoch it belongs to.
struct Open
{
    std::int64_t index;
    std::uint64_t epoch;
};
thread_local std::vector<Open> t_open;
} // namespace

void trace_push( const char * tag )
{
    nvtxRangePushA( tag );
    std::int64_t index = -1;
    std::uint64_t epoch = 0;
    if( g_recording.load( std::memory_order_relaxed ) )
    {
        std::lock_guard<std::mutex> lock( g_mutex );
        epoch = g_epoch.load( std::memory_order_relaxed );
        if( g_records.size() < kMaxNames )
        {
            index = static_cast<std::int64_t>( g_records.size() );
            g_records.push_back( Record{ tag, Clock::now(), {}, false } );
        }
    }
    t_open.push_back( Open{ index, epoch } );
}

void trace_pop()
{
    nvtxRangePop();
    if( t_open.empty() ) { return; }
    const Open o = t_open.back();
    t_open.pop_back();
    if( o.index < 0 ) { return; }
    const auto now = Clock::now();
    std::lock_guard<std::mutex> lock( g_mutex );
    if( o.epoch == g_epoch.load( std::memory_order_relaxed ) && o.index < static_cast<std::int64_t>( g_records.size() ) )
    {
        g_records[static_cast<size_t>( o.index )].end = now;
        g_records[static_cast<size_t>( o.index )].closed = true;
    }
}

} // namespace tb

extern "C" {

int tb_trace_record( int32_t enabled )
{
    std::lock_guard<std::mutex> lock( tb::g_mutex );
    tb::g_records.clear();
    tb::g_epoch.fetch_add( 1 );
    tb::g_recording.store( enabled != 0 );
    return TB_OK;
}

int64_t tb_trace_names( char * buf, int64_t cap )
{
    std::lock_guard<std::mutex> lock( tb::g_mutex );
    std::string all;
    for( const auto & r : tb::g_records ) { all += r.name; all += '\n'; }
    if( buf != nullptr && cap > 0 )
    {
        const size_t m = std::min<size_t>( all.size(), static_cast<size_t>( cap - 1 ) );
        std::memcpy( buf, all.data(), m );
        buf[m] = '\0';
    }
    return static_cast<int64_t>( all.size() ) + 1;
}

int64_t tb_trace_times( double * ms, int64_t cap )
{
    std::lock_guard<std::mutex> lock( tb::g_mutex );
    const std::int64_t n = static_cast<std::int64_t>( tb::g_records.size() );
    if( ms != nullptr )
    {
        for( std::int64_t i = 0; i < std::min( n, cap ); ++i )
        {
            const auto & r = tb::g_records[static_cast<size_t>( i )];
            ms[i] = r.closed ? std::chrono::duration<double, std::milli>( r.end - r.begin ).count() : -1.0;
        }
    }
    return n;
}

} // extern "C"
