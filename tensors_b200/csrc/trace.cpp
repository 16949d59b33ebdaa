// Phase ranges: NVTX push/pop plus an optional host-side record (trace.hpp).
#include "trace.hpp"

#include <nvtx3/nvToolsExt.h>

#include <atomic>
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
std::atomic<bool> g_recording{ false };
std::mutex g_mutex;
std::vector<std::string> g_names;
constexpr size_t kMaxNames = 1 << 16;
} // namespace

void trace_push( const char * tag )
{
    nvtxRangePushA( tag );
    if( g_recording.load( std::memory_order_relaxed ) )
    {
        std::lock_guard<std::mutex> lock( g_mutex );
        if( g_names.size() < kMaxNames ) { g_names.emplace_back( tag ); }
    }
}

void trace_pop() { nvtxRangePop(); }

} // namespace tb

extern "C" {

int tb_trace_record( int32_t enabled )
{
    std::lock_guard<std::mutex> lock( tb::g_mutex );
    tb::g_names.clear();
    tb::g_recording.store( enabled != 0 );
    return TB_OK;
}

int64_t tb_trace_names( char * buf, int64_t cap )
{
    std::lock_guard<std::mutex> lock( tb::g_mutex );
    std::string all;
    for( const auto & s : tb::g_names ) { all += s; all += '\n'; }
    if( buf != nullptr && cap > 0 )
    {
        const size_t m = std::min<size_t>( all.size(), static_cast<size_t>( cap - 1 ) );
        std::memcpy( buf, all.data(), m );
        buf[m] = '\0';
    }
    return static_cast<int64_t>( all.size() ) + 1;
}

} // extern "C"
