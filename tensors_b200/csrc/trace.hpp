// Named phase ranges for timeline tools.  Each range carries the tag of the
// reference's TOOLS_PTIMER at the same phase (for example
// "CholeskyDecomposition::NumericFactorization", Numeric.hpp:34), is an NVTX
// push/pop range (header-only NVTX 3: free unless a profiler such as Nsight
// Systems is attached), and, while recording is switched on
// (tb_trace_record), is also appended to a host-side list that
// tb_trace_names returns, so the ranges can be checked without a profiler.
#pragma once

#include <string>

namespace tb
{

void trace_push( const char * tag );
void trace_pop();

struct TraceRange
{
    explicit TraceRange( const char * tag ) { trace_push( tag ); }
    ~TraceRange() { trace_pop(); }
    TraceRange( const TraceRange & ) = delete;
    TraceRange & operator=( const TraceRange & ) = delete;
};

} // namespace tb
