// Status codes and small shared helpers of the tensors_b200 library.
#pragma once

#include <cstdint>
#include <string>

#include "../../include/tensors_b200.h"

namespace tb
{
constexpr std::int64_t ceil_div( std::int64_t a, std::int64_t b ) { return (a + b - 1) / b; }
// Message of the last failing call on this thread (tb_last_error).
void set_last_error( const std::string & msg );
} // namespace tb
