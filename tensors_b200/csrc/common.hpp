// Status codes and small shared helpers of the tensors_b200 library.
#pragma once

#include <cstdint>

#include "../../include/tensors_b200.h"

namespace tb
{
constexpr std::int64_t ceil_div( std::int64_t a, std::int64_t b ) { return (a + b - 1) / b; }
} // namespace tb
