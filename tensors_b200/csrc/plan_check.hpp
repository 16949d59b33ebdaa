// Host-side bounds check of a device plan (see plan_check.cpp).
#pragma once

#include <string>

#include "plan.hpp"
#include "symbolic.hpp"

namespace tb
{
// Empty string when every task stays within its buffers, else a description
// of the first violation.
std::string check_plan( const Symbolic & sym, const Plan & pl );
} // namespace tb
