// Static list scheduling of the factorization's task graph (schedule.cpp).
#pragma once

#include "plan.hpp"

namespace tb
{

// Reorders plan.dag into the start order of a simulated run on `workers`
// CTAs (critical-path first); records the simulated makespan in
// plan.dag_makespan_us.  Leaves the list unchanged if it cannot be ordered.
void schedule_task_graph( Plan & plan, int workers );

} // namespace tb
