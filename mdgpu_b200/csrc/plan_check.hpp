// Host self-check of a plan's tables (see plan_check.cpp).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "plan.hpp"

namespace mdgpu {

// Empty when every invariant holds, else what failed (and for which front).
std::string check_plan(const Plan& P, const Symbolic& S, const SolveScheduleHost& Q,
                       const std::vector<int>& level, const std::vector<int>& csr_rowptr,
                       const int* csr_col, const int* csr_src, int64_t csr_nnz);

// The panel launches' task lists (tile T, panel width PW): per OP_PANEL every
// row tile of the level's fronts that have the panel once, each task after
// the diagonal tasks it waits on, counters and flags in range.
std::string check_panel_schedule(const Plan& P, const PanelSchedule& S,
                                 const std::vector<int>& level, int T, int PW);

}  // namespace mdgpu
