// Shared helpers of the C ABI implementation (host and device parts).
#pragma once
#include <exception>
#include <string>

#include "../../../include/tigerci_sigma.h"
#include "plan.h"

namespace tci {
void set_error(const std::string& m);
int guard_status(const std::exception_ptr& ep);
void build_space_from_c(const tci_deck* d, CsfSpace& sp);
void operator_from_c(const tci_operator* op, const CsfSpace& sp, Operator& out);
}  // namespace tci
