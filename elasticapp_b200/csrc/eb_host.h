// Host-side helpers shared between the simulator (eb_capi.cu) and the server
// (serve.cu).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/elastica_b200.h"
#include "eb_internal.h"

namespace eb {

// One straight rod from its initializer, in the local slot layout: field row f
// of the rod at [f * (n + 1), (f + 1) * (n + 1)).
struct HostRodData {
  int64_t n = 0;
  bool damped = false;
  std::vector<double> state;  // kStateFields rows
  std::vector<double> param;  // kParamFields rows
};
eb_status host_straight_rod(const eb_straight_rod& p, HostRodData& out);

// records the message eb_last_error() returns on this thread
void set_last_error(const std::string& message);

}  // namespace eb
