// Internal declarations shared by the host-side translation units.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "../../include/hmotif.h"

namespace hm {

// Records a message for hm_last_error() on the calling thread and returns
// the status code so call sites can write `return set_error(...)`.
int set_error(int status, const char* fmt, ...);

}  // namespace hm

// A host-side hypergraph (generator output, files read or written).
struct hm_hostgraph {
  std::vector<uint64_t> offsets;
  std::vector<uint32_t> members;
  std::vector<int64_t> times;
  uint32_t n_nodes = 0;
  uint64_t redraws = 0;
};

