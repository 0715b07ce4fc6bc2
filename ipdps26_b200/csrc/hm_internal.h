// Internal declarations shared by the host-side translation units.
#pragma once

#include <cstddef>
#include <cstdint>

#include "../../include/hmotif.h"

namespace hm {

// Records a message for hm_last_error() on the calling thread and returns
// the status code so call sites can write `return set_error(...)`.
int set_error(int status, const char* fmt, ...);

}  // namespace hm
