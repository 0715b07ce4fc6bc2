// Status codes and the per-thread last-error message.
#include <cstdarg>
#include <cstdio>

#include "hm_internal.h"

namespace {
thread_local char g_last_error[512] = "";
}

namespace hm {

int set_error(int status, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return status;
}

}  // namespace hm

extern "C" const char* hm_last_error(void) { return g_last_error; }

extern "C" const char* hm_status_string(int status) {
  switch (status) {
    case HM_OK: return "ok";
    case HM_ERR_INVALID: return "invalid argument";
    case HM_ERR_CUDA: return "CUDA runtime error";
    case HM_ERR_NOMEM: return "out of device memory or over budget";
    case HM_ERR_CAPACITY: return "output buffer too small";
    case HM_ERR_NOT_LIVE: return "hyperedge id not live";
    case HM_ERR_TIMEOUT: return "bounded device wait expired";
    case HM_ERR_STATE: return "invalid object state";
    case HM_ERR_LIMIT: return "input beyond a documented size limit";
    default: return "unknown status";
  }
}
