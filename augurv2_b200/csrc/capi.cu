// Library-wide C ABI: error reporting and version.
#include <string.h>

#include "common.cuh"

namespace ab {

static thread_local char g_last_error[512] = "";

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

int cuda_status(cudaError_t e, const char* what) {
  return fail(AB_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

}  // namespace ab

extern "C" const char* ab_last_error(void) { return ab::g_last_error; }

extern "C" const char* ab_version(void) { return "augurv2_b200 0.1 (sm_100a)"; }
