// tp_capi.cu -- version, status text, per-thread error detail, device queries.
#include <stdarg.h>
#include <stdio.h>

#include "tp_common.cuh"

namespace tp {

static thread_local char g_err[512] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int sm_count() {
  static int cached = 0;
  if (cached) return cached;
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1)
    return 148;
  cached = n;
  return n;
}

}  // namespace tp

extern "C" int tp_version(void) { return 10000; }

extern "C" const char* tp_status_string(int status) {
  switch (status) {
    case TP_OK: return "ok";
    case TP_ERR_ARG: return "invalid argument";
    case TP_ERR_CUDA: return "CUDA error";
    case TP_ERR_INDEX: return "index out of range";
    case TP_ERR_DEGENERATE: return "degenerate cell";
    case TP_ERR_CAPACITY: return "capacity exceeded";
    case TP_ERR_NOT_CONVERGED: return "not converged";
    case TP_ERR_BREAKDOWN: return "Krylov breakdown (operator not SPD)";
    case TP_ERR_NONFINITE: return "non-finite value";
    case TP_ERR_TIMEOUT: return "device wait timed out";
    default: return "unknown status";
  }
}

extern "C" const char* tp_last_error(void) { return tp::g_err; }

extern "C" int tp_device_sm_count(void) { return tp::sm_count(); }
