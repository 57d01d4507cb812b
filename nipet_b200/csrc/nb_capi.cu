// nb_capi.cu -- status strings and the per-thread last-error message of the C ABI.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include "nb_internal.cuh"

static thread_local char g_last_error[1024] = "";

void nb_set_error_msg(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

int nb_cuda_fail(cudaError_t e, const char *what, const char *file, int line) {
  nb_set_error_msg("%s failed: %s (%s) at %s:%d", what, cudaGetErrorName(e),
                   cudaGetErrorString(e), file, line);
  return e == cudaErrorMemoryAllocation ? NB_ERR_NOMEM : NB_ERR_CUDA;
}

extern "C" int nb_version(void) { return 10000; }

extern "C" const char *nb_last_error(void) { return g_last_error; }

extern "C" const char *nb_strerror(int status) {
  switch (status) {
  case NB_OK: return "success";
  case NB_ERR_ARG: return "invalid argument";
  case NB_ERR_CUDA: return "CUDA runtime error";
  case NB_ERR_NOMEM: return "out of device memory";
  case NB_ERR_DEVICE: return "device-side error";
  case NB_ERR_UNSUPPORTED: return "unsupported";
  case NB_ERR_DATA: return "malformed input data";
  default: return "unknown status";
  }
}
