// Error reporting and launch helpers of libcbmv.
#include <stdarg.h>

#include "common.cuh"

namespace cbmv {

static thread_local char g_err[512] = "";

int set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(CBMV_ECUDA, "%s launch: %s", what, cudaGetErrorString(e));
  return CBMV_OK;
}

unsigned grid_for(int64_t n, int block) {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
      sms = 148;
  }
  int64_t g = (n + block - 1) / block;
  const int64_t cap = (int64_t)sms * 32;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (unsigned)g;
}

}  // namespace cbmv

extern "C" const char* cbmv_last_error(void) { return cbmv::g_err; }
extern "C" const char* cbmv_version(void) { return "cbmv-b200 0.1"; }
extern "C" int cbmv_sync(void* stream) {
  CBMV_CUDA(cudaStreamSynchronize(cbmv::as_stream(stream)));
  return CBMV_OK;
}
