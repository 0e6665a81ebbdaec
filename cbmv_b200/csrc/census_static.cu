// cbmv_census_static: the census matcher with its scratch memory in a
// fixed device array instead of a per-call allocation.
//
// cbmv_census needs two descriptor images (16 bytes per pixel each) as
// scratch and allocates them on every call.  Some callers cannot allocate
// device memory at the point where they call the matcher: code running
// under a memory manager that owns the whole device heap (a serving
// runtime's arena, a framework's caching allocator that must see every
// byte), code that records launches into a CUDA graph while capture forbids
// allocation, or embedded hosts whose plugin interface hands out only
// input and output buffers.  This entry point allocates nothing: the
// descriptors live in g_census_scratch below, a file-scope device array of
// kStaticCensusMaxPixels pixels per image (32 MiB in all) that every GPU
// loading this library holds from module load until the process exits.
#include <mutex>

#include "common.cuh"
#include "pipeline.cuh"

namespace cbmv {
namespace {

constexpr int64_t kStaticCensusMaxPixels = int64_t(1) << 20;  // per image

// Descriptors of the left image in [0, max), of the right image in
// [max, 2 max).  Shared by every call of cbmv_census_static on a device.
__device__ __align__(256) ulonglong2 g_census_scratch[2 * kStaticCensusMaxPixels];

// The array's device address, looked up once per device: in host code the
// symbol g_census_scratch names a host-side stand-in, not device memory, so
// it must never be passed to a kernel directly.  The cache lives as long as
// the process: after cudaDeviceReset the module (and the array) is loaded
// anew at another address, so a process that resets a device must not call
// cbmv_census_static again.
std::mutex g_mu;
void* g_addr[64] = {};

int scratch_address(ulonglong2** out) {
  int dev = 0;
  CBMV_CUDA(cudaGetDevice(&dev));
  CBMV_REQUIRE(dev >= 0 && dev < 64, CBMV_ERANGE, "device ordinal %d beyond 63", dev);
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_census_scratch);
    if (e != cudaSuccess || !p)
      return set_error(CBMV_ECUDA, "cudaGetSymbolAddress(g_census_scratch): %s",
                       cudaGetErrorString(e));
    g_addr[dev] = p;
  }
  *out = static_cast<ulonglong2*>(g_addr[dev]);
  return CBMV_OK;
}

}  // namespace
}  // namespace cbmv

using namespace cbmv;

extern "C" int64_t cbmv_census_static_max_pixels(void) { return kStaticCensusMaxPixels; }

extern "C" int cbmv_census_static(const uint8_t* L, const uint8_t* R, int64_t H, int64_t W, int D,
                                  int wsize, void* out, int dtype, int layout, void* stream) {
  int rc = check_common(L, R, out, H, W, D, wsize, dtype, layout, 11);  // as cbmv_census
  if (rc) return rc;
  // W <= max / H first, so that H * W cannot overflow
  CBMV_REQUIRE(W <= kStaticCensusMaxPixels / H, CBMV_ERANGE,
               "cbmv_census_static: image of %lld x %lld pixels exceeds its fixed scratch of %lld pixels "
               "(use cbmv_census)",
               (long long)W, (long long)H, (long long)kStaticCensusMaxPixels);
  ulonglong2* dl = nullptr;
  rc = scratch_address(&dl);
  if (rc) return rc;
  ulonglong2* dr = dl + kStaticCensusMaxPixels;
  cudaStream_t st = as_stream(stream);
  // Every descriptor the cost kernel reads is written by this call first
  // (both lie in the valid window region), so nothing needs clearing.
  if ((rc = launch_census_desc(L, H, W, wsize, dl, st))) return rc;
  if ((rc = launch_census_desc(R, H, W, wsize, dr, st))) return rc;
  return dtype == CBMV_F64 ? launch_census_cost(dl, dr, H, W, D, wsize, layout, (double*)out, st)
                           : launch_census_cost(dl, dr, H, W, D, wsize, layout, (float*)out, st);
}
