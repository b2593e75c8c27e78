// Allocation-free per-column dot products of device blocks.
//
// Some callers cannot let a library allocate device memory while they run:
// their device memory is owned by their own pool (an outer L-BFGS or Krylov
// driver that keeps its vectors on the GPU), and a cudaMalloc would
// synchronise the device or break their memory accounting.  This entry point
// serves them: it runs the same deterministic two-stage reduction as the
// library's column dots (coldot_kernel + reduce_partials_kernel), but keeps the
// per-block partial sums in the file-scope device array below instead of
// context-owned memory, and it calls no allocating routine.
//
// The array is 296 blocks x 64 columns of doubles (148 KB) and every GPU that
// loads the library holds it until the process exits.  All calls share it and
// it keeps the last call's contents; each call overwrites every partial it
// later reads, so nothing needs clearing, but calls that overlap on the GPU
// (different streams, no ordering between them) race on it.
//
// The module is loaded lazily: the first call on a device loads it, which is
// when the array and the kernels' own device memory are reserved.  A caller
// that owns its device pool makes one warm-up call per device before it hands
// the device to the pool.  The array's name in host
// code is a host-side stand-in, not a device address, so every call asks the
// runtime for the address with the device current; once the module is loaded
// the lookup allocates nothing, and it stays right when a device reset or a
// new primary context reloads the module at another address.
#include <string>

#include "../../include/invdft_force.h"
#include "kernels.cuh"

namespace invdft {
void set_thread_error(const std::string &msg);  // capi.cu: message of invdft_last_error(NULL)
}

namespace {

constexpr int kNoallocBlocks = 296;  // 2 x 148 SMs
constexpr int kNoallocMaxCols = 64;
static __device__ __align__(256) double g_noalloc_partials[kNoallocBlocks * kNoallocMaxCols];

}  // namespace

extern "C" invdft_status invdft_coldot_noalloc(const double *d_a, const double *d_b, int64_t n, int32_t B,
                                               double *d_out, void *stream) {
  if (!d_a || !d_b || !d_out || n < 0) {
    invdft::set_thread_error("invdft_coldot_noalloc: null pointer or negative length");
    return INVDFT_BAD_ARG;
  }
  if (B < 1 || B > kNoallocMaxCols) {
    invdft::set_thread_error("invdft_coldot_noalloc: block width must be in [1, 64] (the size of its "
                             "static scratch), got " + std::to_string(B));
    return INVDFT_BAD_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    invdft::set_thread_error("invdft_coldot_noalloc: no usable current CUDA device");
    return INVDFT_CUDA_ERROR;
  }
  // the device address of the array in the current device's context
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
  if (e != cudaSuccess || !p) {
    invdft::set_thread_error(std::string("invdft_coldot_noalloc: cudaGetSymbolAddress failed on device ") +
                             std::to_string(dev) + ": " + cudaGetErrorString(e));
    return INVDFT_CUDA_ERROR;
  }
  double *scratch = static_cast<double *>(p);
  try {
    invdft::launch_coldot(d_a, d_b, n, B, scratch, kNoallocBlocks, d_out, static_cast<cudaStream_t>(stream));
  } catch (const std::exception &ex) {
    invdft::set_thread_error(std::string("invdft_coldot_noalloc: ") + ex.what());
    return INVDFT_CUDA_ERROR;
  }
  return INVDFT_OK;
}
