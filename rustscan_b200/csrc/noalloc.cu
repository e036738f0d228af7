// noalloc.cu — an inclusive prefix sum that allocates nothing.
//
// Some callers cannot let a library allocate device memory. A host framework
// that owns the whole device memory budget through its own pool has to
// account for every byte, and a side allocation either breaks that
// accounting or fails with out-of-memory in the middle of a run. Deployments
// that fix their memory use at start-up forbid allocation after
// initialisation for the same reason. Creating a gsr context allocates its
// scratch, so those callers cannot use gsr_prefix_sum_u32.
//
// gsr_prefix_sum_u32_noalloc runs the same single-pass look-back scan, but
// its scratch is a fixed array compiled into this library (file scope,
// __device__, 64 KiB of look-back states plus a control block and status
// words). Every GPU that loads the library holds that array until the
// process exits. The caller passes only the input and the output.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/gsr.h"
#include "gsr_kernels.h"

using namespace gsr;

namespace {

// Largest input: 2^24 values, i.e. 8192 partitions of 2048 values, one
// 64-bit look-back state each.
constexpr uint32_t kNoAllocMaxN = 1u << 24;
constexpr uint32_t kNoAllocStates = kNoAllocMaxN / 2048;

struct NoAllocScratch {
  unsigned long long states[kNoAllocStates];
  LookbackCtl ctl;
  DevStatus status;
};

// Zero-initialised when the module loads. The look-back states are tagged
// with a launch epoch kept in `ctl`, so stale states from an earlier call
// never need clearing; the status words are cleared at every call.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Device address of the array per device ordinal, looked up once per device
// with that device current (the host-side name of a __device__ variable is
// not a device address).
constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
NoAllocScratch* g_scratch_ptr[kMaxDevices] = {};
int g_num_sms[kMaxDevices] = {};

gsr_status setup_device(int dev, NoAllocScratch** out, int* num_sms) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) {
      (void)cudaGetLastError();
      return GSR_ERR_CUDA;
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) {
      (void)cudaGetLastError();
      return GSR_ERR_CUDA;
    }
    g_num_sms[dev] = sms;
    g_scratch_ptr[dev] = static_cast<NoAllocScratch*>(p);
  }
  *out = g_scratch_ptr[dev];
  *num_sms = g_num_sms[dev];
  return GSR_OK;
}

}  // namespace

extern "C" GSR_API gsr_status gsr_prefix_sum_u32_noalloc(const uint32_t* in, uint32_t* out, uint32_t n,
                                                          void* stream) {
  if (n == 0) return GSR_OK;
  if (!in || !out || in == out) return GSR_ERR_INVALID_ARG;
  if (n > kNoAllocMaxN) return GSR_ERR_INVALID_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    (void)cudaGetLastError();
    return GSR_ERR_CUDA;
  }
  NoAllocScratch* scratch = nullptr;
  int num_sms = 0;
  gsr_status rs = setup_device(dev, &scratch, &num_sms);
  if (rs != GSR_OK) return rs;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(&scratch->status, 0, sizeof(DevStatus), st) != cudaSuccess) {
    (void)cudaGetLastError();
    return GSR_ERR_CUDA;
  }
  if (inclusive_scan_u32_scratch(in, out, n, scratch->states, kNoAllocStates, &scratch->ctl, &scratch->status,
                                 num_sms, st) != cudaSuccess) {
    (void)cudaGetLastError();
    return GSR_ERR_CUDA;
  }
  return GSR_OK;
}
