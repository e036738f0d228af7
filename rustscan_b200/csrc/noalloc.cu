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
#include <cuda.h>
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

// Device address of the array, looked up with cudaGetSymbolAddress (the
// host-side name of a __device__ variable is not a device address). The
// address belongs to the module as loaded into one CUDA context: after
// cudaDeviceReset, or under another context of the same device, the module
// is loaded anew, possibly elsewhere. So the lookup is cached per device
// together with the unique ID of the context it was made in (cuCtxGetId,
// reached through the runtime's driver entry points, so no link against
// libcuda), and made again whenever the calling thread's current context
// has another ID. Without those entry points (a driver older than CUDA 12.0)
// the address is looked up at every call: a host-side query that allocates
// nothing.
constexpr int kMaxDevices = 64;

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

struct DeviceSlot {
  bool valid;
  unsigned long long ctx_id;
  NoAllocScratch* ptr;
  int num_sms;
};

std::mutex g_setup_mutex;
DeviceSlot g_slots[kMaxDevices] = {};
std::once_flag g_entry_once;
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

void load_entry_points() {
  void* f = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
      q == cudaDriverEntryPointSuccess)
    g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f);
  f = nullptr;
  if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
      q == cudaDriverEntryPointSuccess)
    g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f);
  (void)cudaGetLastError();
}

// ID of the calling thread's current context; false if it cannot be told.
bool current_context_id(unsigned long long* id) {
  std::call_once(g_entry_once, load_entry_points);
  if (!g_ctx_get_current || !g_ctx_get_id) return false;
  CUcontext ctx = nullptr;
  if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return false;
  return g_ctx_get_id(ctx, id) == CUDA_SUCCESS;
}

gsr_status lookup(int dev, NoAllocScratch** out, int* num_sms) {
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
  *out = static_cast<NoAllocScratch*>(p);
  *num_sms = sms;
  return GSR_OK;
}

// Set-up, with device `dev` current: the array's address in the current
// context, from the cache when it was looked up in this very context.
gsr_status setup_device(int dev, NoAllocScratch** out, int* num_sms) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  DeviceSlot& s = g_slots[dev];
  unsigned long long id = 0;
  if (current_context_id(&id) && s.valid && s.ctx_id == id) {
    *out = s.ptr;
    *num_sms = s.num_sms;
    return GSR_OK;
  }
  // The lookup creates the device's primary context if none is current yet,
  // so the context is asked for again afterwards.
  gsr_status rs = lookup(dev, out, num_sms);
  if (rs != GSR_OK) return rs;
  s.valid = current_context_id(&id);
  s.ctx_id = id;
  s.ptr = *out;
  s.num_sms = *num_sms;
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
