// gsr_internal.cuh — shared device-side building blocks of the rasterizer:
// per-view descriptors, device status flags, bounded waits and the
// decoupled look-back used by the compaction, the scans and the radix sort.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "gsr_math.h"

namespace gsr {

constexpr int kWarp = 32;

// Device status words (zeroed by the host, read by gsr_sync_status).
struct DevStatus {
  uint32_t overflow;       // an intersection list did not fit
  uint32_t timeout;        // a bounded wait gave up
  uint32_t timeout_where;  // which wait gave up (kernel id)
  uint32_t bad_input;      // an input index out of range (topology plan)
  unsigned long long required;  // largest intersection count requested
  uint32_t internal;       // an internal consistency check failed (a sort position outside its segment)
};

enum : uint32_t { kWaitCompact = 1, kWaitScan = 2, kWaitSort = 3, kWaitSelfTest = 4 };

// Per-view camera and layout, in device memory.
struct ViewDesc {
  float rot[9];  // rot[col*3 + row]
  float trans[3];
  float fx, fy, cx, cy;
  uint32_t w, h;
  float campos[3];
  uint32_t tiles_x, tiles_y;
  uint32_t tile_base;  // first work item of this view in the persistent raster
  uint64_t pix_base;   // first pixel of this view in the packed image buffer
};

template <class F> __device__ __forceinline__ Cam<F> cam_from_desc(const ViewDesc& d) {
  Cam<F> c;
  for (int col = 0; col < 3; ++col)
    for (int row = 0; row < 3; ++row) c.rot.m[col][row] = F(d.rot[col * 3 + row]);
  c.trans.x = F(d.trans[0]);
  c.trans.y = F(d.trans[1]);
  c.trans.z = F(d.trans[2]);
  c.focal.x = F(d.fx);
  c.focal.y = F(d.fy);
  c.pc.x = F(d.cx);
  c.pc.y = F(d.cy);
  c.w = d.w;
  c.h = d.h;
  c.campos.x = F(d.campos[0]);
  c.campos.y = F(d.campos[1]);
  c.campos.z = F(d.campos[2]);
  return c;
}

// ---------------------------------------------------------------------------
// Bounded waits. Every spin on another block's progress gives up after a
// fixed number of polls, records where, and lets the kernel finish (with
// wrong data) so that the context stays usable and the host sees
// GSR_ERR_TIMEOUT.
// ---------------------------------------------------------------------------
constexpr uint32_t kMaxPolls = 1u << 22;

__device__ __forceinline__ void report_timeout(DevStatus* st, uint32_t where) {
  atomicExch(&st->timeout, 1u);
  atomicExch(&st->timeout_where, where);
}

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) { return *(const volatile uint32_t*)p; }
__device__ __forceinline__ void st_volatile(uint32_t* p, uint32_t v) { *(volatile uint32_t*)p = v; }

// ---------------------------------------------------------------------------
// Decoupled look-back. A 64-bit state word packs a 30-bit launch epoch, a
// 2-bit flag (1: this partition's aggregate, 2: inclusive prefix through this
// partition) and a 32-bit count. A word whose epoch differs from the
// launch's is "not yet published", so state arrays never need clearing —
// also under CUDA-graph replay, because the epoch lives in device memory and
// advances once per launch (see LookbackCtl).
// ---------------------------------------------------------------------------
constexpr unsigned long long kFlagAgg = 1ull << 32;
constexpr unsigned long long kFlagPre = 2ull << 32;

__device__ __forceinline__ unsigned long long ld_volatile64(const unsigned long long* p) {
  return *(const volatile unsigned long long*)p;
}
__device__ __forceinline__ void st_volatile64(unsigned long long* p, unsigned long long v) {
  *(volatile unsigned long long*)p = v;
}

// Publishes `agg` for partition `part` of a chain whose states are
// states[part * stride] and returns the exclusive prefix of the partition.
__device__ __forceinline__ uint32_t lookback(unsigned long long* states, uint32_t stride, uint32_t part, uint32_t agg,
                                             uint32_t epoch, DevStatus* status, uint32_t where,
                                             uint32_t max_polls = kMaxPolls) {
  const unsigned long long tag = (unsigned long long)(epoch & 0x3fffffffu) << 34;
  if (part == 0) {
    st_volatile64(states, tag | kFlagPre | agg);
    return 0;
  }
  st_volatile64(states + (size_t)part * stride, tag | kFlagAgg | agg);
  // Walk back over the predecessors kLookbackWindow states per round trip:
  // the window's loads are independent and in flight together; the states
  // are then consumed in order up to the first inclusive prefix (done) or
  // the first predecessor that has not published yet (poll again from it).
  constexpr int kLookbackWindow = 8;
  uint32_t sum = 0;
  int64_t j = (int64_t)part - 1;
  uint32_t polls = 0;
  bool done = false;
  while (j >= 0 && !done) {
    unsigned long long w[kLookbackWindow];
#pragma unroll
    for (int k = 0; k < kLookbackWindow; ++k) w[k] = j - k >= 0 ? ld_volatile64(states + (size_t)(j - k) * stride) : 0ull;
    int used = 0;
#pragma unroll
    for (int k = 0; k < kLookbackWindow; ++k) {
      if (done || used < k || j - k < 0) continue;
      const unsigned long long s = w[k];
      if ((s >> 34) != (tag >> 34) || ((s >> 32) & 3ull) == 0) continue;  // not published: stop consuming
      sum += (uint32_t)s;
      used = k + 1;
      if (((s >> 32) & 3ull) == 2ull) done = true;
    }
    j -= used;
    if (!done && used < kLookbackWindow && j >= 0) {
      // Stopped at an unpublished predecessor.
      if (++polls > max_polls) {
        report_timeout(status, where);
        break;
      }
      if (used == 0) __nanosleep(20);
    }
  }
  st_volatile64(states + (size_t)part * stride, tag | kFlagPre | (uint32_t)(sum + agg));
  return sum;
}

// Launch epoch and work tickets shared by all blocks of one look-back kernel
// launch (one control block per context; launches on its stream are
// serialised). A kernel reads the device epoch at entry and tags its states
// with epoch+1; the last block to exit stores epoch+1 back and clears the
// tickets, so the next launch starts fresh without a memset.
constexpr int kMaxSegments = 64;
struct LookbackCtl {
  uint32_t epoch;
  uint32_t done;
  uint32_t ticket[kMaxSegments];
};

__device__ __forceinline__ uint32_t epoch_begin(const LookbackCtl* e) { return ld_volatile(&e->epoch) + 1u; }

// Every thread of every block calls this once, after the block's last
// look-back state write.
__device__ __forceinline__ void epoch_end(LookbackCtl* e, uint32_t epoch) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const uint32_t prev = atomicAdd(&e->done, 1u);
    if (prev == gridDim.x * gridDim.y * gridDim.z - 1) {
      for (int i = 0; i < kMaxSegments; ++i) e->ticket[i] = 0;
      e->done = 0;
      __threadfence();
      st_volatile(&e->epoch, epoch);
    }
  }
}

// Next work ticket of segment `seg` for this block (broadcast through smem).
__device__ __forceinline__ uint32_t next_ticket(LookbackCtl* e, uint32_t seg, uint32_t* smem_slot) {
  __syncthreads();
  if (threadIdx.x == 0) *smem_slot = atomicAdd(&e->ticket[seg], 1u);
  __syncthreads();
  return *smem_slot;
}

// ---------------------------------------------------------------------------
// Block-wide exclusive scan of one u32 per thread (blockDim.x <= 1024,
// multiple of 32). `scratch` holds 32 words. Returns the exclusive prefix;
// *total receives the block sum.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* scratch, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) scratch[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = (lane < nw) ? scratch[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) scratch[lane] = w;
  }
  __syncthreads();
  const uint32_t wbase = (warp > 0) ? scratch[warp - 1] : 0u;
  *total = scratch[nw - 1];
  __syncthreads();
  return wbase + x - v;
}

// Number of SMs of the current device (cached by the host and passed in).
struct LaunchInfo {
  int num_sms;
};

}  // namespace gsr
