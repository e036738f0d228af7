// k_frames.cu — training targets from 8-bit colour frames
// (frame_targets.rs:44-62, resize_rgb_u8_to_f32).
//
// The reference decodes a frame to RGB bytes, converts it on the host to
// f32 (each byte / 255, then a box-average resize when the frame size differs
// from the training resolution) and uploads the f32 image every step
// (engine/trainer.rs:94-107, 265-268). Here the bytes cross PCIe (a quarter
// of the f32 volume) and this kernel does the conversion on the device, for
// all views of a step in one launch: one thread per output pixel, the
// reference's box bounds and summation order, so the targets are the same
// floats as the host conversion's. The file builds without multiply-add
// contraction.
#include "gsr_kernels.h"

namespace gsr {

namespace {

struct FrameDesc {
  uint64_t src;  // byte offset of the frame
  uint64_t dst;  // float offset of the view's [H,W,3] target
  uint32_t sw, sh, dw, dh;
};
struct FrameBlock {
  FrameDesc f[kMaxViews];
};

constexpr int kFrameThreads = 256;

__global__ void __launch_bounds__(kFrameThreads) frames_to_targets_kernel(const uint8_t* frames, float* out,
                                                                          FrameBlock blk) {
  const FrameDesc d = blk.f[blockIdx.y];
  const uint64_t p = (uint64_t)blockIdx.x * kFrameThreads + threadIdx.x;
  if (p >= (uint64_t)d.dw * d.dh) return;
  const uint8_t* src = frames + d.src;
  float* dst = out + d.dst + p * 3;
  if (d.sw == d.dw && d.sh == d.dh) {
#pragma unroll
    for (int c = 0; c < 3; ++c) dst[c] = (float)src[p * 3 + c] / 255.0f;
    return;
  }
  // resize_rgb: output pixel (dx, dy) averages the source pixels
  // [sx0, sx1) x [sy0, sy1), at least one, clamped to the frame.
  const uint64_t dy = p / d.dw, dx = p % d.dw;
  const uint64_t sy0 = dy * d.sh / d.dh;
  const uint64_t sy1 = min(max((dy + 1) * d.sh / d.dh, sy0 + 1), (uint64_t)d.sh);
  const uint64_t sx0 = dx * d.sw / d.dw;
  const uint64_t sx1 = min(max((dx + 1) * d.sw / d.dw, sx0 + 1), (uint64_t)d.sw);
  float acc[3] = {0.f, 0.f, 0.f};
  uint32_t count = 0;
  for (uint64_t sy = sy0; sy < sy1; ++sy)
    for (uint64_t sx = sx0; sx < sx1; ++sx) {
      const uint8_t* s = src + (sy * d.sw + sx) * 3;
#pragma unroll
      for (int c = 0; c < 3; ++c) acc[c] = acc[c] + (float)s[c] / 255.0f;
      ++count;
    }
  const float inv = 1.0f / (float)(count > 0 ? count : 1);
#pragma unroll
  for (int c = 0; c < 3; ++c) dst[c] = acc[c] * inv;
}

}  // namespace

cudaError_t launch_frames_to_targets(const uint8_t* frames, const FrameSpec* spec, uint32_t n_views, float* out,
                                     cudaStream_t st) {
  if (n_views == 0) return cudaSuccess;
  if (n_views > (uint32_t)kMaxViews) return cudaErrorInvalidValue;
  FrameBlock blk{};
  uint64_t pmax = 0, dst = 0;
  for (uint32_t v = 0; v < n_views; ++v) {
    FrameDesc& d = blk.f[v];
    d.src = spec[v].src_offset;
    d.dst = dst;
    d.sw = spec[v].src_w;
    d.sh = spec[v].src_h;
    d.dw = spec[v].dst_w;
    d.dh = spec[v].dst_h;
    const uint64_t P = (uint64_t)d.dw * d.dh;
    dst += P * 3;
    if (P > pmax) pmax = P;
  }
  if (pmax == 0) return cudaSuccess;
  const uint64_t bx = (pmax + kFrameThreads - 1) / kFrameThreads;
  if (bx > 0x7fffffffull) return cudaErrorInvalidValue;
  frames_to_targets_kernel<<<dim3((unsigned)bx, n_views), kFrameThreads, 0, st>>>(frames, out, blk);
  return cudaGetLastError();
}

}  // namespace gsr
