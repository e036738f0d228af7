// k_raster.cu — front-to-back blending (rasterize.wgsl:21-99) and its
// reverse-walk adjoint.
//
// One CTA per (view, tile) work item across all views of the launch; one
// thread per pixel, warps laid out as 8x4 pixel blocks so that a warp's
// pixels terminate together. Each batch of the tile's depth-sorted list is
// staged in shared memory (three float4 per Gaussian), every pixel walks it,
// and the CTA stops as soon as all its pixels are saturated
// (__syncthreads_and). A Gaussian whose sigma exceeds log(255*opacity) plus
// a margin is rejected before the exponential; that never changes a decision
// (see kRejectMargin), so the contributor sets are those of the oracle.
//
// The forward records per pixel the final transmittance and the list index
// of the last contributor. The backward re-walks each tile from the largest
// last index down, recovers the transmittance before each contributor by
// division (T_i = T_{i+1} / (1 - alpha_i)), keeps the colour accumulated
// behind it, and forms per-pixel gradients (blend_step_grad). Per Gaussian
// the 12 gradient sums over the warp's pixels come from a reduce-scatter
// butterfly (16 shuffles), over the CTA's warps from shared memory in warp
// order, and over tiles from float4 atomics (or, in deterministic mode,
// per-intersection records reduced later in a fixed order).
#include "gsr_kernels.h"

namespace gsr {

namespace {

struct RasterArgs {
  ViewSet vs;
  FwdBufs b;
  float bg[3];
  float* out_rgba;
  const float* v_rgba;
  int ref_mode;
  int det;
};

__device__ __forceinline__ uint32_t find_view(const ViewSet& vs, uint32_t item) {
  uint32_t v = 0;
  for (uint32_t i = 1; i < vs.n_views; ++i)
    if (vs.views[i].tile_base <= item) v = i;
  return v;
}

template <int TW, int TH> struct PixelMap {
  static constexpr int kWarpsX = TW / 8;
  __device__ static void local(int tid, int& lx, int& ly) {
    const int w = tid >> 5, lane = tid & 31;
    lx = (w % kWarpsX) * 8 + (lane & 7);
    ly = (w / kWarpsX) * 4 + (lane >> 3);
  }
};

template <int TW, int TH, int BATCH>
__global__ void __launch_bounds__(TW* TH) raster_fwd_kernel(RasterArgs a) {
  constexpr int NT = TW * TH;
  __shared__ float4 s_a[BATCH];  // x, y, conic a, conic b
  __shared__ float4 s_b[BATCH];  // conic c, reject cut, opacity, -
  __shared__ float4 s_c[BATCH];  // r, g, b, -
  __shared__ uint32_t s_cidx[BATCH];
  __shared__ int s_hit[BATCH];
  const uint32_t item = blockIdx.x;
  const uint32_t v = find_view(a.vs, item);
  const ViewDesc& vd = a.vs.views[v];
  const uint32_t t = item - vd.tile_base;
  const uint32_t tx = t % vd.tiles_x, ty = t / vd.tiles_x;
  int lx, ly;
  PixelMap<TW, TH>::local(threadIdx.x, lx, ly);
  const uint32_t px = tx * TW + lx, py = ty * TH + ly;
  const bool inside = px < vd.w && py < vd.h;
  const float pcx = (float)px + 0.5f, pcy = (float)py + 0.5f;
  const uint32_t* ranges = slice(a.b.ranges, 2 * a.b.Tcap, v);
  const uint32_t s0 = ranges[2 * t], s1 = ranges[2 * t + 1];
  const uint32_t* vals = slice(a.b.isect_val, a.b.Icap, v);
  const float4* rec = slice(a.b.rec, a.b.Vcap * 3, v);
  uint8_t* vis = slice(a.b.visible_c, a.b.Vcap, v);
  float T = 1.f, C0 = 0.f, C1 = 0.f, C2 = 0.f;
  uint32_t last = 0, nc = 0, stop = s1;
  bool done = !inside;
  for (uint32_t b0 = s0; b0 < s1; b0 += BATCH) {
    const uint32_t nb = min((uint32_t)BATCH, s1 - b0);
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < nb; j += NT) {
      const uint32_t c = vals[b0 + j];
      const float4 r0 = rec[(size_t)c * 3 + 0];
      const float4 r1 = rec[(size_t)c * 3 + 1];
      const float4 r2 = rec[(size_t)c * 3 + 2];
      s_a[j] = r0;
      s_b[j] = make_float4(r1.x, r2.y + kRejectMargin, r1.y, 0.f);
      s_c[j] = make_float4(r1.z, r1.w, r2.x, 0.f);
      s_cidx[j] = c;
      s_hit[j] = 0;
    }
    __syncthreads();
    if (!done) {
      for (uint32_t j = 0; j < nb; ++j) {
        const float4 A = s_a[j];
        const float4 B = s_b[j];
        const float sigma = blend_sigma(A.x - pcx, A.y - pcy, A.z, A.w, B.x);
        if (sigma > B.y) continue;
        float gauss;
        const float alpha = blend_alpha_of(sigma, B.z, gauss);
        if (alpha < 0.f) continue;
        const float4 Cc = s_c[j];
        const float visw = alpha * T;
        C0 = C0 + fmaxf(Cc.x, 0.f) * visw;
        C1 = C1 + fmaxf(Cc.y, 0.f) * visw;
        C2 = C2 + fmaxf(Cc.z, 0.f) * visw;
        T = T * (1.f - alpha);
        last = b0 + j + 1;
        ++nc;
        s_hit[j] = 1;
        if (T < 1e-4f) {
          done = true;
          stop = b0 + j + 1;
          break;
        }
      }
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < nb; j += NT)
      if (s_hit[j]) vis[s_cidx[j]] = 1;
    if (__syncthreads_and(done)) break;
  }
  if (inside) {
    const size_t pix = (size_t)py * vd.w + px;
    float4* out = reinterpret_cast<float4*>(a.out_rgba) + vd.pix_base + pix;
    *out = make_float4(C0 + T * a.bg[0], C1 + T * a.bg[1], C2 + T * a.bg[2], 1.f - T);
    slice(a.b.tfinal, a.b.Pcap, v)[pix] = T;
    slice(a.b.last, a.b.Pcap, v)[pix] = last;
    slice(a.b.ncontrib, a.b.Pcap, v)[pix] = nc;
    slice(a.b.nvisit, a.b.Pcap, v)[pix] = stop - s0;
  }
}

// Reduce-scatter of 16 per-lane values over the warp: returns in every lane
// the warp total of slot (lane >> 1). Summation order is fixed.
__device__ __forceinline__ float warp_reduce_scatter16(float (&x)[16], int lane) {
  const uint32_t full = 0xffffffffu;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const bool hi = lane & 16;
    const float send = hi ? x[i] : x[i + 8];
    const float keep = hi ? x[i + 8] : x[i];
    x[i] = keep + __shfl_xor_sync(full, send, 16);
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const bool hi = lane & 8;
    const float send = hi ? x[i] : x[i + 4];
    const float keep = hi ? x[i + 4] : x[i];
    x[i] = keep + __shfl_xor_sync(full, send, 8);
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const bool hi = lane & 4;
    const float send = hi ? x[i] : x[i + 2];
    const float keep = hi ? x[i + 2] : x[i];
    x[i] = keep + __shfl_xor_sync(full, send, 4);
  }
  {
    const bool hi = lane & 2;
    const float send = hi ? x[0] : x[1];
    const float keep = hi ? x[1] : x[0];
    x[0] = keep + __shfl_xor_sync(full, send, 2);
  }
  return x[0] + __shfl_xor_sync(full, x[0], 1);
}

template <int TW, int TH, int BATCH>
__global__ void __launch_bounds__(TW* TH) raster_bwd_kernel(RasterArgs a) {
  constexpr int NT = TW * TH;
  constexpr int NW = NT / 32;
  __shared__ float4 s_a[BATCH];
  __shared__ float4 s_b[BATCH];
  __shared__ float4 s_c[BATCH];
  __shared__ uint32_t s_cidx[BATCH];
  __shared__ float s_part[NW][BATCH][12];
  __shared__ uint32_t s_max;
  const uint32_t item = blockIdx.x;
  const uint32_t v = find_view(a.vs, item);
  const ViewDesc& vd = a.vs.views[v];
  const uint32_t t = item - vd.tile_base;
  const uint32_t tx = t % vd.tiles_x, ty = t / vd.tiles_x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int lx, ly;
  PixelMap<TW, TH>::local(threadIdx.x, lx, ly);
  const uint32_t px = tx * TW + lx, py = ty * TH + ly;
  const bool inside = px < vd.w && py < vd.h;
  const float pcx = (float)px + 0.5f, pcy = (float)py + 0.5f;
  const uint32_t* ranges = slice(a.b.ranges, 2 * a.b.Tcap, v);
  const uint32_t s0 = ranges[2 * t];
  const uint32_t* vals = slice(a.b.isect_val, a.b.Icap, v);
  const float4* rec = slice(a.b.rec, a.b.Vcap * 3, v);
  float4* sgrad = slice(a.b.sgrad, a.b.Vcap * 3, v);
  float* part = a.b.sgrad_part + (size_t)a.b.Icap * 12 * v;
  uint32_t last = 0;
  float T = 1.f, K = 0.f;
  float vrgb[3] = {0.f, 0.f, 0.f};
  float S[3] = {0.f, 0.f, 0.f};
  if (inside) {
    const size_t pix = (size_t)py * vd.w + px;
    last = slice(a.b.last, a.b.Pcap, v)[pix];
    T = slice(a.b.tfinal, a.b.Pcap, v)[pix];
    const float4 g = reinterpret_cast<const float4*>(a.v_rgba)[vd.pix_base + pix];
    vrgb[0] = g.x;
    vrgb[1] = g.y;
    vrgb[2] = g.z;
    K = (vrgb[0] * a.bg[0] + vrgb[1] * a.bg[1] + vrgb[2] * a.bg[2] - g.w) * T;
  }
  if (threadIdx.x == 0) s_max = 0;
  __syncthreads();
  const uint32_t wmax = __reduce_max_sync(0xffffffffu, last);
  if (lane == 0) atomicMax(&s_max, wmax);
  __syncthreads();
  const uint32_t smax = s_max;
  for (uint32_t be = smax; be > s0;) {
    const uint32_t bs = (be - s0 > (uint32_t)BATCH) ? be - BATCH : s0;
    const uint32_t nb = be - bs;
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < nb; j += NT) {
      const uint32_t c = vals[bs + j];
      const float4 r0 = rec[(size_t)c * 3 + 0];
      const float4 r1 = rec[(size_t)c * 3 + 1];
      const float4 r2 = rec[(size_t)c * 3 + 2];
      s_a[j] = r0;
      s_b[j] = make_float4(r1.x, r2.y + kRejectMargin, r1.y, 0.f);
      s_c[j] = make_float4(r1.z, r1.w, r2.x, 0.f);
      s_cidx[j] = c;
    }
    __syncthreads();
    for (int j = (int)nb - 1; j >= 0; --j) {
      const uint32_t s = bs + (uint32_t)j;
      SplatGrad<float> g;
      bool contrib = false;
      if (s < last) {
        const float4 A = s_a[j];
        const float4 B = s_b[j];
        const float dx = A.x - pcx, dy = A.y - pcy;
        const float sigma = blend_sigma(dx, dy, A.z, A.w, B.x);
        if (sigma <= B.y) {
          float gauss;
          const float alpha = blend_alpha_of(sigma, B.z, gauss);
          if (alpha >= 0.f) {
            const float4 Cc = s_c[j];
            const bool skip = a.ref_mode && (T <= 1e-4f);
            blend_step_grad(dx, dy, A.z, A.w, B.x, Cc.x, Cc.y, Cc.z, B.z, gauss, alpha, T, S, vrgb, K, skip, g);
            contrib = !skip;
          }
        }
      }
      if (__any_sync(0xffffffffu, contrib)) {
        float x[16];
        if (contrib) {
          x[0] = g.v_xy[0];
          x[1] = g.v_xy[1];
          x[2] = g.v_conic[0];
          x[3] = g.v_conic[1];
          x[4] = g.v_conic[2];
          x[5] = g.v_rgb[0];
          x[6] = g.v_rgb[1];
          x[7] = g.v_rgb[2];
          x[8] = g.v_opac;
          x[9] = g.abs_xy[0];
          x[10] = g.abs_xy[1];
          x[11] = g.count;
        } else {
#pragma unroll
          for (int k = 0; k < 12; ++k) x[k] = 0.f;
        }
        x[12] = x[13] = x[14] = x[15] = 0.f;
        const float r = warp_reduce_scatter16(x, lane);
        const int slot = lane >> 1;
        if ((lane & 1) == 0 && slot < 12) s_part[warp][j][slot] = r;
      } else if (lane < 12) {
        s_part[warp][j][lane] = 0.f;
      }
    }
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < nb * 3; q += NT) {
      const uint32_t j = q / 3, k = q % 3;
      float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int w = 0; w < NW; ++w) {
        f.x = f.x + s_part[w][j][4 * k + 0];
        f.y = f.y + s_part[w][j][4 * k + 1];
        f.z = f.z + s_part[w][j][4 * k + 2];
        f.w = f.w + s_part[w][j][4 * k + 3];
      }
      if (a.det) {
        reinterpret_cast<float4*>(part + (size_t)(bs + j) * 12)[k] = f;
      } else if (f.x != 0.f || f.y != 0.f || f.z != 0.f || f.w != 0.f) {
        atomicAdd(sgrad + (size_t)s_cidx[j] * 3 + k, f);
      }
    }
    be = bs;
  }
  // Deterministic mode: list entries of this tile that no pixel reached keep
  // zero partial records.
  if (a.det) {
    const uint32_t s1 = ranges[2 * t + 1];
    for (uint32_t s = smax > s0 ? smax : s0; s + threadIdx.x < s1; s += NT) {
      float4* p4 = reinterpret_cast<float4*>(part + (size_t)(s + threadIdx.x) * 12);
      p4[0] = p4[1] = p4[2] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
}

template <int TW, int TH>
cudaError_t launch_fwd_shape(const RasterArgs& a, uint32_t items, cudaStream_t st) {
  raster_fwd_kernel<TW, TH, 256><<<items, TW * TH, 0, st>>>(a);
  return cudaGetLastError();
}
template <int TW, int TH>
cudaError_t launch_bwd_shape(const RasterArgs& a, uint32_t items, cudaStream_t st) {
  raster_bwd_kernel<TW, TH, 64><<<items, TW * TH, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_raster_fwd(const ViewSet& vs, FwdBufs& b, const float* bg, float* out_rgba, const Scratch& s,
                              cudaStream_t st) {
  (void)s;
  RasterArgs a{};
  a.vs = vs;
  a.b = b;
  a.bg[0] = bg[0];
  a.bg[1] = bg[1];
  a.bg[2] = bg[2];
  a.out_rgba = out_rgba;
  cudaError_t e = cudaMemsetAsync(b.visible_c, 0, b.Vcap * vs.n_views, st);
  if (e != cudaSuccess) return e;
  if (vs.total_tiles == 0) return cudaSuccess;
  if (vs.tile_w == 16 && vs.tile_h == 16) return launch_fwd_shape<16, 16>(a, vs.total_tiles, st);
  if (vs.tile_w == 8 && vs.tile_h == 8) return launch_fwd_shape<8, 8>(a, vs.total_tiles, st);
  if (vs.tile_w == 32 && vs.tile_h == 8) return launch_fwd_shape<32, 8>(a, vs.total_tiles, st);
  return cudaErrorInvalidValue;
}

cudaError_t launch_raster_bwd(const ViewSet& vs, FwdBufs& b, const float* bg, const float* v_rgba, int ref_mode,
                              int deterministic, const Scratch& s, cudaStream_t st) {
  (void)s;
  RasterArgs a{};
  a.vs = vs;
  a.b = b;
  a.bg[0] = bg[0];
  a.bg[1] = bg[1];
  a.bg[2] = bg[2];
  a.v_rgba = v_rgba;
  a.ref_mode = ref_mode;
  a.det = deterministic;
  if (!deterministic) {
    cudaError_t e = cudaMemsetAsync(b.sgrad, 0, sizeof(float4) * 3 * b.Vcap * vs.n_views, st);
    if (e != cudaSuccess) return e;
  }
  if (vs.total_tiles == 0) return cudaSuccess;
  if (vs.tile_w == 16 && vs.tile_h == 16) return launch_bwd_shape<16, 16>(a, vs.total_tiles, st);
  if (vs.tile_w == 8 && vs.tile_h == 8) return launch_bwd_shape<8, 8>(a, vs.total_tiles, st);
  if (vs.tile_w == 32 && vs.tile_h == 8) return launch_bwd_shape<32, 8>(a, vs.total_tiles, st);
  return cudaErrorInvalidValue;
}

}  // namespace gsr
