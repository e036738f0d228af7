// k_raster.cu — front-to-back blending (rasterize.wgsl:21-99) and its
// reverse-walk adjoint.
//
// One CTA per (view, tile) work item across all views of the launch. Each
// warp owns an 8 x 4*PPL pixel block of the tile; each lane owns PPL pixels
// of one column (rows y, y+4, ...), so the per-Gaussian terms a*dx*dx and
// 2b*dx are formed once for all of them. The tile's depth-sorted list is staged in
// shared memory batch by batch; while staging, every Gaussian's padded
// axis-aligned box of its {sigma <= log(255*opacity) + 1e-3} ellipse
// (footprint_box, written into the record by the emission kernel) gives a
// bit per warp block it can reach.
// Each warp then walks, in order, only the Gaussians whose bit it holds
// (ballot compaction into a per-warp list). The box is conservative and
// sigma is evaluated with the same expression tree as the oracle, so every
// contributor decision is unchanged: culled Gaussians could not pass the
// alpha >= 1/255 test (see kRejectMargin).
//
// The forward records per pixel the final transmittance and the list index
// of the last contributor. The backward walks the same per-warp lists from
// the tile's largest last index down, recovers the transmittance before each
// contributor by division (T_i = T_{i+1} / (1 - alpha_i)), keeps the colour
// accumulated behind it, and forms per-pixel gradients (blend_step_grad).
// Per Gaussian the gradient sums over a warp's pixels come from a
// reduce-scatter butterfly (16 shuffles), over the CTA's warps from shared
// memory in warp order, and over tiles from float4 atomics (or, in
// deterministic mode, per-intersection records reduced later in a fixed
// order).
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

// Warp w of a TW-wide tile owns the 8 x (4*PPL) block at (x0, y0); lane l
// owns column x0 + (l & 7) and rows y0 + (l >> 3) + 4q, q = 0..PPL-1.
template <int TW, int PPL> struct WarpBlock {
  static constexpr int kWarpsX = TW / 8;
  static constexpr int kRows = 4 * PPL;
  __device__ static int x0(int w) { return (w % kWarpsX) * 8; }
  __device__ static int y0(int w) { return (w / kWarpsX) * kRows; }
};

// Stages one Gaussian: records in shared memory plus the bit mask of warp
// blocks its padded footprint box overlaps (half-widths written by the
// emission kernel into r2.zw; negative means no box, never cull). The
// forward stages colours clamped at zero, the backward raw colours.
template <int TW, int PPL, int NW, bool CLAMP>
__device__ __forceinline__ uint32_t stage_one(const float4* rec, uint32_t c, float tx0, float ty0, float4& A, float4& B,
                                              float4& Cc) {
  const float4 r0 = rec[(size_t)c * 3 + 0];
  const float4 r1 = rec[(size_t)c * 3 + 1];
  const float4 r2 = rec[(size_t)c * 3 + 2];
  A = make_float4(r0.x, r0.y, r0.z, 2.f * r0.w);  // 2b is exact
  B = make_float4(r1.x, r2.y + kRejectMargin, r1.y, 0.f);
  Cc = CLAMP ? make_float4(fmaxf(r1.z, 0.f), fmaxf(r1.w, 0.f), fmaxf(r2.x, 0.f), 0.f)
             : make_float4(r1.z, r1.w, r2.x, 0.f);
  const float rx = r2.z, ry = r2.w;
  if (!(rx >= 0.f) || !(ry >= 0.f)) return (1u << NW) - 1u;
  uint32_t mask = 0;
  constexpr float kSpanY = (float)(4 * PPL - 1);
#pragma unroll
  for (int w = 0; w < NW; ++w) {
    const float bx0 = tx0 + (float)WarpBlock<TW, PPL>::x0(w) + 0.5f;
    const float by0 = ty0 + (float)WarpBlock<TW, PPL>::y0(w) + 0.5f;
    const bool out = (r0.x + rx < bx0) || (r0.x - rx > bx0 + 7.f) || (r0.y + ry < by0) || (r0.y - ry > by0 + kSpanY);
    if (!out) mask |= 1u << w;
  }
  return mask;
}

// Order-preserving compaction of the batch entries whose mask has bit w.
__device__ __forceinline__ int build_list(const uint8_t* s_mask, uint32_t nb, int w, int lane, uint16_t* list) {
  int cnt = 0;
  for (uint32_t base = 0; base < nb; base += 32) {
    const uint32_t j = base + lane;
    const bool bit = j < nb && ((s_mask[j] >> w) & 1u);
    const uint32_t bal = __ballot_sync(0xffffffffu, bit);
    if (bit) list[cnt + __popc(bal & ((1u << lane) - 1u))] = (uint16_t)j;
    cnt += __popc(bal);
  }
  __syncwarp();
  return cnt;
}

template <int TW, int TH, int PPL, int BATCH>
__global__ void __launch_bounds__(TW* TH / PPL) raster_fwd_kernel(RasterArgs a) {
  constexpr int NT = TW * TH / PPL;
  constexpr int NW = NT / 32;
  __shared__ float4 s_a[BATCH];  // x, y, conic a, 2 conic b
  __shared__ float4 s_b[BATCH];  // conic c, reject cut, opacity, -
  __shared__ float4 s_c[BATCH];  // max(r,0), max(g,0), max(b,0), -
  __shared__ uint32_t s_cidx[BATCH];
  __shared__ uint8_t s_mask[BATCH];
  __shared__ uint8_t s_hit[BATCH];
  __shared__ uint16_t s_list[NW][BATCH];
  const uint32_t item = blockIdx.x;
  const uint32_t v = find_view(a.vs, item);
  const ViewDesc& vd = a.vs.views[v];
  const uint32_t t = item - vd.tile_base;
  const uint32_t tx = t % vd.tiles_x, ty = t / vd.tiles_x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t px = tx * TW + WarpBlock<TW, PPL>::x0(warp) + (lane & 7);
  const uint32_t pyb = ty * TH + WarpBlock<TW, PPL>::y0(warp) + (lane >> 3);
  const float pcx = (float)px + 0.5f;
  const uint32_t* ranges = slice(a.b.ranges, 2 * a.b.Tcap, v);
  const uint32_t s0 = ranges[2 * t], s1 = ranges[2 * t + 1];
  const uint32_t* vals = slice(a.b.isect_val, a.b.Icap, v);
  const float4* rec = slice(a.b.rec, a.b.Vcap * 3, v);
  uint8_t* vis = slice(a.b.visible_c, a.b.Vcap, v);
  const float tx0 = (float)(tx * TW), ty0 = (float)(ty * TH);
  float T[PPL], C0[PPL], C1[PPL], C2[PPL], pcy[PPL];
  uint32_t last[PPL], nc[PPL], stop[PPL];
  bool done[PPL];
  bool all_done = true;
#pragma unroll
  for (int q = 0; q < PPL; ++q) {
    const uint32_t py = pyb + 4 * q;
    T[q] = 1.f;
    C0[q] = C1[q] = C2[q] = 0.f;
    pcy[q] = (float)py + 0.5f;
    last[q] = nc[q] = 0;
    stop[q] = s1;
    done[q] = !(px < vd.w && py < vd.h);
    all_done = all_done && done[q];
  }
  for (uint32_t b0 = s0; b0 < s1; b0 += BATCH) {
    const uint32_t nb = min((uint32_t)BATCH, s1 - b0);
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < nb; j += NT) {
      const uint32_t c = vals[b0 + j];
      float4 A, B, Cc;
      s_mask[j] = (uint8_t)stage_one<TW, PPL, NW, true>(rec, c, tx0, ty0, A, B, Cc);
      s_a[j] = A;
      s_b[j] = B;
      s_c[j] = Cc;
      s_cidx[j] = c;
      s_hit[j] = 0;
    }
    __syncthreads();
    if (!__all_sync(0xffffffffu, all_done)) {
      const int cnt = build_list(s_mask, nb, warp, lane, s_list[warp]);
      for (int k = 0; k < cnt; ++k) {
        const uint32_t j = s_list[warp][k];
        const float4 A = s_a[j];
        const float4 B = s_b[j];
        const float dx = esub(A.x, pcx);
        const float t1 = emul(emul(A.z, dx), dx);
        const float t2 = emul(A.w, dx);
#pragma unroll
        for (int q = 0; q < PPL; ++q) {
          if (done[q]) continue;
          const float dy = esub(A.y, pcy[q]);
          // blend_sigma's expression tree with a*dx*dx and 2b*dx shared.
          const float sigma = blend_sigma_shared(t1, t2, dy, B.x);
          if (sigma > B.y) continue;
          float gauss;
          const float alpha = blend_alpha_of(sigma, B.z, gauss);
          if (alpha < 0.f) continue;
          const float4 Cc = s_c[j];
          const float w = emul(alpha, T[q]);
          C0[q] = fmaf(Cc.x, w, C0[q]);  // blend_accum; Cc was clamped at staging
          C1[q] = fmaf(Cc.y, w, C1[q]);
          C2[q] = fmaf(Cc.z, w, C2[q]);
          T[q] = emul(T[q], esub(1.f, alpha));
          last[q] = b0 + j + 1;
          ++nc[q];
          s_hit[j] = 1;
          if (T[q] < 1e-4f) {
            done[q] = true;
            stop[q] = b0 + j + 1;
          }
        }
        all_done = true;
#pragma unroll
        for (int q = 0; q < PPL; ++q) all_done = all_done && done[q];
        if (__all_sync(0xffffffffu, all_done)) break;
      }
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < nb; j += NT)
      if (s_hit[j]) vis[s_cidx[j]] = 1;
    if (__syncthreads_and(all_done)) break;
  }
  float4* out = reinterpret_cast<float4*>(a.out_rgba) + vd.pix_base;
#pragma unroll
  for (int q = 0; q < PPL; ++q) {
    const uint32_t py = pyb + 4 * q;
    if (!(px < vd.w && py < vd.h)) continue;
    const size_t pix = (size_t)py * vd.w + px;
    out[pix] = make_float4(C0[q] + T[q] * a.bg[0], C1[q] + T[q] * a.bg[1], C2[q] + T[q] * a.bg[2], 1.f - T[q]);
    slice(a.b.tfinal, a.b.Pcap, v)[pix] = T[q];
    slice(a.b.last, a.b.Pcap, v)[pix] = last[q];
    slice(a.b.ncontrib, a.b.Pcap, v)[pix] = nc[q];
    slice(a.b.nvisit, a.b.Pcap, v)[pix] = stop[q] - s0;
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

// Per-pixel state of the reverse walk.
struct BwdPixel {
  uint32_t last;
  float T, K;
  float vrgb[3];
  float S[3];
};

__device__ __forceinline__ void load_bwd_pixel(const RasterArgs& a, const ViewDesc& vd, uint32_t v, uint32_t px,
                                               uint32_t py, BwdPixel& p) {
  p.last = 0;
  p.T = 1.f;
  p.K = 0.f;
  p.vrgb[0] = p.vrgb[1] = p.vrgb[2] = 0.f;
  p.S[0] = p.S[1] = p.S[2] = 0.f;
  if (!(px < vd.w && py < vd.h)) return;
  const size_t pix = (size_t)py * vd.w + px;
  p.last = slice(a.b.last, a.b.Pcap, v)[pix];
  p.T = slice(a.b.tfinal, a.b.Pcap, v)[pix];
  const float4 g = reinterpret_cast<const float4*>(a.v_rgba)[vd.pix_base + pix];
  p.vrgb[0] = g.x;
  p.vrgb[1] = g.y;
  p.vrgb[2] = g.z;
  p.K = (g.x * a.bg[0] + g.y * a.bg[1] + g.z * a.bg[2] - g.w) * p.T;
}

// One pixel's step of the reverse walk; adds its gradient into x[0..11)
// (the contributor count is taken from a ballot).
__device__ __forceinline__ bool bwd_step(BwdPixel& p, uint32_t s, float dx, float t1, float t2, float pcy,
                                         const float4& A, const float4& B, const float4& Cc, int ref_mode,
                                         float (&x)[16]) {
  if (s >= p.last) return false;
  const float dy = esub(A.y, pcy);
  const float sigma = blend_sigma_shared(t1, t2, dy, B.x);
  if (sigma > B.y) return false;
  float gauss;
  const float alpha = blend_alpha_of(sigma, B.z, gauss);
  if (alpha < 0.f) return false;
  const bool skip = ref_mode && (p.T <= 1e-4f);
  SplatGrad<float> g;
  blend_step_grad(dx, dy, A.z, 0.5f * A.w, B.x, Cc.x, Cc.y, Cc.z, B.z, gauss, alpha, p.T, p.S, p.vrgb, p.K, skip, g);
  if (skip) return false;
  x[0] += g.v_xy[0];
  x[1] += g.v_xy[1];
  x[2] += g.v_conic[0];
  x[3] += g.v_conic[1];
  x[4] += g.v_conic[2];
  x[5] += g.v_rgb[0];
  x[6] += g.v_rgb[1];
  x[7] += g.v_rgb[2];
  x[8] += g.v_opac;
  x[9] += g.abs_xy[0];
  x[10] += g.abs_xy[1];
  return true;
}

template <int TW, int TH, int PPL, int BATCH>
__global__ void __launch_bounds__(TW* TH / PPL) raster_bwd_kernel(RasterArgs a) {
  constexpr int NT = TW * TH / PPL;
  constexpr int NW = NT / 32;
  __shared__ float4 s_a[BATCH];
  __shared__ float4 s_b[BATCH];
  __shared__ float4 s_c[BATCH];
  __shared__ uint32_t s_cidx[BATCH];
  __shared__ uint8_t s_mask[BATCH];
  __shared__ uint16_t s_list[NW][BATCH];
  __shared__ float s_part[NW][BATCH][12];
  __shared__ uint32_t s_max;
  const uint32_t item = blockIdx.x;
  const uint32_t v = find_view(a.vs, item);
  const ViewDesc& vd = a.vs.views[v];
  const uint32_t t = item - vd.tile_base;
  const uint32_t tx = t % vd.tiles_x, ty = t / vd.tiles_x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t px = tx * TW + WarpBlock<TW, PPL>::x0(warp) + (lane & 7);
  const uint32_t pyb = ty * TH + WarpBlock<TW, PPL>::y0(warp) + (lane >> 3);
  const float pcx = (float)px + 0.5f;
  const uint32_t* ranges = slice(a.b.ranges, 2 * a.b.Tcap, v);
  const uint32_t s0 = ranges[2 * t];
  const uint32_t* vals = slice(a.b.isect_val, a.b.Icap, v);
  const float4* rec = slice(a.b.rec, a.b.Vcap * 3, v);
  float4* sgrad = slice(a.b.sgrad, a.b.Vcap * 3, v);
  float* part = a.b.sgrad_part + (size_t)a.b.Icap * 12 * v;
  const float tx0 = (float)(tx * TW), ty0 = (float)(ty * TH);
  BwdPixel pp[PPL];
  uint32_t mylast = 0;
#pragma unroll
  for (int q = 0; q < PPL; ++q) {
    load_bwd_pixel(a, vd, v, px, pyb + 4 * q, pp[q]);
    mylast = max(mylast, pp[q].last);
  }
  if (threadIdx.x == 0) s_max = 0;
  __syncthreads();
  const uint32_t wmax = __reduce_max_sync(0xffffffffu, mylast);
  if (lane == 0) atomicMax(&s_max, wmax);
  __syncthreads();
  const uint32_t smax = s_max;
  for (uint32_t be = smax; be > s0;) {
    const uint32_t bs = (be - s0 > (uint32_t)BATCH) ? be - BATCH : s0;
    const uint32_t nb = be - bs;
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < nb; j += NT) {
      const uint32_t c = vals[bs + j];
      float4 A, B, Cc;
      s_mask[j] = (uint8_t)stage_one<TW, PPL, NW, false>(rec, c, tx0, ty0, A, B, Cc);
      s_a[j] = A;
      s_b[j] = B;
      s_c[j] = Cc;
      s_cidx[j] = c;
    }
    for (uint32_t q = threadIdx.x; q < (uint32_t)NW * nb * 12; q += NT) {
      const uint32_t w = q / (nb * 12), r = q % (nb * 12);
      s_part[w][r / 12][r % 12] = 0.f;
    }
    __syncthreads();
    if (bs < wmax) {
      const int cnt = build_list(s_mask, nb, warp, lane, s_list[warp]);
      for (int k = cnt - 1; k >= 0; --k) {
        const uint32_t j = s_list[warp][k];
        const uint32_t s = bs + j;
        if (s >= wmax) continue;  // warp-uniform
        const float4 A = s_a[j];
        const float4 B = s_b[j];
        const float4 Cc = s_c[j];
        const float dx = esub(A.x, pcx);
        const float t1 = emul(emul(A.z, dx), dx);
        const float t2 = emul(A.w, dx);
        float x[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) x[i] = 0.f;
        uint32_t ncontrib = 0;
#pragma unroll
        for (int q = 0; q < PPL; ++q) {
          const bool c = bwd_step(pp[q], s, dx, t1, t2, (float)(pyb + 4 * q) + 0.5f, A, B, Cc, a.ref_mode, x);
          ncontrib += __popc(__ballot_sync(0xffffffffu, c));
        }
        if (ncontrib) {
          const float r = warp_reduce_scatter16(x, lane);
          const int slot = lane >> 1;
          if ((lane & 1) == 0 && slot < 11) s_part[warp][j][slot] = r;
          if (lane == 0) s_part[warp][j][11] = (float)ncontrib;
        }
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

template <int TW, int TH, int PPL>
cudaError_t launch_fwd_shape(const RasterArgs& a, uint32_t items, cudaStream_t st) {
  raster_fwd_kernel<TW, TH, PPL, 128><<<items, TW * TH / PPL, 0, st>>>(a);
  return cudaGetLastError();
}
template <int TW, int TH, int PPL>
cudaError_t launch_bwd_shape(const RasterArgs& a, uint32_t items, cudaStream_t st) {
  raster_bwd_kernel<TW, TH, PPL, 64><<<items, TW * TH / PPL, 0, st>>>(a);
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
  if (vs.tile_w == 16 && vs.tile_h == 16) return launch_fwd_shape<16, 16, 2>(a, vs.total_tiles, st);
  if (vs.tile_w == 8 && vs.tile_h == 8) return launch_fwd_shape<8, 8, 2>(a, vs.total_tiles, st);
  if (vs.tile_w == 32 && vs.tile_h == 8) return launch_fwd_shape<32, 8, 2>(a, vs.total_tiles, st);
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
  if (vs.tile_w == 16 && vs.tile_h == 16) return launch_bwd_shape<16, 16, 2>(a, vs.total_tiles, st);
  if (vs.tile_w == 8 && vs.tile_h == 8) return launch_bwd_shape<8, 8, 2>(a, vs.total_tiles, st);
  if (vs.tile_w == 32 && vs.tile_h == 8) return launch_bwd_shape<32, 8, 2>(a, vs.total_tiles, st);
  return cudaErrorInvalidValue;
}

}  // namespace gsr
