// k_loss.cu — 0.8 * L1 + 0.2 * (1 - SSIM) and its gradient
// (engine/loss.rs:42-76, 112-142, 233-276, default settings).
//
// SSIM uses an 11-tap sigma-1.5 normalised Gaussian window applied
// separably (horizontal, then vertical) with replicate padding, C1 = 1e-4,
// C2 = 9e-4 and denominators clamped at 1e-8. The reference builds it from
// ~10 burn ops and differentiates through burn autodiff; here two tiled
// kernels do the work:
//  pass 1: per 32x32 output tile and channel, the four blurred moments in
//          shared memory, the SSIM map, its partial derivatives with respect
//          to (mu_x, E[x^2], E[xy]) and per-tile partial sums of SSIM and L1;
//  pass 2: the adjoint of the padded separable blur applied to the three
//          partial maps, combined with the L1 sign into d loss / d pred.
// A last kernel reduces the per-tile sums in a fixed order (double).
#include "gsr_kernels.h"

namespace gsr {

namespace {

constexpr int LTX = 32, LTY = 32, R = 5, WIN = 11;
constexpr int HX = LTX + 2 * R, HY = LTY + 2 * R;
constexpr int kLT = 256;                          // threads per loss block
constexpr int kHaloIt = (HX * HY + kLT - 1) / kLT;  // halo elements per thread

struct LossArgs {
  const ViewDesc* views;
  const float* pred;    // RGBA per view (pix_base)
  const float* target;  // RGB per view (pix_base)
  float* v_pred;
  float* maps;          // [view][3 ch][3 maps][Pcap]
  float* partial;       // [view][3 ch][tiles][2]
  uint64_t Pcap;
  uint32_t tiles_cap;
  float k[WIN];
  float l1_w, ssim_w;
};

__device__ __forceinline__ int clampi(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// Pass 1. Shared memory holds the two input planes (x, y) of the
// replicate-padded halo, then the four horizontally blurred planes (x, y,
// x^2 + y^2, xy; the products are formed as the row is read). SSIM needs
// E[x^2] and E[y^2] only through their sum (in sigma_x^2 + sigma_y^2), and
// its derivatives with respect to both are equal, so one blurred plane
// carries the sum. Each thread
// blurs two adjacent columns at once with paired FP32 arithmetic, sliding
// one load per tap along the row (horizontal) or down the column pair
// (vertical, two output rows per thread).
struct SsimFwdSmem {
  float p[2][HY][HX];
  float h[4][HY][LTX];
  float red[2][8];
};

__global__ void __launch_bounds__(kLT, 5) ssim_fwd_kernel(LossArgs a) {
  extern __shared__ float4 smem_raw[];
  SsimFwdSmem& S = *reinterpret_cast<SsimFwdSmem*>(smem_raw);
  const uint32_t v = blockIdx.z, ch = blockIdx.y;
  const ViewDesc& vd = a.views[v];
  const int W = (int)vd.w, H = (int)vd.h;
  const int tiles_x = (W + LTX - 1) / LTX, tiles_y = (H + LTY - 1) / LTY;
  const int tile = blockIdx.x;
  if (tile >= tiles_x * tiles_y) return;
  const int x0 = (tile % tiles_x) * LTX, y0 = (tile / tiles_x) * LTY;
  const float* pred = a.pred + vd.pix_base * 4;
  const float* tgt = a.target + vd.pix_base * 3;
  {
    // All of a thread's halo loads are issued before the first store.
    float xs[kHaloIt], ys[kHaloIt];
#pragma unroll
    for (int it = 0; it < kHaloIt; ++it) {
      const int i = threadIdx.x + it * kLT;
      if (i < HX * HY) {
        const int hy = i / HX, hx = i % HX;
        const int gx = clampi(x0 + hx - R, 0, W - 1), gy = clampi(y0 + hy - R, 0, H - 1);
        const size_t p = (size_t)gy * W + gx;
        xs[it] = pred[p * 4 + ch];
        ys[it] = tgt[p * 3 + ch];
      }
    }
#pragma unroll
    for (int it = 0; it < kHaloIt; ++it) {
      const int i = threadIdx.x + it * kLT;
      if (i < HX * HY) {
        const int hy = i / HX, hx = i % HX;
        S.p[0][hy][hx] = xs[it];
        S.p[1][hy][hx] = ys[it];
      }
    }
  }
  __syncthreads();
  // Horizontal pass: every halo row, output columns in pairs; the four
  // moment values of each input are formed once from x and y.
  for (int i = threadIdx.x; i < HY * (LTX / 2); i += blockDim.x) {
    const int hy = i / (LTX / 2), ox = 2 * (i % (LTX / 2));
    const float* rx = &S.p[0][hy][ox];
    const float* ry = &S.p[1][hy][ox];
    float2 acc[4];
    float prev[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) acc[m] = f2(0.f);
    {
      const float x = rx[0], y = ry[0];
      prev[0] = x;
      prev[1] = y;
      prev[2] = x * x + y * y;
      prev[3] = x * y;
    }
#pragma unroll
    for (int t = 0; t < WIN; ++t) {
      const float x = rx[t + 1], y = ry[t + 1];
      const float next[4] = {x, y, x * x + y * y, x * y};
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        acc[m] = fma2(f2(a.k[t]), make_float2(prev[m], next[m]), acc[m]);
        prev[m] = next[m];
      }
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) *reinterpret_cast<float2*>(&S.h[m][hy][ox]) = acc[m];
  }
  __syncthreads();
  // Vertical pass and the SSIM map: a column pair times two rows per thread.
  const float C1 = 1e-4f, C2 = 9e-4f;
  float ssum = 0.f, lsum = 0.f;
  float* maps = a.maps + ((size_t)v * 3 + ch) * 3 * a.Pcap;
  {
    const int ox = 2 * (threadIdx.x % (LTX / 2)), oy = 2 * (threadIdx.x / (LTX / 2));  // 16 x 16 tasks
    float2 mo[4][2];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      float2 r0 = f2(0.f), r1 = f2(0.f);
      float2 prev = *reinterpret_cast<const float2*>(&S.h[m][oy][ox]);
#pragma unroll
      for (int t = 0; t < WIN; ++t) {
        const float2 next = *reinterpret_cast<const float2*>(&S.h[m][oy + t + 1][ox]);
        r0 = fma2(f2(a.k[t]), prev, r0);
        r1 = fma2(f2(a.k[t]), next, r1);
        prev = next;
      }
      mo[m][0] = r0;
      mo[m][1] = r1;
    }
#pragma unroll
    for (int ry = 0; ry < 2; ++ry) {
#pragma unroll
      for (int cx = 0; cx < 2; ++cx) {
        const int gx = x0 + ox + cx, gy = y0 + oy + ry;
        if (gx >= W || gy >= H) continue;
        const float mx = cx ? mo[0][ry].y : mo[0][ry].x, my = cx ? mo[1][ry].y : mo[1][ry].x;
        const float ess = cx ? mo[2][ry].y : mo[2][ry].x;  // E[x^2] + E[y^2]
        const float exy = cx ? mo[3][ry].y : mo[3][ry].x;
        const float sxy = exy - mx * my;
        const float A = 2.f * mx * my + C1, B = 2.f * sxy + C2;
        const float Cr = mx * mx + my * my + C1, Dr = ((ess - mx * mx) - my * my) + C2;
        const float Cc = fmaxf(Cr, 1e-8f), Dc = fmaxf(Dr, 1e-8f);
        const float inv = 1.f / (Cc * Dc);
        const float s = (A * B) * inv;
        const float dC = Cr > 1e-8f ? 1.f : 0.f, dD = Dr > 1e-8f ? 1.f : 0.f;
        const float gmx = (2.f * my * B + A * (-2.f * my)) * inv - s * ((2.f * mx * dC) * Dc + Cc * (-2.f * mx * dD)) * inv;
        const size_t p = (size_t)gy * W + gx;
        maps[p] = gmx;
        maps[a.Pcap + p] = -s * dD / Dc;
        maps[2 * a.Pcap + p] = 2.f * A * inv;
        ssum += s;
        lsum += fabsf(S.p[0][oy + ry + R][ox + cx + R] - S.p[1][oy + ry + R][ox + cx + R]);
      }
    }
  }
  // Fixed-order block reduction.
  for (int o = 16; o > 0; o >>= 1) {
    ssum += __shfl_xor_sync(0xffffffffu, ssum, o);
    lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  }
  if ((threadIdx.x & 31) == 0) {
    S.red[0][threadIdx.x >> 5] = ssum;
    S.red[1][threadIdx.x >> 5] = lsum;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float a0 = 0.f, a1 = 0.f;
    for (int w = 0; w < 8; ++w) {
      a0 += S.red[0][w];
      a1 += S.red[1][w];
    }
    float* pp = a.partial + (((size_t)v * 3 + ch) * a.tiles_cap + tile) * 2;
    pp[0] = a0;
    pp[1] = a1;
  }
}

// Weight of output q in the adjoint of a replicate-padded 11-tap
// correlation at input p along an axis of length n (k is symmetric, so for
// interior p it is k[R + q - p]; the border inputs collect the clamped taps).
__device__ __forceinline__ float adj_weight(const float* k, int p, int q, int n) {
  if (p > 0 && p < n - 1) {
    const int d = q - p;
    return (d >= -R && d <= R) ? k[R + d] : 0.f;
  }
  float w = 0.f;
#pragma unroll
  for (int t = 0; t < WIN; ++t)
    if (clampi(q + t - R, 0, n - 1) == p) w += k[t];
  return w;
}

// Pass 2: the adjoint of the padded separable blur on the three partial
// maps (vertical, then horizontal), combined with the L1 sign. Interior
// rows and column pairs take the symmetric-kernel fast path with paired
// arithmetic; rows and columns on the image border use adj_weight.
struct SsimBwdSmem {
  float g[3][HY][HX];
  float v[3][LTY][HX];
};

__global__ void __launch_bounds__(kLT, 5) ssim_bwd_kernel(LossArgs a) {
  extern __shared__ float4 smem_raw[];
  SsimBwdSmem& S = *reinterpret_cast<SsimBwdSmem*>(smem_raw);
  const uint32_t v = blockIdx.z, ch = blockIdx.y;
  const ViewDesc& vd = a.views[v];
  const int W = (int)vd.w, H = (int)vd.h;
  const int tiles_x = (W + LTX - 1) / LTX, tiles_y = (H + LTY - 1) / LTY;
  const int tile = blockIdx.x;
  if (tile >= tiles_x * tiles_y) return;
  const int x0 = (tile % tiles_x) * LTX, y0 = (tile / tiles_x) * LTY;
  const float* maps = a.maps + ((size_t)v * 3 + ch) * 3 * a.Pcap;
  const float* pred = a.pred + vd.pix_base * 4;
  const float* tgt = a.target + vd.pix_base * 3;
  // The prediction and target values of this thread's output pixels (read
  // at the end) are loaded now, with the halo of the three maps.
  constexpr int kOutIt = LTY * (LTX / 2) / kLT;
  float px_x[kOutIt][2], px_y[kOutIt][2];
#pragma unroll
  for (int it = 0; it < kOutIt; ++it) {
    const int i = threadIdx.x + it * kLT;
    const int oy = i / (LTX / 2), ox = 2 * (i % (LTX / 2));
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const int px = x0 + ox + c, py = y0 + oy;
      const bool ok = px < W && py < H;
      const size_t p = (size_t)py * W + px;
      px_x[it][c] = ok ? pred[p * 4 + ch] : 0.f;
      px_y[it][c] = ok ? tgt[p * 3 + ch] : 0.f;
    }
  }
  {
    float gs[kHaloIt][3];
#pragma unroll
    for (int it = 0; it < kHaloIt; ++it) {
      const int i = threadIdx.x + it * kLT;
      const int hy = i / HX, hx = i % HX;
      const int gx = x0 + hx - R, gy = y0 + hy - R;
      const bool ok = i < HX * HY && gx >= 0 && gx < W && gy >= 0 && gy < H;
      const size_t p = (size_t)gy * W + gx;
#pragma unroll
      for (int m = 0; m < 3; ++m) gs[it][m] = ok ? maps[m * a.Pcap + p] : 0.f;
    }
#pragma unroll
    for (int it = 0; it < kHaloIt; ++it) {
      const int i = threadIdx.x + it * kLT;
      if (i < HX * HY) {
        const int hy = i / HX, hx = i % HX;
#pragma unroll
        for (int m = 0; m < 3; ++m) S.g[m][hy][hx] = gs[it][m];
      }
    }
  }
  __syncthreads();
  // Adjoint of the vertical pass: tile rows, all halo columns (in pairs).
  // When every output row and its taps lie strictly inside the image (no
  // border row, no clamped tap), each tap weighs k[R + d] and no check is
  // needed: a thread then slides down a column pair over four output rows,
  // adding each loaded halo row into the rows it reaches (14 loads per plane
  // for 4 rows instead of 44). Every output sums its taps in tap order, as
  // the per-row loop of border tiles does.
  const bool rows_inside = y0 >= R + 1 && y0 + LTY + R <= H - 1;
  if (rows_inside) {
    constexpr int kRows = 4;
    for (int i = threadIdx.x; i < (LTY / kRows) * (HX / 2); i += blockDim.x) {
      const int oy = kRows * (i / (HX / 2)), hx = 2 * (i % (HX / 2));
      float2 acc[3][kRows];
#pragma unroll
      for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int j = 0; j < kRows; ++j) acc[m][j] = f2(0.f);
#pragma unroll
      for (int r = 0; r < WIN + kRows - 1; ++r) {
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          const float2 val = *reinterpret_cast<const float2*>(&S.g[m][oy + r][hx]);
#pragma unroll
          for (int j = 0; j < kRows; ++j)
            if (r - j >= 0 && r - j < WIN) acc[m][j] = fma2(f2(a.k[r - j]), val, acc[m][j]);
        }
      }
#pragma unroll
      for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int j = 0; j < kRows; ++j) *reinterpret_cast<float2*>(&S.v[m][oy + j][hx]) = acc[m][j];
    }
  }
  for (int i = threadIdx.x; !rows_inside && i < LTY * (HX / 2); i += blockDim.x) {
    const int oy = i / (HX / 2), hx = 2 * (i % (HX / 2));
    const int py = y0 + oy;
    float2 acc[3] = {f2(0.f), f2(0.f), f2(0.f)};
    if (py < H) {
      const bool interior = py > 0 && py < H - 1;
#pragma unroll
      for (int d = -R; d <= R; ++d) {
        const int qy = py + d;
        if (qy < 0 || qy >= H) continue;  // zero rows outside the image
        const float w = interior ? a.k[R + d] : adj_weight(a.k, py, qy, H);
#pragma unroll
        for (int m = 0; m < 3; ++m)
          acc[m] = fma2(f2(w), *reinterpret_cast<const float2*>(&S.g[m][oy + R + d][hx]), acc[m]);
      }
    }
#pragma unroll
    for (int m = 0; m < 3; ++m) *reinterpret_cast<float2*>(&S.v[m][oy][hx]) = acc[m];
  }
  __syncthreads();
  float* out = a.v_pred + vd.pix_base * 4;
  const float M = 3.f * (float)W * (float)H;
  const float kl = a.l1_w / M, ks = -a.ssim_w / M;
#pragma unroll
  for (int it = 0; it < kOutIt; ++it) {
    const int i = threadIdx.x + it * kLT;
    const int oy = i / (LTX / 2), ox = 2 * (i % (LTX / 2));
    const int px = x0 + ox, py = y0 + oy;
    if (px >= W || py >= H) continue;
    float2 acc[3] = {f2(0.f), f2(0.f), f2(0.f)};
    if (px > 0 && px + 1 < W - 1) {
      // Both columns interior: the symmetric kernel, paired. Each loaded
      // value serves both columns, weights (k[j], k[j - 1]); a zero weight
      // adds an exact +0, so each column sums its taps in tap order.
#pragma unroll
      for (int j = 0; j <= 2 * R + 1; ++j) {
        const float2 w = make_float2(j <= 2 * R ? a.k[j] : 0.f, j >= 1 ? a.k[j - 1] : 0.f);
#pragma unroll
        for (int m = 0; m < 3; ++m) acc[m] = fma2(w, f2(S.v[m][oy][ox + j]), acc[m]);
      }
    } else {
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int pc = px + c;
        if (pc >= W) continue;
        float s3[3] = {0.f, 0.f, 0.f};
        for (int d = -R; d <= R; ++d) {
          const int qx = pc + d;
          if (qx < 0 || qx >= W) continue;
          const float w = adj_weight(a.k, pc, qx, W);
#pragma unroll
          for (int m = 0; m < 3; ++m) s3[m] = s3[m] + w * S.v[m][oy][ox + c + R + d];
        }
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          if (c) acc[m].y = s3[m];
          else acc[m].x = s3[m];
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const int pc = px + c;
      if (pc >= W) continue;
      const float a0 = c ? acc[0].y : acc[0].x, a1 = c ? acc[1].y : acc[1].x, a2 = c ? acc[2].y : acc[2].x;
      const size_t p = (size_t)py * W + pc;
      const float x = px_x[it][c], y = px_y[it][c];
      const float dlt = x - y;
      const float sg = dlt > 0.f ? 1.f : (dlt < 0.f ? -1.f : 0.f);
      out[p * 4 + ch] = kl * sg + ks * (a0 + 2.f * x * a1 + y * a2);
      if (ch == 0) out[p * 4 + 3] = 0.f;
    }
  }
}

// One block per view: strided partial sums in double, then a fixed-order
// tree over the block (deterministic).
__global__ void __launch_bounds__(256) loss_reduce_kernel(LossArgs a, uint32_t n_views, float* loss) {
  __shared__ double s_ss[256], s_l1[256];
  const uint32_t v = blockIdx.x;
  if (v >= n_views) return;
  const ViewDesc& vd = a.views[v];
  const int W = (int)vd.w, H = (int)vd.h;
  const int tiles = ((W + LTX - 1) / LTX) * ((H + LTY - 1) / LTY);
  double ss = 0.0, l1 = 0.0;
  for (int i = threadIdx.x; i < 3 * tiles; i += blockDim.x) {
    const int ch = i / tiles, t = i % tiles;
    const float* pp = a.partial + (((size_t)v * 3 + ch) * a.tiles_cap + t) * 2;
    ss += pp[0];
    l1 += pp[1];
  }
  s_ss[threadIdx.x] = ss;
  s_l1[threadIdx.x] = l1;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      s_ss[threadIdx.x] += s_ss[threadIdx.x + o];
      s_l1[threadIdx.x] += s_l1[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double M = 3.0 * (double)W * (double)H;
    loss[v] = (float)((double)a.l1_w * (s_l1[0] / M) + (double)a.ssim_w * (1.0 - s_ss[0] / M));
  }
}

}  // namespace

void ssim_window(float* k) {
  // loss.rs:233-250: values in f64, stored as f32, normalised in f32.
  float vals[WIN], sum = 0.0f;
  for (int o = -R; o <= R; ++o) {
    vals[o + R] = (float)exp(-(double)(o * o) / (2.0 * 1.5 * 1.5));
    sum += vals[o + R];
  }
  for (int i = 0; i < WIN; ++i) k[i] = vals[i] / (sum > 1e-8f ? sum : 1e-8f);
}

uint32_t loss_tiles(uint32_t w, uint32_t h) { return ((w + LTX - 1) / LTX) * ((h + LTY - 1) / LTY); }

cudaError_t launch_loss(const ViewSet& vs, const ViewDesc* host_views, const float* pred, const float* target,
                        float l1_w, float ssim_w, float* loss, float* v_pred, float* work, uint64_t work_floats,
                        cudaStream_t st) {
  LossArgs a{};
  a.views = vs.views;
  a.pred = pred;
  a.target = target;
  a.v_pred = v_pred;
  uint64_t pmax = 0;
  uint32_t tmax = 0;
  for (uint32_t v = 0; v < vs.n_views; ++v) {
    const uint64_t p = (uint64_t)host_views[v].w * host_views[v].h;
    if (p > pmax) pmax = p;
    const uint32_t t = loss_tiles(host_views[v].w, host_views[v].h);
    if (t > tmax) tmax = t;
  }
  a.Pcap = pmax;
  a.tiles_cap = tmax;
  const uint64_t need = (uint64_t)vs.n_views * 9 * pmax + (uint64_t)vs.n_views * 3 * tmax * 2;
  if (need > work_floats) return cudaErrorInvalidValue;
  a.maps = work;
  a.partial = work + (uint64_t)vs.n_views * 9 * pmax;
  ssim_window(a.k);
  a.l1_w = l1_w;
  a.ssim_w = ssim_w;
  if (tmax == 0) return cudaSuccess;
  dim3 grid(tmax, 3, vs.n_views);
  // More than the 48 KB default of dynamic shared memory (set for the current device).
  cudaFuncSetAttribute(ssim_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SsimFwdSmem));
  cudaFuncSetAttribute(ssim_bwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SsimBwdSmem));
  ssim_fwd_kernel<<<grid, kLT, sizeof(SsimFwdSmem), st>>>(a);
  ssim_bwd_kernel<<<grid, kLT, sizeof(SsimBwdSmem), st>>>(a);
  loss_reduce_kernel<<<vs.n_views, 256, 0, st>>>(a, vs.n_views, loss);
  return cudaGetLastError();
}

}  // namespace gsr
