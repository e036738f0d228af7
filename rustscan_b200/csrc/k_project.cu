// k_project.cu — projection, SH colour, tile counting and compaction.
//
// Three passes over every Gaussian and every view of the launch
// (project_forward.wgsl:19-96, project_visible.wgsl:130-214):
//  1. visibility: one thread per Gaussian projects it in every view and
//     records warp ballot words and per-block visible counts (the block
//     stages its 256 x 40-byte transform rows with 128-bit loads);
//  2. one block per view scans the block counts;
//  3. records: the visible Gaussians' compact indices follow in global-id
//     order from the block base, the earlier warps' and lanes' bits; the
//     projection is recomputed and the SH colour evaluated from the block's
//     SH rows, staged in shared memory with coalesced asynchronous copies.
// No block waits on another. The tiles each visible Gaussian touches are
// counted afterwards by the warp-cooperative walk over the compact records.
// This replaces the atomic compaction of project_forward.wgsl:94-96
// (nondeterministic order) and fuses the separate project_visible pass.
//
// Projected record, three float4 per visible Gaussian:
//   r0 = (x, y, conic_a, conic_b)
//   r1 = (conic_c, opacity, red, green)
//   r2 = (blue, log(255*opacity), tile box x0 | x1 << 16, tile box y0 | y1 << 16)
#include <cuda_bf16.h>

#include "gsr_kernels.h"

namespace gsr {

namespace {

constexpr int kProjThreads = (int)kProjBlock;

struct ProjectArgs {
  SplatsDev sp;
  ViewSet vs;
  float cov_blur;
  int hp;
  FwdBufs b;
  uint32_t parts;       // blocks of kProjThreads Gaussians
  uint32_t words;       // visibility words per view (parts * warps per block)
  uint32_t* vis_bits;   // [views][words]
  uint32_t* blk_count;  // [views][parts]
  uint32_t* blk_base;   // [views][parts]
};

// The block's SH rows live in shared memory as FP32 with an odd row stride,
// so that the 32 threads of a warp reading coefficient j of their own rows
// hit 32 different banks.
template <int DEG> struct ShRows {
  static constexpr int kN = 3 * (DEG + 1) * (DEG + 1);
  static constexpr int kStride = kN | 1;
  static constexpr size_t kBytes = sizeof(float) * kProjThreads * kStride;
};

__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}

// Stages the SH rows of Gaussians g0 .. g0 + rows - 1 (global element order,
// coalesced). FP32 rows are copied asynchronously (completed by
// sh_rows_wait); BF16 rows are widened on the way.
template <int DEG>
__device__ __forceinline__ void sh_rows_issue(const float* sh, uint32_t g0, uint32_t rows, float* s_sh) {
  using L = ShRows<DEG>;
  const float* src = sh + (size_t)g0 * L::kN;
  for (uint32_t e = threadIdx.x; e < rows * L::kN; e += kProjThreads)
    cp_async4(s_sh + (e / L::kN) * L::kStride + (e % L::kN), src + e);
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int DEG>
__device__ __forceinline__ void sh_rows_issue(const __nv_bfloat16* sh, uint32_t g0, uint32_t rows, float* s_sh) {
  using L = ShRows<DEG>;
  const __nv_bfloat16* src = sh + (size_t)g0 * L::kN;
  for (uint32_t e = threadIdx.x; e < rows * L::kN; e += kProjThreads)
    s_sh[(e / L::kN) * L::kStride + (e % L::kN)] = __bfloat162float(src[e]);
}
__device__ __forceinline__ void sh_rows_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Stages the block's 256 transform rows (10 floats each, 16-byte aligned)
// with 128-bit loads and reads this thread's parameters.
struct GaussParams {
  V3<float> mean{0.f, 0.f, 0.f};
  V4<float> quat{1.f, 0.f, 0.f, 0.f};
  V3<float> ls{0.f, 0.f, 0.f};
  float raw = 0.f;
};
__device__ __forceinline__ GaussParams stage_params(const SplatsDev& sp, uint32_t g0, uint32_t rows, float4* s_tr4) {
  float* s_tr = reinterpret_cast<float*>(s_tr4);
  const float* src = sp.transforms + (size_t)g0 * 10;
  if (rows == kProjThreads) {
    const float4* src4 = reinterpret_cast<const float4*>(src);
    for (int i = threadIdx.x; i < kProjThreads * 10 / 4; i += kProjThreads) s_tr4[i] = __ldg(src4 + i);
  } else {
    for (uint32_t i = threadIdx.x; i < rows * 10; i += kProjThreads) s_tr[i] = __ldg(src + i);
  }
  __syncthreads();
  GaussParams q;
  if (threadIdx.x < rows) {
    const float* t = s_tr + threadIdx.x * 10;
    q.mean = V3<float>{t[0], t[1], t[2]};
    q.quat = V4<float>{t[3], t[4], t[5], t[6]};
    q.ls = V3<float>{t[7], t[8], t[9]};
    q.raw = __ldg(sp.raw_opac + g0 + threadIdx.x);
  }
  return q;
}

// Pass 1: visibility of every Gaussian in every view. Each warp's ballot
// word goes to vis_bits[view][warp], each block's count to
// blk_count[view][block].
__global__ void __launch_bounds__(kProjThreads) visibility_kernel(ProjectArgs a) {
  constexpr int kWarps = kProjThreads / 32;
  __shared__ float4 s_tr4[kProjThreads * 10 / 4];
  __shared__ uint32_t s_cnt[kMaxViews][kWarps];
  const uint32_t n = a.sp.n, nv = a.vs.n_views;
  const uint32_t part = blockIdx.x;
  const uint32_t g0 = part * kProjThreads;
  const uint32_t rows = min(n - g0, (uint32_t)kProjThreads);
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const GaussParams q = stage_params(a.sp, g0, rows, s_tr4);
  const bool valid = threadIdx.x < rows;
  const TileShape ts{a.vs.tile_w, a.vs.tile_h};
  const GaussWorld<float> gw = gauss_world(q.quat, q.ls, q.raw);  // once for all views
  for (uint32_t v = 0; v < nv; ++v) {
    const ViewDesc& vd = a.vs.views[v];
    const Cam<float> cam = cam_from_desc<float>(vd);
    bool vis = false;
    if (valid)
      vis = project_gaussian_w(cam, q.mean, gw, a.cov_blur, ts, vd.tiles_x, vd.tiles_y, a.hp != 0)
                .visible;
    const uint32_t m = __ballot_sync(0xffffffffu, vis);
    if (lane == 0) {
      a.vis_bits[(size_t)v * a.words + part * kWarps + warp] = m;
      s_cnt[v][warp] = (uint32_t)__popc(m);
    }
  }
  __syncthreads();
  if (threadIdx.x < nv) {
    uint32_t tot = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) tot += s_cnt[threadIdx.x][w];
    a.blk_count[(size_t)threadIdx.x * a.parts + part] = tot;
  }
}

// Pass 2: per view (one block each), the exclusive scan of the block counts
// in block order and the view's visible count.
constexpr int kBlkScanThreads = 1024;
__global__ void __launch_bounds__(kBlkScanThreads) block_scan_kernel(ProjectArgs a) {
  __shared__ uint32_t s_scan[32];
  __shared__ uint32_t s_carry;
  const uint32_t v = blockIdx.x;
  const uint32_t* cnt = a.blk_count + (size_t)v * a.parts;
  uint32_t* base = a.blk_base + (size_t)v * a.parts;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (uint32_t p0 = 0; p0 < a.parts; p0 += kBlkScanThreads) {
    const uint32_t p = p0 + threadIdx.x;
    const uint32_t x = p < a.parts ? cnt[p] : 0u;
    uint32_t tot;
    const uint32_t e = block_exclusive_scan(x, s_scan, &tot);
    const uint32_t carry = s_carry;
    if (p < a.parts) base[p] = carry + e;
    __syncthreads();
    if (threadIdx.x == 0) s_carry = carry + tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) a.b.vcount[v * 4 + 0] = s_carry;
}

// Pass 3: the visible Gaussians' records at their compact indices in
// global-id order (block base + warps before + lanes before); the
// projection is recomputed (the same expression on the same inputs), the SH
// colour is evaluated from the block's staged SH rows.
template <class SHT, int DEG>
__global__ void __launch_bounds__(kProjThreads) records_kernel(ProjectArgs a) {
  constexpr int kWarps = kProjThreads / 32;
  extern __shared__ float s_sh[];  // [kProjThreads][ShRows<DEG>::kStride]
  __shared__ float4 s_tr4[kProjThreads * 10 / 4];
  __shared__ uint32_t s_mask[kMaxViews][kWarps];
  __shared__ uint32_t s_wpre[kMaxViews][kWarps];
  __shared__ uint32_t s_base[kMaxViews];
  const uint32_t n = a.sp.n, nv = a.vs.n_views;
  const uint32_t part = blockIdx.x;
  const uint32_t g0 = part * kProjThreads;
  const uint32_t g = g0 + threadIdx.x;
  const uint32_t rows = min(n - g0, (uint32_t)kProjThreads);
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  sh_rows_issue<DEG>(reinterpret_cast<const SHT*>(a.sp.sh), g0, rows, s_sh);
  for (uint32_t i = threadIdx.x; i < nv * kWarps; i += kProjThreads) {
    const uint32_t v = i / kWarps, w = i % kWarps;
    s_mask[v][w] = a.vis_bits[(size_t)v * a.words + part * kWarps + w];
  }
  if (threadIdx.x < nv) s_base[threadIdx.x] = a.blk_base[(size_t)threadIdx.x * a.parts + part];
  const GaussParams q = stage_params(a.sp, g0, rows, s_tr4);  // synchronises the block
  if (threadIdx.x < nv) {
    uint32_t tot = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      s_wpre[threadIdx.x][w] = tot;
      tot += (uint32_t)__popc(s_mask[threadIdx.x][w]);
    }
  }
  sh_rows_wait();
  __syncthreads();
  const bool valid = threadIdx.x < rows;
  const TileShape ts{a.vs.tile_w, a.vs.tile_h};
  const GaussWorld<float> gw = gauss_world(q.quat, q.ls, q.raw);  // once for all views
  const float* shg = s_sh + threadIdx.x * ShRows<DEG>::kStride;
  for (uint32_t v = 0; v < nv; ++v) {
    const uint32_t m = s_mask[v][warp];
    const bool vis = (m >> lane) & 1u;
    const uint32_t c = s_base[v] + s_wpre[v][warp] + (uint32_t)__popc(m & ((1u << lane) - 1u));
    if (valid) slice(a.b.c_of_gid, a.b.Ncap, v)[g] = vis ? (int32_t)c : -1;
    if (vis) {
      const ViewDesc& vd = a.vs.views[v];
      const Cam<float> cam = cam_from_desc<float>(vd);
      const Projected<float> p =
          project_gaussian_w(cam, q.mean, gw, a.cov_blur, ts, vd.tiles_x, vd.tiles_y, a.hp != 0);
      auto coeff = [&](int k, int ch) { return shg[k * 3 + ch]; };
      const V3<float> rgb = sh_to_color<float>(DEG, view_dir(cam, q.mean), coeff);
      float4* r = slice(a.b.rec, a.b.Vcap * 3, v) + (size_t)c * 3;
      r[0] = make_float4(p.mean2d.x, p.mean2d.y, p.conic.x, p.conic.y);
      r[1] = make_float4(p.conic.z, p.opacity, rgb.x, rgb.y);
      r[2] = make_float4(rgb.z, p.thr, __uint_as_float(p.box.x0 | (p.box.x1 << 16)),
                         __uint_as_float(p.box.y0 | (p.box.y1 << 16)));
      slice(a.b.gid_of_c, a.b.Vcap, v)[c] = g;
      slice(a.b.depth_key, a.b.Vcap, v)[c] = __float_as_uint(p.depth);
      // Tiles of the box: the intersection slots of the slot layout (the
      // counting walk replaces them by passing-tile counts otherwise).
      const uint32_t bw = p.box.x1 > p.box.x0 ? p.box.x1 - p.box.x0 : 0u;
      slice(a.b.count, a.b.Vcap, v)[c] = bw * (p.box.y1 > p.box.y0 ? p.box.y1 - p.box.y0 : 0u);
    }
  }
}

template <class SHT, int DEG>
cudaError_t launch_deg(dim3 grid, cudaStream_t st, const ProjectArgs& a) {
  const size_t bytes = ShRows<DEG>::kBytes;
  cudaError_t e = cudaFuncSetAttribute(records_kernel<SHT, DEG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return e;
  records_kernel<SHT, DEG><<<grid, kProjThreads, bytes, st>>>(a);
  return cudaGetLastError();
}

template <class SHT>
cudaError_t dispatch(int degree, dim3 grid, cudaStream_t st, const ProjectArgs& a) {
  switch (degree) {
    case 0: return launch_deg<SHT, 0>(grid, st, a);
    case 1: return launch_deg<SHT, 1>(grid, st, a);
    case 2: return launch_deg<SHT, 2>(grid, st, a);
    case 3: return launch_deg<SHT, 3>(grid, st, a);
    default: return launch_deg<SHT, 4>(grid, st, a);
  }
}

}  // namespace

cudaError_t launch_project(const SplatsDev& sp, const ViewSet& vs, float cov_blur, int fp64_conic, FwdBufs& b,
                           const Scratch& s, cudaStream_t st) {
  (void)s;
  if (sp.n == 0) {
    // No Gaussians: every view has zero visible.
    for (uint32_t v = 0; v < vs.n_views; ++v) {
      cudaError_t e = cudaMemsetAsync(b.vcount + v * 4, 0, 4 * sizeof(uint32_t), st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  ProjectArgs a;
  a.sp = sp;
  a.vs = vs;
  a.cov_blur = cov_blur;
  a.hp = fp64_conic;
  a.b = b;
  a.parts = (sp.n + kProjThreads - 1) / kProjThreads;
  a.words = a.parts * (kProjThreads / 32);
  if (a.parts > b.proj_parts_cap) return cudaErrorInvalidValue;
  a.vis_bits = b.vis_bits;
  a.blk_count = b.blk_count;
  a.blk_base = b.blk_base;
  visibility_kernel<<<a.parts, kProjThreads, 0, st>>>(a);
  block_scan_kernel<<<vs.n_views, kBlkScanThreads, 0, st>>>(a);
  const dim3 grid(a.parts);
  return sp.sh_bf16 ? dispatch<__nv_bfloat16>(sp.degree, grid, st, a) : dispatch<float>(sp.degree, grid, st, a);
}

}  // namespace gsr
