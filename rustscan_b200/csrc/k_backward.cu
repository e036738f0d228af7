// k_backward.cu — projection backward (project_backwards.wgsl:12-151) over
// all views of the last forward, the densification statistics
// (engine/trainer.rs:651-728) and the bias-corrected Adam update
// (engine/optimizer.rs:122-162).
//
// Two passes: one thread per (view, visible Gaussian) forms that view's
// projection adjoint into a pair record; one thread per Gaussian then sums
// its records over the views in a fixed order and writes the gradient once.
// Rows of Gaussians no view sees get zero gradients, as the reference
// zero-fills. Adam is a separate element-wise pass with 16-byte accesses.
#include <cuda_bf16.h>

#include "gsr_kernels.h"

namespace gsr {

namespace {

// ---------------------------------------------------------------------------
// Kernel A: one thread per (view, visible Gaussian). The projection adjoint
// of that view (everything but the SH view-direction term) goes into a
// 96-byte pair record, stored as six planes of float4 ([view][6][Vcap]) so
// that a warp reading one part for consecutive Gaussians reads 512
// contiguous bytes:
//   q0 = (v_mean, v_raw_opacity)   q1 = v_quat
//   q2 = (v_log_scale, depth)      q3 = (view direction, visible flag)
//   q4 = (v_rgb, pixel count)      q5 = (v_xy, |v_xy| sums)
// ---------------------------------------------------------------------------
struct PairArgs {
  SplatsDev sp;
  ViewSet vs;
  float cov_blur;
  FwdBufs b;
  int exact;
  int hp;
};

struct NoCoeff {
  __device__ float operator()(int, int) const { return 0.f; }
};

__global__ void __launch_bounds__(128, 6) pair_bwd_kernel(PairArgs a) {
  const uint32_t v = blockIdx.y;
  const uint32_t V = a.b.vcount[v * 4 + 0];
  const ViewDesc& vd = a.vs.views[v];
  const Cam<float> cam = cam_from_desc<float>(vd);
  const uint32_t* gid_of_c = slice(a.b.gid_of_c, a.b.Vcap, v);
  const float4* sgrad = slice(a.b.sgrad, a.b.Vcap * 3, v);
  const uint8_t* vis = slice(a.b.visible_c, a.b.Vcap, v);
  float4* pair = slice(a.b.pair, a.b.Vcap * 6, v);
  const uint32_t stride = gridDim.x * blockDim.x;
  uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t g_next = c < V ? gid_of_c[c] : 0u;
  for (; c < V; c += stride) {
    const uint32_t g = g_next;
    if (c + stride < V) g_next = gid_of_c[c + stride];  // the next row's id is in flight during this one
    const float2* t2 = reinterpret_cast<const float2*>(a.sp.transforms + (size_t)g * 10);
    const float2 t01 = t2[0], t23 = t2[1], t45 = t2[2], t67 = t2[3], t89 = t2[4];
    const float4 q0 = sgrad[(size_t)c * 3 + 0], q1 = sgrad[(size_t)c * 3 + 1], q2 = sgrad[(size_t)c * 3 + 2];
    const ParamGrad<float> pg = project_backward(
        cam, V3<float>{t01.x, t01.y, t23.x}, V4<float>{t23.y, t45.x, t45.y, t67.x}, V3<float>{t67.y, t89.x, t89.y},
        a.sp.raw_opac[g], a.cov_blur, V2<float>{q0.x, q0.y}, V3<float>{q0.z, q0.w, q1.x}, V3<float>{q1.y, q1.z, q1.w},
        q2.x, a.sp.degree, NoCoeff(), a.exact != 0, false, a.hp != 0);
    const size_t cap = a.b.Vcap;
    pair[0 * cap + c] = make_float4(pg.v_mean.x, pg.v_mean.y, pg.v_mean.z, pg.v_raw_opac);
    pair[1 * cap + c] = make_float4(pg.v_quat.x, pg.v_quat.y, pg.v_quat.z, pg.v_quat.w);
    pair[2 * cap + c] = make_float4(pg.v_log_scale.x, pg.v_log_scale.y, pg.v_log_scale.z, pg.depth);
    pair[3 * cap + c] = make_float4(pg.viewdir.x, pg.viewdir.y, pg.viewdir.z, vis[c] ? 1.f : 0.f);
    pair[4 * cap + c] = make_float4(q1.y, q1.z, q1.w, q2.w);
    pair[5 * cap + c] = make_float4(q0.x, q0.y, q2.y, q2.z);
  }
}

// ---------------------------------------------------------------------------
// Kernel B: one thread per Gaussian, views in a fixed order. Sums the pair
// records (plus the SH view-direction term, which needs the coefficients),
// writes the per-view statistics and the densification sums, and writes the
// summed gradient (times grad_scale) as [n][10], [n][3K], [n]. Compaction
// runs in global-id order, so consecutive threads read consecutive pair
// records of a view: every load is coalesced and no staging is needed.
// ---------------------------------------------------------------------------
struct GatherArgs {
  SplatsDev sp;
  ViewSet vs;
  FwdBufs b;
  float* v_tr;
  float* v_sh;
  float* v_op;
  float* stats;
  float* acc;
  int use_visible;
  float grad_scale;
  int exact;
};

__device__ __forceinline__ float to_f(float x) { return x; }
__device__ __forceinline__ float to_f(__nv_bfloat16 x) { return __bfloat162float(x); }

// A block owns kGT consecutive Gaussians. Shared memory holds, per Gaussian,
// one row of its SH values (read by the view-direction term; staged with
// coalesced loads) that is reused for its SH gradients on the way out, plus a
// row of transform and opacity gradients, so that every global write is
// coalesced too.
constexpr int kGT = 128;

template <int K> struct GatherSmem {
  static constexpr int kSh = 3 * K + 1;  // odd stride: conflict-free rows
  static constexpr int kTr = 11;
  static constexpr size_t kPairOff = sizeof(float) * (kGT * kSh + kGT * kTr);  // a multiple of 16
  static constexpr size_t kBytes = kPairOff + sizeof(float4) * 2 * 6 * kGT;   // + two stages of pair records
};

__device__ __forceinline__ void cp_async16(float4* dst, const float4* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Starts the copy of this thread's six pair records of view v (compact index
// c, none if c < 0) into its slots of stage `stage`; one commit group per
// view whether or not it copies anything.
__device__ __forceinline__ void pair_issue(const FwdBufs& b, uint32_t v, int32_t c, float4* s_pair, int stage,
                                           uint32_t r) {
  if (c >= 0) {
    const float4* P = slice(b.pair, b.Vcap * 6, v) + c;
#pragma unroll
    for (int q = 0; q < 6; ++q) cp_async16(s_pair + (stage * 6 + q) * kGT + r, P + q * b.Vcap);
  }
  cp_async_commit();
}

// Copies rows x NSH SH values (global element order, coalesced) into
// shared-memory rows of stride STR as FP32. All of a thread's loads are in
// flight at once: asynchronous copies for FP32, a batch of register loads
// for BF16.
template <int NSH, int STR>
__device__ __forceinline__ void stage_sh_rows(const float* src, uint32_t rows, float* s_row) {
  for (uint32_t e = threadIdx.x; e < rows * NSH; e += kGT) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(s_row + (e / NSH) * STR + (e % NSH));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src + e) : "memory");
  }
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}
template <int NSH, int STR>
__device__ __forceinline__ void stage_sh_rows(const __nv_bfloat16* src, uint32_t rows, float* s_row) {
  constexpr int kB = 8;
  const uint32_t total = rows * NSH;
  for (uint32_t e0 = threadIdx.x; e0 < total; e0 += kB * kGT) {
    float x[kB];
#pragma unroll
    for (int i = 0; i < kB; ++i) {
      const uint32_t e = e0 + i * kGT;
      x[i] = e < total ? __bfloat162float(src[e]) : 0.f;
    }
#pragma unroll
    for (int i = 0; i < kB; ++i) {
      const uint32_t e = e0 + i * kGT;
      if (e < total) s_row[(e / NSH) * STR + (e % NSH)] = x[i];
    }
  }
}

template <class SHT, int DEG>
__global__ void __launch_bounds__(kGT, DEG >= 4 ? 2 : 4) gather_kernel(GatherArgs a) {
  constexpr int K = (DEG + 1) * (DEG + 1);
  constexpr int NSH = 3 * K;
  using L = GatherSmem<K>;
  extern __shared__ float smem[];
  float* s_row = smem;                 // [kGT][kSh]: SH values, then SH gradients
  float* s_tg = smem + kGT * L::kSh;   // [kGT][kTr]: transform + opacity gradients
  // [2][6][kGT]: each thread's pair records of the current and the next view
  float4* s_pair = reinterpret_cast<float4*>(reinterpret_cast<char*>(smem) + L::kPairOff);
  const uint32_t n = a.sp.n;
  const uint32_t nv = a.vs.n_views;
  const float sc = a.grad_scale;
  const SHT* sh = reinterpret_cast<const SHT*>(a.sp.sh);
  const bool dir_term = a.exact != 0 && DEG > 0;
  const uint32_t r = threadIdx.x;
  for (uint32_t g0 = blockIdx.x * kGT; g0 < n; g0 += gridDim.x * kGT) {
    const uint32_t rows = min((uint32_t)kGT, n - g0);
    const uint32_t g = g0 + r;
    const bool own = r < rows;
    __syncthreads();
    if (dir_term) stage_sh_rows<NSH, L::kSh>(sh + (size_t)g0 * NSH, rows, s_row);
    __syncthreads();
    V3<float> mean{0.f, 0.f, 0.f};
    if (own && dir_term) {
      const float* t = a.sp.transforms + (size_t)g * 10;
      mean = V3<float>{t[0], t[1], t[2]};
    }
    const float* cf = s_row + r * L::kSh;
    auto coeff = [&](int k, int ch) { return cf[k * 3 + ch]; };
    float sg[NSH];
#pragma unroll
    for (int i = 0; i < NSH; ++i) sg[i] = 0.f;
    float gt[10], gop = 0.f;
#pragma unroll
    for (int k = 0; k < 10; ++k) gt[k] = 0.f;
    float ac[9];
    if (own && a.acc) {
#pragma unroll
      for (int k = 0; k < 9; ++k) ac[k] = a.acc[k * (size_t)n + g];
    }
    // The pair records of view v + 1 are in flight while view v is summed
    // (each thread copies and reads only its own slots).
    int32_t c_cur = (own && nv > 0) ? a.b.c_of_gid[g] : -1;
    if (nv > 0) pair_issue(a.b, 0, c_cur, s_pair, 0, r);
    int32_t c_nxt = (own && nv > 1) ? slice(a.b.c_of_gid, a.b.Ncap, 1)[g] : -1;
    for (uint32_t v = 0; v < nv; ++v) {
      const int32_t c = c_cur;
      if (v + 1 < nv)
        pair_issue(a.b, v + 1, c_nxt, s_pair, (v + 1) & 1, r);
      else
        cp_async_commit();
      c_cur = c_nxt;
      c_nxt = (own && v + 2 < nv) ? slice(a.b.c_of_gid, a.b.Ncap, v + 2)[g] : -1;
      cp_async_wait1();  // view v's records have landed
      float st[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      float g2d = 0.f, gcol = 0.f, visf = 0.f;
      if (c >= 0) {
        const float4* P = s_pair + (v & 1) * 6 * kGT + r;
        const float4 q0 = P[0], q1 = P[kGT], q2 = P[2 * kGT], q3 = P[3 * kGT], q4 = P[4 * kGT], q5 = P[5 * kGT];
        V3<float> vm{q0.x, q0.y, q0.z};
        const V3<float> dir{q3.x, q3.y, q3.z};
        if (dir_term) {
          const Cam<float> cam = cam_from_desc<float>(a.vs.views[v]);
          const V3<float> d = sh_viewdir_vjp(cam, mean, dir, DEG, V3<float>{q4.x, q4.y, q4.z}, coeff);
          vm.x += d.x;
          vm.y += d.y;
          vm.z += d.z;
        }
        gt[0] += vm.x;
        gt[1] += vm.y;
        gt[2] += vm.z;
        gt[3] += q1.x;
        gt[4] += q1.y;
        gt[5] += q1.z;
        gt[6] += q1.w;
        gt[7] += q2.x;
        gt[8] += q2.y;
        gt[9] += q2.z;
        gop += q0.w;
        float bas[25];
        sh_basis<float>(DEG, dir.x, dir.y, dir.z, bas);
        float csum = 0.f;
#pragma unroll
        for (int k = 0; k < K; ++k) {
          const float s0 = bas[k] * q4.x, s1 = bas[k] * q4.y, s2 = bas[k] * q4.z;
          sg[k * 3 + 0] += s0;
          sg[k * 3 + 1] += s1;
          sg[k * 3 + 2] += s2;
          csum += fabsf(s0) + fabsf(s1) + fabsf(s2);
        }
        // Densification quantities of this view (engine/trainer.rs:660-727).
        g2d = (fabsf(vm.x) + fabsf(vm.y) + fabsf(vm.z)) / 3.0f;
        gcol = csum * (1.0f / (float)(3 * K));  // mean over coefficients of the channel mean
        // project_backwards.wgsl:33-36, 105-108.
        st[0] = q5.x;
        st[1] = q5.y;
        st[2] = q5.z;
        st[3] = q5.w;
        st[4] = q4.w * sqrtf(q5.z * q5.z + q5.w * q5.w);
        st[5] = q4.w;
        st[6] = q4.w * q2.w;
        visf = q3.w;
      }
      if (own && a.stats) {
        float* so = a.stats + ((size_t)v * n + g) * 7;
#pragma unroll
        for (int k = 0; k < 7; ++k) so[k] = st[k];
      }
      if (a.acc) {
        // One view at a time, in view order, as a per-view accumulation does.
        ac[0] += g2d;
        ac[1] += sqrtf(st[0] * st[0] + st[1] * st[1]);
        ac[2] += sqrtf(st[2] * st[2] + st[3] * st[3]);
        ac[3] += st[4];
        ac[4] += st[5];
        ac[5] += st[6];
        ac[6] += gcol;
        ac[7] += 1.0f;
        ac[8] += a.use_visible ? visf : 1.0f;
      }
    }
    if (own && a.acc) {
#pragma unroll
      for (int k = 0; k < 9; ++k) a.acc[k * (size_t)n + g] = ac[k];
    }
    __syncthreads();  // every thread is done with the SH values in s_row
    float* tg = s_tg + r * L::kTr;
#pragma unroll
    for (int k = 0; k < 10; ++k) tg[k] = gt[k] * sc;
    tg[10] = gop * sc;
    float* sgr = s_row + r * L::kSh;
#pragma unroll
    for (int i = 0; i < NSH; ++i) sgr[i] = sg[i] * sc;
    __syncthreads();
    float* vt = a.v_tr + (size_t)g0 * 10;
    for (uint32_t e = r; e < rows * 10; e += kGT) vt[e] = s_tg[(e / 10) * L::kTr + (e % 10)];
    float* vs = a.v_sh + (size_t)g0 * NSH;
    for (uint32_t e = r; e < rows * NSH; e += kGT) vs[e] = s_row[(e / NSH) * L::kSh + (e % NSH)];
    if (own) a.v_op[g] = tg[10];
  }
}

template <class SHT, int DEG> void launch_gather(int blocks, cudaStream_t st, const GatherArgs& a) {
  constexpr int K = (DEG + 1) * (DEG + 1);
  const size_t bytes = GatherSmem<K>::kBytes;
  cudaFuncSetAttribute(gather_kernel<SHT, DEG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  gather_kernel<SHT, DEG><<<blocks, kGT, bytes, st>>>(a);
}

template <class SHT>
void dispatch_gather(int degree, int blocks, cudaStream_t st, const GatherArgs& a) {
  switch (degree) {
    case 0: launch_gather<SHT, 0>(blocks, st, a); break;
    case 1: launch_gather<SHT, 1>(blocks, st, a); break;
    case 2: launch_gather<SHT, 2>(blocks, st, a); break;
    case 3: launch_gather<SHT, 3>(blocks, st, a); break;
    default: launch_gather<SHT, 4>(blocks, st, a); break;
  }
}

// engine/optimizer.rs:141-161 with the bias corrections applied as
// multiplications by their f32 reciprocals; every operation rounded on its
// own (the file builds with multiply-add contraction; Adam must match the
// oracle bit for bit).
__device__ __forceinline__ float adam_one(float p, float g, float& m, float& v, float lr, const AdamScalars& a) {
  const float m1 = eadd(emul(m, a.beta1), emul(g, esub(1.0f, a.beta1)));
  const float m2 = eadd(emul(v, a.beta2), emul(emul(g, g), esub(1.0f, a.beta2)));
  m = m1;
  v = m2;
  const float mh = emul(m1, a.rbc1), vh = emul(m2, a.rbc2);
  const float upd = __fdiv_rn(mh, eadd(__fsqrt_rn(vh), a.eps));
  return esub(p, emul(upd, lr));
}

__device__ __forceinline__ float group_lr(const AdamScalars& a, int group, uint32_t col) {
  if (group == 0) return col < 3 ? a.lr_pos : (col < 7 ? a.lr_rot : a.lr_scale);
  return group == 1 ? a.lr_color : a.lr_opac;
}

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ float4 ld4(const __nv_bfloat16* p) {
  const uint2 u = *reinterpret_cast<const uint2*>(p);
  const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.x));
  const float2 hi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.y));
  return make_float4(lo.x, lo.y, hi.x, hi.y);
}
__device__ __forceinline__ void st4(float* p, float4 x) { *reinterpret_cast<float4*>(p) = x; }
__device__ __forceinline__ void st4(__nv_bfloat16* p, float4 x) {
  __nv_bfloat162 lo, hi;
  lo.x = __float2bfloat16_rn(x.x);
  lo.y = __float2bfloat16_rn(x.y);
  hi.x = __float2bfloat16_rn(x.z);
  hi.y = __float2bfloat16_rn(x.w);
  uint2 u;
  u.x = *reinterpret_cast<uint32_t*>(&lo);
  u.y = *reinterpret_cast<uint32_t*>(&hi);
  *reinterpret_cast<uint2*>(p) = u;
}
__device__ __forceinline__ void store_sh(float* p, float x) { *p = x; }
__device__ __forceinline__ void store_sh(__nv_bfloat16* p, float x) { *p = __float2bfloat16_rn(x); }

// Element-wise Adam over one parameter group (0 transforms: columns 3
// position, 4 rotation, 3 scale; 1 SH coefficients; 2 opacities). Four
// elements per thread with 16-byte loads and stores when every array is
// aligned for them (vec), the remainder one by one.
template <class PT>
__global__ void __launch_bounds__(256) adam_kernel(PT* p, const float* g, float* m, float* v, uint64_t n, int group,
                                                   int vec, const AdamScalars* scal) {
  const AdamScalars a = *scal;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t t0 = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t nq = vec ? n / 4 : 0;
  for (uint64_t q = t0; q < nq; q += stride) {
    const uint64_t i = q * 4;
    float4 P = ld4(p + i);
    const float4 G = ld4(g + i);
    float4 M = ld4(m + i), Vv = ld4(v + i);
    uint32_t col = group == 0 ? (uint32_t)(i % 10u) : 0u;
    auto step = [&](float& pp, float gg, float& mm, float& vv) {
      pp = adam_one(pp, gg, mm, vv, group_lr(a, group, col), a);
      if (++col == 10u) col = 0u;
    };
    step(P.x, G.x, M.x, Vv.x);
    step(P.y, G.y, M.y, Vv.y);
    step(P.z, G.z, M.z, Vv.z);
    step(P.w, G.w, M.w, Vv.w);
    st4(p + i, P);
    st4(m + i, M);
    st4(v + i, Vv);
  }
  for (uint64_t i = nq * 4 + t0; i < n; i += stride) {
    const uint32_t col = group == 0 ? (uint32_t)(i % 10u) : 0u;
    store_sh(p + i, adam_one(to_f(p[i]), g[i], m[i], v[i], group_lr(a, group, col), a));
  }
}

__global__ void set_scalars_kernel(AdamScalars* dst, AdamScalars v) { *dst = v; }

__global__ void densify_kernel(const float* v_tr, const float* stats, const float* v_sh, const float* visible,
                               uint32_t n, int K, int use_visible, float* acc) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float* t = v_tr + (size_t)i * 10;
    const float* s = stats + (size_t)i * 7;
    const float g2 = (fabsf(t[0]) + fabsf(t[1]) + fabsf(t[2])) / 3.0f;
    float gc = 0.f;
    for (int k = 0; k < K; ++k) {
      const float* c = v_sh + ((size_t)i * K + k) * 3;
      gc = gc + (fabsf(c[0]) + fabsf(c[1]) + fabsf(c[2])) / 3.0f;
    }
    gc = gc / (float)K;
    acc[0 * (size_t)n + i] += g2;
    acc[1 * (size_t)n + i] += sqrtf(s[0] * s[0] + s[1] * s[1]);
    acc[2 * (size_t)n + i] += sqrtf(s[2] * s[2] + s[3] * s[3]);
    acc[3 * (size_t)n + i] += s[4];
    acc[4 * (size_t)n + i] += s[5];
    acc[5 * (size_t)n + i] += s[6];
    acc[6 * (size_t)n + i] += gc;
    acc[7 * (size_t)n + i] += 1.0f;
    acc[8 * (size_t)n + i] += use_visible ? visible[i] : 1.0f;
  }
}

}  // namespace

cudaError_t launch_set_scalars(AdamScalars* dst, const AdamScalars& v, cudaStream_t st) {
  set_scalars_kernel<<<1, 1, 0, st>>>(dst, v);
  return cudaGetLastError();
}

cudaError_t launch_project_bwd(const SplatsDev& sp, const ViewSet& vs, float cov_blur, FwdBufs& b,
                               const ProjBwdArgs& pa, cudaStream_t st, int num_sms) {
  if (sp.n == 0) return cudaSuccess;
  PairArgs pr{};
  pr.sp = sp;
  pr.vs = vs;
  pr.cov_blur = cov_blur;
  pr.b = b;
  pr.exact = pa.exact;
  pr.hp = pa.hp;
  int px = num_sms * 16 / (int)vs.n_views;
  if (px < 1) px = 1;
  pair_bwd_kernel<<<dim3(px, vs.n_views), 128, 0, st>>>(pr);
  GatherArgs a{};
  a.sp = sp;
  a.vs = vs;
  a.b = b;
  a.v_tr = pa.v_tr;
  a.v_sh = pa.v_sh;
  a.v_op = pa.v_op;
  a.stats = pa.stats;
  a.acc = pa.densify_acc;
  a.use_visible = pa.use_visible;
  a.grad_scale = pa.grad_scale;
  a.exact = pa.exact;
  int blocks = (int)((sp.n + kGT - 1) / kGT);
  const int cap = num_sms * 8;
  if (blocks > cap) blocks = cap;
  if (sp.sh_bf16)
    dispatch_gather<__nv_bfloat16>(sp.degree, blocks, st, a);
  else
    dispatch_gather<float>(sp.degree, blocks, st, a);
  return cudaGetLastError();
}

namespace {
bool aligned(const void* p, uintptr_t to) { return (reinterpret_cast<uintptr_t>(p) & (to - 1)) == 0; }

template <class PT>
void adam_group(PT* p, const float* g, float* m, float* v, uint64_t n, int group, const AdamScalars* scal,
                cudaStream_t st, int num_sms) {
  if (n == 0) return;
  const int vec = aligned(p, 4 * sizeof(PT)) && aligned(g, 16) && aligned(m, 16) && aligned(v, 16);
  const uint64_t units = vec ? (n + 3) / 4 : n;
  uint64_t blocks = (units + 255) / 256;
  const uint64_t cap = (uint64_t)num_sms * 8;
  if (blocks > cap) blocks = cap;
  adam_kernel<PT><<<(unsigned)blocks, 256, 0, st>>>(p, g, m, v, n, group, vec, scal);
}
}  // namespace

cudaError_t launch_adam(const AdamArgs& a, const float* g_tr, const float* g_sh, const float* g_op, uint32_t n,
                        int degree, int sh_bf16, cudaStream_t st, int num_sms) {
  if (n == 0) return cudaSuccess;
  const uint64_t nsh = (uint64_t)n * (degree + 1) * (degree + 1) * 3;
  adam_group<float>(a.transforms, g_tr, a.m_tr, a.v_tr, (uint64_t)n * 10, 0, a.scal, st, num_sms);
  if (sh_bf16)
    adam_group<__nv_bfloat16>(reinterpret_cast<__nv_bfloat16*>(a.sh), g_sh, a.m_sh, a.v_sh, nsh, 1, a.scal, st,
                              num_sms);
  else
    adam_group<float>(reinterpret_cast<float*>(a.sh), g_sh, a.m_sh, a.v_sh, nsh, 1, a.scal, st, num_sms);
  adam_group<float>(a.raw_opac, g_op, a.m_op, a.v_op, n, 2, a.scal, st, num_sms);
  return cudaGetLastError();
}

cudaError_t launch_densify(const float* v_tr, const float* stats, const float* v_sh, const float* visible, uint32_t n,
                           int degree, int use_visible, float* acc, cudaStream_t st, int num_sms) {
  if (n == 0) return cudaSuccess;
  const int K = (degree + 1) * (degree + 1);
  densify_kernel<<<num_sms * 8, 256, 0, st>>>(v_tr, stats, v_sh, visible, n, K, use_visible, acc);
  return cudaGetLastError();
}

}  // namespace gsr
