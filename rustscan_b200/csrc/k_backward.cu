// k_backward.cu — projection backward (project_backwards.wgsl:12-151) over
// all views of the last forward, optionally fused with the bias-corrected
// Adam update (engine/optimizer.rs:122-162) and the densification
// statistics (engine/trainer.rs:651-728).
//
// One thread per Gaussian, views in a fixed order: the gradient of the sum
// over views is formed in registers and written once (or consumed by Adam in
// place, so the [N, 10+3K+1] gradient never touches memory in a training
// step). Rows of Gaussians no view sees get zero gradients, as the reference
// zero-fills.
#include <cuda_bf16.h>

#include "gsr_kernels.h"

namespace gsr {

namespace {

struct PBArgs {
  SplatsDev sp;
  ViewSet vs;
  float cov_blur;
  FwdBufs b;
  float* v_tr;
  float* v_sh;
  float* v_op;
  float* stats;
  AdamArgs adam;
  int do_adam;
  float* acc;
  int use_visible;
  float grad_scale;
  int exact;
};

__device__ __forceinline__ float adam_one(float p, float g, float* m, float* v, float lr, const AdamScalars& a) {
  const float m1 = *m * a.beta1 + g * (1.0f - a.beta1);
  const float m2 = *v * a.beta2 + (g * g) * (1.0f - a.beta2);
  *m = m1;
  *v = m2;
  const float mh = m1 / a.bc1, vh = m2 / a.bc2;
  const float upd = mh / (sqrtf(vh) + a.eps);
  return p - upd * lr;
}

__device__ __forceinline__ float to_f(float x) { return x; }
__device__ __forceinline__ float to_f(__nv_bfloat16 x) { return __bfloat162float(x); }
__device__ __forceinline__ void store_sh(float* p, float x) { *p = x; }
__device__ __forceinline__ void store_sh(__nv_bfloat16* p, float x) { *p = __float2bfloat16_rn(x); }

template <class SHT, int DEG>
__global__ void __launch_bounds__(128) project_bwd_kernel(PBArgs a) {
  constexpr int K = (DEG + 1) * (DEG + 1);
  const uint32_t n = a.sp.n;
  const SHT* sh = reinterpret_cast<const SHT*>(a.sp.sh);
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
    const float* t = a.sp.transforms + (size_t)g * 10;
    float tp[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) tp[k] = t[k];
    const V3<float> mean{tp[0], tp[1], tp[2]};
    const V4<float> quat{tp[3], tp[4], tp[5], tp[6]};
    const V3<float> ls{tp[7], tp[8], tp[9]};
    const float raw = a.sp.raw_opac[g];
    const SHT* shg = sh + (size_t)g * K * 3;
    float coef[K * 3];
#pragma unroll
    for (int k = 0; k < K * 3; ++k) coef[k] = to_f(shg[k]);
    auto coeff = [&](int k, int ch) { return coef[k * 3 + ch]; };
    float gt[10], gsh[K * 3], gop = 0.f;
#pragma unroll
    for (int k = 0; k < 10; ++k) gt[k] = 0.f;
#pragma unroll
    for (int k = 0; k < K * 3; ++k) gsh[k] = 0.f;
    for (uint32_t v = 0; v < a.vs.n_views; ++v) {
      const int32_t c = slice(a.b.c_of_gid, a.b.Ncap, v)[g];
      float st[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      float g2d = 0.f, gcol = 0.f, visf = 0.f;
      if (c >= 0) {
        const float4* sgp = slice(a.b.sgrad, a.b.Vcap * 3, v) + (size_t)c * 3;
        const float4 q0 = sgp[0], q1 = sgp[1], q2 = sgp[2];
        const ViewDesc& vd = a.vs.views[v];
        const Cam<float> cam = cam_from_desc<float>(vd);
        const ParamGrad<float> pg =
            project_backward(cam, mean, quat, ls, raw, a.cov_blur, V2<float>{q0.x, q0.y}, V3<float>{q0.z, q0.w, q1.x},
                             V3<float>{q1.y, q1.z, q1.w}, q2.x, DEG, coeff, a.exact != 0);
        float bas[25];
        sh_basis<float>(DEG, pg.viewdir.x, pg.viewdir.y, pg.viewdir.z, bas);
        const float vg[10] = {pg.v_mean.x, pg.v_mean.y, pg.v_mean.z, pg.v_quat.x, pg.v_quat.y,
                              pg.v_quat.z, pg.v_quat.w, pg.v_log_scale.x, pg.v_log_scale.y, pg.v_log_scale.z};
#pragma unroll
        for (int k = 0; k < 10; ++k) gt[k] = gt[k] + vg[k];
        gop = gop + pg.v_raw_opac;
        float csum = 0.f;
#pragma unroll
        for (int k = 0; k < K; ++k) {
          const float s0 = bas[k] * q1.y, s1 = bas[k] * q1.z, s2 = bas[k] * q1.w;
          gsh[k * 3 + 0] = gsh[k * 3 + 0] + s0;
          gsh[k * 3 + 1] = gsh[k * 3 + 1] + s1;
          gsh[k * 3 + 2] = gsh[k * 3 + 2] + s2;
          csum = csum + (fabsf(s0) + fabsf(s1) + fabsf(s2)) / 3.0f;
        }
        gcol = csum / (float)K;
        g2d = (fabsf(vg[0]) + fabsf(vg[1]) + fabsf(vg[2])) / 3.0f;
        // project_backwards.wgsl:192-205, 274-277.
        st[0] = q0.x;
        st[1] = q0.y;
        st[2] = q2.y;
        st[3] = q2.z;
        const float abs_score = sqrtf(q2.y * q2.y + q2.z * q2.z);
        st[4] = q2.w * abs_score;
        st[5] = q2.w;
        st[6] = q2.w * pg.depth;
        visf = slice(a.b.visible_c, a.b.Vcap, v)[c] ? 1.f : 0.f;
      }
      if (a.stats) {
        float* so = a.stats + ((size_t)v * n + g) * 7;
#pragma unroll
        for (int k = 0; k < 7; ++k) so[k] = st[k];
      }
      if (a.acc) {
        // engine/trainer.rs:660-727 for this view.
        float* acc = a.acc;
        acc[0 * (size_t)n + g] += g2d;
        acc[1 * (size_t)n + g] += sqrtf(st[0] * st[0] + st[1] * st[1]);
        acc[2 * (size_t)n + g] += sqrtf(st[2] * st[2] + st[3] * st[3]);
        acc[3 * (size_t)n + g] += st[4];
        acc[4 * (size_t)n + g] += st[5];
        acc[5 * (size_t)n + g] += st[6];
        acc[6 * (size_t)n + g] += gcol;
        acc[7 * (size_t)n + g] += 1.0f;
        acc[8 * (size_t)n + g] += a.use_visible ? visf : 1.0f;
      }
    }
    const float sc = a.grad_scale;
    if (!a.do_adam) {
      float* o = a.v_tr + (size_t)g * 10;
#pragma unroll
      for (int k = 0; k < 10; ++k) o[k] = gt[k] * sc;
      float* os = a.v_sh + (size_t)g * K * 3;
#pragma unroll
      for (int k = 0; k < K * 3; ++k) os[k] = gsh[k] * sc;
      a.v_op[g] = gop * sc;
    } else {
      const AdamArgs& ad = a.adam;
      const AdamScalars sc_ = *ad.scal;
      float* pt = ad.transforms + (size_t)g * 10;
      float* mt = ad.m_tr + (size_t)g * 10;
      float* vt = ad.v_tr + (size_t)g * 10;
#pragma unroll
      for (int k = 0; k < 10; ++k) {
        const float lr = k < 3 ? sc_.lr_pos : (k < 7 ? sc_.lr_rot : sc_.lr_scale);
        pt[k] = adam_one(tp[k], gt[k] * sc, mt + k, vt + k, lr, sc_);
      }
      SHT* ps = reinterpret_cast<SHT*>(ad.sh) + (size_t)g * K * 3;
      float* ms = ad.m_sh + (size_t)g * K * 3;
      float* vs = ad.v_sh + (size_t)g * K * 3;
#pragma unroll
      for (int k = 0; k < K * 3; ++k)
        store_sh(ps + k, adam_one(coef[k], gsh[k] * sc, ms + k, vs + k, sc_.lr_color, sc_));
      ad.raw_opac[g] = adam_one(raw, gop * sc, ad.m_op + g, ad.v_op + g, sc_.lr_opac, sc_);
    }
  }
}

template <class SHT>
void dispatch_pb(int degree, int blocks, cudaStream_t st, const PBArgs& a) {
  switch (degree) {
    case 0: project_bwd_kernel<SHT, 0><<<blocks, 128, 0, st>>>(a); break;
    case 1: project_bwd_kernel<SHT, 1><<<blocks, 128, 0, st>>>(a); break;
    case 2: project_bwd_kernel<SHT, 2><<<blocks, 128, 0, st>>>(a); break;
    case 3: project_bwd_kernel<SHT, 3><<<blocks, 128, 0, st>>>(a); break;
    default: project_bwd_kernel<SHT, 4><<<blocks, 128, 0, st>>>(a); break;
  }
}

// Standalone Adam over one group: group 0 transforms (columns: 3 position,
// 4 rotation, 3 scale), 1 SH coefficients, 2 opacities.
template <class PT>
__global__ void adam_kernel(PT* p, const float* g, float* m, float* v, uint64_t n, int group,
                            const AdamScalars* scal) {
  const AdamScalars a = *scal;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    float lr;
    if (group == 0) {
      const int col = (int)(i % 10u);
      lr = col < 3 ? a.lr_pos : (col < 7 ? a.lr_rot : a.lr_scale);
    } else {
      lr = group == 1 ? a.lr_color : a.lr_opac;
    }
    store_sh(p + i, adam_one(to_f(p[i]), g[i], m + i, v + i, lr, a));
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
                               const ProjBwdArgs& pa, const AdamArgs* adam, cudaStream_t st, int num_sms) {
  if (sp.n == 0) return cudaSuccess;
  PBArgs a{};
  a.sp = sp;
  a.vs = vs;
  a.cov_blur = cov_blur;
  a.b = b;
  a.v_tr = pa.v_tr;
  a.v_sh = pa.v_sh;
  a.v_op = pa.v_op;
  a.stats = pa.stats;
  a.do_adam = adam != nullptr;
  if (adam) a.adam = *adam;
  a.acc = pa.densify_acc;
  a.use_visible = pa.use_visible;
  a.grad_scale = pa.grad_scale;
  a.exact = pa.exact;
  int blocks = (int)((sp.n + 127) / 128);
  const int cap = num_sms * 16;
  if (blocks > cap) blocks = cap;
  if (sp.sh_bf16)
    dispatch_pb<__nv_bfloat16>(sp.degree, blocks, st, a);
  else
    dispatch_pb<float>(sp.degree, blocks, st, a);
  return cudaGetLastError();
}

cudaError_t launch_adam(const AdamArgs& a, const float* g_tr, const float* g_sh, const float* g_op, uint32_t n,
                        int degree, int sh_bf16, cudaStream_t st, int num_sms) {
  if (n == 0) return cudaSuccess;
  const int K = (degree + 1) * (degree + 1);
  const int blocks = num_sms * 8;
  adam_kernel<float><<<blocks, 256, 0, st>>>(a.transforms, g_tr, a.m_tr, a.v_tr, (uint64_t)n * 10, 0, a.scal);
  if (sh_bf16)
    adam_kernel<__nv_bfloat16><<<blocks, 256, 0, st>>>(reinterpret_cast<__nv_bfloat16*>(a.sh), g_sh, a.m_sh, a.v_sh,
                                                       (uint64_t)n * K * 3, 1, a.scal);
  else
    adam_kernel<float><<<blocks, 256, 0, st>>>(reinterpret_cast<float*>(a.sh), g_sh, a.m_sh, a.v_sh,
                                               (uint64_t)n * K * 3, 1, a.scal);
  adam_kernel<float><<<blocks, 256, 0, st>>>(a.raw_opac, g_op, a.m_op, a.v_op, n, 2, a.scal);
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
