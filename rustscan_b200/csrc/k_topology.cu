// k_topology.cu — device-side topology apply (RustGS/src/training/topology/
// apply.rs:10-94): the mutated splat set built on the device from a plan of
// rows (source index, kind, sample scalar), without the reference's round
// trip through a host snapshot. One thread per output row; the SH row is
// copied unchanged (f32 or bf16 bits).
#include <cuda_bf16.h>

#include "gsr_kernels.h"

namespace gsr {

namespace {

struct TopoArgs {
  const float* tr;
  const void* sh;
  const float* op;
  uint32_t n;
  const TopoRow* rows;
  uint32_t m;
  uint32_t sh_elems;  // SH scalars per row (3K)
  int sh_bf16;
  TopoParams p;
  float* otr;
  void* osh;
  float* oop;
  DevStatus* status;
};

__global__ void __launch_bounds__(256) topology_kernel(TopoArgs a) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.m; i += gridDim.x * blockDim.x) {
    const TopoRow row = a.rows[i];
    if (row.source >= a.n) {
      // A plan row naming a splat that does not exist: flag it, write zeros.
      atomicExch(&a.status->bad_input, 1u);
      for (int k = 0; k < 10; ++k) a.otr[(size_t)i * 10 + k] = 0.f;
      a.oop[i] = 0.f;
      continue;
    }
    float t[10];
    for (int k = 0; k < 10; ++k) t[k] = a.tr[(size_t)row.source * 10 + k];
    float logit = a.op[row.source];
    topo_mutate(t, logit, row.kind, row.sample, a.p);
    for (int k = 0; k < 10; ++k) a.otr[(size_t)i * 10 + k] = t[k];
    a.oop[i] = logit;
    if (a.sh_bf16) {
      const uint16_t* src = static_cast<const uint16_t*>(a.sh) + (size_t)row.source * a.sh_elems;
      uint16_t* dst = static_cast<uint16_t*>(a.osh) + (size_t)i * a.sh_elems;
      for (uint32_t k = 0; k < a.sh_elems; ++k) dst[k] = src[k];
    } else {
      const uint32_t* src = static_cast<const uint32_t*>(a.sh) + (size_t)row.source * a.sh_elems;
      uint32_t* dst = static_cast<uint32_t*>(a.osh) + (size_t)i * a.sh_elems;
      for (uint32_t k = 0; k < a.sh_elems; ++k) dst[k] = src[k];
    }
  }
}

}  // namespace

cudaError_t launch_topology(const SplatsDev& sp, const TopoRow* rows, uint32_t m, const TopoParams& p, float* otr,
                            void* osh, float* oop, DevStatus* status, cudaStream_t st, int num_sms) {
  if (m == 0) return cudaSuccess;
  TopoArgs a{};
  a.tr = sp.transforms;
  a.sh = sp.sh;
  a.op = sp.raw_opac;
  a.n = sp.n;
  a.rows = rows;
  a.m = m;
  const uint32_t K = (uint32_t)((sp.degree + 1) * (sp.degree + 1));
  a.sh_elems = 3 * K;
  a.sh_bf16 = sp.sh_bf16;
  a.p = p;
  a.otr = otr;
  a.osh = osh;
  a.oop = oop;
  a.status = status;
  int blocks = (int)((m + 255) / 256);
  if (blocks > num_sms * 8) blocks = num_sms * 8;
  topology_kernel<<<blocks, 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace gsr
