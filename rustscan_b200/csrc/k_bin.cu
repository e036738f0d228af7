// k_bin.cu — tile binning around the sorts: intersection emission
// (map_gaussian_to_intersects.wgsl), tile ranges (get_tile_offsets.wgsl),
// the visibility export and the deterministic-mode gradient reduction.
//
// Emission walks Gaussians in depth order and writes, for every tile that
// passes the contribution test, the tile id as key and the compact index as
// value at the Gaussian's scanned offset. The test reads the exact float
// values the counting pass used (stored in the projected record), so the
// emitted set always matches the counts (the reference recomputes the extent
// from the inverted conic here, which can disagree with its count pass).
#include <cstring>

#include "gsr_kernels.h"

namespace gsr {

namespace {

__device__ __forceinline__ TileBox unpack_box(float4 r2) {
  const uint32_t bx = __float_as_uint(r2.z), by = __float_as_uint(r2.w);
  TileBox b;
  b.x0 = bx & 0xffffu;
  b.x1 = bx >> 16;
  b.y0 = by & 0xffffu;
  b.y1 = by >> 16;
  return b;
}

__global__ void __launch_bounds__(256) emit_kernel(ViewSet vs, FwdBufs b, int det) {
  const uint32_t v = blockIdx.y;
  const uint32_t V = b.vcount[v * 4 + 0];
  const ViewDesc& vd = vs.views[v];
  const TileShape ts{vs.tile_w, vs.tile_h};
  const uint32_t* perm = slice(b.perm, b.Vcap, v);
  const uint32_t* off = slice(b.offset, b.Vcap, v);
  float4* rec_w = slice(b.rec, b.Vcap * 3, v);
  const float4* rec = rec_w;
  uint32_t* keys = slice(b.isect_key_raw, b.Icap, v);
  uint32_t* vals = slice(b.isect_val_raw, b.Icap, v);
  uint32_t* emit_c = det ? slice(b.inv_perm, b.Icap, v) : nullptr;
  const uint64_t cap = b.Icap;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < V; r += gridDim.x * blockDim.x) {
    const uint32_t c = perm[r];
    uint64_t o = off[r];
    const float4 r0 = rec[(size_t)c * 3 + 0];
    const float4 r1 = rec[(size_t)c * 3 + 1];
    const float4 r2 = rec[(size_t)c * 3 + 2];
    const V2<float> mean{r0.x, r0.y};
    const V3<float> conic{r0.z, r0.w, r1.x};
    const float thr = r2.y;
    const TileBox box = unpack_box(r2);
    for (uint32_t ty = box.y0; ty < box.y1; ++ty)
      for (uint32_t tx = box.x0; tx < box.x1; ++tx)
        if (will_primitive_contribute(tx, ty, ts, mean, conic, thr)) {
          if (o < cap) {
            keys[o] = tx + ty * vd.tiles_x;
            if (det) {
              vals[o] = (uint32_t)o;
              emit_c[o] = c;
            } else {
              vals[o] = c;
            }
          }
          ++o;
        }
    // The tile box is no longer needed: the record's last two slots now
    // carry the footprint half-widths the rasterizer culls warp blocks with
    // (negative: no box, never cull).
    float rx = -1.f, ry = -1.f;
    if (!footprint_box(conic.x, conic.y, conic.z, thr + kRejectMargin, rx, ry)) rx = ry = -1.f;
    float4* rw = rec_w + (size_t)c * 3 + 2;
    rw->z = rx;
    rw->w = ry;
  }
}

// Deterministic mode: the sort carried emission indices; turn them back into
// compact indices and record where each emission landed.
__global__ void __launch_bounds__(256) remap_kernel(FwdBufs b) {
  const uint32_t v = blockIdx.y;
  const uint32_t I = b.vcount[v * 4 + 1];
  uint32_t* vals = slice(b.isect_val, b.Icap, v);
  uint32_t* inv = slice(b.inv_perm, b.Icap, v);
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < I; s += gridDim.x * blockDim.x) {
    const uint32_t e = vals[s];
    const uint32_t c = inv[e];
    inv[e] = s;
    vals[s] = c;
  }
}

// get_tile_offsets.wgsl:11-30. ranges must be zeroed beforehand.
__global__ void __launch_bounds__(256) ranges_kernel(FwdBufs b) {
  const uint32_t v = blockIdx.y;
  const uint32_t I = b.vcount[v * 4 + 1];
  const uint32_t* keys = slice(b.isect_key, b.Icap, v);
  uint32_t* ranges = slice(b.ranges, 2 * b.Tcap, v);
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < I; s += gridDim.x * blockDim.x) {
    const uint32_t t = keys[s];
    if (t >= b.Tcap) continue;
    if (s == 0 || t != keys[s - 1]) ranges[2 * t] = s;
    if (s + 1 == I || t != keys[s + 1]) ranges[2 * t + 1] = s + 1;
  }
}

// visible[v][gid] = 1 for Gaussians that contributed to a pixel of view v
// (the `visible` output of rasterize.wgsl:270). out must be zeroed.
__global__ void __launch_bounds__(256) visible_kernel(FwdBufs b, uint32_t n, float* out) {
  const uint32_t v = blockIdx.y;
  const uint32_t V = b.vcount[v * 4 + 0];
  const uint8_t* vis = slice(b.visible_c, b.Vcap, v);
  const uint32_t* gid = slice(b.gid_of_c, b.Vcap, v);
  float* o = out + (size_t)n * v;
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < V; c += gridDim.x * blockDim.x)
    if (vis[c]) o[gid[c]] = 1.0f;
}

// Deterministic mode: per Gaussian, sum the per-intersection partial
// gradients in emission order (tiles in row-major box order).
__global__ void __launch_bounds__(256) reduce_det_kernel(FwdBufs b) {
  const uint32_t v = blockIdx.y;
  const uint32_t V = b.vcount[v * 4 + 0];
  const uint32_t* perm = slice(b.perm, b.Vcap, v);
  const uint32_t* off = slice(b.offset, b.Vcap, v);
  const uint32_t* cnt = slice(b.count, b.Vcap, v);
  const uint32_t* inv = slice(b.inv_perm, b.Icap, v);
  const float* part = b.sgrad_part + (size_t)b.Icap * 12 * v;
  float4* sg = slice(b.sgrad, b.Vcap * 3, v);
  const uint64_t cap = b.Icap;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < V; r += gridDim.x * blockDim.x) {
    const uint32_t c = perm[r];
    const uint64_t o = off[r];
    float acc[12];
    for (int k = 0; k < 12; ++k) acc[k] = 0.f;
    for (uint32_t i = 0; i < cnt[c]; ++i) {
      const uint64_t e = o + i;
      if (e >= cap) break;
      const float* p = part + (size_t)inv[e] * 12;
      for (int k = 0; k < 12; ++k) acc[k] = acc[k] + p[k];
    }
    sg[(size_t)c * 3 + 0] = make_float4(acc[0], acc[1], acc[2], acc[3]);
    sg[(size_t)c * 3 + 1] = make_float4(acc[4], acc[5], acc[6], acc[7]);
    sg[(size_t)c * 3 + 2] = make_float4(acc[8], acc[9], acc[10], acc[11]);
  }
}

__global__ void set_views_kernel(ViewDesc* dst, ViewDescBlock blk, uint32_t n) {
  if (threadIdx.x < n) dst[threadIdx.x] = blk.v[threadIdx.x];
}

dim3 grid_for(const ViewSet& vs, int num_sms) {
  int x = num_sms * 8 / (int)vs.n_views;
  if (x < 1) x = 1;
  return dim3(x, vs.n_views);
}

}  // namespace

cudaError_t launch_set_views(ViewDesc* dst, const ViewDesc* host, uint32_t n, cudaStream_t st) {
  if (n > (uint32_t)kMaxViews) return cudaErrorInvalidValue;
  ViewDescBlock blk;
  memset(&blk, 0, sizeof(blk));
  for (uint32_t i = 0; i < n; ++i) blk.v[i] = host[i];
  set_views_kernel<<<1, kMaxViews, 0, st>>>(dst, blk, n);
  return cudaGetLastError();
}

cudaError_t launch_emit(const ViewSet& vs, FwdBufs& b, const Scratch& s, int deterministic, cudaStream_t st) {
  emit_kernel<<<grid_for(vs, s.num_sms), 256, 0, st>>>(vs, b, deterministic);
  return cudaGetLastError();
}

cudaError_t launch_remap(const ViewSet& vs, FwdBufs& b, const Scratch& s, cudaStream_t st) {
  remap_kernel<<<grid_for(vs, s.num_sms), 256, 0, st>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_ranges(const ViewSet& vs, FwdBufs& b, const Scratch& s, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(b.ranges, 0, sizeof(uint32_t) * 2 * b.Tcap * vs.n_views, st);
  if (e != cudaSuccess) return e;
  ranges_kernel<<<grid_for(vs, s.num_sms), 256, 0, st>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_visible_out(const ViewSet& vs, FwdBufs& b, uint32_t n, float* out, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float) * (size_t)n * vs.n_views, st);
  if (e != cudaSuccess) return e;
  visible_kernel<<<dim3(256, vs.n_views), 256, 0, st>>>(b, n, out);
  return cudaGetLastError();
}

cudaError_t launch_reduce_det(const ViewSet& vs, FwdBufs& b, const Scratch& s, cudaStream_t st) {
  reduce_det_kernel<<<grid_for(vs, s.num_sms), 256, 0, st>>>(b);
  return cudaGetLastError();
}

}  // namespace gsr
