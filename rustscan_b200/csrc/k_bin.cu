// k_bin.cu — tile binning around the sorts: intersection emission
// (map_gaussian_to_intersects.wgsl), tile ranges (get_tile_offsets.wgsl),
// the visibility export and the deterministic-mode gradient reduction.
//
// Counting (the per-Gaussian tile count of project_forward.wgsl:79-91) and
// emission both run the contribution test on the exact float values stored
// in the projected record, so the emitted set always matches the counts (the
// reference recomputes the extent from the inverted conic at emission, which
// can disagree with its count pass).
#include <cstring>

#include "gsr_kernels.h"

namespace gsr {

namespace {

// Warp-cooperative tile walk. The 32 Gaussians of a warp have boxes of very
// different sizes (one tile to thousands), so a loop per thread would leave
// most lanes idle. The warp flattens its Gaussians' boxes into one item list
// (lane-major, row-major within a box: the emission order) and every pass
// tests 32 consecutive items, one per lane. Passing items are ranked within
// their Gaussian with ballots, so each Gaussian's tiles keep their row-major
// order and the output is the same as a per-Gaussian loop.
struct WalkWarp {
  uint4 box[32];      // exclusive prefix of box sizes, box width, box origin x, y
  float4 g0[32];      // mean x, y, conic a, b
  float4 g1[32];      // conic c, cut, 1 / box width, -
  uint32_t run[32];  // passing tiles found so far, per Gaussian
  uint32_t off[32];  // emission offset, per Gaussian
  uint32_t cid[32];  // compact index, per Gaussian
  uint32_t lane_of_rank[32];  // lanes of the Gaussians with a non-empty box, in lane order
};

constexpr int kWalkThreads = 256;
constexpr int kWalkWarps = kWalkThreads / 32;
// Walk blocks per SM in the launch (4 are resident at a time). Box sizes
// vary by orders of magnitude between Gaussians, and many short blocks
// balance them better than a few long grid-stride ones: emission of the
// 8-view step took 0.52 ms at 4, 0.43 at 8, 0.41 at 16 and 0.39 at 24 to
// 48, where the per-block tile-count flush starts to cost what balance gains.
constexpr int kWalkBlocksPerSm = 24;

// EMIT = false: count the passing tiles of every compact index (gid order).
// EMIT = true: walk the Gaussians in depth order and write, for every
// passing tile, the tile id as key and the compact index as value at the
// Gaussian's scanned offset; then replace the record's tile box with the
// footprint half-widths the rasterizer culls warp blocks with (negative: no
// box, never cull).
// SLOTS (emission only): every box tile of a Gaussian has a slot at its
// row-major position after the Gaussian's offset (offsets scanned from box
// sizes, no counting walk); a passing tile writes its key there (packed, or
// the tile id with the compact index as value), a failing one the all-ones
// key, which sorts after every tile.
template <bool EMIT, bool HIST = false, bool SLOTS = false>
// 5 resident blocks per SM (48 registers): emission of the 8-view step 0.395
// -> 0.382 ms against 4 (54 registers); 6 spills and is slower.
__global__ void __launch_bounds__(kWalkThreads, 5) tile_walk_kernel(ViewSet vs, FwdBufs b, int det) {
  __shared__ WalkWarp s_w[kWalkWarps];
  extern __shared__ uint32_t s_th[];  // HIST: per-tile counts of this block's emitted intersections
  const uint32_t v = blockIdx.y;
  const uint32_t V = b.vcount[v * 4 + 0];
  const ViewDesc& vd = vs.views[v];
  const TileShape ts{vs.tile_w, vs.tile_h};
  const uint32_t* perm = slice(b.perm, b.Vcap, v);
  const uint32_t* off = slice(b.offset, b.Vcap, v);
  float4* rec_w = slice(b.rec, b.Vcap * 3, v);
  const float4* rec = rec_w;
  uint32_t* count = slice(b.count, b.Vcap, v);
  uint32_t* keys = slice(b.isect_key_raw, b.Icap, v);
  uint32_t* vals = slice(b.isect_val_raw, b.Icap, v);
  uint32_t* emit_c = det ? slice(b.inv_perm, b.Icap, v) : nullptr;
  const uint64_t cap = b.Icap;
  const uint32_t lane = threadIdx.x & 31u;
  WalkWarp& S = s_w[threadIdx.x >> 5];
  const uint32_t T = vd.tiles_x * vd.tiles_y;
  if (HIST) {
    for (uint32_t t = threadIdx.x; t < T; t += kWalkThreads) s_th[t] = 0u;
    __syncthreads();
  }
  const uint32_t stride = gridDim.x * kWalkWarps * 32u;
  for (uint32_t base = (blockIdx.x * kWalkWarps + (threadIdx.x >> 5)) * 32u; base < V; base += stride) {
    const uint32_t r = base + lane;
    uint32_t nb = 0u, c = 0u, x0 = 0u, y0 = 0u, w = 0u, o0 = 0u;
    V2<float> mean{0.f, 0.f};
    V3<float> conic{0.f, 0.f, 0.f};
    float thr = 0.f;
    if (r < V) {
      c = EMIT ? perm[r] : r;
      const float4 r0 = rec[(size_t)c * 3 + 0];
      const float4 r1 = rec[(size_t)c * 3 + 1];
      const float4 r2 = rec[(size_t)c * 3 + 2];
      mean = V2<float>{r0.x, r0.y};
      conic = V3<float>{r0.z, r0.w, r1.x};
      thr = r2.y;
      const uint32_t bx = __float_as_uint(r2.z), by = __float_as_uint(r2.w);
      x0 = bx & 0xffffu;
      y0 = by & 0xffffu;
      const uint32_t x1 = bx >> 16, y1 = by >> 16;
      w = x1 > x0 ? x1 - x0 : 0u;
      nb = w * (y1 > y0 ? y1 - y0 : 0u);
      if (EMIT) o0 = off[r];
    }
    uint32_t incl = nb;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= (uint32_t)d) incl += t;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    __syncwarp();  // the previous round's readers of S are done
    S.box[lane] = make_uint4(incl - nb, w, x0, y0);
    S.g0[lane] = make_float4(mean.x, mean.y, conic.x, conic.y);
    S.g1[lane] = make_float4(conic.z, thr, w ? 1.0f / (float)w : 0.f, 0.f);
    S.run[lane] = 0u;
    S.off[lane] = o0;
    S.cid[lane] = c;
    const uint32_t nzm = __ballot_sync(0xffffffffu, nb > 0u);
    if (nb > 0u) S.lane_of_rank[__popc(nzm & ((1u << lane) - 1u))] = lane;
    __syncwarp();
    const uint32_t ex = incl - nb;
    for (uint32_t t0 = 0; t0 < total; t0 += 32u) {
      const uint32_t t = t0 + lane;
      const bool live = t < total;
      // Owner of item t: the Gaussians with a non-empty box own consecutive
      // item runs. The run starts inside [t0, t0 + 32) mark bits; the owner of
      // t0 is the first Gaussian whose run ends after t0, and every start at
      // positions 1..lane moves the owner of t0 + lane one Gaussian further.
      const uint32_t sbit = (nb > 0u && ex >= t0 && ex < t0 + 32u) ? (1u << (ex - t0)) : 0u;
      const uint32_t starts = __reduce_or_sync(0xffffffffu, sbit);
      const uint32_t r0 = (uint32_t)__popc(__ballot_sync(0xffffffffu, nb > 0u && incl <= t0));
      uint32_t owner = 0u, tx = 0u, ty = 0u, local = 0u;
      bool pass = false;
      if (live) {
        const uint32_t upto = ((2u << lane) - 1u) & ~1u;  // positions 1..lane
        owner = S.lane_of_rank[r0 + (uint32_t)__popc(starts & upto)];
        const uint4 bx = S.box[owner];
        const float4 ga = S.g0[owner], gb = S.g1[owner];
        local = t - bx.x;
        // Row and column of the item in its box: the quotient from the
        // float reciprocal is within one of the exact one for local < 2^24,
        // and the remainder's range fixes it.
        const uint32_t ow = bx.y;
        uint32_t ry, rx;
        if (local < (1u << 24)) {
          ry = __float2uint_rz(__uint2float_rn(local) * gb.z);
          rx = local - ry * ow;
          if ((int32_t)rx < 0) {
            --ry;
            rx += ow;
          } else if (rx >= ow) {
            ++ry;
            rx -= ow;
          }
        } else {
          ry = local / ow;
          rx = local - ry * ow;
        }
        tx = bx.z + rx;
        ty = bx.w + ry;
        pass = will_primitive_contribute(tx, ty, ts, V2<float>{ga.x, ga.y}, V3<float>{ga.z, ga.w, gb.x}, gb.y);
      }
      if (SLOTS) {
        if (live) {
          const uint64_t o = (uint64_t)S.off[owner] + local;
          if (o < cap) {
            if (pass) {
              if (HIST) atomicAdd(&s_th[tx + ty * vd.tiles_x], 1u);
              keys[o] = b.pack_bits ? ((tx + ty * vd.tiles_x) << b.pack_bits) | S.cid[owner] : tx + ty * vd.tiles_x;
            } else {
              keys[o] = 0xffffffffu;
            }
            if (!b.pack_bits) vals[o] = S.cid[owner];
          }
        }
        continue;
      }
      const uint32_t pm = __ballot_sync(0xffffffffu, pass);
      const uint32_t prev = __shfl_up_sync(0xffffffffu, owner, 1);
      const bool start = live && (lane == 0u || prev != owner);
      const uint32_t sm = __ballot_sync(0xffffffffu, start);
      if (EMIT && pass) {
        const uint32_t first = 31u - (uint32_t)__clz(sm & ((2u << lane) - 1u));
        const uint32_t before = pm & ((1u << lane) - 1u) & ~((1u << first) - 1u);
        const uint64_t o = (uint64_t)S.off[owner] + S.run[owner] + (uint32_t)__popc(before);
        if (o < cap) {
          if (HIST) atomicAdd(&s_th[tx + ty * vd.tiles_x], 1u);
          if (b.pack_bits) {
            keys[o] = ((tx + ty * vd.tiles_x) << b.pack_bits) | S.cid[owner];
          } else if (det) {
            keys[o] = tx + ty * vd.tiles_x;
            vals[o] = (uint32_t)o;
            emit_c[o] = S.cid[owner];
          } else {
            keys[o] = tx + ty * vd.tiles_x;
            vals[o] = S.cid[owner];
          }
        }
      }
      __syncwarp();
      if (start) {
        const uint32_t later = sm & ~((2u << lane) - 1u);
        const uint32_t seg_hi = later ? ((1u << (__ffs(later) - 1)) - 1u) : 0xffffffffu;
        S.run[owner] += (uint32_t)__popc(pm & seg_hi & ~((1u << lane) - 1u));
      }
      __syncwarp();
    }
    if (r < V) {
      if (!EMIT) {
        count[c] = S.run[lane];
      } else {
        float rx = -1.f, ry = -1.f;
        if (!footprint_box(conic.x, conic.y, conic.z, thr + kRejectMargin, rx, ry)) rx = ry = -1.f;
        float4* rw = rec_w + (size_t)c * 3 + 2;
        rw->z = rx;
        rw->w = ry;
      }
    }
  }
  if (HIST) {
    __syncthreads();
    uint32_t* th = slice(b.tile_hist, b.Tcap, v);
    for (uint32_t t = threadIdx.x; t < T; t += kWalkThreads)
      if (s_th[t]) atomicAdd(th + t, s_th[t]);
  }
}

// From the per-tile counts of one view: the tile ranges
// (get_tile_offsets.wgsl:11-30 — [start, end) per tile, 0,0 when empty) and
// the digit histograms of the tile sort's (at most two) passes over the
// tile id's digits, in the sort's histogram layout.
constexpr int kHistThreads = 1024;
__global__ void __launch_bounds__(kHistThreads) tile_hist_finish_kernel(ViewSet vs, FwdBufs b, uint32_t* hist,
                                                                         uint32_t dbits, uint32_t dbits1, int slots) {
  __shared__ uint32_t s_scan[32];
  __shared__ uint32_t s_h[2][256];
  const uint32_t v = blockIdx.x;
  const ViewDesc& vd = vs.views[v];
  const uint32_t T = vd.tiles_x * vd.tiles_y;
  const uint32_t* th = slice(b.tile_hist, b.Tcap, v);
  uint32_t* ranges = slice(b.ranges, 2 * b.Tcap, v);
  for (int i = threadIdx.x; i < 512; i += kHistThreads) (&s_h[0][0])[i] = 0u;
  constexpr uint32_t kPer = kHistMaxTiles / kHistThreads;
  const uint32_t t0 = threadIdx.x * kPer;
  uint32_t loc[kPer];
  uint32_t sum = 0;
#pragma unroll
  for (uint32_t i = 0; i < kPer; ++i) {
    loc[i] = t0 + i < T ? th[t0 + i] : 0u;
    sum += loc[i];
  }
  uint32_t all;
  uint32_t run = block_exclusive_scan(sum, s_scan, &all);  // its barriers also order the zeroing above
#pragma unroll
  for (uint32_t i = 0; i < kPer; ++i) {
    const uint32_t t = t0 + i;
    if (t < T) {
      ranges[2 * t] = loc[i] ? run : 0u;
      ranges[2 * t + 1] = loc[i] ? run + loc[i] : 0u;
      if (loc[i]) {
        atomicAdd(&s_h[0][t & ((1u << dbits) - 1u)], loc[i]);
        atomicAdd(&s_h[1][(t >> dbits) & ((1u << dbits1) - 1u)], loc[i]);
      }
    }
    run += loc[i];
  }
  if (slots && threadIdx.x == 0) {
    // Slot layout: the sort covers every slot written (the scanned box
    // sizes, clamped to capacity); the slots of failing tiles hold the
    // all-ones key. Either the sort drops those in its first pass (slots ==
    // 2, digits below 8 bits) and the histograms count the real keys only,
    // or they are sorted along (slots == 1): their digits are then counted
    // as the sort takes them, from bit pack_bits (0 for pairs) in
    // dbits-wide steps (the top digit of a packed key can be narrower than
    // dbits); over the sorted bits the key exceeds every tile id, so it
    // sorts last. The view's intersection count becomes the real one.
    const uint32_t written = b.vcount[v * 4 + 1];
    if (slots == 1) {
      atomicAdd(&s_h[0][(uint32_t)(0xffffffffull >> b.pack_bits) & ((1u << dbits) - 1u)], written - all);
      atomicAdd(&s_h[1][(uint32_t)(0xffffffffull >> (b.pack_bits + dbits)) & ((1u << dbits1) - 1u)], written - all);
    }  // slots == 2: the sort drops the sentinels in its first pass
    b.vcount[v * 4 + 3] = written;
    b.vcount[v * 4 + 1] = all;
    b.vcount[v * 4 + 2] = all;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 1024; i += kHistThreads) {
    const int p = i >> 8;
    hist[(size_t)v * 1024 + i] = p < 2 ? s_h[p][i & 255] : 0u;
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

// Packed intersections of one view back to (tile id, compact index) pairs
// (inspection exports).
__global__ void __launch_bounds__(256) unpack_isects_kernel(const uint32_t* packed, uint32_t n, uint32_t bits,
                                                            uint32_t* tiles, uint32_t* vals) {
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const uint32_t k = packed[s];
    tiles[s] = k >> bits;
    vals[s] = k & ((1u << bits) - 1u);
  }
}

// Passing-tile counts per compact index from the sorted packed keys of one
// view (the slot layout has no counting walk); count must be zeroed.
__global__ void __launch_bounds__(256) count_from_isects_kernel(const uint32_t* keys, const uint32_t* n_isects,
                                                                uint32_t mask, uint32_t* count) {
  const uint32_t n = *n_isects;
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x)
    atomicAdd(count + (keys[s] & mask), 1u);
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
// (the `visible` output of rasterize.wgsl:79). out must be zeroed.
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

dim3 grid_for(const ViewSet& vs, int num_sms, int per_sm = 8) {
  int x = num_sms * per_sm / (int)vs.n_views;
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

cudaError_t launch_count(const ViewSet& vs, FwdBufs& b, const Scratch& s, cudaStream_t st) {
  tile_walk_kernel<false><<<grid_for(vs, s.num_sms, kWalkBlocksPerSm), kWalkThreads, 0, st>>>(vs, b, 0);
  return cudaGetLastError();
}

cudaError_t launch_emit(const ViewSet& vs, FwdBufs& b, const Scratch& s, int deterministic, cudaStream_t st) {
  tile_walk_kernel<true><<<grid_for(vs, s.num_sms, kWalkBlocksPerSm), kWalkThreads, 0, st>>>(vs, b, deterministic);
  return cudaGetLastError();
}

cudaError_t launch_emit_hist(const ViewSet& vs, FwdBufs& b, const Scratch& s, int deterministic, bool slots,
                             cudaStream_t st) {
  if (vs.max_tiles > kHistMaxTiles) return cudaErrorInvalidValue;
  if (slots && deterministic) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(b.tile_hist, 0, sizeof(uint32_t) * b.Tcap * vs.n_views, st);
  if (e != cudaSuccess) return e;
  const size_t smem = sizeof(uint32_t) * vs.max_tiles;
  // The per-tile counts may take the static walk state past the 48 KB
  // default: allow the largest histogram.
  if (slots) {
    e = cudaFuncSetAttribute(tile_walk_kernel<true, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(uint32_t) * kHistMaxTiles));
    if (e != cudaSuccess) return e;
    tile_walk_kernel<true, true, true><<<grid_for(vs, s.num_sms, kWalkBlocksPerSm), kWalkThreads, smem, st>>>(vs, b, 0);
  } else {
    e = cudaFuncSetAttribute(tile_walk_kernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(uint32_t) * kHistMaxTiles));
    if (e != cudaSuccess) return e;
    tile_walk_kernel<true, true><<<grid_for(vs, s.num_sms, kWalkBlocksPerSm), kWalkThreads, smem, st>>>(vs, b, deterministic);
  }
  return cudaGetLastError();
}

cudaError_t launch_tile_hist_finish(const ViewSet& vs, FwdBufs& b, const Scratch& s, int tile_bits, bool slots,
                                   bool drop_sentinels, cudaStream_t st) {
  if (vs.max_tiles > kHistMaxTiles || sort_passes(tile_bits) > 2) return cudaErrorInvalidValue;
  const int d0 = tile_first_digit_bits(tile_bits);
  tile_hist_finish_kernel<<<vs.n_views, kHistThreads, 0, st>>>(vs, b, s.hist, (uint32_t)d0,
                                                                (uint32_t)(tile_bits > d0 ? tile_bits - d0 : d0),
                                                                slots ? (drop_sentinels ? 2 : 1) : 0);
  return cudaGetLastError();
}

cudaError_t launch_count_from_isects(FwdBufs& b, uint32_t view, uint32_t n_visible, cudaStream_t st) {
  uint32_t* count = slice(b.count, b.Vcap, view);
  cudaError_t e = cudaMemsetAsync(count, 0, sizeof(uint32_t) * n_visible, st);
  if (e != cudaSuccess) return e;
  count_from_isects_kernel<<<1024, 256, 0, st>>>(isect_index_src(b, view), b.vcount + view * 4 + 1,
                                                 isect_index_mask_host(b), count);
  return cudaGetLastError();
}

cudaError_t launch_unpack_isects(const FwdBufs& b, uint32_t view, uint32_t n, uint32_t* tiles, uint32_t* vals,
                                 cudaStream_t st) {
  if (!b.pack_bits || n == 0) return cudaSuccess;
  const uint32_t blocks = (n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096;
  unpack_isects_kernel<<<blocks, 256, 0, st>>>(slice(b.isect_key, b.Icap, view), n, b.pack_bits, tiles, vals);
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
