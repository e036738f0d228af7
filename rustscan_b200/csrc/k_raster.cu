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
// of the last contributor, and per list entry a bit for each warp block in
// which some pixel took the Gaussian. The backward walks, per warp, only the
// entries whose forward bit covers its block (its contributor decisions
// repeat the forward's, so no other entry can contribute there), from
// the tile's largest last index down, recovers the transmittance before each
// contributor by division (T_i = T_{i+1} / (1 - alpha_i)), keeps the colour
// accumulated behind it, and forms per-pixel gradients (blend_step_grad).
// Per Gaussian the gradient sums over a warp's pixels come from a
// reduce-scatter butterfly (13 shuffles), over the CTA's warps from shared
// memory in warp order, and over tiles from float4 atomics (or, in
// deterministic mode, per-intersection records reduced later in a fixed
// order).
//
// Work items are the (view, tile) pairs of the launch. With the persistent
// schedule the raster kernels run as many CTAs as the SMs hold at once, each
// taking the next item from an atomic ticket, in decreasing order of an
// estimated cost, so the longest tiles start first and the launch does not
// end in a tail of long tiles on a few SMs; views of different sizes and
// visible counts share one queue. The backward's cost is the number of list
// entries up to the tile's last contributor: the forward appends each item
// to the list of its cost's bit length (33 lists), and a backward ticket
// walks the lists from the longest costs down. A persistent forward orders
// its items by list length with a single-block counting sort first.
// Otherwise one CTA per item runs in item order.
#include <algorithm>

#include <type_traits>

#include "gsr_kernels.h"

namespace gsr {

namespace {

// Pixels per lane. The forward gains nothing from more than 2. The
// backward of 16x16 tiles runs one warp per tile with 8 pixels per lane
// (raster_bwd_tile_kernel) when the launch has tiles enough to fill the
// GPU several times over with one-warp CTAs, so that each Gaussian's warp
// reduction serves the whole tile; otherwise two warps per tile with 4
// pixels per lane (raster_bwd_kernel), which keeps twice the warps busy on a
// small view. The other tile shapes run raster_bwd_kernel with 2.
constexpr int kFwdPPL = 2;
static_assert(4 * kFwdPPL == 8, "forward warp blocks, and so the exported hit bits, are 8x8 pixels");
constexpr int kBwdPPL = 2;
constexpr int kBwdPPL16 = 4;
// One-warp CTA waves (the tile kernel's residency times the SMs) a launch
// must fill before the 16x16 backward runs one warp per tile.
constexpr uint32_t kTileKernelWaves = 4;
// The one-warp backward's batch (entries staged per round, double-buffered)
// and its resident CTAs per SM: 64 entries take 13 KB of shared memory, so
// that 16 CTAs fit an SM, the register bound of 16 (at most 128 a thread).
constexpr int kTileBwdBatch = 64;
constexpr int kTileBwdBlocks = 16;

struct RasterArgs {
  ViewSet vs;
  FwdBufs b;
  float bg[3];
  float* out_rgba;
  const float* v_rgba;
  int ref_mode;
  int det;
  int persist;  // 0: one CTA per item; 1: persistent, items from sched_order; 2: persistent, items from the cost lists
};

__device__ __forceinline__ uint32_t find_view(const ViewSet& vs, uint32_t item) {
  uint32_t v = 0;
  for (uint32_t i = 1; i < vs.n_views; ++i)
    if (vs.views[i].tile_base <= item) v = i;
  return v;
}

constexpr uint32_t kNoItem = 0xffffffffu;

constexpr int kCostLists = 33;  // bit lengths 0..32 of a cost

__device__ __forceinline__ uint32_t cost_bucket(uint32_t cost) { return cost ? 32u - (uint32_t)__clz(cost) : 0u; }

// Per CTA, for the cost lists: each list's length and its first ticket
// (lists in decreasing cost order). Read once per launch.
struct CostListView {
  uint32_t count[kCostLists];
  uint32_t first[kCostLists];
};
__device__ __forceinline__ void load_cost_lists(const RasterArgs& a, CostListView* s) {
  if (a.persist != 2) return;
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    for (int k = kCostLists - 1; k >= 0; --k) {
      const uint32_t n = a.b.sched_lcount[k];
      s->count[k] = n;
      s->first[k] = run;
      run += n;
    }
  }
}

// The next work item of this CTA (block-uniform; kNoItem when done). In
// the grid schedule a CTA runs item blockIdx.x once; in the persistent one
// thread 0 takes a ticket and reads the item at that place of the cost
// order. The leading barrier keeps the previous item's shared state intact
// until every thread is done with it (and publishes load_cost_lists).
__device__ __forceinline__ uint32_t next_item(const RasterArgs& a, uint32_t round, uint32_t* s_item,
                                              const CostListView* lists) {
  if (!a.persist) return round == 0 ? blockIdx.x : kNoItem;
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t slot = atomicAdd(a.b.sched_ticket, 1u);
    uint32_t item = kNoItem;
    if (slot < a.vs.total_tiles) {
      if (a.persist == 1) {
        item = a.b.sched_order[slot];
      } else {
        for (int k = kCostLists - 1; k >= 0; --k) {
          if (slot - lists->first[k] < lists->count[k]) {
            item = a.b.sched_lists[(size_t)k * a.b.sched_items_cap + (slot - lists->first[k])];
            break;
          }
        }
      }
    }
    *s_item = item;
  }
  __syncthreads();
  return *s_item;
}

// One block: the work items of a persistent forward in decreasing order of
// cost bucket (bit length of the list length; order within a bucket is
// arbitrary), and the ticket reset.
constexpr int kOrderThreads = 1024;
__global__ void __launch_bounds__(kOrderThreads) sched_order_kernel(ViewSet vs, FwdBufs b) {
  __shared__ uint32_t s_hist[kCostLists];
  __shared__ uint32_t s_start[kCostLists];
  if (threadIdx.x < kCostLists) s_hist[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t total = vs.total_tiles;
  auto cost_of = [&](uint32_t item) -> uint32_t {
    const uint32_t v = find_view(vs, item);
    const uint32_t t = item - vs.views[v].tile_base;
    const uint32_t* r = slice(b.ranges, 2 * b.Tcap, v);
    return r[2 * t + 1] - r[2 * t];
  };
  for (uint32_t i = threadIdx.x; i < total; i += kOrderThreads) atomicAdd(&s_hist[cost_bucket(cost_of(i))], 1u);
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    for (int k = kCostLists - 1; k >= 0; --k) {
      s_start[k] = run;
      run += s_hist[k];
    }
    *b.sched_ticket = 0u;
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < total; i += kOrderThreads)
    b.sched_order[atomicAdd(&s_start[cost_bucket(cost_of(i))], 1u)] = i;
}

// Warp w of a TW-wide tile owns the 8 x (4*PPL) block at (x0, y0); lane l
// owns column x0 + (l & 7) and rows y0 + (l >> 3) + 4q, q = 0..PPL-1.
template <int TW, int PPL> struct WarpBlock {
  static_assert(TW % 8 == 0, "tile width is a multiple of the 8-pixel warp block");
  static constexpr int kWarpsX = TW / 8;
  static constexpr int kRows = 4 * PPL;
  __device__ static int x0(int w) { return (w % kWarpsX) * 8; }
  __device__ static int y0(int w) { return (w / kWarpsX) * kRows; }
};

// Stages one Gaussian for the forward: its blend terms (colours clamped at
// zero) plus the bit mask of warp blocks its padded footprint box overlaps
// (half-widths written by the emission kernel into r2.zw; negative means no
// box, never cull).
template <int TW, int PPL, int NW>
__device__ __forceinline__ uint32_t stage_one(const float4* rec, uint32_t c, float tx0, float ty0, float4& A, float4& B,
                                              float4& Cc) {
  const float4 r0 = rec[(size_t)c * 3 + 0];
  const float4 r1 = rec[(size_t)c * 3 + 1];
  const float4 r2 = rec[(size_t)c * 3 + 2];
  A = make_float4(r0.x, r0.y, r0.z, 2.f * r0.w);  // 2b is exact
  B = make_float4(r1.x, r2.y + kRejectMargin, r1.y, 0.f);
  Cc = make_float4(fmaxf(r1.z, 0.f), fmaxf(r1.w, 0.f), fmaxf(r2.x, 0.f), 0.f);
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

// Order-preserving compaction of the batch entries whose mask has a bit of
// wsel.
__device__ __forceinline__ int build_list(const uint8_t* s_mask, uint32_t nb, uint32_t wsel, int lane,
                                          uint16_t* list) {
  int cnt = 0;
  for (uint32_t base = 0; base < nb; base += 32) {
    const uint32_t j = base + lane;
    const bool bit = j < nb && (s_mask[j] & wsel) != 0u;
    const uint32_t bal = __ballot_sync(0xffffffffu, bit);
    if (bit) list[cnt + __popc(bal & ((1u << lane) - 1u))] = (uint16_t)j;
    cnt += __popc(bal);
  }
  __syncwarp();
  return cnt;
}

// Paired FP32 arithmetic: every lane owns its pixels in pairs (rows y + 8k and
// y + 8k + 4 of one column), and the per-pixel arithmetic of a pair runs as
// two-wide operations (fma2 is a fused multiply-add per half, add2 and mul2
// round per half like the scalar operations).
//
// The compiler contracts a paired multiply feeding a paired add into one
// fused multiply-add, even when written as PTX with .rn and with contraction
// switched off (--fmad=false; measured: the paired and the fused results
// agree bit for bit, the separately rounded scalar chain does not). The
// decision arithmetic is therefore defined with its multiply-adds fused
// (sigma and the range reduction of the exponential, gsr_math.h), and the
// kernels spell those as fma2, which is then exact by construction; no
// decision depends on a paired multiply feeding a paired add. The file is
// built without contraction, like the CPU oracle, so that the remaining
// scalar expressions keep their written rounding.
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

// blend_sigma_shared for the two pixels of a pair (same column: same t1,
// t2): the same operations in the same order, each half rounded on its own.
__device__ __forceinline__ float2 sigma2(float t1, float t2, float2 dy, float cc) {
  return mul2(f2(0.5f), fma2(mul2(f2(cc), dy), dy, fma2(f2(t2), dy, f2(t1))));
}

// blend_expf(-sigma) for both pixels, without its range clamps: for every
// sigma the contribution test can accept (0 <= sigma <= log(255) + margin)
// they change nothing, so there the result is bit-identical to blend_expf.
// For a pixel outside that range the value is meaningless (possibly not
// finite); every use of it is selected away by the pixel's contribution
// flags, never multiplied in.
__device__ __forceinline__ float2 blend_exp2(float2 sigma) {
  const float2 x = make_float2(-sigma.x, -sigma.y);
  const float2 t = fma2(x, f2(bexp::kLog2e), f2(bexp::kMagic));
  const float2 n = add2(t, f2(-bexp::kMagic));
  // 2^n by exponent-field addition, as blend_expf: t's bits are those of
  // 1.5 * 2^23 plus n, and a left shift by 23 drops the constant (its low 22
  // bits are zero), leaving n << 23 modulo 2^32.
  static_assert((bexp::kMagicBits << 23) == 0u, "the constant part shifts out");
  const uint32_t ex = __float_as_uint(t.x) << 23;
  const uint32_t ey = __float_as_uint(t.y) << 23;
  float2 r = fma2(neg2(n), f2(bexp::kLn2Hi), x);
  r = fma2(neg2(n), f2(bexp::kLn2Lo), r);
  float2 p = f2(bexp::kC6);
  p = fma2(p, r, f2(bexp::kC5));
  p = fma2(p, r, f2(bexp::kC4));
  p = fma2(p, r, f2(bexp::kC3));
  p = fma2(p, r, f2(bexp::kC2));
  p = fma2(p, r, f2(1.0f));
  p = fma2(p, r, f2(1.0f));
  return make_float2(__uint_as_float(__float_as_uint(p.x) + ex), __uint_as_float(__float_as_uint(p.y) + ey));
}

// Per-entry terms of a forward step for one pixel pair.
struct FwdPre {
  float2 sg;       // sigma of both pixels
  float opac;
  float ax, ay;    // alpha of both pixels
  bool l0, l1;     // within the cut
  bool c0, c1;     // contributes (before the pixel-state gate)
};

template <int TW, int TH, int PPL, int BATCH>
__global__ void __launch_bounds__(TW* TH / PPL) raster_fwd_kernel(RasterArgs a) {
  static_assert(PPL % 2 == 0, "pixels per lane come in pairs");
  static_assert(TH % (4 * PPL) == 0 && (TW * TH / PPL) % 32 == 0, "warp blocks tile the tile");
  constexpr int NT = TW * TH / PPL;
  constexpr int NW = NT / 32;
  constexpr int NP = PPL / 2;
  __shared__ float4 s_a[BATCH];  // x, y, conic a, 2 conic b
  __shared__ float4 s_b[BATCH];  // conic c, reject cut, opacity, -
  __shared__ float4 s_c[BATCH];  // max(r,0), max(g,0), max(b,0), -
  __shared__ uint32_t s_cidx[BATCH];
  __shared__ uint8_t s_mask[BATCH];
  __shared__ uint8_t s_hit[NW][BATCH];  // warp w took entry j
  __shared__ uint16_t s_list[NW][BATCH];
  __shared__ uint32_t s_item;
  __shared__ uint32_t s_work;
  __shared__ CostListView s_lists;
  if (threadIdx.x == 0) s_work = 0u;
  load_cost_lists(a, &s_lists);
  for (uint32_t round = 0;; ++round) {
    const uint32_t item = next_item(a, round, &s_item, &s_lists);
    if (item == kNoItem) break;
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
    const uint32_t* vals = isect_index_src(a.b, v);
    const uint32_t vmask = isect_index_mask(a.b);
    const float4* rec = slice(a.b.rec, a.b.Vcap * 3, v);
    uint8_t* vis = slice(a.b.visible_c, a.b.Vcap, v);
    uint8_t* hitw = slice(a.b.hitw, a.b.Icap, v);
    const float tx0 = (float)(tx * TW), ty0 = (float)(ty * TH);
    // Pixel q = 2k + h sits at row pyb + 4q and is half h of pair k.
    float2 T[NP], C0[NP], C1[NP], C2[NP], npcy[NP];
    uint32_t last[PPL], nc[PPL];  // a pixel that saturates stops at its last contributor
    bool done[PPL];
    bool all_done = true;
  #pragma unroll
    for (int k = 0; k < NP; ++k) {
      T[k] = f2(1.f);
      C0[k] = C1[k] = C2[k] = f2(0.f);
      npcy[k] = make_float2(-((float)(pyb + 8 * k) + 0.5f), -((float)(pyb + 8 * k + 4) + 0.5f));
    }
  #pragma unroll
    for (int q = 0; q < PPL; ++q) {
      const uint32_t py = pyb + 4 * q;
      last[q] = nc[q] = 0;
      done[q] = !(px < vd.w && py < vd.h);
      all_done = all_done && done[q];
    }
    for (uint32_t b0 = s0; b0 < s1; b0 += BATCH) {
      const uint32_t nb = min((uint32_t)BATCH, s1 - b0);
      __syncthreads();
      for (uint32_t j = threadIdx.x; j < nb; j += NT) {
        const uint32_t c = vals[b0 + j] & vmask;
        float4 A, B, Cc;
        s_mask[j] = (uint8_t)stage_one<TW, PPL, NW>(rec, c, tx0, ty0, A, B, Cc);
        s_a[j] = A;
        s_b[j] = B;
        s_c[j] = Cc;
        s_cidx[j] = c;
  #pragma unroll
        for (int w = 0; w < NW; ++w) s_hit[w][j] = 0;
      }
      __syncthreads();
      if (!__all_sync(0xffffffffu, all_done)) {
        const int cnt = build_list(s_mask, nb, 1u << warp, lane, s_list[warp]);
        // Entries go two at a time: the sigma, cut test, exponential and
        // contribution test of both (independent of the pixel state) form one
        // straight-line block whose chains interleave; the blends then apply
        // in list order, the second gated by the pixel state the first left.
        for (int e = 0; e < cnt; e += 2) {
          const bool two = e + 1 < cnt;  // warp-uniform
          const uint32_t jj[2] = {s_list[warp][e], two ? s_list[warp][e + 1] : s_list[warp][e]};
          FwdPre pre[2][NP];
          uint32_t need = 0;
  #pragma unroll
          for (int u = 0; u < 2; ++u) {
            const float4 A = s_a[jj[u]];
            const float4 B = s_b[jj[u]];
            const float dx = esub(A.x, pcx);
            const float t1 = emul(emul(A.z, dx), dx);
            const float t2 = emul(A.w, dx);
  #pragma unroll
            for (int k = 0; k < NP; ++k) {
              FwdPre& q = pre[u][k];
              const float2 dy = add2(f2(A.y), npcy[k]);
              q.sg = sigma2(t1, t2, dy, B.x);
              q.l0 = !(q.sg.x > B.y);
              q.l1 = !(q.sg.y > B.y);
              q.opac = B.z;
              if (__any_sync(0xffffffffu, (q.l0 && !done[2 * k]) || (q.l1 && !done[2 * k + 1])) && (u == 0 || two))
                need |= 1u << (u * NP + k);
            }
          }
          // blend_alpha_of (sigma >= 0 and alpha >= 1/255) and the blend of
          // entry u, pair k. A pixel that does not take the Gaussian blends
          // with alpha 0, which leaves its colour and transmittance bit for bit
          // unchanged.
          auto alpha = [&](FwdPre& q) {
            const float2 og = mul2(f2(q.opac), blend_exp2(q.sg));
            q.ax = fminf(0.999f, og.x);
            q.ay = fminf(0.999f, og.y);
            q.c0 = q.l0 && q.sg.x >= 0.f && q.ax >= (float)(1.0 / 255.0);
            q.c1 = q.l1 && q.sg.y >= 0.f && q.ay >= (float)(1.0 / 255.0);
          };
          auto blend = [&](int u, int k) {
            const FwdPre& q = pre[u][k];
            const bool c0 = q.c0 && !done[2 * k], c1 = q.c1 && !done[2 * k + 1];
            if (!(c0 || c1)) return;
            const uint32_t j = jj[u];
            const float2 am = make_float2(c0 ? q.ax : 0.f, c1 ? q.ay : 0.f);
            const float4 Cc = s_c[j];
            const float2 w = mul2(am, T[k]);
            C0[k] = fma2(f2(Cc.x), w, C0[k]);  // blend_accum; Cc was clamped at staging
            C1[k] = fma2(f2(Cc.y), w, C1[k]);
            C2[k] = fma2(f2(Cc.z), w, C2[k]);
            T[k] = mul2(T[k], add2(f2(1.f), neg2(am)));
            s_hit[warp][j] = 1;
            if (c0) {
              last[2 * k] = b0 + j + 1;
              ++nc[2 * k];
              if (T[k].x < 1e-4f) done[2 * k] = true;
            }
            if (c1) {
              last[2 * k + 1] = b0 + j + 1;
              ++nc[2 * k + 1];
              if (T[k].y < 1e-4f) done[2 * k + 1] = true;
            }
          };
          static_assert(NP == 1, "the forward runs one pixel pair per lane");
          if (need == 3u) {
            alpha(pre[0][0]);
            alpha(pre[1][0]);
            blend(0, 0);
            blend(1, 0);
          } else if (need == 1u) {
            alpha(pre[0][0]);
            blend(0, 0);
          } else if (need == 2u) {
            alpha(pre[1][0]);
            blend(1, 0);
          }
          all_done = true;
  #pragma unroll
          for (int q = 0; q < PPL; ++q) all_done = all_done && done[q];
          if (__all_sync(0xffffffffu, all_done)) break;
        }
      }
      __syncthreads();
      for (uint32_t j = threadIdx.x; j < nb; j += NT) {
        uint32_t bits = 0;
  #pragma unroll
        for (int w = 0; w < NW; ++w) bits |= (uint32_t)s_hit[w][j] << w;
        hitw[b0 + j] = (uint8_t)bits;  // bit w: the 8x8 block of warp w
        if (bits) vis[s_cidx[j]] = 1;
      }
      if (__syncthreads_and(all_done)) break;
    }
    float4* out = reinterpret_cast<float4*>(a.out_rgba) + vd.pix_base;
  #pragma unroll
    for (int q = 0; q < PPL; ++q) {
      const uint32_t py = pyb + 4 * q;
      if (!(px < vd.w && py < vd.h)) continue;
      const size_t pix = (size_t)py * vd.w + px;
      const int k = q / 2;
      const float Tq = (q & 1) ? T[k].y : T[k].x;
      const float c0 = (q & 1) ? C0[k].y : C0[k].x;
      const float c1 = (q & 1) ? C1[k].y : C1[k].x;
      const float c2 = (q & 1) ? C2[k].y : C2[k].x;
      out[pix] = make_float4(c0 + Tq * a.bg[0], c1 + Tq * a.bg[1], c2 + Tq * a.bg[2], 1.f - Tq);
      slice(a.b.tfinal, a.b.Pcap, v)[pix] = Tq;
      slice(a.b.last, a.b.Pcap, v)[pix] = last[q];
      slice(a.b.ncontrib, a.b.Pcap, v)[pix] = nc[q];
      slice(a.b.nvisit, a.b.Pcap, v)[pix] = (done[q] ? last[q] : s1) - s0;
    }
    // The backward's cost of this item: list entries up to the tile's
    // largest last contributor.
    uint32_t ml = 0;
#pragma unroll
    for (int q = 0; q < PPL; ++q) ml = max(ml, last[q]);
    ml = __reduce_max_sync(0xffffffffu, ml);
    if (lane == 0 && ml) atomicMax(&s_work, ml);
    __syncthreads();
    if (threadIdx.x == 0) {
      const uint32_t cost = s_work > s0 ? s_work - s0 : 0u;
      const uint32_t k = cost_bucket(cost);
      a.b.sched_lists[(size_t)k * a.b.sched_items_cap + atomicAdd(a.b.sched_lcount + k, 1u)] = item;
      s_work = 0u;
    }
  }
}

// Reduce-scatter of 12 per-lane values over the warp in 13 shuffles. Lane
// l ends with the warp total of value reduce12_slot(l) (lanes whose bit 1 is
// set and bit 2 differs hold the same value; the fixed summation order makes
// them equal). Stages: xor 16 halves 12 -> 6, xor 8 halves 6 -> 3, xor 4
// splits values 0 and 2 and sums value 1 in both lanes, xor 2 splits the two
// left, xor 1 completes the sum.
__device__ __forceinline__ int reduce12_slot(int lane) {
  const int g16 = (lane >> 4) & 1, g8 = (lane >> 3) & 1, g4 = (lane >> 2) & 1, g2 = (lane >> 1) & 1;
  return (g2 ? 1 : (g4 ? 2 : 0)) + 3 * g8 + 6 * g16;
}
__device__ __forceinline__ float warp_reduce_scatter12(float (&x)[12], int lane) {
  const uint32_t full = 0xffffffffu;
  {
    const bool hi = lane & 16;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      const float send = hi ? x[i] : x[i + 6];
      const float keep = hi ? x[i + 6] : x[i];
      x[i] = keep + __shfl_xor_sync(full, send, 16);
    }
  }
  {
    const bool hi = lane & 8;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const float send = hi ? x[i] : x[i + 3];
      const float keep = hi ? x[i + 3] : x[i];
      x[i] = keep + __shfl_xor_sync(full, send, 8);
    }
  }
  float w0, w1;
  {
    const bool hi = lane & 4;
    const float send = hi ? x[0] : x[2];
    const float keep = hi ? x[2] : x[0];
    w0 = keep + __shfl_xor_sync(full, send, 4);
    w1 = x[1] + __shfl_xor_sync(full, x[1], 4);
  }
  float u;
  {
    const bool hi = lane & 2;
    const float send = hi ? w0 : w1;
    const float keep = hi ? w1 : w0;
    u = keep + __shfl_xor_sync(full, send, 2);
  }
  return u + __shfl_xor_sync(full, u, 1);
}

// Per-pair state of the reverse walk (pixel q = 2k + h is half h of pair k).
struct BwdPair {
  uint32_t last0, last1;
  float2 T;             // transmittance
  float2 SK;            // the background term plus dot(colour accumulated behind the current Gaussian,
                        // upstream colour gradient)
  float2 vr, vg, vb;    // upstream colour gradient
};

__device__ __forceinline__ void load_bwd_pair(const RasterArgs& a, const ViewDesc& vd, uint32_t v, uint32_t px,
                                              uint32_t py0, BwdPair& p) {
  float T[2] = {1.f, 1.f}, K[2] = {0.f, 0.f}, g[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
  uint32_t last[2] = {0u, 0u};
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint32_t py = py0 + 4 * h;
    if (!(px < vd.w && py < vd.h)) continue;
    const size_t pix = (size_t)py * vd.w + px;
    last[h] = slice(a.b.last, a.b.Pcap, v)[pix];
    T[h] = slice(a.b.tfinal, a.b.Pcap, v)[pix];
    const float4 u = reinterpret_cast<const float4*>(a.v_rgba)[vd.pix_base + pix];
    g[h][0] = u.x;
    g[h][1] = u.y;
    g[h][2] = u.z;
    K[h] = (u.x * a.bg[0] + u.y * a.bg[1] + u.z * a.bg[2] - u.w) * T[h];
  }
  p.last0 = last[0];
  p.last1 = last[1];
  p.T = make_float2(T[0], T[1]);
  p.SK = make_float2(K[0], K[1]);
  p.vr = make_float2(g[0][0], g[1][0]);
  p.vg = make_float2(g[0][1], g[1][1]);
  p.vb = make_float2(g[0][2], g[1][2]);
}

__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// A lane's sums over its pixels for the current Gaussian. With dx shared
// by the lane's column and vs the gradient with respect to sigma at each
// pixel, the mean and conic gradient sums factor through three moments,
// M0 = sum vs, M1 = sum vs dy, M2 = sum vs dy^2:
//   sum vs (a dx + b dy) = a S1 + b S2,   sum vs (b dx + c dy) = b S1 + c S2,
//   sum vs dx^2 / 2 = S3 / 2,   sum vs dx dy = S4,   sum vs dy^2 / 2 = S5 / 2,
// with S1 = dx M0, S2 = M1, S3 = dx^2 M0, S4 = dx M1 and S5 = M2 per lane.
// The S sums are what the warp reduces; the conic combination runs once per
// tile, on the CTA's totals. Where the pixel's alpha is not clamped, alpha =
// opacity * G, so the opacity-path gradient sum va * G over those pixels is
// -(sum vs) / opacity: M0 serves for both. The absolute mean-gradient sums
// (densification statistics) stay per pixel.
struct BwdMom {
  float2 m0, m1, m2;
};
struct BwdAcc {
  float2 cr, cg, cb;  // colour gradients
  float2 ax, ay;      // sums of |d/dx| and |d/dy| of the per-pixel mean gradients
  uint32_t n;         // contributing pixels
};

// The first part of a reverse-walk step for both pixels of a pair: the
// offsets and sigma, and whether each pixel can take the Gaussian at all
// (it is before its last contributor and sigma is within the cut).
struct PairPre {
  float2 dy, sg;
  bool l0, l1;
};
__device__ __forceinline__ PairPre bwd_pair_pre(const BwdPair& p, float2 npcy, uint32_t s, float t1, float t2,
                                                const float4& A, const float4& B) {
  PairPre q;
  const bool in0 = s < p.last0, in1 = s < p.last1;
  q.dy = add2(f2(A.y), npcy);
  q.sg = sigma2(t1, t2, q.dy, B.x);
  q.l0 = in0 && !(q.sg.x > B.y);
  q.l1 = in1 && !(q.sg.y > B.y);
  return q;
}

// The rest of the step: the contribution decisions repeat the forward's bit
// for bit; the gradient follows blend_step_grad (rasterize_backwards, exact
// adjoint), with the transmittance recovered with a Newton-refined hardware
// reciprocal. Adds the pair's terms into mom and acc (FIRST_MOM, FIRST_ACC:
// sets them to the terms). Straight-line code: a pixel that does not take
// the Gaussian contributes zeros and keeps its state. With REF (the
// reference semantics) a pixel whose transmittance fell to 1e-4 no longer
// counts as a contributor and gets no gradient.
template <bool REF, bool FIRST_MOM, bool FIRST_ACC>
__device__ __forceinline__ void bwd_pair_rest(BwdPair& p, const PairPre& q, float adx, float bdx, float cb,
                                              const float4& B, const float2 cpv, const float2 vr, const float2 vg,
                                              const float2 vb, BwdMom& mom, BwdAcc& acc) {
  const float2 dy = q.dy;
  const float2 gs = blend_exp2(q.sg);
  const float2 og = mul2(f2(B.z), gs);
  const float ax = fminf(0.999f, og.x), ay = fminf(0.999f, og.y);
  const bool c0 = q.l0 && q.sg.x >= 0.f && ax >= (float)(1.0 / 255.0);
  const bool c1 = q.l1 && q.sg.y >= 0.f && ay >= (float)(1.0 / 255.0);
  const bool sk0 = REF && p.T.x <= 1e-4f, sk1 = REF && p.T.y <= 1e-4f;
  const float2 al = make_float2(ax, ay);
  const float2 am = make_float2(c0 ? ax : 0.f, c1 ? ay : 0.f);
  const float2 om = add2(f2(1.f), neg2(am));
  // Hardware reciprocal refined by one Newton step (r + r(1 - om r)); a
  // pixel that does not take this Gaussian keeps its transmittance exactly.
#ifdef GSR_EXACT_RCP
  float2 ra = make_float2(__frcp_rn(om.x), __frcp_rn(om.y));
#else
  float2 ra = make_float2(rcp_approx(om.x), rcp_approx(om.y));
  ra = fma2(ra, fma2(neg2(om), ra, f2(1.f)), ra);
#endif
  // A pixel that does not take the Gaussian has om = 1 exactly, so ra = 1
  // exactly (the refined reciprocal of 1 is 1) and its state is unchanged.
  const float2 Ti = mul2(p.T, ra);
  const float2 vis = mul2(am, Ti);
  // The colour behind only enters through its dot product with the
  // upstream gradient, which accumulates directly: sum vis_i * dot(c_i, v).
  const float2 va = fma2(Ti, cpv, neg2(mul2(p.SK, ra)));
  p.SK = fma2(vis, cpv, p.SK);
  p.T = Ti;
  const bool gm0 = c0 && !sk0, gm1 = c1 && !sk1;
  const bool gg0 = gm0 && og.x <= 0.999f, gg1 = gm1 && og.y <= 0.999f;
  // vis is zero where the pixel does not take the Gaussian; only the
  // reference semantics drop contributors beyond that.
  const float2 visg = REF ? make_float2(gm0 ? vis.x : 0.f, gm1 ? vis.y : 0.f) : vis;
  const float2 av = mul2(al, va);
  const float2 vs = make_float2(gg0 ? -av.x : 0.f, gg1 ? -av.y : 0.f);
  const float2 vsdy = mul2(vs, dy);
  // |vs (a dx + b dy)| and |vs (b dx + c dy)| per pixel.
  const float2 avs = make_float2(fabsf(vs.x), fabsf(vs.y));
  const float2 g0 = fma2(f2(cb), dy, f2(adx)), g1 = fma2(f2(B.x), dy, f2(bdx));
  const float2 ag0 = make_float2(fabsf(g0.x), fabsf(g0.y)), ag1 = make_float2(fabsf(g1.x), fabsf(g1.y));
  const uint32_t nc = (gm0 ? 1u : 0u) + (gm1 ? 1u : 0u);
  if constexpr (FIRST_MOM) {
    mom.m0 = vs;
    mom.m1 = vsdy;
    mom.m2 = mul2(vsdy, dy);
  } else {
    mom.m0 = add2(mom.m0, vs);
    mom.m1 = add2(mom.m1, vsdy);
    mom.m2 = fma2(vsdy, dy, mom.m2);
  }
  if constexpr (FIRST_ACC) {
    acc.ax = mul2(avs, ag0);
    acc.ay = mul2(avs, ag1);
    acc.cr = mul2(visg, vr);
    acc.cg = mul2(visg, vg);
    acc.cb = mul2(visg, vb);
    acc.n = nc;
  } else {
    acc.ax = fma2(avs, ag0, acc.ax);
    acc.ay = fma2(avs, ag1, acc.ay);
    acc.cr = fma2(visg, vr, acc.cr);
    acc.cg = fma2(visg, vg, acc.cg);
    acc.cb = fma2(visg, vb, acc.cb);
    acc.n += nc;
  }
}

// Maps the forward's per-entry warp-block bits (blocks of kFwdPPL pixels
// per lane) onto the warp blocks of a backward with PB pixels per lane: a
// backward block is the union of the forward blocks of its column span and
// rows.
// The forward warp block (8x8 pixels) that holds pixel pair k of backward
// warp w with PB pixels per lane (its rows 8k .. 8k + 7).
template <int TW, int PB>
__device__ __forceinline__ int fwd_block_of(int w, int k) {
  constexpr int KX = TW / 8;
  return (w % KX) + ((w / KX) * (PB / 2) + k) * KX;
}

template <int TW, int TH, int PB>
__device__ __forceinline__ uint32_t hit_bits_for(uint32_t f) {
  constexpr int PF = kFwdPPL;
  static_assert(PB % PF == 0, "backward warp blocks are unions of forward ones");
  constexpr int NWF = TW * TH / PF / 32;
  constexpr int KX = TW / 8;
  if (PB == PF) return f;
  uint32_t m = 0;
#pragma unroll
  for (int fw = 0; fw < NWF; ++fw) m |= ((f >> fw) & 1u) << ((fw % KX) + ((fw / KX) * PF / PB) * KX);
  return m;
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// The backward walks the tile's list from its largest last-contributor
// index down in batches. Batches are double-buffered: while batch k is
// evaluated, the raw records of batch k + 1 are in flight (asynchronous
// copies into the other buffer) and the list entries of batch k + 2 (hit
// bits and compact indices) are loaded into registers.
template <int TW, int TH, int PPL, int BATCH, bool REF>
__global__ void __launch_bounds__(TW* TH / PPL) raster_bwd_kernel(RasterArgs a) {
  static_assert(PPL % 2 == 0, "pixels per lane come in pairs");
  static_assert(TH % (4 * PPL) == 0 && (TW * TH / PPL) % 32 == 0, "warp blocks tile the tile");
  constexpr int NT = TW * TH / PPL;
  constexpr int NW = NT / 32;
  constexpr int NP = PPL / 2;
  constexpr int kSI = (BATCH + NT - 1) / NT;  // entries a thread stages per batch
  __shared__ float4 s_rec[2][BATCH][3];        // raw records
  __shared__ uint32_t s_cidx[2][BATCH];
  __shared__ uint8_t s_mask[2][BATCH];         // warp blocks that take the entry
  __shared__ uint16_t s_list[NW][BATCH];
  __shared__ float4 s_part[NW][BATCH][3];      // written by the warps whose bit is set
  __shared__ uint32_t s_max;
  __shared__ uint32_t s_item;
  __shared__ CostListView s_lists;
  load_cost_lists(a, &s_lists);
  for (uint32_t round = 0;; ++round) {
    const uint32_t item = next_item(a, round, &s_item, &s_lists);
    if (item == kNoItem) break;
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
    const uint32_t* vals = isect_index_src(a.b, v);
    const uint32_t vmask = isect_index_mask(a.b);
    const float4* rec = slice(a.b.rec, a.b.Vcap * 3, v);
    const uint8_t* hitw = slice(a.b.hitw, a.b.Icap, v);
    float4* sgrad = slice(a.b.sgrad, a.b.Vcap * 3, v);
    float* part = a.b.sgrad_part + (size_t)a.b.Icap * 12 * v;
    BwdPair pp[NP];
    uint32_t mylast = 0;
  #pragma unroll
    for (int k = 0; k < NP; ++k) {
      load_bwd_pair(a, vd, v, px, pyb + 8 * k, pp[k]);
      mylast = max(mylast, max(pp[k].last0, pp[k].last1));
    }
    if (threadIdx.x == 0) s_max = 0;
    __syncthreads();
    const uint32_t wmax = __reduce_max_sync(0xffffffffu, mylast);
    if (lane == 0) atomicMax(&s_max, wmax);
    __syncthreads();
    const uint32_t smax = s_max;
    const int slot = reduce12_slot(lane);                          // the gradient value this lane ends with
    const bool writer = (lane & 1) == 0 && !((lane & 2) && (lane & 4));  // one lane per value
    uint32_t wsel = 0;  // the forward blocks inside this warp's block
  #pragma unroll
    for (int k = 0; k < NP; ++k) wsel |= 1u << fwd_block_of<TW, PPL>(warp, k);
    const uint32_t b0 = fwd_block_of<TW, PPL>(warp, 0);
    auto batch_lo = [&](uint32_t e) { return (e - s0 > (uint32_t)BATCH) ? e - BATCH : s0; };
    // List entries [lo, hi) of a batch into registers.
    uint32_t pc[kSI], ph[kSI];
    auto fetch = [&](uint32_t lo, uint32_t hi) {
  #pragma unroll
      for (int it = 0; it < kSI; ++it) {
        const uint32_t s = lo + threadIdx.x + it * NT;
        const bool ok = threadIdx.x + it * NT < (uint32_t)BATCH && s < hi;
        ph[it] = ok ? hitw[s] : 0u;
        pc[it] = ok ? (vals[s] & vmask) : 0u;
      }
    };
    // Masks, indices and record copies of the fetched batch [lo, hi) into
    // buffer `buf`; one commit group per call.
    auto issue = [&](uint32_t lo, uint32_t hi, int buf) {
  #pragma unroll
      for (int it = 0; it < kSI; ++it) {
        const uint32_t j = threadIdx.x + it * NT;
        if (j < (uint32_t)BATCH && lo + j < hi) {
          s_mask[buf][j] = (uint8_t)ph[it];  // the forward's 8x8 block bits
          if (ph[it]) {
            s_cidx[buf][j] = pc[it];
            const float4* r = rec + (size_t)pc[it] * 3;
            cp_async16(&s_rec[buf][j][0], r);
            cp_async16(&s_rec[buf][j][1], r + 1);
            cp_async16(&s_rec[buf][j][2], r + 2);
          }
        }
      }
      cp_async_commit();
    };
    uint32_t be = smax, bs = be > s0 ? batch_lo(be) : s0;
    if (be > s0) {
      fetch(bs, be);
      issue(bs, be, 0);
    }
    uint32_t nbe = bs, nbs = nbe > s0 ? batch_lo(nbe) : s0;
    if (nbe > s0) fetch(nbs, nbe);
    int buf = 0;
    while (be > s0) {
      const uint32_t nb = be - bs;
      if (nbe > s0)
        issue(nbs, nbe, buf ^ 1);
      else
        cp_async_commit();
      const uint32_t n2e = nbs, n2s = n2e > s0 ? batch_lo(n2e) : s0;
      if (n2e > s0) fetch(n2s, n2e);
      cp_async_wait1();  // this thread's copies of the current batch have landed
      __syncthreads();
      if (bs < wmax) {
        const int cnt = build_list(s_mask[buf], nb, wsel, lane, s_list[warp]);
        for (int e = cnt - 1; e >= 0; --e) {
          const uint32_t j = s_list[warp][e];
          const uint32_t s = bs + j;
          const float4 r0 = s_rec[buf][j][0], r1 = s_rec[buf][j][1], r2 = s_rec[buf][j][2];
          const float4 A = make_float4(r0.x, r0.y, r0.z, 2.f * r0.w);  // 2b is exact
          const float4 B = make_float4(r1.x, r2.y + kRejectMargin, r1.y, 0.f);
          const float4 Cc = make_float4(r1.z, r1.w, r2.x, 0.f);
          const float dx = esub(A.x, pcx);
          const float t1 = emul(emul(A.z, dx), dx);
          const float t2 = emul(A.w, dx);
          const float cb = r0.w;  // the conic's b
          const float adx = A.z * dx, bdx = cb * dx;
          BwdMom mom;  // set by the first pair evaluated
          BwdAcc acc;
          const float cp0 = fmaxf(Cc.x, 0.f), cp1 = fmaxf(Cc.y, 0.f), cp2 = fmaxf(Cc.z, 0.f);
          // The pairs of this warp whose 8x8 block had a pixel take the
          // Gaussian in the forward (the others contribute nothing here).
          const uint32_t mraw = s_mask[buf][j];
          // Pair k takes part when its forward block took the Gaussian (a
          // warp-uniform test); the first pair evaluated sets the sums.
          auto rest = [&](int k, auto first) {
            const float2 npcy = make_float2(-((float)(pyb + 8 * k) + 0.5f), -((float)(pyb + 8 * k + 4) + 0.5f));
            const PairPre pre = bwd_pair_pre(pp[k], npcy, s, t1, t2, A, B);
            const float2 cpv =
                fma2(f2(cp2), pp[k].vb, fma2(f2(cp1), pp[k].vg, mul2(f2(cp0), pp[k].vr)));
            constexpr bool kF = decltype(first)::value;
            bwd_pair_rest<REF, kF, kF>(pp[k], pre, adx, bdx, cb, B, cpv, pp[k].vr, pp[k].vg, pp[k].vb, mom, acc);
          };
          constexpr std::integral_constant<bool, true> kFirst{};
          constexpr std::integral_constant<bool, false> kNext{};
          if constexpr (NP == 1) {
            rest(0, kFirst);  // listed entries take part in the warp's one pair
          } else if constexpr (NP == 2) {
            // Pair k of this warp lies in forward block b0 + k * KX; the
            // needed pairs run as one straight-line block, so that their
            // independent chains interleave.
            constexpr uint32_t KX = TW / 8, both = 1u | (1u << KX);
            const uint32_t need = (mraw >> b0) & both;  // listed entries have at least one
            if (need == both) {
              rest(0, kFirst);
              rest(1, kNext);
            } else if (need == 1u) {
              rest(0, kFirst);
            } else {
              rest(1, kFirst);
            }
          } else {
            mom.m0 = mom.m1 = mom.m2 = acc.cr = acc.cg = acc.cb = acc.ax = acc.ay = f2(0.f);
            acc.n = 0u;
  #pragma unroll
            for (int k = 0; k < NP; ++k)
              if ((mraw >> fwd_block_of<TW, PPL>(warp, k)) & 1u) rest(k, kNext);
          }
          const float M0 = mom.m0.x + mom.m0.y, M1 = mom.m1.x + mom.m1.y, M2 = mom.m2.x + mom.m2.y;
          float x[12];
          x[0] = dx * M0;  // S1..S5 (the conic combination follows the CTA sum)
          x[1] = M1;
          x[2] = dx * x[0];
          x[3] = dx * M1;
          x[4] = M2;
          x[5] = acc.cr.x + acc.cr.y;
          x[6] = acc.cg.x + acc.cg.y;
          x[7] = acc.cb.x + acc.cb.y;
          x[8] = M0;
          x[9] = acc.ax.x + acc.ax.y;
          x[10] = acc.ay.x + acc.ay.y;
          x[11] = (float)acc.n;
          const float r = warp_reduce_scatter12(x, lane);
          float* sp = reinterpret_cast<float*>(&s_part[warp][j][0]);
          if (writer) sp[slot] = r;
        }
      }
      __syncthreads();
      for (uint32_t q = threadIdx.x; q < nb * 3; q += NT) {
        const uint32_t j = q / 3, k = q % 3;
        const uint32_t m = hit_bits_for<TW, TH, PPL>(s_mask[buf][j]);  // warps that wrote a slot
        float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
        bool any = false;
  #pragma unroll
        for (int w = 0; w < NW; ++w) {
          if (!((m >> w) & 1u)) continue;
          const float4 g = s_part[w][j][k];
          if (!any) {
            f = g;
            any = true;
          } else {
            f.x = f.x + g.x;
            f.y = f.y + g.y;
            f.z = f.z + g.z;
            f.w = f.w + g.w;
          }
        }
        if (any) {
          // The tile's S sums and sum vs into the screen-space gradients.
          if (k == 0) {
            const float4 r0 = s_rec[buf][j][0];
            const float cc = s_rec[buf][j][1].x;
            f = make_float4(r0.z * f.x + r0.w * f.y, r0.w * f.x + cc * f.y, 0.5f * f.z, f.w);
          } else if (k == 1) {
            // v_rgb is zero for a channel whose raw colour is negative.
            const float4 r1 = s_rec[buf][j][1];
            const float rb = s_rec[buf][j][2].x;
            f = make_float4(0.5f * f.x, r1.z < 0.f ? 0.f : f.y, r1.w < 0.f ? 0.f : f.z, rb < 0.f ? 0.f : f.w);
          } else {
            f.x = f.x != 0.f ? -f.x / s_rec[buf][j][1].y : 0.f;
          }
        }
        if (a.det) {
          reinterpret_cast<float4*>(part + (size_t)(bs + j) * 12)[k] = f;
        } else if (f.x != 0.f || f.y != 0.f || f.z != 0.f || f.w != 0.f) {
          atomicAdd(sgrad + (size_t)s_cidx[buf][j] * 3 + k, f);
        }
      }
      __syncthreads();  // the next batch's copies reuse this buffer
      be = bs;
      bs = nbs;
      nbe = n2e;
      nbs = n2s;
      buf ^= 1;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");  // no copy may outlive the block
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
}

// The backward of 16x16 tiles with one warp per tile. Lane l owns, in each
// of the tile's four 8x8 blocks q (block column q & 1, block row q >> 1), the
// pixel pair (8 (q & 1) + (l & 7), 8 (q >> 1) + (l >> 3) + {0, 4}), so that
// pair q lies in the forward's warp block q and an entry's block bits say
// which pairs need it. Against two warps per tile, each list entry is staged,
// set up and reduced once per tile rather than once per warp whose block it
// reaches, and the tile's sum needs no second warp. The pairs of a block
// column share dx and the terms that depend on it; the sigma-gradient
// moments are kept per column (S1 = dx0 M0_0 + dx1 M0_1 and so on).
template <int BATCH, bool REF>
__global__ void __launch_bounds__(32, kTileBwdBlocks) raster_bwd_tile_kernel(RasterArgs a) {
  constexpr int NT = 32;
  constexpr int kSI = BATCH / NT;  // entries a lane stages per batch
  static_assert(BATCH % NT == 0, "whole batches per lane");
  __shared__ float4 s_rec[2][BATCH][3];  // raw records
  __shared__ uint32_t s_cidx[2][BATCH];
  __shared__ uint8_t s_mask[2][BATCH];  // forward blocks that take the entry
  __shared__ uint16_t s_list[BATCH];
  __shared__ float4 s_part[BATCH][3];   // the tile's reduced sums of listed entries
  __shared__ float2 s_v[4][3][32];      // upstream colour gradient of each lane's pairs (read only)
  __shared__ uint32_t s_item;
  __shared__ CostListView s_lists;
  load_cost_lists(a, &s_lists);
  const int lane = threadIdx.x;
  const int slot = reduce12_slot(lane);                          // the gradient value this lane ends with
  const bool writer = (lane & 1) == 0 && !((lane & 2) && (lane & 4));  // one lane per value
  for (uint32_t round = 0;; ++round) {
    const uint32_t item = next_item(a, round, &s_item, &s_lists);
    if (item == kNoItem) break;
    const uint32_t v = find_view(a.vs, item);
    const ViewDesc& vd = a.vs.views[v];
    const uint32_t t = item - vd.tile_base;
    const uint32_t tx = t % vd.tiles_x, ty = t / vd.tiles_x;
    const uint32_t px0 = tx * 16 + (lane & 7), py0 = ty * 16 + (lane >> 3);
    const float pcx0 = (float)px0 + 0.5f, pcx1 = (float)(px0 + 8) + 0.5f;
    // Negated pixel-centre rows of the lane's pairs: block row h, half u at
    // row py0 + 8 h + 4 u (small integers plus 0.5: exact).
    const float npy[4] = {-((float)py0 + 0.5f), -((float)(py0 + 4) + 0.5f), -((float)(py0 + 8) + 0.5f),
                          -((float)(py0 + 12) + 0.5f)};
    const uint32_t* ranges = slice(a.b.ranges, 2 * a.b.Tcap, v);
    const uint32_t s0 = ranges[2 * t];
    const uint32_t* vals = isect_index_src(a.b, v);
    const uint32_t vmask = isect_index_mask(a.b);
    const float4* rec = slice(a.b.rec, a.b.Vcap * 3, v);
    const uint8_t* hitw = slice(a.b.hitw, a.b.Icap, v);
    float4* sgrad = slice(a.b.sgrad, a.b.Vcap * 3, v);
    float* part = a.b.sgrad_part + (size_t)a.b.Icap * 12 * v;
    BwdPair pp[4];
    uint32_t mylast = 0;
  #pragma unroll
    for (int q = 0; q < 4; ++q) {
      load_bwd_pair(a, vd, v, px0 + 8 * (q & 1), py0 + 8 * (q >> 1), pp[q]);
      mylast = max(mylast, max(pp[q].last0, pp[q].last1));
      s_v[q][0][lane] = pp[q].vr;  // kept in shared memory, not registers
      s_v[q][1][lane] = pp[q].vg;
      s_v[q][2][lane] = pp[q].vb;
    }
    const uint32_t smax = __reduce_max_sync(0xffffffffu, mylast);
    auto batch_lo = [&](uint32_t e) { return (e - s0 > (uint32_t)BATCH) ? e - BATCH : s0; };
    uint32_t pc[kSI], ph[kSI];
    auto fetch = [&](uint32_t lo, uint32_t hi) {
  #pragma unroll
      for (int it = 0; it < kSI; ++it) {
        const uint32_t s = lo + lane + it * NT;
        const bool ok = s < hi;
        ph[it] = ok ? hitw[s] : 0u;
        pc[it] = ok ? (vals[s] & vmask) : 0u;
      }
    };
    auto issue = [&](uint32_t lo, uint32_t hi, int buf) {
  #pragma unroll
      for (int it = 0; it < kSI; ++it) {
        const uint32_t j = lane + it * NT;
        if (lo + j < hi) {
          s_mask[buf][j] = (uint8_t)ph[it];
          if (ph[it]) {
            s_cidx[buf][j] = pc[it];
            const float4* r = rec + (size_t)pc[it] * 3;
            cp_async16(&s_rec[buf][j][0], r);
            cp_async16(&s_rec[buf][j][1], r + 1);
            cp_async16(&s_rec[buf][j][2], r + 2);
          }
        }
      }
      cp_async_commit();
    };
    uint32_t be = smax, bs = be > s0 ? batch_lo(be) : s0;
    if (be > s0) {
      fetch(bs, be);
      issue(bs, be, 0);
    }
    uint32_t nbe = bs, nbs = nbe > s0 ? batch_lo(nbe) : s0;
    if (nbe > s0) fetch(nbs, nbe);
    int buf = 0;
    while (be > s0) {
      const uint32_t nb = be - bs;
      if (nbe > s0)
        issue(nbs, nbe, buf ^ 1);
      else
        cp_async_commit();
      const uint32_t n2e = nbs, n2s = n2e > s0 ? batch_lo(n2e) : s0;
      if (n2e > s0) fetch(n2s, n2e);
      cp_async_wait1();  // this lane's copies of the current batch have landed
      __syncthreads();   // and every lane's
      const int cnt = build_list(s_mask[buf], nb, 0xfu, lane, s_list);
      for (int e = cnt - 1; e >= 0; --e) {
        const uint32_t j = s_list[e];
        const uint32_t s = bs + j;
        const float4 r0 = s_rec[buf][j][0], r1 = s_rec[buf][j][1], r2 = s_rec[buf][j][2];
        const float4 A = make_float4(r0.x, r0.y, r0.z, 2.f * r0.w);  // 2b is exact
        const float4 B = make_float4(r1.x, r2.y + kRejectMargin, r1.y, 0.f);
        const float cb = r0.w;  // the conic's b
        const float cp0 = fmaxf(r1.z, 0.f), cp1 = fmaxf(r1.w, 0.f), cp2 = fmaxf(r2.x, 0.f);
        const uint32_t need = s_mask[buf][j];  // bit q: pair q takes part
        const float dx0 = esub(A.x, pcx0), dx1 = esub(A.x, pcx1);
        BwdMom mom0, mom1;
        BwdAcc acc;
        constexpr std::integral_constant<bool, true> kT{};
        constexpr std::integral_constant<bool, false> kF{};
        // The pairs of block column c (q = c upper, q = c + 2 lower) as one
        // straight-line block; FM: the column's first pair sets its moments,
        // FA: the entry's first pair sets the shared sums.
        auto column = [&](auto cc, auto fa, BwdMom& mom) {
          constexpr int c = decltype(cc)::value;
          constexpr bool FA = decltype(fa)::value;
          const float dx = c ? dx1 : dx0;
          const float t1 = emul(emul(A.z, dx), dx);
          const float t2 = emul(A.w, dx);
          const float adx = A.z * dx, bdx = cb * dx;
          auto rest = [&](auto qq, auto fm, auto fa2) {
            constexpr int q = decltype(qq)::value;
            const float2 npcy = make_float2(npy[2 * (q >> 1)], npy[2 * (q >> 1) + 1]);
            const PairPre pre = bwd_pair_pre(pp[q], npcy, s, t1, t2, A, B);
            const float2 vr = s_v[q][0][lane], vg = s_v[q][1][lane], vb = s_v[q][2][lane];
            const float2 cpv = fma2(f2(cp2), vb, fma2(f2(cp1), vg, mul2(f2(cp0), vr)));
            bwd_pair_rest<REF, decltype(fm)::value, decltype(fa2)::value>(pp[q], pre, adx, bdx, cb, B, cpv, vr, vg,
                                                                          vb, mom, acc);
          };
          const uint32_t nc = (need >> c) & 5u;  // bit 0: upper pair, bit 2: lower pair
          if (nc == 5u) {
            rest(std::integral_constant<int, c>{}, kT, std::integral_constant<bool, FA>{});
            rest(std::integral_constant<int, c + 2>{}, kF, kF);
          } else if (nc == 1u) {
            rest(std::integral_constant<int, c>{}, kT, std::integral_constant<bool, FA>{});
          } else {
            rest(std::integral_constant<int, c + 2>{}, kT, std::integral_constant<bool, FA>{});
          }
        };
        if (need & 5u) {
          column(std::integral_constant<int, 0>{}, kT, mom0);
        } else {
          mom0.m0 = mom0.m1 = mom0.m2 = acc.cr = acc.cg = acc.cb = acc.ax = acc.ay = f2(0.f);
          acc.n = 0u;
        }
        if (need & 10u)
          column(std::integral_constant<int, 1>{}, kF, mom1);
        else
          mom1.m0 = mom1.m1 = mom1.m2 = f2(0.f);
        const float M00 = mom0.m0.x + mom0.m0.y, M01 = mom1.m0.x + mom1.m0.y;
        const float M10 = mom0.m1.x + mom0.m1.y, M11 = mom1.m1.x + mom1.m1.y;
        const float e0 = dx0 * M00, e1 = dx1 * M01;
        float x[12];
        x[0] = e0 + e1;  // S1..S5 (the conic combination follows the reduction)
        x[1] = M10 + M11;
        x[2] = dx0 * e0 + dx1 * e1;
        x[3] = dx0 * M10 + dx1 * M11;
        x[4] = (mom0.m2.x + mom0.m2.y) + (mom1.m2.x + mom1.m2.y);
        x[5] = acc.cr.x + acc.cr.y;
        x[6] = acc.cg.x + acc.cg.y;
        x[7] = acc.cb.x + acc.cb.y;
        x[8] = M00 + M01;
        x[9] = acc.ax.x + acc.ax.y;
        x[10] = acc.ay.x + acc.ay.y;
        x[11] = (float)acc.n;
        const float r = warp_reduce_scatter12(x, lane);
        if (writer) reinterpret_cast<float*>(&s_part[j][0])[slot] = r;
      }
      __syncwarp();
      for (uint32_t qi = lane; qi < nb * 3; qi += NT) {
        const uint32_t j = qi / 3, k = qi % 3;
        float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
        if (s_mask[buf][j]) {
          f = s_part[j][k];
          if (k == 0) {
            const float4 r0 = s_rec[buf][j][0];
            const float cc = s_rec[buf][j][1].x;
            f = make_float4(r0.z * f.x + r0.w * f.y, r0.w * f.x + cc * f.y, 0.5f * f.z, f.w);
          } else if (k == 1) {
            // v_rgb is zero for a channel whose raw colour is negative.
            const float4 r1 = s_rec[buf][j][1];
            const float rb = s_rec[buf][j][2].x;
            f = make_float4(0.5f * f.x, r1.z < 0.f ? 0.f : f.y, r1.w < 0.f ? 0.f : f.z, rb < 0.f ? 0.f : f.w);
          } else {
            f.x = f.x != 0.f ? -f.x / s_rec[buf][j][1].y : 0.f;
          }
        }
        if (a.det) {
          reinterpret_cast<float4*>(part + (size_t)(bs + j) * 12)[k] = f;
        } else if (f.x != 0.f || f.y != 0.f || f.z != 0.f || f.w != 0.f) {
          atomicAdd(sgrad + (size_t)s_cidx[buf][j] * 3 + k, f);
        }
      }
      __syncthreads();  // the next batch's copies reuse this buffer
      be = bs;
      bs = nbs;
      nbe = n2e;
      nbs = n2s;
      buf ^= 1;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");  // no copy may outlive the block
    if (a.det) {
      const uint32_t s1 = ranges[2 * t + 1];
      for (uint32_t s = smax > s0 ? smax : s0; s + lane < s1; s += NT) {
        float4* p4 = reinterpret_cast<float4*>(part + (size_t)(s + lane) * 12);
        p4[0] = p4[1] = p4[2] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
  }
}

// Gaussians per shared-memory batch: 0 selects the tuned defaults (128 in
// the forward, 64 in the backward); other values round up to 64, 128 or 256.
// The backward of shapes with two or more warps per tile caps at 128 (its
// double-buffered records and per-warp partial sums would not fit the 48 KB
// of static shared memory).
inline int pick_batch(uint32_t want, int dflt) {
  if (want == 0) return dflt;
  return want <= 64 ? 64 : (want <= 128 ? 128 : 256);
}

// Launches kernel over the launch's work items: one CTA per item (grid
// schedule), or as many CTAs as the SMs hold at once (persistent schedule;
// the residency of each instantiation is looked up once).
// Resident CTAs per SM of a raster kernel instantiation, looked up once
// (context creation warms it up, so that a first launch inside a stream
// capture needs no lookup).
template <void (*Kernel)(RasterArgs)> int resident_per_sm(int threads) {
  static int per_sm = 0;  // one per kernel instantiation
  if (per_sm <= 0) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, Kernel, threads, 0) != cudaSuccess || n < 1) {
      (void)cudaGetLastError();
      n = 1;
    }
    per_sm = n;
  }
  return per_sm;
}

template <void (*Kernel)(RasterArgs)>
cudaError_t launch_items(int threads, const RasterArgs& a, int num_sms, cudaStream_t st) {
  uint32_t grid = a.vs.total_tiles;
  if (a.persist)
    grid = std::min<uint32_t>(grid, (uint32_t)resident_per_sm<Kernel>(threads) * (uint32_t)std::max(num_sms, 1));
  if (grid == 0) return cudaSuccess;  // a warm-up call (no items)
  Kernel<<<grid, threads, 0, st>>>(a);
  return cudaGetLastError();
}

template <int TW, int TH, int PPL>
cudaError_t launch_fwd_shape(const RasterArgs& a, uint32_t batch, int num_sms, cudaStream_t st) {
  constexpr int NT = TW * TH / PPL;
  switch (pick_batch(batch, 128)) {
    case 64: return launch_items<raster_fwd_kernel<TW, TH, PPL, 64>>(NT, a, num_sms, st);
    case 128: return launch_items<raster_fwd_kernel<TW, TH, PPL, 128>>(NT, a, num_sms, st);
    default: return launch_items<raster_fwd_kernel<TW, TH, PPL, 256>>(NT, a, num_sms, st);
  }
}
template <int TW, int TH, int PPL, bool REF>
cudaError_t launch_bwd_mode(const RasterArgs& a, uint32_t batch, int num_sms, cudaStream_t st) {
  constexpr int NT = TW * TH / PPL;
  constexpr int kMaxBatch = NT / 32 >= 2 ? 128 : 256;
  int b = pick_batch(batch, 64);
  if (b > kMaxBatch) b = kMaxBatch;
  switch (b) {
    case 64: return launch_items<raster_bwd_kernel<TW, TH, PPL, 64, REF>>(NT, a, num_sms, st);
    case 128: return launch_items<raster_bwd_kernel<TW, TH, PPL, 128, REF>>(NT, a, num_sms, st);
    default:
      return launch_items<raster_bwd_kernel<TW, TH, PPL, (kMaxBatch > 128 ? 256 : 128), REF>>(NT, a, num_sms, st);
  }
}
// The 16x16 backward stages 64 entries per batch whatever the forward's
// batch: 13 KB of shared memory and at most 128 registers per one-warp CTA
// let 16 CTAs share an SM (a 128-entry batch would fit 9).
template <bool REF>
cudaError_t launch_bwd_tile16(const RasterArgs& a, int num_sms, cudaStream_t st) {
  return launch_items<raster_bwd_tile_kernel<kTileBwdBatch, REF>>(32, a, num_sms, st);
}
template <int TW, int TH, int PPL>
cudaError_t launch_bwd_shape(const RasterArgs& a, uint32_t batch, int num_sms, cudaStream_t st) {
  return a.ref_mode ? launch_bwd_mode<TW, TH, PPL, true>(a, batch, num_sms, st)
                    : launch_bwd_mode<TW, TH, PPL, false>(a, batch, num_sms, st);
}
// 16x16 tiles: one warp per tile on large launches, two otherwise.
cudaError_t launch_bwd_16(const RasterArgs& a, uint32_t batch, int num_sms, cudaStream_t st) {
  const uint32_t wave =
      (uint32_t)resident_per_sm<raster_bwd_tile_kernel<kTileBwdBatch, false>>(32) * (uint32_t)std::max(num_sms, 1);
  if (a.vs.total_tiles >= kTileKernelWaves * wave || a.vs.total_tiles == 0)
    return a.ref_mode ? launch_bwd_tile16<true>(a, num_sms, st) : launch_bwd_tile16<false>(a, num_sms, st);
  return launch_bwd_shape<16, 16, kBwdPPL16>(a, batch, num_sms, st);
}

}  // namespace

void raster_warm_up(uint32_t tile_w, uint32_t tile_h, uint32_t batch, int num_sms) {
  RasterArgs a{};
  a.persist = 1;  // total_tiles 0: the launchers only look up the residency
  a.vs.batch = batch;
  for (int ref = 0; ref < 2; ++ref) {
    a.ref_mode = ref;
    if (tile_w == 16 && tile_h == 16) {
      (void)launch_fwd_shape<16, 16, kFwdPPL>(a, batch, num_sms, nullptr);
      (void)launch_bwd_16(a, batch, num_sms, nullptr);
      (void)launch_bwd_shape<16, 16, kBwdPPL16>(a, batch, num_sms, nullptr);
    } else if (tile_w == 8 && tile_h == 8) {
      (void)launch_fwd_shape<8, 8, kFwdPPL>(a, batch, num_sms, nullptr);
      (void)launch_bwd_shape<8, 8, kBwdPPL>(a, batch, num_sms, nullptr);
    } else if (tile_w == 32 && tile_h == 8) {
      (void)launch_fwd_shape<32, 8, kFwdPPL>(a, batch, num_sms, nullptr);
      (void)launch_bwd_shape<32, 8, kBwdPPL>(a, batch, num_sms, nullptr);
    }
  }
}

cudaError_t launch_raster_fwd(const ViewSet& vs, FwdBufs& b, const float* bg, float* out_rgba, const Scratch& s,
                              cudaStream_t st) {
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
  // The forward appends every item to the cost list of its backward cost.
  e = cudaMemsetAsync(b.sched_lcount, 0, sizeof(uint32_t) * kCostLists, st);
  if (e != cudaSuccess) return e;
  a.persist = (vs.persistent & kPersistFwd) != 0 ? 1 : 0;
  if (a.persist) {
    sched_order_kernel<<<1, kOrderThreads, 0, st>>>(vs, b);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (vs.tile_w == 16 && vs.tile_h == 16) return launch_fwd_shape<16, 16, kFwdPPL>(a, vs.batch, s.num_sms, st);
  if (vs.tile_w == 8 && vs.tile_h == 8) return launch_fwd_shape<8, 8, kFwdPPL>(a, vs.batch, s.num_sms, st);
  if (vs.tile_w == 32 && vs.tile_h == 8) return launch_fwd_shape<32, 8, kFwdPPL>(a, vs.batch, s.num_sms, st);
  return cudaErrorInvalidValue;
}

cudaError_t launch_raster_bwd(const ViewSet& vs, FwdBufs& b, const float* bg, const float* v_rgba, int ref_mode,
                              int deterministic, const Scratch& s, cudaStream_t st) {
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
  a.persist = (vs.persistent & kPersistBwd) != 0 ? 2 : 0;
  if (a.persist) {
    cudaError_t e = cudaMemsetAsync(b.sched_ticket, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
  }
  if (vs.tile_w == 16 && vs.tile_h == 16) return launch_bwd_16(a, vs.batch, s.num_sms, st);
  if (vs.tile_w == 8 && vs.tile_h == 8) return launch_bwd_shape<8, 8, kBwdPPL>(a, vs.batch, s.num_sms, st);
  if (vs.tile_w == 32 && vs.tile_h == 8) return launch_bwd_shape<32, 8, kBwdPPL>(a, vs.batch, s.num_sms, st);
  return cudaErrorInvalidValue;
}

}  // namespace gsr
