// k_sort.cu — segmented LSD radix sort of (u32 key, u32 value) pairs and
// decoupled-look-back scans.
//
// The reference sorts with a bitonic network (radix_sort.wgsl, 2 +
// log2(P)(log2(P)+1)/2 launches of P = next_pow2(n) threads) and scans with
// Hillis-Steele steps (prefix_sum.wgsl, 1 + log2(n) launches). Here:
//  - one histogram pass over the keys computes the digit counts of every
//    radix pass at once;
//  - each radix pass is one persistent launch: blocks take 4096-key
//    partitions by ticket, rank keys stably inside the block (peer lanes
//    of a digit by match_any, or by one ballot per digit bit where the
//    digits are near-random; warps in order), publish per-digit counts and look
//    back across partitions for their global offsets, then scatter through
//    shared memory so that every digit's run is written contiguously;
//  - scans are single-pass with the same look-back.
// Keys are u32; `bits` (from bit shift0) set the passes: ceil(bits / 8)
// passes of equal digits of at most 8 bits (12 bits: two 6-bit passes, whose
// 64 digit runs per partition are written in longer stretches than 256). Stability (ties in input order) is what the reference's index
// tie-break provides (radix_sort.wgsl:21-26). Without values, the keys are
// sorted alone (the binning packs tile id and compact index into one key
// when both fit in 32 bits).
#include <algorithm>

#include "gsr_kernels.h"

namespace gsr {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kWarpKeys = kSortItems * 32;  // 512 keys per warp

__device__ __forceinline__ uint32_t seg_count(const uint32_t* counts, uint32_t stride, uint32_t seg, uint32_t n_host,
                                              uint64_t cap) {
  if (!counts) return n_host;
  const uint64_t c = counts[(size_t)seg * stride];
  return (uint32_t)(c < cap ? c : cap);
}

__global__ void __launch_bounds__(256) sort_hist_kernel(const uint32_t* keys, uint64_t seg_stride,
                                                        const uint32_t* counts, uint32_t count_stride,
                                                        uint32_t n_host, uint64_t cap, int passes, uint32_t shift0,
                                                        uint32_t dbits, uint32_t* hist) {
  __shared__ uint32_t h[4][256];
  for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x) (&h[0][0])[i] = 0;
  __syncthreads();
  const uint32_t seg = blockIdx.y;
  const uint32_t n = seg_count(counts, count_stride, seg, n_host, cap);
  const uint32_t* k = keys + (size_t)seg * seg_stride;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t key = k[i];
    for (int p = 0; p < passes; ++p) atomicAdd(&h[p][(key >> (shift0 + dbits * p)) & ((1u << dbits) - 1u)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * 256; i += blockDim.x) {
    const uint32_t c = (&h[0][0])[i];
    if (c) atomicAdd(hist + (size_t)seg * 1024 + i, c);
  }
}

__global__ void __launch_bounds__(256) sort_hist_scan_kernel(const uint32_t* hist, uint32_t* base) {
  __shared__ uint32_t s_scan[32];
  const uint32_t p = blockIdx.x, seg = blockIdx.y;
  const size_t o = (size_t)seg * 1024 + p * 256 + threadIdx.x;
  uint32_t tot;
  base[o] = block_exclusive_scan(hist[o], s_scan, &tot);
}

struct SortPassArgs {
  const uint32_t* keys_in;
  const uint32_t* vals_in;  // null: values are the input positions
  uint32_t* keys_out;
  uint32_t* vals_out;
  uint64_t seg_stride;
  const uint32_t* counts;
  uint32_t count_stride;
  uint32_t n_host;
  uint64_t cap;
  uint32_t shift;
  uint32_t dmask;  // digit mask: (1 << digit bits) - 1, at most 255
  uint32_t pass;
  const uint32_t* base;  // [seg][4][256]
  uint32_t drop;         // 1: keys equal to 0xffffffff take digit dmask + 1 and are not written (dmask < 255)
  unsigned long long* states;
  uint32_t parts_cap;
  LookbackCtl* ctl;
  DevStatus* status;
};

// KV: values travel with the keys; otherwise the keys are sorted alone.
template <bool KV>
__global__ void __launch_bounds__(kSortThreads, KV ? 2 : 4) sort_pass_kernel(SortPassArgs a) {
  __shared__ uint32_t s_keys[kSortTile];
  __shared__ uint32_t s_vals[KV ? kSortTile : 1];
  __shared__ uint32_t s_whist[kSortWarps][256];
  __shared__ uint32_t s_dstart[256];
  __shared__ uint32_t s_gbase[256];
  __shared__ uint32_t s_scan[32];
  __shared__ uint32_t s_ticket;
  __shared__ uint32_t s_dropped;
  const uint32_t epoch = epoch_begin(a.ctl);
  const unsigned long long tag = (unsigned long long)(epoch & 0x3fffffffu) << 34;
  const int dbits = __popc(a.dmask);
  const int rbits = dbits + (a.drop ? 1 : 0);  // digit bits ranked (the dropped keys' digit is dmask + 1)
  const uint32_t kDropDigit = a.dmask + 1u;
  const uint32_t seg = blockIdx.y;
  const uint32_t n = seg_count(a.counts, a.count_stride, seg, a.n_host, a.cap);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt_mask = (1u << lane) - 1u;
  const uint32_t* kin = a.keys_in + (size_t)seg * a.seg_stride;
  const uint32_t* vin = a.vals_in ? a.vals_in + (size_t)seg * a.seg_stride : nullptr;
  uint32_t* kout = a.keys_out + (size_t)seg * a.seg_stride;
  uint32_t* vout = a.vals_out + (size_t)seg * a.seg_stride;
  unsigned long long* states = a.states + (size_t)seg * a.parts_cap * 256;
  const uint32_t* gbase = a.base + (size_t)seg * 1024 + a.pass * 256;
  for (;;) {
    const uint32_t part = next_ticket(a.ctl, seg, &s_ticket);
    if ((uint64_t)part * kSortTile >= n) break;
    const uint32_t tile0 = part * kSortTile;
    uint32_t key[kSortItems], val[kSortItems], lrank[kSortItems];
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
      const uint32_t idx = tile0 + warp * kWarpKeys + i * 32 + lane;
      const bool ok = idx < n;
      key[i] = ok ? kin[idx] : 0xffffffffu;
      val[i] = (KV && ok) ? (vin ? vin[idx] : idx) : 0u;
    }
    for (int j = lane; j < 256; j += 32) s_whist[warp][j] = 0;
    __syncwarp();
    // Stable rank within the warp: rounds in order, lanes in order.
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
      const uint32_t idx = tile0 + warp * kWarpKeys + i * 32 + lane;
      const bool ok = idx < n;
      uint32_t d, peers;
      if (KV) {
        // Near-random digits (depth keys): one ballot per digit bit.
        d = (a.drop && key[i] == 0xffffffffu) ? kDropDigit : (key[i] >> a.shift) & a.dmask;
        const uint32_t okm = __ballot_sync(0xffffffffu, ok);  // every lane, also past the end
        peers = ok ? okm : (1u << lane);
#pragma unroll
        for (int bit = 0; bit < 8; ++bit) {
          if (bit < rbits) {
            const bool set = (d >> bit) & 1u;
            const uint32_t bb = __ballot_sync(0xffffffffu, set);
            peers &= set ? bb : ~bb;
          }
        }
      } else {
        // Clustered digits (tile ids of neighbouring boxes): few distinct
        // values per warp, where match_any is cheaper.
        d = ok ? ((a.drop && key[i] == 0xffffffffu) ? kDropDigit : ((key[i] >> a.shift) & a.dmask)) : (256u + lane);
        peers = __match_any_sync(0xffffffffu, d);
      }
      const uint32_t below = peers & lt_mask;
      uint32_t b = 0;
      if (ok) b = s_whist[warp][d];
      __syncwarp();
      if (ok && below == 0) s_whist[warp][d] = b + __popc(peers);
      __syncwarp();
      lrank[i] = b + __popc(below);
    }
    __syncthreads();
    // Per digit (one per thread): warp offsets and the block count.
    const uint32_t d = threadIdx.x;
    uint32_t sum = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
      const uint32_t t = s_whist[w][d];
      s_whist[w][d] = sum;
      sum += t;
    }
    // The digit counts are published before the block scan, so that later
    // partitions can sum past this one as early as possible; only the
    // pass's digits look back.
    if (d <= a.dmask) st_volatile64(states + (size_t)part * 256 + d, tag | (part == 0 ? kFlagPre : kFlagAgg) | sum);
    uint32_t tot;
    const uint32_t dstart = block_exclusive_scan(sum, s_scan, &tot);
    const uint32_t excl = d <= a.dmask ? lookback(states + d, 256, part, sum, epoch, a.status, kWaitSort) : 0u;
    s_dstart[d] = dstart;
    s_gbase[d] = gbase[d] + excl - dstart;
    // The dropped keys are placed last in the block and never written (one
    // thread sets the count: the drop digit's, or thread 0 when nothing drops).
    if (d == (a.drop ? kDropDigit : 0u)) s_dropped = a.drop ? sum : 0u;
    // This partition writes digit d's keys to gbase[d] + excl onwards; a
    // position past the segment would mean the digit histogram did not
    // describe these keys. Such a partition writes nothing and is reported
    // through the status words.
    const bool outside = d <= a.dmask && sum != 0u && s_gbase[d] + dstart + sum > n;  // each term is below 2^30
    if (__syncthreads_or(outside)) {
      if (threadIdx.x == 0) atomicOr(&a.status->internal, 1u);
      continue;
    }
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
      const uint32_t idx = tile0 + warp * kWarpKeys + i * 32 + lane;
      if (idx < n) {
        const uint32_t dd = (a.drop && key[i] == 0xffffffffu) ? kDropDigit : (key[i] >> a.shift) & a.dmask;
        const uint32_t pos = s_dstart[dd] + s_whist[warp][dd] + lrank[i];
        s_keys[pos] = key[i];
        if (KV) s_vals[pos] = val[i];
      }
    }
    __syncthreads();
    const uint32_t nvalid = min((uint32_t)kSortTile, n - tile0) - s_dropped;
    for (uint32_t j = threadIdx.x; j < nvalid; j += kSortThreads) {
      const uint32_t k = s_keys[j];
      const uint32_t dst = s_gbase[(k >> a.shift) & a.dmask] + j;
      kout[dst] = k;
      if (KV) vout[dst] = s_vals[j];
    }
  }
  epoch_end(a.ctl, epoch);
}

// ---------------------------------------------------------------------------
// Decoupled look-back scan: 2048 elements per partition, thread-striped
// rounds. in[gather[i]] when gather is set. Exclusive or inclusive output.
// Per segment totals: totals[seg * tstride + 0] = min(total, cap_total),
// totals[seg * tstride + 1] = total; overflow is flagged when total exceeds
// cap_total.
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

struct ScanArgs {
  const uint32_t* in;
  const uint32_t* gather;
  uint32_t* out;
  uint64_t seg_stride;
  const uint32_t* counts;
  uint32_t count_stride;
  uint32_t n_host;
  uint64_t cap;
  int inclusive;
  uint32_t* totals;
  uint32_t totals_stride;
  uint64_t cap_total;
  unsigned long long* states;
  uint32_t parts_cap;
  LookbackCtl* ctl;
  DevStatus* status;
  uint32_t seg_base;  // segment of blockIdx.y == 0
};

__global__ void __launch_bounds__(kScanThreads) scan_kernel(ScanArgs a) {
  __shared__ uint32_t s_scan[32];
  __shared__ uint32_t s_ticket, s_excl;
  const uint32_t epoch = epoch_begin(a.ctl);
  const uint32_t seg = a.seg_base + blockIdx.y;
  const uint32_t n = seg_count(a.counts, a.count_stride, seg, a.n_host, a.cap);
  const uint32_t* in = a.in + (size_t)seg * a.seg_stride;
  const uint32_t* ga = a.gather ? a.gather + (size_t)seg * a.seg_stride : nullptr;
  uint32_t* out = a.out + (size_t)seg * a.seg_stride;
  unsigned long long* states = a.states + (size_t)seg * a.parts_cap;
  const uint32_t nparts = (n + kScanTile - 1) / kScanTile;
  if (n == 0 && a.totals && blockIdx.x == 0 && threadIdx.x == 0) {
    a.totals[(size_t)seg * a.totals_stride + 0] = 0;
    a.totals[(size_t)seg * a.totals_stride + 1] = 0;
  }
  for (;;) {
    const uint32_t part = next_ticket(a.ctl, seg, &s_ticket);
    if (part >= nparts) break;
    const uint32_t tile0 = part * kScanTile;
    uint32_t v[kScanItems];
    uint32_t local = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
      const uint32_t idx = tile0 + i * kScanThreads + threadIdx.x;
      v[i] = (idx < n) ? (ga ? in[ga[idx]] : in[idx]) : 0u;
    }
    // Rounds in order; within a round threads in order.
    uint32_t round_base[kScanItems];
    uint32_t carry = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
      uint32_t tot;
      const uint32_t e = block_exclusive_scan(v[i], s_scan, &tot);
      round_base[i] = carry + e;
      carry += tot;
    }
    local = carry;
    if (threadIdx.x == 0) s_excl = lookback(states, 1, part, local, epoch, a.status, kWaitScan);
    __syncthreads();
    const uint32_t excl = s_excl;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
      const uint32_t idx = tile0 + i * kScanThreads + threadIdx.x;
      if (idx < n) out[idx] = excl + round_base[i] + (a.inclusive ? v[i] : 0u);
    }
    if (part == nparts - 1 && threadIdx.x == 0 && a.totals) {
      const uint64_t total = (uint64_t)excl + local;
      a.totals[(size_t)seg * a.totals_stride + 0] = (uint32_t)(total < a.cap_total ? total : a.cap_total);
      a.totals[(size_t)seg * a.totals_stride + 1] = (uint32_t)total;
      if (total > a.cap_total) {
        atomicExch(&a.status->overflow, 1u);
        atomicMax(&a.status->required, (unsigned long long)total);
      }
    }
  }
  epoch_end(a.ctl, epoch);
}

int persistent_blocks(int num_sms, uint32_t segments, int per_sm) {
  const int total = num_sms * per_sm;
  const int per = total / (int)(segments ? segments : 1);
  return per < 1 ? 1 : per;
}

}  // namespace

cudaError_t radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out, uint32_t* vals_out,
                             uint32_t* keys_tmp, uint32_t* vals_tmp, uint64_t seg_stride, uint32_t segments,
                             const uint32_t* counts, uint32_t count_stride, uint32_t n_host, uint64_t cap_per_segment,
                             int bits, const Scratch& s, cudaStream_t st, bool hist_ready, uint32_t shift0,
                             const uint32_t* counts_dropped, int first_bits) {
  if (segments == 0 || segments > (uint32_t)kMaxSegments) return cudaErrorInvalidValue;
  if (shift0 >= 32 || (keys_in == nullptr)) return cudaErrorInvalidValue;
  const bool kv = vals_out != nullptr;
  const int passes = sort_passes(bits);
  // Digit widths: uniform, or (with histograms from the caller and two
  // passes) first_bits for the first pass and the rest for the second.
  const bool split = first_bits > 0 && hist_ready && passes == 2 && first_bits < bits && bits - first_bits <= 8;
  const int dbits = split ? first_bits : sort_digit_bits(bits);
  auto pass_bits = [&](int p) { return split ? (p == 0 ? first_bits : bits - first_bits) : dbits; };
  // Dropping the all-ones keys in the first pass needs a spare digit value.
  const bool drop = counts_dropped != nullptr;
  if (drop && (dbits >= 8 || !hist_ready)) return cudaErrorInvalidValue;
  const uint32_t parts_cap = (uint32_t)((cap_per_segment + kSortTile - 1) / kSortTile);
  if ((uint64_t)parts_cap * 256 * segments > s.lb_states_words) return cudaErrorInvalidValue;
  if (!hist_ready) {
    cudaError_t e = cudaMemsetAsync(s.hist, 0, sizeof(uint32_t) * 1024 * segments, st);
    if (e != cudaSuccess) return e;
    dim3 grid(persistent_blocks(s.num_sms, segments, 4), segments);
    sort_hist_kernel<<<grid, 256, 0, st>>>(keys_in, seg_stride, counts, count_stride, n_host, cap_per_segment, passes,
                                           shift0, (uint32_t)dbits, s.hist);
  }
  sort_hist_scan_kernel<<<dim3(passes, segments), 256, 0, st>>>(s.hist, s.hist_base);
  // Ping-pong so that the last pass writes keys_out/vals_out.
  const uint32_t* ki = keys_in;
  const uint32_t* vi = vals_in;
  for (int p = 0; p < passes; ++p) {
    const bool to_out = ((passes - 1 - p) % 2) == 0;
    uint32_t* ko = to_out ? keys_out : keys_tmp;
    uint32_t* vo = to_out ? vals_out : vals_tmp;
    SortPassArgs a;
    a.keys_in = ki;
    a.vals_in = vi;
    a.keys_out = ko;
    a.vals_out = vo;
    a.seg_stride = seg_stride;
    a.counts = (drop && p > 0) ? counts_dropped : counts;
    a.count_stride = count_stride;
    a.drop = (drop && p == 0) ? 1u : 0u;
    a.n_host = n_host;
    a.cap = cap_per_segment;
    a.shift = shift0 + dbits * p;  // a split's second pass starts after the first's bits
    a.dmask = (1u << pass_bits(p)) - 1u;
    a.pass = p;
    a.base = s.hist_base;
    a.states = s.lb_states;
    a.parts_cap = parts_cap;
    a.ctl = s.ctl;
    a.status = s.status;
    dim3 grid(persistent_blocks(s.num_sms, segments, kv ? 3 : 4), segments);
    if (kv)
      sort_pass_kernel<true><<<grid, kSortThreads, 0, st>>>(a);
    else
      sort_pass_kernel<false><<<grid, kSortThreads, 0, st>>>(a);
    ki = ko;
    vi = vo;
  }
  return cudaGetLastError();
}

cudaError_t inclusive_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n_host, const Scratch& s,
                               cudaStream_t st) {
  if (n_host == 0) return cudaSuccess;
  ScanArgs a{};
  a.in = in;
  a.gather = nullptr;
  a.out = out;
  a.seg_stride = 0;
  a.counts = nullptr;
  a.n_host = n_host;
  a.cap = n_host;
  a.inclusive = 1;
  a.totals = nullptr;
  a.parts_cap = (n_host + kScanTile - 1) / kScanTile;
  if (a.parts_cap > s.lb_states_words) return cudaErrorInvalidValue;
  a.states = s.lb_states;
  a.ctl = s.ctl;
  a.status = s.status;
  scan_kernel<<<dim3(persistent_blocks(s.num_sms, 1, 4), 1), kScanThreads, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t inclusive_scan_u32_scratch(const uint32_t* in, uint32_t* out, uint32_t n_host, unsigned long long* states,
                                       uint64_t states_words, LookbackCtl* ctl, DevStatus* status, int num_sms,
                                       cudaStream_t st) {
  if (n_host == 0) return cudaSuccess;
  ScanArgs a{};
  a.in = in;
  a.gather = nullptr;
  a.out = out;
  a.seg_stride = 0;
  a.counts = nullptr;
  a.n_host = n_host;
  a.cap = n_host;
  a.inclusive = 1;
  a.totals = nullptr;
  a.parts_cap = (n_host + kScanTile - 1) / kScanTile;
  if (a.parts_cap > states_words) return cudaErrorInvalidValue;
  a.states = states;
  a.ctl = ctl;
  a.status = status;
  scan_kernel<<<dim3(persistent_blocks(num_sms, 1, 4), 1), kScanThreads, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_offsets(const ViewSet& vs, FwdBufs& b, const Scratch& s, cudaStream_t st) {
  ScanArgs a{};
  a.in = b.count;
  a.gather = b.perm;
  a.out = b.offset;
  a.seg_stride = b.Vcap;
  a.counts = b.vcount;
  a.count_stride = 4;
  a.cap = b.Vcap;
  a.inclusive = 0;
  a.totals = b.vcount + 1;
  a.totals_stride = 4;
  a.cap_total = b.Icap;
  a.parts_cap = (uint32_t)((b.Vcap + kScanTile - 1) / kScanTile);
  if ((uint64_t)a.parts_cap * vs.n_views > s.lb_states_words) return cudaErrorInvalidValue;
  a.states = s.lb_states;
  a.ctl = s.ctl;
  a.status = s.status;
  // The scan gathers the counts through the depth order, one 4-byte read
  // per random index. Views are scanned in groups whose count arrays fit in
  // about a third of L2 together, so each 32-byte sector is fetched from
  // DRAM once rather than once per element read from it.
  constexpr uint64_t kGatherBytes = 40ull << 20;
  const uint32_t per = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(vs.n_views, kGatherBytes / (4 * b.Vcap)));
  for (uint32_t v0 = 0; v0 < vs.n_views; v0 += per) {
    const uint32_t nv = std::min(per, vs.n_views - v0);
    a.seg_base = v0;
    scan_kernel<<<dim3(persistent_blocks(s.num_sms, nv, 4), nv), kScanThreads, 0, st>>>(a);
  }
  return cudaGetLastError();
}

}  // namespace gsr

// ---------------------------------------------------------------------------
// Self-test of the bounded wait: one thread plays partition 1 of a look-back
// whose partition 0 never publishes (its state word carries another epoch),
// so the wait must give up after max_polls polls, flag the status and return.
// ---------------------------------------------------------------------------
namespace gsr {
namespace {
__global__ void lookback_timeout_probe_kernel(unsigned long long* states, DevStatus* status, uint32_t max_polls,
                                              uint32_t* out) {
  if (threadIdx.x == 0) {
    states[0] = 0ull;  // epoch 0: never the probe's epoch below
    *out = lookback(states, 1, 1, 7u, 0x3fffffffu, status, kWaitSelfTest, max_polls);
  }
}
}  // namespace

cudaError_t launch_lookback_timeout_probe(unsigned long long* states, DevStatus* status, uint32_t max_polls,
                                          uint32_t* out, cudaStream_t st) {
  lookback_timeout_probe_kernel<<<1, 32, 0, st>>>(states, status, max_polls, out);
  return cudaGetLastError();
}
}  // namespace gsr
