// gsr_kernels.h — host-side launchers of the rasterizer kernels and the
// device buffer layout they share. Internal to libgsr.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "gsr_internal.cuh"

namespace gsr {

constexpr int kMaxViews = kMaxSegments;

// Per-view scratch of one forward/backward. Every array is sized for
// max_views slots; view v's slice starts at v * <capacity>.
struct FwdBufs {
  float4* rec;             // [V][3] projected record (see k_project.cu)
  uint32_t* gid_of_c;      // [V] global id of compact index c (global-id order)
  uint32_t* depth_key;     // [V] f32 depth bits of c
  uint32_t* perm;          // [V] compact index of depth rank r
  uint32_t* depth_sorted;  // [V] sorted depth keys (sort output, unused after)
  uint32_t* key_tmp;       // [max(V, I)] sort double buffers
  uint32_t* val_tmp;
  uint32_t* count;         // [V] tile count of c
  uint32_t* offset;        // [V] first intersection of rank r
  int32_t* c_of_gid;       // [N] compact index of a global id, -1 if culled
  uint32_t* isect_key;     // [I] tile id, sorted (packed: tile id << pack_bits | compact index)
  uint32_t* isect_val;     // [I] compact index, sorted (unused when packed)
  uint32_t* isect_key_raw; // [I] emission order
  uint32_t* isect_val_raw;
  uint32_t* ranges;        // [2T]
  uint32_t* tile_hist;     // [T] intersections per tile (counted during emission)
  float* tfinal;           // [P] final transmittance
  uint32_t* last;          // [P] last contributor list index + 1
  uint32_t* ncontrib;      // [P]
  uint32_t* nvisit;        // [P]
  uint8_t* visible_c;      // [V]
  uint8_t* hitw;           // [I] per list entry: forward warp blocks with a pixel that took it
  uint32_t* vis_bits;      // projection: [views][proj_parts_cap * 8] visibility ballot words
  uint32_t* blk_count;     // projection: [views][proj_parts_cap] visible per projection block
  uint32_t* blk_base;      // projection: [views][proj_parts_cap] exclusive scan of blk_count
  uint32_t proj_parts_cap;
  float4* sgrad;           // [V][3] screen-space gradient sums (12 floats)
  float4* pair;            // [views][6][Vcap]: six float4 planes of projection adjoint records
  float* sgrad_part;       // [I][12] per-intersection partial sums (deterministic mode)
  uint32_t* inv_perm;      // [I] emission index -> sorted position (deterministic mode)
  uint32_t* vcount;        // [4] visible, intersections (clamped), intersections required, pad
  uint32_t* sched_order;   // [views * Tcap] persistent forward: work items in issue order
  uint32_t* sched_lists;   // [33][sched_items_cap] work items by the bit length of their backward cost
  uint32_t* sched_lcount;  // [33] items in each of those lists (appended by the forward)
  uint32_t* sched_ticket;  // [1] next ticket a persistent raster CTA takes
  uint64_t sched_items_cap;
  uint64_t Vcap, Ncap, Icap, Tcap, Pcap;
  uint32_t pack_bits;      // > 0: intersections are packed keys (see isect_key), else (tile, index) pairs
  bool slots;              // slot layout: one key per box tile, sentinel keys last; vcount[3] = keys sorted
};

// The compact index of intersection s (packed keys or pairs).
__host__ __device__ __forceinline__ const uint32_t* isect_index_src(const FwdBufs& b, uint32_t v) {
  return b.pack_bits ? b.isect_key + (size_t)b.Icap * v : b.isect_val + (size_t)b.Icap * v;
}
__device__ __forceinline__ uint32_t isect_index_mask(const FwdBufs& b) {
  return b.pack_bits ? (1u << b.pack_bits) - 1u : 0xffffffffu;
}
inline uint32_t isect_index_mask_host(const FwdBufs& b) { return b.pack_bits ? (1u << b.pack_bits) - 1u : 0xffffffffu; }

struct ViewSet {
  const ViewDesc* views;  // device
  uint32_t n_views;
  uint32_t tile_w, tile_h;
  uint32_t batch;         // Gaussians per shared-memory batch of the rasterizer (0: tuned defaults)
  uint32_t total_tiles;   // sum over views of tiles_x * tiles_y
  uint32_t max_tiles;     // max over views
  int persistent;         // kPersist* bits: raster kernels whose CTAs take cost-ordered items persistently
};
// Bits of ViewSet::persistent (otherwise one CTA per work item).
constexpr int kPersistFwd = 1, kPersistBwd = 2;

struct SplatsDev {
  const float* transforms;
  const void* sh;
  const float* raw_opac;
  uint32_t n;
  int degree;
  int sh_bf16;
};

// Pointers to a view's slice of a per-view array.
template <class T> __host__ __device__ __forceinline__ T* slice(T* base, uint64_t cap, uint32_t v) {
  return base + (size_t)cap * v;
}

struct Scratch {
  unsigned long long* lb_states;  // look-back states
  uint64_t lb_states_words;
  uint32_t* hist;                 // radix histograms [segments][4][256]
  uint32_t* hist_base;            // their exclusive scans
  LookbackCtl* ctl;
  DevStatus* status;
  int num_sms;
};

// Gaussians per projection block (visibility, per-block counts, records).
// 128 (staged SH rows of 25 KB, 7 records blocks per SM in place of 3) made
// the projection 0.009 ms faster per 8-view step of 1M Gaussians but the
// step no faster: the sorts that follow it lost as much.
constexpr uint32_t kProjBlock = 256;

// ---- launchers (return cudaGetLastError()) ----
cudaError_t launch_project(const SplatsDev& sp, const ViewSet& vs, float cov_blur, int fp64_conic, FwdBufs& b,
                           const Scratch& s, cudaStream_t st);

// Stable LSD radix sort of (key, value) pairs in `segments` segments of
// seg_stride elements; segment i holds counts[i * count_stride] elements
// (or n_host when counts is null). vals_in == nullptr means values 0..n-1;
// vals_out == nullptr sorts the keys alone. The digits are `bits` bits
// from bit shift0 up. The result lands in keys_out/vals_out; tmp buffers
// are clobbered. With counts_dropped (histograms from the caller, digits
// below 8 bits), keys equal to 0xffffffff are dropped in the first pass:
// the histograms must not count them, and counts_dropped[i * count_stride]
// gives segment i's count without them (the sorted output's length).
// Radix passes and digit width for a sort over `bits` key bits.
inline int sort_passes(int bits) {
  const int p = (bits + 7) / 8;
  return p < 1 ? 1 : (p > 4 ? 4 : p);
}
inline int sort_digit_bits(int bits) {
  const int p = sort_passes(bits);
  const int d = (bits + p - 1) / p;
  return d < 1 ? 1 : (d > 8 ? 8 : d);
}
// Digit widths of the tile sort (histograms from emission): the tile-id
// digits of consecutive keys are spread in the low bits and clustered in the
// high ones, so the second pass takes up to kTileSecondDigit bits and the
// first the rest. Equal to sort_digit_bits for one pass.
constexpr int kTileSecondDigit = 8;
inline int tile_first_digit_bits(int bits) {
  if (sort_passes(bits) != 2) return sort_digit_bits(bits);
  const int d1 = kTileSecondDigit < bits - 1 ? kTileSecondDigit : bits - 1;
  return bits - d1;
}
cudaError_t radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                             uint32_t* vals_out, uint32_t* keys_tmp, uint32_t* vals_tmp, uint64_t seg_stride,
                             uint32_t segments, const uint32_t* counts, uint32_t count_stride, uint32_t n_host,
                             uint64_t cap_per_segment, int bits, const Scratch& s, cudaStream_t st,
                             bool hist_ready = false, uint32_t shift0 = 0, const uint32_t* counts_dropped = nullptr,
                             int first_bits = 0);

// Bounded-wait self-test: a look-back whose predecessor never publishes
// (look-back states 0 and 1 are overwritten); gives up after max_polls.
cudaError_t launch_lookback_timeout_probe(unsigned long long* states, DevStatus* status, uint32_t max_polls,
                                          uint32_t* out, cudaStream_t st);

// Inclusive scan of n_host values (prefix sum primitive).
cudaError_t inclusive_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n_host, const Scratch& s,
                               cudaStream_t st);

// The same scan with caller-provided look-back scratch (no context).
cudaError_t inclusive_scan_u32_scratch(const uint32_t* in, uint32_t* out, uint32_t n_host, unsigned long long* states,
                                       uint64_t states_words, LookbackCtl* ctl, DevStatus* status, int num_sms,
                                       cudaStream_t st);

// Per view: offset[r] = exclusive scan of count[perm[r]], sets vcount[1..2].
cudaError_t launch_offsets(const ViewSet& vs, FwdBufs& b, const Scratch& s, cudaStream_t st);

// Per-view tile counts of the compact records (count[c], gid order).
cudaError_t launch_count(const ViewSet& vs, FwdBufs& b, const Scratch& s, cudaStream_t st);
cudaError_t launch_emit(const ViewSet& vs, FwdBufs& b, const Scratch& s, int deterministic, cudaStream_t st);
// Emission that also counts the emitted intersections per tile (tile_hist),
// then, from those counts, the tile ranges and the tile sort's per-pass digit
// histograms (Scratch::hist), replacing the sort's histogram pass and the
// ranges kernel. For views of at most kHistMaxTiles tiles.
constexpr uint32_t kHistMaxTiles = 8192;
// slots: the slot layout (offsets from box sizes, failing tiles write the
// sentinel key); packed keys only.
cudaError_t launch_emit_hist(const ViewSet& vs, FwdBufs& b, const Scratch& s, int deterministic, bool slots,
                             cudaStream_t st);
// Tile ranges and the tile sort's digit histograms (digits of
// sort_digit_bits(bits_for(max tiles)) bits) from emission's tile counts.
cudaError_t launch_tile_hist_finish(const ViewSet& vs, FwdBufs& b, const Scratch& s, int tile_bits, bool slots,
                                   bool drop_sentinels,
                                   cudaStream_t st);
// Packed mode only: the passing-tile counts of a view's compact indices,
// recounted from its sorted intersections into b.count.
cudaError_t launch_count_from_isects(FwdBufs& b, uint32_t view, uint32_t n_visible, cudaStream_t st);
// Packed mode only: intersections [0, n) of a view as separate tile ids and
// compact indices.
cudaError_t launch_unpack_isects(const FwdBufs& b, uint32_t view, uint32_t n, uint32_t* tiles, uint32_t* vals,
                                 cudaStream_t st);
cudaError_t launch_remap(const ViewSet& vs, FwdBufs& b, const Scratch& s, cudaStream_t st);
cudaError_t launch_ranges(const ViewSet& vs, FwdBufs& b, const Scratch& s, cudaStream_t st);

// Looks up the residency of the raster kernels of a tile shape and batch
// (persistent schedule) outside any stream capture; enqueues nothing.
void raster_warm_up(uint32_t tile_w, uint32_t tile_h, uint32_t batch, int num_sms);
cudaError_t launch_raster_fwd(const ViewSet& vs, FwdBufs& b, const float* bg, float* out_rgba, const Scratch& s,
                              cudaStream_t st);
cudaError_t launch_raster_bwd(const ViewSet& vs, FwdBufs& b, const float* bg, const float* v_rgba, int ref_mode,
                              int deterministic, const Scratch& s, cudaStream_t st);
cudaError_t launch_reduce_det(const ViewSet& vs, FwdBufs& b, const Scratch& s, cudaStream_t st);

// Copies view descriptors to device memory through a kernel argument (safe
// to enqueue repeatedly and to capture in a graph).
struct ViewDescBlock {
  ViewDesc v[kMaxViews];
};
cudaError_t launch_set_views(ViewDesc* dst, const ViewDesc* host, uint32_t n, cudaStream_t st);

cudaError_t launch_visible_out(const ViewSet& vs, FwdBufs& b, uint32_t n, float* out_visible, cudaStream_t st);

// 8-bit RGB frames to f32 training targets (views packed back to back).
struct FrameSpec {
  uint64_t src_offset;     // byte offset of the frame in the frame buffer
  uint32_t src_w, src_h;   // frame size
  uint32_t dst_w, dst_h;   // training resolution of the view
};
cudaError_t launch_frames_to_targets(const uint8_t* frames, const FrameSpec* spec, uint32_t n_views, float* out,
                                     cudaStream_t st);

// Per-step optimizer scalars, read by the kernels from device memory so that
// a captured step can be replayed with new values.
struct AdamScalars {
  float lr_pos, lr_rot, lr_scale, lr_color, lr_opac;
  float beta1, beta2, eps;
  float rbc1, rbc2;  // 1 / (1 - beta^step), rounded to f32
};

struct AdamArgs {
  float* transforms;
  void* sh;
  float* raw_opac;
  float* m_tr;
  float* v_tr;
  float* m_sh;
  float* v_sh;
  float* m_op;
  float* v_op;
  const AdamScalars* scal;  // device
};

// Writes the scalars to device memory (a one-thread kernel, so the values
// travel as launch arguments and the call is safe to issue per step).
cudaError_t launch_set_scalars(AdamScalars* dst, const AdamScalars& v, cudaStream_t st);

// Project backward over all Gaussians for all views of the last forward:
// writes the gradients (summed over views, scaled by grad_scale), optional
// per-view stats, and optionally accumulates the densification statistics
// view by view.
struct ProjBwdArgs {
  float* v_tr;
  float* v_sh;
  float* v_op;
  float* stats;        // [views][n][7] or null
  float* densify_acc;  // [9][n] or null
  int use_visible;
  float grad_scale;
  int exact;
  int hp;  // FP64 conic mode of the forward
};
cudaError_t launch_project_bwd(const SplatsDev& sp, const ViewSet& vs, float cov_blur, FwdBufs& b,
                               const ProjBwdArgs& a, cudaStream_t st, int num_sms);

cudaError_t launch_adam(const AdamArgs& a, const float* g_tr, const float* g_sh, const float* g_op, uint32_t n,
                        int degree, int sh_bf16, cudaStream_t st, int num_sms);
cudaError_t launch_densify(const float* v_tr, const float* stats, const float* v_sh, const float* visible, uint32_t n,
                           int degree, int use_visible, float* acc, cudaStream_t st, int num_sms);

// Topology apply: output row i from plan row i (source, kind, sample).
struct TopoRow {
  uint32_t source;
  int32_t kind;
  float sample;
  uint32_t pad;
};
cudaError_t launch_topology(const SplatsDev& sp, const TopoRow* rows, uint32_t m, const TopoParams& p, float* otr,
                            void* osh, float* oop, DevStatus* status, cudaStream_t st, int num_sms);

// Loss: per view, l1_w*L1 + ssim_w*(1-SSIM); writes loss[v] and v_pred (RGBA).
cudaError_t launch_loss(const ViewSet& vs, const ViewDesc* host_views, const float* pred, const float* target,
                        float l1_w, float ssim_w, float* loss, float* v_pred, float* work, uint64_t work_floats,
                        cudaStream_t st);

}  // namespace gsr
