// api.cu — the C ABI of include/gsr.h: context, scratch ownership and the
// orchestration of the forward (render_forward, RustGS/src/training/forward/
// mod.rs:156-294), the backward (RenderBackward::backward, backward/
// autodiff.rs:85-141), the loss, Adam and the training step
// (WgpuTrainer::train_step, engine/trainer.rs:253-440).
//
// Unlike the reference, no stage reads a count back to the host: every
// kernel takes the visible and intersection counts from device memory and
// runs over capacity-sized buffers, so a whole step can be enqueued (and
// captured in a CUDA graph) without a synchronisation. An intersection count
// above capacity is clamped, flagged on the device and reported by
// gsr_sync_status.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/gsr.h"
#include "gsr_kernels.h"

using namespace gsr;

namespace gsr {
void ssim_window(float* k);
uint32_t loss_tiles(uint32_t w, uint32_t h);
}  // namespace gsr

struct gsr_ctx {
  gsr_config cfg{};
  int device = 0;
  int num_sms = 148;
  std::string err;
  // per-view scratch
  FwdBufs b{};
  Scratch s{};
  ViewDesc* d_views = nullptr;
  std::vector<void*> allocs;
  uint64_t states_words = 0;
  // last forward
  bool have_fwd = false;
  uint32_t fwd_views = 0;
  uint32_t fwd_n = 0;
  int fwd_degree = 0;
  std::vector<ViewDesc> fwd_desc;
  ViewSet fwd_vs{};
  // training-step buffers
  float* render = nullptr;  // [views][Pcap][4]
  float* v_render = nullptr;
  float* loss_work = nullptr;
  uint64_t loss_work_floats = 0;
  float* grad_work = nullptr;  // summed gradient of a training step: [N][10], [N][3K<=75], [N] (16-byte aligned)
  uint64_t grad_sh_off = 0, grad_op_off = 0;
  AdamScalars* d_scal = nullptr;
  // graph cache of the training step: the whole step, or (when the step
  // waits on a targets-ready event) its forward here and the rest in
  // graph_exec_rest
  cudaGraphExec_t graph_exec = nullptr;
  cudaGraphExec_t graph_exec_rest = nullptr;
  std::vector<uint8_t> graph_key;
  int graph_kernels = 0;
  cudaStream_t capture_stream = nullptr;  // graphs are recorded here (the legacy default stream cannot capture)
  // optional stage timing (events recorded between stages; never in a graph)
  bool prof_on = false;
  std::vector<int> prof_stage;
  std::vector<cudaEvent_t> prof_ev;
  size_t prof_used = 0;
};

namespace {

gsr_status fail(gsr_ctx* c, gsr_status st, const std::string& msg) {
  if (c) c->err = msg;
  return st;
}

gsr_status cuda_fail(gsr_ctx* c, cudaError_t e, const char* where) {
  if (c) c->err = std::string(where) + ": " + cudaGetErrorString(e);
  (void)cudaGetLastError();
  return GSR_ERR_CUDA;
}

#define GSR_CUDA(ctx, call)                                  \
  do {                                                       \
    cudaError_t _e = (call);                                 \
    if (_e != cudaSuccess) return cuda_fail(ctx, _e, #call); \
  } while (0)

template <class T> bool dalloc(gsr_ctx* c, T** p, uint64_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  void* q = nullptr;
  if (cudaMalloc(&q, sizeof(T) * count) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  c->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return true;
}

// Stage ids reported by gsr_profile_read (see include/gsr.h).
enum Stage { kStProject = 0, kStDepthSort, kStOffsets, kStEmit, kStTileSort, kStRanges, kStRasterFwd, kStVisible,
             kStLoss, kStRasterBwd, kStReduce, kStProjectBwd, kStAdam, kStCount };

void prof_mark(gsr_ctx* c, int stage, cudaStream_t st) {
  if (!c->prof_on) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
  if (c->prof_used == c->prof_ev.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    c->prof_ev.push_back(e);
    c->prof_stage.push_back(stage);
  }
  c->prof_stage[c->prof_used] = stage;
  cudaEventRecord(c->prof_ev[c->prof_used], st);
  ++c->prof_used;
}

void free_all(gsr_ctx* c) {
  for (cudaEvent_t e : c->prof_ev) cudaEventDestroy(e);
  c->prof_ev.clear();
  c->prof_stage.clear();
  c->prof_used = 0;
  for (void* p : c->allocs) cudaFree(p);
  c->allocs.clear();
  if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
  c->graph_exec = nullptr;
  if (c->graph_exec_rest) cudaGraphExecDestroy(c->graph_exec_rest);
  c->graph_exec_rest = nullptr;
  if (c->capture_stream) cudaStreamDestroy(c->capture_stream);
  c->capture_stream = nullptr;
}

uint64_t tcap_for(const gsr_config& cfg) { return cfg.max_pixels / ((uint64_t)cfg.tile_w * cfg.tile_h) + 4096; }

gsr_status allocate(gsr_ctx* c) {
  const gsr_config& cfg = c->cfg;
  const uint64_t V = cfg.max_splats, N = cfg.max_splats, I = cfg.max_isects, P = cfg.max_pixels;
  const uint64_t T = tcap_for(cfg);
  const uint64_t nv = cfg.max_views;
  FwdBufs& b = c->b;
  b.Vcap = V;
  b.Ncap = N;
  b.Icap = I;
  b.Tcap = T;
  b.Pcap = P;
  const uint64_t VI = std::max(V, I);
  bool ok = dalloc(c, &b.rec, nv * V * 3) && dalloc(c, &b.gid_of_c, nv * V) && dalloc(c, &b.depth_key, nv * V) &&
            dalloc(c, &b.perm, nv * V) && dalloc(c, &b.depth_sorted, nv * V) && dalloc(c, &b.key_tmp, nv * VI) &&
            dalloc(c, &b.val_tmp, nv * VI) && dalloc(c, &b.count, nv * V) && dalloc(c, &b.offset, nv * V) &&
            dalloc(c, &b.c_of_gid, nv * N) && dalloc(c, &b.isect_key, nv * I) && dalloc(c, &b.isect_val, nv * I) &&
            dalloc(c, &b.isect_key_raw, nv * I) && dalloc(c, &b.isect_val_raw, nv * I) &&
            dalloc(c, &b.ranges, nv * 2 * T) && dalloc(c, &b.tfinal, nv * P) && dalloc(c, &b.last, nv * P) &&
            dalloc(c, &b.ncontrib, nv * P) && dalloc(c, &b.nvisit, nv * P) && dalloc(c, &b.visible_c, nv * V) &&
            dalloc(c, &b.sgrad, nv * V * 3) && dalloc(c, &b.pair, nv * V * 6) && dalloc(c, &b.vcount, nv * 4) &&
            dalloc(c, &b.tile_hist, nv * T) && dalloc(c, &b.hitw, nv * I) && dalloc(c, &b.sched_order, nv * T) &&
            dalloc(c, &b.sched_lists, 33 * nv * T) && dalloc(c, &b.sched_lcount, 33) && dalloc(c, &b.sched_ticket, 1);
  b.sched_items_cap = nv * T;
  b.proj_parts_cap = (uint32_t)((N + kProjBlock - 1) / kProjBlock);
  ok = ok && dalloc(c, &b.vis_bits, nv * b.proj_parts_cap * 8) && dalloc(c, &b.blk_count, nv * b.proj_parts_cap) &&
       dalloc(c, &b.blk_base, nv * b.proj_parts_cap);
  if (ok && cfg.deterministic)
    ok = dalloc(c, &b.sgrad_part, nv * I * 12) && dalloc(c, &b.inv_perm, nv * I);
  else {
    b.sgrad_part = nullptr;
    b.inv_perm = nullptr;
  }
  // Look-back states: the largest of the compaction (256 Gaussians per
  // partition), the scans (2048) and the sorts (4096 keys, 256 digits).
  const uint64_t w_proj = ((N + 255) / 256) * nv;
  const uint64_t w_sort = ((VI + 4095) / 4096) * 256 * nv;
  const uint64_t w_scan = ((std::max<uint64_t>(V, 1u << 20) + 2047) / 2048) * nv;
  c->states_words = std::max(std::max(w_proj, w_sort), w_scan);
  ok = ok && dalloc(c, &c->s.lb_states, c->states_words) && dalloc(c, &c->s.hist, 64 * 1024) &&
       dalloc(c, &c->s.hist_base, 64 * 1024) && dalloc(c, &c->s.ctl, 1) && dalloc(c, &c->s.status, 1) &&
       dalloc(c, &c->d_views, nv) && dalloc(c, &c->d_scal, 1);
  const uint64_t lt = loss_tiles(1, 1) + P / (32 * 16) + 2 * (P / 16) + 64;
  c->loss_work_floats = nv * 9 * P + nv * 3 * lt * 2;
  c->grad_sh_off = (N * 10 + 3) & ~uint64_t(3);
  c->grad_op_off = c->grad_sh_off + ((N * 75 + 3) & ~uint64_t(3));
  ok = ok && dalloc(c, &c->render, nv * P * 4) && dalloc(c, &c->v_render, nv * P * 4) &&
       dalloc(c, &c->loss_work, c->loss_work_floats) && dalloc(c, &c->grad_work, c->grad_op_off + N);
  if (!ok) return fail(c, GSR_ERR_OOM, "device allocation failed (reduce max_splats/max_isects/max_pixels)");
  c->s.lb_states_words = c->states_words;
  c->s.num_sms = c->num_sms;
  // Zero the look-back states (epoch 0 never matches a launch), the control
  // block and the status words.
  if (cudaMemset(c->s.lb_states, 0, sizeof(unsigned long long) * c->states_words) != cudaSuccess ||
      cudaMemset(c->s.ctl, 0, sizeof(LookbackCtl)) != cudaSuccess ||
      cudaMemset(c->s.status, 0, sizeof(DevStatus)) != cudaSuccess ||
      cudaMemset(b.vcount, 0, sizeof(uint32_t) * 4 * nv) != cudaSuccess ||
      cudaMemset(b.sched_lcount, 0, sizeof(uint32_t) * 33) != cudaSuccess)
    return cuda_fail(c, cudaGetLastError(), "cudaMemset");
  raster_warm_up(cfg.tile_w, cfg.tile_h, cfg.batch, c->num_sms);
  return GSR_OK;
}

bool valid_tile(uint32_t w, uint32_t h) { return (w == 16 && h == 16) || (w == 8 && h == 8) || (w == 32 && h == 8); }

// Builds the per-view descriptors; fails if a view exceeds the capacities.
gsr_status build_views(gsr_ctx* c, const gsr_camera* cams, uint32_t n_views, std::vector<ViewDesc>& out,
                       ViewSet& vs) {
  if (!cams || n_views == 0) return fail(c, GSR_ERR_INVALID_ARG, "no cameras");
  if (n_views > c->cfg.max_views) return fail(c, GSR_ERR_INVALID_ARG, "n_views exceeds max_views");
  out.resize(n_views);
  uint32_t tile_base = 0, max_tiles = 0;
  uint64_t pix_base = 0;
  for (uint32_t v = 0; v < n_views; ++v) {
    const gsr_camera& cm = cams[v];
    ViewDesc& d = out[v];
    memset(&d, 0, sizeof(d));
    if (cm.width == 0 || cm.height == 0) return fail(c, GSR_ERR_INVALID_ARG, "empty image");
    if ((uint64_t)cm.width * cm.height > c->cfg.max_pixels) return fail(c, GSR_ERR_INVALID_ARG, "view exceeds max_pixels");
    if (!(cm.fx > 0.f) || !(cm.fy > 0.f)) return fail(c, GSR_ERR_INVALID_ARG, "focal length must be positive");
    for (int col = 0; col < 3; ++col)
      for (int row = 0; row < 3; ++row) d.rot[col * 3 + row] = cm.viewmat[col * 4 + row];
    d.trans[0] = cm.viewmat[12];
    d.trans[1] = cm.viewmat[13];
    d.trans[2] = cm.viewmat[14];
    d.fx = cm.fx;
    d.fy = cm.fy;
    d.cx = cm.cx;
    d.cy = cm.cy;
    d.w = cm.width;
    d.h = cm.height;
    d.campos[0] = cm.campos[0];
    d.campos[1] = cm.campos[1];
    d.campos[2] = cm.campos[2];
    d.tiles_x = (cm.width + c->cfg.tile_w - 1) / c->cfg.tile_w;
    d.tiles_y = (cm.height + c->cfg.tile_h - 1) / c->cfg.tile_h;
    const uint64_t nt = (uint64_t)d.tiles_x * d.tiles_y;
    if (nt > c->b.Tcap || d.tiles_x > 65535 || d.tiles_y > 65535)
      return fail(c, GSR_ERR_INVALID_ARG, "view has too many tiles");
    d.tile_base = tile_base;
    d.pix_base = pix_base;
    tile_base += (uint32_t)nt;
    max_tiles = std::max<uint32_t>(max_tiles, (uint32_t)nt);
    pix_base += (uint64_t)cm.width * cm.height;
  }
  vs.views = c->d_views;
  vs.n_views = n_views;
  vs.tile_w = c->cfg.tile_w;
  vs.tile_h = c->cfg.tile_h;
  vs.batch = c->cfg.batch;
  vs.total_tiles = tile_base;
  vs.max_tiles = max_tiles;
  // The default runs the backward persistently and the forward as a grid:
  // on the 8-view 1280x720 step the cost order shortens the backward by 5%,
  // while the forward, whose cost (entries up to saturation) the list length
  // predicts poorly, is 2% faster as a grid.
  vs.persistent = c->cfg.schedule == GSR_SCHEDULE_PERSISTENT ? (kPersistFwd | kPersistBwd)
                  : c->cfg.schedule == GSR_SCHEDULE_GRID     ? 0
                                                             : kPersistBwd;
  return GSR_OK;
}

int bits_for(uint32_t n) {
  int b = 1;
  while (b < 32 && (1ull << b) < (uint64_t)n) ++b;
  return b;
}

SplatsDev splats_dev(const gsr_ctx* c, const gsr_splats* sp) {
  SplatsDev d;
  d.transforms = sp->transforms;
  d.sh = sp->sh;
  d.raw_opac = sp->raw_opacity;
  d.n = sp->n;
  d.degree = (int)sp->sh_degree;
  d.sh_bf16 = c->cfg.sh_dtype == GSR_SH_BF16;
  return d;
}

gsr_status check_splats(gsr_ctx* c, const gsr_splats* sp) {
  if (!sp) return fail(c, GSR_ERR_INVALID_ARG, "null splats");
  if (sp->n > c->cfg.max_splats) return fail(c, GSR_ERR_INVALID_ARG, "n exceeds max_splats");
  if (sp->sh_degree > 4) return fail(c, GSR_ERR_INVALID_ARG, "sh_degree must be 0..4");
  if (sp->n > 0 && (!sp->transforms || !sp->sh || !sp->raw_opacity))
    return fail(c, GSR_ERR_INVALID_ARG, "null parameter pointer");
  if (sp->n > 0 && (reinterpret_cast<uintptr_t>(sp->transforms) & 15u))
    return fail(c, GSR_ERR_INVALID_ARG, "transforms must be 16-byte aligned");
  return GSR_OK;
}

// Enqueues the whole forward. out_rgba is the packed image buffer.
gsr_status forward_impl(gsr_ctx* c, const gsr_splats* sp, const gsr_camera* cams, uint32_t n_views, float* out_rgba,
                        float* out_visible, cudaStream_t st) {
  gsr_status rs = check_splats(c, sp);
  if (rs != GSR_OK) return rs;
  if (!out_rgba) return fail(c, GSR_ERR_INVALID_ARG, "null out_rgba");
  std::vector<ViewDesc> desc;
  ViewSet vs;
  rs = build_views(c, cams, n_views, desc, vs);
  if (rs != GSR_OK) return rs;
  GSR_CUDA(c, launch_set_views(c->d_views, desc.data(), n_views, st));
  const SplatsDev sd = splats_dev(c, sp);
  FwdBufs& b = c->b;
  prof_mark(c, kStProject, st);
  GSR_CUDA(c, launch_project(sd, vs, c->cfg.cov_blur, c->cfg.fp64_conic, b, c->s, st));
  prof_mark(c, kStDepthSort, st);
  GSR_CUDA(c, radix_sort_pairs(b.depth_key, nullptr, b.depth_sorted, b.perm, b.key_tmp, b.val_tmp, b.Vcap, n_views,
                               b.vcount, 4, 0, b.Vcap, 31, c->s, st));
  // Up to kHistMaxTiles tiles a view, emission also counts intersections
  // per tile: the tile ranges and the tile sort's digit histograms follow
  // from those counts (no histogram pass, no ranges pass).
  const bool tile_counts = vs.max_tiles <= kHistMaxTiles;
  // With tile counts from emission and no deterministic bookkeeping, an
  // intersection whose tile id and compact index fit in 32 bits together is
  // one packed key (tile id high, index low), sorted alone.
  const int tbits = bits_for(vs.max_tiles), ibits = bits_for(sp->n);
  b.pack_bits = (tile_counts && !c->cfg.deterministic && tbits + ibits <= 32) ? (uint32_t)ibits : 0u;
  // With tile counts from emission, no deterministic bookkeeping and a
  // spare tile id, the slot layout: every box tile gets a slot (offsets from
  // the box sizes the projection wrote), failing tiles hold a sentinel key
  // that sorts last, and no counting walk runs. Keys are packed when tile id
  // and compact index fit in 32 bits, else (tile id, compact index) pairs.
  b.slots = tile_counts && !c->cfg.deterministic && vs.max_tiles < (1u << tbits);
  prof_mark(c, kStOffsets, st);
  if (!b.slots) GSR_CUDA(c, launch_count(vs, b, c->s, st));
  GSR_CUDA(c, launch_offsets(vs, b, c->s, st));
  prof_mark(c, kStEmit, st);
  // In the slot layout the tile sort drops the failing tiles' sentinel keys
  // in its first pass when its digits leave a spare digit value (below 8
  // bits), so the second pass and the scatter move real intersections only.
  const bool drop_sentinels = b.slots && tile_first_digit_bits(tbits) < 8;
  if (tile_counts) {
    GSR_CUDA(c, launch_emit_hist(vs, b, c->s, c->cfg.deterministic, b.slots, st));
    GSR_CUDA(c, launch_tile_hist_finish(vs, b, c->s, tbits, b.slots, drop_sentinels, st));
  } else {
    GSR_CUDA(c, launch_emit(vs, b, c->s, c->cfg.deterministic, st));
  }
  prof_mark(c, kStTileSort, st);
  const uint32_t* real_counts = drop_sentinels ? b.vcount + 1 : nullptr;
  if (b.pack_bits)
    GSR_CUDA(c, radix_sort_pairs(b.isect_key_raw, nullptr, b.isect_key, nullptr, b.key_tmp, nullptr, b.Icap, n_views,
                                 b.vcount + (b.slots ? 3 : 1), 4, 0, b.Icap, tbits, c->s, st, true, b.pack_bits,
                                 real_counts, tile_first_digit_bits(tbits)));
  else
    GSR_CUDA(c, radix_sort_pairs(b.isect_key_raw, b.isect_val_raw, b.isect_key, b.isect_val, b.key_tmp, b.val_tmp,
                                 b.Icap, n_views, b.vcount + (b.slots ? 3 : 1), 4, 0, b.Icap, tbits, c->s, st,
                                 tile_counts, 0, real_counts, tile_counts ? tile_first_digit_bits(tbits) : 0));
  if (c->cfg.deterministic) GSR_CUDA(c, launch_remap(vs, b, c->s, st));
  prof_mark(c, kStRanges, st);
  if (!tile_counts) GSR_CUDA(c, launch_ranges(vs, b, c->s, st));
  prof_mark(c, kStRasterFwd, st);
  GSR_CUDA(c, launch_raster_fwd(vs, b, c->cfg.background, out_rgba, c->s, st));
  prof_mark(c, kStVisible, st);
  if (out_visible) GSR_CUDA(c, launch_visible_out(vs, b, sp->n, out_visible, st));
  c->have_fwd = true;
  c->fwd_views = n_views;
  c->fwd_n = sp->n;
  c->fwd_degree = (int)sp->sh_degree;
  c->fwd_desc = desc;
  c->fwd_vs = vs;
  return GSR_OK;
}

gsr_status raster_backward_impl(gsr_ctx* c, const float* v_rgba, cudaStream_t st) {
  FwdBufs& b = c->b;
  prof_mark(c, kStRasterBwd, st);
  GSR_CUDA(c, launch_raster_bwd(c->fwd_vs, b, c->cfg.background, v_rgba, c->cfg.adjoint == GSR_ADJOINT_REFERENCE,
                                c->cfg.deterministic, c->s, st));
  prof_mark(c, kStReduce, st);
  if (c->cfg.deterministic) GSR_CUDA(c, launch_reduce_det(c->fwd_vs, b, c->s, st));
  return GSR_OK;
}

}  // namespace

extern "C" {

const char* gsr_version(void) { return "gsr 0.1 (sm_100a)"; }

const char* gsr_last_error(const gsr_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

gsr_status gsr_create(const gsr_config* cfg_in, gsr_ctx** out) {
  if (!out) return GSR_ERR_INVALID_ARG;
  *out = nullptr;
  gsr_ctx* c = new (std::nothrow) gsr_ctx();
  if (!c) return GSR_ERR_OOM;
  gsr_config cfg{};
  if (cfg_in) cfg = *cfg_in;
  if (cfg.tile_w == 0 && cfg.tile_h == 0) {
    cfg.tile_w = 16;
    cfg.tile_h = 16;
  }
  if (cfg.max_views == 0) cfg.max_views = 1;
  if (cfg.max_splats == 0) cfg.max_splats = 1u << 16;
  if (cfg.max_pixels == 0) cfg.max_pixels = 1920ull * 1080ull;
  if (cfg.max_isects == 0) cfg.max_isects = std::min<uint64_t>(std::max<uint64_t>(16 * cfg.max_splats, 1u << 20), 1ull << 29);
  c->cfg = cfg;
  gsr_status st = GSR_OK;
  if (!valid_tile(cfg.tile_w, cfg.tile_h)) st = fail(c, GSR_ERR_INVALID_ARG, "tile shape must be 16x16, 8x8 or 32x8");
  else if (cfg.max_views > (uint32_t)kMaxViews) st = fail(c, GSR_ERR_INVALID_ARG, "max_views exceeds 64");
  else if (cfg.max_splats >= (1ull << 30) || cfg.max_isects >= (1ull << 30))
    st = fail(c, GSR_ERR_INVALID_ARG, "capacities must stay below 2^30");
  else if (cfg.sh_dtype != GSR_SH_F32 && cfg.sh_dtype != GSR_SH_BF16)
    st = fail(c, GSR_ERR_INVALID_ARG, "unknown sh_dtype");
  else if (!(cfg.cov_blur >= 0.f))
    st = fail(c, GSR_ERR_INVALID_ARG, "cov_blur must be >= 0");
  else if (cfg.schedule != GSR_SCHEDULE_DEFAULT && cfg.schedule != GSR_SCHEDULE_PERSISTENT &&
           cfg.schedule != GSR_SCHEDULE_GRID)
    st = fail(c, GSR_ERR_INVALID_ARG, "unknown schedule");
  if (st != GSR_OK) {
    gsr_status r = st;
    delete c;
    return r;
  }
  if (cudaGetDevice(&c->device) != cudaSuccess ||
      cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess) {
    (void)cudaGetLastError();
    delete c;
    return GSR_ERR_CUDA;
  }
  st = allocate(c);
  if (st != GSR_OK) {
    free_all(c);
    delete c;
    return st;
  }
  *out = c;
  return GSR_OK;
}

void gsr_destroy(gsr_ctx* ctx) {
  if (!ctx) return;
  free_all(ctx);
  delete ctx;
}

gsr_status gsr_sync_status(gsr_ctx* c, void* stream, uint64_t* required) {
  if (!c) return GSR_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  DevStatus h{};
  GSR_CUDA(c, cudaMemcpyAsync(&h, c->s.status, sizeof(DevStatus), cudaMemcpyDeviceToHost, st));
  GSR_CUDA(c, cudaStreamSynchronize(st));
  GSR_CUDA(c, cudaMemsetAsync(c->s.status, 0, sizeof(DevStatus), st));
  GSR_CUDA(c, cudaStreamSynchronize(st));
  if (required) *required = h.required;
  if (h.timeout) {
    char buf[96];
    snprintf(buf, sizeof(buf), "bounded device wait gave up (site %u)", h.timeout_where);
    return fail(c, GSR_ERR_TIMEOUT, buf);
  }
  if (h.bad_input) return fail(c, GSR_ERR_INVALID_ARG, "a topology plan row names a source splat out of range");
  if (h.internal) return fail(c, GSR_ERR_CUDA, "internal check failed: a sort position fell outside its segment");
  if (h.overflow) {
    char buf[128];
    snprintf(buf, sizeof(buf), "intersection capacity %llu exceeded: %llu required",
             (unsigned long long)c->b.Icap, (unsigned long long)h.required);
    return fail(c, GSR_ERR_CAPACITY, buf);
  }
  return GSR_OK;
}

gsr_status gsr_reserve_isects(gsr_ctx* c, uint64_t max_isects) {
  if (!c) return GSR_ERR_INVALID_ARG;
  if (max_isects <= c->cfg.max_isects) return GSR_OK;
  if (max_isects >= (1ull << 30)) return fail(c, GSR_ERR_INVALID_ARG, "capacity must stay below 2^30");
  if (cudaDeviceSynchronize() != cudaSuccess) return cuda_fail(c, cudaGetLastError(), "cudaDeviceSynchronize");
  free_all(c);
  c->cfg.max_isects = max_isects;
  c->have_fwd = false;
  c->graph_key.clear();
  return allocate(c);
}

gsr_status gsr_prefix_sum_u32(gsr_ctx* c, const uint32_t* in, uint32_t* out, uint32_t n, void* stream) {
  if (!c) return GSR_ERR_INVALID_ARG;
  if (n == 0) return GSR_OK;
  if (!in || !out || in == out) return fail(c, GSR_ERR_INVALID_ARG, "bad prefix-sum buffers");
  if (n >= (1u << 30)) return fail(c, GSR_ERR_INVALID_ARG, "n must stay below 2^30");
  if ((uint64_t)((n + 2047) / 2048) > c->states_words)
    return fail(c, GSR_ERR_INVALID_ARG, "n exceeds the context's scan capacity");
  GSR_CUDA(c, inclusive_scan_u32(in, out, n, c->s, (cudaStream_t)stream));
  return GSR_OK;
}

gsr_status gsr_radix_sort_by_key_u32(gsr_ctx* c, const uint32_t* keys_in, const uint32_t* vals_in,
                                     uint32_t* keys_out, uint32_t* vals_out, uint32_t n, void* stream) {
  if (!c) return GSR_ERR_INVALID_ARG;
  if (n == 0) return GSR_OK;
  if (!keys_in || !vals_in || !keys_out || !vals_out) return fail(c, GSR_ERR_INVALID_ARG, "null sort buffer");
  if (keys_in == keys_out || vals_in == vals_out) return fail(c, GSR_ERR_INVALID_ARG, "sort buffers may not alias");
  if (n >= (1u << 30)) return fail(c, GSR_ERR_INVALID_ARG, "n must stay below 2^30");
  const uint64_t tmp_cap = std::max(c->b.Vcap, c->b.Icap) * c->cfg.max_views;
  if (n > tmp_cap || (uint64_t)((n + 4095) / 4096) * 256 > c->states_words)
    return fail(c, GSR_ERR_INVALID_ARG, "n exceeds the context's sort capacity");
  GSR_CUDA(c, radix_sort_pairs(keys_in, vals_in, keys_out, vals_out, c->b.key_tmp, c->b.val_tmp, 0, 1, nullptr, 0, n,
                               n, 32, c->s, (cudaStream_t)stream));
  return GSR_OK;
}

gsr_status gsr_render_forward(gsr_ctx* c, const gsr_splats* sp, const gsr_camera* cams, uint32_t n_views,
                              float* out_rgba, float* out_visible, void* stream) {
  if (!c) return GSR_ERR_INVALID_ARG;
  return forward_impl(c, sp, cams, n_views, out_rgba, out_visible, (cudaStream_t)stream);
}

gsr_status gsr_render_backward(gsr_ctx* c, const gsr_splats* sp, const float* v_rgba, const gsr_grads* grads,
                               float* stats, void* stream) {
  if (!c) return GSR_ERR_INVALID_ARG;
  if (!c->have_fwd) return fail(c, GSR_ERR_NOT_READY, "backward without a forward");
  gsr_status rs = check_splats(c, sp);
  if (rs != GSR_OK) return rs;
  if (sp->n != c->fwd_n || (int)sp->sh_degree != c->fwd_degree)
    return fail(c, GSR_ERR_INVALID_ARG, "splats differ from the last forward");
  // With no Gaussians the gradient arrays are empty and may be null.
  if (!v_rgba || !grads || (sp->n > 0 && (!grads->v_transforms || !grads->v_sh || !grads->v_raw_opacity)))
    return fail(c, GSR_ERR_INVALID_ARG, "null gradient buffer");
  cudaStream_t st = (cudaStream_t)stream;
  rs = raster_backward_impl(c, v_rgba, st);
  if (rs != GSR_OK) return rs;
  ProjBwdArgs pa{};
  pa.v_tr = grads->v_transforms;
  pa.v_sh = grads->v_sh;
  pa.v_op = grads->v_raw_opacity;
  pa.stats = stats;
  pa.densify_acc = nullptr;
  pa.grad_scale = 1.0f;
  pa.exact = c->cfg.adjoint == GSR_ADJOINT_EXACT;
  pa.hp = c->cfg.fp64_conic;
  prof_mark(c, kStProjectBwd, st);
  GSR_CUDA(c, launch_project_bwd(splats_dev(c, sp), c->fwd_vs, c->cfg.cov_blur, c->b, pa, st, c->num_sms));
  prof_mark(c, kStCount, st);
  return GSR_OK;
}

gsr_status gsr_export(gsr_ctx* c, uint32_t view, int32_t what, void* dst, uint64_t bytes, void* stream) {
  if (!c) return GSR_ERR_INVALID_ARG;
  if (!c->have_fwd) return fail(c, GSR_ERR_NOT_READY, "no forward to export");
  if (view >= c->fwd_views || !dst) return fail(c, GSR_ERR_INVALID_ARG, "bad view or destination");
  cudaStream_t st = (cudaStream_t)stream;
  FwdBufs& b = c->b;
  uint32_t cnt[4];
  GSR_CUDA(c, cudaMemcpyAsync(cnt, b.vcount + view * 4, sizeof(cnt), cudaMemcpyDeviceToHost, st));
  GSR_CUDA(c, cudaStreamSynchronize(st));
  const uint64_t V = cnt[0], I = cnt[1];
  const ViewDesc& d = c->fwd_desc[view];
  const uint64_t P = (uint64_t)d.w * d.h, T = (uint64_t)d.tiles_x * d.tiles_y;
  const void* src = nullptr;
  uint64_t need = 0;
  switch (what) {
    case 0: {
      if (bytes < 8) return fail(c, GSR_ERR_INVALID_ARG, "destination too small");
      uint32_t two[2] = {cnt[0], cnt[2]};
      GSR_CUDA(c, cudaMemcpy(dst, two, 8, cudaMemcpyDefault));
      return GSR_OK;
    }
    case 1: src = slice(b.gid_of_c, b.Vcap, view); need = 4 * V; break;
    case 2: src = slice(b.perm, b.Vcap, view); need = 4 * V; break;
    case 3:
    case 4:
      if (b.pack_bits) {
        // Packed keys: unpacked into the (idle) sort double buffers first.
        uint32_t* tiles = slice(b.key_tmp, std::max(b.Vcap, b.Icap), view);
        uint32_t* idx = slice(b.val_tmp, std::max(b.Vcap, b.Icap), view);
        GSR_CUDA(c, launch_unpack_isects(b, view, (uint32_t)I, tiles, idx, st));
        src = what == 3 ? tiles : idx;
      } else {
        src = what == 3 ? slice(b.isect_key, b.Icap, view) : slice(b.isect_val, b.Icap, view);
      }
      need = 4 * I;
      break;
    case 5: src = slice(b.ranges, 2 * b.Tcap, view); need = 8 * T; break;
    case 6: src = slice(b.tfinal, b.Pcap, view); need = 4 * P; break;
    case 7: src = slice(b.last, b.Pcap, view); need = 4 * P; break;
    case 8: src = slice(b.ncontrib, b.Pcap, view); need = 4 * P; break;
    case 9: src = slice(b.sgrad, b.Vcap * 3, view); need = 48 * V; break;
    case 10: src = slice(b.nvisit, b.Pcap, view); need = 4 * P; break;
    case 11:
      // The slot layout keeps box sizes there; the passing-tile counts are
      // recounted from the sorted intersections.
      if (b.slots) GSR_CUDA(c, launch_count_from_isects(b, view, (uint32_t)V, st));
      src = slice(b.count, b.Vcap, view);
      need = 4 * V;
      break;
    case 12: src = slice(b.hitw, b.Icap, view); need = I; break;
    default: return fail(c, GSR_ERR_INVALID_ARG, "unknown export selector");
  }
  if (bytes < need) return fail(c, GSR_ERR_INVALID_ARG, "destination too small");
  if (need) GSR_CUDA(c, cudaMemcpyAsync(dst, src, need, cudaMemcpyDefault, st));
  GSR_CUDA(c, cudaStreamSynchronize(st));
  return GSR_OK;
}

gsr_status gsr_frames_to_targets(gsr_ctx* c, const uint8_t* frames, const gsr_frame* desc, const gsr_camera* cams,
                                 uint32_t n_views, float* targets, void* stream) {
  if (!c) return GSR_ERR_INVALID_ARG;
  if (n_views == 0) return GSR_OK;
  if (!frames || !desc || !cams || !targets) return fail(c, GSR_ERR_INVALID_ARG, "null frame or target buffer");
  if (n_views > (uint32_t)kMaxViews) return fail(c, GSR_ERR_INVALID_ARG, "at most 64 frames per call");
  std::vector<FrameSpec> spec(n_views);
  for (uint32_t v = 0; v < n_views; ++v) {
    if (desc[v].width == 0 || desc[v].height == 0) return fail(c, GSR_ERR_INVALID_ARG, "empty frame");
    if (cams[v].width == 0 || cams[v].height == 0) return fail(c, GSR_ERR_INVALID_ARG, "empty target view");
    spec[v].src_offset = desc[v].offset;
    spec[v].src_w = desc[v].width;
    spec[v].src_h = desc[v].height;
    spec[v].dst_w = cams[v].width;
    spec[v].dst_h = cams[v].height;
  }
  GSR_CUDA(c, launch_frames_to_targets(frames, spec.data(), n_views, targets, (cudaStream_t)stream));
  return GSR_OK;
}

gsr_status gsr_loss(gsr_ctx* c, const float* pred, const float* target, const gsr_camera* cams, uint32_t n_views,
                    float l1_w, float ssim_w, float* loss, float* v_pred, void* stream) {
  if (!c) return GSR_ERR_INVALID_ARG;
  if (!pred || !target || !loss || !v_pred) return fail(c, GSR_ERR_INVALID_ARG, "null loss buffer");
  std::vector<ViewDesc> desc;
  ViewSet vs;
  gsr_status rs = build_views(c, cams, n_views, desc, vs);
  if (rs != GSR_OK) return rs;
  cudaStream_t st = (cudaStream_t)stream;
  GSR_CUDA(c, launch_set_views(c->d_views, desc.data(), n_views, st));
  GSR_CUDA(c, launch_loss(vs, desc.data(), pred, target, l1_w, ssim_w, loss, v_pred, c->loss_work,
                          c->loss_work_floats, st));
  // The descriptors of the last forward stay valid for its backward.
  if (c->have_fwd) GSR_CUDA(c, launch_set_views(c->d_views, c->fwd_desc.data(), c->fwd_views, st));
  return GSR_OK;
}

static AdamScalars make_scalars(const gsr_lr* lr, int32_t step) {
  AdamScalars s;
  s.lr_pos = lr->position;
  s.lr_rot = lr->rotation;
  s.lr_scale = lr->scale;
  s.lr_color = lr->color;
  s.lr_opac = lr->opacity;
  s.beta1 = lr->beta1;
  s.beta2 = lr->beta2;
  s.eps = lr->eps;
  // engine/optimizer.rs:144-147: 1 - beta^step with f32 powi; the kernels
  // multiply by the f32 reciprocals.
  s.rbc1 = 1.0f / (1.0f - powi_f32(lr->beta1, step));
  s.rbc2 = 1.0f / (1.0f - powi_f32(lr->beta2, step));
  return s;
}

gsr_status gsr_adam_step(gsr_ctx* c, float* transforms, void* sh, float* raw_opacity, uint32_t n, uint32_t sh_degree,
                         const gsr_grads* g, const gsr_adam_state* state, const gsr_lr* lr, int32_t step,
                         void* stream) {
  if (!c) return GSR_ERR_INVALID_ARG;
  if (!g || !state || !lr || step < 1 || sh_degree > 4) return fail(c, GSR_ERR_INVALID_ARG, "bad Adam arguments");
  if (n == 0) return GSR_OK;
  cudaStream_t st = (cudaStream_t)stream;
  AdamArgs a{};
  a.transforms = transforms;
  a.sh = sh;
  a.raw_opac = raw_opacity;
  a.m_tr = state->m_transforms;
  a.v_tr = state->v_transforms;
  a.m_sh = state->m_sh;
  a.v_sh = state->v_sh;
  a.m_op = state->m_opacity;
  a.v_op = state->v_opacity;
  a.scal = c->d_scal;
  GSR_CUDA(c, launch_set_scalars(c->d_scal, make_scalars(lr, step), st));
  GSR_CUDA(c, launch_adam(a, g->v_transforms, g->v_sh, g->v_raw_opacity, n, (int)sh_degree,
                          c->cfg.sh_dtype == GSR_SH_BF16, st, c->num_sms));
  return GSR_OK;
}

gsr_status gsr_accumulate_densify(gsr_ctx* c, const gsr_grads* g, const float* stats, const float* visible, uint32_t n,
                                  uint32_t sh_degree, int32_t use_visible, float* acc, void* stream) {
  if (!c) return GSR_ERR_INVALID_ARG;
  if (!g || !stats || !acc || (use_visible && !visible)) return fail(c, GSR_ERR_INVALID_ARG, "bad densify arguments");
  GSR_CUDA(c, launch_densify(g->v_transforms, stats, g->v_sh, visible, n, (int)sh_degree, use_visible, acc,
                             (cudaStream_t)stream, c->num_sms));
  return GSR_OK;
}

// The step after its forward: loss, raster backward, projection backward
// with the densification statistics, Adam.
static gsr_status train_rest(gsr_ctx* c, const gsr_splats* sp, float* transforms, void* sh, float* raw_opacity,
                             const gsr_adam_state* state, uint32_t n_views, const float* targets,
                             const gsr_train_params* p, float* densify_acc, float* loss, cudaStream_t st) {
  prof_mark(c, kStLoss, st);
  GSR_CUDA(c, launch_loss(c->fwd_vs, c->fwd_desc.data(), c->render, targets, p->l1_weight, p->ssim_weight, loss,
                          c->v_render, c->loss_work, c->loss_work_floats, st));
  const gsr_status rs = raster_backward_impl(c, c->v_render, st);
  if (rs != GSR_OK) return rs;
  AdamArgs a{};
  a.transforms = transforms;
  a.sh = sh;
  a.raw_opac = raw_opacity;
  a.m_tr = state->m_transforms;
  a.v_tr = state->v_transforms;
  a.m_sh = state->m_sh;
  a.v_sh = state->v_sh;
  a.m_op = state->m_opacity;
  a.v_op = state->v_opacity;
  a.scal = c->d_scal;
  ProjBwdArgs pa{};
  pa.v_tr = c->grad_work;
  pa.v_sh = c->grad_work + c->grad_sh_off;
  pa.v_op = c->grad_work + c->grad_op_off;
  pa.densify_acc = densify_acc;
  pa.use_visible = p->use_visible;
  pa.grad_scale = 1.0f / (float)n_views;
  pa.exact = c->cfg.adjoint == GSR_ADJOINT_EXACT;
  pa.hp = c->cfg.fp64_conic;
  prof_mark(c, kStProjectBwd, st);
  GSR_CUDA(c, launch_project_bwd(splats_dev(c, sp), c->fwd_vs, c->cfg.cov_blur, c->b, pa, st, c->num_sms));
  prof_mark(c, kStAdam, st);
  GSR_CUDA(c, launch_adam(a, pa.v_tr, pa.v_sh, pa.v_op, sp->n, (int)sp->sh_degree, c->cfg.sh_dtype == GSR_SH_BF16,
                          st, c->num_sms));
  prof_mark(c, kStCount, st);
  return GSR_OK;
}

// Captures what `body` launches on the capture stream into an executable
// graph and adds its kernel nodes to c->graph_kernels.
extern "C++" template <class Body>
gsr_status capture_graph(gsr_ctx* c, Body body, cudaGraphExec_t* out) {
  if (!c->capture_stream) GSR_CUDA(c, cudaStreamCreateWithFlags(&c->capture_stream, cudaStreamNonBlocking));
  cudaStream_t cs = c->capture_stream;
  cudaGraph_t graph = nullptr;
  GSR_CUDA(c, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  gsr_status rs = body(cs);
  cudaError_t e = cudaStreamEndCapture(cs, &graph);
  if (rs != GSR_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rs;
  }
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
  size_t nn = 0;
  if (cudaGraphGetNodes(graph, nullptr, &nn) == cudaSuccess && nn > 0) {
    std::vector<cudaGraphNode_t> nodes(nn);
    if (cudaGraphGetNodes(graph, nodes.data(), &nn) == cudaSuccess)
      for (size_t i = 0; i < nn; ++i) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++c->graph_kernels;
      }
  }
  e = cudaGraphInstantiate(out, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    *out = nullptr;
    return cuda_fail(c, e, "cudaGraphInstantiate");
  }
  return GSR_OK;
}

static gsr_status train_step_impl(gsr_ctx* c, float* transforms, void* sh, float* raw_opacity, uint32_t n,
                                  uint32_t sh_degree, const gsr_adam_state* state, const gsr_camera* cams,
                                  uint32_t n_views, const float* targets, const gsr_train_params* p,
                                  float* densify_acc, float* loss, int32_t use_graph, cudaEvent_t ready,
                                  cudaStream_t st) {
  if (!c) return GSR_ERR_INVALID_ARG;
  if (!state || !p || !targets || !loss || p->step < 1) return fail(c, GSR_ERR_INVALID_ARG, "bad training arguments");
  gsr_splats sp{transforms, sh, raw_opacity, n, sh_degree};
  GSR_CUDA(c, launch_set_scalars(c->d_scal, make_scalars(&p->lr, p->step), st));
  auto fwd = [&](cudaStream_t s) { return forward_impl(c, &sp, cams, n_views, c->render, nullptr, s); };
  auto rest = [&](cudaStream_t s) {
    return train_rest(c, &sp, transforms, sh, raw_opacity, state, n_views, targets, p, densify_acc, loss, s);
  };
  if (!use_graph) {
    gsr_status rs = fwd(st);
    if (rs != GSR_OK) return rs;
    if (ready) GSR_CUDA(c, cudaStreamWaitEvent(st, ready, 0));
    return rest(st);
  }
  // Graph key: everything baked into the captured launches, and whether the
  // step is split at the event wait.
  const uint8_t split = ready != nullptr;
  std::vector<uint8_t> key;
  auto put = [&](const void* d, size_t sz) {
    const uint8_t* q = static_cast<const uint8_t*>(d);
    key.insert(key.end(), q, q + sz);
  };
  put(&transforms, sizeof(void*));
  put(&sh, sizeof(void*));
  put(&raw_opacity, sizeof(void*));
  put(&n, 4);
  put(&sh_degree, 4);
  put(state, sizeof(*state));
  put(&n_views, 4);
  put(cams, sizeof(gsr_camera) * n_views);
  put(&targets, sizeof(void*));
  put(&densify_acc, sizeof(void*));
  put(&loss, sizeof(void*));
  put(&p->l1_weight, 4);
  put(&p->ssim_weight, 4);
  put(&p->use_visible, 4);
  put(&split, 1);
  if (c->graph_exec == nullptr || key != c->graph_key) {
    for (cudaGraphExec_t* g : {&c->graph_exec, &c->graph_exec_rest})
      if (*g) {
        cudaGraphExecDestroy(*g);
        *g = nullptr;
      }
    c->graph_key.clear();
    std::vector<ViewDesc> desc;
    ViewSet vs;
    gsr_status rs = build_views(c, cams, n_views, desc, vs);
    if (rs != GSR_OK) return rs;
    c->graph_kernels = 0;
    if (split) {
      rs = capture_graph(c, fwd, &c->graph_exec);
      if (rs == GSR_OK) rs = capture_graph(c, rest, &c->graph_exec_rest);
    } else {
      rs = capture_graph(
          c,
          [&](cudaStream_t s) {
            gsr_status r = fwd(s);
            return r != GSR_OK ? r : rest(s);
          },
          &c->graph_exec);
    }
    if (rs != GSR_OK) {
      for (cudaGraphExec_t* g : {&c->graph_exec, &c->graph_exec_rest})
        if (*g) {
          cudaGraphExecDestroy(*g);
          *g = nullptr;
        }
      return rs;
    }
    c->graph_key = key;
  }
  GSR_CUDA(c, cudaGraphLaunch(c->graph_exec, st));
  if (split) {
    GSR_CUDA(c, cudaStreamWaitEvent(st, ready, 0));
    GSR_CUDA(c, cudaGraphLaunch(c->graph_exec_rest, st));
  }
  return GSR_OK;
}

gsr_status gsr_train_step(gsr_ctx* c, float* transforms, void* sh, float* raw_opacity, uint32_t n, uint32_t sh_degree,
                          const gsr_adam_state* state, const gsr_camera* cams, uint32_t n_views, const float* targets,
                          const gsr_train_params* p, float* densify_acc, float* loss, int32_t use_graph,
                          void* stream) {
  return train_step_impl(c, transforms, sh, raw_opacity, n, sh_degree, state, cams, n_views, targets, p, densify_acc,
                         loss, use_graph, nullptr, (cudaStream_t)stream);
}

gsr_status gsr_train_step_after(gsr_ctx* c, float* transforms, void* sh, float* raw_opacity, uint32_t n,
                                uint32_t sh_degree, const gsr_adam_state* state, const gsr_camera* cams,
                                uint32_t n_views, const float* targets, const gsr_train_params* p,
                                float* densify_acc, float* loss, int32_t use_graph, void* targets_ready,
                                void* stream) {
  return train_step_impl(c, transforms, sh, raw_opacity, n, sh_degree, state, cams, n_views, targets, p, densify_acc,
                         loss, use_graph, (cudaEvent_t)targets_ready, (cudaStream_t)stream);
}

gsr_status gsr_profile(gsr_ctx* c, int32_t enable) {
  if (!c) return GSR_ERR_INVALID_ARG;
  c->prof_on = enable != 0;
  c->prof_used = 0;
  return GSR_OK;
}

gsr_status gsr_profile_read(gsr_ctx* c, float* ms_per_stage, int32_t n_stages, void* stream) {
  if (!c || !ms_per_stage || n_stages < (int)kStCount) return fail(c, GSR_ERR_INVALID_ARG, "bad profile buffer");
  GSR_CUDA(c, cudaStreamSynchronize((cudaStream_t)stream));
  for (int i = 0; i < n_stages; ++i) ms_per_stage[i] = 0.f;
  for (size_t i = 0; i + 1 < c->prof_used; ++i) {
    float ms = 0.f;
    GSR_CUDA(c, cudaEventElapsedTime(&ms, c->prof_ev[i], c->prof_ev[i + 1]));
    const int st = c->prof_stage[i];
    if (st >= 0 && st < (int)kStCount) ms_per_stage[st] += ms;
  }
  c->prof_used = 0;
  return GSR_OK;
}

int32_t gsr_graph_kernel_count(const gsr_ctx* c) { return c ? c->graph_kernels : 0; }

gsr_status gsr_selftest_wait_timeout(gsr_ctx* c, uint32_t max_polls, void* stream) {
  if (!c) return GSR_ERR_INVALID_ARG;
  if (max_polls < 1 || max_polls > kMaxPolls) return fail(c, GSR_ERR_INVALID_ARG, "max_polls outside 1..2^22");
  if (c->s.lb_states_words < 2) return fail(c, GSR_ERR_INVALID_ARG, "no look-back scratch");
  // The probe overwrites look-back states 0 and 1; every look-back launch
  // tags its states with a fresh epoch, so later launches are unaffected.
  GSR_CUDA(c, launch_lookback_timeout_probe(c->s.lb_states, c->s.status, max_polls, c->b.vcount + 3,
                                            (cudaStream_t)stream));
  return gsr_sync_status(c, stream, nullptr);
}

gsr_status gsr_topology_apply(gsr_ctx* c, const gsr_splats* sp, const gsr_topo_row* rows, uint32_t m,
                              const gsr_topo_params* params, float* dst_transforms, void* dst_sh,
                              float* dst_raw_opacity, void* stream) {
  if (!c) return GSR_ERR_INVALID_ARG;
  gsr_status rs = check_splats(c, sp);
  if (rs != GSR_OK) return rs;
  if (m > 0 && (!rows || !params || !dst_transforms || !dst_sh || !dst_raw_opacity))
    return fail(c, GSR_ERR_INVALID_ARG, "null topology buffer");
  if (m == 0) return GSR_OK;
  static_assert(sizeof(gsr_topo_row) == sizeof(TopoRow), "plan row layout");
  TopoParams p{};
  p.has_decay = params->has_refine_decay;
  p.scale_decay = params->scale_decay;
  p.opacity_decay = params->opacity_decay;
  p.train_t = params->train_t;
  p.opacity_reset = params->opacity_reset;
  p.reset_cap = params->opacity_reset_cap;
  GSR_CUDA(c, launch_topology(splats_dev(c, sp), reinterpret_cast<const TopoRow*>(rows), m, p, dst_transforms, dst_sh,
                              dst_raw_opacity, c->s.status, (cudaStream_t)stream, c->num_sms));
  return GSR_OK;
}

gsr_status gsr_autotune(const gsr_config* base, const gsr_splats* sp, const gsr_camera* cams, uint32_t n_views,
                        int32_t reps, gsr_tune_result* out, void* stream) {
  if (!base || !sp || !cams || !out || n_views == 0 || reps < 1 || sp->sh_degree > 4) return GSR_ERR_INVALID_ARG;
  memset(out, 0, sizeof(*out));
  cudaStream_t st = (cudaStream_t)stream;
  uint64_t pix = 0;
  for (uint32_t v = 0; v < n_views; ++v) pix += (uint64_t)cams[v].width * cams[v].height;
  const uint64_t n = sp->n, K = (uint64_t)(sp->sh_degree + 1) * (sp->sh_degree + 1);
  float *rgba = nullptr, *vrgba = nullptr, *grads = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  auto release = [&]() {
    if (rgba) cudaFree(rgba);
    if (vrgba) cudaFree(vrgba);
    if (grads) cudaFree(grads);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  };
  if (cudaMalloc(&rgba, sizeof(float) * 4 * std::max<uint64_t>(pix, 1)) != cudaSuccess ||
      cudaMalloc(&vrgba, sizeof(float) * 4 * std::max<uint64_t>(pix, 1)) != cudaSuccess ||
      cudaMalloc(&grads, sizeof(float) * std::max<uint64_t>(n * (11 + 3 * K), 1)) != cudaSuccess ||
      cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    release();
    return GSR_ERR_OOM;
  }
  // A fixed upstream gradient (every float 0x3f3f3f3f, about 0.75): the work
  // of the backward does not depend on its values.
  if (cudaMemsetAsync(vrgba, 0x3f, sizeof(float) * 4 * pix, st) != cudaSuccess) {
    release();
    return GSR_ERR_CUDA;
  }
  const gsr_grads g{grads, grads + n * 10, grads + n * (10 + 3 * K)};
  static const uint32_t kShapes[3][2] = {{16, 16}, {8, 8}, {32, 8}};
  static const uint32_t kBatches[3] = {64, 128, 256};
  float best = -1.f;
  gsr_status first_err = GSR_OK;
  for (int si = 0; si < 3; ++si) {
    for (int bi = 0; bi < 3; ++bi) {
      gsr_tune_candidate& cd = out->candidates[si * 3 + bi];
      cd.tile_w = kShapes[si][0];
      cd.tile_h = kShapes[si][1];
      cd.batch = kBatches[bi];
      cd.ms_per_view = -1.f;
      gsr_config cfg = *base;
      cfg.tile_w = cd.tile_w;
      cfg.tile_h = cd.tile_h;
      cfg.batch = cd.batch;
      if (cfg.max_views < n_views) cfg.max_views = n_views;
      gsr_ctx* c = nullptr;
      gsr_status rs = gsr_create(&cfg, &c);
      auto once = [&]() -> gsr_status {
        gsr_status r = gsr_render_forward(c, sp, cams, n_views, rgba, nullptr, stream);
        return r != GSR_OK ? r : gsr_render_backward(c, sp, vrgba, &g, nullptr, stream);
      };
      uint64_t req = 0;
      if (rs == GSR_OK) rs = once();
      if (rs == GSR_OK) rs = gsr_sync_status(c, stream, &req);
      if (rs == GSR_ERR_CAPACITY) {
        // Smaller tiles duplicate more keys: grow the capacity once.
        rs = gsr_reserve_isects(c, std::min<uint64_t>(req + req / 8 + 4096, (1ull << 30) - 1));
        if (rs == GSR_OK) rs = once();
        if (rs == GSR_OK) rs = gsr_sync_status(c, stream, &req);
      }
      if (rs == GSR_OK) {
        cudaEventRecord(e0, st);
        for (int r = 0; r < reps && rs == GSR_OK; ++r) rs = once();
        cudaEventRecord(e1, st);
        if (rs == GSR_OK) rs = gsr_sync_status(c, stream, &req);
        float ms = 0.f;
        if (rs == GSR_OK && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) {
          cd.ms_per_view = ms / (float)reps / (float)n_views;
          if (best < 0.f || cd.ms_per_view < best) {
            best = cd.ms_per_view;
            out->tile_w = cd.tile_w;
            out->tile_h = cd.tile_h;
            out->batch = cd.batch;
            out->ms_per_view = best;
          }
        }
      }
      cd.status = rs;
      if (rs != GSR_OK && first_err == GSR_OK) first_err = rs;
      if (c) gsr_destroy(c);
    }
  }
  release();
  if (best < 0.f) return first_err != GSR_OK ? first_err : GSR_ERR_CUDA;
  return GSR_OK;
}

}  // extern "C"
