/* gsr.h — C ABI of the sm_100a differentiable Gaussian-splatting rasterizer.
 *
 * This is the drop-in boundary for RustGS's training render op. Each entry
 * point names the reference interface it replaces (paths relative to the
 * RustScan repository). A Rust backend binds these functions through a thin
 * FFI crate; the reference's nine burn Backend extension traits collapse onto
 * gsr_render_forward / gsr_render_backward plus the two primitives.
 *
 * Conventions
 *  - All tensor arguments are device pointers (CUDA global memory) in the
 *    RustGS layouts: transforms [N,10] f32 = position xyz + quaternion wxyz
 *    + log-scale xyz; sh [N,K,3] (K = (degree+1)^2) f32 or bf16; raw
 *    opacity [N] f32 logits (RustGS/src/training/engine/splats.rs:7-18).
 *  - Images are [H,W,4] f32 RGBA, row-major, one view after another.
 *  - Streams are cudaStream_t passed as void*. Calls only enqueue work; only
 *    gsr_sync_status, gsr_export, gsr_profile_read and gsr_reserve_isects
 *    synchronise the host, as their comments say.
 *  - The caller owns every parameter, gradient and image buffer. The
 *    context owns all scratch (keys, ranges, saved forward state).
 *  - Errors are returned as gsr_status; nothing aborts or panics across the
 *    ABI. gsr_last_error() gives a human-readable message.
 *  - One context serves one stream at a time.
 */
#ifndef GSR_H
#define GSR_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GSR_API __attribute__((visibility("default")))
#else
#define GSR_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gsr_status {
  GSR_OK = 0,
  GSR_ERR_INVALID_ARG = 1, /* bad pointer, size or configuration */
  GSR_ERR_OOM = 2,         /* device allocation failed */
  GSR_ERR_CAPACITY = 3,    /* intersection capacity exceeded; see gsr_sync_status */
  GSR_ERR_CUDA = 4,        /* a CUDA call failed */
  GSR_ERR_TIMEOUT = 5,     /* a bounded device-side wait gave up */
  GSR_ERR_NOT_READY = 6    /* backward without a matching forward */
} gsr_status;

typedef struct gsr_ctx gsr_ctx;

enum { GSR_SH_F32 = 0, GSR_SH_BF16 = 1 };
enum { GSR_ADJOINT_EXACT = 0, GSR_ADJOINT_REFERENCE = 1 };
/* Raster work scheduling. Work items are the (view, tile) pairs of a launch.
 * PERSISTENT: as many CTAs as the GPU holds at once take items from a queue
 * ordered by decreasing estimated cost (the forward by list length, the
 * backward by the list entries up to the tile's last contributor, which the
 * forward records), so the longest tiles start first and the launch ends
 * without a tail of long tiles. GRID: one CTA per item in view and tile
 * order, scheduled by the hardware. DEFAULT: the backward persistent, the
 * forward as a grid (the forward's cost, its entries up to saturation, is
 * not known before it runs). The results are the same; with float atomics
 * (deterministic = 0) the gradient sums may differ in the last bits. */
enum { GSR_SCHEDULE_DEFAULT = 0, GSR_SCHEDULE_PERSISTENT = 1, GSR_SCHEDULE_GRID = 2 };

/* Context configuration. Replaces the rasterizer fields of RustGS's
 * TrainingConfig (RustGS/src/training/config.rs:7, raster_cov_blur) and the
 * fixed TILE_WIDTH of RustGS/src/training/forward/mod.rs:25-26. Zero fields
 * take the defaults noted. */
typedef struct gsr_config {
  float cov_blur;          /* screen-space covariance blur in px^2 (0.3) */
  float background[3];     /* background colour (0,0,0) */
  uint32_t tile_w, tile_h; /* tile shape: 16x16 (default), 8x8 or 32x8 */
  uint32_t batch;          /* Gaussians staged in shared memory per raster batch: 64, 128 or 256
                              (rounded up; 0: tuned defaults, 128 forward / 64 backward; the
                              16x16 backward always stages 64) */
  int32_t sh_dtype;        /* GSR_SH_F32 or GSR_SH_BF16 storage of SH coefficients */
  int32_t adjoint;         /* GSR_ADJOINT_EXACT (default) or GSR_ADJOINT_REFERENCE */
  int32_t deterministic;   /* 1: fixed-order gradient reduction, bitwise reruns */
  int32_t fp64_conic;      /* 1: 2x2 covariance inversion in FP64 */
  uint64_t max_splats;     /* capacity in Gaussians */
  uint32_t max_views;      /* views per forward (1) */
  uint32_t schedule;       /* GSR_SCHEDULE_*: raster work scheduling */
  uint64_t max_pixels;     /* capacity in pixels per view */
  uint64_t max_isects;     /* tile intersections per view (0: 16 * max_splats, at least 2^20) */
} gsr_config;

/* Pinhole camera. viewmat is the column-major world->camera matrix
 * (GaussianCamera::view_matrix, RustGS/src/core/camera.rs:30-32); campos is
 * the world-space camera centre (GaussianCamera::position, :34-37). +Z is
 * forward, +Y down, pixel centres at integer + 0.5. */
typedef struct gsr_camera {
  float viewmat[16];
  float fx, fy, cx, cy;
  uint32_t width, height;
  float campos[3];
  float _pad;
} gsr_camera;

/* Gaussian parameters (DeviceSplats, RustGS/src/training/engine/splats.rs:13-18). */
typedef struct gsr_splats {
  const float* transforms; /* [n,10] */
  const void* sh;          /* [n,K,3] f32 or bf16 per gsr_config.sh_dtype */
  const float* raw_opacity;/* [n] */
  uint32_t n;
  uint32_t sh_degree;      /* 0..4 */
} gsr_splats;

/* Gradients, same layouts as the parameters (f32). */
typedef struct gsr_grads {
  float* v_transforms;  /* [n,10] */
  float* v_sh;          /* [n,K,3] */
  float* v_raw_opacity; /* [n] */
} gsr_grads;

/* ---- context ------------------------------------------------------------ */
GSR_API gsr_status gsr_create(const gsr_config* cfg, gsr_ctx** out);
GSR_API void gsr_destroy(gsr_ctx* ctx);
GSR_API const char* gsr_last_error(const gsr_ctx* ctx);
GSR_API const char* gsr_version(void);

/* Synchronises the stream, then reports device-side conditions of the work
 * enqueued so far: GSR_ERR_CAPACITY with *required set to the intersection
 * capacity that did not fit, GSR_ERR_TIMEOUT if a bounded wait gave up.
 * Clears the conditions. Host-synchronising. The capacity counts the
 * binning's slots: the intersections themselves, or, when the tile id and
 * the compact index pack into one 32-bit key with a tile id to spare (the
 * common case, no counting pass), every tile of each visible Gaussian's
 * tile box. */
GSR_API gsr_status gsr_sync_status(gsr_ctx* ctx, void* stream, uint64_t* required);

/* Grows the per-view intersection capacity (frees and reallocates scratch;
 * call between steps). */
GSR_API gsr_status gsr_reserve_isects(gsr_ctx* ctx, uint64_t max_isects);

/* ---- primitives (RustGS/src/training/gpu_primitives) --------------------- */
/* Inclusive scan of n u32 values.
 * Replaces PrefixSumBackend::prefix_sum_u32_primitive
 * (RustGS/src/training/gpu_primitives/prefix_sum.rs:41-45). in and out may
 * not alias. n <= 2^30. */
GSR_API gsr_status gsr_prefix_sum_u32(gsr_ctx* ctx, const uint32_t* in, uint32_t* out, uint32_t n, void* stream);

/* Inclusive scan of n u32 values that allocates no device memory and needs no
 * context. No counterpart in the reference: it exists for callers that must
 * not have a library allocate on their behalf, such as host frameworks that
 * own the whole device memory budget through their own pool (an allocation
 * outside it breaks their accounting or fails mid-run) and deployments that
 * fix their memory use at start-up.
 * Limits and behaviour:
 *  - n <= 16,777,216 (2^24); larger n returns GSR_ERR_INVALID_ARG.
 *  - Scratch is a 64 KiB array compiled into libgsr (a file-scope __device__
 *    variable) that every GPU loading the library keeps until process exit.
 *  - The first call on each device looks up that array's device address
 *    (cudaGetSymbolAddress) with the device current; make that first call
 *    before any stream capture. The address is cached with the ID of the
 *    context it was found in and looked up again when the calling thread's
 *    current context differs (after cudaDeviceReset, or under a context
 *    other than the device's primary one); make the first call in each new
 *    context before any stream capture as well.
 *  - All calls on a device share the one array: the look-back states, the
 *    launch-epoch control block and the status words that each call clears
 *    first. Calls whose work overlaps on the GPU (different streams, or
 *    threads) race on all of them and give wrong results. Serialise them,
 *    e.g. on one stream.
 *  - It only enqueues work; a device-side wait that gives up cannot be
 *    reported here (results are then wrong but the call still finishes).
 * in and out are device pointers and may not alias. */
GSR_API gsr_status gsr_prefix_sum_u32_noalloc(const uint32_t* in, uint32_t* out, uint32_t n, void* stream);

/* Stable ascending sort of (key, value) pairs; equal keys keep input order.
 * Replaces RadixSortBackend::radix_sort_by_key_u32_primitive
 * (RustGS/src/training/gpu_primitives/radix_sort.rs:48-53). Inputs are not
 * modified; outputs must not alias inputs. n <= 2^30. */
GSR_API gsr_status gsr_radix_sort_by_key_u32(gsr_ctx* ctx, const uint32_t* keys_in, const uint32_t* vals_in,
                                     uint32_t* keys_out, uint32_t* vals_out, uint32_t n, void* stream);

/* ---- render op ------------------------------------------------------------ */
/* Forward render of n_views views: projection + SH, tile binning, depth and
 * tile sorts, tile ranges and front-to-back blending, all enqueued without a
 * host synchronisation. out_rgba receives the views' [H,W,4] images one
 * after another; out_visible (nullable) receives [n_views, n] flags (1 if the
 * Gaussian contributed to a pixel). The context keeps the state the backward
 * needs until the next forward.
 * Replaces render_forward (RustGS/src/training/forward/mod.rs:156-294) and,
 * below it, ProjectionBackend (projection.rs:44-50), SortingBackend
 * (sorting.rs:8-12), ProjectVisibleBackend (project_visible.rs:36-45),
 * TileMappingBackend (tile_mapping.rs:82-95) and RasterizeBackend
 * (rasterize.rs:48-59). */
GSR_API gsr_status gsr_render_forward(gsr_ctx* ctx, const gsr_splats* splats, const gsr_camera* cams, uint32_t n_views,
                              float* out_rgba, float* out_visible, void* stream);

/* Backward of the last forward for upstream image gradients v_rgba (same
 * layout as out_rgba). Writes the parameter gradients of the sum over views
 * (rows of Gaussians no view sees are zero) and, if stats is not NULL, the
 * [n_views, n, 7] densification statistics (project_backwards.wgsl:33-36, 105-108).
 * With n == 0 the gradient arrays are empty and may be NULL.
 * Replaces RenderBackward::backward (RustGS/src/training/backward/autodiff.rs:82-142)
 * and, below it, RasterizeBwdBackend (rasterize_bwd.rs:41-54) and
 * ProjectBwdBackend (project_bwd.rs:44-52). */
GSR_API gsr_status gsr_render_backward(gsr_ctx* ctx, const gsr_splats* splats, const float* v_rgba, const gsr_grads* grads,
                               float* stats, void* stream);

/* Copies internal state of view `view` of the last forward to a device or
 * host buffer for inspection (tests, tools). `what` selects:
 *  0 counts (u32 x2: visible, intersections)          [host-synchronising]
 *  1 visible global ids in compact order (u32 x V)
 *  2 depth order: compact index per rank (u32 x V)
 *  3 sorted intersection tile ids (u32 x I)
 *  4 sorted intersection compact indices (u32 x I)
 *  5 tile ranges (u32 x 2T)
 *  6 per-pixel final transmittance (f32 x H*W)
 *  7 per-pixel last contributor list index + 1 (u32 x H*W, 0: none)
 *  8 per-pixel contributor counts (u32 x H*W)
 *  9 per-Gaussian screen-space gradient sums of the last backward (f32 x 12V)
 * 10 per-pixel list entries evaluated (u32 x H*W)
 * 11 per-Gaussian tile counts in compact order (u32 x V)
 * 12 per-intersection 8x8 pixel blocks of its tile (bit x + (y * tile_w / 8),
 *    blocks row-major) holding a pixel that took the Gaussian (u8 x I; defined
 *    for entries before the tile's largest last-contributor index)
 * `bytes` is the destination size; the call fails if it is too small. */
GSR_API gsr_status gsr_export(gsr_ctx* ctx, uint32_t view, int32_t what, void* dst, uint64_t bytes, void* stream);

/* ---- training targets from 8-bit frames ----------------------------------- */
/* One decoded colour frame: width x height RGB bytes (row-major, 3 bytes a
 * pixel) at byte `offset` of a frame buffer. */
typedef struct gsr_frame {
  uint64_t offset;
  uint32_t width, height;
} gsr_frame;

/* Converts n_views (at most 64) decoded 8-bit RGB frames into the targets
 * gsr_loss and gsr_train_step read: per view [H,W,3] f32 with W, H from
 * cams[v], views packed one after another. Replaces the host-side
 * resize_rgb_u8_to_f32 (RustGS/src/training/data/frame_targets.rs:44-62)
 * before the per-step f32 upload (engine/trainer.rs:94-107, 265-268): the
 * caller uploads the bytes (a quarter of the f32 volume) and the conversion
 * runs on the device. A frame of the camera's size maps each byte b to
 * b / 255; any other size is box-averaged with the reference's bounds
 * (output (x, y) averages source columns [x*sw/dw, max((x+1)*sw/dw,
 * x*sw/dw + 1)) and the same rows, clamped to the frame) and summation
 * order, so the results equal the reference's floats. frames and targets
 * are device pointers; desc and cams host arrays. Enqueue only. */
GSR_API gsr_status gsr_frames_to_targets(gsr_ctx* ctx, const uint8_t* frames, const gsr_frame* desc,
                                         const gsr_camera* cams, uint32_t n_views, float* targets, void* stream);

/* ---- loss (RustGS/src/training/engine/loss.rs:112-142) -------------------- */
/* l1_w * mean|pred - target| + ssim_w * (1 - mean SSIM) with an 11-tap
 * sigma-1.5 Gaussian window, replicate padding and C1 = 0.01^2,
 * C2 = 0.03^2, for n_views images. pred is RGBA [H,W,4] per view (the render
 * output), target RGB [H,W,3] per view. Writes loss[n_views] and the
 * gradient v_pred in RGBA layout (alpha gradient 0). Replaces
 * combined_loss_with_kernel and its burn autodiff backward with the default
 * (non-robust, unmasked) settings. */
GSR_API gsr_status gsr_loss(gsr_ctx* ctx, const float* pred, const float* target, const gsr_camera* cams, uint32_t n_views,
                    float l1_w, float ssim_w, float* loss, float* v_pred, void* stream);

/* ---- optimizer (RustGS/src/training/engine/optimizer.rs:45-163) ----------- */
typedef struct gsr_adam_state {
  float* m_transforms; float* v_transforms; /* [n,10] */
  float* m_sh; float* v_sh;                 /* [n,K,3] */
  float* m_opacity; float* v_opacity;       /* [n] */
} gsr_adam_state;

typedef struct gsr_lr {
  float position, rotation, scale, color, opacity; /* learning rates per column group */
  float beta1, beta2, eps;                         /* 0.9, 0.999, 1e-8 */
} gsr_lr;

/* Bias-corrected Adam with per-column learning rates on all three parameter
 * groups; step is the 1-based step count shared by the groups.
 * Parameters are updated in place (the SH storage dtype is honoured).
 * Replaces AdamScaled::step_device_splats (optimizer.rs:80-120). */
GSR_API gsr_status gsr_adam_step(gsr_ctx* ctx, float* transforms, void* sh, float* raw_opacity, uint32_t n,
                         uint32_t sh_degree, const gsr_grads* grads, const gsr_adam_state* state, const gsr_lr* lr,
                         int32_t step, void* stream);

/* ---- densification statistics (RustGS/src/training/engine/trainer.rs:651-728) */
/* acc holds 9 arrays of n floats: grad_2d, screen_grad_2d, abs_grad_2d,
 * abs_pixel_grad_2d, pixel_coverage, camera_depth, grad_color,
 * num_observations, visible_observations. visible may be NULL when
 * use_visible is 0. Replaces WgpuTrainer::accumulate_gradients. */
GSR_API gsr_status gsr_accumulate_densify(gsr_ctx* ctx, const gsr_grads* grads, const float* stats, const float* visible,
                                  uint32_t n, uint32_t sh_degree, int32_t use_visible, float* acc, void* stream);

/* ---- training step (RustGS/src/training/engine/trainer.rs:253-440) ------- */
typedef struct gsr_train_params {
  gsr_lr lr;
  int32_t step;        /* 1-based Adam step */
  float l1_weight;     /* 0.8 */
  float ssim_weight;   /* 0.2 */
  int32_t use_visible; /* densification visible_observations from render visibility */
} gsr_train_params;

/* One training step over n_views views: forward, loss, backward, the
 * densification accumulators (per view) and one fused Adam update of all
 * parameters with the gradient of the mean loss over the views. targets are
 * RGB [H,W,3] per view on the device; loss[n_views] receives the per-view
 * losses (device). With use_graph != 0 the step is recorded into a CUDA graph
 * on first use for this (splats, cameras, sizes) signature and replayed
 * afterwards. */
GSR_API gsr_status gsr_train_step(gsr_ctx* ctx, float* transforms, void* sh, float* raw_opacity, uint32_t n,
                          uint32_t sh_degree, const gsr_adam_state* state, const gsr_camera* cams, uint32_t n_views,
                          const float* targets, const gsr_train_params* params, float* densify_acc, float* loss,
                          int32_t use_graph, void* stream);

/* gsr_train_step whose loss waits on targets_ready (a cudaEvent_t, or NULL
 * for no wait): the forward is launched first and the stream waits on the
 * event's latest record before the loss reads targets, so that the targets'
 * upload and conversion on another stream overlap the forward (the
 * reference uploads them before its forward, engine/trainer.rs:265-268).
 * With use_graph != 0 and an event, the forward and the rest are recorded
 * as two graphs with the wait between their launches. */
GSR_API gsr_status gsr_train_step_after(gsr_ctx* ctx, float* transforms, void* sh, float* raw_opacity, uint32_t n,
                                uint32_t sh_degree, const gsr_adam_state* state, const gsr_camera* cams,
                                uint32_t n_views, const float* targets, const gsr_train_params* params,
                                float* densify_acc, float* loss, int32_t use_graph, void* targets_ready,
                                void* stream);

/* ---- topology (RustGS/src/training/topology/apply.rs) -------------------- */
/* A topology plan row: the output splat copies splat `source`, as is
 * (GSR_TOPO_EXISTING) or as one half of a split, moved by -offset
 * (GSR_TOPO_REFINE_EXISTING) or +offset (GSR_TOPO_REFINE_NEW), where offset
 * is the source's scale times sample_scalar rotated by its quaternion; split
 * halves have their largest scale axis halved and opacity 1 - sqrt(1 - o).
 * Mirrors TopologyPlanRow (topology/mod.rs:831-843). */
enum { GSR_TOPO_EXISTING = 0, GSR_TOPO_REFINE_EXISTING = 1, GSR_TOPO_REFINE_NEW = 2 };
typedef struct gsr_topo_row {
  uint32_t source;
  int32_t kind;
  float sample_scalar;
  uint32_t _pad;
} gsr_topo_row;
/* Plan-wide options (TopologyMutationPlan::refine_decay and the opacity-reset
 * aftermath; topology/mod.rs:776-780, 863-870). */
typedef struct gsr_topo_params {
  int32_t has_refine_decay;
  float scale_decay, opacity_decay, train_t;
  int32_t opacity_reset;
  float opacity_reset_cap; /* 0.01 in the reference (LITEGS_OPACITY_RESET_CAP) */
} gsr_topo_params;

/* Builds the mutated splat set on the device: output row i from rows[i]
 * (rows in device memory, m of them; pruning is a source that no row
 * names). Writes dst_transforms [m,10], dst_sh [m,K,3] (same storage type as
 * src) and dst_raw_opacity [m]; the destinations may not alias the source.
 * Replaces apply_mutations (topology/apply.rs:10-27) with its host round
 * trip (topology/bridge.rs:25-146). A row whose source is out of range is
 * reported by gsr_sync_status as GSR_ERR_INVALID_ARG. Adam moments and the
 * densification accumulators are the caller's to reset, as the reference
 * resets them on topology changes (engine/trainer.rs:851-853). */
GSR_API gsr_status gsr_topology_apply(gsr_ctx* ctx, const gsr_splats* src, const gsr_topo_row* rows, uint32_t m,
                                      const gsr_topo_params* params, float* dst_transforms, void* dst_sh,
                                      float* dst_raw_opacity, void* stream);

/* ---- autotuner (no counterpart in the reference) ------------------------ */
/* Candidates: tile shapes 16x16, 8x8, 32x8 times raster batches 64, 128,
 * 256 (9 entries, in that order). */
enum { GSR_TUNE_CANDIDATES = 9 };
typedef struct gsr_tune_candidate {
  uint32_t tile_w, tile_h, batch;
  int32_t status;   /* GSR_OK, or why the candidate could not run */
  float ms_per_view; /* forward + backward, mean over the timed repetitions */
  uint32_t _pad;
} gsr_tune_candidate;
typedef struct gsr_tune_result {
  uint32_t tile_w, tile_h, batch; /* the fastest candidate */
  float ms_per_view;
  gsr_tune_candidate candidates[GSR_TUNE_CANDIDATES];
} gsr_tune_result;

/* Times forward + backward (a fixed upstream gradient) of the given splats
 * and views for every candidate, each in a temporary context built from
 * *base with that tile shape and batch (and max_isects grown as needed), and
 * reports the fastest; base->tile_w/tile_h/batch are ignored. reps >= 1 timed
 * repetitions after one warm-up. Allocates and frees device memory and
 * synchronises the stream: call it once per scene/resolution mix, outside
 * any stream capture, then create the working context with the result. */
GSR_API gsr_status gsr_autotune(const gsr_config* base, const gsr_splats* splats, const gsr_camera* cams,
                                uint32_t n_views, int32_t reps, gsr_tune_result* out, void* stream);

/* ---- instrumentation (no counterpart in the reference) ------------------ */
/* Stage timing: when enabled, the context records CUDA events on the stream
 * between pipeline stages of the calls that follow (never inside a graph
 * capture). gsr_profile_read synchronises the stream and writes the
 * milliseconds per stage, summed since the last read, in this order:
 * project, depth_sort, offsets, emit, tile_sort, ranges, raster_fwd,
 * visible, loss, raster_bwd, reduce, project_bwd, adam (13 entries). */
enum { GSR_PROFILE_STAGES = 13 };
GSR_API gsr_status gsr_profile(gsr_ctx* ctx, int32_t enable);
GSR_API gsr_status gsr_profile_read(gsr_ctx* ctx, float* ms_per_stage, int32_t n_stages, void* stream);
/* Self-test of the bounded device waits (no counterpart in the reference):
 * runs one look-back whose predecessor never publishes, which must give up
 * after max_polls polls (1..2^22). Returns GSR_ERR_TIMEOUT when the wait gave
 * up as it should (the context stays usable), GSR_OK if it did not.
 * Synchronises the stream. */
GSR_API gsr_status gsr_selftest_wait_timeout(gsr_ctx* ctx, uint32_t max_polls, void* stream);
/* Kernel nodes in the captured training-step graph (0 before a capture). */
GSR_API int32_t gsr_graph_kernel_count(const gsr_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* GSR_H */
