// CPU ORACLE — test infrastructure only, never the product path.
//
// A C++ restatement of RustGS's differentiable Gaussian-splatting rasterizer
// (RustGS/src/training/shaders/*.wgsl and the Rust orchestration around
// them), instantiated in float (the parity oracle) and double (the FP64
// reference for image/gradient error reports and finite differences). Only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg call it.
//
// The per-Gaussian EWA formulas come from the shared header gsr_math.h (the
// same expression trees the CUDA kernels evaluate); everything else here —
// culling and compaction order, depth and tile ordering, intersection
// emission, tile ranges, the blend loops, both backward walks, the loss, Adam
// and the densification statistics — is restated in plain loops, each block
// citing the reference lines it follows.
//
// Parity pins: the sort/scan primitives follow the reference's own known
// answer tests (gpu_primitives/radix_sort/tests.rs, prefix_sum/tests.rs);
// images and gradients are unpinned by the reference (no test fixes their
// values) and are checked against the FP64 instantiation and central finite
// differences instead.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include "../rustscan_b200/csrc/gsr_math.h"

using namespace gsr;

extern "C" {
// Layout shared with include/gsr.h's gsr_camera.
typedef struct {
  float viewmat[16];  // column-major world->camera
  float fx, fy, cx, cy;
  uint32_t width, height;
  float campos[3];  // camera centre in world space
  float _pad;
} orc_camera;
}

namespace {

template <class F> Cam<F> make_cam(const orc_camera& c) {
  Cam<F> k;
  for (int col = 0; col < 3; ++col)
    for (int row = 0; row < 3; ++row) k.rot.m[col][row] = F(c.viewmat[col * 4 + row]);
  k.trans.x = F(c.viewmat[12]);
  k.trans.y = F(c.viewmat[13]);
  k.trans.z = F(c.viewmat[14]);
  k.focal.x = F(c.fx);
  k.focal.y = F(c.fy);
  k.pc.x = F(c.cx);
  k.pc.y = F(c.cy);
  k.w = c.width;
  k.h = c.height;
  k.campos.x = F(c.campos[0]);
  k.campos.y = F(c.campos[1]);
  k.campos.z = F(c.campos[2]);
  return k;
}

template <class F> struct Splats {
  int n = 0, degree = 0, K = 1;
  const F* transforms = nullptr;  // [n,10]
  const F* sh = nullptr;          // [n,K,3]
  const F* raw_opac = nullptr;    // [n]
};

template <class F> struct FwdState {
  // inputs kept for the backward
  Splats<F> sp;
  orc_camera camera;
  Cam<F> cam;
  F cov_blur;
  bool hp = false;  // FP64 2D-covariance compensation and inversion
  F bg[3];
  TileShape ts;
  uint32_t tiles_x = 0, tiles_y = 0;
  // projection, in compact (global-id) order
  std::vector<int32_t> gid_of_c;
  std::vector<Projected<F>> proj;
  std::vector<V3<F>> rgb;
  std::vector<uint32_t> count;
  // depth order: order[r] = compact index of rank r
  std::vector<int32_t> order;
  std::vector<uint32_t> isect_tile, isect_c;  // sorted by (tile, depth, gid)
  std::vector<uint32_t> ranges;               // [2T]
  // per pixel
  std::vector<F> image;  // [H,W,4]
  std::vector<F> tfinal;
  std::vector<uint32_t> last;      // list index of the last contributor + 1 (0: none)
  std::vector<uint32_t> ncontrib;  // number of contributors
  std::vector<uint32_t> nvisit;    // list entries evaluated before termination
  std::vector<F> visible;          // [n]
  // per intersection: bit (lx/8) + (ly/8)*(tile_w/8) for each 8x8 pixel block
  // of the tile holding a pixel that took the Gaussian (test inspection)
  std::vector<uint32_t> hit_blocks;
};

// ---------------------------------------------------------------------------
// Forward: project_forward.wgsl + project_visible.wgsl (projection, computed
// once per Gaussian), sorting.rs:34-61 (depth order, ties by global id),
// prefix_sum.wgsl (inclusive scan), map_gaussian_to_intersects.wgsl (emission
// with the count pass's tile test), tile_mapping.rs:206-215 (stable tile
// sort), get_tile_offsets.wgsl and rasterize.wgsl.
// ---------------------------------------------------------------------------
template <class F> void forward(FwdState<F>& st) {
  const Splats<F>& sp = st.sp;
  const Cam<F>& cam = st.cam;
  const uint32_t W = cam.w, H = cam.h;
  st.tiles_x = (W + st.ts.tw - 1) / st.ts.tw;
  st.tiles_y = (H + st.ts.th - 1) / st.ts.th;
  const uint32_t T = st.tiles_x * st.tiles_y;

  // project_forward.wgsl:13-96, one Gaussian at a time.
  std::vector<Projected<F>> all(sp.n);
  std::vector<uint32_t> cnt(sp.n, 0);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int g = 0; g < sp.n; ++g) {
    const F* t = sp.transforms + (size_t)g * 10;
    V3<F> mean{t[0], t[1], t[2]};
    V4<F> q{t[3], t[4], t[5], t[6]};
    V3<F> ls{t[7], t[8], t[9]};
    all[g] = project_gaussian(cam, mean, q, ls, sp.raw_opac[g], st.cov_blur, st.ts, st.tiles_x, st.tiles_y, st.hp);
    if (all[g].visible) cnt[g] = count_tiles(all[g], st.ts);
  }
  // Compaction in global-id order (replaces the atomic compaction of
  // project_forward.wgsl:94-96, whose order is nondeterministic).
  st.gid_of_c.clear();
  for (int g = 0; g < sp.n; ++g)
    if (all[g].visible) st.gid_of_c.push_back(g);
  const size_t V = st.gid_of_c.size();
  st.proj.resize(V);
  st.count.resize(V);
  st.rgb.resize(V);
#pragma omp parallel for schedule(static)
  for (long c = 0; c < (long)V; ++c) {
    const int g = st.gid_of_c[c];
    st.proj[c] = all[g];
    st.count[c] = cnt[g];
    // project_visible.wgsl:168-208: SH colour for the visible Gaussian.
    const F* t = sp.transforms + (size_t)g * 10;
    V3<F> mean{t[0], t[1], t[2]};
    const F* shg = sp.sh + (size_t)g * sp.K * 3;
    auto coeff = [&](int k, int ch) { return shg[k * 3 + ch]; };
    st.rgb[c] = sh_to_color<F>(sp.degree, view_dir(cam, mean), coeff);
  }
  // sorting.rs:34-61 + radix_sort.wgsl:21-26: ascending depth bits, ties by
  // the pre-sort index (here the global id, via compact order).
  st.order.resize(V);
  std::iota(st.order.begin(), st.order.end(), 0);
  std::stable_sort(st.order.begin(), st.order.end(), [&](int a, int b) {
    if (sizeof(F) == 4) {
      const uint32_t ka = float_to_bits((float)st.proj[a].depth), kb = float_to_bits((float)st.proj[b].depth);
      return ka < kb;
    }
    return st.proj[a].depth < st.proj[b].depth;
  });
  // prefix_sum.wgsl over counts in depth order -> emission offsets.
  std::vector<uint64_t> off(V + 1, 0);
  for (size_t r = 0; r < V; ++r) off[r + 1] = off[r] + st.count[st.order[r]];
  const size_t I = off[V];
  std::vector<uint32_t> et(I), ec(I);
  // map_gaussian_to_intersects.wgsl:17-48, with the tile test of the count
  // pass (one tile-set function for both passes).
#pragma omp parallel for schedule(dynamic, 256)
  for (long r = 0; r < (long)V; ++r) {
    const int c = st.order[r];
    const Projected<F>& p = st.proj[c];
    uint64_t o = off[r];
    for (uint32_t ty = p.box.y0; ty < p.box.y1; ++ty)
      for (uint32_t tx = p.box.x0; tx < p.box.x1; ++tx)
        if (will_primitive_contribute(tx, ty, st.ts, p.mean2d, p.conic, p.thr)) {
          et[o] = tx + ty * st.tiles_x;
          ec[o] = (uint32_t)c;
          ++o;
        }
  }
  // Stable sort by tile id (tile_mapping.rs:206-215) as a counting sort.
  std::vector<uint64_t> tstart(T + 1, 0);
  for (size_t i = 0; i < I; ++i) tstart[et[i] + 1]++;
  for (uint32_t t = 0; t < T; ++t) tstart[t + 1] += tstart[t];
  st.isect_tile.resize(I);
  st.isect_c.resize(I);
  {
    std::vector<uint64_t> cur(tstart.begin(), tstart.end() - 1);
    for (size_t i = 0; i < I; ++i) {
      const uint64_t d = cur[et[i]]++;
      st.isect_tile[d] = et[i];
      st.isect_c[d] = ec[i];
    }
  }
  // get_tile_offsets.wgsl:11-30 (untouched tiles keep 0, 0).
  st.ranges.assign(2 * (size_t)T, 0);
  for (size_t i = 0; i < I; ++i) {
    const uint32_t t = st.isect_tile[i];
    if (i == 0 || t != st.isect_tile[i - 1]) st.ranges[2 * t] = (uint32_t)i;
    if (i + 1 == I || t != st.isect_tile[i + 1]) st.ranges[2 * t + 1] = (uint32_t)(i + 1);
  }
  // rasterize.wgsl:21-99.
  st.image.assign((size_t)W * H * 4, F(0));
  st.tfinal.assign((size_t)W * H, F(1));
  st.last.assign((size_t)W * H, 0);
  st.ncontrib.assign((size_t)W * H, 0);
  st.nvisit.assign((size_t)W * H, 0);
  st.hit_blocks.assign(I, 0);
  std::vector<uint8_t> vis_c(V, 0);
#pragma omp parallel for schedule(dynamic, 4)
  for (long tile = 0; tile < (long)T; ++tile) {
    const uint32_t tx = (uint32_t)tile % st.tiles_x, ty = (uint32_t)tile / st.tiles_x;
    const uint32_t s0 = st.ranges[2 * tile], s1 = st.ranges[2 * tile + 1];
    for (uint32_t ly = 0; ly < st.ts.th; ++ly)
      for (uint32_t lx = 0; lx < st.ts.tw; ++lx) {
        const uint32_t px = tx * st.ts.tw + lx, py = ty * st.ts.th + ly;
        if (px >= W || py >= H) continue;
        const F pcx = F(px) + F(0.5), pcy = F(py) + F(0.5);
        F Tr = F(1), C[3] = {F(0), F(0), F(0)};
        uint32_t last = 0, nc = 0, nv = 0;
        for (uint32_t s = s0; s < s1; ++s) {
          const uint32_t c = st.isect_c[s];
          const Projected<F>& p = st.proj[c];
          ++nv;
          F gauss;
          const F alpha =
              blend_alpha(pcx, pcy, p.mean2d.x, p.mean2d.y, p.conic.x, p.conic.y, p.conic.z, p.opacity, gauss);
          if (alpha < F(0)) continue;
          const F vis = alpha * Tr;
          C[0] = blend_accum(C[0], st.rgb[c].x, vis);
          C[1] = blend_accum(C[1], st.rgb[c].y, vis);
          C[2] = blend_accum(C[2], st.rgb[c].z, vis);
          Tr = Tr * (F(1) - alpha);
          vis_c[c] = 1;  // benign race: every writer stores 1
          st.hit_blocks[s] |= 1u << ((lx / 8) + (ly / 8) * ((st.ts.tw + 7) / 8));  // entry s belongs to this tile only
          last = s + 1;
          ++nc;
          if (Tr < F(1e-4)) break;
        }
        const size_t pix = (size_t)py * W + px;
        st.image[pix * 4 + 0] = C[0] + Tr * st.bg[0];
        st.image[pix * 4 + 1] = C[1] + Tr * st.bg[1];
        st.image[pix * 4 + 2] = C[2] + Tr * st.bg[2];
        st.image[pix * 4 + 3] = F(1) - Tr;
        st.tfinal[pix] = Tr;
        st.last[pix] = last;
        st.ncontrib[pix] = nc;
        st.nvisit[pix] = nv;
      }
  }
  st.visible.assign(sp.n, F(0));
  for (size_t c = 0; c < V; ++c)
    if (vis_c[c]) st.visible[st.gid_of_c[c]] = F(1);
}

// ---------------------------------------------------------------------------
// Backward.
// mode 0: exact adjoint, reverse walk from each pixel's last contributor with
//         the transmittance recovered by division (follows the forward's
//         termination), then the exact projection adjoint.
// mode 1: reverse walk with the reference's semantics: the Gaussian that
//         takes T to <= 1e-4 and all after it get no gradient
//         (rasterize_backwards.wgsl:108-112) and the projection adjoint omits
//         the compensation and view-direction terms (project_backwards.wgsl).
// mode 2: literal restatement of rasterize_backwards.wgsl:26-169 (front to
//         back, colour-behind from the final colour) + mode-1 projection.
// ---------------------------------------------------------------------------
template <class F> struct BwdOut {
  std::vector<SplatGrad<F>> sg;  // per compact index
};

template <class F> void raster_backward(const FwdState<F>& st, const F* v_rgba, int mode, BwdOut<F>& out) {
  const uint32_t W = st.cam.w, H = st.cam.h, T = st.tiles_x * st.tiles_y;
  const size_t V = st.gid_of_c.size(), I = st.isect_c.size();
  // Per intersection partial sums over the tile's pixels, then a reduction in
  // sorted-intersection order: deterministic under OpenMP.
  std::vector<SplatGrad<F>> part(I);
  std::memset((void*)part.data(), 0, sizeof(SplatGrad<F>) * I);
#pragma omp parallel for schedule(dynamic, 4)
  for (long tile = 0; tile < (long)T; ++tile) {
    const uint32_t tx = (uint32_t)tile % st.tiles_x, ty = (uint32_t)tile / st.tiles_x;
    const uint32_t s0 = st.ranges[2 * tile], s1 = st.ranges[2 * tile + 1];
    for (uint32_t ly = 0; ly < st.ts.th; ++ly)
      for (uint32_t lx = 0; lx < st.ts.tw; ++lx) {
        const uint32_t px = tx * st.ts.tw + lx, py = ty * st.ts.th + ly;
        if (px >= W || py >= H) continue;
        const size_t pix = (size_t)py * W + px;
        const F pcx = F(px) + F(0.5), pcy = F(py) + F(0.5);
        const F* vo = v_rgba + pix * 4;
        if (mode == 2) {
          // rasterize_backwards.wgsl:48-165.
          const F* fc = &st.image[pix * 4];
          const F Tf = F(1) - fc[3];
          const F fin[3] = {fc[0] - Tf * st.bg[0], fc[1] - Tf * st.bg[1], fc[2] - Tf * st.bg[2]};
          const F vrgb[3] = {vo[0], vo[1], vo[2]};
          const F va = (vo[3] - (st.bg[0] * vo[0] + st.bg[1] * vo[1] + st.bg[2] * vo[2])) * Tf;
          F po[3] = {F(0), F(0), F(0)}, pa = F(1);
          for (uint32_t s = s0; s < s1; ++s) {
            const uint32_t c = st.isect_c[s];
            const Projected<F>& p = st.proj[c];
            const F r3[3] = {st.rgb[c].x, st.rgb[c].y, st.rgb[c].z};
            const F cp[3] = {gmax(r3[0], F(0)), gmax(r3[1], F(0)), gmax(r3[2], F(0))};
            const F dx = p.mean2d.x - pcx, dy = p.mean2d.y - pcy;
            const F sigma = F(0.5) * (p.conic.x * dx * dx + p.conic.z * dy * dy) + p.conic.y * dx * dy;
            const F gauss = gexp(-sigma);
            const F alpha = gmin(F(0.999), p.opacity * gauss);
            if (sigma < F(0) || alpha < F(1.0 / 255.0)) continue;
            const F nT = pa * (F(1) - alpha);
            if (nT <= F(1e-4)) break;
            const F vis = alpha * pa;
            SplatGrad<F>& g = part[s];
            for (int k = 0; k < 3; ++k) g.v_rgb[k] = g.v_rgb[k] + ((r3[k] >= F(0)) ? vis * vrgb[k] : F(0));
            for (int k = 0; k < 3; ++k) po[k] = po[k] + vis * cp[k];
            const F ra = F(1) / (F(1) - alpha);
            F v_alpha = F(0);
            for (int k = 0; k < 3; ++k) v_alpha = v_alpha + (pa * cp[k] + (po[k] - fin[k]) * ra) * vrgb[k];
            v_alpha = v_alpha + va * ra;
            const F vs = -alpha * v_alpha;
            if (p.opacity * gauss <= F(0.999)) {
              const F vx = vs * (p.conic.x * dx + p.conic.y * dy);
              const F vy = vs * (p.conic.y * dx + p.conic.z * dy);
              g.v_conic[0] = g.v_conic[0] + F(0.5) * vs * dx * dx;
              g.v_conic[1] = g.v_conic[1] + vs * dx * dy;
              g.v_conic[2] = g.v_conic[2] + F(0.5) * vs * dy * dy;
              g.v_xy[0] = g.v_xy[0] + vx;
              g.v_xy[1] = g.v_xy[1] + vy;
              g.v_opac = g.v_opac + v_alpha * gauss;
              g.abs_xy[0] = g.abs_xy[0] + gabs(vx);
              g.abs_xy[1] = g.abs_xy[1] + gabs(vy);
            }
            g.count = g.count + F(1);
            pa = nT;
          }
          continue;
        }
        // Reverse walk (modes 0 and 1).
        const uint32_t last = st.last[pix];
        if (last == 0) continue;
        const F vrgb[3] = {vo[0], vo[1], vo[2]};
        const F Tf = st.tfinal[pix];
        const F K = (vrgb[0] * st.bg[0] + vrgb[1] * st.bg[1] + vrgb[2] * st.bg[2] - vo[3]) * Tf;
        F Tr = Tf, S[3] = {F(0), F(0), F(0)};
        for (uint32_t s = last; s-- > s0;) {
          const uint32_t c = st.isect_c[s];
          const Projected<F>& p = st.proj[c];
          F gauss;
          const F alpha =
              blend_alpha(pcx, pcy, p.mean2d.x, p.mean2d.y, p.conic.x, p.conic.y, p.conic.z, p.opacity, gauss);
          if (alpha < F(0)) continue;
          const bool skip = (mode == 1) && (Tr <= F(1e-4));
          SplatGrad<F> g;
          blend_step_grad(p.mean2d.x - pcx, p.mean2d.y - pcy, p.conic.x, p.conic.y, p.conic.z, st.rgb[c].x,
                          st.rgb[c].y, st.rgb[c].z, p.opacity, gauss, alpha, Tr, S, vrgb, K, skip, g);
          SplatGrad<F>& acc = part[s];
          acc.v_xy[0] += g.v_xy[0];
          acc.v_xy[1] += g.v_xy[1];
          for (int k = 0; k < 3; ++k) acc.v_conic[k] += g.v_conic[k];
          for (int k = 0; k < 3; ++k) acc.v_rgb[k] += g.v_rgb[k];
          acc.v_opac += g.v_opac;
          acc.abs_xy[0] += g.abs_xy[0];
          acc.abs_xy[1] += g.abs_xy[1];
          acc.count += g.count;
        }
      }
  }
  out.sg.assign(V, SplatGrad<F>());
  std::memset((void*)out.sg.data(), 0, sizeof(SplatGrad<F>) * V);
  for (size_t s = 0; s < I; ++s) {
    SplatGrad<F>& a = out.sg[st.isect_c[s]];
    const SplatGrad<F>& b = part[s];
    a.v_xy[0] += b.v_xy[0];
    a.v_xy[1] += b.v_xy[1];
    for (int k = 0; k < 3; ++k) a.v_conic[k] += b.v_conic[k];
    for (int k = 0; k < 3; ++k) a.v_rgb[k] += b.v_rgb[k];
    a.v_opac += b.v_opac;
    a.abs_xy[0] += b.abs_xy[0];
    a.abs_xy[1] += b.abs_xy[1];
    a.count += b.count;
  }
}

// project_backwards.wgsl:12-151 for every visible Gaussian; rows of
// non-visible Gaussians stay zero (project_bwd.rs zero-fills).
template <class F>
void project_backward_all(const FwdState<F>& st, const BwdOut<F>& bo, bool exact, F* v_tr, F* v_sh, F* v_op,
                          F* stats) {
  const Splats<F>& sp = st.sp;
  const int K = sp.K;
  std::memset(v_tr, 0, sizeof(F) * 10 * (size_t)sp.n);
  std::memset(v_sh, 0, sizeof(F) * 3 * (size_t)K * sp.n);
  std::memset(v_op, 0, sizeof(F) * (size_t)sp.n);
  std::memset(stats, 0, sizeof(F) * 7 * (size_t)sp.n);
  const long V = (long)st.gid_of_c.size();
#pragma omp parallel for schedule(static)
  for (long c = 0; c < V; ++c) {
    const int g = st.gid_of_c[c];
    const SplatGrad<F>& sg = bo.sg[c];
    const F* t = sp.transforms + (size_t)g * 10;
    const F* shg = sp.sh + (size_t)g * K * 3;
    auto coeff = [&](int k, int ch) { return shg[k * 3 + ch]; };
    V3<F> mean{t[0], t[1], t[2]};
    V4<F> q{t[3], t[4], t[5], t[6]};
    V3<F> ls{t[7], t[8], t[9]};
    V2<F> vxy{sg.v_xy[0], sg.v_xy[1]};
    V3<F> vcon{sg.v_conic[0], sg.v_conic[1], sg.v_conic[2]};
    V3<F> vcol{sg.v_rgb[0], sg.v_rgb[1], sg.v_rgb[2]};
    const ParamGrad<F> pg = project_backward(st.cam, mean, q, ls, sp.raw_opac[g], st.cov_blur, vxy, vcon, vcol,
                                             sg.v_opac, sp.degree, coeff, exact, true, st.hp);
    // helpers.wgsl:289-380: SH coefficient gradients.
    F b[25];
    sh_basis<F>(sp.degree, pg.viewdir.x, pg.viewdir.y, pg.viewdir.z, b);
    for (int k = 0; k < K; ++k) {
      v_sh[((size_t)g * K + k) * 3 + 0] = b[k] * vcol.x;
      v_sh[((size_t)g * K + k) * 3 + 1] = b[k] * vcol.y;
      v_sh[((size_t)g * K + k) * 3 + 2] = b[k] * vcol.z;
    }
    F* o = v_tr + (size_t)g * 10;
    o[0] = pg.v_mean.x;
    o[1] = pg.v_mean.y;
    o[2] = pg.v_mean.z;
    o[3] = pg.v_quat.x;
    o[4] = pg.v_quat.y;
    o[5] = pg.v_quat.z;
    o[6] = pg.v_quat.w;
    o[7] = pg.v_log_scale.x;
    o[8] = pg.v_log_scale.y;
    o[9] = pg.v_log_scale.z;
    v_op[g] = pg.v_raw_opac;
    // project_backwards.wgsl:33-36, 105-108.
    F* s = stats + (size_t)g * 7;
    s[0] = sg.v_xy[0];
    s[1] = sg.v_xy[1];
    s[2] = sg.abs_xy[0];
    s[3] = sg.abs_xy[1];
    const F abs_score = gsqrt(sg.abs_xy[0] * sg.abs_xy[0] + sg.abs_xy[1] * sg.abs_xy[1]);
    s[4] = sg.count * abs_score;
    s[5] = sg.count;
    s[6] = sg.count * pg.depth;
  }
}

// ---------------------------------------------------------------------------
// Loss (engine/loss.rs:42-76, 144-196, 233-276 with the default weights:
// 0.8 * L1 + 0.2 * (1 - SSIM), 11-tap sigma 1.5 Gaussian window, replicate
// padding, C1 = 0.01^2, C2 = 0.03^2, denominators clamped at 1e-8).
// pred has pstride floats per pixel (3 or 4); target has 3.
// ---------------------------------------------------------------------------
template <class F> void gauss_kernel(F* k) {
  // loss.rs:233-250: values computed in f64, stored as f32, normalised in f32.
  float vals[11], sum = 0.0f;
  for (int o = -5; o <= 5; ++o) {
    vals[o + 5] = (float)std::exp(-(double)(o * o) / (2.0 * 1.5 * 1.5));
    sum += vals[o + 5];
  }
  for (int i = 0; i < 11; ++i) k[i] = F(vals[i] / std::max(sum, 1e-8f));
}

// Separable blur with replicate padding, horizontal then vertical (loss.rs:252-276).
template <class F> void blur(const std::vector<F>& in, std::vector<F>& out, int H, int W, const F* k) {
  std::vector<F> tmp((size_t)H * W);
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      F s = F(0);
      for (int t = 0; t < 11; ++t) {
        const int xx = std::min(std::max(x + t - 5, 0), W - 1);
        s = s + k[t] * in[(size_t)y * W + xx];
      }
      tmp[(size_t)y * W + x] = s;
    }
  out.resize((size_t)H * W);
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      F s = F(0);
      for (int t = 0; t < 11; ++t) {
        const int yy = std::min(std::max(y + t - 5, 0), H - 1);
        s = s + k[t] * tmp[(size_t)yy * W + x];
      }
      out[(size_t)y * W + x] = s;
    }
}

// Adjoint of blur.
template <class F> void blur_adj(const std::vector<F>& g, std::vector<F>& out, int H, int W, const F* k) {
  std::vector<F> tmp((size_t)H * W, F(0));
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x)
      for (int t = 0; t < 11; ++t) {
        const int yy = std::min(std::max(y + t - 5, 0), H - 1);
        tmp[(size_t)yy * W + x] += k[t] * g[(size_t)y * W + x];
      }
  out.assign((size_t)H * W, F(0));
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x)
      for (int t = 0; t < 11; ++t) {
        const int xx = std::min(std::max(x + t - 5, 0), W - 1);
        out[(size_t)y * W + xx] += k[t] * tmp[(size_t)y * W + x];
      }
}

template <class F>
double loss_fwd_bwd(const F* pred, int pstride, const F* tgt, int H, int W, double l1w, double ssimw, F* v_pred) {
  F k[11];
  gauss_kernel(k);
  const size_t P = (size_t)H * W;
  const F C1 = F(0.0001), C2 = F(0.0009);
  double l1 = 0.0, ssim_sum = 0.0;
  const double M = 3.0 * (double)P;
  for (size_t i = 0; i < P * (size_t)pstride; ++i) v_pred[i] = F(0);
  for (int ch = 0; ch < 3; ++ch) {
    std::vector<F> x(P), y(P), xx(P), yy(P), xy(P);
    for (size_t i = 0; i < P; ++i) {
      x[i] = pred[i * pstride + ch];
      y[i] = tgt[i * 3 + ch];
      xx[i] = x[i] * x[i];
      yy[i] = y[i] * y[i];
      xy[i] = x[i] * y[i];
    }
    std::vector<F> mx, my, exx, eyy, exy;
    blur(x, mx, H, W, k);
    blur(y, my, H, W, k);
    blur(xx, exx, H, W, k);
    blur(yy, eyy, H, W, k);
    blur(xy, exy, H, W, k);
    std::vector<F> gmx(P), gexx(P), gexy(P);
    for (size_t i = 0; i < P; ++i) {
      const F mux = mx[i], muy = my[i];
      const F sxx = exx[i] - mux * mux, syy = eyy[i] - muy * muy, sxy = exy[i] - mux * muy;
      const F A = F(2) * mux * muy + C1, B = F(2) * sxy + C2;
      const F Cr = mux * mux + muy * muy + C1, Dr = sxx + syy + C2;
      const F Cc = gmax(Cr, F(1e-8)), Dc = gmax(Dr, F(1e-8));
      const F s = (A * B) / (Cc * Dc);
      ssim_sum += (double)s;
      // d s / d(mx, exx, exy) with sxx = exx - mx^2, sxy = exy - mx*my.
      const F inv = F(1) / (Cc * Dc);
      const F dC = (Cr > F(1e-8)) ? F(1) : F(0), dD = (Dr > F(1e-8)) ? F(1) : F(0);
      const F dA_dmx = F(2) * muy, dB_dmx = F(-2) * muy;
      const F dC_dmx = F(2) * mux * dC, dD_dmx = F(-2) * mux * dD;
      gmx[i] = (dA_dmx * B + A * dB_dmx) * inv - s * (dC_dmx * Dc + Cc * dD_dmx) / (Cc * Dc);
      gexx[i] = -s * dD / Dc;
      gexy[i] = F(2) * A * inv;
      l1 += std::fabs((double)(x[i] - y[i]));
    }
    std::vector<F> amx, aexx, aexy;
    blur_adj(gmx, amx, H, W, k);
    blur_adj(gexx, aexx, H, W, k);
    blur_adj(gexy, aexy, H, W, k);
    const F ks = F(-ssimw / M), kl = F(l1w / M);
    for (size_t i = 0; i < P; ++i) {
      const F d = x[i] - y[i];
      const F sg = (d > F(0)) ? F(1) : ((d < F(0)) ? F(-1) : F(0));
      v_pred[i * pstride + ch] = kl * sg + ks * (amx[i] + F(2) * x[i] * aexx[i] + y[i] * aexy[i]);
    }
  }
  return l1w * (l1 / M) + ssimw * (1.0 - ssim_sum / M);
}

}  // namespace

// ===========================================================================
// C ABI for ctypes.
// ===========================================================================
extern "C" {

struct orc_fwd_f32 {
  FwdState<float> st;
};
struct orc_fwd_f64 {
  FwdState<double> st;
};

#define ORC_EXPORT __attribute__((visibility("default")))

// ---- frame targets (training/data/frame_targets.rs) ----
// resize_rgb_u8_to_f32 (:44-62): each byte / 255; a frame of another size is
// then box-averaged by resize_rgb (:1-42), rows and columns in order.
ORC_EXPORT void orc_frame_to_target(const uint8_t* src, uint32_t sw, uint32_t sh, uint32_t dw, uint32_t dh,
                                    float* dst) {
  if (sw == dw && sh == dh) {
    for (uint64_t i = 0; i < (uint64_t)sw * sh * 3; ++i) dst[i] = (float)src[i] / 255.0f;
    return;
  }
  for (uint64_t dy = 0; dy < dh; ++dy) {
    const uint64_t sy0 = dy * sh / dh;
    const uint64_t sy1 = std::min(std::max((dy + 1) * sh / dh, sy0 + 1), (uint64_t)sh);
    for (uint64_t dx = 0; dx < dw; ++dx) {
      const uint64_t sx0 = dx * sw / dw;
      const uint64_t sx1 = std::min(std::max((dx + 1) * sw / dw, sx0 + 1), (uint64_t)sw);
      float acc[3] = {0.f, 0.f, 0.f};
      uint64_t count = 0;
      for (uint64_t sy = sy0; sy < sy1; ++sy)
        for (uint64_t sx = sx0; sx < sx1; ++sx) {
          const uint8_t* q = src + (sy * sw + sx) * 3;
          for (int c = 0; c < 3; ++c) acc[c] = acc[c] + (float)q[c] / 255.0f;
          ++count;
        }
      const float inv = 1.0f / (float)(count > 0 ? count : 1);
      float* o = dst + (dy * dw + dx) * 3;
      for (int c = 0; c < 3; ++c) o[c] = acc[c] * inv;
    }
  }
}

// ---- primitives (gpu_primitives/*) ----
// Inclusive scan (prefix_sum.rs:53-136).
ORC_EXPORT void orc_prefix_sum_u32(const uint32_t* in, uint32_t* out, uint64_t n) {
  uint32_t acc = 0;
  for (uint64_t i = 0; i < n; ++i) {
    acc += in[i];
    out[i] = acc;
  }
}
// Stable sort by key with ties in input order (radix_sort.wgsl:21-26).
ORC_EXPORT void orc_sort_pairs_u32(const uint32_t* keys, const uint32_t* vals, uint32_t* ko, uint32_t* vo,
                                   uint64_t n) {
  std::vector<uint64_t> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](uint64_t a, uint64_t b) { return keys[a] < keys[b]; });
  for (uint64_t i = 0; i < n; ++i) {
    ko[i] = keys[idx[i]];
    vo[i] = vals[idx[i]];
  }
}
ORC_EXPORT float orc_expf(float x) { return portable_expf(x); }
ORC_EXPORT float orc_blend_expf(float x) { return blend_expf(x); }
ORC_EXPORT float orc_logf(float x) { return portable_logf(x); }

// ---- forward ----
#define ORC_FWD_IMPL(SUF, F)                                                                                    \
  ORC_EXPORT orc_fwd_##SUF* orc_forward_##SUF(const F* transforms, const F* sh, const F* raw_opac, int n,         \
                                              int degree, const orc_camera* cam, F cov_blur, const F* bg,         \
                                              uint32_t tile_w, uint32_t tile_h, int hp) {                         \
    orc_fwd_##SUF* h = new orc_fwd_##SUF();                                                                       \
    FwdState<F>& st = h->st;                                                                                      \
    st.sp.n = n;                                                                                                  \
    st.sp.degree = degree;                                                                                        \
    st.sp.K = num_sh_coeffs(degree);                                                                              \
    st.sp.transforms = transforms;                                                                                \
    st.sp.sh = sh;                                                                                                \
    st.sp.raw_opac = raw_opac;                                                                                    \
    st.camera = *cam;                                                                                             \
    st.cam = make_cam<F>(*cam);                                                                                   \
    st.cov_blur = cov_blur;                                                                                       \
    st.hp = hp != 0;                                                                                              \
    st.bg[0] = bg[0];                                                                                             \
    st.bg[1] = bg[1];                                                                                             \
    st.bg[2] = bg[2];                                                                                             \
    st.ts.tw = tile_w;                                                                                            \
    st.ts.th = tile_h;                                                                                            \
    forward(st);                                                                                                  \
    return h;                                                                                                     \
  }                                                                                                               \
  ORC_EXPORT void orc_free_##SUF(orc_fwd_##SUF* h) { delete h; }                                                  \
  ORC_EXPORT void orc_sizes_##SUF(const orc_fwd_##SUF* h, uint64_t* out) {                                        \
    out[0] = h->st.gid_of_c.size();                                                                               \
    out[1] = h->st.isect_c.size();                                                                                \
    out[2] = h->st.tiles_x;                                                                                       \
    out[3] = h->st.tiles_y;                                                                                       \
  }                                                                                                               \
  /* per visible Gaussian (compact order): gid, count, depth, mean2d, conic, opacity, thr, rgb, box */           \
  ORC_EXPORT void orc_visible_##SUF(const orc_fwd_##SUF* h, int32_t* gid, uint32_t* count, F* depth, F* rec,       \
                                    uint32_t* box) {                                                               \
    const FwdState<F>& st = h->st;                                                                                \
    for (size_t c = 0; c < st.gid_of_c.size(); ++c) {                                                             \
      const Projected<F>& p = st.proj[c];                                                                         \
      gid[c] = st.gid_of_c[c];                                                                                    \
      count[c] = st.count[c];                                                                                     \
      depth[c] = p.depth;                                                                                         \
      F* r = rec + c * 10;                                                                                        \
      r[0] = p.mean2d.x;                                                                                          \
      r[1] = p.mean2d.y;                                                                                          \
      r[2] = p.conic.x;                                                                                           \
      r[3] = p.conic.y;                                                                                           \
      r[4] = p.conic.z;                                                                                           \
      r[5] = p.opacity;                                                                                           \
      r[6] = p.thr;                                                                                               \
      r[7] = st.rgb[c].x;                                                                                         \
      r[8] = st.rgb[c].y;                                                                                         \
      r[9] = st.rgb[c].z;                                                                                         \
      box[c * 4 + 0] = p.box.x0;                                                                                  \
      box[c * 4 + 1] = p.box.y0;                                                                                  \
      box[c * 4 + 2] = p.box.x1;                                                                                  \
      box[c * 4 + 3] = p.box.y1;                                                                                  \
    }                                                                                                             \
  }                                                                                                               \
  ORC_EXPORT void orc_order_##SUF(const orc_fwd_##SUF* h, int32_t* order) {                                       \
    std::copy(h->st.order.begin(), h->st.order.end(), order);                                                     \
  }                                                                                                               \
  ORC_EXPORT void orc_isects_##SUF(const orc_fwd_##SUF* h, uint32_t* tiles, uint32_t* cs, uint32_t* ranges) {     \
    std::copy(h->st.isect_tile.begin(), h->st.isect_tile.end(), tiles);                                           \
    std::copy(h->st.isect_c.begin(), h->st.isect_c.end(), cs);                                                    \
    std::copy(h->st.ranges.begin(), h->st.ranges.end(), ranges);                                                  \
  }                                                                                                               \
  ORC_EXPORT void orc_pixels_##SUF(const orc_fwd_##SUF* h, F* image, F* tfinal, uint32_t* last, uint32_t* nc,     \
                                   uint32_t* nv, F* visible) {                                                    \
    const FwdState<F>& st = h->st;                                                                                \
    std::copy(st.image.begin(), st.image.end(), image);                                                           \
    std::copy(st.tfinal.begin(), st.tfinal.end(), tfinal);                                                        \
    std::copy(st.last.begin(), st.last.end(), last);                                                              \
    std::copy(st.ncontrib.begin(), st.ncontrib.end(), nc);                                                        \
    std::copy(st.nvisit.begin(), st.nvisit.end(), nv);                                                            \
    std::copy(st.visible.begin(), st.visible.end(), visible);                                                     \
  }                                                                                                               \
  ORC_EXPORT void orc_hit_blocks_##SUF(const orc_fwd_##SUF* h, uint32_t* bits) {                                 \
    std::copy(h->st.hit_blocks.begin(), h->st.hit_blocks.end(), bits);                                            \
  }                                                                                                               \
  /* backward: mode 0 exact, 1 reference semantics (reverse walk), 2 literal WGSL walk */                         \
  ORC_EXPORT void orc_backward_##SUF(const orc_fwd_##SUF* h, const F* v_rgba, int mode, F* v_tr, F* v_sh, F* v_op, \
                                     F* stats, F* splat_grads) {                                                  \
    BwdOut<F> bo;                                                                                                 \
    raster_backward(h->st, v_rgba, mode, bo);                                                                     \
    project_backward_all(h->st, bo, mode == 0, v_tr, v_sh, v_op, stats);                                          \
    if (splat_grads) {                                                                                            \
      for (size_t c = 0; c < bo.sg.size(); ++c) {                                                                 \
        const SplatGrad<F>& g = bo.sg[c];                                                                         \
        F* o = splat_grads + c * 12;                                                                              \
        o[0] = g.v_xy[0];                                                                                         \
        o[1] = g.v_xy[1];                                                                                         \
        o[2] = g.v_conic[0];                                                                                      \
        o[3] = g.v_conic[1];                                                                                      \
        o[4] = g.v_conic[2];                                                                                      \
        o[5] = g.v_rgb[0];                                                                                        \
        o[6] = g.v_rgb[1];                                                                                        \
        o[7] = g.v_rgb[2];                                                                                        \
        o[8] = g.v_opac;                                                                                          \
        o[9] = g.abs_xy[0];                                                                                       \
        o[10] = g.abs_xy[1];                                                                                      \
        o[11] = g.count;                                                                                          \
      }                                                                                                           \
    }                                                                                                             \
  }                                                                                                               \
  ORC_EXPORT double orc_loss_##SUF(const F* pred, int pstride, const F* tgt, int H, int W, double l1w,            \
                                   double ssimw, F* v_pred) {                                                     \
    return loss_fwd_bwd<F>(pred, pstride, tgt, H, W, l1w, ssimw, v_pred);                                         \
  }

ORC_FWD_IMPL(f32, float)
ORC_FWD_IMPL(f64, double)

// ---- optimizer (engine/optimizer.rs:122-162) ----
// p -= (m_hat / (sqrt(v_hat) + eps)) * lr[i % ncols] with the bias
// corrections 1 - beta^step of the given step (1-based).
ORC_EXPORT void orc_adam_f32(float* p, const float* g, float* m, float* v, uint64_t n, const float* lr, int ncols,
                             int step, float beta1, float beta2, float eps) {
  const float omb1 = 1.0f - beta1, omb2 = 1.0f - beta2;
  // The bias corrections are applied as multiplications by their f32
  // reciprocals (the reference divides; the two differ by at most an ulp).
  const float rbc1 = 1.0f / (1.0f - powi_f32(beta1, step)), rbc2 = 1.0f / (1.0f - powi_f32(beta2, step));
  for (uint64_t i = 0; i < n; ++i) {
    const float gi = g[i];
    const float m1 = m[i] * beta1 + gi * omb1;
    const float m2 = v[i] * beta2 + (gi * gi) * omb2;
    m[i] = m1;
    v[i] = m2;
    const float mh = m1 * rbc1, vh = m2 * rbc2;
    const float upd = mh / (sqrtf(vh) + eps);
    p[i] = p[i] - upd * lr[i % (uint64_t)ncols];
  }
}

// ---- densification statistics (engine/trainer.rs:651-728) ----
// acc is 9 arrays of n floats: grad_2d, screen_grad_2d, abs_grad_2d,
// abs_pixel_grad_2d, pixel_coverage, camera_depth, grad_color,
// num_observations, visible_observations.
// topology/apply.rs:29-94 restated through the shared topo_mutate: output
// row i copies source rows[i*3] with kind rows[i*3+1] and sample scalar
// (bits) rows[i*3+2]; SH rows are copied (sh_elems floats each).
ORC_EXPORT int orc_topology_apply_f32(const float* tr, const float* sh, const float* op, uint32_t n, uint32_t sh_elems,
                                      const uint32_t* rows, uint32_t m, int has_decay, float scale_decay,
                                      float opacity_decay, float train_t, int opacity_reset, float reset_cap,
                                      float* otr, float* osh, float* oop) {
  TopoParams p{};
  p.has_decay = has_decay;
  p.scale_decay = scale_decay;
  p.opacity_decay = opacity_decay;
  p.train_t = train_t;
  p.opacity_reset = opacity_reset;
  p.reset_cap = reset_cap;
  for (uint32_t i = 0; i < m; ++i) {
    const uint32_t src = rows[(size_t)i * 3];
    const int kind = (int)rows[(size_t)i * 3 + 1];
    float sample;
    memcpy(&sample, &rows[(size_t)i * 3 + 2], 4);
    if (src >= n) return -1;
    float t[10];
    for (int k = 0; k < 10; ++k) t[k] = tr[(size_t)src * 10 + k];
    float logit = op[src];
    topo_mutate(t, logit, kind, sample, p);
    for (int k = 0; k < 10; ++k) otr[(size_t)i * 10 + k] = t[k];
    oop[i] = logit;
    for (uint32_t k = 0; k < sh_elems; ++k) osh[(size_t)i * sh_elems + k] = sh[(size_t)src * sh_elems + k];
  }
  return 0;
}

ORC_EXPORT void orc_densify_f32(const float* v_tr, const float* stats, const float* v_sh, const float* visible,
                                int n, int K, int use_visible, float* acc) {
  for (int i = 0; i < n; ++i) {
    const float* t = v_tr + (size_t)i * 10;
    const float* s = stats + (size_t)i * 7;
    const float g2 = (fabsf(t[0]) + fabsf(t[1]) + fabsf(t[2])) / 3.0f;
    const float sg = sqrtf(s[0] * s[0] + s[1] * s[1]);
    const float ag = sqrtf(s[2] * s[2] + s[3] * s[3]);
    float gc = 0.0f;
    for (int k = 0; k < K; ++k) {
      const float* c = v_sh + ((size_t)i * K + k) * 3;
      gc += (fabsf(c[0]) + fabsf(c[1]) + fabsf(c[2])) / 3.0f;
    }
    gc = gc / (float)K;
    acc[0 * (size_t)n + i] += g2;
    acc[1 * (size_t)n + i] += sg;
    acc[2 * (size_t)n + i] += ag;
    acc[3 * (size_t)n + i] += s[4];
    acc[4 * (size_t)n + i] += s[5];
    acc[5 * (size_t)n + i] += s[6];
    acc[6 * (size_t)n + i] += gc;
    acc[7 * (size_t)n + i] += 1.0f;
    acc[8 * (size_t)n + i] += use_visible ? visible[i] : 1.0f;
  }
}

}  // extern "C"
