// ref_cpu_forward.cpp — TEST INFRASTRUCTURE (timed CPU baseline only).
//
// A restatement of the reference's shipped CPU forward renderer,
// RustGS/src/render/tiled_renderer.rs:174-386 (TiledRenderer::
// render_camera_splats, project_camera_splats, compute_tile_bounds,
// render_projected_with_background), projection tiled_renderer.rs:389-490,
// and the CPU SH evaluation RustGS/src/sh.rs:35-112 (its f32 constants).
// Its semantics differ from the GPU training path (no Jacobian clamp, a
// 3-sigma box of the 4x covariance, d^2 < 9 and weight > 0.001 cutoffs,
// saturation at accumulated alpha 0.999, colour clamped to [0, 1], a depth
// output), so it is never a parity reference: bench.py times it,
// single-threaded as shipped, beside the oracle. Only tests and bench.py
// load this library.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

struct Proj {
  float x, y, depth, cxx, cxy, cyy, opacity, rgb[3];
};

// sh.rs:35-112 (degree <= 4; coefficients [k][c]; + 0.5 bias, unclamped).
void sh_rgb(const float* c, int degree, const float d[3], float out[3]) {
  const float x = d[0], y = d[1], z = d[2];
  for (int ch = 0; ch < 3; ++ch) out[ch] = 0.2820948f * c[ch];
  auto add = [&](int k, float s) {
    for (int ch = 0; ch < 3; ++ch) out[ch] += c[k * 3 + ch] * s;
  };
  if (degree >= 1) {
    add(1, 0.48860252f * -y);
    add(2, 0.48860252f * z);
    add(3, 0.48860252f * -x);
  }
  if (degree >= 2) {
    const float z2 = z * z, t0b = -1.0925485f * z, t1a = 0.54627424f;
    const float c1 = x * x - y * y, s1 = 2.0f * x * y;
    add(4, t1a * s1);
    add(5, t0b * y);
    add(6, 0.9461747f * z2 - 0.31539157f);
    add(7, t0b * x);
    add(8, t1a * c1);
    if (degree >= 3) {
      const float t0c = -2.285229f * z2 + 0.4570458f, t1b = 1.4453057f * z, t2a = -0.5900436f;
      const float c2 = x * c1 - y * s1, s2 = x * s1 + y * c1;
      add(9, t2a * s2);
      add(10, t1b * s1);
      add(11, t0c * y);
      add(12, z * (1.8658817f * z2 - 1.119529f));
      add(13, t0c * x);
      add(14, t1b * c1);
      add(15, t2a * c2);
      if (degree >= 4) {
        const float t0d = z * (-4.683326f * z2 + 2.0071397f), t1c = 3.3116114f * z2 - 0.47308734f;
        const float t2b = -1.7701308f * z, t3a = 0.6258357f;
        const float c3 = x * c2 - y * s2, s3 = x * s2 + y * c2;
        const float p12 = z * (1.8658817f * z2 - 1.119529f), p6 = 0.9461747f * z2 - 0.31539157f;
        add(16, t3a * s3);
        add(17, t2b * s2);
        add(18, t1c * s1);
        add(19, t0d * y);
        add(20, 1.9843135f * z * p12 - 1.0062306f * p6);
        add(21, t0d * x);
        add(22, t1c * c1);
        add(23, t2b * c2);
        add(24, t3a * c3);
      }
    }
  }
  for (int ch = 0; ch < 3; ++ch) out[ch] += 0.5f;
}

// tiled_renderer.rs:389-475: EWA projection without the Jacobian clamp.
bool project(const float pos[3], const float scale[3], const float q[4], float opac, const float r[3][3],
             const float t[3], float fx, float fy, float pcx, float pcy, float blur, Proj& o) {
  const float cx = r[0][0] * pos[0] + r[0][1] * pos[1] + r[0][2] * pos[2] + t[0];
  const float cy = r[1][0] * pos[0] + r[1][1] * pos[1] + r[1][2] * pos[2] + t[1];
  const float cz = r[2][0] * pos[0] + r[2][1] * pos[1] + r[2][2] * pos[2] + t[2];
  if (cz <= 0.0f) return false;
  o.x = fx * cx / cz + pcx;
  o.y = fy * cy / cz + pcy;
  o.depth = cz;
  const float qw = q[0], qx = q[1], qy = q[2], qz = q[3];
  const float R[3][3] = {{1.0f - 2.0f * (qy * qy + qz * qz), 2.0f * (qx * qy - qw * qz), 2.0f * (qx * qz + qw * qy)},
                         {2.0f * (qx * qy + qw * qz), 1.0f - 2.0f * (qx * qx + qz * qz), 2.0f * (qy * qz - qw * qx)},
                         {2.0f * (qx * qz - qw * qy), 2.0f * (qy * qz + qw * qx), 1.0f - 2.0f * (qx * qx + qy * qy)}};
  const float s2[3] = {scale[0] * scale[0], scale[1] * scale[1], scale[2] * scale[2]};
  float W[3][3];  // world covariance R diag(s^2) R^T
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) W[i][j] = R[i][0] * R[j][0] * s2[0] + R[i][1] * R[j][1] * s2[1] + R[i][2] * R[j][2] * s2[2];
  float M[3][3], Cc[3][3];  // camera covariance r W r^T
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) M[i][j] = r[i][0] * W[0][j] + r[i][1] * W[1][j] + r[i][2] * W[2][j];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Cc[i][j] = M[i][0] * r[j][0] + M[i][1] * r[j][1] + M[i][2] * r[j][2];
  const float iz = 1.0f / cz, iz2 = iz * iz;
  const float jx0 = fx * iz, jx2 = -fx * cx * iz2, jy1 = fy * iz, jy2 = -fy * cy * iz2;
  float cxx = jx0 * (Cc[0][0] * jx0 + Cc[0][2] * jx2) + jx2 * (Cc[0][2] * jx0 + Cc[2][2] * jx2);
  const float cxy = jx0 * (Cc[0][1] * jy1 + Cc[0][2] * jy2) + jx2 * (Cc[1][2] * jy1 + Cc[2][2] * jy2);
  float cyy = jy1 * (Cc[1][1] * jy1 + Cc[1][2] * jy2) + jy2 * (Cc[1][2] * jy1 + Cc[2][2] * jy2);
  const float det_raw = cxx * cyy - cxy * cxy;
  cxx += std::max(blur, 0.0f);
  cyy += std::max(blur, 0.0f);
  const float det_blur = std::max(cxx * cyy - cxy * cxy, 1e-12f);
  if (det_raw <= 0.0f) return false;
  o.opacity = opac * std::sqrt(det_raw / det_blur);
  if (o.opacity < 1.0f / 255.0f) return false;
  o.cxx = cxx;
  o.cxy = cxy;
  o.cyy = cyy;
  return true;
}

}  // namespace

extern "C" __attribute__((visibility("default"))) void orc_ref_cpu_forward(
    const float* transforms /*[n,10]*/, const float* sh /*[n,K,3]*/, const float* raw_opac, int n, int degree,
    const float* viewmat /*4x4 column-major world->camera*/, const float* campos, float fx, float fy, float pcx,
    float pcy, int width, int height, float cov_blur, const float* background, float* color /*[h,w,3]*/,
    float* depth /*[h,w]*/) {
  const int K = (degree + 1) * (degree + 1);
  const float r[3][3] = {{viewmat[0], viewmat[4], viewmat[8]},
                         {viewmat[1], viewmat[5], viewmat[9]},
                         {viewmat[2], viewmat[6], viewmat[10]}};
  const float t[3] = {viewmat[12], viewmat[13], viewmat[14]};
  // project_camera_splats (tiled_renderer.rs:187-247)
  std::vector<Proj> proj;
  proj.reserve(n);
  for (int i = 0; i < n; ++i) {
    const float* tr = transforms + (size_t)i * 10;
    float d[3] = {tr[0] - campos[0], tr[1] - campos[1], tr[2] - campos[2]};
    const float len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (len <= 1e-12f) {
      d[0] = 0.0f;
      d[1] = 0.0f;
      d[2] = 1.0f;
    } else {
      d[0] /= len;
      d[1] /= len;
      d[2] /= len;
    }
    Proj p;
    sh_rgb(sh + (size_t)i * K * 3, degree, d, p.rgb);
    const float scale[3] = {std::fabs(std::exp(tr[7])), std::fabs(std::exp(tr[8])), std::fabs(std::exp(tr[9]))};
    const float opac = 1.0f / (1.0f + std::exp(-raw_opac[i]));
    if (project(tr, scale, tr + 3, opac, r, t, fx, fy, pcx, pcy, cov_blur, p)) proj.push_back(p);
  }
  // render_projected_with_background (tiled_renderer.rs:270-386), 16x16 tiles
  const int tw = 16, th = 16, ntx = (width + tw - 1) / tw, nty = (height + th - 1) / th;
  std::vector<float> alpha((size_t)width * height, 0.0f);
  std::fill(color, color + (size_t)width * height * 3, 0.0f);
  std::fill(depth, depth + (size_t)width * height, FLT_MAX);
  std::vector<std::vector<uint32_t>> lists((size_t)ntx * nty);
  for (size_t gi = 0; gi < proj.size(); ++gi) {
    const Proj& g = proj[gi];
    // compute_tile_bounds (tiled_renderer.rs:132-155), tile_alpha 4
    const float sx = std::max(std::sqrt(g.cxx * 4.0f), 1.0f), sy = std::max(std::sqrt(g.cyy * 4.0f), 1.0f);
    auto to_index = [](float v) -> long { return v <= 0.0f || v != v ? 0L : (long)v; };  // Rust `as usize`
    const long x0 = to_index(std::max(g.x - 3.0f * sx, 0.0f));
    const long x1 = to_index(std::min(g.x + 3.0f * sx, (float)width - 1.0f));
    const long y0 = to_index(std::max(g.y - 3.0f * sy, 0.0f));
    const long y1 = to_index(std::min(g.y + 3.0f * sy, (float)height - 1.0f));
    const long tx0 = x0 / tw, tx1 = (x1 + tw - 1) / tw, ty0 = y0 / th, ty1 = (y1 + th - 1) / th;
    for (long ty = ty0; ty < ty1 && ty < nty; ++ty)
      for (long tx = tx0; tx < tx1 && tx < ntx; ++tx) lists[(size_t)ty * ntx + tx].push_back((uint32_t)gi);
  }
  for (int ty = 0; ty < nty; ++ty) {
    for (int tx = 0; tx < ntx; ++tx) {
      std::vector<uint32_t>& L = lists[(size_t)ty * ntx + tx];
      if (L.empty()) continue;
      std::stable_sort(L.begin(), L.end(), [&](uint32_t a, uint32_t b) { return proj[a].depth < proj[b].depth; });
      const int px0 = tx * tw, py0 = ty * th, px1 = std::min(px0 + tw, width), py1 = std::min(py0 + th, height);
      for (uint32_t gi : L) {
        const Proj& g = proj[gi];
        const float det = g.cxx * g.cyy - g.cxy * g.cxy;
        if (det < 1e-10f) continue;
        const float inv_det = 1.0f / det;
        for (int py = py0; py < py1; ++py) {
          for (int px = px0; px < px1; ++px) {
            const size_t i = (size_t)py * width + px;
            if (alpha[i] >= 0.999f) continue;
            const float dx = g.x - ((float)px + 0.5f), dy = g.y - ((float)py + 0.5f);
            const float d2 = (g.cyy * dx * dx - 2.0f * g.cxy * dx * dy + g.cxx * dy * dy) * inv_det;
            if (!(d2 < 9.0f)) continue;
            const float w = std::exp(-0.5f * d2) * g.opacity;
            if (!(w > 0.001f)) continue;
            const float a = w * (1.0f - alpha[i]);
            if (!(a > 0.0f)) continue;
            color[i * 3 + 0] += g.rgb[0] * a;
            color[i * 3 + 1] += g.rgb[1] * a;
            color[i * 3 + 2] += g.rgb[2] * a;
            alpha[i] += a;
            if (depth[i] == FLT_MAX && a > 0.01f) depth[i] = g.depth;
          }
        }
      }
    }
  }
  for (size_t i = 0; i < alpha.size(); ++i) {
    const float tr = 1.0f - alpha[i];
    for (int ch = 0; ch < 3; ++ch) color[i * 3 + ch] = std::min(std::max(color[i * 3 + ch] + background[ch] * tr, 0.0f), 1.0f);
  }
}
