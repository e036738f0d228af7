// gsr_math.h — per-Gaussian EWA splatting math shared by the sm_100a kernels
// (compiled by nvcc as __device__ code) and by the CPU oracle (compiled by g++
// as host code, instantiated for float and double).
//
// Every expression here fixes its evaluation order explicitly (left to right,
// no implicit contraction: kernels build with --fmad=false, the oracle with
// -ffp-contract=off), so the GPU and the CPU evaluate identical expression
// trees and the integer outputs derived from them (visible set, tile counts,
// sort keys, per-pixel contributor counts) match bit for bit.
//
// The formulas restate RustGS/src/training/shaders/helpers.wgsl (cited per
// function). Matrices are column-major like WGSL: m[col][row].
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define GSR_HD __host__ __device__ __forceinline__
#else
#define GSR_HD inline
#include <cmath>
#include <cstring>
#endif

namespace gsr {

// ----------------------------------------------------------------------------
// Scalar primitives (float and double overloads).
// ----------------------------------------------------------------------------
GSR_HD float gmin(float a, float b) { return fminf(a, b); }
GSR_HD double gmin(double a, double b) { return fmin(a, b); }
GSR_HD float gmax(float a, float b) { return fmaxf(a, b); }
GSR_HD double gmax(double a, double b) { return fmax(a, b); }
GSR_HD float gsqrt(float a) { return sqrtf(a); }
GSR_HD double gsqrt(double a) { return sqrt(a); }
GSR_HD float gfma(float a, float b, float c) { return fmaf(a, b, c); }
GSR_HD double gfma(double a, double b, double c) { return fma(a, b, c); }
GSR_HD float gabs(float a) { return fabsf(a); }
GSR_HD double gabs(double a) { return fabs(a); }
template <class F> GSR_HD F clampf(F x, F lo, F hi) { return gmin(gmax(x, lo), hi); }
// Individually rounded float operations that no compiler may fuse into a
// multiply-add, for the expressions whose bits decide integer outputs (the
// blend decisions). Plain operators on the host, where the oracle is built
// with -ffp-contract=off.
GSR_HD float emul(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fmul_rn(a, b);
#else
  return a * b;
#endif
}
GSR_HD float eadd(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fadd_rn(a, b);
#else
  return a + b;
#endif
}
GSR_HD float esub(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fsub_rn(a, b);
#else
  return a - b;
#endif
}
GSR_HD double emul(double a, double b) { return a * b; }
GSR_HD double eadd(double a, double b) { return a + b; }
GSR_HD double esub(double a, double b) { return a - b; }

// 1/x correctly rounded (the same value as the IEEE division on the host).
GSR_HD float grcp(float x) {
#if defined(__CUDA_ARCH__)
  return __frcp_rn(x);
#else
  return 1.0f / x;
#endif
}
GSR_HD double grcp(double x) { return 1.0 / x; }

GSR_HD float bits_to_float(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, 4);
  return f;
#endif
}
GSR_HD uint32_t float_to_bits(float f) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
#endif
}

// exp for float: Cody & Waite (1980) additive range reduction x = n*ln2 + r
// with ln2 split into a short high part and a correction, then e^r by a
// degree-7 Taylor polynomial in Horner form (|r| <= ln2/2, truncation error
// < 0.1 ulp), then scaling by 2^n in two exact power-of-two steps. The same
// sequence of IEEE operations runs on host and device, so results agree bit
// for bit; accuracy is within 2 ulp of the true value (tested against a
// double-precision exp). Inputs below -87.3365 flush to 0.
GSR_HD float portable_expf(float x) {
  if (!(x > -87.3365f)) return (x != x) ? x : 0.0f;
  if (x > 88.7228f) return bits_to_float(0x7f800000u);
  const float n = rintf(x * 1.44269504088896341f);
  float r = fmaf(-n, 0.693145751953125f, x);  // ln2 high part (exact in 17 bits)
  r = fmaf(-n, 1.42860682030941723e-06f, r);  // ln2 - high part
  float p = 1.98412698412698413e-04f;          // 1/7!
  p = fmaf(p, r, 1.38888888888888889e-03f);    // 1/6!
  p = fmaf(p, r, 8.33333333333333333e-03f);    // 1/5!
  p = fmaf(p, r, 4.16666666666666667e-02f);    // 1/4!
  p = fmaf(p, r, 1.66666666666666667e-01f);    // 1/3!
  p = fmaf(p, r, 0.5f);                        // 1/2!
  p = fmaf(p, r, 1.0f);
  p = fmaf(p, r, 1.0f);
  const int ni = (int)n;
  const int n1 = ni >> 1;
  const int n2 = ni - n1;
  p = p * bits_to_float((uint32_t)(n1 + 127) << 23);
  return p * bits_to_float((uint32_t)(n2 + 127) << 23);
}

// natural log for float: x = 2^e * m with m in [sqrt(1/2), sqrt(2)),
// log(m) = 2*atanh(s), s = (m-1)/(m+1), by the odd series
// 2(s + s^3/3 + s^5/5 + s^7/7 + s^9/9) (|s| <= 0.1716, truncation < 1e-9
// relative), then log(x) = e*ln2 + log(m) with the split ln2 of
// portable_expf. Within 2 ulp of the true value away from x == 1 and with
// small absolute error near it (tested against a double-precision log).
GSR_HD float portable_logf(float x) {
  if (!(x > 0.0f)) return (x == 0.0f) ? bits_to_float(0xff800000u) : bits_to_float(0x7fc00000u);
  if (x == bits_to_float(0x7f800000u)) return x;
  int eadj = 0;
  if (x < 1.17549435e-38f) {
    x = x * 8388608.0f;  // 2^23, exact
    eadj = -23;
  }
  const uint32_t b = float_to_bits(x);
  int e = (int)((b >> 23) & 0xffu) - 127;
  float m = bits_to_float((b & 0x007fffffu) | 0x3f800000u);
  if (m > 1.41421356237309505f) {
    m = m * 0.5f;
    e = e + 1;
  }
  const float f = m - 1.0f;
  const float s = f / (2.0f + f);
  const float s2 = s * s;
  float p = fmaf(s2, 1.11111111111111111e-01f, 1.42857142857142857e-01f);  // 1/9, 1/7
  p = fmaf(p, s2, 2.0e-01f);                                               // 1/5
  p = fmaf(p, s2, 3.33333333333333333e-01f);                               // 1/3
  const float two_s = s + s;
  const float lm = fmaf(two_s * s2, p, two_s);
  const float ef = (float)(e + eadj);
  return fmaf(ef, 0.693145751953125f, fmaf(ef, 1.42860682030941723e-06f, lm));
}

GSR_HD float gexp(float x) { return portable_expf(x); }
GSR_HD double gexp(double x) { return exp(x); }
GSR_HD float glog(float x) { return portable_logf(x); }
GSR_HD double glog(double x) { return log(x); }

// Integer power by binary exponentiation in float, the way Rust's f32::powi
// is evaluated for the Adam bias corrections (engine/optimizer.rs:146-147).
GSR_HD float powi_f32(float b, int e) {
  float r = 1.0f, x = b;
  unsigned n = (unsigned)(e < 0 ? -e : e);
  while (n) {
    if (n & 1u) r = r * x;
    n >>= 1;
    if (n) x = x * x;
  }
  return e < 0 ? 1.0f / r : r;
}

// helpers.wgsl:52-54
template <class F> GSR_HD F sigmoid(F x) { return F(1) / (F(1) + gexp(-x)); }

// ----------------------------------------------------------------------------
// Small vectors and column-major matrices.
// ----------------------------------------------------------------------------
template <class F> struct V2 { F x, y; };
template <class F> struct V3 { F x, y, z; };
template <class F> struct V4 { F x, y, z, w; };
// C columns of R rows; m[c][r].
template <class F, int C, int R> struct Mat { F m[C][R]; };
template <class F> using M2 = Mat<F, 2, 2>;
template <class F> using M3 = Mat<F, 3, 3>;
template <class F> using M32 = Mat<F, 3, 2>;  // WGSL mat3x2: 3 columns, 2 rows

// (A * B)[j][i] = sum_k A[k][i] * B[j][k], accumulated left to right.
template <class F, int K, int R, int C>
GSR_HD Mat<F, C, R> mul(const Mat<F, K, R>& a, const Mat<F, C, K>& b) {
  Mat<F, C, R> o;
  for (int j = 0; j < C; ++j)
    for (int i = 0; i < R; ++i) {
      F s = a.m[0][i] * b.m[j][0];
      for (int k = 1; k < K; ++k) s = s + a.m[k][i] * b.m[j][k];
      o.m[j][i] = s;
    }
  return o;
}
template <class F, int C, int R> GSR_HD Mat<F, R, C> transpose(const Mat<F, C, R>& a) {
  Mat<F, R, C> o;
  for (int c = 0; c < C; ++c)
    for (int r = 0; r < R; ++r) o.m[r][c] = a.m[c][r];
  return o;
}
template <class F, int C, int R> GSR_HD Mat<F, C, R> add(const Mat<F, C, R>& a, const Mat<F, C, R>& b) {
  Mat<F, C, R> o;
  for (int c = 0; c < C; ++c)
    for (int r = 0; r < R; ++r) o.m[c][r] = a.m[c][r] + b.m[c][r];
  return o;
}
// mat * vec for a 3x3 matrix: out[i] = sum_k m[k][i] * v[k], left to right.
template <class F> GSR_HD V3<F> mulv(const M3<F>& a, V3<F> v) {
  V3<F> o;
  o.x = a.m[0][0] * v.x + a.m[1][0] * v.y + a.m[2][0] * v.z;
  o.y = a.m[0][1] * v.x + a.m[1][1] * v.y + a.m[2][1] * v.z;
  o.z = a.m[0][2] * v.x + a.m[1][2] * v.y + a.m[2][2] * v.z;
  return o;
}
template <class F> GSR_HD F det2(const M2<F>& a) { return a.m[0][0] * a.m[1][1] - a.m[0][1] * a.m[1][0]; }

// ----------------------------------------------------------------------------
// Camera (per view) in the precision F.
// viewmat is the column-major world->camera matrix; the rotation is its upper
// 3x3 block and the translation its fourth column (helpers.wgsl:7-18).
// ----------------------------------------------------------------------------
template <class F> struct Cam {
  M3<F> rot;
  V3<F> trans;
  V2<F> focal;
  V2<F> pc;  // principal point (pixel_center)
  uint32_t w, h;
  V3<F> campos;
};

// (viewmat * vec4(mean, 1)).xyz with the products summed left to right
// (project_forward.wgsl:33); the final "+ t * 1.0" is exact.
template <class F> GSR_HD V3<F> world_to_cam(const Cam<F>& c, V3<F> p) {
  V3<F> o = mulv(c.rot, p);
  o.x = o.x + c.trans.x;
  o.y = o.y + c.trans.y;
  o.z = o.z + c.trans.z;
  return o;
}

// helpers.wgsl:56-77, quaternion (w, x, y, z) -> rotation matrix.
template <class F> GSR_HD M3<F> quat_to_mat3(V4<F> q) {
  const F w = q.x, x = q.y, y = q.z, z = q.w;
  const F x2 = x * x, y2 = y * y, z2 = z * z;
  const F xy = x * y, xz = x * z, yz = y * z;
  const F wx = w * x, wy = w * y, wz = w * z;
  M3<F> r;
  r.m[0][0] = F(1) - F(2) * (y2 + z2);
  r.m[0][1] = F(2) * (xy + wz);
  r.m[0][2] = F(2) * (xz - wy);
  r.m[1][0] = F(2) * (xy - wz);
  r.m[1][1] = F(1) - F(2) * (x2 + z2);
  r.m[1][2] = F(2) * (yz + wx);
  r.m[2][0] = F(2) * (xz + wy);
  r.m[2][1] = F(2) * (yz - wx);
  r.m[2][2] = F(1) - F(2) * (x2 + y2);
  return r;
}

// R * diag(s): column j scaled by s_j (helpers.wgsl:128-136; the zero terms of
// the full product are exact and are skipped).
template <class F> GSR_HD M3<F> rot_scale(const M3<F>& r, V3<F> s) {
  M3<F> m;
  const F sv[3] = {s.x, s.y, s.z};
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) m.m[j][i] = r.m[j][i] * sv[j];
  return m;
}

// helpers.wgsl:138-154. The limits follow the WGSL expression exactly.
template <class F> GSR_HD M32<F> calc_cam_j(V3<F> mc, const Cam<F>& c) {
  const F limx_pos = (F(1.15) * F(c.w) - c.pc.x) / c.focal.x;
  const F limy_pos = (F(1.15) * F(c.h) - c.pc.y) / c.focal.y;
  const F limx_neg = (F(-0.15) * F(c.w) - c.pc.x) / c.focal.x;
  const F limy_neg = (F(-0.15) * F(c.h) - c.pc.y) / c.focal.y;
  const F rz = F(1) / gmax(mc.z, F(0.01));
  const F u = clampf(mc.x * rz, limx_neg, limx_pos);
  const F v = clampf(mc.y * rz, limy_neg, limy_pos);
  const F dx = c.focal.x * rz, dy = c.focal.y * rz;
  M32<F> j;
  j.m[0][0] = dx;
  j.m[0][1] = F(0);
  j.m[1][0] = F(0);
  j.m[1][1] = dy;
  j.m[2][0] = -dx * u;
  j.m[2][1] = -dy * v;
  return j;
}

// helpers.wgsl:170-183. Returns the opacity compensation and adds the blur.
template <class F> GSR_HD F compensate_cov2d(M2<F>& cov, F blur) {
  const M2<F> start = cov;
  cov.m[0][0] = cov.m[0][0] + blur;
  cov.m[1][1] = cov.m[1][1] + blur;
  const F det_raw = gmax(det2(start), F(0));
  const F det_end = gmax(det2(cov), F(1e-12));
  if (det_raw <= F(0)) return F(0);
  return gsqrt(det_raw / det_end);
}

// helpers.wgsl:185-198. Packed conic (a, b, c) = (inv[0][0], inv[0][1], inv[1][1]).
template <class F> GSR_HD V3<F> inverse2x2_packed(const M2<F>& m) {
  const F a = m.m[0][0] + F(1e-6);
  const F d = m.m[1][1] + F(1e-6);
  const F b = m.m[0][1];
  const F det = a * d - b * m.m[1][0];
  V3<F> o;
  if (det <= F(1e-10)) {
    o.x = o.y = o.z = F(0);
    return o;
  }
  const F inv = F(1) / det;
  o.x = d * inv;
  o.y = -b * inv;
  o.z = a * inv;
  return o;
}

// FP64 variants of the compensation and the inversion for float inputs,
// used for near-degenerate (flattened) covariances where the float
// determinant a*d - b*c cancels catastrophically. The float matrix is
// widened, the determinants and the inverse are formed in double, and the
// results are rounded once to float. For double inputs they are the plain
// functions.
GSR_HD float compensate_cov2d_hp(M2<float>& cov, float blur) {
  const double a = cov.m[0][0], b = cov.m[0][1], c = cov.m[1][0], d = cov.m[1][1];
  cov.m[0][0] = cov.m[0][0] + blur;
  cov.m[1][1] = cov.m[1][1] + blur;
  const double det_raw = fmax(a * d - b * c, 0.0);
  const double det_end = fmax((double)cov.m[0][0] * (double)cov.m[1][1] - b * c, 1e-12);
  if (det_raw <= 0.0) return 0.0f;
  return (float)sqrt(det_raw / det_end);
}
GSR_HD double compensate_cov2d_hp(M2<double>& cov, double blur) { return compensate_cov2d(cov, blur); }
GSR_HD V3<float> inverse2x2_packed_hp(const M2<float>& m) {
  const double a = (double)m.m[0][0] + 1e-6, d = (double)m.m[1][1] + 1e-6, b = m.m[0][1];
  const double det = a * d - b * (double)m.m[1][0];
  V3<float> o;
  if (det <= 1e-10) {
    o.x = o.y = o.z = 0.0f;
    return o;
  }
  const double inv = 1.0 / det;
  o.x = (float)(d * inv);
  o.y = (float)(-b * inv);
  o.z = (float)(a * inv);
  return o;
}
GSR_HD V3<double> inverse2x2_packed_hp(const M2<double>& m) { return inverse2x2_packed(m); }

// helpers.wgsl:218-224.
template <class F> GSR_HD V2<F> bbox_extent(const M2<F>& cov, F thr) {
  const F sp = gmax(thr, F(0));
  V2<F> e;
  e.x = gsqrt(gmax(F(0), F(2) * sp * cov.m[0][0]));
  e.y = gsqrt(gmax(F(0), F(2) * sp * cov.m[1][1]));
  return e;
}

// Tile grid shape. The reference hard-wires 16x16 (helpers.wgsl:3-4); the
// shape is a parameter here and 16x16 reproduces the reference.
struct TileShape {
  uint32_t tw, th;
};

struct TileBox {
  uint32_t x0, y0, x1, y1;  // [x0, x1) x [y0, y1) in tile units
};

// helpers.wgsl:204-216 generalised to tw x th tiles.
template <class F>
GSR_HD TileBox tile_bbox(V2<F> center, V2<F> ext, TileShape ts, uint32_t tiles_x, uint32_t tiles_y) {
  const F cx = center.x / F(ts.tw), cy = center.y / F(ts.th);
  const F ex = ext.x / F(ts.tw), ey = ext.y / F(ts.th);
  TileBox b;
  b.x0 = (uint32_t)clampf(cx - ex, F(0), F(tiles_x));
  b.y0 = (uint32_t)clampf(cy - ey, F(0), F(tiles_y));
  b.x1 = (uint32_t)clampf(cx + ex + F(1), F(0), F(tiles_x));
  b.y1 = (uint32_t)clampf(cy + ey + F(1), F(0), F(tiles_y));
  return b;
}

// helpers.wgsl:232-235 (forward form, also used by rasterize.wgsl:67-72):
// 0.5 * (a*dx*dx + 2*b*dx*dy + c*dy*dy) with delta = point - mean.
template <class F> GSR_HD F calc_sigma(F px, F py, V3<F> conic, V2<F> mean) {
  const F dx = px - mean.x, dy = py - mean.y;
  return F(0.5) * (conic.x * dx * dx + F(2) * conic.y * dx * dy + conic.z * dy * dy);
}

// helpers.wgsl:237-283 for the tile (tx, ty) of a tw x th grid.
template <class F>
GSR_HD bool will_primitive_contribute(uint32_t tx, uint32_t ty, TileShape ts, V2<F> mean, V3<F> conic, F thr) {
  const F rx0 = F(tx * ts.tw), ry0 = F(ty * ts.th);
  const F rx1 = rx0 + F(ts.tw), ry1 = ry0 + F(ts.th);
  const bool x_left = mean.x < rx0;
  const bool x_right = mean.x > rx1;
  const bool in_x = !(x_left || x_right);
  const bool y_above = mean.y < ry0;
  const bool y_below = mean.y > ry1;
  const bool in_y = !(y_above || y_below);
  if (in_x && in_y) return true;
  const F ccx = x_left ? rx0 : rx1;
  const F ccy = y_above ? ry0 : ry1;
  const F width = rx1 - rx0, height = ry1 - ry0;
  const F dxv = x_left ? width : -width;
  const F dyv = y_above ? height : -height;
  const F diffx = mean.x - ccx, diffy = mean.y - ccy;
  F tmx = F(0), tmy = F(0);
  if (!in_y)
    tmx = clampf((dxv * conic.x * diffx + dxv * conic.y * diffy) / gmax(dxv * conic.x * dxv, F(1e-12)), F(0), F(1));
  if (!in_x)
    tmy = clampf((dyv * conic.y * diffx + dyv * conic.z * diffy) / gmax(dyv * conic.z * dyv, F(1e-12)), F(0), F(1));
  const F mpx = ccx + tmx * dxv, mpy = ccy + tmy * dyv;
  return calc_sigma(mpx, mpy, conic, mean) <= thr;
}

// ----------------------------------------------------------------------------
// Spherical harmonics (project_visible.wgsl:44-127 and helpers.wgsl:289-380).
// ----------------------------------------------------------------------------
GSR_HD constexpr int num_sh_coeffs(int degree) { return (degree + 1) * (degree + 1); }

// Basis values b[0..K) for the view direction, expression order as in the
// WGSL colour accumulation. Templated on the scalar so that a dual number can
// carry the direction derivatives (sh_basis_grad).
template <class S> GSR_HD void sh_basis(int degree, S x, S y, S z, S* b) {
  b[0] = S(0.28209479177387814);
  if (degree == 0) return;
  const S a = S(0.48860251190292);
  b[1] = -a * y;
  b[2] = a * z;
  b[3] = -a * x;
  if (degree == 1) return;
  const S z2 = z * z;
  const S t0b = S(-1.092548430592079) * z;
  const S t1a = S(0.5462742152960395);
  const S c1 = x * x - y * y;
  const S s1 = S(2) * x * y;
  b[6] = S(0.9461746957575601) * z2 - S(0.3153915652525201);
  b[7] = t0b * x;
  b[5] = t0b * y;
  b[8] = t1a * c1;
  b[4] = t1a * s1;
  if (degree == 2) return;
  const S t0c = S(-2.285228997322329) * z2 + S(0.4570457994644658);
  const S t1b = S(1.445305721320277) * z;
  const S t2a = S(-0.5900435899266435);
  const S c2 = x * c1 - y * s1;
  const S s2 = x * s1 + y * c1;
  b[12] = z * (S(1.865881662950577) * z2 - S(1.119528997770346));
  b[13] = t0c * x;
  b[11] = t0c * y;
  b[14] = t1b * c1;
  b[10] = t1b * s1;
  b[15] = t2a * c2;
  b[9] = t2a * s2;
  if (degree == 3) return;
  const S t0d = z * (S(-4.683325804901025) * z2 + S(2.007139630671868));
  const S t1c = S(3.31161143515146) * z2 - S(0.47308734787878);
  const S t2b = S(-1.770130769779931) * z;
  const S t3a = S(0.6258357354491763);
  const S c3 = x * c2 - y * s2;
  const S s3 = x * s2 + y * c2;
  b[20] = S(1.984313483298443) * z * b[12] - S(1.006230589874905) * b[6];
  b[21] = t0d * x;
  b[19] = t0d * y;
  b[22] = t1c * c1;
  b[18] = t1c * s1;
  b[23] = t2b * c2;
  b[17] = t2b * s2;
  b[24] = t3a * c3;
  b[16] = t3a * s3;
}

// Colour = sum_k b_k * coeff_k, accumulated band by band in the WGSL order
// (project_visible.wgsl:44-127), then + 0.5 (project_visible.wgsl:208).
// coeff(k, ch) is a functor returning the coefficient as F.
template <class F, class Coeff> GSR_HD V3<F> sh_to_color(int degree, V3<F> dir, const Coeff& coeff) {
  F b[25] = {};
  sh_basis<F>(degree, dir.x, dir.y, dir.z, b);
  V3<F> col;
  F* cp[3] = {&col.x, &col.y, &col.z};
  for (int ch = 0; ch < 3; ++ch) {
    F c = b[0] * coeff(0, ch);
    if (degree >= 1) {
      // fTmp0A * (-y*c1 + z*c2 - x*c3): basis values are (-A y, A z, -A x); the
      // WGSL groups the three products before scaling by A.
      const F a = F(0.48860251190292);
      const F y = dir.y, z = dir.z, x = dir.x;
      c = c + a * (-y * coeff(1, ch) + z * coeff(2, ch) - x * coeff(3, ch));
    }
    if (degree >= 2) c = c + (b[4] * coeff(4, ch) + b[5] * coeff(5, ch) + b[6] * coeff(6, ch) + b[7] * coeff(7, ch) + b[8] * coeff(8, ch));
    if (degree >= 3)
      c = c + (b[9] * coeff(9, ch) + b[10] * coeff(10, ch) + b[11] * coeff(11, ch) + b[12] * coeff(12, ch) +
               b[13] * coeff(13, ch) + b[14] * coeff(14, ch) + b[15] * coeff(15, ch));
    if (degree >= 4)
      c = c + (b[16] * coeff(16, ch) + b[17] * coeff(17, ch) + b[18] * coeff(18, ch) + b[19] * coeff(19, ch) +
               b[20] * coeff(20, ch) + b[21] * coeff(21, ch) + b[22] * coeff(22, ch) + b[23] * coeff(23, ch) +
               b[24] * coeff(24, ch));
    *cp[ch] = c + F(0.5);
  }
  return col;
}

// Forward-mode dual number with three partials, used to differentiate the SH
// basis with respect to the view direction.
template <class F> struct Dual3 {
  F v, d[3];
  GSR_HD Dual3() : v(0), d{0, 0, 0} {}
  GSR_HD Dual3(F c) : v(c), d{0, 0, 0} {}
};
template <class F> GSR_HD Dual3<F> operator+(const Dual3<F>& a, const Dual3<F>& b) {
  Dual3<F> o;
  o.v = a.v + b.v;
  for (int i = 0; i < 3; ++i) o.d[i] = a.d[i] + b.d[i];
  return o;
}
template <class F> GSR_HD Dual3<F> operator-(const Dual3<F>& a, const Dual3<F>& b) {
  Dual3<F> o;
  o.v = a.v - b.v;
  for (int i = 0; i < 3; ++i) o.d[i] = a.d[i] - b.d[i];
  return o;
}
template <class F> GSR_HD Dual3<F> operator-(const Dual3<F>& a) {
  Dual3<F> o;
  o.v = -a.v;
  for (int i = 0; i < 3; ++i) o.d[i] = -a.d[i];
  return o;
}
template <class F> GSR_HD Dual3<F> operator*(const Dual3<F>& a, const Dual3<F>& b) {
  Dual3<F> o;
  o.v = a.v * b.v;
  for (int i = 0; i < 3; ++i) o.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return o;
}

// Basis values and their gradients with respect to (x, y, z).
template <class F> GSR_HD void sh_basis_grad(int degree, V3<F> dir, F* b, F (*db)[3]) {
  Dual3<F> x(dir.x), y(dir.y), z(dir.z);
  x.d[0] = F(1);
  y.d[1] = F(1);
  z.d[2] = F(1);
  Dual3<F> bd[25];
  sh_basis<Dual3<F>>(degree, x, y, z, bd);
  const int k = num_sh_coeffs(degree);
  for (int i = 0; i < k; ++i) {
    b[i] = bd[i].v;
    db[i][0] = bd[i].d[0];
    db[i][1] = bd[i].d[1];
    db[i][2] = bd[i].d[2];
  }
}

// ----------------------------------------------------------------------------
// Projection of one Gaussian (project_forward.wgsl:19-96 and
// project_visible.wgsl:130-214, computed once).
// ----------------------------------------------------------------------------
template <class F> struct Projected {
  bool visible;
  F depth;     // camera-space z
  V2<F> mean2d;
  V3<F> conic;
  F opacity;   // sigmoid(raw) * compensation
  F thr;       // log(255 * opacity), the contribution power threshold
  TileBox box;
};

// Geometric part of the projection. The quaternion is normalised by the
// reciprocal square root of its squared norm (project_forward.wgsl:38-42).
// The view-independent part: the 3D covariance from the normalised
// quaternion and the scales, and the opacity (ok = false for a degenerate
// quaternion, which no view projects).
template <class F> struct GaussWorld {
  M3<F> cov3d;
  F opacity;
  bool ok;
};
template <class F>
GSR_HD GaussWorld<F> gauss_world(V4<F> quat, V3<F> log_scale, F raw_opac) {
  GaussWorld<F> w;
  const F qn = quat.x * quat.x + quat.y * quat.y + quat.z * quat.z + quat.w * quat.w;
  w.ok = !(qn < F(1e-6));
  const F rs = F(1) / gsqrt(w.ok ? qn : F(1));
  quat.x = quat.x * rs;
  quat.y = quat.y * rs;
  quat.z = quat.z * rs;
  quat.w = quat.w * rs;
  V3<F> scale;
  scale.x = gexp(log_scale.x);
  scale.y = gexp(log_scale.y);
  scale.z = gexp(log_scale.z);
  w.opacity = sigmoid(raw_opac);
  const M3<F> m = rot_scale(quat_to_mat3(quat), scale);
  w.cov3d = mul(m, transpose(m));
  return w;
}

// project_gaussian with the view-independent part computed once (kernels
// that project one Gaussian into many views).
template <class F>
GSR_HD Projected<F> project_gaussian_w(const Cam<F>& cam, V3<F> mean, const GaussWorld<F>& gw, F cov_blur,
                                       TileShape ts, uint32_t tiles_x, uint32_t tiles_y, bool hp = false) {
  Projected<F> p;
  p.visible = false;
  const V3<F> mc = world_to_cam(cam, mean);
  p.depth = mc.z;
  if (mc.z < F(0.01) || mc.z > F(1e10)) return p;
  if (!gw.ok) return p;
  F opacity = gw.opacity;
  const M3<F> cov_cam = mul(mul(cam.rot, gw.cov3d), transpose(cam.rot));
  const M32<F> j = calc_cam_j(mc, cam);
  M2<F> cov2d = mul(mul(j, cov_cam), transpose(j));
  opacity = opacity * (hp ? compensate_cov2d_hp(cov2d, cov_blur) : compensate_cov2d(cov2d, cov_blur));
  if (opacity < F(1.0 / 255.0)) return p;
  const F rz = F(1) / mc.z;
  V2<F> mean2d;
  mean2d.x = cam.focal.x * mc.x * rz + cam.pc.x;
  mean2d.y = cam.focal.y * mc.y * rz + cam.pc.y;
  const V3<F> conic = hp ? inverse2x2_packed_hp(cov2d) : inverse2x2_packed(cov2d);
  const F thr = glog(opacity * F(255));
  const V2<F> ext = bbox_extent(cov2d, thr);
  if (ext.x < F(0) || ext.y < F(0)) return p;
  if (mean2d.x + ext.x <= F(0) || mean2d.x - ext.x >= F(cam.w) || mean2d.y + ext.y <= F(0) ||
      mean2d.y - ext.y >= F(cam.h))
    return p;
  p.visible = true;
  p.mean2d = mean2d;
  p.conic = conic;
  p.opacity = opacity;
  p.thr = thr;
  p.box = tile_bbox(mean2d, ext, ts, tiles_x, tiles_y);
  return p;
}

template <class F>
GSR_HD Projected<F> project_gaussian(const Cam<F>& cam, V3<F> mean, V4<F> quat, V3<F> log_scale, F raw_opac,
                                     F cov_blur, TileShape ts, uint32_t tiles_x, uint32_t tiles_y,
                                     bool hp = false) {
  return project_gaussian_w(cam, mean, gauss_world(quat, log_scale, raw_opac), cov_blur, ts, tiles_x, tiles_y, hp);
}

// Number of tiles of the box that pass the contribution test, visited in
// row-major order (project_forward.wgsl:75-89).
template <class F> GSR_HD uint32_t count_tiles(const Projected<F>& p, TileShape ts) {
  uint32_t n = 0;
  for (uint32_t ty = p.box.y0; ty < p.box.y1; ++ty)
    for (uint32_t tx = p.box.x0; tx < p.box.x1; ++tx)
      if (will_primitive_contribute(tx, ty, ts, p.mean2d, p.conic, p.thr)) ++n;
  return n;
}

// View direction for SH (project_visible.wgsl:168-169).
template <class F> GSR_HD V3<F> view_dir(const Cam<F>& cam, V3<F> mean) {
  V3<F> d;
  d.x = mean.x - cam.campos.x;
  d.y = mean.y - cam.campos.y;
  d.z = mean.z - cam.campos.z;
  const F n2 = d.x * d.x + d.y * d.y + d.z * d.z;
  const F r = F(1) / gsqrt(gmax(n2, F(1e-12)));
  d.x = d.x * r;
  d.y = d.y * r;
  d.z = d.z * r;
  return d;
}

// ----------------------------------------------------------------------------
// Per-pixel blend step (rasterize.wgsl:65-85).
// ----------------------------------------------------------------------------
// sigma = 0.5 * (a*dx*dx + 2*b*dx*dy + c*dy*dy) with d = mean - pixel centre,
// evaluated left to right with the two multiply-adds contracted, as WGSL
// lets an implementation do: t1 = (a*dx)*dx and t2 = (2b)*dx, then
// 0.5 * fma((c*dy), dy, fma(t2, dy, t1)). Every other operation is rounded on
// its own. The fused form is spelled out (fmaf on the host, the same fused
// operation on the device), so host and device agree bit for bit whatever
// the compiler contracts; it also lets the kernels run a pixel pair's sigma
// as paired fused multiply-adds. blend_sigma_shared takes the per-column
// terms t1 and t2 precomputed (kernels share them between the pixels of a
// column).
template <class F> GSR_HD F blend_sigma_shared(F t1, F t2, F dy, F cc) {
  return emul(F(0.5), gfma(emul(cc, dy), dy, gfma(t2, dy, t1)));
}
template <class F> GSR_HD F blend_sigma(F dx, F dy, F ca, F cb, F cc) {
  return blend_sigma_shared(emul(emul(ca, dx), dx), emul(emul(F(2), cb), dx), dy, cc);
}

// exp(x) for the blend, where x = -sigma <= 0 matters (x > 0 only occurs
// for sigma < 0, which the contribution test rejects whatever the value):
// the Cody-Waite reduction of portable_expf and a degree-6 polynomial (one
// multiply-add fewer than portable_expf's Taylor form), with n = round(x*log2(e))
// taken by one fused multiply-add of 1.5*2^23 (round-to-nearest-even of the
// exact product, for |x*log2e| < 2^22; its integer then sits in the low
// mantissa bits) and the scaling by 2^n done by adding n to the exponent
// field, exact because the result stays a normal number for x >= -87.33.
// Same IEEE operations on host and device.
// Constants of blend_expf (shared with the paired device version).
namespace bexp {
constexpr float kLog2e = 1.44269504088896341f;
constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23
constexpr uint32_t kMagicBits = 0x4B400000u;
constexpr float kLn2Hi = 0.693145751953125f;
constexpr float kLn2Lo = 1.42860682030941723e-06f;
// exp(r) ~ 1 + r + r^2 (kC2 + r (kC3 + r (kC4 + r (kC5 + r kC6)))) on
// [-ln2/2, ln2/2]: coefficients fitted for minimal relative error
// (iteratively reweighted least squares, 3.1e-9 before rounding to float);
// the whole float evaluation is within 0.87 ulp of exp over x in [-87, 0].
constexpr float kC6 = 1.381453942e-03f;
constexpr float kC5 = 8.368745446e-03f;
constexpr float kC4 = 4.166838899e-02f;
constexpr float kC3 = 1.666652113e-01f;
constexpr float kC2 = 4.999999404e-01f;
constexpr float kLow = -87.3365f;                 // below: the result would not be normal
}  // namespace bexp

GSR_HD float blend_expf(float x) {
  x = fminf(x, 0.0f);
  if (!(x > bexp::kLow)) return (x != x) ? x : 0.0f;
  const float t = fmaf(x, bexp::kLog2e, bexp::kMagic);
  const float n = esub(t, bexp::kMagic);
  const int ni = (int)(float_to_bits(t) - bexp::kMagicBits);
  float r = fmaf(-n, bexp::kLn2Hi, x);
  r = fmaf(-n, bexp::kLn2Lo, r);
  float p = bexp::kC6;
  p = fmaf(p, r, bexp::kC5);
  p = fmaf(p, r, bexp::kC4);
  p = fmaf(p, r, bexp::kC3);
  p = fmaf(p, r, bexp::kC2);
  p = fmaf(p, r, 1.0f);
  p = fmaf(p, r, 1.0f);
  return bits_to_float(float_to_bits(p) + ((uint32_t)ni << 23));
}
GSR_HD double blend_expf(double x) { return exp(x); }

// alpha = min(0.999, opac * exp(-sigma)); returns it when the Gaussian
// contributes (sigma >= 0 and alpha >= 1/255), else -1. gauss = exp(-sigma).
template <class F> GSR_HD F blend_alpha_of(F sigma, F opac, F& gauss) {
  gauss = blend_expf(-sigma);
  const F alpha = gmin(F(0.999), emul(opac, gauss));
  if (sigma >= F(0) && alpha >= F(1.0 / 255.0)) return alpha;
  return F(-1);
}
template <class F> GSR_HD F blend_alpha(F px, F py, F mx, F my, F ca, F cb, F cc, F opac, F& gauss) {
  return blend_alpha_of(blend_sigma(mx - px, my - py, ca, cb, cc), opac, gauss);
}
// Colour accumulation C += max(c, 0) * w as one fused multiply-add.
template <class F> GSR_HD F blend_accum(F C, F c, F w) { return gfma(gmax(c, F(0)), w, C); }

// Padded half-widths of the box around the ellipse {0.5 d^T C d <= cut}
// (C = conic): sqrt(2 cut (C^-1)_ii), determinant in double, widened by 0.1%
// plus 0.01 px so that float rounding can never put a pixel of the true
// ellipse outside it. Returns false (no box) for non-positive-definite
// conics or non-finite input.
GSR_HD bool footprint_box(float a, float b, float c, float cut, float& rx, float& ry) {
  const double det = (double)a * (double)c - (double)b * (double)b;
  if (!(det > 0.0) || !(a > 0.0f) || !(c > 0.0f) || !(cut > 0.0f)) return false;
  const double q = 2.0 * (double)cut / det;
  rx = (float)(sqrt(q * (double)c) * 1.001 + 0.01);
  ry = (float)(sqrt(q * (double)a) * 1.001 + 0.01);
  return rx == rx && ry == ry && rx < 3.0e38f && ry < 3.0e38f;
}

// A Gaussian whose sigma exceeds log(255 * opac) + kRejectMargin cannot pass
// the alpha >= 1/255 test: its exact alpha is below (1/255) * exp(-1e-3),
// far outside the few-ulp error of the float exp and log. Kernels use this
// to skip the exponential without changing any decision.
constexpr float kRejectMargin = 1e-3f;

// ----------------------------------------------------------------------------
// Backward helpers (helpers.wgsl:79-118, 200-202, 382-427).
// ----------------------------------------------------------------------------

// helpers.wgsl:79-102: gradient of quat_to_mat3 with respect to (w, x, y, z).
template <class F> GSR_HD V4<F> quat_to_mat3_vjp(V4<F> q, const M3<F>& v) {
  const F w = q.x, x = q.y, y = q.z, z = q.w;
  V4<F> o;
  o.x = x * (v.m[1][2] - v.m[2][1]) + y * (v.m[2][0] - v.m[0][2]) + z * (v.m[0][1] - v.m[1][0]);
  o.y = F(-2) * x * (v.m[1][1] + v.m[2][2]) + y * (v.m[0][1] + v.m[1][0]) + z * (v.m[0][2] + v.m[2][0]) +
        w * (v.m[1][2] - v.m[2][1]);
  o.z = x * (v.m[0][1] + v.m[1][0]) - F(2) * y * (v.m[0][0] + v.m[2][2]) + z * (v.m[1][2] + v.m[2][1]) +
        w * (v.m[2][0] - v.m[0][2]);
  o.w = x * (v.m[0][2] + v.m[2][0]) + y * (v.m[1][2] + v.m[2][1]) - F(2) * z * (v.m[0][0] + v.m[1][1]) +
        w * (v.m[0][1] - v.m[1][0]);
  o.x = o.x * F(2);
  o.y = o.y * F(2);
  o.z = o.z * F(2);
  o.w = o.w * F(2);
  return o;
}

// helpers.wgsl:104-118 applied to a vector: d(v/|v|)^T * g.
template <class F> GSR_HD V4<F> normalize_vjp_apply(V4<F> v, V4<F> g) {
  const F sx = v.x * v.x, sy = v.y * v.y, sz = v.z * v.z, sw = v.w * v.w;
  const F l2 = v.x * v.x + v.y * v.y + v.z * v.z + v.w * v.w;
  const F l = gsqrt(gmax(l2, F(1e-20)));
  const F ccx = -v.x * v.y, ccy = -v.y * v.z, ccz = -v.z * v.x;  // -v.xyz * v.yzx
  const F csx = -v.x * v.w, csy = -v.y * v.w, csz = -v.z * v.w;  // -v.xyz * v.w
  const F k = F(1) / (l * l2);
  // Columns of the symmetric WGSL matrix; mat * vec sums column_i * g_i.
  const F c0[4] = {l2 - sx, ccx, ccz, csx};
  const F c1[4] = {ccx, l2 - sy, ccy, csy};
  const F c2[4] = {ccz, ccy, l2 - sz, csz};
  const F c3[4] = {csx, csy, csz, l2 - sw};
  F o[4];
  for (int i = 0; i < 4; ++i) o[i] = (c0[i] * k) * g.x + (c1[i] * k) * g.y + (c2[i] * k) * g.z + (c3[i] * k) * g.w;
  V4<F> r;
  r.x = o[0];
  r.y = o[1];
  r.z = o[2];
  r.w = o[3];
  return r;
}

// Full 2x2 inverse of helpers.wgsl:185-198 (both off-diagonals use m_reg[0][1]).
template <class F> GSR_HD M2<F> inverse2x2(const M2<F>& m) {
  const V3<F> c = inverse2x2_packed(m);
  M2<F> o;
  o.m[0][0] = c.x;
  o.m[0][1] = c.y;
  o.m[1][0] = c.y;
  o.m[1][1] = c.z;
  return o;
}

// helpers.wgsl:200-202: -m_inv * v * m_inv.
template <class F> GSR_HD M2<F> inverse2x2_vjp(const M2<F>& mi, const M2<F>& v) {
  M2<F> n;
  n.m[0][0] = -mi.m[0][0];
  n.m[0][1] = -mi.m[0][1];
  n.m[1][0] = -mi.m[1][0];
  n.m[1][1] = -mi.m[1][1];
  return mul(mul(n, v), mi);
}

// helpers.wgsl:382-427: gradient of (mean2d, cov2d) with respect to the
// camera-space mean, with the Jacobian clip branches.
template <class F>
GSR_HD V3<F> persp_proj_vjp(const M32<F>& j, V3<F> mc, const M3<F>& cov, const Cam<F>& c, const M2<F>& v_cov2d,
                            V2<F> v_mean2d) {
  const F x = mc.x, y = mc.y, z = mc.z;
  const F rz = F(1) / gmax(gabs(z), F(0.01));
  const F rz2 = rz * rz;
  V3<F> o;
  o.x = c.focal.x * rz * v_mean2d.x;
  o.y = c.focal.y * rz * v_mean2d.y;
  o.z = -(c.focal.x * x * v_mean2d.x + c.focal.y * y * v_mean2d.y) * rz2;
  const Mat<F, 3, 2> vj = add(mul(mul(v_cov2d, j), transpose(cov)), mul(mul(transpose(v_cov2d), j), cov));
  const F limx_pos = (F(1.15) * F(c.w) - c.pc.x) / c.focal.x;
  const F limy_pos = (F(1.15) * F(c.h) - c.pc.y) / c.focal.y;
  const F limx_neg = (F(-0.15) * F(c.w) - c.pc.x) / c.focal.x;
  const F limy_neg = (F(-0.15) * F(c.h) - c.pc.y) / c.focal.y;
  if (x * rz <= limx_pos && x * rz >= limx_neg) {
    o.x = o.x + -c.focal.x * rz2 * vj.m[2][0];
    o.z = o.z + F(2) * c.focal.x * x * rz2 * rz * vj.m[2][0];
  } else {
    const F cx = clampf(x * rz, limx_neg, limx_pos);
    o.z = o.z + c.focal.x * cx * rz2 * vj.m[2][0];
  }
  if (y * rz <= limy_pos && y * rz >= limy_neg) {
    o.y = o.y + -c.focal.y * rz2 * vj.m[2][1];
    o.z = o.z + F(2) * c.focal.y * y * rz2 * rz * vj.m[2][1];
  } else {
    const F cy = clampf(y * rz, limy_neg, limy_pos);
    o.z = o.z + c.focal.y * cy * rz2 * vj.m[2][1];
  }
  o.z = o.z + (-c.focal.x * rz2 * vj.m[0][0] - c.focal.y * rz2 * vj.m[1][1]);
  return o;
}

// Gradient of sqrt(max(det(A),0) / max(det(A + bI), 1e-12)) with respect to A
// (the opacity compensation of helpers.wgsl:170-183). The reference backward
// omits this term; the exact adjoint includes it.
template <class F> GSR_HD M2<F> compensate_vjp(const M2<F>& start, F blur, F v_fc) {
  M2<F> g;
  g.m[0][0] = g.m[0][1] = g.m[1][0] = g.m[1][1] = F(0);
  M2<F> end = start;
  end.m[0][0] = end.m[0][0] + blur;
  end.m[1][1] = end.m[1][1] + blur;
  const F d0 = det2(start), d1r = det2(end);
  const F det_raw = gmax(d0, F(0));
  const F det_end = gmax(d1r, F(1e-12));
  if (det_raw <= F(0)) return g;
  const F fc = gsqrt(det_raw / det_end);
  const F k0 = v_fc * fc / (F(2) * det_raw);
  g.m[0][0] = k0 * start.m[1][1];
  g.m[1][1] = k0 * start.m[0][0];
  g.m[0][1] = -k0 * start.m[1][0];
  g.m[1][0] = -k0 * start.m[0][1];
  if (d1r > F(1e-12)) {
    const F k1 = v_fc * fc / (F(2) * det_end);
    g.m[0][0] = g.m[0][0] - k1 * end.m[1][1];
    g.m[1][1] = g.m[1][1] - k1 * end.m[0][0];
    g.m[0][1] = g.m[0][1] + k1 * end.m[1][0];
    g.m[1][0] = g.m[1][0] + k1 * end.m[0][1];
  }
  return g;
}

// Screen-space gradients of one Gaussian summed over the pixels it touches
// (the per-Gaussian record written by rasterize_backwards.wgsl:145-162).
template <class F> struct SplatGrad {
  F v_xy[2];
  F v_conic[3];
  F v_rgb[3];
  F v_opac;
  F abs_xy[2];
  F count;
};

// Parameter gradients of one Gaussian (project_backwards.wgsl:51-151).
template <class F> struct ParamGrad {
  V3<F> v_mean;
  V4<F> v_quat;
  V3<F> v_log_scale;
  F v_raw_opac;
  V3<F> viewdir;  // for the SH coefficient gradients b_k(viewdir) * v_rgb
  F depth;        // camera-space z, for the densification statistics
};

// exact == false reproduces the reference approximations: no gradient
// through the opacity compensation with respect to the covariance and none
// through the SH view direction with respect to the mean. With exact == true
// both terms are included and the result is the true adjoint of
// project_gaussian + sh_to_color. coeff(k, ch) gives SH coefficients (read
// only when exact).
// Gradient of f(d) = sum_{k>=1} w_k b_k(d) with respect to the direction
// d = (x, y, z), from the derivatives of the basis polynomials of sh_basis
// (degrees 1-3 written out; degree 4 goes through dual numbers).
template <class F> GSR_HD V3<F> sh_weighted_grad(int degree, F x, F y, F z, const F* w) {
  V3<F> g;
  g.x = g.y = g.z = F(0);
  if (degree <= 0) return g;
  if (degree >= 4) {
    F b[25], db[25][3];
    V3<F> d;
    d.x = x;
    d.y = y;
    d.z = z;
    sh_basis_grad<F>(degree, d, b, db);
    for (int k = 1; k < num_sh_coeffs(degree); ++k) {
      g.x = g.x + w[k] * db[k][0];
      g.y = g.y + w[k] * db[k][1];
      g.z = g.z + w[k] * db[k][2];
    }
    return g;
  }
  const F A = F(0.48860251190292);
  g.x = -A * w[3];
  g.y = -A * w[1];
  g.z = A * w[2];
  if (degree == 1) return g;
  const F t1a = F(0.5462742152960395), c0b = F(1.092548430592079), c6 = F(0.9461746957575601);
  // b4 = t1a 2xy, b5 = -c0b zy, b6 = c6 z^2 - c, b7 = -c0b zx, b8 = t1a (x^2 - y^2)
  g.x = g.x + w[4] * (F(2) * t1a * y) - w[7] * (c0b * z) + w[8] * (F(2) * t1a * x);
  g.y = g.y + w[4] * (F(2) * t1a * x) - w[5] * (c0b * z) - w[8] * (F(2) * t1a * y);
  g.z = g.z - w[5] * (c0b * y) + w[6] * (F(2) * c6 * z) - w[7] * (c0b * x);
  if (degree == 2) return g;
  const F t2a = F(-0.5900435899266435), c1b = F(1.445305721320277), c0c = F(2.285228997322329);
  const F c0c0 = F(0.4570457994644658), c12a = F(1.865881662950577), c12b = F(1.119528997770346);
  const F t0c = -c0c * z * z + c0c0;
  const F x2 = x * x, y2 = y * y;
  // b9 = t2a (3x^2 y - y^3), b10 = c1b z 2xy, b11 = t0c y, b12 = z (c12a z^2 - c12b),
  // b13 = t0c x, b14 = c1b z (x^2 - y^2), b15 = t2a (x^3 - 3 x y^2)
  g.x = g.x + w[9] * (t2a * F(6) * x * y) + w[10] * (c1b * F(2) * y * z) + w[13] * t0c +
        w[14] * (c1b * F(2) * x * z) + w[15] * (t2a * F(3) * (x2 - y2));
  g.y = g.y + w[9] * (t2a * F(3) * (x2 - y2)) + w[10] * (c1b * F(2) * x * z) + w[11] * t0c -
        w[14] * (c1b * F(2) * y * z) - w[15] * (t2a * F(6) * x * y);
  g.z = g.z + w[10] * (c1b * F(2) * x * y) - w[11] * (F(2) * c0c * z * y) +
        w[12] * (F(3) * c12a * z * z - c12b) - w[13] * (F(2) * c0c * z * x) + w[14] * (c1b * (x2 - y2));
  return g;
}

// Gradient of the SH colour with respect to the mean through the view
// direction (dir = normalize(mean - campos)): sum_k (sum_ch v_color_ch *
// coeff_k,ch) * d b_k / d dir, chained through the normalisation. The
// reference omits this term.
template <class F, class Coeff>
GSR_HD V3<F> sh_viewdir_vjp(const Cam<F>& cam, V3<F> mean, V3<F> vd, int degree, V3<F> v_color, const Coeff& coeff) {
  V3<F> out;
  out.x = out.y = out.z = F(0);
  if (degree <= 0) return out;
  const int k = num_sh_coeffs(degree);
  F w[25];
  w[0] = F(0);
  for (int i = 1; i < k; ++i) w[i] = v_color.x * coeff(i, 0) + v_color.y * coeff(i, 1) + v_color.z * coeff(i, 2);
  const V3<F> gg = sh_weighted_grad<F>(degree, vd.x, vd.y, vd.z, w);
  const F gv[3] = {gg.x, gg.y, gg.z};
  // d(d/|d|) = (I - u u^T) / |d| with u the unit view direction.
  V3<F> d;
  d.x = mean.x - cam.campos.x;
  d.y = mean.y - cam.campos.y;
  d.z = mean.z - cam.campos.z;
  const F n2 = d.x * d.x + d.y * d.y + d.z * d.z;
  if (n2 > F(1e-12)) {
    const F inv = F(1) / gsqrt(n2);
    const F ug = vd.x * gv[0] + vd.y * gv[1] + vd.z * gv[2];
    out.x = (gv[0] - vd.x * ug) * inv;
    out.y = (gv[1] - vd.y * ug) * inv;
    out.z = (gv[2] - vd.z * ug) * inv;
  } else {
    const F inv = F(1) / gsqrt(F(1e-12));
    out.x = gv[0] * inv;
    out.y = gv[1] * inv;
    out.z = gv[2] * inv;
  }
  return out;
}

// exact == false reproduces the reference approximations (see above);
// hp selects the FP64 compensation and inversion of the forward's
// high-precision conic mode;
// sh_dir == false leaves out only the view-direction term even when exact
// (callers that add sh_viewdir_vjp themselves).
template <class F, class Coeff>
GSR_HD ParamGrad<F> project_backward(const Cam<F>& cam, V3<F> mean, V4<F> quat_unorm, V3<F> log_scale, F raw_opac,
                                     F cov_blur, V2<F> v_xy, V3<F> v_conic, V3<F> v_color, F v_opac, int degree,
                                     const Coeff& coeff, bool exact, bool sh_dir = true, bool hp = false) {
  ParamGrad<F> g;
  const V3<F> vd = view_dir(cam, mean);
  g.viewdir = vd;
  const V3<F> mc = world_to_cam(cam, mean);
  g.depth = mc.z;
  const F qn = quat_unorm.x * quat_unorm.x + quat_unorm.y * quat_unorm.y + quat_unorm.z * quat_unorm.z +
               quat_unorm.w * quat_unorm.w;
  const F rs = F(1) / gsqrt(qn);
  V4<F> quat;
  quat.x = quat_unorm.x * rs;
  quat.y = quat_unorm.y * rs;
  quat.z = quat_unorm.z * rs;
  quat.w = quat_unorm.w * rs;
  V3<F> scale;
  scale.x = gexp(log_scale.x);
  scale.y = gexp(log_scale.y);
  scale.z = gexp(log_scale.z);
  const M3<F> rotmat = quat_to_mat3(quat);
  const M3<F> m = rot_scale(rotmat, scale);
  const M3<F> cov3d = mul(m, transpose(m));
  const M3<F> cov_cam = mul(mul(cam.rot, cov3d), transpose(cam.rot));
  const M32<F> j = calc_cam_j(mc, cam);
  const M2<F> cov_start = mul(mul(j, cov_cam), transpose(j));
  M2<F> cov2d = cov_start;
  const F fc = hp ? compensate_cov2d_hp(cov2d, cov_blur) : compensate_cov2d(cov2d, cov_blur);
  const F opac = sigmoid(raw_opac);
  g.v_raw_opac = fc * v_opac * opac * (F(1) - opac);
  M2<F> cinv;
  {
    // The conic the forward used (FP64 inversion in high-precision mode).
    const V3<F> c = hp ? inverse2x2_packed_hp(cov2d) : inverse2x2_packed(cov2d);
    cinv.m[0][0] = c.x;
    cinv.m[0][1] = c.y;
    cinv.m[1][0] = c.y;
    cinv.m[1][1] = c.z;
  }
  M2<F> vci;
  vci.m[0][0] = v_conic.x;
  vci.m[0][1] = F(0.5) * v_conic.y;
  vci.m[1][0] = F(0.5) * v_conic.y;
  vci.m[1][1] = v_conic.z;
  M2<F> v_cov2d = inverse2x2_vjp(cinv, vci);
  if (exact) v_cov2d = add(v_cov2d, compensate_vjp(cov_start, cov_blur, v_opac * opac));
  const V3<F> v_mc = persp_proj_vjp(j, mc, cov_cam, cam, v_cov2d, v_xy);
  const M3<F> v_cov_cam = mul(mul(transpose(j), v_cov2d), j);
  const M3<F> v_cov3d = mul(mul(transpose(cam.rot), v_cov_cam), cam.rot);
  const M3<F> v_m = mul(add(v_cov3d, transpose(v_cov3d)), m);
  V3<F> v_scale;
  v_scale.x = rotmat.m[0][0] * v_m.m[0][0] + rotmat.m[0][1] * v_m.m[0][1] + rotmat.m[0][2] * v_m.m[0][2];
  v_scale.y = rotmat.m[1][0] * v_m.m[1][0] + rotmat.m[1][1] * v_m.m[1][1] + rotmat.m[1][2] * v_m.m[1][2];
  v_scale.z = rotmat.m[2][0] * v_m.m[2][0] + rotmat.m[2][1] * v_m.m[2][1] + rotmat.m[2][2] * v_m.m[2][2];
  g.v_log_scale.x = v_scale.x * scale.x;
  g.v_log_scale.y = v_scale.y * scale.y;
  g.v_log_scale.z = v_scale.z * scale.z;
  g.v_quat = normalize_vjp_apply(quat_unorm, quat_to_mat3_vjp(quat, rot_scale(v_m, scale)));
  g.v_mean = mulv(transpose(cam.rot), v_mc);
  if (exact && sh_dir && degree > 0) {
    const V3<F> vm = sh_viewdir_vjp(cam, mean, vd, degree, v_color, coeff);
    g.v_mean.x = g.v_mean.x + vm.x;
    g.v_mean.y = g.v_mean.y + vm.y;
    g.v_mean.z = g.v_mean.z + vm.z;
  }
  return g;
}

// Reverse-walk adjoint of one blend step. T is the transmittance after this
// Gaussian on entry and before it on return; S is the colour accumulated
// behind it (unnormalised) and gains this Gaussian's share. vrgb is the
// pixel's upstream colour gradient and K = (dot(vrgb, bg) - v_alpha) * T_final.
// Writes the per-pixel contribution of this Gaussian into g (overwriting).
// With ref_skip the gradient is zeroed but S and T still advance.
template <class F>
GSR_HD void blend_step_grad(F dx, F dy, F ca, F cb, F cc, F r, F gcol, F bcol, F opac, F gauss, F alpha, F& T,
                            F S[3], const F vrgb[3], F K, bool ref_skip, SplatGrad<F>& g) {
  const F ra = grcp(F(1) - alpha);
  const F Ti = T * ra;
  const F cp[3] = {gmax(r, F(0)), gmax(gcol, F(0)), gmax(bcol, F(0))};
  const F craw[3] = {r, gcol, bcol};
  const F vis = alpha * Ti;
  const F v_alpha = Ti * (cp[0] * vrgb[0] + cp[1] * vrgb[1] + cp[2] * vrgb[2]) -
                    (S[0] * vrgb[0] + S[1] * vrgb[1] + S[2] * vrgb[2] + K) * ra;
  for (int c = 0; c < 3; ++c) S[c] = S[c] + cp[c] * vis;
  T = Ti;
  if (ref_skip) {
    g.v_xy[0] = g.v_xy[1] = F(0);
    g.v_conic[0] = g.v_conic[1] = g.v_conic[2] = F(0);
    g.v_rgb[0] = g.v_rgb[1] = g.v_rgb[2] = F(0);
    g.v_opac = F(0);
    g.abs_xy[0] = g.abs_xy[1] = F(0);
    g.count = F(0);
    return;
  }
  for (int c = 0; c < 3; ++c) g.v_rgb[c] = (craw[c] >= F(0)) ? vis * vrgb[c] : F(0);
  g.count = F(1);
  if (opac * gauss <= F(0.999)) {
    const F vs = -alpha * v_alpha;
    g.v_conic[0] = F(0.5) * vs * dx * dx;
    g.v_conic[1] = vs * dx * dy;
    g.v_conic[2] = F(0.5) * vs * dy * dy;
    g.v_xy[0] = vs * (ca * dx + cb * dy);
    g.v_xy[1] = vs * (cb * dx + cc * dy);
    g.v_opac = v_alpha * gauss;
  } else {
    g.v_conic[0] = g.v_conic[1] = g.v_conic[2] = F(0);
    g.v_xy[0] = g.v_xy[1] = F(0);
    g.v_opac = F(0);
  }
  g.abs_xy[0] = gabs(g.v_xy[0]);
  g.abs_xy[1] = gabs(g.v_xy[1]);
}

// ----------------------------------------------------------------------------
// Topology mutation of one splat row (RustGS/src/training/topology/apply.rs:
// 29-176): a row copies a source splat, optionally refined as one half of a
// split (moved by -/+ the rotated, scaled sample offset, its largest axis
// halved, opacity 1 - sqrt(1 - o)), optionally decayed (scale and opacity
// shrink with the remaining training fraction) and optionally opacity-reset
// (capped). Logits go through the numerically stable sigmoid of apply.rs.
// ----------------------------------------------------------------------------
enum TopoKind { kTopoExisting = 0, kTopoRefineExisting = 1, kTopoRefineNew = 2 };
struct TopoParams {
  int has_decay;
  float scale_decay, opacity_decay, train_t;
  int opacity_reset;
  float reset_cap;
};

template <class F> GSR_HD F stable_sigmoid(F x) {
  if (x >= F(0)) {
    const F e = gexp(-x);
    return F(1) / (F(1) + e);
  }
  const F e = gexp(x);
  return e / (F(1) + e);
}
template <class F> GSR_HD F clamp_to(F x, F lo, F hi) { return gmin(gmax(x, lo), hi); }

// Rotation of v by the quaternion (w, x, y, z), normalised first; a zero
// quaternion is the identity (apply.rs:97-106).
template <class F> GSR_HD V3<F> quat_rotate(V4<F> q, V3<F> v) {
  const F n2 = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
  if (!(n2 > F(0))) return v;
  const F r = F(1) / gsqrt(n2);
  const F w = q.x * r, x = q.y * r, y = q.z * r, z = q.w * r;
  // v + 2w (u x v) + 2 u x (u x v), u = (x, y, z)
  const F cx = y * v.z - z * v.y, cy = z * v.x - x * v.z, cz = x * v.y - y * v.x;
  const F dx = y * cz - z * cy, dy = z * cx - x * cz, dz = x * cy - y * cx;
  V3<F> o;
  o.x = v.x + F(2) * (w * cx + dx);
  o.y = v.y + F(2) * (w * cy + dy);
  o.z = v.z + F(2) * (w * cz + dz);
  return o;
}

// One output row from its source row: transforms t[10] (position, quaternion
// w x y z, log scale) and the opacity logit, in place.
template <class F> GSR_HD void topo_mutate(F* t, F& logit, int kind, F sample, const TopoParams& p) {
  if (kind == kTopoRefineExisting || kind == kTopoRefineNew) {
    V3<F> sc;
    sc.x = gexp(t[7]);
    sc.y = gexp(t[8]);
    sc.z = gexp(t[9]);
    V3<F> sv;
    sv.x = sc.x * sample;
    sv.y = sc.y * sample;
    sv.z = sc.z * sample;
    const V3<F> off = quat_rotate(V4<F>{t[3], t[4], t[5], t[6]}, sv);
    const F sgn = kind == kTopoRefineNew ? F(1) : F(-1);
    t[0] = t[0] + sgn * off.x;
    t[1] = t[1] + sgn * off.y;
    t[2] = t[2] + sgn * off.z;
    // The largest axis (first on ties) halves (apply.rs:108-118).
    F r[3] = {sc.x, sc.y, sc.z};
    int m = 0;
    for (int a = 1; a < 3; ++a)
      if (r[a] > r[m]) m = a;
    r[m] = r[m] * F(0.5);
    for (int a = 0; a < 3; ++a) t[7 + a] = glog(gmax(r[a], F(1e-6)));
    // apply.rs:120-124
    const F lo = F(1.0 / 255.0), hi = F(1) - F(1.0 / 255.0);
    const F o = clamp_to(stable_sigmoid(logit), lo, hi);
    const F rf = clamp_to(F(1) - gsqrt(F(1) - o), lo, hi);
    logit = glog(rf / (F(1) - rf));
  }
  if (p.has_decay) {
    // apply.rs:132-153
    const F shrink = F(1) - clamp_to(F(p.train_t), F(0), F(1));
    if (F(p.scale_decay) > F(0)) {
      const F scaling = gmax(F(1) - F(p.scale_decay) * shrink, F(1e-6));
      for (int a = 0; a < 3; ++a) t[7 + a] = glog(gmax(gexp(t[7 + a]) * scaling, F(1e-12)));
    }
    if (F(p.opacity_decay) > F(0)) {
      const F o = stable_sigmoid(logit);
      const F d = clamp_to(o - F(p.opacity_decay) * shrink, F(1e-12), F(1) - F(1e-12));
      logit = glog(d / (F(1) - d));
    }
  }
  if (p.opacity_reset) {
    // apply.rs:126-130
    const F o = clamp_to(stable_sigmoid(logit), F(1e-12), F(1) - F(1e-12));
    const F r = gmin(o, F(p.reset_cap));
    logit = glog(r / (F(1) - r));
  }
}

}  // namespace gsr
