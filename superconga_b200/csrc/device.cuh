// Device-side building blocks of the B200 self-consistency path: complex
// arithmetic, the midpoint Riccati step, the local Green functions and the
// bilinear lookups into the reference grid.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace scb {

constexpr int MAX_COMP = 4;

template <typename R>
struct Cx {
  R re, im;
};

// Per-angle constants of one trajectory frame.
struct AngleParams {
  double cD, sD;  // order parameter into the frame (float trig, promoted)
  double cA, sA;  // induced vector potential into the frame
  double cB, sB;  // frame back to the reference grid
  double cE, sE;  // external vector potential coordinates (double trig)
  double vx, vy;  // Fermi velocity
  double w;       // Fermi-surface integrand factor
  double hs;      // Riccati step h / |v_F| (RiccatiSolverConfined.h:525-527)
  double sx, sy;  // vx * w, vy * w
  double eta[MAX_COMP];  // basis function of every component at this angle
};

template <typename R>
__device__ __forceinline__ Cx<R> cmul(Cx<R> a, Cx<R> b) {
  return Cx<R>{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}

// Precision-specific primitives: IEEE-rounded reciprocal and accurate
// reciprocal square root in FP64; the fast MUFU approximations in FP32.
// FP64 reciprocal: the hardware approximation r (relative error about 2^-20)
// refined by one third-order step of the series 1/x = r / (1 - e) with
// e = 1 - x r, truncated after e^2: r (1 + e + e^2), error O(e^3) (measured on
// B200: within 2 ulp of IEEE 1/x; the arguments here are finite and nonzero).
__device__ __forceinline__ double rcp_(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  const double e = fma(-x, r, 1.0);
  return fma(r, fma(e, e, e), r);
}
__device__ __forceinline__ float rcp_(float x) { return __fdividef(1.0f, x); }
// FP64 reciprocal square root of a positive normal argument: the hardware
// approximation r refined by one third-order step of the binomial series
// 1/sqrt(x) = r (1 - e)^(-1/2) with e = 1 - x r^2, truncated after e^2:
// r (1 + e/2 + 3 e^2/8), error O(e^3) (measured on B200: within 3 ulp).
__device__ __forceinline__ double rsqrt_(double x) {
  double r;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  const double e = fma(-x * r, r, 1.0);
  return fma(r, e * fma(0.375, e, 0.5), r);
}
__device__ __forceinline__ float rsqrt_(float x) { return rsqrtf(x); }
// FP64 square root of a non-negative argument as x / sqrt(x); the estimate is
// taken of max(x, smallest normal), which gives 0 for x = 0 with no branch and
// leaves every normal argument unchanged.
__device__ __forceinline__ double sqrt_(double x) {
  return x * rsqrt_(fmax(x, 2.2250738585072014e-308));
}
// FP32 square root of a non-negative argument: the hardware approximation
// (sqrt.approx; 0 for 0), one instruction.
__device__ __forceinline__ float sqrt_(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Principal square root, branch cut on the negative real axis, through one
// square root and one reciprocal square root:
//   u = (|z| + |x|)/2, t = sqrt(u), v = |y| / (2 t);
//   sqrt(z) = (t, sign(y) v) for x >= 0 and (v, sign(y) t) otherwise.
// u = 0 only for z = 0, where the estimate of max(u, smallest normal) is
// finite and t = v = 0: the root 0 with no branch.
template <typename R>
__device__ __forceinline__ Cx<R> csqrt_dev(R x, R y) {
  const R m = sqrt_(x * x + y * y);
  const R u = R(0.5) * (m + fabs(x));
  const R r = rsqrt_(fmax(u, R(sizeof(R) == 8 ? 2.2250738585072014e-308 : 1.17549435e-38)));
  const R t = u * r;
  const R v = R(0.5) * fabs(y) * r;
  const bool pos = x >= R(0);
  return Cx<R>{pos ? t : v, copysign(pos ? v : t, y)};
}

// Midpoint Riccati step, riccati::computeStep (RiccatiSolutions.h:65-94):
//   a = i h/4 conj(D), b = 2 a g0 + i h e - 1, c = (a g0 + i h e + 1) g0 + i h D,
//   g1 = 2 c / (-b + sqrt(b^2 - 4 a c)).
// The products with the purely imaginary step are written out (they are exact).
// With u = a g0 and B = i h e the discriminant reduces to
//   b^2 - 4 a c = (B - 1)^2 + h^2 |D|^2 - 8 u,
// because a (i h D) = -(h^2 / 4) |D|^2 is real; that form skips two complex
// products and avoids the cancellation of b^2 against 4 a c.
template <typename R>
__device__ __forceinline__ Cx<R> riccati_step(R dre, R dim, R ere, R eim, Cx<R> g, R h) {
  const R q = R(0.25) * h;
  const Cx<R> a{q * dim, q * dre};
  const R ser = -h * eim, sei = h * ere;  // (i h) * e
  const Cx<R> ag = cmul(a, g);
  const Cx<R> b{R(2) * ag.re + ser - R(1), R(2) * ag.im + sei};
  const Cx<R> t{ag.re + ser + R(1), ag.im + sei};
  const Cx<R> tg = cmul(t, g);
  const Cx<R> c{tg.re - h * dim, tg.im + h * dre};
  const R bm = ser - R(1);
  const R s0 = h * h * (dre * dre + dim * dim) - sei * sei;  // the site's part: shared by all energies
  const Cx<R> disc = csqrt_dev<R>((bm * bm + s0) - R(8) * ag.re, (R(2) * bm) * sei - R(8) * ag.im);
  const R den_re = disc.re - b.re, den_im = disc.im - b.im;
  const R inv = rcp_(den_re * den_re + den_im * den_im);
  const R c2r = R(2) * c.re, c2i = R(2) * c.im;
  return Cx<R>{(c2r * den_re + c2i * den_im) * inv, (c2i * den_re - c2r * den_im) * inv};
}

// Two energies of one thread, lane by lane in FP32 pairs:
// re = (Re z_j, Re z_j+1), im = (Im z_j, Im z_j+1).  sm_100 executes one
// FFMA2 / FMUL2 / FADD2 instruction for both lanes, so the FP32 arithmetic of
// the mixed-precision sweep takes half the issue slots; the square roots and
// reciprocals stay one MUFU instruction per lane.  Each lane is rounded as the
// scalar FP32 operation would be.
struct Cx2 {
  float2 re, im;
};
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ Cx2 pack2(Cx<float> a, Cx<float> b) {
  return Cx2{make_float2(a.re, b.re), make_float2(a.im, b.im)};
}
__device__ __forceinline__ void unpack2(Cx2 v, Cx<float> &a, Cx<float> &b) {
  a = Cx<float>{v.re.x, v.im.x};
  b = Cx<float>{v.re.y, v.im.y};
}

// csqrt_dev of both lanes.
__device__ __forceinline__ Cx2 csqrt2(float2 x, float2 y) {
  const float2 xx = fma2(x, x, mul2(y, y));
  const float2 m = make_float2(sqrt_(xx.x), sqrt_(xx.y));
  const float2 u = mul2(bc2(0.5f), add2(m, make_float2(fabsf(x.x), fabsf(x.y))));
  const float2 r = make_float2(rsqrt_(fmaxf(u.x, 1.17549435e-38f)), rsqrt_(fmaxf(u.y, 1.17549435e-38f)));
  const float2 t = mul2(u, r);
  const float2 v = mul2(mul2(bc2(0.5f), make_float2(fabsf(y.x), fabsf(y.y))), r);
  const bool p0 = x.x >= 0.0f, p1 = x.y >= 0.0f;
  return Cx2{make_float2(p0 ? t.x : v.x, p1 ? t.y : v.y),
             make_float2(copysignf(p0 ? v.x : t.x, y.x), copysignf(p1 ? v.y : t.y, y.y))};
}

// riccati_step<float> of two energies e = ere + i eim (ere: the real part
// with the site's Doppler shift added; Matsubara energies have ere = the
// shift alone) at the same site fields and step h.
__device__ __forceinline__ Cx2 riccati_step2(float dre, float dim, float2 ere, float2 eim, Cx2 g, float h) {
  const float q = 0.25f * h;
  const float2 ar = bc2(q * dim), ai = bc2(q * dre);
  const float2 ser = mul2(bc2(-h), eim);  // Re of (i h) * e
  const float2 sei = mul2(bc2(h), ere);   // Im of (i h) * e
  const float2 agre = fma2(ar, g.re, mul2(neg2(ai), g.im));
  const float2 agim = fma2(ar, g.im, mul2(ai, g.re));
  const float2 bm = add2(ser, bc2(-1.0f));
  const float2 bre = fma2(bc2(2.0f), agre, bm);
  const float2 bim = fma2(bc2(2.0f), agim, sei);
  const float2 tre = add2(agre, add2(ser, bc2(1.0f)));
  const float2 tim = add2(agim, sei);
  const float2 cre = fma2(tre, g.re, fma2(neg2(tim), g.im, bc2(-h * dim)));
  const float2 cim = fma2(tre, g.im, fma2(tim, g.re, bc2(h * dre)));
  const float2 s0 = fma2(neg2(sei), sei, bc2(h * h * (dre * dre + dim * dim)));
  const Cx2 disc = csqrt2(fma2(bc2(-8.0f), agre, fma2(bm, bm, s0)),
                          fma2(bc2(-8.0f), agim, mul2(add2(bm, bm), sei)));
  const float2 dr = add2(disc.re, neg2(bre)), di = add2(disc.im, neg2(bim));
  const float2 s = fma2(dr, dr, mul2(di, di));
  // 2 c / den = 2 c conj(den) / |den|^2 (the factor 2 is exact, so it goes with 1/|den|^2).
  const float2 inv2 = mul2(bc2(2.0f), make_float2(rcp_(s.x), rcp_(s.y)));
  return Cx2{mul2(fma2(cre, dr, mul2(cim, di)), inv2), mul2(fma2(cim, dr, mul2(neg2(cre), di)), inv2)};
}

// local_greens<float> of two energies, before the signs: with p = g gt and
// w = 2 / |1 + p|^2, fre = w Im p, fim = w (1 + Re p); then
//   Re g = -fre, f + f~* = (fre ure - fim uim, -(fre vim + fim vre)),
//   Im I = -(Re D uim + Im D vre),
// u = gt - g, v = g + gt.  Returns fre, F.re, nfim = fre vim + fim vre
// (F.im = -nfim) and ni = Re D uim + Im D vre (Im I = -ni).
__device__ __forceinline__ void local_greens2(Cx2 g, Cx2 gt, float dre, float dim, float2 &fre,
                                              float2 &Fre, float2 &nfim, float2 &ni) {
  const float2 pre = fma2(g.re, gt.re, mul2(neg2(g.im), gt.im));
  const float2 pim = fma2(g.re, gt.im, mul2(g.im, gt.re));
  const float2 den_re = add2(bc2(1.0f), pre);
  const float2 s = fma2(den_re, den_re, mul2(pim, pim));
  const float2 w = mul2(bc2(2.0f), make_float2(rcp_(s.x), rcp_(s.y)));
  fre = mul2(pim, w);
  const float2 fim = mul2(den_re, w);
  const float2 ure = add2(gt.re, neg2(g.re)), uim = add2(gt.im, neg2(g.im));
  const float2 vre = add2(g.re, gt.re), vim = add2(g.im, gt.im);
  Fre = fma2(fre, ure, mul2(neg2(fim), uim));
  nfim = fma2(fre, vim, mul2(fim, vre));
  ni = fma2(bc2(dre), uim, mul2(bc2(dim), vre));
}

// greens_g_im<float> of two real energies: Im g = -[(1 - Re p)(1 + Re p) - (Im p)^2] / |1 + p|^2.
__device__ __forceinline__ float2 greens_g_im2(Cx2 g, Cx2 gt) {
  const float2 pre = fma2(g.re, gt.re, mul2(neg2(g.im), gt.im));
  const float2 pim = fma2(g.re, gt.im, mul2(g.im, gt.re));
  const float2 den_re = add2(bc2(1.0f), pre), nr = add2(bc2(1.0f), neg2(pre));
  const float2 s = fma2(den_re, den_re, mul2(pim, pim));
  const float2 inv = make_float2(rcp_(s.x), rcp_(s.y));
  return mul2(fma2(nr, den_re, mul2(neg2(pim), pim)), neg2(inv));
}

// Homogeneous solutions, riccati::computeHomogeneous (RiccatiSolutions.h:36-54).
template <typename R>
__device__ __forceinline__ void riccati_homogeneous(R dre, R dim, R ere, R eim, Cx<R> &g,
                                                    Cx<R> &gt) {
  const R nd = dre * dre + dim * dim;
  const R e2re = ere * ere - eim * eim, e2im = ere * eim + eim * ere;
  const Cx<R> om = csqrt_dev<R>(nd - e2re, -e2im);
  const R dr = ere - om.im, di = eim + om.re;  // energy + i * Omega
  const R inv = rcp_(dr * dr + di * di);
  const Cx<R> invd{dr * inv, -di * inv};
  g = cmul(Cx<R>{-dre, -dim}, invd);
  gt = cmul(Cx<R>{dre, -dim}, invd);
}

// Local Green functions of one energy (LocalGreens.h:32-70) and the free-energy
// kernel (ComputeFreeEnergy.h:95-103): returns f + f~* in F, Re g and Im I.
// With p = g gt and w = 2 / |1 + p|^2, the common factor i 2 / (1 + p) of f
// and f~ is fac = w (Im p, 1 + Re p), and
//   Re g = Re[-i (1 - p) / (1 + p)] = -2 Im p / |1 + p|^2 = -Re fac,
//   f + f~* = -fac g + conj(fac gt) = (Re[fac (gt - g)], -Im[fac (g + gt)]),
//   Im I = Im[conj(D) g - D gt] = Re D Im(g - gt) - Im D Re(g + gt),
// the same quantities as the reference's in fewer operations.
template <typename R>
__device__ __forceinline__ void local_greens(Cx<R> g, Cx<R> gt, R dre, R dim, Cx<R> &F,
                                             R &g_re, R &i_im) {
  const Cx<R> p = cmul(g, gt);
  const R den_re = R(1) + p.re, den_im = p.im;
  const R w = R(2) * rcp_(den_re * den_re + den_im * den_im);
  const R fre = den_im * w, fim = den_re * w;
  g_re = -fre;
  const R ure = gt.re - g.re, uim = gt.im - g.im;  // gt - g
  const R vre = g.re + gt.re, vim = g.im + gt.im;  // g + gt
  F = Cx<R>{fre * ure - fim * uim, -(fre * vim + fim * vre)};
  i_im = -(dre * uim + dim * vre);
}

// Im g of one real energy, g = -i (1 - g gt) / (1 + g gt) (LocalGreens.h:32-43).
template <typename R>
__device__ __forceinline__ R greens_g_im(Cx<R> g, Cx<R> gt) {
  const Cx<R> p = cmul(g, gt);
  const R den_re = R(1) + p.re, den_im = p.im;
  const R inv = rcp_(den_re * den_re + den_im * den_im);
  const R nr = R(1) - p.re, ni = -p.im;
  return -(nr * den_re + ni * den_im) * inv;
}

// Bilinear lookup of insertRotatedGrid(_Additive)_kernel
// (GridFunctions_GPU.h:436-546): coordinates of site (x, y) of an n_out grid in
// an n_in grid rotated by the angle whose (cos, sin) of minus the angle are
// (c, s).  Returns false when the reference leaves the site untouched.
struct Bilinear {
  int i00;  // index of the lower-left corner in the input grid
  double xf, yf;
};
__device__ __forceinline__ bool rotated_lookup(int x, int y, int n_out, int n_in, double c,
                                               double s, Bilinear &b) {
  const double xt = (double)(n_in - n_out) / 2.0;
  const double sh = (double)(n_in - 1) / 2.0;
  const double X = (double)x + xt - sh, Y = (double)y + xt - sh;
  const double xr = X * c - Y * s + sh;
  const double yr = X * s + Y * c + sh;
  const int xi = (int)xr, yi = (int)yr;
  if (xi >= 0 && xi + 1 < n_in && yi >= 0 && yi + 1 < n_in) {
    b.i00 = yi * n_in + xi;
    b.xf = xr - (double)xi;
    b.yf = yr - (double)yi;
    return true;
  }
  return false;
}
__device__ __forceinline__ double bilerp(double v00, double v01, double v10, double v11,
                                         double xf, double yf) {
  const double x1 = (1.0 - xf) * v00 + xf * v01;
  const double x2 = (1.0 - xf) * v10 + xf * v11;
  return (1.0 - yf) * x1 + yf * x2;
}

}  // namespace scb
