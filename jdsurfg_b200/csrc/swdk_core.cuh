// swdk_core.cuh -- device numerics of the surface-wave forward model.
//
// Everything here is __host__ __device__ so the same arithmetic can be
// exercised on the CPU by developer probes; the product runs it only inside
// the CUDA kernels of swdk_kernels.cu.
//
// Reference semantics (JDSurfG, src/SWD):
//   * secular functions dltar4 (Rayleigh, Dunkin delta matrix) and dltar1
//     (Love, Haskell) follow surfdisp96.f:712-1095;
//   * the period/mode continuation, bracket scan and refinement follow
//     surfdisp96.f:57-370 (surfdisp96) and :400-708 (getsol/nevill/half);
//   * eigenfunctions and energy integrals follow sregn96.f90:193-1629 and
//     slegn96.f90:179-670.
// Restructuring relative to the Fortran (same mathematics):
//   * per-layer divisions by rho, ra, rb become one reciprocal each;
//   * E/E^-1 and the f/g/h layer integrals are formed once per layer and
//     shared by the six intijr integrals (the reference rebuilds them per
//     integral);
//   * the up/down compound-matrix vectors in the eigenfunction pass are
//     normalised by powers of two with an integer exponent instead of
//     max-division + log (exact scaling, no log per layer);
//   * the Rayleigh down pass, svfunc and energy are fused in one top-down
//     sweep; node kernels are formed by _ParamConvert on the fly.
#pragma once
#include <cstdint>
#include <cmath>

#ifdef __CUDACC__
#define SWDK_HD __host__ __device__ __forceinline__
#define SWDK_HDI __host__ __device__
#else
#define SWDK_HD inline
#define SWDK_HDI inline
#endif

namespace swdk {

#ifndef __CUDACC__
// host builds of these headers (CPU test harnesses): the device's rsqrt
inline double rsqrt(double x) { return 1.0 / std::sqrt(x); }
using std::signbit;
#endif

// ---------------------------------------------------------------------------
// status codes (per output slot)
// ---------------------------------------------------------------------------
enum : int32_t {
  ST_OK = 0,
  ST_NO_ROOT = 1,      // no root after the per-period retry (the reference exits)
  ST_RETRIED = 2,      // found by the reference's single-period retry
  ST_NAN_INPUT = 3,    // non-finite or non-positive model values
  ST_ITER_LIMIT = 4,   // refinement hit its iteration cap (reference: 100 in nevill)
};

constexpr int KMAX_CHAIN = 128;   // periods per chain (host checks)
constexpr double TWOPI = 2.0 * 3.141592653589793;
constexpr double PI_F = 3.1415927410125732;  // REAL*4 pi of sregn96/slegn96

// ---------------------------------------------------------------------------
// small double complex with Fortran (Smith) division
// ---------------------------------------------------------------------------
struct cx {
  double re, im;
};
SWDK_HD cx mkc(double r, double i = 0.0) { cx z; z.re = r; z.im = i; return z; }
SWDK_HD cx operator+(cx a, cx b) { return mkc(a.re + b.re, a.im + b.im); }
SWDK_HD cx operator-(cx a, cx b) { return mkc(a.re - b.re, a.im - b.im); }
SWDK_HD cx operator-(cx a) { return mkc(-a.re, -a.im); }
SWDK_HD cx operator*(cx a, cx b) { return mkc(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
SWDK_HD cx operator*(double s, cx a) { return mkc(s * a.re, s * a.im); }
SWDK_HD cx operator*(cx a, double s) { return mkc(a.re * s, a.im * s); }
SWDK_HD cx operator/(cx a, double s) { return mkc(a.re / s, a.im / s); }
SWDK_HD cx operator+(cx a, double s) { return mkc(a.re + s, a.im); }
SWDK_HD cx operator+(double s, cx a) { return mkc(s + a.re, a.im); }
SWDK_HD cx operator-(double s, cx a) { return mkc(s - a.re, -a.im); }
SWDK_HD cx operator/(cx a, cx b) {
  if (fabs(b.re) >= fabs(b.im)) {
    double r = b.im / b.re, den = b.re + b.im * r;
    return mkc((a.re + a.im * r) / den, (a.im - a.re * r) / den);
  } else {
    double r = b.re / b.im, den = b.im + b.re * r;
    return mkc((a.re * r + a.im) / den, (a.im * r - a.re) / den);
  }
}
SWDK_HD cx operator/(double s, cx b) { return mkc(s) / b; }
SWDK_HD cx csqrt_real(double x) { return x >= 0.0 ? mkc(sqrt(x), 0.0) : mkc(0.0, sqrt(-x)); }
SWDK_HD cx cexpc(cx z) {
  double e = exp(z.re);
  if (z.im == 0.0) return mkc(e, 0.0);
  double s, c;
  sincos(z.im, &s, &c);
  return mkc(e * c, e * s);
}
SWDK_HD double cabsc(cx z) { return hypot(z.re, z.im); }
SWDK_HD double dsign1(double x) { return copysign(1.0, x); }

// exact power-of-two normalisation: v *= 2^-e where 2^e ~ max|v|
SWDK_HD int pow2_exponent(double t) {
  int e;
  frexp(t, &e);
  return e;
}

// Element (layer counted from the half-space up, column) of a layer table.
// Column-major: each column's layers are contiguous, half-space first, so a
// secular evaluation (half-space upward) streams its column forward and a
// lane's consecutive layers share cache sectors whatever column the other
// lanes of its warp work on.
SWDK_HD size_t layer_index(int up, int ncol, int col, int lstride) {
#ifdef SWDK_LAYER_ROWMAJOR
  (void)lstride;
  return (size_t)up * ncol + col;
#else
  (void)ncol;
  return (size_t)col * lstride + up;
#endif
}

// ---------------------------------------------------------------------------
// secular functions on the flattened REAL*4 layer model
//   lay[layer_index(mp, ncol, col, lstride)] = (d, a, b, rho), mp = 0 is the
//   half-space and mp counts layers upward
// ---------------------------------------------------------------------------
// Flattening of one sublayer of the standard grid (grid2LayerModel without
// fluid nodes, then surfdisp96's sphere()): the flattened thickness, the
// velocity factor and the Rayleigh / Love density factors.  They depend on
// the depth grid only, so one table serves every column.
struct DepthLayer {
  double tmp;       // a, b -> (float)((double)a * tmp)
  float d, fR, fL;  // flattened thickness; rho -> rho * fR (Rayleigh) or * fL (Love)
  float pad_;
};

struct LayerView {
  const float4* lay;   // (d, a, b, rho) REAL*4 as surfdisp96 holds them
  int fast;            // 1: secular_fast (recip()-based), 0: dltar1/dltar4 as written
  int ncol, col;
  int lstride;  // layer slots per column of the table (column-major layout)
  int L;    // layers including the half-space
  int llw;  // 2 when the top layer is fluid (surfdisp96.f:143-144)
  // node source (null: the layer table): the column's grid nodes
  // (vp, vs, rho, -) and the depth grid's flattening factors
  const float4* nodes;
  const DepthLayer* dl;
  int wave;  // 2 Rayleigh, 1 Love: which density factor
  SWDK_HD size_t idx(int m) const { return layer_index(L - 1 - m, ncol, col, lstride); }
  // layer m (top-down) of the flattened REAL*4 model, from the table or
  // rebuilt from the nodes with the arithmetic of the model preparation:
  // sublayer j of node interval i is v_i + (2j+1)(v_{i+1} - v_i)/8 in REAL*4
  // (grid2LayerModel, SurfaceWave.cpp:113-155), then a, b times tmp and rho
  // times the wave's density factor (sphere(), surfdisp96.f:499-571)
  SWDK_HD float4 layer(int m) const {
    if (!nodes) return lay[idx(m)];
    if (m == L - 1) {
      const float4 n = nodes[nnode() - 1];
      return flatten(n.x, n.y, n.z, m);
    }
    return from_nodes(nodes[m >> 2], nodes[(m >> 2) + 1], m);
  }
  SWDK_HD int nnode() const { return (L + 3) >> 2; }
  // sublayer m < L-1 of node interval m/4 (nodes n0 above, n1 below)
  SWDK_HD float4 from_nodes(const float4& n0, const float4& n1, int m) const {
    const float w = (float)(2 * (m & 3) + 1);
    float ai, bi, ri;
#ifdef __CUDA_ARCH__
    // The preparation forms v0 + d/8 (d = w (v1 - v0) in REAL*4) in double
    // and rounds it to REAL*4.  d/8 is exact in REAL*4 (a power-of-two
    // scaling of a normal number), so that is the correctly rounded REAL*4
    // sum of v0 and d/8, which one IEEE single-precision addition also
    // gives: the same bits without FP64 conversions in the layer walk.
    ai = __fadd_rn(n0.x, __fmul_rn(0.125f, __fmul_rn(w, __fsub_rn(n1.x, n0.x))));
    bi = __fadd_rn(n0.y, __fmul_rn(0.125f, __fmul_rn(w, __fsub_rn(n1.y, n0.y))));
    ri = __fadd_rn(n0.z, __fmul_rn(0.125f, __fmul_rn(w, __fsub_rn(n1.z, n0.z))));
#else
    ai = (float)((double)n0.x + (double)(w * (n1.x - n0.x)) * 0.125);
    bi = (float)((double)n0.y + (double)(w * (n1.y - n0.y)) * 0.125);
    ri = (float)((double)n0.z + (double)(w * (n1.z - n0.z)) * 0.125);
#endif
    return flatten(ai, bi, ri, m);
  }
  SWDK_HD float4 flatten(float ai, float bi, float ri, int m) const {
    const DepthLayer& q = dl[m];
    float4 out;
    out.x = q.d;
#ifdef __CUDA_ARCH__
    out.y = (float)__dmul_rn((double)ai, q.tmp);
    out.z = (float)__dmul_rn((double)bi, q.tmp);
    out.w = __fmul_rn(ri, wave == 2 ? q.fR : q.fL);
#else
    out.y = (float)((double)ai * q.tmp);
    out.z = (float)((double)bi * q.tmp);
    out.w = ri * (wave == 2 ? q.fR : q.fL);
#endif
    return out;
  }
  // A walk over consecutive layers (DIR -1: upward, m decreasing; +1:
  // downward) that loads ahead of use.  From the nodes it holds the current
  // interval's two nodes and the next interval's far node, which is loaded
  // one interval (four sublayers) before it is needed; from a table it holds
  // the next layer, loaded one layer early.  Layers L-1 (the half-space)
  // and below are not walked.
  struct Walk {
    float4 n0, n1, nn;
    int i;
  };
  template <int DIR, bool NODES>
  SWDK_HD void walk_start(Walk& w, int m) const {
    if (!NODES) { w.nn = lay[idx(m)]; return; }
    w.i = m >> 2;
    w.n0 = nodes[w.i];
    w.n1 = nodes[w.i + 1];
    const int j = DIR < 0 ? w.i - 1 : w.i + 2;
    if (j >= 0 && j < nnode()) w.nn = nodes[j];
  }
  // layer m of the walk: the call before was walk_start(m) or walk_layer(m - DIR)
  template <int DIR, bool NODES>
  SWDK_HD float4 walk_layer(Walk& w, int m) const {
    if (!NODES) {
      const float4 r = w.nn;
      const int j = m + DIR;
      if (j >= 0 && j < L) w.nn = lay[idx(j)];
      return r;
    }
    const int i = m >> 2;
    if (i != w.i) {
      if (DIR < 0) { w.n1 = w.n0; w.n0 = w.nn; }
      else { w.n0 = w.n1; w.n1 = w.nn; }
      w.i = i;
      const int j = DIR < 0 ? i - 1 : i + 2;
      if (j >= 0 && j < nnode()) w.nn = nodes[j];
    }
    return from_nodes(w.n0, w.n1, m);
  }
  SWDK_HD float4 get(int m) const {  // m: reference (top-down, 0-based) index
    return lay[idx(m)];
  }
};

// dltar4 (surfdisp96.f:798-898)
SWDK_HDI double dltar4(const LayerView& V, double wvno, double omga) {
  double omega = omga;
  if (omega < 1.0e-4) omega = 1.0e-4;
  const double wvno2 = wvno * wvno;
  const double iom = 1.0 / omega;
  float4 h = V.get(V.L - 1);
  double a = h.y, b = h.z, rho1 = h.w;
  double xka = omega / a, xkb = omega / b;
  double ra = sqrt((wvno + xka) * fabs(wvno - xka));
  double rb = sqrt((wvno + xkb) * fabs(wvno - xkb));
  double t = b * iom;
  double gammk = 2.0 * t * t;
  double gam = gammk * wvno2;
  double gamm1 = gam - 1.0;
  double e0 = rho1 * rho1 * (gamm1 * gamm1 - gam * gammk * ra * rb);
  double e1 = -rho1 * ra;
  double e2 = rho1 * (gamm1 - gammk * ra * rb);
  double e3 = rho1 * rb;
  double e4 = wvno2 - ra * rb;
  for (int m = V.L - 2; m >= V.llw - 1; --m) {
    float4 ly = V.get(m);
    const double dpth = ly.x;
    a = ly.y;
    b = ly.z;
    const double rho = ly.w;
    xka = omega / a;
    xkb = omega / b;
    t = b * iom;
    gammk = 2.0 * t * t;
    gam = gammk * wvno2;
    ra = sqrt((wvno + xka) * fabs(wvno - xka));
    rb = sqrt((wvno + xkb) * fabs(wvno - xkb));
    const double p = ra * dpth, q = rb * dpth;
    // var (surfdisp96.f:901-1018)
    double w, x, cosp, y, z, cosq, pex = 0.0, sex = 0.0;
    if (wvno < xka) {
      double sp, cp;
      sincos(p, &sp, &cp);
      w = sp / ra; x = -ra * sp; cosp = cp;
    } else if (wvno == xka) {
      cosp = 1.0; w = dpth; x = 0.0;
    } else {
      pex = p;
      double fac = (p < 16.0) ? exp(-2.0 * p) : 0.0;
      cosp = (1.0 + fac) * 0.5;
      double sp = (1.0 - fac) * 0.5;
      w = sp / ra; x = ra * sp;
    }
    if (wvno < xkb) {
      double sq, cq;
      sincos(q, &sq, &cq);
      y = sq / rb; z = -rb * sq; cosq = cq;
    } else if (wvno == xkb) {
      cosq = 1.0; y = dpth; z = 0.0;
    } else {
      sex = q;
      double fac = (q < 16.0) ? exp(-2.0 * q) : 0.0;
      cosq = (1.0 + fac) * 0.5;
      double sq = (1.0 - fac) * 0.5;
      y = sq / rb; z = rb * sq;
    }
    const double exa = pex + sex;
    const double a0 = (exa < 60.0) ? exp(-exa) : 0.0;
    const double cpcq = cosp * cosq, cpy = cosp * y, cpz = cosp * z, cqw = cosq * w, cqx = cosq * x;
    const double xy = x * y, xz = x * z, wy = w * y, wz = w * z;
    // dnka (surfdisp96.f:1051-1095)
    const double irho = 1.0 / rho;
    gamm1 = gam - 1.0;
    const double twgm1 = gam + gamm1, gmgmk = gam * gammk, gmgm1 = gam * gamm1, gm1sq = gamm1 * gamm1;
    const double rho2 = rho * rho, irho2 = irho * irho;
    const double a0pq = a0 - cpcq;
    const double c11 = cpcq - 2.0 * gmgm1 * a0pq - gmgmk * xz - wvno2 * gm1sq * wy;
    const double c12 = (wvno2 * cpy - cqx) * irho;
    const double c13 = -(twgm1 * a0pq + gammk * xz + wvno2 * gamm1 * wy) * irho;
    const double c14 = (cpz - wvno2 * cqw) * irho;
    const double c15 = -(2.0 * wvno2 * a0pq + xz + wvno2 * wvno2 * wy) * irho2;
    const double c21 = (gmgmk * cpz - gm1sq * cqw) * rho;
    const double c22 = cpcq;
    const double c23 = gammk * cpz - gamm1 * cqw;
    const double c24 = -wz;
    const double c41 = (gm1sq * cpy - gmgmk * cqx) * rho;
    const double c42 = -xy;
    const double c43 = gamm1 * cpy - gammk * cqx;
    const double c51 = -(2.0 * gmgmk * gm1sq * a0pq + gmgmk * gmgmk * xz + gm1sq * gm1sq * wy) * rho2;
    const double c53 = -(gammk * gamm1 * twgm1 * a0pq + gam * gammk * gammk * xz + gamm1 * gm1sq * wy) * rho;
    const double tt = -2.0 * wvno2;
    const double c31 = tt * c53, c32 = tt * c43, c33 = a0 + 2.0 * (cpcq - c11), c34 = tt * c23, c35 = tt * c13;
    // ee(i) = sum_j e(j) ca(j,i); ca rows: 1:(c11..c15) 2:(c21,c22,c23,c24,c14)
    // 3:(c31..c35) 4:(c41,c42,c43,c22,c12) 5:(c51,c41,c53,c21,c11)
    double f0 = e0 * c11 + e1 * c21 + e2 * c31 + e3 * c41 + e4 * c51;
    double f1 = e0 * c12 + e1 * c22 + e2 * c32 + e3 * c42 + e4 * c41;
    double f2 = e0 * c13 + e1 * c23 + e2 * c33 + e3 * c43 + e4 * c53;
    double f3 = e0 * c14 + e1 * c24 + e2 * c34 + e3 * c22 + e4 * c21;
    double f4 = e0 * c15 + e1 * c14 + e2 * c35 + e3 * c12 + e4 * c11;
    // normc (surfdisp96.f:1022-1047): divide by the largest magnitude
    double t1 = fmax(fmax(fmax(fabs(f0), fabs(f1)), fmax(fabs(f2), fabs(f3))), fabs(f4));
    if (t1 < 1.e-40) t1 = 1.0;
    const double it1 = 1.0 / t1;
    e0 = f0 * it1; e1 = f1 * it1; e2 = f2 * it1; e3 = f3 * it1; e4 = f4 * it1;
  }
  if (V.llw != 1) {
    float4 ly = V.get(0);
    const double a0l = ly.y, dpth = ly.x, rho = ly.w;
    xka = omega / a0l;
    ra = sqrt((wvno + xka) * fabs(wvno - xka));
    const double p = ra * dpth;
    double w, cosp;
    if (wvno < xka) {
      double sp, cp;
      sincos(p, &sp, &cp);
      w = sp / ra; cosp = cp;
    } else if (wvno == xka) {
      cosp = 1.0; w = dpth;
    } else {
      double fac = (p < 16.0) ? exp(-2.0 * p) : 0.0;
      cosp = (1.0 + fac) * 0.5;
      w = ((1.0 - fac) * 0.5) / ra;
    }
    const double w0 = -rho * w;
    return cosp * e0 + w0 * e1;
  }
  return e0;
}

// dltar1 (surfdisp96.f:734-794)
SWDK_HDI double dltar1(const LayerView& V, double wvno, double omega) {
  float4 h = V.get(V.L - 1);
  double beta1 = h.z, rho1 = h.w;
  double xkb = omega / beta1;
  double rb = sqrt((wvno + xkb) * fabs(wvno - xkb));
  double e1 = rho1 * rb;
  double e2 = 1.0 / (beta1 * beta1);
  for (int m = V.L - 2; m >= V.llw - 1; --m) {
    float4 ly = V.get(m);
    beta1 = ly.z;
    rho1 = ly.w;
    const double dpth = ly.x;
    const double xmu = rho1 * beta1 * beta1;
    xkb = omega / beta1;
    rb = sqrt((wvno + xkb) * fabs(wvno - xkb));
    const double q = dpth * rb;
    double cosq, y, z;
    if (wvno < xkb) {
      double sq, cq;
      sincos(q, &sq, &cq);
      y = sq / rb; z = -rb * sq; cosq = cq;
    } else if (wvno == xkb) {
      cosq = 1.0; y = dpth; z = 0.0;
    } else {
      double fac = (q < 16.0) ? exp(-2.0 * q) : 0.0;
      cosq = (1.0 + fac) * 0.5;
      double sq = (1.0 - fac) * 0.5;
      y = sq / rb; z = rb * sq;
    }
    const double e10 = e1 * cosq + e2 * xmu * z;
    const double e20 = e1 * y / xmu + e2 * cosq;
    double xnor = fmax(fabs(e10), fabs(e20));
    if (xnor < 1.e-40) xnor = 1.0;
    const double ix = 1.0 / xnor;
    e1 = e10 * ix;
    e2 = e20 * ix;
  }
  return e1;
}

// 1/x for the positive, normal layer parameters: the hardware estimate
// (PTX rcp.approx.ftz.f64) refined by two Newton-Raphson steps
// r <- r + r (1 - x r), each with fused multiply-adds; the relative error
// is then below one unit in the last place.  Computing the reciprocals here
// instead of reading FP64 tables keeps one float4 per layer as the only
// memory traffic of an evaluation.
SWDK_HD double recip(double x) {
#ifdef __CUDA_ARCH__
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  double e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  e = fma(-x, r, 1.0);
  return fma(r, e, r);
#else
  return 1.0 / x;
#endif
}

// dltar4 with the per-layer reciprocals (1/a, 1/b, 1/rho) from recip(), the
// vertical wavenumber and its reciprocal from one rsqrt, exp(-(p+q)) as
// exp(-p) exp(-q), and the max-normalisation applied every NORM layers
// (NORM = 1 is surfdisp96's per-layer normc; larger NORM rescales the
// propagated vector by a different positive factor, which changes neither
// the sign nor the continuity of the period equation in c).
struct LayerCoef {
  double a0, cpcq, cpy, cpz, cqw, cqx, xy, xz, wy, wz, gam, gammk, rho, irho;
};

SWDK_HD LayerCoef layer_coef(const float4 ly, double wvno, double wvno2, double omega, double iom) {
  LayerCoef k;
  k.irho = recip((double)ly.w);
  const double dpth = ly.x;
  k.rho = ly.w;
  const double xka = omega * recip((double)ly.y), xkb = omega * recip((double)ly.z);
  const double t = (double)ly.z * iom;
  k.gammk = 2.0 * t * t;
  k.gam = k.gammk * wvno2;
  const double Xa = (wvno + xka) * fabs(wvno - xka);
  const double Xb = (wvno + xkb) * fabs(wvno - xkb);
  // var (surfdisp96.f:901-1018); ep = exp(-pex), eq = exp(-sex)
  double w, x, cosp, y, z, cosq, ep = 1.0, eq = 1.0, pex = 0.0, sex = 0.0;
  if (wvno < xka) {
    const double ir = rsqrt(Xa), r = Xa * ir;
    double sp, cp;
    sincos(r * dpth, &sp, &cp);
    w = sp * ir; x = -r * sp; cosp = cp;
  } else if (wvno == xka) {
    cosp = 1.0; w = dpth; x = 0.0;
  } else {
    const double ir = rsqrt(Xa), r = Xa * ir, p = r * dpth;
    pex = p;
    ep = (p < 60.0) ? exp(-p) : 0.0;
    const double fac = (p < 16.0) ? ep * ep : 0.0;
    cosp = (1.0 + fac) * 0.5;
    const double sp = (1.0 - fac) * 0.5;
    w = sp * ir; x = r * sp;
  }
  if (wvno < xkb) {
    const double ir = rsqrt(Xb), r = Xb * ir;
    double sq, cq;
    sincos(r * dpth, &sq, &cq);
    y = sq * ir; z = -r * sq; cosq = cq;
  } else if (wvno == xkb) {
    cosq = 1.0; y = dpth; z = 0.0;
  } else {
    const double ir = rsqrt(Xb), r = Xb * ir, q = r * dpth;
    sex = q;
    eq = (q < 60.0) ? exp(-q) : 0.0;
    const double fac = (q < 16.0) ? eq * eq : 0.0;
    cosq = (1.0 + fac) * 0.5;
    const double sq = (1.0 - fac) * 0.5;
    y = sq * ir; z = r * sq;
  }
  // a0 = exp(-(pex+sex)) when pex+sex < 60 (both factors then below 60)
  k.a0 = (pex + sex < 60.0) ? ep * eq : 0.0;
  k.cpcq = cosp * cosq; k.cpy = cosp * y; k.cpz = cosp * z; k.cqw = cosq * w; k.cqx = cosq * x;
  k.xy = x * y; k.xz = x * z; k.wy = w * y; k.wz = w * z;
  return k;
}

// e <- e * Dunkin(k) (surfdisp96.f:1051-1095 and dltar4's product)
SWDK_HD void apply_dunkin(const LayerCoef& k, double wvno2, double& e0, double& e1, double& e2, double& e3,
                          double& e4) {
  const double gam = k.gam, gammk = k.gammk, rho = k.rho, irho = k.irho;
  const double gamm1 = gam - 1.0;
  const double twgm1 = gam + gamm1, gmgmk = gam * gammk, gmgm1 = gam * gamm1, gm1sq = gamm1 * gamm1;
  const double rho2 = rho * rho, irho2 = irho * irho;
  const double a0pq = k.a0 - k.cpcq;
  const double c11 = k.cpcq - 2.0 * gmgm1 * a0pq - gmgmk * k.xz - wvno2 * gm1sq * k.wy;
  const double c12 = (wvno2 * k.cpy - k.cqx) * irho;
  const double c13 = -(twgm1 * a0pq + gammk * k.xz + wvno2 * gamm1 * k.wy) * irho;
  const double c14 = (k.cpz - wvno2 * k.cqw) * irho;
  const double c15 = -(2.0 * wvno2 * a0pq + k.xz + wvno2 * wvno2 * k.wy) * irho2;
  const double c21 = (gmgmk * k.cpz - gm1sq * k.cqw) * rho;
  const double c22 = k.cpcq;
  const double c23 = gammk * k.cpz - gamm1 * k.cqw;
  const double c24 = -k.wz;
  const double c41 = (gm1sq * k.cpy - gmgmk * k.cqx) * rho;
  const double c42 = -k.xy;
  const double c43 = gamm1 * k.cpy - gammk * k.cqx;
  const double c51 = -(2.0 * gmgmk * gm1sq * a0pq + gmgmk * gmgmk * k.xz + gm1sq * gm1sq * k.wy) * rho2;
  const double c53 = -(gammk * gamm1 * twgm1 * a0pq + gam * gammk * gammk * k.xz + gamm1 * gm1sq * k.wy) * rho;
  const double tt = -2.0 * wvno2;
  const double c31 = tt * c53, c32 = tt * c43, c33 = k.a0 + 2.0 * (k.cpcq - c11), c34 = tt * c23, c35 = tt * c13;
  const double f0 = e0 * c11 + e1 * c21 + e2 * c31 + e3 * c41 + e4 * c51;
  const double f1 = e0 * c12 + e1 * c22 + e2 * c32 + e3 * c42 + e4 * c41;
  const double f2 = e0 * c13 + e1 * c23 + e2 * c33 + e3 * c43 + e4 * c53;
  const double f3 = e0 * c14 + e1 * c24 + e2 * c34 + e3 * c22 + e4 * c21;
  const double f4 = e0 * c15 + e1 * c14 + e2 * c35 + e3 * c12 + e4 * c11;
  e0 = f0; e1 = f1; e2 = f2; e3 = f3; e4 = f4;
}

template <int NORM, bool NODES>
SWDK_HDI double dltar4_fast(const LayerView& V, double wvno, double omga) {
  double omega = omga;
  if (omega < 1.0e-4) omega = 1.0e-4;
  const double wvno2 = wvno * wvno;
  const double iom = 1.0 / omega;
  const int hs = V.L - 1;  // the half-space
  const float4 h = V.layer(hs);
  double xka = omega * recip((double)h.y), xkb = omega * recip((double)h.z);
  const double ra = sqrt((wvno + xka) * fabs(wvno - xka));
  const double rb = sqrt((wvno + xkb) * fabs(wvno - xkb));
  const double t = (double)h.z * iom;
  const double gammk = 2.0 * t * t;
  const double gam = gammk * wvno2;
  const double gamm1 = gam - 1.0;
  const double rho1 = h.w;
  double e0 = rho1 * rho1 * (gamm1 * gamm1 - gam * gammk * ra * rb);
  double e1 = -rho1 * ra;
  double e2 = rho1 * (gamm1 - gammk * ra * rb);
  double e3 = rho1 * rb;
  double e4 = wvno2 - ra * rb;
  const int mlo = V.llw - 1;
  int since = 0;
  LayerView::Walk wk;
  auto norm_e = [&](int m) {
    if (++since >= NORM || m == mlo) {
      since = 0;
      double t1 = fmax(fmax(fmax(fabs(e0), fabs(e1)), fmax(fabs(e2), fabs(e3))), fabs(e4));
      if (t1 < 1.e-40) t1 = 1.0;
      if (NORM == 1) {
        e0 = e0 / t1; e1 = e1 / t1; e2 = e2 / t1; e3 = e3 / t1; e4 = e4 / t1;
      } else {
        const double it1 = 1.0 / t1;
        e0 *= it1; e1 *= it1; e2 *= it1; e3 *= it1; e4 *= it1;
      }
    }
  };
  if (hs - 1 >= mlo) {
    V.walk_start<-1, NODES>(wk, hs - 1);
    LayerCoef cur = layer_coef(V.walk_layer<-1, NODES>(wk, hs - 1), wvno, wvno2, omega, iom);
    int m = hs - 1;
    for (; m > mlo; --m) {
      // the next layer's coefficients do not depend on e: computed while
      // this layer's product runs (root search 336 -> 327 ms per step)
      const float4 nly = V.walk_layer<-1, NODES>(wk, m - 1);
      apply_dunkin(cur, wvno2, e0, e1, e2, e3, e4);
      cur = layer_coef(nly, wvno, wvno2, omega, iom);
      norm_e(m);
    }
    apply_dunkin(cur, wvno2, e0, e1, e2, e3, e4);
    norm_e(m);
  }
  if (V.llw != 1) {
    const float4 ly = V.layer(0);
    const double dpth = ly.x, rho = ly.w;
    xka = omega * recip((double)ly.y);
    const double Xa = (wvno + xka) * fabs(wvno - xka);
    double w, cosp;
    if (wvno < xka) {
      const double ir = rsqrt(Xa), r = Xa * ir;
      double sp, cp;
      sincos(r * dpth, &sp, &cp);
      w = sp * ir; cosp = cp;
    } else if (wvno == xka) {
      cosp = 1.0; w = dpth;
    } else {
      const double ir = rsqrt(Xa), r = Xa * ir, p = r * dpth;
      const double fac = (p < 16.0) ? exp(-2.0 * p) : 0.0;
      cosp = (1.0 + fac) * 0.5;
      w = ((1.0 - fac) * 0.5) * ir;
    }
    const double w0 = -rho * w;
    return cosp * e0 + w0 * e1;
  }
  return e0;
}

// dltar1 with 1/b and 1/(rho b^2) from recip()
template <int NORM, bool NODES>
SWDK_HDI double dltar1_fast(const LayerView& V, double wvno, double omega) {
  const int hs = V.L - 1;  // the half-space
  float4 h = V.layer(hs);
  double beta1 = h.z, rho1 = h.w;
  double xkb = omega * recip(beta1);
  double rb = sqrt((wvno + xkb) * fabs(wvno - xkb));
  double e1 = rho1 * rb;
  double e2 = 1.0 / (beta1 * beta1);
  int since = 0;
  const int mlo = V.llw - 1;
  LayerView::Walk wk;
  if (hs - 1 >= mlo) V.walk_start<-1, NODES>(wk, hs - 1);
  for (int m = hs - 1; m >= mlo; --m) {
    const float4 ly = V.walk_layer<-1, NODES>(wk, m);
    beta1 = ly.z;
    rho1 = ly.w;
    const double dpth = ly.x;
    const double xmu = rho1 * beta1 * beta1;
    const double ixmu = recip(xmu);
    xkb = omega * recip(beta1);
    const double Xb = (wvno + xkb) * fabs(wvno - xkb);
    double cosq, y, z;
    if (wvno < xkb) {
      const double ir = rsqrt(Xb), r = Xb * ir;
      double sq, cq;
      sincos(dpth * r, &sq, &cq);
      y = sq * ir; z = -r * sq; cosq = cq;
    } else if (wvno == xkb) {
      cosq = 1.0; y = dpth; z = 0.0;
    } else {
      const double ir = rsqrt(Xb), r = Xb * ir, q = dpth * r;
      const double fac = (q < 16.0) ? exp(-2.0 * q) : 0.0;
      cosq = (1.0 + fac) * 0.5;
      const double sq = (1.0 - fac) * 0.5;
      y = sq * ir; z = r * sq;
    }
    const double e10 = e1 * cosq + e2 * xmu * z;
    const double e20 = e1 * y * ixmu + e2 * cosq;
    if (++since >= NORM || m == V.llw - 1) {
      since = 0;
      double xnor = fmax(fabs(e10), fabs(e20));
      if (xnor < 1.e-40) xnor = 1.0;
      if (NORM == 1) { e1 = e10 / xnor; e2 = e20 / xnor; }
      else { const double ix2 = 1.0 / xnor; e1 = e10 * ix2; e2 = e20 * ix2; }
    } else {
      e1 = e10; e2 = e20;
    }
  }
  return e1;
}

SWDK_HD double secular(const LayerView& V, int iwave, double wvno, double omega) {
  return (iwave == 1) ? dltar1(V, wvno, omega) : dltar4(V, wvno, omega);
}

// production secular function: reciprocal-table variants; the reference
// refinement keeps per-layer normalisation like surfdisp96
SWDK_HD double secular_fast(const LayerView& V, int iwave, int refine, double wvno, double omega) {
  if (V.nodes) {
    if (refine == 0) return (iwave == 1) ? dltar1_fast<1, true>(V, wvno, omega) : dltar4_fast<1, true>(V, wvno, omega);
    return (iwave == 1) ? dltar1_fast<4, true>(V, wvno, omega) : dltar4_fast<4, true>(V, wvno, omega);
  }
  if (refine == 0) return (iwave == 1) ? dltar1_fast<1, false>(V, wvno, omega) : dltar4_fast<1, false>(V, wvno, omega);
  return (iwave == 1) ? dltar1_fast<4, false>(V, wvno, omega) : dltar4_fast<4, false>(V, wvno, omega);
}

// ---------------------------------------------------------------------------
// surfdisp96 period/mode continuation as a flat state machine.  Each call of
// chain_advance() runs control logic until it needs one secular-function
// value (returns true with s.creq set) or the chain is finished (false).
// ---------------------------------------------------------------------------
enum Phase : int {
  PH_CHAIN_START, PH_PERIOD_START, PH_GS_START, PH_GS_FIRST, PH_SCAN, PH_SCAN_GOT, PH_REFINE_START,
  PH_NEV_A, PH_NEV_TOP, PH_NEV_BODY_GOT, PH_NEV_BODY, PH_NEV_HALF_GOT, PH_NEV_NEV_GOT, PH_BRENT_STEP,
  PH_BRENT_GOT, PH_REFINE_DONE, PH_GS_OK, PH_GS_FAIL, PH_PERIOD_OUT, PH_FAIL, PH_MODE_END, PH_CHAIN_END,
  PH_RETRY_NEXT, PH_PROP_LO, PH_PROP_HI, PH_PROP_CHECK, PH_PROP_DOWN, PH_PROP_DOWN_GOT, PH_PROP_C1_GOT, PH_FIRST_NEXT, PH_FIRST_GOT, PH_DONE
};

struct ChainParams {
  const double* t;  // periods of the chain
  double rtol;      // Brent bracket tolerance (relative)
  double cc;        // start value 0.95*0.90*c_R(slowest layer), surfdisp96.f:206-226
  float betmx;      // largest shear velocity of the flattened model
  int16_t kmax;     // periods (<= KMAX_CHAIN)
  int16_t nmode;    // modes 1..nmode (surfdisp96 "mode")
  int8_t igr;       // 0 phase; >0 numerical group velocity (surfdisp96.f:241-248)
  int8_t iwave;     // 1 Love, 2 Rayleigh
  int8_t refine;    // 0 reference nevill, 1 Brent
  int8_t sngl;      // REAL*4 output like the reference
  int8_t retry;     // surfdisp()'s single-period retries (surfdisp.cpp:94-109): RETRY_*
};

// The chain state, parameters and output addressing of the root kernels live
// in shared memory (one of each per lane, 352 bytes together, 45 KB per
// 128-thread block); integer fields are as narrow as their ranges allow
// (periods <= KMAX_CHAIN, scan steps <= SCAN_CAP + 32, Brent steps <= 201,
// Neville points <= 10).
struct ChainState {
  double last;    // value of the last requested secular evaluation
  double creq;    // requested phase velocity
  double omega;   // 2 pi / t1 of the current root
  // surfdisp96 locals
  double t1;
  double c1, c2, clow, cm, del1, del2, del1st;
  // refinement
  double c3, del3, ra_, fa, rb_, fb, rc_, fc, rd, re;
  // learned proposals
  double plo, phi, fplo, c1s, del1s;
  // retries
  double sub_out;
  float t1a, t1b;
  int nevals;
  int16_t phase, next;
  int16_t iq, k, ift;
  int16_t nctrl, nscan;
  int16_t pm, nprop_ok, nprop_fail;
  int16_t pj;  // first-period proposal: grid index of the last coarse point checked
  int16_t rq_m, rq_k, iterlim;
  int8_t ierr, ifirst, idir, gpass;
  int8_t nev, m, sub;
};

// Output callback: slot (mode iq, period k) gets value v; the caller owns
// storage.  out(mode-1, k-1) addressing is done by the kernel.
struct ChainIO {
  double* c;    // [KMAX_CHAIN] continuation array (surfdisp96 c())
  double* cb;   // [KMAX_CHAIN] group continuation (surfdisp96 cb())
  double* out;  // out[(iq-1)*stride + (k-1)*ostride]
  int stride, ostride;
  int32_t* st;  // status, same addressing as out
  const float2* prop;  // learned (c, half-width) per (mode, period), same addressing; may be null
};

// Retries of failed periods (surfdisp.cpp:94-109): none; inline, one after
// the other at the end of the chain; deferred, i.e. the caller collects the
// failed slots of a chain with ierr != 0 and runs each as its own work item;
// one such item (a single-period chain for slot (rq_m, rq_k)).
constexpr int RETRY_NONE = 0, RETRY_INLINE = 1, RETRY_DEFERRED = 2, RETRY_ONE = 3;

constexpr double ONE_DC = 1.0e-2;  // surfdisp96 "one"
constexpr double ONEA = 1.5;       // dble(sone0)
constexpr double DC = (double)0.005f;
constexpr float HGR = 0.005f;
constexpr int SCAN_CAP = 20000;    // guard against non-finite inputs (legit scans need < 2000)

SWDK_HD double& out_at(const ChainIO& io, int iq, int k) {
  return io.out[(size_t)(iq - 1) * io.stride + (size_t)(k - 1) * io.ostride];
}
SWDK_HD int32_t& st_at(const ChainIO& io, int iq, int k) {
  return io.st[(size_t)(iq - 1) * io.stride + (size_t)(k - 1) * io.ostride];
}

// a single-period retry of slot (mode m, period k) as its own chain
SWDK_HD void chain_init_retry(ChainState& s, int m, int k);

SWDK_HD void chain_init(ChainState& s) {
  s.phase = PH_CHAIN_START;
  s.nprop_ok = 0;
  s.nprop_fail = 0;
  s.sub = 0;
  s.iterlim = 0;
  s.nevals = 0;
  s.last = 0.0;
  s.del1st = 0.0;
}

SWDK_HD void chain_init_retry(ChainState& s, int m, int k) {
  chain_init(s);
  s.sub = 1;
  s.rq_m = m;
  s.rq_k = k;
}

// Learned proposals live on the reference's scan grid g_j = c1 + j*dc
// (surfdisp96.f:452-470).  For period k > 1 of a mode, taking the scan to go
// upward from c1 (f(c1) with the mode's polarity del1st; f(c1) itself is
// evaluated only when the walk reaches c1 or the proposal is dropped), the
// network's anchored estimate
//   c* = c(k-1) + (mu(k) - mu(k-1))
// (a bias of the network that is smooth in period cancels) names the grid
// cell [g_m, g_m+1] expected to hold the root.  f is evaluated at both cell
// ends: a sign change from the polarity del1st to the opposite one is the
// cell the scan would have reached; otherwise the scan walks from that cell
// up or down, one grid step at a time, to the sign change.  The cell and
// hence the refinement are the plain scan's own.  The stretch [c1, g_m]
// is not walked step by step, so the proposal is used only where that
// saves steps (m >= 2) and the stretch is short: m*dc <= PROP_GAP_PER_S * T.
constexpr double PROP_GAP_PER_S = 0.01;

SWDK_HD bool proposal_cell(const ChainState& s, const ChainParams& P, const ChainIO& io, int& m) {
  if (!io.prop || s.sub || P.igr > 0 || P.refine != 1 || s.k < 2 || s.gpass != 0 || s.del1st == 0.0) return false;
  const size_t base = (size_t)(s.iq - 1) * io.stride;
  const float2 pr = io.prop[base + (size_t)(s.k - 1) * io.ostride];
  const float2 pp = io.prop[base + (size_t)(s.k - 2) * io.ostride];
  if (!(pr.y > 0.0f) || !(pr.y <= 0.25f) || !(pp.y > 0.0f)) return false;
  const double cs = io.c[s.k - 2] + ((double)pr.x - (double)pp.x);
  const double x = (cs - s.c1) / DC;
  if (!(x >= 2.0) || !(x < 1.0e4)) return false;
  m = (int)floor(x);
  if ((double)m * DC > PROP_GAP_PER_S * s.t1) return false;
  return s.c1 + (double)(m + 1) * DC < (double)P.betmx + DC;
}

// The first period of a Rayleigh chain's first mode scans from cc, on
// average about 90 grid steps below the root.  There the proposal is the
// network's absolute estimate c* (no previous root to anchor it), and the
// stretch [c1, g_m] below its cell is checked at every FIRST_STRIDE-th grid
// point instead of being skipped: each checked point must keep the
// polarity of f(c1); the first that does not ends the check, and the
// reference's scan resumes one grid step at a time from the checked point
// below it, so it reaches the first sign change of the plain scan.  This
// holds unless the first two roots lie inside one coarse interval (and the
// estimate lies above both): the fundamental and first higher Rayleigh
// modes are at least 0.05 km/s apart at 1-2 s on the default and 0.2 km/s
// on the production grid, above the coarse interval of 0.02 km/s.  Love
// chains keep the plain scan: their first two modes come as close as
// 0.001 km/s at short periods; so do higher Rayleigh modes, whose first
// period scans up from the mode below (modes 1 and 2 as close as
// 0.0002 km/s).
constexpr int FIRST_STRIDE = 4;

SWDK_HD bool first_cell(const ChainState& s, const ChainParams& P, const ChainIO& io, int& m) {
  if (!io.prop || s.sub || P.igr > 0 || P.refine != 1 || P.iwave != 2 || s.k != 1 || s.iq != 1 || s.gpass != 0 ||
      s.ifirst != 1 || s.del1st == 0.0)
    return false;
  const float2 pr = io.prop[0];  // (mode 1, period 1)
  if (!(pr.y > 0.0f) || !(pr.y <= 0.25f)) return false;
  const double x = ((double)pr.x - s.c1) / DC;
  if (!(x >= 4.0 * FIRST_STRIDE) || !(x < 1.0e4)) return false;
  m = (int)floor(x);
  return s.c1 + (double)(m + 1) * DC < (double)P.betmx + DC;
}

// grid point c1 + j*dc, accumulated like the scan does
SWDK_HD double scan_grid(double c1, int j) {
  double c = c1;
  for (int i = 0; i < j; ++i) c = c + DC;
  return c;
}

// Evaluation phases counted by the root kernels' statistics: the getsol
// scan of a mode's first period, the scan of later periods (and of group
// passes and dropped proposals), the learned cell's two ends, the walk from
// a learned cell, the refinement, and the single-period retries.
constexpr int EV_SCAN_FIRST = 0, EV_SCAN = 1, EV_CELL = 2, EV_WALK = 3, EV_REFINE = 4, EV_RETRY = 5;
constexpr int NPHASE_EV = 6;

// request a secular-function value at c; continue with phase nxt
#define SWDK_REQ(cv, nxt) do { s.creq = (cv); s.next = (nxt); return true; } while (0)

SWDK_HDI bool chain_advance(ChainState& s, const ChainParams& P, const ChainIO& io) {
  for (;;) {
    // parameters of the active chain: the main chain or a single-period retry
    const double* tp = s.sub ? (P.t + (s.rq_k - 1)) : P.t;
    const int kmax = s.sub ? 1 : P.kmax;
    const int nmode = s.sub ? s.rq_m : P.nmode;
    switch (s.phase) {
      case PH_CHAIN_START: {
        s.ift = 999;
        s.ierr = 0;
        s.iq = 1;
        s.k = 1;
        s.cm = P.cc;
        s.c1 = P.cc;
        s.clow = P.cc;
        for (int i = 0; i < kmax; ++i) { io.c[i] = 0.0; io.cb[i] = 0.0; }
        s.phase = PH_PERIOD_START;
        break;
      }
      case PH_PERIOD_START: {
        if (s.k > kmax) { s.phase = PH_MODE_END; break; }
        if (s.k >= s.ift) { s.phase = PH_FAIL; break; }
        double t1 = tp[s.k - 1];
        if (P.igr > 0) {
          s.t1a = (float)(t1 / (double)(1.0f + HGR));
          s.t1b = (float)(t1 / (double)(1.0f - HGR));
          t1 = (double)s.t1a;
        } else {
          s.t1a = (float)t1;
        }
        s.t1 = t1;
        const int k = s.k, iq = s.iq;
        if (k == 1 && iq == 1) { s.c1 = P.cc; s.clow = P.cc; s.ifirst = 1; }
        else if (k == 1 && iq > 1) { s.c1 = io.c[0] + ONE_DC * DC; s.clow = s.c1; s.ifirst = 1; }
        else if (k > 1 && iq > 1) {
          s.ifirst = 0;
          s.clow = io.c[k - 1] + ONE_DC * DC;
          s.c1 = io.c[k - 2];
          if (s.c1 < s.clow) s.c1 = s.clow;
        } else {
          s.ifirst = 0;
          s.c1 = io.c[k - 2] - ONEA * DC;
          s.clow = s.cm;
        }
        s.gpass = 0;
        s.pj = -1;  // the first-period jump is tried once per period (a fallback rescans from c1)
        s.phase = PH_GS_START;
        int m;
        if (proposal_cell(s, P, io, m)) {
          // learned cell: f(c1) is evaluated only if the walk or a fallback
          // needs it; until then the scan is taken to go up, i.e. f(c1) to
          // have the mode's polarity del1st (surfdisp96.f:446-451)
          s.omega = TWOPI / s.t1;
          s.c1s = s.c1;
          s.del1s = s.del1st;
          s.idir = 1;
          s.nscan = 0;
          s.pm = m;
          s.plo = scan_grid(s.c1, m);
          s.phi = s.plo + DC;
          s.phase = PH_PROP_LO;
        }
        break;
      }
      case PH_PROP_LO: {
        SWDK_REQ(s.plo, PH_PROP_HI);
      }
      case PH_PROP_HI: {
        s.fplo = s.last;
        SWDK_REQ(s.phi, PH_PROP_CHECK);
      }
      case PH_PROP_CHECK: {
        const double fphi = s.last;
        const bool lo_same = dsign1(s.fplo) == dsign1(s.del1s), hi_same = dsign1(fphi) == dsign1(s.del1s);
        if (lo_same && !hi_same) {  // the cell of the sign change
          s.nprop_ok++;
          s.c1 = s.plo; s.del1 = s.fplo; s.c2 = s.phi; s.del2 = fphi;
          s.phase = PH_REFINE_START;
        } else if (lo_same) {  // root above the cell: scan on upward from g_m+1
          s.nprop_ok++;
          s.c1 = s.phi; s.del1 = fphi;
          s.phase = PH_SCAN;
        } else if (!hi_same) {  // root below the cell: walk down from g_m
          s.nprop_ok++;
          s.c2 = s.plo; s.del2 = s.fplo;
          s.pm = s.pm - 1;
          s.phase = PH_PROP_DOWN;
        } else {  // two sign changes inside one cell: the plain search from c1
          s.nprop_fail++;
          s.c1 = s.c1s;
          s.phase = PH_GS_START;
        }
        break;
      }
      case PH_PROP_DOWN: {  // c2 = g_pm+1 has the opposite sign; try g_pm
        if (s.pm <= 0) {  // cell [c1, g_1]: f(c1) itself is needed now
          SWDK_REQ(s.c1s, PH_PROP_C1_GOT);
        }
        s.plo = scan_grid(s.c1s, s.pm);
        SWDK_REQ(s.plo, PH_PROP_DOWN_GOT);
      }
      case PH_PROP_C1_GOT: {
        if (dsign1(s.last) == dsign1(s.del1s)) {  // as assumed: the cell [c1, g_1]
          s.c1 = s.c1s; s.del1 = s.last;
          s.phase = PH_REFINE_START;
        } else {  // f(c1) has the other polarity: the reference scans down from c1
          s.nprop_fail++;
          s.c1 = s.c1s;
          s.phase = PH_GS_START;
        }
        break;
      }
      case PH_PROP_DOWN_GOT: {
        if (dsign1(s.last) == dsign1(s.del1s)) {  // sign change in [g_pm, g_pm+1]
          s.c1 = s.plo; s.del1 = s.last;
          s.phase = PH_REFINE_START;
        } else {
          s.c2 = s.plo; s.del2 = s.last;
          s.pm = s.pm - 1;
          s.phase = PH_PROP_DOWN;
        }
        break;
      }
      case PH_GS_START: {  // getsol entry (surfdisp96.f:439-451)
        s.omega = TWOPI / s.t1;
        s.nscan = 0;
        SWDK_REQ(s.c1, PH_GS_FIRST);
      }
      case PH_GS_FIRST: {
        s.del1 = s.last;
        if (s.ifirst == 1) s.del1st = s.del1;
        const double plmn = dsign1(s.del1st) * dsign1(s.del1);
        if (s.ifirst == 1) s.idir = 1;
        else if (plmn >= 0.0) s.idir = 1;
        else s.idir = -1;
        s.phase = PH_SCAN;
        int m;
        if (s.pj == -1 && first_cell(s, P, io, m)) {  // the first period: checked jump to the learned cell
          s.c1s = s.c1;
          s.del1s = s.del1st;
          s.pm = m;
          s.pj = 0;
          s.plo = s.c1;
          s.fplo = s.del1;
          s.phase = PH_FIRST_NEXT;
        }
        break;
      }
      case PH_FIRST_NEXT: {  // next coarse point below the cell, or the cell
        if (s.pj + FIRST_STRIDE < s.pm) {
          double c = s.plo;
          for (int i = 0; i < FIRST_STRIDE; ++i) c = c + DC;
          s.phi = c;
          SWDK_REQ(c, PH_FIRST_GOT);
        }
        // every checked point kept the polarity: the cell [g_m, g_m+1]
        double c = s.plo;
        for (int i = s.pj; i < s.pm; ++i) c = c + DC;
        s.plo = c;
        s.phi = c + DC;
        s.idir = 1;
        s.nscan = s.pm;
        s.phase = PH_PROP_LO;
        break;
      }
      case PH_FIRST_GOT: {
        if (dsign1(s.last) == dsign1(s.del1s)) {
          s.plo = s.phi;
          s.fplo = s.last;
          s.pj = s.pj + FIRST_STRIDE;
          s.phase = PH_FIRST_NEXT;
          break;
        }
        // a sign change in (plo, phi]: the reference's scan from plo
        s.nprop_fail++;
        s.c1 = s.plo;
        s.del1 = s.fplo;
        s.idir = 1;
        s.nscan = s.pj;
        s.phase = PH_SCAN;
        break;
      }
      case PH_SCAN: {  // label 1000
        s.c2 = (s.idir > 0) ? s.c1 + DC : s.c1 - DC;
        if (s.c2 <= s.clow) { s.idir = 1; s.c1 = s.clow; break; }
        if (++s.nscan > SCAN_CAP) { s.phase = PH_GS_FAIL; break; }
        SWDK_REQ(s.c2, PH_SCAN_GOT);
      }
      case PH_SCAN_GOT: {
        s.del2 = s.last;
        if (dsign1(s.del1) != dsign1(s.del2)) { s.phase = PH_REFINE_START; break; }
        s.c1 = s.c2;
        s.del1 = s.del2;
        if (s.c1 < s.cm || s.c1 >= ((double)P.betmx + DC) || !(s.c1 == s.c1)) { s.phase = PH_GS_FAIL; break; }
        s.phase = PH_SCAN;
        break;
      }
      case PH_REFINE_START: {
        if (P.refine == 0) {
          s.c3 = 0.5 * (s.c1 + s.c2);
          SWDK_REQ(s.c3, PH_NEV_A);
        }
        s.ra_ = s.c1; s.fa = s.del1; s.rb_ = s.c2; s.fb = s.del2;
        s.rc_ = s.ra_; s.fc = s.fa; s.rd = s.rb_ - s.ra_; s.re = s.rd;
        s.nctrl = 0;
        s.phase = PH_BRENT_STEP;
        break;
      }
      // ---- nevill (surfdisp96.f:575-694), bracket kept in c1/c2 ----
      case PH_NEV_A: {
        s.del3 = s.last;
        s.nev = 1; s.nctrl = 1; s.m = 1;
        s.phase = PH_NEV_TOP;
        break;
      }
      case PH_NEV_TOP: {
        s.nctrl = s.nctrl + 1;
        if (s.nctrl >= 100) { s.iterlim++; s.phase = PH_REFINE_DONE; break; }
        if (s.c3 < fmin(s.c1, s.c2) || s.c3 > fmax(s.c1, s.c2)) {
          s.nev = 0;
          s.c3 = 0.5 * (s.c1 + s.c2);
          SWDK_REQ(s.c3, PH_NEV_BODY_GOT);
        }
        s.phase = PH_NEV_BODY;
        break;
      }
      case PH_NEV_BODY_GOT: {
        s.del3 = s.last;
        s.phase = PH_NEV_BODY;
        break;
      }
      case PH_NEV_BODY: {
        const double s13 = s.del1 - s.del3;
        const double s32 = s.del3 - s.del2;
        if (dsign1(s.del3) * dsign1(s.del1) < 0.0) { s.c2 = s.c3; s.del2 = s.del3; }
        else { s.c1 = s.c3; s.del1 = s.del3; }
        if (fabs(s.c1 - s.c2) <= 1.e-6 * s.c1) { s.phase = PH_REFINE_DONE; break; }
        if (dsign1(s13) != dsign1(s32)) s.nev = 0;
        const double ss1 = fabs(s.del1), s1 = (double)0.01f * ss1;
        const double ss2 = fabs(s.del2), s2 = (double)0.01f * ss2;
        if (s1 > ss2 || s2 > ss1 || s.nev == 0) {
          s.c3 = 0.5 * (s.c1 + s.c2);
          SWDK_REQ(s.c3, PH_NEV_HALF_GOT);
        }
        // Neville on x(y) (surfdisp96.f:654-682); x/y held in io.cb tail
        double* x = io.cb + KMAX_CHAIN;
        double* y = x + 12;
        int m = s.m;
        if (s.nev == 2) { x[m] = s.c3; y[m] = s.del3; }
        else { x[0] = s.c1; y[0] = s.del1; x[1] = s.c2; y[1] = s.del2; m = 1; }
        s.m = m;
        bool bad = false;
        for (int kk = 1; kk <= m; ++kk) {
          const int j = m - kk + 1;
          const double denom = y[m] - y[j - 1];
          if (fabs(denom) < 1.0e-10 * fabs(y[m])) { bad = true; break; }
          x[j - 1] = (-y[j - 1] * x[j] + y[m] * x[j - 1]) / denom;
        }
        if (bad) {
          s.c3 = 0.5 * (s.c1 + s.c2);
          SWDK_REQ(s.c3, PH_NEV_HALF_GOT);
        }
        s.c3 = x[0];
        SWDK_REQ(s.c3, PH_NEV_NEV_GOT);
      }
      case PH_NEV_HALF_GOT: {
        s.del3 = s.last;
        s.nev = 1; s.m = 1;
        s.phase = PH_NEV_TOP;
        break;
      }
      case PH_NEV_NEV_GOT: {
        s.del3 = s.last;
        s.nev = 2;
        s.m = s.m + 1;
        if (s.m > 10) s.m = 10;
        s.phase = PH_NEV_TOP;
        break;
      }
      // ---- tight refinement: Brent's zeroin on the scan bracket ----
      case PH_BRENT_STEP: {
        if (signbit(s.fb) == signbit(s.fc)) { s.rc_ = s.ra_; s.fc = s.fa; s.rd = s.rb_ - s.ra_; s.re = s.rd; }
        if (fabs(s.fc) < fabs(s.fb)) {
          s.ra_ = s.rb_; s.rb_ = s.rc_; s.rc_ = s.ra_;
          s.fa = s.fb; s.fb = s.fc; s.fc = s.fa;
        }
        const double eps = 2.220446049250313e-16;
        const double tol1 = 2.0 * eps * fabs(s.rb_) + 0.5 * P.rtol * fabs(s.rb_);
        const double xm = 0.5 * (s.rc_ - s.rb_);
        if (fabs(xm) <= tol1 || s.fb == 0.0) { s.c3 = s.rb_; s.phase = PH_REFINE_DONE; break; }
        if (++s.nctrl > 200) { s.iterlim++; s.c3 = s.rb_; s.phase = PH_REFINE_DONE; break; }
        if (fabs(s.re) >= tol1 && fabs(s.fa) > fabs(s.fb)) {
          const double sr = s.fb / s.fa;
          double p, q;
          if (s.ra_ == s.rc_) { p = 2.0 * xm * sr; q = 1.0 - sr; }
          else {
            const double qq = s.fa / s.fc, r = s.fb / s.fc;
            p = sr * (2.0 * xm * qq * (qq - r) - (s.rb_ - s.ra_) * (r - 1.0));
            q = (qq - 1.0) * (r - 1.0) * (sr - 1.0);
          }
          if (p > 0.0) q = -q;
          p = fabs(p);
          if (2.0 * p < fmin(3.0 * xm * q - fabs(tol1 * q), fabs(s.re * q))) { s.re = s.rd; s.rd = p / q; }
          else { s.rd = xm; s.re = s.rd; }
        } else { s.rd = xm; s.re = s.rd; }
        s.ra_ = s.rb_; s.fa = s.fb;
        if (fabs(s.rd) > tol1) s.rb_ = s.rb_ + s.rd;
        else s.rb_ = s.rb_ + copysign(tol1, xm);
        SWDK_REQ(s.rb_, PH_BRENT_GOT);
      }
      case PH_BRENT_GOT: {
        s.fb = s.last;
        s.phase = PH_BRENT_STEP;
        break;
      }
      case PH_REFINE_DONE: {  // getsol tail (surfdisp96.f:487-491)
        s.c1 = s.c3;
        if (s.c1 > (double)P.betmx || !(s.c1 == s.c1)) { s.phase = PH_GS_FAIL; break; }
        s.phase = PH_GS_OK;
        break;
      }
      case PH_GS_OK: {
        if (s.gpass == 0) {
          io.c[s.k - 1] = s.c1;
          if (P.igr > 0) {
            s.t1 = (double)s.t1b;
            s.ifirst = 0;
            s.clow = io.cb[s.k - 1] + ONE_DC * DC;
            s.c1 = s.c1 - ONEA * DC;
            s.gpass = 1;
            s.phase = PH_GS_START;
            break;
          }
          s.c1 = 0.0;
        } else {
          io.cb[s.k - 1] = s.c1;
        }
        s.phase = PH_PERIOD_OUT;
        break;
      }
      case PH_GS_FAIL: {
        if (s.gpass == 0) { s.phase = PH_FAIL; break; }
        s.c1 = io.c[s.k - 1];
        io.cb[s.k - 1] = s.c1;
        s.phase = PH_PERIOD_OUT;
        break;
      }
      case PH_PERIOD_OUT: {  // surfdisp96.f:307-319
        const double ck = io.c[s.k - 1];
        double v;
        if (P.sngl) {
          const float cc0 = (float)ck, cc1 = (float)s.c1;
          if (P.igr == 0) v = (double)cc0;
          else v = (double)((1.0f / s.t1a - 1.0f / s.t1b) / (1.0f / (s.t1a * cc0) - 1.0f / (s.t1b * cc1)));
        } else {
          if (P.igr == 0) v = ck;
          else {
            const double ta = s.t1a, tb = s.t1b;
            v = (1.0 / ta - 1.0 / tb) / (1.0 / (ta * ck) - 1.0 / (tb * s.c1));
          }
        }
        if (s.sub) { if (s.iq == nmode) s.sub_out = v; }
        else { out_at(io, s.iq, s.k) = v; st_at(io, s.iq, s.k) = ST_OK; }
        s.k = s.k + 1;
        s.phase = PH_PERIOD_START;
        break;
      }
      case PH_FAIL: {  // labels 1700/1750
        if (s.iq <= 1) s.ierr = 1;
        s.ift = s.k;
        if (s.sub) { if (s.iq == nmode) s.sub_out = 0.0; }
        else for (int i = s.k; i <= kmax; ++i) { out_at(io, s.iq, i) = 0.0; st_at(io, s.iq, i) = ST_NO_ROOT; }
        s.phase = PH_MODE_END;
        break;
      }
      case PH_MODE_END: {
        s.iq = s.iq + 1;
        s.k = 1;
        s.phase = (s.iq > nmode) ? PH_CHAIN_END : PH_PERIOD_START;
        break;
      }
      case PH_CHAIN_END: {
        if (s.sub) {  // a single-period retry finished (surfdisp.cpp:97-108)
          const double v = s.sub_out;
          const bool ok = (s.ierr == 0) && v != 0.0 && (v == v);
          out_at(io, s.rq_m, s.rq_k) = ok ? v : 0.0;
          st_at(io, s.rq_m, s.rq_k) = ok ? ST_RETRIED : ST_NO_ROOT;
          s.rq_k = s.rq_k + 1;
          s.phase = (P.retry == RETRY_ONE) ? PH_DONE : PH_RETRY_NEXT;
          break;
        }
        if (s.ierr == 0 || P.retry != RETRY_INLINE) { s.phase = PH_DONE; break; }
        s.rq_m = 1; s.rq_k = 1;
        s.phase = PH_RETRY_NEXT;
        break;
      }
      case PH_RETRY_NEXT: {
        s.sub = 0;
        bool found = false;
        while (s.rq_m <= P.nmode && !found) {
          while (s.rq_k <= P.kmax) {
            const double v = out_at(io, s.rq_m, s.rq_k);
            if (v == 0.0 || !(v == v)) { found = true; break; }
            s.rq_k++;
          }
          if (!found) { s.rq_m++; s.rq_k = 1; }
        }
        if (!found) { s.phase = PH_DONE; break; }
        s.sub = 1;
        s.phase = PH_CHAIN_START;
        break;
      }
      case PH_DONE:
      default:
        return false;
    }
  }
}
#undef SWDK_REQ

// phase of the evaluation a chain has just requested (s.next set)
SWDK_HD int eval_phase(const ChainState& s) {
  if (s.sub) return EV_RETRY;
  switch (s.next) {
    case PH_GS_FIRST:
    case PH_SCAN_GOT: return (s.k == 1 && s.gpass == 0) ? EV_SCAN_FIRST : EV_SCAN;
    case PH_PROP_HI:
    case PH_PROP_CHECK: return EV_CELL;
    case PH_FIRST_GOT: return EV_SCAN_FIRST;
    case PH_PROP_DOWN_GOT:
    case PH_PROP_C1_GOT: return EV_WALK;
    default: return EV_REFINE;
  }
}

// Runs a whole chain.  io.cb must have KMAX_CHAIN + 24 doubles (Neville x/y).
// On the device every lane of the warp must call this (active = false for
// lanes without a chain): a full-warp vote at the top of each iteration
// reconverges the warp so that the secular function -- nearly all of the
// work -- runs once for all lanes that need a value, instead of once per
// divergent group of lanes.
SWDK_HDI void run_chain(const LayerView& V, const ChainParams& P, const ChainIO& io, ChainState& s, bool active) {
  chain_init(s);
#ifdef __CUDA_ARCH__
  for (;;) {
    const bool need = active && chain_advance(s, P, io);
    if (!need) active = false;
    if (__ballot_sync(0xffffffffu, need) == 0u) break;
    if (need) {
      s.last = V.fast ? secular_fast(V, P.iwave, P.refine, s.omega / s.creq, s.omega)
                     : secular(V, P.iwave, s.omega / s.creq, s.omega);
      s.nevals++;
      s.phase = s.next;
    }
  }
#else
  if (!active) return;
  while (chain_advance(s, P, io)) {
    s.last = V.fast ? secular_fast(V, P.iwave, P.refine, s.omega / s.creq, s.omega)
                   : secular(V, P.iwave, s.omega / s.creq, s.omega);
    s.nevals++;
    s.phase = s.next;
  }
#endif
}

}  // namespace swdk
