// Test harness: the GPU's eigenfunction / energy-integral passes
// (jdsurfg_b200/csrc/swdk_eigen.cuh) compiled for the host, one
// (layer model, period, phase velocity) at a time, so tests can compare the
// raw layer kernels and group velocity with the oracle's sregn96 / slegn96
// on the CPU.  Built by tests/test_eigen_host.py.
#include <cmath>
#include <vector>

#include <vector_types.h>  // float2 / float4 of the CUDA headers (plain host structs)

#include "swdk_eigen.cuh"

using namespace swdk;

namespace {
// records each layer's raw kernels (before the pass's normaliser)
struct LayerSink {
  double *da, *db, *dr;
  void add(int l, double, double, double xa, double xb, double xr) const {
    da[l] = xa;
    db[l] = xb;
    dr[l] = xr;
  }
  void start() const {}
  void finish() const {}
};

// the node sums as a per-layer accumulation: kp[n] += w * (...) in layer
// order, the arithmetic NodeSink keeps in registers
struct TentSink {
  double* kp;
  const float2* crs;
  int L, nw;
  void start() const {}
  void finish() const {}
  void add(int l, double fa, double fr, double xa, double xb, double xr) const {
    if (nw > 0 && l == 0) return;
    const int lp = (nw > 0) ? l - 1 : l;
    const int n0 = (lp >> 2) + nw;
    const double xbf = xb * fa, xaf = xa * fa, xrf = xr * fr;
    const double t = (double)(2 * (lp & 3) + 1) / 8.0;
    const double w0 = (l == L - 1) ? 4.875 : 1.0 - t;
    kp[n0] += w0 * (xbf + xaf * (double)crs[n0].x + xrf * (double)crs[n0].y * (double)crs[n0].x);
    if (l != L - 1)
      kp[n0 + 1] += t * (xbf + xaf * (double)crs[n0 + 1].x + xrf * (double)crs[n0 + 1].y * (double)crs[n0 + 1].x);
  }
};
}  // namespace

// wave 1 Love, 2 Rayleigh.  The layer model (top-down, last = half-space)
// becomes the pass's model as the eigen kernel builds it: flat, or with the
// earth-flattening transform of bldsph (ar = 6371) when sphere != 0.
// Returns the flat group velocity, the normaliser and per-layer raw kernels;
// trunc_q is the pass's depth-truncation threshold (0: every layer).
extern "C" int eig_host_pass(int wave, int L, const float* thk, const float* vp, const float* vs, const float* rho,
                             int sphere, double t, double c, double trunc_q, double* ugr, double* norm, double* da,
                             double* db, double* dr) {
  if (L < 2 || L > LMAX) return -1;
  std::vector<double> drs(L), zd(L), za(L), zb(L), zr(L), vtp(L), rtp(L);
  double acc = 0.0;
  for (int i = 0; i < L; ++i) {
    acc = acc + ((i == L - 1) ? 1.0 : (double)thk[i]);
    drs[i] = acc;
  }
  const double ar = 6371.0;
  for (int i = 0; i < L; ++i) {
    if (sphere) {
      const double r0 = (i == 0) ? ar : ar - drs[i - 1];
      const double r1 = ar - drs[i];
      const double z0 = ar * std::log(ar / r0), z1 = ar * std::log(ar / r1);
      const double tmp = (2.0 * ar) / (r0 + r1);
      vtp[i] = tmp;
      const double t2 = tmp * tmp, t4 = t2 * t2, t5 = t4 * tmp;
      rtp[i] = (wave == 1) ? 1.0 / t5 : std::pow(tmp, (double)(-2.275f));
      za[i] = (double)vp[i] * tmp;
      zb[i] = (double)vs[i] * tmp;
      zr[i] = (double)rho[i] * rtp[i];
      zd[i] = (i == L - 1) ? 0.0 : z1 - z0;
    } else {
      vtp[i] = 1.0;
      rtp[i] = 1.0;
      za[i] = vp[i];
      zb[i] = vs[i];
      zr[i] = rho[i];
      zd[i] = thk[i];
    }
  }

  const double omega = 2.0 * PI_F / t, wvno = omega / c;
  LayerSink sink{da, db, dr};
  for (int i = 0; i < L; ++i) { da[i] = 0.0; db[i] = 0.0; dr[i] = 0.0; }
  if (wave == 1) {
    std::vector<LoveLayer> lay(L);
    for (int i = 0; i < L; ++i) make_love_layer(lay[i], zd[i], zb[i], zr[i], vtp[i], rtp[i]);
    LoveScratch scr;
    love_pass(lay.data(), L, omega, wvno, scr, *ugr, *norm, sink, trunc_q);
  } else {
    std::vector<RayLayer> lay(L);
    for (int i = 0; i < L; ++i) make_ray_layer(lay[i], zd[i], za[i], zb[i], zr[i], vtp[i], rtp[i]);
    RayScratch scr;
    rayleigh_pass(lay.data(), L, omega, wvno, scr, *ugr, *norm, sink, trunc_q);
  }
  return 0;
}

// The node sums of one pass through NodeSink (kp) and through TentSink
// (kref) on the same flat layer model; nw fluid nodes merged into layer 0,
// crs holds nz (dalpha/dbeta, drho/dalpha) pairs.
extern "C" int eig_host_nodesums(int wave, int L, const float* thk, const float* vp, const float* vs,
                                 const float* rho, int nw, int nz, const float* crs, double t, double c,
                                 double trunc_q, double* kp, double* kref) {
  if (L < 2 || L > LMAX || nz < 2) return -1;
  const double omega = 2.0 * PI_F / t, wvno = omega / c;
  std::vector<float2> cr(nz);
  for (int i = 0; i < nz; ++i) { cr[i].x = crs[2 * i]; cr[i].y = crs[2 * i + 1]; }
  for (int i = 0; i < nz; ++i) { kp[i] = 0.0; kref[i] = 0.0; }
  NodeSink ns{kp, cr.data(), L, nw, nz};
  TentSink ts{kref, cr.data(), L, nw};
  double ugr, norm;
  if (wave == 1) {
    std::vector<LoveLayer> lay(L);
    for (int i = 0; i < L; ++i) make_love_layer(lay[i], thk[i], vs[i], rho[i], 1.0, 1.0);
    LoveScratch scr;
    love_pass(lay.data(), L, omega, wvno, scr, ugr, norm, ns, trunc_q);
    love_pass(lay.data(), L, omega, wvno, scr, ugr, norm, ts, trunc_q);
  } else {
    std::vector<RayLayer> lay(L);
    for (int i = 0; i < L; ++i) make_ray_layer(lay[i], thk[i], vp[i], vs[i], rho[i], 1.0, 1.0);
    RayScratch scr;
    rayleigh_pass(lay.data(), L, omega, wvno, scr, ugr, norm, ns, trunc_q);
    rayleigh_pass(lay.data(), L, omega, wvno, scr, ugr, norm, ts, trunc_q);
  }
  return 0;
}
