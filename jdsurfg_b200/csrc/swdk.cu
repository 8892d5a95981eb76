// swdk.cu -- kernels and C-ABI of the B200 surface-wave engine (libswdk.so).
//
// Pipeline of one SurfTime::get_1d_kernel call (SurfaceWave.cpp:458-502):
//   k_prep   : one thread per column: Brocher vp/rho (empirical.cpp:9-18),
//              grid2LayerModel (SurfaceWave.cpp:113-155), surfdisp96's
//              sphere() flattening (surfdisp96.f:499-571) and start value
//              (surfdisp96.f:154-226); writes the REAL*4 layer model
//              half-space first and column by column, so each secular
//              evaluation streams its own column forward.
//   k_roots  : one thread per (column, root chain); a chain is one
//              surfdisp96 call (wave, period list, modes 1..M) with the
//              reference's retry (surfdisp.cpp:94-109); identical chains of
//              different slot types are computed once.
//   k_eigen  : one block per (column, wave-type group of output slots), one
//              thread per slot: sregn96 /
//              sregnpu / slegn96 / slegnpu passes, sphericity, _ParamConvert
//              and the empirical chain rule (SurfaceWave.cpp:491-500).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "swdk.h"
#include "swdk_core.cuh"
#include "swdk_eigen.cuh"

using namespace swdk;

namespace {

constexpr int FEAT_NODES = 64, FEAT_DIM = 320;  // proposal network input (see swdk_mlp.cu)
constexpr double FEAT_C0 = 3.5;                  // phase velocity offset of the network target

// statistics counters of a call (device array, copied to the host):
// [0] secular evaluations, [1]/[2] Rayleigh/Love layer-evaluations,
// [3]/[4] learned cells used / dropped, [5..10] evaluations by phase
// (EV_* below)
constexpr int NCOUNT = 11;
constexpr int EV_BASE = 5;

struct ColInfo {
  double cc;    // surfdisp96 start value cc (surfdisp96.f:222)
  float betmx;  // largest flattened shear velocity
  float pad_;
  int L;        // sublayers incl. half-space
  int llw;      // 2 if the top layer is fluid
  int nw;       // leading fluid grid nodes
  int valid;
};

struct ChainDesc {
  int t_off;    // first period in the period array
  int np;       // periods
  int nmode;    // modes 1..nmode
  int iwave;    // 1 Love, 2 Rayleigh
  int igr;      // surfdisp96 igr
  int out_off;  // root slot of (mode 1, period 0)
};

// output slots grouped by wave type (Rc, Rg, Lc, Lg order); the eigen
// kernel runs one block per (column, group), so a block's warps all do the
// same kind of pass and finish together
struct SlotGroups {
  int n;         // non-empty groups
  int start[4];  // first slot of group g in the plan's slot array
  int count[4];  // slots of group g
};

struct SlotDesc {
  int wtype;        // 0 Rc, 1 Rg, 2 Lc, 3 Lg
  int oslot;        // output slot (0..kmax-1)
  int r0, r1, r2;   // root slots of T, T(1+0.005), T(1-0.005)
  double t, t1, t2;
};

// ---------------------------------------------------------------------------
// exact-order arithmetic for the model preparation (matches the CPU order)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// correctly rounded x^5 for x exactly representable in float (x^2 is exact)
__device__ __forceinline__ double pow5_cr(double x) {
  const double x2 = dmul(x, x);
  const double hi = dmul(x2, x2);
  const double lo = fma(x2, x2, -hi);
  return fma(hi, x, dmul(lo, x));
}

// empirical_relation (empirical.cpp:9-18); std::pow(float,int) is evaluated
// in double and, for float arguments, the exact-then-rounded products below
// equal glibc's correctly rounded pow.
__device__ void brocher(float vsz, float& vpz, float& rhoz) {
  const double v = vsz, v2 = dmul(v, v), v3 = dmul(v2, v), v4 = dmul(v2, v2);
  vpz = (float)dsub(dadd(dsub(dadd(0.9409, dmul(2.0947, v)), dmul(0.8206, v2)), dmul(0.2683, v3)),
                    dmul(0.0251, v4));
  const double p = vpz, p2 = dmul(p, p), p3 = dmul(p2, p), p4 = dmul(p2, p2), p5 = pow5_cr(p);
  rhoz = (float)dadd(dsub(dadd(dsub(dmul(1.6612, p), dmul(0.4721, p2)), dmul(0.0671, p3)), dmul(0.0043, p4)),
                     dmul(0.000106, p5));
}

// empirical_deriv (empirical.cpp:26-34)
__device__ void brocher_deriv(float vp, float vs, float& drda, float& dadb) {
  const double p = vp, p2 = dmul(p, p), p3 = dmul(p2, p), p4 = dmul(p2, p2);
  drda = (float)dadd(dsub(dadd(dsub(1.6612, dmul(0.4721 * 2, p)), dmul(0.0671 * 3, p2)), dmul(0.0043 * 4, p3)),
                     dmul(0.000106 * 5, p4));
  const double s = vs, s2 = dmul(s, s), s3 = dmul(s2, s);
  dadb = (float)dsub(dadd(dsub(2.0947, dmul(0.8206 * 2, s)), dmul(0.2683 * 3, s2)), dmul(0.0251 * 4, s3));
}

// gtsolh (surfdisp96.f:377-398), REAL*4
__device__ float gtsolh(float a, float b) {
  float c = fmul(0.95f, b);
  for (int i = 0; i < 5; ++i) {
    const float gamma = fdiv(b, a);
    const float kappa = fdiv(c, b);
    const float k2 = fmul(kappa, kappa);
    const float gk = fmul(gamma, kappa);
    const float gk2 = fmul(gk, gk);
    const float fac1 = __fsqrt_rn(fsub(1.0f, gk2));
    const float fac2 = __fsqrt_rn(fsub(1.0f, k2));
    const float tk = fsub(2.0f, k2);
    const float fr = fsub(fmul(tk, tk), fmul(fmul(4.0f, fac1), fac2));
    float frp = fadd(fadd(-fmul(fmul(4.0f, fsub(2.0f, k2)), kappa),
                          fdiv(fmul(fmul(fmul(fmul(4.0f, fac2), gamma), gamma), kappa), fac1)),
                     fdiv(fmul(fmul(4.0f, fac1), kappa), fac2));
    frp = fdiv(frp, b);
    c = fsub(c, fdiv(fr, frp));
  }
  return c;
}

// surfdisp96 model set-up for one column: sphere() (ar = 6370) when
// sphere != 0, extremal velocities and the start value.  d/a/b/r are the
// layer arrays (top-down, length L) and are flattened in place; rhoR/rhoL
// receive the Rayleigh/Love density mappings.
__device__ void sd96_setup(int L, int sphere, float* d, float* a, float* b, const float* r, float* rhoR, float* rhoL,
                           ColInfo& ci) {
  if (sphere) {
    const double ar = 6370.0;
    double dr = 0.0, r0 = ar;
    d[L - 1] = 1.0f;
    for (int i = 0; i < L; ++i) {
      dr = dadd(dr, (double)d[i]);
      const double r1 = dsub(ar, dr);
      const double z0 = dmul(ar, log(ddiv(ar, r0)));
      const double z1 = dmul(ar, log(ddiv(ar, r1)));
      d[i] = (float)dsub(z1, z0);
      const double tmp = ddiv(dadd(ar, ar), dadd(r0, r1));
      a[i] = (float)dmul((double)a[i], tmp);
      b[i] = (float)dmul((double)b[i], tmp);
      const float btp = (float)tmp;
      rhoR[i] = fmul(r[i], (float)pow((double)btp, (double)(-2.275f)));
      const float b2 = fmul(btp, btp), b4 = fmul(b2, b2), b5 = fmul(b4, btp);
      rhoL[i] = fmul(r[i], fdiv(1.0f, b5));
      r0 = r1;
    }
    d[L - 1] = 0.0f;
  } else {
    for (int i = 0; i < L; ++i) { rhoR[i] = r[i]; rhoL[i] = r[i]; }
  }
  ci.llw = (b[0] <= 0.0f) ? 2 : 1;
  int jmn = 0, jsol = 1;
  float betmx = -1.e20f, betmn = 1.e20f;
  for (int i = 0; i < L; ++i) {
    if (b[i] > 0.01f && b[i] < betmn) { betmn = b[i]; jmn = i; jsol = 1; }
    else if (b[i] <= 0.01f && a[i] < betmn) { betmn = a[i]; jmn = i; jsol = 0; }
    if (b[i] > betmx) betmx = b[i];
  }
  float cc1 = (jsol == 0) ? betmn : gtsolh(a[jmn], b[jmn]);
  cc1 = fmul(0.95f, cc1);
  cc1 = fmul(0.90f, cc1);
  ci.cc = (double)cc1;
  ci.betmx = betmx;
}

__device__ __forceinline__ bool finitef(float x) { return isfinite(x); }

// REAL*4 layers (h, alpha, beta, rho), half-space first (layer_index), of the
// flattened model, one table per wave type (the density transform differs)
__device__ void write_layers(int L, int ncol, int col, int lstride, const float* th, const float* a, const float* b,
                             const float* rR, const float* rL, float4* layR, float4* layL) {
  for (int m = 0; m < L; ++m) {
    const size_t o = layer_index(L - 1 - m, ncol, col, lstride);
    layR[o] = make_float4(th[m], a[m], b[m], rR[m]);
    layL[o] = make_float4(th[m], a[m], b[m], rL[m]);
  }
}

// ---------------------------------------------------------------------------
// k_prep: node model -> layer models (one thread per column)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_prep(int ncol, int ldi, int nz, const float* __restrict__ vs_in,
                                              const float* __restrict__ vp_in, const float* __restrict__ rho_in,
                                              const float* __restrict__ depth, int sphere, int Lmax,
                                              float4* __restrict__ layR, float4* __restrict__ layL,
                                              float4* __restrict__ lay0,
                                              ColInfo* __restrict__ info, float2* __restrict__ chainrule,
                                              float4* __restrict__ nodefeat, float4* __restrict__ nodes) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  float v[NZMAX], vp[NZMAX], rho[NZMAX], dep[NZMAX];
  bool valid = true;
  for (int k = 0; k < nz; ++k) {
    v[k] = vs_in[col + (size_t)ldi * k];
    dep[k] = depth[k];
    if (vp_in) {
      vp[k] = vp_in[col + (size_t)ldi * k];
      rho[k] = rho_in[col + (size_t)ldi * k];
    } else {
      brocher(v[k], vp[k], rho[k]);
    }
    if (!finitef(v[k]) || !finitef(vp[k]) || !finitef(rho[k]) || v[k] < 0.0f || !(vp[k] > 0.0f) || !(rho[k] > 0.0f))
      valid = false;
  }
  int nw = 0;
  while (nw < nz - 1 && v[nw] == 0.0f) ++nw;
  for (int k = nw; k < nz; ++k)
    if (!(v[k] > 0.0f)) valid = false;
  if (nodefeat) {  // proposal-network input: 64 nodes x (vs, vp, rho, thickness), normalised
    for (int i = 0; i < FEAT_NODES; ++i) {
      const int k = i < nz ? i : nz - 1;
      const float thk = (i < nz - 1) ? dep[i + 1] - dep[i] : 0.0f;
      nodefeat[(size_t)col * FEAT_NODES + i] = make_float4(v[k] / 4.5f, vp[k] / 8.0f, rho[k] / 3.3f, thk / 5.0f);
    }
  }
  for (int k = 0; k < nz; ++k) {
    float drda = 0.0f, dadb = 0.0f;
    brocher_deriv(vp[k], v[k], drda, dadb);
    chainrule[(size_t)k * ncol + col] = make_float2(dadb, drda);
  }
  // grid2LayerModel (SurfaceWave.cpp:113-155), fluid nodes merged into one layer
  float th[LMAX], a[LMAX], b[LMAX], r[LMAX], rR[LMAX], rL[LMAX];
  const int n = 4;
  int L, istart, k = 0;
  if (nw > 0) {
    L = (nz - nw) + (nz - nw - 1) * 3 + 1;
    istart = nw;
    th[0] = fsub(dep[nw], dep[0]);
    r[0] = rho[0];
    b[0] = 0.0f;
    a[0] = vp[0];
    k = 1;
  } else {
    L = nz + (nz - 1) * 3;
    istart = 0;
  }
  for (int i = istart; i < nz - 1; ++i) {
    const float thk = fdiv(fsub(dep[i + 1], dep[i]), (float)n);
    const float dvp = fsub(vp[i + 1], vp[i]), dvs = fsub(v[i + 1], v[i]), drh = fsub(rho[i + 1], rho[i]);
    for (int j = 0; j < n; ++j) {
      const float w = (float)(2 * j + 1);
      th[k] = thk;
      a[k] = (float)dadd((double)vp[i], ddiv((double)fmul(w, dvp), 2.0 * n));
      b[k] = (float)dadd((double)v[i], ddiv((double)fmul(w, dvs), 2.0 * n));
      r[k] = (float)dadd((double)rho[i], ddiv((double)fmul(w, drh), 2.0 * n));
      ++k;
    }
  }
  th[L - 1] = 0.0f;
  a[L - 1] = vp[nz - 1];
  b[L - 1] = v[nz - 1];
  r[L - 1] = rho[nz - 1];
  for (int m = 0; m < L; ++m) lay0[(size_t)col * Lmax + m] = make_float4(th[m], a[m], b[m], r[m]);
  // the grid nodes, from which the root search rebuilds the flattened
  // sublayers of columns without fluid nodes (LayerView::layer)
  if (nodes)
    for (int k2 = 0; k2 < nz; ++k2) nodes[(size_t)col * nz + k2] = make_float4(vp[k2], v[k2], rho[k2], 0.0f);
  ColInfo ci;
  ci.L = L;
  ci.nw = nw;
  ci.valid = valid ? 1 : 0;
  sd96_setup(L, sphere, th, a, b, r, rR, rL, ci);
  write_layers(L, ncol, col, Lmax, th, a, b, rR, rL, layR, layL);
  info[col] = ci;
}

// k_prep_layers: layered models (surfdisp96_ input) -> layer models
__global__ void k_prep_layers(int nmodel, int nlayer, const float* __restrict__ thk, const float* __restrict__ vp,
                              const float* __restrict__ vs, const float* __restrict__ rho, int sphere,
                              float4* __restrict__ layR, float4* __restrict__ layL, ColInfo* __restrict__ info) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= nmodel) return;
  float th[LMAX], a[LMAX], b[LMAX], r[LMAX], rR[LMAX], rL[LMAX];
  bool valid = true;
  for (int m = 0; m < nlayer; ++m) {
    const size_t o = (size_t)col * nlayer + m;
    th[m] = thk[o]; a[m] = vp[o]; b[m] = vs[o]; r[m] = rho[o];
    if (!finitef(th[m]) || !finitef(a[m]) || !finitef(b[m]) || !finitef(r[m])) valid = false;
  }
  ColInfo ci;
  ci.L = nlayer;
  ci.nw = (b[0] <= 0.0f) ? 1 : 0;
  ci.valid = valid ? 1 : 0;
  sd96_setup(nlayer, sphere, th, a, b, r, rR, rL, ci);
  write_layers(nlayer, nmodel, col, nlayer, th, a, b, rR, rL, layR, layL);
  info[col] = ci;
}

// The flattening of the standard sublayer grid (no fluid nodes) of a depth
// vector: thicknesses as grid2LayerModel makes them (4 per node interval,
// SurfaceWave.cpp:113-155), then sphere()'s loop (surfdisp96.f:499-571,
// ar = 6370) in the same arithmetic as sd96_setup; one thread.
__global__ void k_depth_table(int nz, const float* __restrict__ depth, int sphere, DepthLayer* __restrict__ dl) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const int L = 4 * nz - 3;
  const double ar = 6370.0;
  double dr = 0.0, r0 = ar;
  for (int m = 0; m < L; ++m) {
    float th;
    if (m == L - 1) th = sphere ? 1.0f : 0.0f;  // sphere(): the half-space counts 1 km in the depth sum
    else {
      const int i = m >> 2;
      th = fdiv(fsub(depth[i + 1], depth[i]), 4.0f);
    }
    DepthLayer q;
    q.pad_ = 0.0f;
    if (sphere) {
      dr = dadd(dr, (double)th);
      const double r1 = dsub(ar, dr);
      const double z0 = dmul(ar, log(ddiv(ar, r0)));
      const double z1 = dmul(ar, log(ddiv(ar, r1)));
      q.d = (m == L - 1) ? 0.0f : (float)dsub(z1, z0);
      q.tmp = ddiv(dadd(ar, ar), dadd(r0, r1));
      const float btp = (float)q.tmp;
      q.fR = (float)pow((double)btp, (double)(-2.275f));
      const float b2 = fmul(btp, btp), b4 = fmul(b2, b2), b5 = fmul(b4, btp);
      q.fL = fdiv(1.0f, b5);
      r0 = r1;
    } else {
      q.d = th;
      q.tmp = 1.0;
      q.fR = 1.0f;
      q.fL = 1.0f;
    }
    dl[m] = q;
  }
}

// ---------------------------------------------------------------------------
// proposal-network rows: row = slot * ncol + col; a half-warp per row:
// lane h < 8 loads nodes 8h .. 8h+7 once and writes their four components
// (four 16-byte chunks of 8 columns), lanes 8 .. 15 write the period
// features and the zero padding
//   x[0:64) vs, [64:128) vp, [128:192) rho, [192:256) thickness,
//   x[256] log(T)/log(100), x[257] (mode-1)/2, zero to 320
// tiled = 0: row-major (n, 320); tiled = 1: the 128-row tile images
// swdk_mlp_propose reads (128-byte swizzled K-major, 81920 bytes per tile)
// ---------------------------------------------------------------------------
static_assert(FEAT_NODES == 64 && FEAT_DIM == 320, "k_features packs 64 nodes x 4 components + 64 columns");
__device__ __forceinline__ void feat_store(__nv_bfloat16* x, int tiled, int w, int c0, const float* v, bool inr) {
  uint32_t pk[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const __nv_bfloat162 b2 = __floats2bfloat162_rn(inr ? v[2 * e] : 0.0f, inr ? v[2 * e + 1] : 0.0f);
    pk[e] = *reinterpret_cast<const uint32_t*>(&b2);
  }
  uint8_t* dst;
  if (tiled) {
    const int t = w >> 7, r = w & 127, kb = c0 >> 6, j = (c0 & 63) >> 3;
    dst = reinterpret_cast<uint8_t*>(x) + (size_t)t * (128 * FEAT_DIM * 2) + kb * (128 * 128) + r * 128 +
          ((j ^ (r & 7)) << 4);
  } else {
    dst = reinterpret_cast<uint8_t*>(x + (size_t)w * FEAT_DIM + c0);
  }
  *reinterpret_cast<uint4*>(dst) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
}

__global__ void k_features(int64_t row0, int nrows, int ncol, int64_t rowmax, const float4* __restrict__ slotfeat,
                           const float4* __restrict__ nodefeat, const int64_t* __restrict__ rowlist,
                           __nv_bfloat16* __restrict__ x, int tiled) {
  const int w = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 4), h = threadIdx.x & 15;
  if (w >= nrows) return;
  const int64_t row = rowlist ? rowlist[w] : row0 + w;
  const bool inr = row >= 0 && row < rowmax;
  const int s = inr ? (int)(row / ncol) : 0, col = inr ? (int)(row % ncol) : 0;
  float v[8];
  if (h < 8) {
    const float4* nf = nodefeat + (size_t)col * FEAT_NODES + 8 * h;
    float4 n[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) n[e] = nf[e];
#pragma unroll
    for (int e = 0; e < 8; ++e) v[e] = n[e].x;
    feat_store(x, tiled, w, 8 * h, v, inr);
#pragma unroll
    for (int e = 0; e < 8; ++e) v[e] = n[e].y;
    feat_store(x, tiled, w, FEAT_NODES + 8 * h, v, inr);
#pragma unroll
    for (int e = 0; e < 8; ++e) v[e] = n[e].z;
    feat_store(x, tiled, w, 2 * FEAT_NODES + 8 * h, v, inr);
#pragma unroll
    for (int e = 0; e < 8; ++e) v[e] = n[e].w;
    feat_store(x, tiled, w, 3 * FEAT_NODES + 8 * h, v, inr);
  } else {
    const float4 sf = slotfeat[s];
    const int c0 = 4 * FEAT_NODES + 8 * (h - 8);
#pragma unroll
    for (int e = 0; e < 8; ++e) v[e] = (c0 + e == 256) ? sf.x : (c0 + e == 257) ? sf.y : 0.0f;
    feat_store(x, tiled, w, c0, v, inr);
  }
}

// swdk_set_proposal_shift: every proposed phase velocity (rows with a
// bracket, half-width > 0) moved by shift km/s
__global__ void k_shift_prop(int n, float2* __restrict__ prop, float shift) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && prop[i].y > 0.0f) prop[i].x += shift;
}

// training targets of chosen rows: y = c_flat - FEAT_C0
__global__ void k_targets(int n, int64_t rowmax, const int64_t* __restrict__ rows, const double* __restrict__ croot,
                          float* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t r = rows[i];
  y[i] = (r >= 0 && r < rowmax) ? (float)(croot[r] - FEAT_C0) : 0.0f;
}

// ---------------------------------------------------------------------------
// k_roots: one thread per (column, chain)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void roots_body(const ChainDesc cd, int ncol, const double* __restrict__ periods,
                                           const float4* __restrict__ layR, const float4* __restrict__ layL,
                                           const ColInfo* __restrict__ info, int refine, double rtol, int sngl,
                                           int retry, double* __restrict__ croot, int32_t* __restrict__ cstat,
                                           int32_t* __restrict__ ierr_out, unsigned long long* __restrict__ nevals) {
  // nevals[0]: evaluations, nevals[1]: Rayleigh layer-evaluations,
  // nevals[2]: Love layer-evaluations
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long my_evals = 0;
  // every lane runs run_chain (its warp vote needs the full warp); lanes
  // past the last column or with an invalid model take part inactive
  const bool inrange = col < ncol;
  const int ccol = inrange ? col : 0;
  const ColInfo ci = info[ccol];
  const bool active = inrange && ci.valid;
  double* outp = croot + (size_t)cd.out_off * ncol + ccol;
  int32_t* stp = cstat + (size_t)cd.out_off * ncol + ccol;
  if (inrange && !ci.valid) {
    for (int i = 0; i < cd.nmode * cd.np; ++i) { outp[(size_t)i * ncol] = 0.0; stp[(size_t)i * ncol] = ST_NAN_INPUT; }
    if (ierr_out) ierr_out[col] = 1;
  }
  LayerView V;
  V.lay = (cd.iwave == 2) ? layR : layL;
  V.fast = 0;  // dltar1/dltar4 as the reference writes them
  V.ncol = ncol;
  V.col = ccol;
  V.lstride = ci.L;  // tables of k_prep_layers: nlayer slots per model
  V.nodes = nullptr;
  V.dl = nullptr;
  V.wave = cd.iwave;
  V.L = ci.L;
  V.llw = ci.llw;
  ChainParams P;
  P.t = periods + cd.t_off;
  P.kmax = cd.np;
  P.nmode = cd.nmode;
  P.igr = cd.igr;
  P.iwave = cd.iwave;
  P.refine = refine;
  P.rtol = rtol;
  P.sngl = sngl;
  P.cc = ci.cc;
  P.betmx = ci.betmx;
  P.retry = retry;
  double cbuf[KMAX_CHAIN];
  double cbbuf[KMAX_CHAIN + 24];
  ChainIO io;
  io.c = cbuf;
  io.cb = cbbuf;
  io.out = outp;
  io.st = stp;
  io.stride = cd.np * ncol;
  io.ostride = ncol;
  io.prop = nullptr;
  ChainState s;
  run_chain(V, P, io, s, active);
  if (active) {
    if (s.iterlim)
      for (int i = 0; i < cd.nmode * cd.np; ++i)
        if (stp[(size_t)i * ncol] == ST_OK) stp[(size_t)i * ncol] = ST_ITER_LIMIT;
    if (ierr_out) ierr_out[col] = s.ierr;
    my_evals = (unsigned long long)s.nevals;
  }
  // layers per evaluation: the half-space, L-2-(llw-1)+1 propagated layers
  // and the fluid top when llw = 2 -- i.e. L for every evaluation
  unsigned long long my_layers = my_evals * (unsigned long long)(active ? ci.L : 0);
  for (int o = 16; o > 0; o >>= 1) {
    my_evals += __shfl_down_sync(0xffffffffu, my_evals, o);
    my_layers += __shfl_down_sync(0xffffffffu, my_layers, o);
  }
  if ((threadIdx.x & 31) == 0 && my_evals && nevals) {
    atomicAdd(nevals, my_evals);
    atomicAdd(nevals + (cd.iwave == 2 ? 1 : 2), my_layers);
  }
}

// one thread per (column, chain); chain = blockIdx.y
__global__ void __launch_bounds__(128) k_roots(int ncol, const ChainDesc* __restrict__ chains,
                                               const double* __restrict__ periods, const float4* __restrict__ layR,
                                               const float4* __restrict__ layL, const ColInfo* __restrict__ info,
                                               int refine, double rtol, int sngl, int retry, double* __restrict__ croot,
                                               int32_t* __restrict__ cstat, int32_t* __restrict__ ierr_out,
                                               unsigned long long* __restrict__ nevals) {
  roots_body(chains[blockIdx.y], ncol, periods, layR, layL, info, refine, rtol, sngl, retry,
             croot, cstat, ierr_out, nevals);
}

// the same for one chain passed by value
__global__ void __launch_bounds__(128) k_roots_one(ChainDesc cd, int ncol, const double* __restrict__ periods,
                                                   const float4* __restrict__ layR, const float4* __restrict__ layL,
                                                   const ColInfo* __restrict__ info, int refine, double rtol, int sngl,
                                                   double* __restrict__ croot, int32_t* __restrict__ cstat,
                                                   int32_t* __restrict__ ierr_out) {
  roots_body(cd, ncol, periods, layR, layL, info, refine, rtol, sngl, 0, croot, cstat,
             ierr_out, nullptr);
}

// ---------------------------------------------------------------------------
// Ragged batches: many models (own grids, depth vectors, period tables) in
// one launch of each kernel.  The work items of the root search are (model,
// chain, column); a block of items is one (model, chain) with the model's
// ncol columns, blocks ordered Rayleigh chains first.  Each model's arrays
// live at offsets in shared buffers.
// ---------------------------------------------------------------------------
struct RModel {
  int ncol, nz, Lmax, pad_;
  long long col0;   // first column of the model in per-column arrays (ColInfo, node features)
  long long lay0;   // float4 offset of its layer tables (layR / layL / lay0, Lmax*ncol each)
  long long crs0;   // float2 offset of its chain-rule factors (nz*ncol)
  long long root0;  // offset of its root slots in croot / cstat / prop (nroot*ncol)
  long long node0;  // float4 offset of its grid nodes (nz*ncol)
  long long dl0;    // offset of its depth table (Lmax DepthLayer)
  double *vc, *vout, *kernel;
  int32_t* status;
};

struct RBlock {
  long long item0;  // first work item of the block
  int model, chain;  // chain: index into the batch's combined chain array
};

// eigen launch of one wave type over a ragged batch: blocks [blk0, blk0+ncol)
// are model `model`'s columns, its slots of this wave type at [g0, g0+gn)
struct REBlock {
  long long blk0;
  int model, g0, gn, pad_;
};

struct RaggedMap {
  const RBlock* blocks;  // null: one model, items = order[item / ncol] x columns
  const RModel* models;
  int nblocks;
  int lstride;           // one model: layer slots per column of its tables (Lmax)
};

template <class T>
__device__ __forceinline__ int ragged_find(const T* tab, int n, long long key, long long T::*field) {
  int lo = 0, hi = n - 1;  // last entry with tab[i].*field <= key
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tab[mid].*field <= key) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Persistent root kernel: lanes take (chain, column) items from a queue
// (chains in `order`, Rayleigh first, columns consecutive) whenever their
// current chain is finished, so lanes stay busy while long chains run.
// queue[0] is the next item; the launch covers the GPU once.
// Dynamic shared memory of k_roots_queue and k_retry (128 threads): 55 KB,
// above the 48 KB a launch gets without opting in; four blocks fit an SM's
// 228 KB.
constexpr size_t ROOTS_SMEM = 128 * (sizeof(ChainState) + sizeof(ChainParams) + sizeof(ChainIO));

#ifndef SWDK_ROOTS_MINB
#define SWDK_ROOTS_MINB 4  // 127 registers, no spill (shared memory allows 4 blocks too); 3 blocks measured slower
#endif
#ifndef SWDK_RETRY_MINB
#define SWDK_RETRY_MINB 3  // retries, one record per warp: 168 registers (48 B of spill loads); 2 blocks (202 registers) measured 8 ms per step slower, 4 (128 registers, more spill) the same as 3
#endif
#ifndef SWDK_EIGEN_MINB
#define SWDK_EIGEN_MINB 3  // Rayleigh passes: 168 registers, no spill (2: 183, 3: 171, 4: 180, 5: 227 ms of eigen per step)
#endif
#ifndef SWDK_EIGEN_MINB_LOVE
#define SWDK_EIGEN_MINB_LOVE 5  // Love passes
#endif
__global__ void __launch_bounds__(128, SWDK_ROOTS_MINB) k_roots_queue(int ncol, int nitems, const int* __restrict__ order,
                                                     const ChainDesc* __restrict__ chains,
                                                     const double* __restrict__ periods,
                                                     const float4* __restrict__ layR, const float4* __restrict__ layL,
                                                     const ColInfo* __restrict__ info, int refine, double rtol,
                                                     int sngl, int retry, double* __restrict__ croot,
                                                     int32_t* __restrict__ cstat, unsigned int* __restrict__ queue,
                                                     const float2* __restrict__ prop,
                                                     int2* __restrict__ retry_list, unsigned int* __restrict__ retry_count,
                                                     unsigned int retry_cap,
                                                     unsigned long long* __restrict__ nevals, RaggedMap rg,
                                                     const float4* __restrict__ nodes,
                                                     const DepthLayer* __restrict__ dl) {
  double cbuf[KMAX_CHAIN];
  double cbbuf[KMAX_CHAIN + 24];
  // dynamic shared memory (ROOTS_SMEM): the chain states, and the chains'
  // parameters and output addressing, which the state machine reads between
  // evaluations instead of holding them in registers across them
  extern __shared__ __align__(16) unsigned char roots_smem[];
  ChainState* sst = reinterpret_cast<ChainState*>(roots_smem);
  ChainParams* sprm = reinterpret_cast<ChainParams*>(sst + 128);
  ChainIO* sio = reinterpret_cast<ChainIO*>(sprm + 128);
  __shared__ unsigned long long phase_ev[NPHASE_EV];
  // evaluations, Rayleigh and Love layer evaluations, proposals used and
  // refused: block totals, added at each chain's end (no registers held)
  __shared__ unsigned long long blk_ev[5];
  if (threadIdx.x < NPHASE_EV) phase_ev[threadIdx.x] = 0ull;
  if (threadIdx.x < 5) blk_ev[threadIdx.x] = 0ull;
  __syncthreads();
  ChainState& s = sst[threadIdx.x];
  ChainParams& P = sprm[threadIdx.x];
  ChainIO& io = sio[threadIdx.x];
  LayerView V;
  int col = 0, item_of = 0;
  bool have = false, exhausted = false;
  io.c = cbuf;
  io.cb = cbbuf;
  for (;;) {
    bool need = false;
    for (;;) {
      if (!have) {
        if (exhausted) break;
        const unsigned int item = atomicAdd(queue, 1u);
        if (item >= (unsigned int)nitems) { exhausted = true; break; }
        item_of = (int)item;
        // the item's model (a ragged batch) or the single model's arrays
        int mcol = ncol, lstride = rg.lstride;
        ChainDesc cd;
        long long o_col = 0, o_lay = 0, o_root = 0, o_node = 0, o_dl = 0;
        if (rg.blocks) {
          const RBlock B = rg.blocks[ragged_find(rg.blocks, rg.nblocks, (long long)item, &RBlock::item0)];
          const RModel& M = rg.models[B.model];
          cd = chains[B.chain];
          col = (int)((long long)item - B.item0);
          mcol = M.ncol;
          lstride = M.Lmax;
          o_col = M.col0; o_lay = M.lay0; o_root = M.root0; o_node = M.node0; o_dl = M.dl0;
        } else {
          cd = chains[order[item / ncol]];
          col = item % ncol;
        }
        const ColInfo ci = info[o_col + col];
        double* outp = croot + o_root + (size_t)cd.out_off * mcol + col;
        int32_t* stp = cstat + o_root + (size_t)cd.out_off * mcol + col;
        if (!ci.valid) {
          for (int i = 0; i < cd.nmode * cd.np; ++i) { outp[(size_t)i * mcol] = 0.0; stp[(size_t)i * mcol] = ST_NAN_INPUT; }
          continue;
        }
        V.lay = ((cd.iwave == 2) ? layR : layL) + o_lay;
        V.fast = 1;
        V.ncol = mcol;
        V.col = col;
        V.lstride = lstride;
        V.L = ci.L;
        V.llw = ci.llw;
        V.nodes = (nodes && ci.nw == 0) ? nodes + o_node + (size_t)col * ((lstride + 3) / 4) : nullptr;
        V.dl = dl + o_dl;
        V.wave = cd.iwave;
        P.t = periods + cd.t_off;
        P.kmax = cd.np;
        P.nmode = cd.nmode;
        P.igr = cd.igr;
        P.iwave = cd.iwave;
        P.refine = refine;
        P.rtol = rtol;
        P.sngl = sngl;
        P.cc = ci.cc;
        P.betmx = ci.betmx;
        P.retry = retry;
        io.out = outp;
        io.st = stp;
        io.stride = cd.np * mcol;
        io.ostride = mcol;
        io.prop = prop ? prop + o_root + (size_t)cd.out_off * mcol + col : nullptr;
        chain_init(s);
        have = true;
      }
      need = chain_advance(s, P, io);
      if (need) break;
      // chain finished
      if (s.iterlim)
        for (int i = 0; i < P.nmode * P.kmax; ++i)
          if (io.st[(size_t)i * io.ostride] == ST_OK) io.st[(size_t)i * io.ostride] = ST_ITER_LIMIT;
      if (retry == RETRY_DEFERRED && s.ierr != 0) {
        // failed slots become single-period work items for k_retry
        for (int m = 1; m <= P.nmode; ++m)
          for (int k = 1; k <= P.kmax; ++k) {
            const double v = out_at(io, m, k);
            if (v == 0.0 || !(v == v)) {
              const unsigned int r = atomicAdd(retry_count, 1u);
              if (r < retry_cap) retry_list[r] = make_int2(item_of, (m << 16) | k);
            }
          }
      }
      atomicAdd(&blk_ev[0], (unsigned long long)s.nevals);
      atomicAdd(&blk_ev[P.iwave == 2 ? 1 : 2], (unsigned long long)s.nevals * V.L);
      if (s.nprop_ok) atomicAdd(&blk_ev[3], (unsigned long long)s.nprop_ok);
      if (s.nprop_fail) atomicAdd(&blk_ev[4], (unsigned long long)s.nprop_fail);
      have = false;
    }
    if (__ballot_sync(0xffffffffu, need) == 0u) break;
    if (need) {
      atomicAdd(&phase_ev[eval_phase(s)], 1ull);
      s.last = secular_fast(V, P.iwave, P.refine, s.omega / s.creq, s.omega);
      s.nevals++;
      s.phase = s.next;
    }
  }
  __syncthreads();
  if (threadIdx.x < NPHASE_EV && nevals && phase_ev[threadIdx.x])
    atomicAdd(nevals + EV_BASE + threadIdx.x, phase_ev[threadIdx.x]);
  if (threadIdx.x < 5 && nevals && blk_ev[threadIdx.x]) atomicAdd(nevals + threadIdx.x, blk_ev[threadIdx.x]);
}

// One round of the getsol scan (surfdisp96.f:452-486) by a whole warp.  The
// chain machine has just asked for f at the next scan point c2 = s.creq (the
// point counted in s.nscan).  Lane j evaluates the point j steps further on,
// accumulated step by step exactly as the scan does; lanes past a point the
// scan would not evaluate (below clow going down, beyond the scan cap) stay
// idle.  The first point, in scan order, with a sign change from its
// predecessor or failing the range test ends the round: the state becomes the
// one the sequential scan reaches there (refinement bracket or failure), so
// the root is the sequential scan's.  Without such a point the scan goes on
// from the last evaluated point.  Every lane holds the same state and leaves
// with the same state.  Returns the evaluations the sequential scan makes.
__device__ int retry_scan(ChainState& s, const ChainParams& P, const LayerView& V, int lane) {
  const unsigned FULL = 0xffffffffu;
  const double step = s.idir > 0 ? DC : -DC;
  double p = s.creq;
  for (int i = 0; i < lane; ++i) p = p + step;
  const bool valid = lane == 0 || ((s.idir > 0 || p > s.clow) && s.nscan + lane <= SCAN_CAP);
  const double f = valid ? secular_fast(V, P.iwave, P.refine, s.omega / p, s.omega) : 0.0;
  double fprev = __shfl_up_sync(FULL, f, 1);
  if (lane == 0) fprev = s.del1;
  const bool sc = valid && dsign1(fprev) != dsign1(f);
  const bool fail = valid && !sc && (p < s.cm || p >= ((double)P.betmx + DC) || !(p == p));
  const unsigned ev = __ballot_sync(FULL, sc || fail);
  const int nvalid = __popc(__ballot_sync(FULL, valid));  // the valid lanes are a prefix
  const int e = ev ? __ffs(ev) - 1 : nvalid - 1;          // the point the round ends at
  const double pe = __shfl_sync(FULL, p, e), fe = __shfl_sync(FULL, f, e);
  const double pb = __shfl_sync(FULL, p, e > 0 ? e - 1 : 0), fb = __shfl_sync(FULL, f, e > 0 ? e - 1 : 0);
  const bool sce = __shfl_sync(FULL, sc ? 1 : 0, e) != 0;
  s.nscan += e;
  s.last = fe;
  if (ev && sce) {  // sign change between the previous point and pe: refine
    if (e > 0) { s.c1 = pb; s.del1 = fb; }
    s.c2 = pe;
    s.del2 = fe;
    s.phase = PH_REFINE_START;
  } else {  // the scan moved on to pe: failed there, or continues from it
    s.c1 = pe; s.del1 = fe;
    s.c2 = pe; s.del2 = fe;
    s.phase = ev ? PH_GS_FAIL : PH_SCAN;
  }
  return e + 1;
}

// k_retry: the deferred single-period retries (surfdisp.cpp:94-109), one
// record per warp.  A retry re-runs the reference's search for one period
// from its start value, a scan of often several hundred dc steps; the warp's
// lanes hold the same chain state and take the scan 32 points at a time
// (retry_scan), the other requests (start point, refinement) are evaluated
// by all lanes alike.
__global__ void __launch_bounds__(128, SWDK_RETRY_MINB) k_retry(int ncol, const int* __restrict__ order,
                                                               const ChainDesc* __restrict__ chains,
                                                               const double* __restrict__ periods,
                                                               const float4* __restrict__ layR,
                                                               const float4* __restrict__ layL,
                                                               const ColInfo* __restrict__ info, int refine,
                                                               double rtol, int sngl, double* __restrict__ croot,
                                                               int32_t* __restrict__ cstat,
                                                               const int2* __restrict__ retry_list,
                                                               const unsigned int* __restrict__ retry_count,
                                                               unsigned int retry_cap, unsigned int* __restrict__ queue,
                                                               unsigned long long* __restrict__ nevals, RaggedMap rg,
                                                               const float4* __restrict__ nodes,
                                                               const DepthLayer* __restrict__ dl) {
  // dynamic shared memory (ROOTS_SMEM): one copy of the warp's chain state,
  // parameters and output addressing per lane
  extern __shared__ __align__(16) unsigned char roots_smem[];
  ChainState* sst = reinterpret_cast<ChainState*>(roots_smem);
  ChainParams* sprm = reinterpret_cast<ChainParams*>(sst + 128);
  ChainIO* sio = reinterpret_cast<ChainIO*>(sprm + 128);
  __shared__ unsigned long long blk_ev[3];  // evaluations, Rayleigh and Love layer evaluations
  if (threadIdx.x < 3) blk_ev[threadIdx.x] = 0ull;
  __syncthreads();
  double cbuf[KMAX_CHAIN];
  double cbbuf[KMAX_CHAIN + 24];
  const unsigned int n = min(*retry_count, retry_cap);
  const int lane = threadIdx.x & 31;
  for (;;) {
    unsigned int r = 0;
    if (lane == 0) r = atomicAdd(queue, 1u);
    r = __shfl_sync(0xffffffffu, r, 0);
    if (r >= n) break;
    ChainState& s = sst[threadIdx.x];
    ChainParams& P = sprm[threadIdx.x];
    ChainIO& io = sio[threadIdx.x];
    LayerView V;
    const int2 rec = retry_list[r];
    const int m = rec.y >> 16, k = rec.y & 0xffff;
    int mcol = ncol, col, lstride = rg.lstride;
    long long o_col = 0, o_lay = 0, o_root = 0, o_node = 0, o_dl = 0;
    ChainDesc cd;
    if (rg.blocks) {
      const RBlock B = rg.blocks[ragged_find(rg.blocks, rg.nblocks, (long long)rec.x, &RBlock::item0)];
      const RModel& M = rg.models[B.model];
      cd = chains[B.chain];
      col = (int)((long long)rec.x - B.item0);
      mcol = M.ncol;
      lstride = M.Lmax;
      o_col = M.col0; o_lay = M.lay0; o_root = M.root0; o_node = M.node0; o_dl = M.dl0;
    } else {
      cd = chains[order[rec.x / ncol]];
      col = rec.x % ncol;
    }
    const ColInfo ci = info[o_col + col];
    V.lay = ((cd.iwave == 2) ? layR : layL) + o_lay;
    V.fast = 1;
    V.ncol = mcol;
    V.col = col;
    V.lstride = lstride;
    V.L = ci.L;
    V.llw = ci.llw;
    V.nodes = (nodes && ci.nw == 0) ? nodes + o_node + (size_t)col * ((lstride + 3) / 4) : nullptr;
    V.dl = dl + o_dl;
    V.wave = cd.iwave;
    P.t = periods + cd.t_off;
    P.kmax = cd.np;
    P.nmode = cd.nmode;
    P.igr = cd.igr;
    P.iwave = cd.iwave;
    P.refine = refine;
    P.rtol = rtol;
    P.sngl = sngl;
    P.cc = ci.cc;
    P.betmx = ci.betmx;
    P.retry = RETRY_ONE;
    io.c = cbuf;
    io.cb = cbbuf;
    io.out = croot + o_root + (size_t)cd.out_off * mcol + col;
    io.st = cstat + o_root + (size_t)cd.out_off * mcol + col;
    io.stride = cd.np * mcol;
    io.ostride = mcol;
    io.prop = nullptr;
    chain_init_retry(s, m, k);
    unsigned long long nev = 0;
    while (chain_advance(s, P, io)) {  // the same decision in every lane
      if (s.next == PH_SCAN_GOT) {
        nev += retry_scan(s, P, V, lane);
        continue;
      }
      s.last = secular_fast(V, P.iwave, P.refine, s.omega / s.creq, s.omega);
      nev++;
      s.phase = s.next;
    }
    __syncwarp();
    if (lane == 0) {
      if (s.iterlim && st_at(io, m, k) != ST_NO_ROOT) st_at(io, m, k) = ST_ITER_LIMIT;
      atomicAdd(&blk_ev[0], nev);
      atomicAdd(&blk_ev[P.iwave == 2 ? 1 : 2], nev * V.L);
    }
  }
  __syncthreads();
  if (threadIdx.x < 3 && nevals && blk_ev[threadIdx.x]) atomicAdd(nevals + threadIdx.x, blk_ev[threadIdx.x]);
  if (threadIdx.x == 0 && nevals && blk_ev[0]) atomicAdd(nevals + EV_BASE + EV_RETRY, blk_ev[0]);
}

// Opts k_roots_queue and k_retry in to ROOTS_SMEM on the current device and
// returns k_roots_queue's resident blocks per SM.
cudaError_t roots_occupancy(int* per) {
  cudaError_t e = cudaFuncSetAttribute(k_roots_queue, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ROOTS_SMEM);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_retry, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ROOTS_SMEM);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per, k_roots_queue, 128, ROOTS_SMEM);
  return e;
}


// recip() on an array (its accuracy test)
__global__ void k_recip(int n, const double* __restrict__ x, double* __restrict__ r) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r[i] = recip(x[i]);
}

// cg(k, m) of model m = last mode's roots (surfdisp96's cg), model-major
__global__ void k_copy_last_mode(int nmodel, int kmax, int mode, const double* __restrict__ croot,
                                 double* __restrict__ cg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nmodel * kmax) return;
  const int m = i / kmax, k = i % kmax;
  cg[i] = croot[((size_t)(mode - 1) * kmax + k) * nmodel + m];
}

// ---------------------------------------------------------------------------
// k_eigen: one block per (column, slot group), threads over the group's slots
// ---------------------------------------------------------------------------
__device__ __forceinline__ int worst_status(int a, int b) {
  // NO_ROOT / NAN dominate, then ITER_LIMIT, then RETRIED
  auto rank = [](int s) { return s == ST_NAN_INPUT ? 4 : s == ST_NO_ROOT ? 3 : s == ST_ITER_LIMIT ? 2 : s == ST_RETRIED ? 1 : 0; };
  return rank(a) >= rank(b) ? a : b;
}

// _flat2sphere (surfdisp.cpp:17-51)
__device__ __forceinline__ double flat2sphere(double t, double c, int love, int group) {
  const double ar = 6371.0;
  const double omega = 2.0 * 3.141592653589793 / t;
  const double x = (love ? 1.5 : 0.5) * c / (ar * omega);
  const double tm = sqrt(1. + x * x);
  return group ? c * tm : c / tm;
}

// specialised per wave type WT (0 Rc, 1 Rg, 2 Lc, 3 Lg) and PATH (0
// get_1d_kernel, 1 get_2d_map): one launch per slot group, so each kernel
// carries only the passes it runs (the all-in-one kernel missed in the
// instruction cache)
// one block's work: column col of a model with ncol columns (its arrays
// passed at the model's offsets)
template <int WT, int PATH>
__device__ __noinline__ void eigen_column(int col, int ncol, int nz, int Lmax, const float4* __restrict__ lay0,
                                             const ColInfo* __restrict__ info, const float2* __restrict__ chainrule,
                                             const SlotDesc* __restrict__ slots, int g0, int gn,
                                             const double* __restrict__ croot, const int32_t* __restrict__ cstat,
                                             int sphere, double* __restrict__ vc, double* __restrict__ vout,
                                             double* __restrict__ kernel, int32_t* __restrict__ status, int ldo) {
  constexpr int path = PATH;
  constexpr bool love = WT >= 2;
  using Layer = typename std::conditional<love, LoveLayer, RayLayer>::type;
  extern __shared__ double sm[];
  const ColInfo ci = info[col];
  const int L = ci.L;
  Layer* lay = reinterpret_cast<Layer*>(sm);
  float2* crs = reinterpret_cast<float2*>(lay + L);  // nz chain-rule factors
  const float4* lc = lay0 + (size_t)col * Lmax;
  for (int i = threadIdx.x; i < nz; i += blockDim.x) crs[i] = chainrule[(size_t)i * ncol + col];
  // bldsph (sregn96.f90:130-184 / slegn96.f90:107-167), ar = 6371: the layer
  // records every slot of the column reads.  Each thread sums the
  // thicknesses above its layers itself, in the same order as one running
  // sum, so the depths are those of the sequential loop.
  const double ar = 6371.0;
  for (int i = threadIdx.x; i < L; i += blockDim.x) {
    const float4 l = lc[i];
    double zd, za, zb, zr, vtp, rt;
    if (sphere) {
      double dr = 0.0;
      for (int j = 0; j < i; ++j) dr = dr + (double)lc[j].x;
      const double r0 = (i == 0) ? ar : ar - dr;
      dr = dr + ((i == L - 1) ? 1.0 : (double)l.x);
      const double r1 = ar - dr;
      const double z0 = ar * log(ar / r0), z1 = ar * log(ar / r1);
      const double tmp = (2.0 * ar) / (r0 + r1);
      vtp = tmp;
      if (love) {
        const double t2 = tmp * tmp, t4 = t2 * t2, t5 = t4 * tmp;
        rt = 1.0 / t5;
      } else {
        rt = pow(tmp, (double)(-2.275f));
      }
      za = (double)l.y * tmp;
      zb = (double)l.z * tmp;
      zr = (double)l.w * rt;
      zd = (i == L - 1) ? 0.0 : z1 - z0;
    } else {
      vtp = 1.0; rt = 1.0;
      za = l.y; zb = l.z; zr = l.w;
      zd = l.x;
    }
    if constexpr (love) make_love_layer(lay[i], zd, zb, zr, vtp, rt);
    else make_ray_layer(lay[i], zd, za, zb, zr, vtp, rt);
  }
  __syncthreads();

  using Scratch = typename std::conditional<love, LoveScratch, RayScratch>::type;
  Scratch scr;  // up-pass checkpoints and the segment being consumed (per slot thread)
  double kp[NZMAX];  // one pass's node sums; the scaled sums accumulate in the output
  NodeSink sink;
  sink.kp = (path == 0) ? kp : nullptr;
  sink.crs = crs;
  sink.L = L;
  sink.nw = ci.nw;
  sink.nz = nz;
  const NodeSink nosink = {nullptr, crs, L, ci.nw, nz};
  for (int s = threadIdx.x; s < gn; s += blockDim.x) {
    const SlotDesc sd = slots[g0 + s];
    constexpr bool group = (WT == 1 || WT == 3);
    const double c0 = croot[(size_t)sd.r0 * ncol + col];
    int st = cstat[(size_t)sd.r0 * ncol + col];
    double c1 = 0.0, c2 = 0.0;
    const bool three = (path == 0) && group;
    if (three) {
      c1 = croot[(size_t)sd.r1 * ncol + col];
      c2 = croot[(size_t)sd.r2 * ncol + col];
      st = worst_status(st, cstat[(size_t)sd.r1 * ncol + col]);
      st = worst_status(st, cstat[(size_t)sd.r2 * ncol + col]);
    }
    const size_t oo = (size_t)sd.oslot * ldo + col;  // outputs: row stride ldo (>= ncol)
    bool dead = !ci.valid || c0 == 0.0 || (three && (c1 == 0.0 || c2 == 0.0));
    if (!ci.valid) st = ST_NAN_INPUT;
    else if (dead) st = ST_NO_ROOT;
    if (status) status[oo] = st;
    if (dead) {
      vc[oo] = 0.0;
      vout[oo] = 0.0;
      if (path == 0)
        for (int i = 0; i < nz; ++i) kernel[((size_t)sd.oslot * nz + i) * ldo + col] = 0.0;
      continue;
    }
    if constexpr (PATH == 1) {  // get_2d_map: disp1D (SurfaceWave.cpp:177-255)
      if (!group) {
        const double v = sphere ? flat2sphere(sd.t, c0, love, 0) : c0;
        vc[oo] = v;
        vout[oo] = v;
      } else {
        vc[oo] = sphere ? flat2sphere(sd.t, c0, love, 0) : c0;
        const double omega = 2.0 * PI_F / sd.t, wvno = omega / c0;
        double ugr, norm;
        if constexpr (love) love_pass(lay, L, omega, wvno, scr, ugr, norm, nosink);
        else rayleigh_pass(lay, L, omega, wvno, scr, ugr, norm, nosink);
        double tm = 1.0;
        if (sphere) {
          const double x = (love ? 3.0 : 1.0) * c0 / (2. * ar * omega);
          tm = sqrt(1. + x * x);
        }
        vout[oo] = ugr * tm;
      }
    } else {
    // ---- get_1d_kernel: kernel1D (SurfaceWave.cpp:266-412) ----
    double* kout = kernel + (size_t)sd.oslot * nz * ldo + col;  // node i at kout[i * ldo]
    if (!group) {
      const double omega = 2.0 * PI_F / sd.t, wvno = omega / c0;
      double ugr, norm;
      for (int i = 0; i < nz; ++i) kp[i] = 0.0;
      if constexpr (love) love_pass(lay, L, omega, wvno, scr, ugr, norm, sink);
      else rayleigh_pass(lay, L, omega, wvno, scr, ugr, norm, sink);
      double tm = 1.0;
      if (sphere) {
        const double x = (love ? 3.0 : 1.0) * c0 / (2. * ar * omega);
        tm = sqrt(1. + x * x);
      }
      const double s1 = 1.0 / (norm * tm * tm * tm);
      for (int i = 0; i < nz; ++i) kout[(size_t)i * ldo] = kp[i] * s1;
      const double cs = c0 / tm;
      vc[oo] = cs;
      vout[oo] = cs;
    } else {
      // sregnpu / slegnpu (sregn96.f90:1737-1878, slegn96.f90:785-918)
      const double twopi = 2.0 * PI_F;
      const double cp = c0;
      double cg = 0.0, f1 = 0.0, f2 = 0.0, dtt = 1.0, tm = 1.0, tm1 = 0.0;
      for (int pass = 0; pass < 3; ++pass) {
        const double tt = (pass == 0) ? sd.t : (pass == 1) ? sd.t1 : sd.t2;
        const double cc = (pass == 0) ? c0 : (pass == 1) ? c1 : c2;
        const double omega = twopi / tt, wvno = omega / cc;
        double ugr, norm;
        for (int i = 0; i < nz; ++i) kp[i] = 0.0;
        if constexpr (love) love_pass(lay, L, omega, wvno, scr, ugr, norm, sink);
        else rayleigh_pass(lay, L, omega, wvno, scr, ugr, norm, sink);
        double coef;
        if (pass == 0) {
          cg = ugr;
          const double uc1 = cg / cp;
          dtt = sd.t2 - sd.t1;
          f1 = uc1 * (2.0 - uc1);
          f2 = uc1 * uc1 * sd.t;
          if (sphere) {
            const double om0 = twopi / sd.t;
            const double k = love ? 1.5 : 0.5;
            const double x = (love ? 3.0 : 1.0) * cp / (2. * ar * om0);
            tm = sqrt(1. + x * x);
            const double y = k / (ar * om0);
            tm1 = (y * y) / tm;
            coef = cg * cp * tm1;
          } else {
            coef = 0.0;
          }
        } else if (pass == 1) {
          coef = tm * (f2 / dtt);
        } else {
          coef = tm * (f1 - f2 / dtt);
        }
        // the sum over the passes, from 0, in the output
        if (coef != 0.0) {
          const double s1 = coef / norm;
          for (int i = 0; i < nz; ++i) {
            const double prev = (pass == 0) ? 0.0 : kout[(size_t)i * ldo];
            kout[(size_t)i * ldo] = prev + kp[i] * s1;
          }
        } else if (pass == 0) {
          for (int i = 0; i < nz; ++i) kout[(size_t)i * ldo] = 0.0;
        }
      }
      vc[oo] = cp / tm;
      vout[oo] = cg * tm;
    }
    // water / merged fluid nodes carry no kernel (SurfaceWave.cpp:495)
    for (int i = 0; i < ci.nw; ++i) kout[(size_t)i * ldo] = 0.0;
    }  // get_1d_kernel
  }
}

template <int WT, int PATH>
__global__ void __launch_bounds__(128, (WT >= 2) ? SWDK_EIGEN_MINB_LOVE : SWDK_EIGEN_MINB) k_eigen(int ncol, int nz, int Lmax, const float4* __restrict__ lay0,
                                               const ColInfo* __restrict__ info, const float2* __restrict__ chainrule,
                                               const SlotDesc* __restrict__ slots, int g0, int gn,
                                               const double* __restrict__ croot, const int32_t* __restrict__ cstat,
                                               int sphere, double* __restrict__ vc, double* __restrict__ vout,
                                               double* __restrict__ kernel, int32_t* __restrict__ status, int ldo,
                                               int col0) {
  eigen_column<WT, PATH>(col0 + (int)blockIdx.x, ncol, nz, Lmax, lay0, info, chainrule, slots, g0, gn, croot, cstat, sphere, vc,
                         vout, kernel, status, ldo);
}

// the same over a ragged batch: block b is column b - blk0 of the model of
// the REBlock entry holding b
template <int WT, int PATH>
__global__ void __launch_bounds__(128, (WT >= 2) ? SWDK_EIGEN_MINB_LOVE : SWDK_EIGEN_MINB)
    k_eigen_ragged(const REBlock* __restrict__ eb, int neb, const RModel* __restrict__ models,
                   const float4* __restrict__ lay0, const ColInfo* __restrict__ info,
                   const float2* __restrict__ chainrule, const SlotDesc* __restrict__ slots,
                   const double* __restrict__ croot, const int32_t* __restrict__ cstat, int sphere) {
  const long long b = blockIdx.x;
  const REBlock E = eb[ragged_find(eb, neb, b, &REBlock::blk0)];
  const RModel M = models[E.model];
  eigen_column<WT, PATH>((int)(b - E.blk0), M.ncol, M.nz, M.Lmax, lay0 + M.lay0, info + M.col0, chainrule + M.crs0,
                         slots, E.g0, E.gn, croot + M.root0, cstat + M.root0, sphere, M.vc, M.vout, M.kernel,
                         M.status, M.ncol);
}

// ---------------------------------------------------------------------------
// Frechet rows (SurfaceWave.cpp:630-659): one block per row
// ---------------------------------------------------------------------------
// rowptr == null: row r at r * n (padded rows); else at rowptr[r] (CSR).
// count_only: only nnz[r] is written.
__global__ void k_frechet(int nx, int ny, int nz, int kmax, const double* __restrict__ kernel, const int32_t* __restrict__ slot,
                          const float* __restrict__ fdm, int32_t* __restrict__ nnz, int32_t* __restrict__ idx,
                          float* __restrict__ val, const int64_t* __restrict__ rowptr, int count_only) {
  const int r = blockIdx.x;
  const int nxi = nx - 2, nyi = ny - 2;
  const int n = nxi * nyi * (nz - 1);
  const size_t ncol = (size_t)nx * ny;
  const int s = slot[r];
  if (s < 0 || s >= kmax) {  // invalid period slot: empty row
    if (threadIdx.x == 0) nnz[r] = 0;
    return;
  }
  const float* f = fdm + (size_t)r * ncol;
  const size_t o0 = rowptr ? (size_t)rowptr[r] : (size_t)r * n;
  int32_t* oi = count_only ? nullptr : idx + o0;
  float* ov = count_only ? nullptr : val + o0;
  __shared__ int base;
  __shared__ int wsum[32];
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int j0 = 0; j0 < n; j0 += blockDim.x) {
    const int j = j0 + threadIdx.x;
    float v = 0.0f;
    bool keep = false;
    if (j < n) {
      const int ix = j % nxi, iy = (j / nxi) % nyi, iz = j / (nxi * nyi);
      const size_t ii = (size_t)(iy + 1) * nx + ix + 1;
      v = (float)((double)f[(ix + 1) + (size_t)nx * (iy + 1)] * kernel[ii + ncol * (iz + (size_t)nz * s)]);
      keep = fabsf(v) > 0.0f;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    const int wpre = __popc(bal & ((1u << lane) - 1u));
    if (lane == 0) wsum[wid] = __popc(bal);
    __syncthreads();
    int off = 0, tot = 0;
    for (int w = 0; w < nw; ++w) { if (w < wid) off += wsum[w]; tot += wsum[w]; }
    if (keep && !count_only) { oi[base + off + wpre] = j; ov[base + off + wpre] = v; }
    __syncthreads();
    if (threadIdx.x == 0) base += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0 && nnz) nnz[r] = base;
}

// LSMR's products with the assembled sensitivity matrix (the reference's
// myaprod_csr, src/shared/parallel.cpp:31-115): FP32 values, FP64 vectors.
// mode 1: y += A x, one warp per row, lanes stride over the row's entries;
// mode 2: x += A^T y, one warp per row scattering with FP64 atomics (the
// reference uses an OpenMP atomic; the summation order is not fixed).
__global__ void k_aprod1(int64_t m, const int64_t* __restrict__ rowptr, const int32_t* __restrict__ idx,
                         const float* __restrict__ val, const double* __restrict__ x, double* __restrict__ y) {
  const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= m) return;
  double acc = 0.0;
  for (int64_t j = rowptr[r] + lane; j < rowptr[r + 1]; j += 32) acc += (double)val[j] * x[idx[j]];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0) y[r] += acc;
}

__global__ void k_aprod2(int64_t m, const int64_t* __restrict__ rowptr, const int32_t* __restrict__ idx,
                         const float* __restrict__ val, double* __restrict__ x, const double* __restrict__ y) {
  const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= m) return;
  const double yr = y[r];
  if (yr == 0.0) return;
  for (int64_t j = rowptr[r] + lane; j < rowptr[r + 1]; j += 32) atomicAdd(&x[idx[j]], (double)val[j] * yr);
}

// exclusive prefix sum of nnz[0..n) into rowptr[0..n] (one block)
// The reference's row-file records (SurfaceWave.cpp:596-603, 641-659) from
// CSR rows: a header (int32 m, int32 n) and per row int32 row id, int32 nnz,
// int32 idx[nnz], float32 val[nnz]; row r starts at word 2 + 2r + 2 rowptr[r].
// One warp per row, the index and value runs copied with coalesced accesses.
__global__ void k_frechet_records(int64_t m, int32_t mh, int32_t n, const int32_t* __restrict__ row_ids, int32_t row0,
                                  const int64_t* __restrict__ rowptr, const int32_t* __restrict__ idx,
                                  const float* __restrict__ val, int32_t* __restrict__ out) {
  const int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (r == 0 && lane == 0) { out[0] = mh; out[1] = n; }
  if (r >= m) return;
  const int64_t a = rowptr[r], b = rowptr[r + 1];
  int32_t* rec = out + 2 + 2 * r + 2 * a;
  if (lane == 0) {
    rec[0] = row_ids ? row_ids[r] : (int32_t)(row0 + r);
    rec[1] = (int32_t)(b - a);
  }
  const int64_t nnz = b - a;
  int32_t* oi = rec + 2;
  int32_t* ov = rec + 2 + nnz;
  for (int64_t k = lane; k < nnz; k += 32) {
    oi[k] = idx[a + k];
    ov[k] = __float_as_int(val[a + k]);
  }
}

__global__ void k_rowptr(int n, const int32_t* __restrict__ nnz, int64_t* __restrict__ rowptr) {
  __shared__ long long part[1024];
  __shared__ long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int a = 0; a < n; a += blockDim.x) {
    const int i = a + threadIdx.x;
    part[threadIdx.x] = (i < n) ? nnz[i] : 0;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1) {  // Hillis-Steele inclusive scan
      const long long v = (threadIdx.x >= (unsigned)o) ? part[threadIdx.x - o] : 0;
      __syncthreads();
      part[threadIdx.x] += v;
      __syncthreads();
    }
    if (i < n) rowptr[i + 1] = carry + part[threadIdx.x];
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry += part[threadIdx.x];
    __syncthreads();
  }
  if (threadIdx.x == 0) rowptr[0] = 0;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct DevBuf {
  void* p = nullptr;
  size_t n = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= n) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaSuccess) n = bytes;
    return e;
  }
  void release() { if (p) cudaFree(p); p = nullptr; n = 0; }
  template <class T> T* as() const { return (T*)p; }
};

struct Plan {
  std::vector<int> order;  // chains queued Rayleigh first
  DevBuf d_order;
  std::vector<ChainDesc> chains;
  std::vector<double> periods;
  std::vector<SlotDesc> slots;  // grouped by wave type
  SlotGroups groups;
  std::vector<float4> rootfeat;  // per root slot: (log T / log 100, mode / 2, Rayleigh, 0)
  std::vector<int> rootwave, rootmode;
  std::vector<double> rootperiod;
  int kmax = 0, nroot = 0, nrootR = 0;  // root slots [0, nrootR) are Rayleigh
  DevBuf d_chains, d_periods, d_slots, d_rootfeat;
};

int nt_of(const double* col, int ntmax) {
  int n = 0;
  while (n < ntmax && col[n] != -1) ++n;
  return n;
}

}  // namespace

#ifndef SWDK_HOST_CHUNKS
#define SWDK_HOST_CHUNKS 16
#endif
// eigen chunks of a host-memory call (e2e on the default workload: 4 chunks
// 14.9, 8 chunks 15.25, 16 chunks 15.33 M slots/s with device time 15.4;
// with the faster eigen stage 16 chunks 17.29, 32 chunks 16.72 M slots/s)
constexpr int HOST_CHUNKS = SWDK_HOST_CHUNKS;

struct swdk_ctx {
  swdk_config cfg;
  cudaStream_t stream = nullptr;
  std::vector<double> tab[4];
  int ntmax[4] = {0, 0, 0, 0}, nmode[4] = {0, 0, 0, 0};
  std::vector<float> depth;
  bool have_periods = false;
  bool dirty = true;
  Plan plan[2];  // 0: get_1d_kernel, 1: get_2d_map
  DevBuf layR, layL, lay0, info, chainrule, croot, cstat, nevals, depth_d, ierr, queue;
  DevBuf nodes, dltab;  // grid nodes and the depth grid's flattening (node-source root search)
  int roots_blocks = 0;
  DevBuf in_vs, in_vp, in_rho, out_vc, out_vout, out_kernel, out_status, in_misc;
  // learned bracket proposals
  swdk_mlp* net[2] = {nullptr, nullptr};  // 0: Rayleigh, 1: Love
  double kappa[2] = {4.0, 4.0};
  double prop_shift = 0.0;  // swdk_set_proposal_shift (testing aid)
  DevBuf nodefeat, pfeat, prop;
  DevBuf retry_list, retry_ctr;  // deferred retries: records and {count, queue}
  int last_ncol = 0, last_path = -1;
  // depth vector on the device (uploaded once per swdk_set_depth)
  const void* depth_dev = nullptr;
  // with split_cols > 0, large calls run as two column halves on two child
  // contexts (own buffers and streams), forked from and joined back into the
  // caller's stream
  swdk_ctx* kids[2] = {nullptr, nullptr};
  cudaEvent_t evfork = nullptr, evjoin[2] = {nullptr, nullptr};
  bool last_split = false;
  // host-memory calls: the copy stream of the chunked output copies and
  // one event per chunk plus one for the end of the copies
  cudaStream_t cstream = nullptr;
  cudaEvent_t evchunk[HOST_CHUNKS + 1] = {};
  // host-memory calls: two streams the eigen chunks alternate on, and
  // their fork/join events
  cudaStream_t estream[2] = {};
  cudaEvent_t evefork = nullptr, evejoin[2] = {};
  // CUDA graph of one call (swdk_graph_capture / swdk_graph_launch)
  bool capturing = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int launches = 0;  // kernels launched by the current call
  // stage marks: 0 start, 1 prep, 5 proposals, 2 roots, 3 eigen, 4 call done
  cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  unsigned long long* h_nevals = nullptr;
  swdk_stats stats;
  bool stats_pending = false;
  std::string err;
};

namespace {

int fail(swdk_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

#define CK(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) return fail(ctx, SWDK_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

int find_chain(Plan& P, std::vector<std::vector<double>>& lists, int iwave, const std::vector<double>& lst, int nmode) {
  for (size_t i = 0; i < P.chains.size(); ++i) {
    if (P.chains[i].iwave == iwave && lists[i] == lst) {
      P.chains[i].nmode = std::max(P.chains[i].nmode, nmode);
      return (int)i;
    }
  }
  ChainDesc d;
  d.t_off = 0;
  d.np = (int)lst.size();
  d.nmode = nmode;
  d.iwave = iwave;
  d.igr = 0;
  d.out_off = 0;
  P.chains.push_back(d);
  lists.push_back(lst);
  return (int)P.chains.size() - 1;
}

int build_plan(swdk_ctx* ctx, int path) {
  Plan& P = ctx->plan[path];
  P.chains.clear();
  P.periods.clear();
  P.slots.clear();
  std::vector<std::vector<double>> lists;
  struct Pending { int w, oslot, ch0, ch1, ch2, mode, k; double t, t1, t2; };
  std::vector<Pending> pend;
  int idx = 0;
  for (int w = 0; w < 4; ++w) {
    if (ctx->ntmax[w] * ctx->nmode[w] <= 0) continue;
    for (int mode = 0; mode < ctx->nmode[w]; ++mode) {
      const double* col = ctx->tab[w].data() + (size_t)mode * ctx->ntmax[w];
      const int nt = nt_of(col, ctx->ntmax[w]);
      if (nt == 0) continue;
      if (nt > SWDK_MAX_PERIODS) return fail(ctx, SWDK_E_LIMIT, "more than SWDK_MAX_PERIODS periods in one list");
      const int iwave = (w < 2) ? 2 : 1;
      std::vector<double> lst(col, col + nt), l1(nt), l2(nt);
      const double dt = 0.01;
      for (int i = 0; i < nt; ++i) { l1[i] = col[i] * (1.0 + 0.5 * dt); l2[i] = col[i] * (1.0 - 0.5 * dt); }
      const int ch0 = find_chain(P, lists, iwave, lst, mode + 1);
      int ch1 = -1, ch2 = -1;
      const bool group = (w == 1 || w == 3);
      if (path == 0 && group) {
        ch1 = find_chain(P, lists, iwave, l1, mode + 1);
        ch2 = find_chain(P, lists, iwave, l2, mode + 1);
      }
      for (int k = 0; k < nt; ++k) pend.push_back({w, idx + k, ch0, ch1, ch2, mode, k, lst[k], l1[k], l2[k]});
      idx += nt;
    }
  }
  P.kmax = idx;
  for (size_t i = 0; i < P.chains.size(); ++i) {
    P.chains[i].t_off = (int)P.periods.size();
    P.periods.insert(P.periods.end(), lists[i].begin(), lists[i].end());
  }
  // root slots: Rayleigh chains first, so one proposal network covers a
  // contiguous row range
  int off = 0;
  P.rootfeat.clear();
  P.rootwave.clear();
  P.rootmode.clear();
  P.rootperiod.clear();
  for (int w = 2; w >= 1; --w) {
    for (size_t i = 0; i < P.chains.size(); ++i) {
      ChainDesc& d = P.chains[i];
      if (d.iwave != w) continue;
      d.out_off = off;
      off += d.nmode * d.np;
      for (int m = 0; m < d.nmode; ++m)
        for (int k = 0; k < d.np; ++k) {
          const double t = lists[i][k];
          P.rootfeat.push_back(make_float4((float)(std::log(t) / std::log(100.0)), 0.5f * (float)m,
                                           w == 2 ? 1.0f : 0.0f, 0.0f));
          P.rootwave.push_back(w);
          P.rootmode.push_back(m);
          P.rootperiod.push_back(t);
        }
    }
    if (w == 2) P.nrootR = off;
  }
  P.nroot = off;
  auto rslot = [&](int ch, int mode, int k) { return ch < 0 ? -1 : P.chains[ch].out_off + mode * P.chains[ch].np + k; };
  for (const Pending& q : pend) {
    SlotDesc s;
    s.wtype = q.w;
    s.oslot = q.oslot;
    s.r0 = rslot(q.ch0, q.mode, q.k);
    s.r1 = rslot(q.ch1, q.mode, q.k);
    s.r2 = rslot(q.ch2, q.mode, q.k);
    s.t = q.t;
    s.t1 = q.t1;
    s.t2 = q.t2;
    P.slots.push_back(s);
  }
  if (P.chains.empty()) return fail(ctx, SWDK_E_NOPERIODS, "no periods");
  std::stable_sort(P.slots.begin(), P.slots.end(), [](const SlotDesc& a, const SlotDesc& b) { return a.wtype < b.wtype; });
  P.groups.n = 0;
  for (size_t i = 0; i < P.slots.size(); ++i) {
    if (i == 0 || P.slots[i].wtype != P.slots[i - 1].wtype) {
      P.groups.start[P.groups.n] = (int)i;
      P.groups.count[P.groups.n] = 0;
      ++P.groups.n;
    }
    ++P.groups.count[P.groups.n - 1];
  }
  P.order.clear();
  for (int w = 2; w >= 1; --w)
    for (size_t i = 0; i < P.chains.size(); ++i)
      if (P.chains[i].iwave == w) P.order.push_back((int)i);
  CK(P.d_order.ensure(P.order.size() * sizeof(int)));
  CK(cudaMemcpy(P.d_order.p, P.order.data(), P.order.size() * sizeof(int), cudaMemcpyHostToDevice));
  CK(P.d_chains.ensure(P.chains.size() * sizeof(ChainDesc)));
  CK(P.d_periods.ensure(P.periods.size() * sizeof(double)));
  CK(P.d_slots.ensure(P.slots.size() * sizeof(SlotDesc)));
  CK(P.d_rootfeat.ensure(P.rootfeat.size() * sizeof(float4)));
  CK(cudaMemcpy(P.d_rootfeat.p, P.rootfeat.data(), P.rootfeat.size() * sizeof(float4), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(P.d_chains.p, P.chains.data(), P.chains.size() * sizeof(ChainDesc), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(P.d_periods.p, P.periods.data(), P.periods.size() * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(P.d_slots.p, P.slots.data(), P.slots.size() * sizeof(SlotDesc), cudaMemcpyHostToDevice));
  return SWDK_OK;
}

int ensure_plans(swdk_ctx* ctx) {
  if (!ctx->have_periods) return fail(ctx, SWDK_E_NOPERIODS, "swdk_set_periods not called");
  if (!ctx->dirty) return SWDK_OK;
  for (int p = 0; p < 2; ++p) {
    int r = build_plan(ctx, p);
    if (r) return r;
  }
  ctx->dirty = false;
  return SWDK_OK;
}

constexpr int PROP_CHUNK = 1 << 20;  // proposal rows per feature/inference launch pair (multiple of 128)

bool proposals_on(const swdk_ctx* ctx) { return ctx->cfg.refine == 1 && (ctx->net[0] || ctx->net[1]); }

// features -> fused network -> (c, half-width) for every root row of plan P
// nodefeat / prop: the node features k_prep wrote and the proposal rows to
// fill (null: the context's own buffers)
int run_proposals(swdk_ctx* ctx, const Plan& P, int ncol, cudaStream_t st, const float4* nodefeat = nullptr,
                  float2* prop = nullptr) {
  const int64_t nrows = (int64_t)P.nroot * ncol;
  if (!prop) {
    CK(ctx->prop.ensure((size_t)nrows * sizeof(float2)));
    prop = ctx->prop.as<float2>();
  }
  if (!nodefeat) nodefeat = ctx->nodefeat.as<float4>();
  CK(ctx->pfeat.ensure((size_t)PROP_CHUNK * FEAT_DIM * sizeof(__nv_bfloat16)));
  const int64_t bound[3] = {0, (int64_t)P.nrootR * ncol, nrows};
  for (int w = 0; w < 2; ++w) {
    const int64_t r0 = bound[w], r1 = bound[w + 1];
    if (r1 <= r0) continue;
    if (!ctx->net[w]) {
      CK(cudaMemsetAsync(prop + r0, 0, (size_t)(r1 - r0) * sizeof(float2), st));
      continue;
    }
    for (int64_t a = r0; a < r1; a += PROP_CHUNK) {
      const int n = (int)std::min<int64_t>(PROP_CHUNK, r1 - a);
      ctx->launches += 2;
      k_features<<<(n + 15) / 16, 256, 0, st>>>(a, n, ncol, nrows, P.d_rootfeat.as<float4>(), nodefeat, nullptr,
                                              ctx->pfeat.as<__nv_bfloat16>(), 1);
      CK(cudaGetLastError());
      int r = swdk_mlp_propose(ctx->net[w], ctx->pfeat.p, n, ctx->kappa[w], prop + a, st);
      if (r) return fail(ctx, r, std::string("proposal inference: ") + swdk_mlp_last_error(ctx->net[w]));
      if (ctx->prop_shift != 0.0) {
        ctx->launches += 1;
        k_shift_prop<<<(n + 255) / 256, 256, 0, st>>>(n, prop + a, (float)ctx->prop_shift);
        CK(cudaGetLastError());
      }
    }
  }
  return SWDK_OK;
}

// model preparation + (proposals) + roots + (eigen) for one call on device
// pointers; path 0 get_1d_kernel, 1 get_2d_map, 2 roots of path 0 only
// ldi / ldo: row strides (in columns) of the input model and of the outputs,
// >= nx*ny; -1 = nx*ny (dense).  A column block of a larger model runs with
// the pointers offset to its first column and the large model's strides.
// Host destination of a host-memory call's outputs: columns c0.. of
// (rows, ld) arrays.
struct HostOut {
  double *vc, *vout, *kernel;
  int32_t* status;
  int ld, c0;
};

int launch_eigen(swdk_ctx* ctx, const Plan& P, int path, int ncol, int nz, int c0, int c1, double* d_vc,
                 double* d_vout, double* d_kernel, int32_t* d_status, int ldo, cudaStream_t st);

int run_device(swdk_ctx* ctx, int path, int nx, int ny, int nz, const float* d_vs, const float* d_vp,
               const float* d_rho, double* d_vc, double* d_vout, double* d_kernel, int32_t* d_status,
               cudaStream_t st, int ldi = -1, int ldo = -1, const HostOut* ho = nullptr) {
  const bool roots_only = (path == 2);
  if (roots_only) path = 0;
  if (nx <= 0 || ny <= 0 || !d_vs || (!roots_only && (!d_vc || !d_vout || (path == 0 && !d_kernel))))
    return fail(ctx, SWDK_E_ARG, "bad arguments");
  if ((d_vp == nullptr) != (d_rho == nullptr)) return fail(ctx, SWDK_E_ARG, "vp and rho must both be given or both NULL");
  if ((int)ctx->depth.size() != nz) return fail(ctx, SWDK_E_NODEPTH, "nz does not match swdk_set_depth");
  if (nz < 2 || nz > SWDK_MAX_NZ || 4 * nz - 3 > SWDK_MAX_LAYERS) return fail(ctx, SWDK_E_LIMIT, "nz out of range");
  int r = ensure_plans(ctx);
  if (r) return r;
  Plan& P = ctx->plan[path];
  const int ncol = nx * ny;
  if (ldi < 0) ldi = ncol;
  if (ldo < 0) ldo = ncol;
  if (ldi < ncol || ldo < ncol) return fail(ctx, SWDK_E_ARG, "row stride below the column count");
  const int Lmax = 4 * nz - 3;
  const bool useprop = proposals_on(ctx);
  const bool wantfeat = useprop || roots_only;
  CK(ctx->layR.ensure((size_t)Lmax * ncol * sizeof(float4)));
  CK(ctx->layL.ensure((size_t)Lmax * ncol * sizeof(float4)));
  CK(ctx->queue.ensure(sizeof(unsigned int)));
  CK(ctx->lay0.ensure((size_t)Lmax * ncol * sizeof(float4)));
  CK(ctx->info.ensure((size_t)ncol * sizeof(ColInfo)));
  CK(ctx->chainrule.ensure((size_t)nz * ncol * sizeof(float2)));
  CK(ctx->croot.ensure((size_t)P.nroot * ncol * sizeof(double)));
  CK(ctx->cstat.ensure((size_t)P.nroot * ncol * sizeof(int32_t)));
  CK(ctx->nevals.ensure(NCOUNT * sizeof(unsigned long long)));
  if (wantfeat) CK(ctx->nodefeat.ensure((size_t)ncol * FEAT_NODES * sizeof(float4)));
  CK(ctx->depth_d.ensure((size_t)nz * sizeof(float)));
  if (ctx->depth_dev != ctx->depth_d.p) {  // first call after swdk_set_depth (never inside a capture)
    if (ctx->capturing) return fail(ctx, SWDK_E_ARG, "depth not on the device before graph capture");
    CK(cudaMemcpyAsync(ctx->depth_d.p, ctx->depth.data(), nz * sizeof(float), cudaMemcpyHostToDevice, st));
    ctx->depth_dev = ctx->depth_d.p;
  }
  const bool use_nodes = ctx->cfg.node_layers != 0;
  if (use_nodes) {
    CK(ctx->nodes.ensure((size_t)nz * ncol * sizeof(float4)));
    CK(ctx->dltab.ensure((size_t)Lmax * sizeof(DepthLayer)));
  }
  CK(cudaMemsetAsync(ctx->nevals.p, 0, NCOUNT * sizeof(unsigned long long), st));
  const bool timing = !ctx->capturing;  // stage events and statistics only on eager calls
  if (timing) CK(cudaEventRecord(ctx->ev[0], st));
  ctx->launches = 0;
  if (use_nodes) {
    ctx->launches += 1;
    k_depth_table<<<1, 32, 0, st>>>(nz, ctx->depth_d.as<float>(), ctx->cfg.sphere, ctx->dltab.as<DepthLayer>());
    CK(cudaGetLastError());
  }
  ctx->launches += 1;
  k_prep<<<(ncol + 127) / 128, 128, 0, st>>>(ncol, ldi, nz, d_vs, d_vp, d_rho, ctx->depth_d.as<float>(), ctx->cfg.sphere,
                                             Lmax, ctx->layR.as<float4>(), ctx->layL.as<float4>(),
                                             ctx->lay0.as<float4>(), ctx->info.as<ColInfo>(),
                                             ctx->chainrule.as<float2>(), wantfeat ? ctx->nodefeat.as<float4>() : nullptr,
                                             use_nodes ? ctx->nodes.as<float4>() : nullptr);
  CK(cudaGetLastError());
  if (timing) CK(cudaEventRecord(ctx->ev[1], st));
  if (useprop) {
    r = run_proposals(ctx, P, ncol, st);
    if (r) return r;
  }
  if (timing) CK(cudaEventRecord(ctx->ev[5], st));
  if (ctx->roots_blocks == 0) {
    int dev = 0, nsm = 0, per = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    CK(roots_occupancy(&per));
    ctx->roots_blocks = std::max(1, nsm * std::max(1, per));
  }
  const int nitems = (int)P.chains.size() * ncol;
  const int rblocks = ctx->cfg.block_roots > 0 ? ctx->cfg.block_roots : ctx->roots_blocks;
  const unsigned int rcap = (unsigned int)std::min<size_t>((size_t)P.nroot * ncol, 0x7fffffffu);
  CK(ctx->retry_list.ensure((size_t)rcap * sizeof(int2)));
  CK(ctx->retry_ctr.ensure(2 * sizeof(unsigned int)));
  CK(cudaMemsetAsync(ctx->queue.p, 0, sizeof(unsigned int), st));
  CK(cudaMemsetAsync(ctx->retry_ctr.p, 0, 2 * sizeof(unsigned int), st));
  unsigned int* rctr = ctx->retry_ctr.as<unsigned int>();
  ctx->launches += 2;
  k_roots_queue<<<std::min(rblocks, (nitems + 127) / 128), 128, ROOTS_SMEM, st>>>(
      ncol, nitems, P.d_order.as<int>(), P.d_chains.as<ChainDesc>(), P.d_periods.as<double>(), ctx->layR.as<float4>(),
      ctx->layL.as<float4>(), ctx->info.as<ColInfo>(), ctx->cfg.refine, ctx->cfg.rtol, ctx->cfg.sngl, RETRY_DEFERRED,
      ctx->croot.as<double>(), ctx->cstat.as<int32_t>(), ctx->queue.as<unsigned int>(),
      useprop ? ctx->prop.as<float2>() : nullptr, ctx->retry_list.as<int2>(), rctr, rcap,
      ctx->nevals.as<unsigned long long>(), RaggedMap{nullptr, nullptr, 0, Lmax},
      use_nodes ? ctx->nodes.as<float4>() : nullptr, ctx->dltab.as<DepthLayer>());
  CK(cudaGetLastError());
  k_retry<<<rblocks, 128, ROOTS_SMEM, st>>>(ncol, P.d_order.as<int>(), P.d_chains.as<ChainDesc>(), P.d_periods.as<double>(),
                                   ctx->layR.as<float4>(), ctx->layL.as<float4>(), ctx->info.as<ColInfo>(),
                                   ctx->cfg.refine, ctx->cfg.rtol, ctx->cfg.sngl, ctx->croot.as<double>(),
                                   ctx->cstat.as<int32_t>(), ctx->retry_list.as<int2>(), rctr, rcap, rctr + 1,
                                   ctx->nevals.as<unsigned long long>(), RaggedMap{nullptr, nullptr, 0, Lmax},
                                   use_nodes ? ctx->nodes.as<float4>() : nullptr, ctx->dltab.as<DepthLayer>());
  CK(cudaGetLastError());
  if (timing) CK(cudaEventRecord(ctx->ev[2], st));
  if (!roots_only) {
    if (!ho) {
      r = launch_eigen(ctx, P, path, ncol, nz, 0, ncol, d_vc, d_vout, d_kernel, d_status, ldo, st);
      if (r) return r;
    } else {
      // host-memory call: the eigen stage in column chunks, each chunk's
      // outputs copied to the host on the copy stream while the next chunk
      // computes
      if (!ctx->cstream) CK(cudaStreamCreateWithFlags(&ctx->cstream, cudaStreamNonBlocking));
      for (int i = 0; i <= HOST_CHUNKS; ++i)
        if (!ctx->evchunk[i]) CK(cudaEventCreateWithFlags(&ctx->evchunk[i], cudaEventDisableTiming));
      for (int i = 0; i < 2; ++i) {
        if (!ctx->estream[i]) CK(cudaStreamCreateWithFlags(&ctx->estream[i], cudaStreamNonBlocking));
        if (!ctx->evejoin[i]) CK(cudaEventCreateWithFlags(&ctx->evejoin[i], cudaEventDisableTiming));
      }
      if (!ctx->evefork) CK(cudaEventCreateWithFlags(&ctx->evefork, cudaEventDisableTiming));
      const int kmax = P.kmax;
      auto chunk = [&](int h, int& a, int& b) {
        a = (int)((long long)ncol * h / HOST_CHUNKS);
        b = (int)((long long)ncol * (h + 1) / HOST_CHUNKS);
      };
      // every chunk is queued before the first copy is issued: a copy to
      // pageable host memory returns only when done, and the chunks behind
      // it must already be on the device by then.  The chunks alternate
      // between two streams, so one chunk's blocks fill the SMs that the
      // other's last wave leaves idle (the outputs are disjoint columns).
      CK(cudaEventRecord(ctx->evefork, st));
      for (int i = 0; i < 2; ++i) CK(cudaStreamWaitEvent(ctx->estream[i], ctx->evefork, 0));
      for (int h = 0; h < HOST_CHUNKS; ++h) {
        int a, b;
        chunk(h, a, b);
        if (b <= a) continue;
        cudaStream_t es = ctx->estream[h & 1];
        r = launch_eigen(ctx, P, path, ncol, nz, a, b, d_vc, d_vout, d_kernel, d_status, ldo, es);
        if (r) return r;
        CK(cudaEventRecord(ctx->evchunk[h], es));
      }
      for (int i = 0; i < 2; ++i) {
        CK(cudaEventRecord(ctx->evejoin[i], ctx->estream[i]));
        CK(cudaStreamWaitEvent(st, ctx->evejoin[i], 0));
      }
      for (int h = 0; h < HOST_CHUNKS; ++h) {
        int a, b;
        chunk(h, a, b);
        if (b <= a) continue;
        CK(cudaStreamWaitEvent(ctx->cstream, ctx->evchunk[h], 0));
        const size_t w = (size_t)(b - a);
        const size_t hp = (size_t)ho->ld;
        CK(cudaMemcpy2DAsync(ho->vc + ho->c0 + a, hp * sizeof(double), d_vc + a, (size_t)ldo * sizeof(double),
                             w * sizeof(double), kmax, cudaMemcpyDeviceToHost, ctx->cstream));
        CK(cudaMemcpy2DAsync(ho->vout + ho->c0 + a, hp * sizeof(double), d_vout + a, (size_t)ldo * sizeof(double),
                             w * sizeof(double), kmax, cudaMemcpyDeviceToHost, ctx->cstream));
        if (ho->status)
          CK(cudaMemcpy2DAsync(ho->status + ho->c0 + a, hp * sizeof(int32_t), d_status + a,
                               (size_t)ldo * sizeof(int32_t), w * sizeof(int32_t), kmax, cudaMemcpyDeviceToHost,
                               ctx->cstream));
        if (path == 0)
          CK(cudaMemcpy2DAsync(ho->kernel + ho->c0 + a, hp * sizeof(double), d_kernel + a,
                               (size_t)ldo * sizeof(double), w * sizeof(double), (size_t)kmax * nz,
                               cudaMemcpyDeviceToHost, ctx->cstream));
      }
    }
  }
  if (timing) {
    CK(cudaEventRecord(ctx->ev[3], st));
    CK(cudaMemcpyAsync(ctx->h_nevals, ctx->nevals.p, NCOUNT * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    CK(cudaEventRecord(ctx->ev[4], st));
    ctx->stats_pending = true;
  }
  if (ho && !roots_only) {  // the call's stream waits for the output copies
    CK(cudaEventRecord(ctx->evchunk[HOST_CHUNKS], ctx->cstream));
    CK(cudaStreamWaitEvent(st, ctx->evchunk[HOST_CHUNKS], 0));
  }
  ctx->stats.nchains = (int)P.chains.size();
  ctx->stats.nslots = P.kmax;
  ctx->stats.kernel_launches = ctx->launches;
  ctx->last_ncol = ncol;
  ctx->last_path = roots_only ? 2 : path;
  return SWDK_OK;
}

void collect_stats(swdk_ctx* ctx) {
  if (!ctx->stats_pending) return;
  if (ctx->last_split) {  // sum of the two halves; stage times are the longer half's
    ctx->stats_pending = false;
    swdk_stats t;
    memset(&t, 0, sizeof(t));
    for (swdk_ctx* k : ctx->kids) {
      if (!k) continue;
      collect_stats(k);
      const swdk_stats& a = k->stats;
      t.secular_evals += a.secular_evals;
      t.layer_evals_rayleigh += a.layer_evals_rayleigh;
      t.layer_evals_love += a.layer_evals_love;
      t.proposals_accepted += a.proposals_accepted;
      t.proposals_rejected += a.proposals_rejected;
      for (int i = 0; i < NPHASE_EV; ++i) t.evals_by_phase[i] += a.evals_by_phase[i];
      t.kernel_launches += a.kernel_launches;
      t.nchains = a.nchains;
      t.nslots = a.nslots;
      t.ms_prep = std::max(t.ms_prep, a.ms_prep);
      t.ms_proposal = std::max(t.ms_proposal, a.ms_proposal);
      t.ms_roots = std::max(t.ms_roots, a.ms_roots);
      t.ms_eigen = std::max(t.ms_eigen, a.ms_eigen);
    }
    ctx->stats = t;
    return;
  }
  cudaEventSynchronize(ctx->ev[4]);
  ctx->stats_pending = false;
  ctx->stats.secular_evals = (int64_t)ctx->h_nevals[0];
  ctx->stats.layer_evals_rayleigh = (int64_t)ctx->h_nevals[1];
  ctx->stats.layer_evals_love = (int64_t)ctx->h_nevals[2];
  ctx->stats.proposals_accepted = (int64_t)ctx->h_nevals[3];
  ctx->stats.proposals_rejected = (int64_t)ctx->h_nevals[4];
  for (int i = 0; i < NPHASE_EV; ++i) ctx->stats.evals_by_phase[i] = (int64_t)ctx->h_nevals[EV_BASE + i];
  cudaEventElapsedTime(&ctx->stats.ms_prep, ctx->ev[0], ctx->ev[1]);
  cudaEventElapsedTime(&ctx->stats.ms_proposal, ctx->ev[1], ctx->ev[5]);
  cudaEventElapsedTime(&ctx->stats.ms_roots, ctx->ev[5], ctx->ev[2]);
  cudaEventElapsedTime(&ctx->stats.ms_eigen, ctx->ev[2], ctx->ev[3]);
}

// the eigen stage over columns [c0, c1): one launch per wave-type slot group
int launch_eigen(swdk_ctx* ctx, const Plan& P, int path, int ncol, int nz, int c0, int c1, double* d_vc,
                 double* d_vout, double* d_kernel, int32_t* d_status, int ldo, cudaStream_t st) {
  using EigFn = void (*)(int, int, int, const float4*, const ColInfo*, const float2*, const SlotDesc*, int, int,
                         const double*, const int32_t*, int, double*, double*, double*, int32_t*, int, int);
  static const EigFn eig[4][2] = {{k_eigen<0, 0>, k_eigen<0, 1>}, {k_eigen<1, 0>, k_eigen<1, 1>},
                                  {k_eigen<2, 0>, k_eigen<2, 1>}, {k_eigen<3, 0>, k_eigen<3, 1>}};
  const int Lmax = 4 * nz - 3;
  for (int g = 0; g < P.groups.n; ++g) {
    const int g0 = P.groups.start[g], gn = P.groups.count[g];
    const int wt = P.slots[g0].wtype;
    const int et = std::min(128, ((gn + 31) / 32) * 32);
    const size_t smem = (size_t)Lmax * (wt >= 2 ? sizeof(LoveLayer) : sizeof(RayLayer)) + (size_t)nz * sizeof(float2);
    ctx->launches += 1;
    eig[wt][path]<<<c1 - c0, et, smem, st>>>(ncol, nz, Lmax, ctx->lay0.as<float4>(), ctx->info.as<ColInfo>(),
                                             ctx->chainrule.as<float2>(), P.d_slots.as<SlotDesc>(), g0, gn,
                                             ctx->croot.as<double>(), ctx->cstat.as<int32_t>(), ctx->cfg.sphere,
                                             d_vc, d_vout, d_kernel, d_status, ldo, c0);
    CK(cudaGetLastError());
  }
  return SWDK_OK;
}

void drop_graph(swdk_ctx* ctx) {
  if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
  if (ctx->graph) cudaGraphDestroy(ctx->graph);
  ctx->gexec = nullptr;
  ctx->graph = nullptr;
}

void drop_kids(swdk_ctx* ctx) {
  for (int i = 0; i < 2; ++i) {
    if (ctx->kids[i]) swdk_destroy(ctx->kids[i]);
    ctx->kids[i] = nullptr;
    if (ctx->evjoin[i]) cudaEventDestroy(ctx->evjoin[i]);
    ctx->evjoin[i] = nullptr;
  }
  if (ctx->evfork) cudaEventDestroy(ctx->evfork);
  ctx->evfork = nullptr;
  ctx->last_split = false;
}

// child contexts with the parent's configuration, period tables, depth
// vector and proposal networks
int ensure_kids(swdk_ctx* ctx) {
  if (ctx->kids[0] && ctx->kids[1]) return SWDK_OK;
  drop_kids(ctx);
  for (int i = 0; i < 2; ++i) {
    swdk_ctx* k = nullptr;
    const int r = swdk_create(&k, &ctx->cfg);
    if (r) { drop_kids(ctx); return fail(ctx, r, "child context creation failed"); }
    for (int w = 0; w < 4; ++w) { k->tab[w] = ctx->tab[w]; k->ntmax[w] = ctx->ntmax[w]; k->nmode[w] = ctx->nmode[w]; }
    k->have_periods = ctx->have_periods;
    k->dirty = true;
    k->depth = ctx->depth;
    k->net[0] = ctx->net[0];
    k->net[1] = ctx->net[1];
    k->kappa[0] = ctx->kappa[0];
    k->kappa[1] = ctx->kappa[1];
    k->prop_shift = ctx->prop_shift;
    ctx->kids[i] = k;
    CK(cudaEventCreateWithFlags(&ctx->evjoin[i], cudaEventDisableTiming));
  }
  CK(cudaEventCreateWithFlags(&ctx->evfork, cudaEventDisableTiming));
  return SWDK_OK;
}

// split_cols 0 (default): no call splits.  Two concurrent persistent root
// searches only contend (577 vs 557 ms per device step on the default
// workload), and a host-memory call streams its outputs back behind the
// eigen stage's column chunks instead (e2e 13.9 M slots/s unsplit, 13.7 M
// split).
bool use_split(const swdk_ctx* ctx, int path, int ncol, bool host) {
  (void)host;
  const int lim = ctx->cfg.split_cols;
  return path != 2 && lim > 0 && ncol >= lim && ncol >= 2;
}

// a device call, as two column halves when it is large enough
int run_split(swdk_ctx* ctx, int path, int nx, int ny, int nz, const float* d_vs, const float* d_vp,
              const float* d_rho, double* d_vc, double* d_vout, double* d_kernel, int32_t* d_status, cudaStream_t st) {
  const int ncol = nx * ny;
  if (!use_split(ctx, path, ncol, false) || nx <= 0 || ny <= 0) {
    ctx->last_split = false;
    return run_device(ctx, path, nx, ny, nz, d_vs, d_vp, d_rho, d_vc, d_vout, d_kernel, d_status, st);
  }
  int r = ensure_plans(ctx);  // argument checks and the parent's plan (kmax) first
  if (r) return r;
  r = ensure_kids(ctx);
  if (r) return r;
  CK(cudaEventRecord(ctx->evfork, st));
  for (int h = 0; h < 2; ++h) {
    swdk_ctx* k = ctx->kids[h];
    const int c0 = h ? ncol / 2 : 0, n = h ? ncol - ncol / 2 : ncol / 2;
    CK(cudaStreamWaitEvent(k->stream, ctx->evfork, 0));
    k->capturing = ctx->capturing;
    r = run_device(k, path, n, 1, nz, d_vs + c0, d_vp ? d_vp + c0 : nullptr, d_rho ? d_rho + c0 : nullptr,
                   d_vc + c0, d_vout + c0, d_kernel ? d_kernel + c0 : nullptr, d_status ? d_status + c0 : nullptr,
                   k->stream, ncol, ncol);
    k->capturing = false;
    if (r) return fail(ctx, r, std::string("column half: ") + k->err);
    CK(cudaEventRecord(ctx->evjoin[h], k->stream));
    CK(cudaStreamWaitEvent(st, ctx->evjoin[h], 0));
  }
  ctx->last_split = true;
  ctx->stats_pending = !ctx->capturing;
  ctx->last_ncol = ncol;
  ctx->last_path = path;
  return SWDK_OK;
}

// host arrays -> device -> host for columns [c0, c0+n) of an ncol-column
// model, on context k's stream and buffers (strided 2-D copies)
int host_piece(swdk_ctx* ctx, swdk_ctx* k, int path, int ncol, int c0, int n, int nz, const float* vs,
               const float* vp, const float* rho, double* vc, double* vout, double* kernel, int32_t* status) {
  int r = ensure_plans(k);
  if (r) return fail(ctx, r, k->err);
  const int kmax = k->plan[path].kmax;
  cudaStream_t st = k->stream;
  CK(k->in_vs.ensure((size_t)n * nz * sizeof(float)));
  if (vp) {
    CK(k->in_vp.ensure((size_t)n * nz * sizeof(float)));
    CK(k->in_rho.ensure((size_t)n * nz * sizeof(float)));
  }
  CK(k->out_vc.ensure((size_t)n * kmax * sizeof(double)));
  CK(k->out_vout.ensure((size_t)n * kmax * sizeof(double)));
  CK(k->out_status.ensure((size_t)n * kmax * sizeof(int32_t)));
  if (path == 0) CK(k->out_kernel.ensure((size_t)n * nz * kmax * sizeof(double)));
  const size_t fw = (size_t)n * sizeof(float), dw = (size_t)n * sizeof(double), iw = (size_t)n * sizeof(int32_t);
  CK(cudaMemcpy2DAsync(k->in_vs.p, fw, vs + c0, ncol * sizeof(float), fw, nz, cudaMemcpyHostToDevice, st));
  if (vp) {
    CK(cudaMemcpy2DAsync(k->in_vp.p, fw, vp + c0, ncol * sizeof(float), fw, nz, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpy2DAsync(k->in_rho.p, fw, rho + c0, ncol * sizeof(float), fw, nz, cudaMemcpyHostToDevice, st));
  }
  // the outputs stream back chunk by chunk behind the eigen stage
  const HostOut ho{vc, vout, kernel, status, ncol, c0};
  r = run_device(k, path, n, 1, nz, k->in_vs.as<float>(), vp ? k->in_vp.as<float>() : nullptr,
                 vp ? k->in_rho.as<float>() : nullptr, k->out_vc.as<double>(), k->out_vout.as<double>(),
                 path == 0 ? k->out_kernel.as<double>() : nullptr, k->out_status.as<int32_t>(), st, -1, -1, &ho);
  if (r) return fail(ctx, r, k->err);
  (void)dw;
  (void)iw;
  return SWDK_OK;
}

int run_host(swdk_ctx* ctx, int path, int nx, int ny, int nz, const float* vs, const float* vp, const float* rho,
             double* vc, double* vout, double* kernel, int32_t* status) {
  if (!ctx || nx <= 0 || ny <= 0 || !vs || !vc || !vout || (path == 0 && !kernel)) return fail(ctx, SWDK_E_ARG, "bad arguments");
  if ((vp == nullptr) != (rho == nullptr)) return fail(ctx, SWDK_E_ARG, "vp and rho must both be given or both NULL");
  CK(cudaSetDevice(ctx->cfg.device));
  int r = ensure_plans(ctx);
  if (r) return r;
  const int ncol = nx * ny;
  if (!use_split(ctx, path, ncol, true)) {
    r = host_piece(ctx, ctx, path, ncol, 0, ncol, nz, vs, vp, rho, vc, vout, kernel, status);
    if (r) return r;
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->last_split = false;
    collect_stats(ctx);
    return SWDK_OK;
  }
  r = ensure_kids(ctx);
  if (r) return r;
  for (int h = 0; h < 2; ++h) {
    const int c0 = h ? ncol / 2 : 0, n = h ? ncol - ncol / 2 : ncol / 2;
    r = host_piece(ctx, ctx->kids[h], path, ncol, c0, n, nz, vs, vp, rho, vc, vout, kernel, status);
    if (r) return r;
  }
  for (int h = 0; h < 2; ++h) CK(cudaStreamSynchronize(ctx->kids[h]->stream));
  ctx->last_split = true;
  ctx->stats_pending = true;
  ctx->last_ncol = ncol;
  ctx->last_path = path;
  collect_stats(ctx);
  return SWDK_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// surfdisp96_ over device-resident models with no device allocation: the
// scratch (layer models, start values, roots of all modes) lives in this
// file-scope array.  Every GPU that loads the library holds it until exit.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_noalloc_scratch[SWDK_NOALLOC_SCRATCH_BYTES];

namespace {
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[256] = {};  // device address of g_noalloc_scratch, per device ordinal

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
}  // namespace

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
extern "C" {

int swdk_config_default(swdk_config* cfg) {
  if (!cfg) return SWDK_E_ARG;
  cfg->device = 0;
  cfg->refine = SWDK_REFINE_TIGHT;
  cfg->rtol = 1e-10;
  cfg->sngl = 1;
  cfg->sphere = 1;
  cfg->block_roots = 0;
  cfg->split_cols = 0;
  cfg->node_layers = 1;
  return SWDK_OK;
}

int swdk_create(swdk_ctx** out, const swdk_config* cfg) {
  if (!out) return SWDK_E_ARG;
  *out = nullptr;
  swdk_ctx* ctx = new swdk_ctx();
  if (cfg) ctx->cfg = *cfg;
  else swdk_config_default(&ctx->cfg);
  if (ctx->cfg.rtol <= 0.0) ctx->cfg.rtol = 1e-10;
  memset(&ctx->stats, 0, sizeof(ctx->stats));
  cudaError_t e = cudaSetDevice(ctx->cfg.device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  for (int i = 0; i < 6 && e == cudaSuccess; ++i) e = cudaEventCreate(&ctx->ev[i]);
  if (e == cudaSuccess) e = cudaMallocHost((void**)&ctx->h_nevals, NCOUNT * sizeof(unsigned long long));
  if (e != cudaSuccess) {
    fprintf(stderr, "swdk_create: %s\n", cudaGetErrorString(e));
    swdk_destroy(ctx);
    return SWDK_E_CUDA;
  }
  for (int i = 0; i < NCOUNT; ++i) ctx->h_nevals[i] = 0;
  *out = ctx;
  return SWDK_OK;
}

void swdk_destroy(swdk_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->cfg.device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  DevBuf* bufs[] = {&ctx->layR, &ctx->layL, &ctx->lay0, &ctx->info, &ctx->chainrule, &ctx->croot, &ctx->cstat,
                    &ctx->nodes, &ctx->dltab,
                    &ctx->nevals, &ctx->depth_d, &ctx->ierr, &ctx->in_vs, &ctx->in_vp, &ctx->in_rho,
                    &ctx->out_vc, &ctx->out_vout, &ctx->out_kernel, &ctx->out_status, &ctx->in_misc,
                    &ctx->queue, &ctx->nodefeat, &ctx->pfeat,
                    &ctx->prop, &ctx->retry_list, &ctx->retry_ctr};
  for (DevBuf* b : bufs) b->release();
  for (int p = 0; p < 2; ++p) {
    ctx->plan[p].d_chains.release();
    ctx->plan[p].d_periods.release();
    ctx->plan[p].d_slots.release();
    ctx->plan[p].d_order.release();
    ctx->plan[p].d_rootfeat.release();
  }
  drop_graph(ctx);
  drop_kids(ctx);
  for (int i = 0; i < 6; ++i)
    if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
  for (cudaEvent_t e : ctx->evchunk)
    if (e) cudaEventDestroy(e);
  if (ctx->cstream) {
    cudaStreamSynchronize(ctx->cstream);
    cudaStreamDestroy(ctx->cstream);
  }
  for (int i = 0; i < 2; ++i) {
    if (ctx->estream[i]) {
      cudaStreamSynchronize(ctx->estream[i]);
      cudaStreamDestroy(ctx->estream[i]);
    }
    if (ctx->evejoin[i]) cudaEventDestroy(ctx->evejoin[i]);
  }
  if (ctx->evefork) cudaEventDestroy(ctx->evefork);
  if (ctx->h_nevals) cudaFreeHost(ctx->h_nevals);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

int swdk_set_periods(swdk_ctx* ctx, const double* tRc, int ntRc, int nmRc, const double* tRg, int ntRg, int nmRg,
                     const double* tLc, int ntLc, int nmLc, const double* tLg, int ntLg, int nmLg) {
  if (!ctx) return SWDK_E_ARG;
  const double* t[4] = {tRc, tRg, tLc, tLg};
  const int nt[4] = {ntRc, ntRg, ntLc, ntLg}, nm[4] = {nmRc, nmRg, nmLc, nmLg};
  for (int w = 0; w < 4; ++w) {
    if (nt[w] < 0 || nm[w] < 0 || (nt[w] * nm[w] > 0 && !t[w])) return fail(ctx, SWDK_E_ARG, "bad period table");
    if (nt[w] > SWDK_MAX_PERIODS) return fail(ctx, SWDK_E_LIMIT, "period table longer than SWDK_MAX_PERIODS");
    ctx->ntmax[w] = nt[w];
    ctx->nmode[w] = nm[w];
    ctx->tab[w].assign(t[w] ? t[w] : nullptr, t[w] ? t[w] + (size_t)nt[w] * nm[w] : nullptr);
    for (double v : ctx->tab[w])
      if (v != -1 && !(v > 0.0)) return fail(ctx, SWDK_E_ARG, "periods must be positive (or -1 padding)");
  }
  ctx->have_periods = true;
  ctx->dirty = true;
  drop_graph(ctx);
  drop_kids(ctx);
  cudaSetDevice(ctx->cfg.device);
  return ensure_plans(ctx);
}

int swdk_set_depth(swdk_ctx* ctx, const float* depth, int nz) {
  if (!ctx || !depth || nz < 2) return SWDK_E_ARG;
  if (nz > SWDK_MAX_NZ) return fail(ctx, SWDK_E_LIMIT, "nz > SWDK_MAX_NZ");
  ctx->depth.assign(depth, depth + nz);
  ctx->depth_dev = nullptr;
  drop_graph(ctx);
  drop_kids(ctx);
  return SWDK_OK;
}

int swdk_kmax(const swdk_ctx* ctx) {
  if (!ctx || !ctx->have_periods) return 0;
  int k = 0;
  for (int w = 0; w < 4; ++w)
    for (int m = 0; m < ctx->nmode[w]; ++m) k += nt_of(ctx->tab[w].data() + (size_t)m * ctx->ntmax[w], ctx->ntmax[w]);
  return k;
}

int swdk_get_1d_kernel(swdk_ctx* ctx, int nx, int ny, int nz, const float* vs, const float* vp, const float* rho,
                       double* vc, double* vout, double* kernel, int32_t* status) {
  return run_host(ctx, 0, nx, ny, nz, vs, vp, rho, vc, vout, kernel, status);
}

int swdk_get_2d_map(swdk_ctx* ctx, int nx, int ny, int nz, const float* vs, const float* vp, const float* rho,
                    double* vc, double* vout, int32_t* status) {
  return run_host(ctx, 1, nx, ny, nz, vs, vp, rho, vc, vout, nullptr, status);
}

int swdk_get_1d_kernel_device(swdk_ctx* ctx, int nx, int ny, int nz, const float* d_vs, const float* d_vp,
                              const float* d_rho, double* d_vc, double* d_vout, double* d_kernel, int32_t* d_status,
                              void* stream) {
  if (!ctx) return SWDK_E_ARG;
  CK(cudaSetDevice(ctx->cfg.device));
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  return run_split(ctx, 0, nx, ny, nz, d_vs, d_vp, d_rho, d_vc, d_vout, d_kernel, d_status, st);
}

int swdk_get_2d_map_device(swdk_ctx* ctx, int nx, int ny, int nz, const float* d_vs, const float* d_vp,
                           const float* d_rho, double* d_vc, double* d_vout, int32_t* d_status, void* stream) {
  if (!ctx) return SWDK_E_ARG;
  CK(cudaSetDevice(ctx->cfg.device));
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  return run_split(ctx, 1, nx, ny, nz, d_vs, d_vp, d_rho, d_vc, d_vout, nullptr, d_status, st);
}

int swdk_surfdisp96_batch(swdk_ctx* ctx, int nmodel, int nlayer, const float* thk, const float* vp, const float* vs,
                          const float* rho, int iflsph, int iwave, int mode, int igr, int kmax, const double* t,
                          double* cg, int32_t* ierr) {
  if (!ctx || nmodel <= 0 || nlayer < 2 || !thk || !vp || !vs || !rho || !t || !cg || kmax <= 0 || mode < 1 ||
      (iwave != 1 && iwave != 2))
    return fail(ctx, SWDK_E_ARG, "bad arguments");
  if (nlayer > SWDK_MAX_LAYERS || kmax > SWDK_MAX_PERIODS) return fail(ctx, SWDK_E_LIMIT, "size beyond limits");
  CK(cudaSetDevice(ctx->cfg.device));
  cudaStream_t st = ctx->stream;
  const size_t nm = nmodel, nin = nm * nlayer;
  CK(ctx->in_misc.ensure(4 * nin * sizeof(float) + kmax * sizeof(double) + sizeof(ChainDesc)));
  float* d_in = ctx->in_misc.as<float>();
  double* d_t = (double*)(d_in + 4 * nin);
  ChainDesc* d_ch = (ChainDesc*)(d_t + kmax);
  CK(cudaMemcpyAsync(d_in, thk, nin * sizeof(float), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d_in + nin, vp, nin * sizeof(float), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d_in + 2 * nin, vs, nin * sizeof(float), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d_in + 3 * nin, rho, nin * sizeof(float), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d_t, t, kmax * sizeof(double), cudaMemcpyHostToDevice, st));
  ChainDesc cd;
  cd.t_off = 0; cd.np = kmax; cd.nmode = mode; cd.iwave = iwave; cd.igr = igr; cd.out_off = 0;
  CK(cudaMemcpyAsync(d_ch, &cd, sizeof(cd), cudaMemcpyHostToDevice, st));
  CK(ctx->layR.ensure(nin * sizeof(float4)));
  CK(ctx->layL.ensure(nin * sizeof(float4)));
  CK(ctx->info.ensure(nm * sizeof(ColInfo)));
  CK(ctx->croot.ensure((size_t)mode * kmax * nm * sizeof(double)));
  CK(ctx->cstat.ensure((size_t)mode * kmax * nm * sizeof(int32_t)));
  CK(ctx->ierr.ensure(nm * sizeof(int32_t)));
  CK(ctx->nevals.ensure(NCOUNT * sizeof(unsigned long long)));
  CK(cudaMemsetAsync(ctx->nevals.p, 0, NCOUNT * sizeof(unsigned long long), st));
  CK(cudaEventRecord(ctx->ev[0], st));
  k_prep_layers<<<(nmodel + 127) / 128, 128, 0, st>>>(nmodel, nlayer, d_in, d_in + nin, d_in + 2 * nin,
                                                       d_in + 3 * nin, iflsph, ctx->layR.as<float4>(),
                                                       ctx->layL.as<float4>(),
                                                       ctx->info.as<ColInfo>());
  CK(cudaGetLastError());
  CK(cudaEventRecord(ctx->ev[1], st));
  CK(cudaEventRecord(ctx->ev[5], st));
  ctx->stats.kernel_launches = 2;
  k_roots<<<dim3((nmodel + 127) / 128, 1), 128, 0, st>>>(nmodel, d_ch, d_t, ctx->layR.as<float4>(),
                                                         ctx->layL.as<float4>(), ctx->info.as<ColInfo>(),
                                                         ctx->cfg.refine, ctx->cfg.rtol, ctx->cfg.sngl, 0,
                                                         ctx->croot.as<double>(), ctx->cstat.as<int32_t>(),
                                                         ctx->ierr.as<int32_t>(),
                                                         ctx->nevals.as<unsigned long long>());
  CK(cudaGetLastError());
  CK(cudaEventRecord(ctx->ev[2], st));
  CK(cudaEventRecord(ctx->ev[3], st));
  // the reference's cg holds the last mode: rows (mode-1)*kmax .. of croot
  std::vector<double> tmp((size_t)kmax * nm);
  CK(cudaMemcpyAsync(tmp.data(), ctx->croot.as<double>() + (size_t)(mode - 1) * kmax * nm,
                     (size_t)kmax * nm * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (ierr) CK(cudaMemcpyAsync(ierr, ctx->ierr.p, nm * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(ctx->h_nevals, ctx->nevals.p, NCOUNT * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  CK(cudaEventRecord(ctx->ev[4], st));
  ctx->stats_pending = true;
  CK(cudaStreamSynchronize(st));
  for (size_t m = 0; m < nm; ++m)
    for (int k = 0; k < kmax; ++k) cg[m * kmax + k] = tmp[(size_t)k * nm + m];
  collect_stats(ctx);
  return SWDK_OK;
}

int swdk_frechet_rows_device(swdk_ctx* ctx, int nx, int ny, int nz, int kmax, const double* d_kernel, int nrows,
                             const int32_t* d_row_slot, const float* d_fdm, int32_t* d_nnz, int32_t* d_indices,
                             float* d_values, void* stream) {
  if (!ctx || nx < 3 || ny < 3 || nz < 2 || kmax <= 0 || nrows < 0 || !d_kernel || !d_row_slot || !d_fdm || !d_nnz ||
      !d_indices || !d_values)
    return fail(ctx, SWDK_E_ARG, "bad arguments");
  if (nrows == 0) return SWDK_OK;
  CK(cudaSetDevice(ctx->cfg.device));
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  k_frechet<<<nrows, 256, 0, st>>>(nx, ny, nz, kmax, d_kernel, d_row_slot, d_fdm, d_nnz, d_indices, d_values, nullptr,
                                   0);
  CK(cudaGetLastError());
  return SWDK_OK;
}

int swdk_frechet_csr_device(swdk_ctx* ctx, int nx, int ny, int nz, int kmax, const double* d_kernel, int nrows,
                            const int32_t* d_row_slot, const float* d_fdm, int64_t* d_rowptr, int32_t* d_indices,
                            float* d_values, int64_t capacity, int64_t* nnz_total, void* stream) {
  if (!ctx || nx < 3 || ny < 3 || nz < 2 || kmax <= 0 || nrows < 0 || !d_kernel || !d_row_slot || !d_fdm ||
      !d_rowptr || capacity < 0 || (capacity > 0 && (!d_indices || !d_values)))
    return fail(ctx, SWDK_E_ARG, "bad arguments");
  CK(cudaSetDevice(ctx->cfg.device));
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  if (nrows == 0) {
    CK(cudaMemsetAsync(d_rowptr, 0, sizeof(int64_t), st));
    if (nnz_total) *nnz_total = 0;
    return SWDK_OK;
  }
  CK(ctx->in_misc.ensure((size_t)nrows * sizeof(int32_t)));
  int32_t* cnt = ctx->in_misc.as<int32_t>();
  // pass 1: entries per row; prefix sum into the row pointer
  k_frechet<<<nrows, 256, 0, st>>>(nx, ny, nz, kmax, d_kernel, d_row_slot, d_fdm, cnt, nullptr, nullptr, nullptr, 1);
  CK(cudaGetLastError());
  k_rowptr<<<1, 1024, 0, st>>>(nrows, cnt, d_rowptr);
  CK(cudaGetLastError());
  int64_t total = 0;
  CK(cudaMemcpyAsync(&total, d_rowptr + nrows, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (nnz_total) *nnz_total = total;
  if (total > capacity) return fail(ctx, SWDK_E_LIMIT, "CSR capacity below the number of nonzeros");
  // pass 2: the rows, compacted
  k_frechet<<<nrows, 256, 0, st>>>(nx, ny, nz, kmax, d_kernel, d_row_slot, d_fdm, nullptr, d_indices, d_values,
                                   d_rowptr, 0);
  CK(cudaGetLastError());
  return SWDK_OK;
}

int swdk_set_proposal(swdk_ctx* ctx, swdk_mlp* rayleigh, swdk_mlp* love, double kappa_rayleigh, double kappa_love) {
  if (!ctx || !(kappa_rayleigh > 0.0) || !(kappa_rayleigh < 1.0e3) || !(kappa_love > 0.0) || !(kappa_love < 1.0e3))
    return fail(ctx, SWDK_E_ARG, "bad arguments");
  drop_graph(ctx);
  drop_kids(ctx);
  ctx->net[0] = rayleigh;
  ctx->net[1] = love;
  ctx->kappa[0] = kappa_rayleigh;
  ctx->kappa[1] = kappa_love;
  return SWDK_OK;
}

int swdk_set_proposal_shift(swdk_ctx* ctx, double shift_km_s) {
  if (!ctx || !(fabs(shift_km_s) <= 10.0)) return fail(ctx, SWDK_E_ARG, "bad arguments");
  drop_graph(ctx);
  drop_kids(ctx);
  ctx->prop_shift = shift_km_s;
  return SWDK_OK;
}

int swdk_roots_device(swdk_ctx* ctx, int nx, int ny, int nz, const float* d_vs, const float* d_vp, const float* d_rho,
                      void* stream) {
  if (!ctx) return SWDK_E_ARG;
  CK(cudaSetDevice(ctx->cfg.device));
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  return run_device(ctx, 2, nx, ny, nz, d_vs, d_vp, d_rho, nullptr, nullptr, nullptr, nullptr, st);
}

int swdk_root_slots(swdk_ctx* ctx, int* nslots, int32_t* wave, int32_t* mode, double* period) {
  if (!ctx || !nslots) return fail(ctx, SWDK_E_ARG, "bad arguments");
  int r = ensure_plans(ctx);
  if (r) return r;
  const Plan& P = ctx->plan[0];
  *nslots = P.nroot;
  for (int i = 0; i < P.nroot; ++i) {
    if (wave) wave[i] = P.rootwave[i];
    if (mode) mode[i] = P.rootmode[i];
    if (period) period[i] = P.rootperiod[i];
  }
  return SWDK_OK;
}

int swdk_last_roots(swdk_ctx* ctx, double* h_c, int32_t* h_status) {
  if (!ctx || ctx->last_ncol <= 0 || ctx->last_path < 0) return fail(ctx, SWDK_E_ARG, "no root search ran yet");
  if (ctx->last_split) return fail(ctx, SWDK_E_ARG, "the last call ran as column halves: use swdk_roots_device");
  CK(cudaSetDevice(ctx->cfg.device));
  const Plan& P = ctx->plan[ctx->last_path == 1 ? 1 : 0];
  const size_t n = (size_t)P.nroot * ctx->last_ncol;
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaDeviceSynchronize());
  if (h_c) CK(cudaMemcpy(h_c, ctx->croot.p, n * sizeof(double), cudaMemcpyDeviceToHost));
  if (h_status) CK(cudaMemcpy(h_status, ctx->cstat.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
  return SWDK_OK;
}

int swdk_training_rows(swdk_ctx* ctx, const int64_t* d_rows, int n, void* d_x, float* d_y, void* stream) {
  if (!ctx || n < 0 || (n > 0 && (!d_rows || !d_x))) return fail(ctx, SWDK_E_ARG, "bad arguments");
  if (ctx->last_path != 2) return fail(ctx, SWDK_E_ARG, "swdk_training_rows needs a preceding swdk_roots_device");
  if (n == 0) return SWDK_OK;
  CK(cudaSetDevice(ctx->cfg.device));
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  const Plan& P = ctx->plan[0];
  const int64_t rowmax = (int64_t)P.nroot * ctx->last_ncol;
  k_features<<<(n + 15) / 16, 256, 0, st>>>(0, n, ctx->last_ncol, rowmax, P.d_rootfeat.as<float4>(),
                                          ctx->nodefeat.as<float4>(), d_rows, (__nv_bfloat16*)d_x, 0);
  CK(cudaGetLastError());
  if (d_y) {
    k_targets<<<(n + 255) / 256, 256, 0, st>>>(n, rowmax, d_rows, ctx->croot.as<double>(), d_y);
    CK(cudaGetLastError());
  }
  return SWDK_OK;
}

int swdk_graph_capture(swdk_ctx* ctx, int path, int nx, int ny, int nz, const float* d_vs, const float* d_vp,
                       const float* d_rho, double* d_vc, double* d_vout, double* d_kernel, int32_t* d_status) {
  if (!ctx || path < 0 || path > 2) return fail(ctx, SWDK_E_ARG, "bad arguments");
  CK(cudaSetDevice(ctx->cfg.device));
  drop_graph(ctx);
  cudaStream_t st = ctx->stream;
  // one eager call sizes every buffer, builds the plans, uploads the depth
  // vector and prepares the proposal networks, so the captured call
  // allocates nothing and copies nothing from pageable memory
  int r = run_split(ctx, path, nx, ny, nz, d_vs, d_vp, d_rho, d_vc, d_vout, d_kernel, d_status, st);
  if (r) return r;
  CK(cudaStreamSynchronize(st));
  collect_stats(ctx);
  CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  ctx->capturing = true;
  r = run_split(ctx, path, nx, ny, nz, d_vs, d_vp, d_rho, d_vc, d_vout, d_kernel, d_status, st);
  ctx->capturing = false;
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(st, &g);
  if (r) {
    if (g) cudaGraphDestroy(g);
    return r;
  }
  if (e != cudaSuccess) return fail(ctx, SWDK_E_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
  ctx->graph = g;
  CK(cudaGraphInstantiate(&ctx->gexec, g, 0));
  return SWDK_OK;
}

struct swdk_graph {
  int device = 0;
  cudaStream_t main = nullptr;
  std::vector<cudaEvent_t> events;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

void swdk_batch_graph_destroy(swdk_graph* g) {
  if (!g) return;
  cudaSetDevice(g->device);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  for (cudaEvent_t e : g->events)
    if (e) cudaEventDestroy(e);
  if (g->main) cudaStreamDestroy(g->main);
  delete g;
}

int swdk_batch_graph_create(int n, swdk_ctx* const* ctxs, const swdk_call* calls, swdk_graph** out) {
  if (!out || n <= 0 || !ctxs || !calls) return SWDK_E_ARG;
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    if (!ctxs[i] || calls[i].path < 0 || calls[i].path > 2 || ctxs[i]->cfg.device != ctxs[0]->cfg.device)
      return SWDK_E_ARG;
    for (int j = 0; j < i; ++j)
      if (ctxs[j] == ctxs[i]) return fail(ctxs[i], SWDK_E_ARG, "a context appears twice in one batch graph");
  }
  swdk_graph* g = new swdk_graph();
  g->device = ctxs[0]->cfg.device;
  auto bail = [&](swdk_ctx* c, int code, const std::string& msg) {
    swdk_batch_graph_destroy(g);
    return fail(c, code, msg);
  };
  swdk_ctx* ctx = ctxs[0];  // for CK's error text
  cudaError_t e = cudaSetDevice(g->device);
  if (e != cudaSuccess) return bail(ctx, SWDK_E_CUDA, cudaGetErrorString(e));
  // eager pass: every context sizes its buffers, builds its plans, uploads
  // its depth vector and prepares its proposal networks
  for (int i = 0; i < n; ++i) {
    const swdk_call& c = calls[i];
    drop_graph(ctxs[i]);
    const int r = run_device(ctxs[i], c.path, c.nx, c.ny, c.nz, c.d_vs, c.d_vp, c.d_rho, c.d_vc, c.d_vout, c.d_kernel,
                             c.d_status, ctxs[i]->stream);
    if (r) { swdk_batch_graph_destroy(g); return r; }
  }
  for (int i = 0; i < n; ++i) {
    e = cudaStreamSynchronize(ctxs[i]->stream);
    if (e != cudaSuccess) return bail(ctxs[i], SWDK_E_CUDA, cudaGetErrorString(e));
    collect_stats(ctxs[i]);
  }
  // capture: fork every context's stream off one main stream, join them back
  e = cudaStreamCreateWithFlags(&g->main, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bail(ctx, SWDK_E_CUDA, cudaGetErrorString(e));
  g->events.assign(n + 1, nullptr);
  for (int i = 0; i <= n && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&g->events[i], cudaEventDisableTiming);
  if (e != cudaSuccess) return bail(ctx, SWDK_E_CUDA, cudaGetErrorString(e));
  e = cudaStreamBeginCapture(g->main, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return bail(ctx, SWDK_E_CUDA, cudaGetErrorString(e));
  int r = SWDK_OK;
  e = cudaEventRecord(g->events[n], g->main);
  for (int i = 0; i < n && e == cudaSuccess && r == SWDK_OK; ++i) {
    const swdk_call& c = calls[i];
    e = cudaStreamWaitEvent(ctxs[i]->stream, g->events[n], 0);
    if (e != cudaSuccess) break;
    ctxs[i]->capturing = true;
    r = run_device(ctxs[i], c.path, c.nx, c.ny, c.nz, c.d_vs, c.d_vp, c.d_rho, c.d_vc, c.d_vout, c.d_kernel, c.d_status,
                   ctxs[i]->stream);
    ctxs[i]->capturing = false;
    if (r) break;
    e = cudaEventRecord(g->events[i], ctxs[i]->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(g->main, g->events[i], 0);
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(g->main, &graph);
  g->graph = graph;
  if (r) { swdk_batch_graph_destroy(g); return r; }
  if (e != cudaSuccess) return bail(ctx, SWDK_E_CUDA, std::string("batch capture: ") + cudaGetErrorString(e));
  if (e2 != cudaSuccess) return bail(ctx, SWDK_E_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e2));
  e = cudaGraphInstantiate(&g->exec, graph, 0);
  if (e != cudaSuccess) return bail(ctx, SWDK_E_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
  *out = g;
  return SWDK_OK;
}

int swdk_batch_graph_launch(swdk_graph* g, void* stream) {
  if (!g || !g->exec) return SWDK_E_ARG;
  if (cudaSetDevice(g->device) != cudaSuccess) return SWDK_E_CUDA;
  return cudaGraphLaunch(g->exec, stream ? (cudaStream_t)stream : g->main) == cudaSuccess ? SWDK_OK : SWDK_E_CUDA;
}

// ---------------------------------------------------------------------------
// Ragged batches (swdk_ragged_*): every model's column preparation, then ONE
// persistent root-search launch over all (model, chain, column) items, one
// retry launch and one eigen launch per wave type over all (model, column)
// blocks; each model's arrays at offsets in shared buffers, its plans
// (chains, periods, slots) concatenated.
// ---------------------------------------------------------------------------
struct swdk_ragged {
  int device = 0, n = 0, path = 0;
  std::vector<swdk_ctx*> ctx;
  std::vector<swdk_call> calls;
  std::vector<RModel> models;
  std::vector<RBlock> blocks;
  std::vector<REBlock> eb[4];
  long long eblocks[4] = {0, 0, 0, 0};
  int et[4] = {0, 0, 0, 0};
  std::vector<ChainDesc> chains;
  std::vector<double> periods;
  std::vector<SlotDesc> slots;
  long long nitems = 0, ncol_tot = 0, lay_tot = 0, crs_tot = 0, root_tot = 0, slots_tot = 0;
  int maxL = 0, maxnz = 0, roots_blocks = 0;
  bool useprop = false;
  DevBuf d_models, d_blocks, d_eb[4], d_chains, d_periods, d_slots;
  DevBuf layR, layL, lay0, info, chainrule, croot, cstat, prop, nodefeat, retry_list, retry_ctr, queue, nevals;
  DevBuf nodes, dltab;
  long long node_tot = 0, dl_tot = 0;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  unsigned long long* h_nevals = nullptr;
  bool stats_pending = false;
  swdk_stats stats;
  int launches = 0;
};

namespace {

// the kernels of one pass over a ragged batch, enqueued on st; timing
// events and the statistics copy only when not capturing
int ragged_enqueue(swdk_ragged* R, cudaStream_t st, bool timing) {
  swdk_ctx* ctx = R->ctx[0];
  const swdk_config& cfg = ctx->cfg;
  CK(cudaMemsetAsync(R->nevals.p, 0, NCOUNT * sizeof(unsigned long long), st));
  CK(cudaMemsetAsync(R->queue.p, 0, sizeof(unsigned int), st));
  CK(cudaMemsetAsync(R->retry_ctr.p, 0, 2 * sizeof(unsigned int), st));
  if (timing) CK(cudaEventRecord(R->ev[0], st));
  R->launches = 0;
  const bool use_nodes = cfg.node_layers != 0;
  for (int i = 0; i < R->n; ++i) {
    const RModel& M = R->models[i];
    const swdk_call& c = R->calls[i];
    if (use_nodes) {
      R->launches += 1;
      k_depth_table<<<1, 32, 0, st>>>(M.nz, R->ctx[i]->depth_d.as<float>(), cfg.sphere,
                                      R->dltab.as<DepthLayer>() + M.dl0);
      CK(cudaGetLastError());
    }
    R->launches += 1;
    k_prep<<<(M.ncol + 127) / 128, 128, 0, st>>>(
        M.ncol, M.ncol, M.nz, c.d_vs, c.d_vp, c.d_rho, R->ctx[i]->depth_d.as<float>(), cfg.sphere, M.Lmax,
        R->layR.as<float4>() + M.lay0, R->layL.as<float4>() + M.lay0, R->lay0.as<float4>() + M.lay0,
        R->info.as<ColInfo>() + M.col0, R->chainrule.as<float2>() + M.crs0,
        R->useprop ? R->nodefeat.as<float4>() + M.col0 * FEAT_NODES : nullptr,
        use_nodes ? R->nodes.as<float4>() + M.node0 : nullptr);
    CK(cudaGetLastError());
  }
  if (timing) CK(cudaEventRecord(R->ev[1], st));
  if (R->useprop) {
    for (int i = 0; i < R->n; ++i) {
      swdk_ctx* c = R->ctx[i];
      const RModel& M = R->models[i];
      const Plan& P = c->plan[R->path];
      float2* dst = R->prop.as<float2>() + M.root0;
      if (!proposals_on(c)) {
        CK(cudaMemsetAsync(dst, 0, (size_t)P.nroot * M.ncol * sizeof(float2), st));
        continue;
      }
      c->launches = 0;
      const int r = run_proposals(c, P, M.ncol, st, R->nodefeat.as<float4>() + M.col0 * FEAT_NODES, dst);
      if (r) return fail(ctx, r, "ragged proposals: " + c->err);
      R->launches += c->launches;
    }
  }
  if (timing) CK(cudaEventRecord(R->ev[5], st));
  const RaggedMap rg{R->d_blocks.as<RBlock>(), R->d_models.as<RModel>(), (int)R->blocks.size(), 0};
  const unsigned int rcap = (unsigned int)std::min<long long>(R->root_tot, 0x7fffffffLL);
  unsigned int* rctr = R->retry_ctr.as<unsigned int>();
  const long long grid = std::min<long long>(R->roots_blocks, (R->nitems + 127) / 128);
  R->launches += 2;
  k_roots_queue<<<(unsigned)std::max(1LL, grid), 128, ROOTS_SMEM, st>>>(
      0, (int)R->nitems, nullptr, R->d_chains.as<ChainDesc>(), R->d_periods.as<double>(), R->layR.as<float4>(),
      R->layL.as<float4>(), R->info.as<ColInfo>(), cfg.refine, cfg.rtol, cfg.sngl, RETRY_DEFERRED,
      R->croot.as<double>(), R->cstat.as<int32_t>(), R->queue.as<unsigned int>(),
      R->useprop ? R->prop.as<float2>() : nullptr, R->retry_list.as<int2>(), rctr, rcap,
      R->nevals.as<unsigned long long>(), rg, use_nodes ? R->nodes.as<float4>() : nullptr,
      R->dltab.as<DepthLayer>());
  CK(cudaGetLastError());
  k_retry<<<R->roots_blocks, 128, ROOTS_SMEM, st>>>(0, nullptr, R->d_chains.as<ChainDesc>(), R->d_periods.as<double>(),
                                           R->layR.as<float4>(), R->layL.as<float4>(), R->info.as<ColInfo>(),
                                           cfg.refine, cfg.rtol, cfg.sngl, R->croot.as<double>(),
                                           R->cstat.as<int32_t>(), R->retry_list.as<int2>(), rctr, rcap, rctr + 1,
                                           R->nevals.as<unsigned long long>(), rg,
                                           use_nodes ? R->nodes.as<float4>() : nullptr, R->dltab.as<DepthLayer>());
  CK(cudaGetLastError());
  if (timing) CK(cudaEventRecord(R->ev[2], st));
  if (R->path != 2) {
    using EigR = void (*)(const REBlock*, int, const RModel*, const float4*, const ColInfo*, const float2*,
                          const SlotDesc*, const double*, const int32_t*, int);
    static const EigR eig[4][2] = {{k_eigen_ragged<0, 0>, k_eigen_ragged<0, 1>},
                                   {k_eigen_ragged<1, 0>, k_eigen_ragged<1, 1>},
                                   {k_eigen_ragged<2, 0>, k_eigen_ragged<2, 1>},
                                   {k_eigen_ragged<3, 0>, k_eigen_ragged<3, 1>}};
    for (int wt = 0; wt < 4; ++wt) {
      if (R->eb[wt].empty()) continue;
      const size_t smem = (size_t)R->maxL * (wt >= 2 ? sizeof(LoveLayer) : sizeof(RayLayer)) +
                          (size_t)R->maxnz * sizeof(float2);
      R->launches += 1;
      eig[wt][R->path]<<<(unsigned)R->eblocks[wt], R->et[wt], smem, st>>>(
          R->d_eb[wt].as<REBlock>(), (int)R->eb[wt].size(), R->d_models.as<RModel>(), R->lay0.as<float4>(),
          R->info.as<ColInfo>(), R->chainrule.as<float2>(), R->d_slots.as<SlotDesc>(), R->croot.as<double>(),
          R->cstat.as<int32_t>(), cfg.sphere);
      CK(cudaGetLastError());
    }
  }
  if (timing) {
    CK(cudaEventRecord(R->ev[3], st));
    CK(cudaMemcpyAsync(R->h_nevals, R->nevals.p, NCOUNT * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    CK(cudaEventRecord(R->ev[4], st));
    R->stats_pending = true;
  }
  return SWDK_OK;
}

void ragged_collect(swdk_ragged* R) {
  if (!R->stats_pending) return;
  cudaEventSynchronize(R->ev[4]);
  R->stats_pending = false;
  swdk_stats& t = R->stats;
  memset(&t, 0, sizeof(t));
  t.secular_evals = (int64_t)R->h_nevals[0];
  t.layer_evals_rayleigh = (int64_t)R->h_nevals[1];
  t.layer_evals_love = (int64_t)R->h_nevals[2];
  t.proposals_accepted = (int64_t)R->h_nevals[3];
  t.proposals_rejected = (int64_t)R->h_nevals[4];
  for (int i = 0; i < NPHASE_EV; ++i) t.evals_by_phase[i] = (int64_t)R->h_nevals[EV_BASE + i];
  t.nchains = (int)R->chains.size();
  t.nslots = (int)R->slots_tot;
  t.kernel_launches = R->launches;
  cudaEventElapsedTime(&t.ms_prep, R->ev[0], R->ev[1]);
  cudaEventElapsedTime(&t.ms_proposal, R->ev[1], R->ev[5]);
  cudaEventElapsedTime(&t.ms_roots, R->ev[5], R->ev[2]);
  cudaEventElapsedTime(&t.ms_eigen, R->ev[2], R->ev[3]);
}

}  // namespace

void swdk_ragged_destroy(swdk_ragged* R) {
  if (!R) return;
  cudaSetDevice(R->device);
  if (R->stream) cudaStreamSynchronize(R->stream);
  if (R->exec) cudaGraphExecDestroy(R->exec);
  if (R->graph) cudaGraphDestroy(R->graph);
  DevBuf* bufs[] = {&R->d_models, &R->d_blocks, &R->d_eb[0], &R->d_eb[1], &R->d_eb[2], &R->d_eb[3], &R->d_chains,
                    &R->d_periods, &R->d_slots, &R->layR, &R->layL, &R->lay0, &R->info, &R->chainrule, &R->croot,
                    &R->cstat, &R->prop, &R->nodefeat, &R->retry_list, &R->retry_ctr, &R->queue, &R->nevals,
                    &R->nodes, &R->dltab};
  for (DevBuf* b : bufs) b->release();
  for (cudaEvent_t& e : R->ev)
    if (e) cudaEventDestroy(e);
  if (R->h_nevals) cudaFreeHost(R->h_nevals);
  if (R->stream) cudaStreamDestroy(R->stream);
  delete R;
}

int swdk_ragged_create(int n, swdk_ctx* const* ctxs, const swdk_call* calls, swdk_ragged** out) {
  if (!out || n <= 0 || !ctxs || !calls) return SWDK_E_ARG;
  *out = nullptr;
  swdk_ctx* ctx = ctxs[0];
  if (!ctx) return SWDK_E_ARG;
  const int path = calls[0].path;
  if (path < 0 || path > 2) return fail(ctx, SWDK_E_ARG, "bad path");
  for (int i = 0; i < n; ++i) {
    const swdk_ctx* c = ctxs[i];
    const swdk_call& k = calls[i];
    if (!c || k.path != path || c->cfg.device != ctx->cfg.device || c->cfg.refine != ctx->cfg.refine ||
        c->cfg.rtol != ctx->cfg.rtol || c->cfg.sngl != ctx->cfg.sngl || c->cfg.sphere != ctx->cfg.sphere ||
        c->cfg.node_layers != ctx->cfg.node_layers)
      return fail(ctx, SWDK_E_ARG, "ragged batch: every model needs the same path, device and root settings");
    if (k.nx <= 0 || k.ny <= 0 || !k.d_vs || (path != 2 && (!k.d_vc || !k.d_vout || (path == 0 && !k.d_kernel))))
      return fail(ctx, SWDK_E_ARG, "ragged batch: bad call arguments");
    if ((k.d_vp == nullptr) != (k.d_rho == nullptr)) return fail(ctx, SWDK_E_ARG, "vp and rho must both be given");
    if ((int)c->depth.size() != k.nz) return fail(ctx, SWDK_E_NODEPTH, "nz does not match swdk_set_depth");
    if (k.nz < 2 || k.nz > SWDK_MAX_NZ || 4 * k.nz - 3 > SWDK_MAX_LAYERS) return fail(ctx, SWDK_E_LIMIT, "nz out of range");
  }
  CK(cudaSetDevice(ctx->cfg.device));
  swdk_ragged* R = new swdk_ragged();
  memset(&R->stats, 0, sizeof(R->stats));
  R->device = ctx->cfg.device;
  R->n = n;
  R->path = path;
  R->ctx.assign(ctxs, ctxs + n);
  R->calls.assign(calls, calls + n);
  auto bail = [&](int code, const std::string& msg) {
    swdk_ragged_destroy(R);
    return fail(ctx, code, msg);
  };
  const int ppath = (path == 2) ? 0 : path;
  std::vector<int> chain0(n), slot0(n);
  for (int i = 0; i < n; ++i) {
    swdk_ctx* c = ctxs[i];
    const int r = ensure_plans(c);
    if (r) { swdk_ragged_destroy(R); return r; }
    const Plan& P = c->plan[ppath];
    const swdk_call& k = calls[i];
    RModel M;
    M.ncol = k.nx * k.ny;
    M.nz = k.nz;
    M.Lmax = 4 * k.nz - 3;
    M.pad_ = 0;
    M.col0 = R->ncol_tot;
    M.lay0 = R->lay_tot;
    M.crs0 = R->crs_tot;
    M.root0 = R->root_tot;
    M.node0 = R->node_tot;
    M.dl0 = R->dl_tot;
    M.vc = k.d_vc;
    M.vout = k.d_vout;
    M.kernel = k.d_kernel;
    M.status = k.d_status;
    R->models.push_back(M);
    R->ncol_tot += M.ncol;
    R->lay_tot += (long long)M.Lmax * M.ncol;
    R->crs_tot += (long long)M.nz * M.ncol;
    R->root_tot += (long long)P.nroot * M.ncol;
    R->node_tot += (long long)M.nz * M.ncol;
    R->dl_tot += M.Lmax;
    R->slots_tot += (long long)P.kmax;
    R->maxL = std::max(R->maxL, M.Lmax);
    R->maxnz = std::max(R->maxnz, M.nz);
    chain0[i] = (int)R->chains.size();
    for (ChainDesc d : P.chains) {
      d.t_off += (int)R->periods.size();
      R->chains.push_back(d);
    }
    R->periods.insert(R->periods.end(), P.periods.begin(), P.periods.end());
    slot0[i] = (int)R->slots.size();
    R->slots.insert(R->slots.end(), P.slots.begin(), P.slots.end());
    for (int g = 0; g < P.groups.n; ++g) {
      const int wt = P.slots[P.groups.start[g]].wtype;
      REBlock E;
      E.blk0 = R->eblocks[wt];
      E.model = i;
      E.g0 = slot0[i] + P.groups.start[g];
      E.gn = P.groups.count[g];
      E.pad_ = 0;
      R->eb[wt].push_back(E);
      R->eblocks[wt] += M.ncol;
      R->et[wt] = std::max(R->et[wt], std::min(128, ((E.gn + 31) / 32) * 32));
    }
    if (proposals_on(c)) R->useprop = true;
    // the model's depth vector on the device (k_prep reads it)
    CK(c->depth_d.ensure((size_t)k.nz * sizeof(float)));
    if (c->depth_dev != c->depth_d.p) {
      CK(cudaMemcpy(c->depth_d.p, c->depth.data(), k.nz * sizeof(float), cudaMemcpyHostToDevice));
      c->depth_dev = c->depth_d.p;
    }
  }
  // root work blocks: every model's Rayleigh chains, then the Love chains,
  // model by model, so the items in flight share a few models' node arrays
  // in L2 (ordering the blocks by cost across models instead measured 4 %
  // slower on the 48-model batch)
  for (int w = 2; w >= 1; --w)
    for (int i = 0; i < n; ++i) {
      const Plan& P = ctxs[i]->plan[ppath];
      for (int ci : P.order) {
        if (P.chains[ci].iwave != w) continue;
        RBlock B;
        B.item0 = R->nitems;
        B.model = i;
        B.chain = chain0[i] + ci;
        R->blocks.push_back(B);
        R->nitems += R->models[i].ncol;
      }
    }
  if (R->nitems >= 0x7fffffffLL) return bail(SWDK_E_LIMIT, "ragged batch: too many work items");
  auto up = [&](DevBuf& b, const void* src, size_t bytes) -> cudaError_t {
    cudaError_t e = b.ensure(std::max<size_t>(bytes, 16));
    if (e == cudaSuccess && bytes) e = cudaMemcpy(b.p, src, bytes, cudaMemcpyHostToDevice);
    return e;
  };
  cudaError_t e = up(R->d_models, R->models.data(), R->models.size() * sizeof(RModel));
  if (e == cudaSuccess) e = up(R->d_blocks, R->blocks.data(), R->blocks.size() * sizeof(RBlock));
  for (int wt = 0; wt < 4 && e == cudaSuccess; ++wt) e = up(R->d_eb[wt], R->eb[wt].data(), R->eb[wt].size() * sizeof(REBlock));
  if (e == cudaSuccess) e = up(R->d_chains, R->chains.data(), R->chains.size() * sizeof(ChainDesc));
  if (e == cudaSuccess) e = up(R->d_periods, R->periods.data(), R->periods.size() * sizeof(double));
  if (e == cudaSuccess) e = up(R->d_slots, R->slots.data(), R->slots.size() * sizeof(SlotDesc));
  if (e == cudaSuccess) e = R->layR.ensure((size_t)R->lay_tot * sizeof(float4));
  if (e == cudaSuccess) e = R->layL.ensure((size_t)R->lay_tot * sizeof(float4));
  if (e == cudaSuccess) e = R->lay0.ensure((size_t)R->lay_tot * sizeof(float4));
  if (e == cudaSuccess) e = R->info.ensure((size_t)R->ncol_tot * sizeof(ColInfo));
  if (e == cudaSuccess) e = R->chainrule.ensure((size_t)R->crs_tot * sizeof(float2));
  if (e == cudaSuccess) e = R->nodes.ensure((size_t)R->node_tot * sizeof(float4));
  if (e == cudaSuccess) e = R->dltab.ensure((size_t)R->dl_tot * sizeof(DepthLayer));
  if (e == cudaSuccess) e = R->croot.ensure((size_t)R->root_tot * sizeof(double));
  if (e == cudaSuccess) e = R->cstat.ensure((size_t)R->root_tot * sizeof(int32_t));
  if (e == cudaSuccess && R->useprop) e = R->prop.ensure((size_t)R->root_tot * sizeof(float2));
  if (e == cudaSuccess && R->useprop) e = R->nodefeat.ensure((size_t)R->ncol_tot * FEAT_NODES * sizeof(float4));
  if (e == cudaSuccess) e = R->retry_list.ensure((size_t)std::min<long long>(R->root_tot, 0x7fffffffLL) * sizeof(int2));
  if (e == cudaSuccess) e = R->retry_ctr.ensure(2 * sizeof(unsigned int));
  if (e == cudaSuccess) e = R->queue.ensure(sizeof(unsigned int));
  if (e == cudaSuccess) e = R->nevals.ensure(NCOUNT * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&R->stream, cudaStreamNonBlocking);
  for (int i = 0; i < 6 && e == cudaSuccess; ++i) e = cudaEventCreate(&R->ev[i]);
  if (e == cudaSuccess) e = cudaMallocHost((void**)&R->h_nevals, NCOUNT * sizeof(unsigned long long));
  if (e != cudaSuccess) return bail(SWDK_E_CUDA, std::string("ragged batch set-up: ") + cudaGetErrorString(e));
  int dev = 0, nsm = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = roots_occupancy(&per);
  if (e != cudaSuccess) return bail(SWDK_E_CUDA, std::string("ragged batch set-up: ") + cudaGetErrorString(e));
  R->roots_blocks = ctx->cfg.block_roots > 0 ? ctx->cfg.block_roots : std::max(1, nsm * std::max(1, per));
  *out = R;
  return SWDK_OK;
}

int swdk_ragged_run(swdk_ragged* R, void* stream) {
  if (!R) return SWDK_E_ARG;
  swdk_ctx* ctx = R->ctx[0];
  CK(cudaSetDevice(R->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : R->stream;
  const int r = ragged_enqueue(R, st, true);
  if (r) return r;
  if (!stream) {
    CK(cudaStreamSynchronize(st));
    ragged_collect(R);
  }
  return SWDK_OK;
}

int swdk_ragged_launch(swdk_ragged* R, void* stream) {
  if (!R) return SWDK_E_ARG;
  swdk_ctx* ctx = R->ctx[0];
  CK(cudaSetDevice(R->device));
  if (!R->exec) {
    // one eager pass first (sizes the proposal scratch of every context),
    // then the same work captured as one graph
    int r = ragged_enqueue(R, R->stream, true);
    if (r) return r;
    CK(cudaStreamSynchronize(R->stream));
    ragged_collect(R);
    CK(cudaStreamBeginCapture(R->stream, cudaStreamCaptureModeThreadLocal));
    r = ragged_enqueue(R, R->stream, false);
    cudaGraph_t g = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(R->stream, &g);
    if (r) {
      if (g) cudaGraphDestroy(g);
      return r;
    }
    if (e2 != cudaSuccess) return fail(ctx, SWDK_E_CUDA, std::string("ragged capture: ") + cudaGetErrorString(e2));
    R->graph = g;
    CK(cudaGraphInstantiate(&R->exec, g, 0));
  }
  CK(cudaGraphLaunch(R->exec, stream ? (cudaStream_t)stream : R->stream));
  return SWDK_OK;
}

int swdk_ragged_stats(swdk_ragged* R, swdk_stats* out) {
  if (!R || !out) return SWDK_E_ARG;
  ragged_collect(R);
  *out = R->stats;
  return SWDK_OK;
}

int swdk_graph_launch(swdk_ctx* ctx, void* stream) {
  if (!ctx || !ctx->gexec) return fail(ctx, SWDK_E_ARG, "no captured graph");
  CK(cudaSetDevice(ctx->cfg.device));
  CK(cudaGraphLaunch(ctx->gexec, stream ? (cudaStream_t)stream : ctx->stream));
  return SWDK_OK;
}

int swdk_autotune(swdk_ctx* ctx, int nx, int ny, int nz, const float* d_vs, const float* d_vp, const float* d_rho,
                  int* blocks_out) {
  if (!ctx) return SWDK_E_ARG;
  CK(cudaSetDevice(ctx->cfg.device));
  drop_graph(ctx);
  cudaStream_t st = ctx->stream;
  int dev = 0, nsm = 0, per = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  CK(roots_occupancy(&per));
  per = std::max(1, per);
  // candidates: resident blocks of the persistent root kernel, 1..per per SM
  // plus one oversubscribed grid (queue items then also spread over waves)
  std::vector<int> cand;
  for (int k = 1; k <= per; ++k) cand.push_back(k * nsm);
  cand.push_back(2 * per * nsm);
  const int saved = ctx->cfg.block_roots;
  int best = 0;
  float best_ms = 1e30f;
  // warm-up (plans, buffers), then each candidate timed on its own call
  ctx->cfg.block_roots = cand.back();
  int r = run_device(ctx, 2, nx, ny, nz, d_vs, d_vp, d_rho, nullptr, nullptr, nullptr, nullptr, st);
  if (r) { ctx->cfg.block_roots = saved; return r; }
  CK(cudaStreamSynchronize(st));
  collect_stats(ctx);
  for (int b : cand) {
    ctx->cfg.block_roots = b;
    r = run_device(ctx, 2, nx, ny, nz, d_vs, d_vp, d_rho, nullptr, nullptr, nullptr, nullptr, st);
    if (r) { ctx->cfg.block_roots = saved; return r; }
    CK(cudaStreamSynchronize(st));
    collect_stats(ctx);
    const float ms = ctx->stats.ms_roots;
    if (ms < best_ms) { best_ms = ms; best = b; }
  }
  ctx->cfg.block_roots = best;
  drop_kids(ctx);  // the column halves are recreated with the tuned grid
  if (blocks_out) *blocks_out = best;
  return SWDK_OK;
}

int swdk_recip_device(const double* d_x, double* d_r, int n, void* stream) {
  if (n < 0 || (n > 0 && (!d_x || !d_r))) return SWDK_E_ARG;
  if (n == 0) return SWDK_OK;
  k_recip<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(n, d_x, d_r);
  return cudaGetLastError() == cudaSuccess ? SWDK_OK : SWDK_E_CUDA;
}

int swdk_frechet_records_device(int64_t m, int32_t m_header, int32_t n, const int32_t* d_row_ids, int32_t row_id0,
                                const int64_t* d_rowptr, const int32_t* d_indices, const float* d_values,
                                int64_t nnz_total, int32_t* d_out, int64_t out_words, void* stream) {
  if (m < 0 || nnz_total < 0 || !d_out || (m > 0 && (!d_rowptr || (nnz_total > 0 && (!d_indices || !d_values)))))
    return SWDK_E_ARG;
  if (out_words < 2 + 2 * m + 2 * nnz_total) return SWDK_E_LIMIT;
  const int64_t blocks = std::max<int64_t>(1, (m + 7) / 8);  // 8 rows (warps) per block of 256
  if (blocks > 0x7fffffff) return SWDK_E_LIMIT;
  k_frechet_records<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(m, m_header, n, d_row_ids, row_id0, d_rowptr,
                                                                          d_indices, d_values, d_out);
  return cudaGetLastError() == cudaSuccess ? SWDK_OK : SWDK_E_CUDA;
}

int swdk_aprod_csr(int mode, int64_t m, int64_t n, const int64_t* d_rowptr, const int32_t* d_indices,
                   const float* d_values, double* d_x, double* d_y, void* stream) {
  if ((mode != 1 && mode != 2) || m < 0 || n < 0 || (m > 0 && (!d_rowptr || !d_x || !d_y))) return SWDK_E_ARG;
  if (m == 0) return SWDK_OK;
  const int64_t blocks = (m + 7) / 8;  // 8 rows (warps) per block of 256
  if (blocks > 0x7fffffff) return SWDK_E_LIMIT;
  cudaStream_t st = (cudaStream_t)stream;
  if (mode == 1) k_aprod1<<<(unsigned)blocks, 256, 0, st>>>(m, d_rowptr, d_indices, d_values, d_x, d_y);
  else k_aprod2<<<(unsigned)blocks, 256, 0, st>>>(m, d_rowptr, d_indices, d_values, d_x, d_y);
  return cudaGetLastError() == cudaSuccess ? SWDK_OK : SWDK_E_CUDA;
}

int swdk_get_stats(swdk_ctx* ctx, swdk_stats* out) {
  if (!ctx || !out) return SWDK_E_ARG;
  collect_stats(ctx);  // waits for the last call's completion event
  *out = ctx->stats;
  return SWDK_OK;
}

const char* swdk_last_error(const swdk_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int swdk_surfdisp96_noalloc(int device, int nmodel, int nlayer, const float* d_thk, const float* d_vp,
                            const float* d_vs, const float* d_rho, int iflsph, int iwave, int mode, int igr, int kmax,
                            const double* d_t, double* d_cg, int32_t* d_ierr, int refine, double rtol, int sngl,
                            void* stream) {
  if (nmodel <= 0 || nlayer < 2 || kmax <= 0 || mode < 1 || (iwave != 1 && iwave != 2) || !d_thk || !d_vp ||
      !d_vs || !d_rho || !d_t || !d_cg || !d_ierr || device < 0 || device >= 256)
    return SWDK_E_ARG;
  if (nlayer > SWDK_MAX_LAYERS || kmax > SWDK_MAX_PERIODS) return SWDK_E_LIMIT;
  // scratch layout: layR | layL | info | croot | cstat, each 256-byte aligned
  const size_t nm = (size_t)nmodel, nin = nm * nlayer, nroot = (size_t)mode * kmax * nm;
  const size_t o_layR = 0;
  const size_t o_layL = align256(o_layR + nin * sizeof(float4));
  const size_t o_info = align256(o_layL + nin * sizeof(float4));
  const size_t o_croot = align256(o_info + nm * sizeof(ColInfo));
  const size_t o_cstat = align256(o_croot + nroot * sizeof(double));
  const size_t need = align256(o_cstat + nroot * sizeof(int32_t));
  if (need > SWDK_NOALLOC_SCRATCH_BYTES) return SWDK_E_LIMIT;
  // an error the caller's thread left pending is the caller's: report it
  // without clearing it, and launch nothing
  if (cudaPeekAtLastError() != cudaSuccess) return SWDK_E_CUDA;
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return SWDK_E_CUDA;
  if (prev != device && cudaSetDevice(device) != cudaSuccess) return SWDK_E_CUDA;
  int rc = SWDK_OK;
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) rc = SWDK_E_CUDA;
      else g_noalloc_ptr[device] = p;
    }
    base = (unsigned char*)g_noalloc_ptr[device];
  }
  if (rc == SWDK_OK) {
    cudaStream_t st = (cudaStream_t)stream;
    float4* layR = (float4*)(base + o_layR);
    float4* layL = (float4*)(base + o_layL);
    ColInfo* info = (ColInfo*)(base + o_info);
    double* croot = (double*)(base + o_croot);
    int32_t* cstat = (int32_t*)(base + o_cstat);
    ChainDesc cd;
    cd.t_off = 0; cd.np = kmax; cd.nmode = mode; cd.iwave = iwave; cd.igr = igr; cd.out_off = 0;
    // each launch is checked as it is made, so the result reflects only
    // this call's own launches
    k_prep_layers<<<(nmodel + 127) / 128, 128, 0, st>>>(nmodel, nlayer, d_thk, d_vp, d_vs, d_rho, iflsph, layR, layL,
                                                         info);
    if (cudaGetLastError() != cudaSuccess) rc = SWDK_E_CUDA;
    if (rc == SWDK_OK) {
      k_roots_one<<<dim3((nmodel + 127) / 128, 1), 128, 0, st>>>(cd, nmodel, d_t, layR, layL, info, refine,
                                                                 rtol > 0.0 ? rtol : 1e-10, sngl, croot, cstat,
                                                                 d_ierr);
      if (cudaGetLastError() != cudaSuccess) rc = SWDK_E_CUDA;
    }
    if (rc == SWDK_OK) {
      const int n = nmodel * kmax;
      k_copy_last_mode<<<(n + 255) / 256, 256, 0, st>>>(nmodel, kmax, mode, croot, d_cg);
      if (cudaGetLastError() != cudaSuccess) rc = SWDK_E_CUDA;
    }
  }
  if (prev != device) cudaSetDevice(prev);
  return rc;
}

}  // extern "C"
