// swdk_eigen.cuh -- eigenfunction / energy-integral passes and node kernels.
//
// Rayleigh: sregn96.f90 svfunc (193-399), up (401-489), dnka (491-647),
//           evalg (649-825), varsv (827-911), hska (913-987), down
//           (989-1059), energy (1061-1196), intijr (1198-1317), ffunc..h2func
//           (1319-1397), getmat (1531-1583), sprayl (1585-1629).
// Love:     slegn96.f90 shfunc (179-246), varl (248-328), up (372-445),
//           energy (447-629), splove (631-670).
// Node kernels: SurfaceWave.cpp _ParamConvert (59-101) with the reference's
//           4.875x half-space weight of the last node kept.
//
// Arithmetic layout (same mathematics as the Fortran):
//   * everything that depends on the layer only (1/alpha^2, 1/beta^2, 1/rho,
//     the REAL*4 rho and 2 b^2 that dnka/hska take, the sphere factors) is
//     formed once per column in a RayLayer / LoveLayer record that every
//     slot of the column reads (shared memory on the device);
//   * every division by a slot constant (wvno, wvno^2, omega^2, rho omega^2)
//     is a multiplication by its reciprocal; 1/sqrt comes from rsqrt;
//   * per layer and sweep the vertical wavenumbers and exp(-r d) (or
//     cos/sin(r d)) are computed once and shared by varsv, dnka / hska and
//     the energy integrals (the Fortran evaluates them up to three times);
//     exp(-2 r d) is exp(-r d)^2 and exp(-(p+q)) is exp(-p) exp(-q);
//   * the energy integrals are formed without E and E^-1 (energy_lean);
//   * the up/down vectors are normalised by exact powers of two.
#pragma once
#include "swdk_core.cuh"

namespace swdk {

constexpr int LMAX = 320;   // sublayers per column (4*80-3 = 317)
constexpr int NZMAX = 96;   // grid nodes per column
constexpr double LN2 = 0.69314718055994530942;

// per-layer constants of one column's flattened Rayleigh model (bldsph of
// sregn96.f90:130-184); rf, rf2 and gq carry the REAL*4 rounding of dnka's
// and hska's arguments (rho, rho*rho and 2 b^2 are REAL*4 there)
struct RayLayer {
  double d, za, zb, zr;  // thickness, alpha, beta, rho
  double izr, ia2, ib2;  // 1/rho, 1/alpha^2, 1/beta^2 (0 for a fluid layer)
  double rf, irf;        // (double)(float)rho and its reciprocal
  double rf2, irf2;      // (double)(rhof*rhof) and its reciprocal
  double gq;             // (double)(2.0f*bf*bf)
  double vtp, rtp;       // _ParamConvert factors of the velocity / density transform
};

// per-layer constants of one column's flattened Love model (slegn96.f90:107-167)
struct LoveLayer {
  double d, zb, zr, ib2;  // thickness, beta, rho, 1/beta^2 (0 for a fluid layer)
  double mu, imu;         // rho beta^2 and its reciprocal
  double vtp, rtp;
};

SWDK_HD void make_ray_layer(RayLayer& y, double d, double za, double zb, double zr, double vtp, double rtp) {
  y.d = d; y.za = za; y.zb = zb; y.zr = zr;
  y.izr = 1.0 / zr;
  y.ia2 = 1.0 / (za * za);
  y.ib2 = (zb > 0.0) ? 1.0 / (zb * zb) : 0.0;
  const float rhof = (float)zr, bf = (float)zb;
  y.rf = (double)rhof;
  y.irf = 1.0 / y.rf;
  y.rf2 = (double)(rhof * rhof);
  y.irf2 = 1.0 / y.rf2;
  y.gq = (double)(2.0f * bf * bf);
  y.vtp = vtp; y.rtp = rtp;
}

SWDK_HD void make_love_layer(LoveLayer& y, double d, double zb, double zr, double vtp, double rtp) {
  y.d = d; y.zb = zb; y.zr = zr;
  y.ib2 = (zb > 0.0) ? 1.0 / (zb * zb) : 0.0;
  y.mu = zr * zb * zb;
  y.imu = (y.mu > 0.0) ? 1.0 / y.mu : 0.0;
  y.vtp = vtp; y.rtp = rtp;
}

// _ParamConvert (SurfaceWave.cpp:59-101) and the empirical chain rule
// (SurfaceWave.cpp:491-500) applied to each layer's raw kernels as the energy
// sweep produces them, so no per-layer kernel array is kept.  With nw = 0,
// layer l feeds node l/4 with weight 1 - (2j+1)/8 and node l/4 + 1 with
// (2j+1)/8, j = l % 4; with nw > 0 leading fluid nodes, solid layer l feeds
// the same pattern shifted to l-1 and nw (the fluid layer feeds a fluid node,
// whose kernel is zero).  The half-space weighs 4.875 (the reference's loop
// adds it once with 7/8 and four more times).  Node n accumulates
//   w * (x_b fa(l) + x_a fa(l) dalpha/dbeta(n) + x_r fr(l) drho/dalpha(n) dalpha/dbeta(n))
// with fa = vtp, fr = rtp; the pass's normaliser divides the sum afterwards.
struct NodeSink {
  double* kp;         // node sums [nz] (null: no kernels wanted)
  const float2* crs;  // (dalpha/dbeta, drho/dalpha) per node
  int L, nw, nz;
  // The sweep visits the sublayers top-down, so the two nodes of the current
  // node interval are the only ones still summing: they are held here and a
  // node is stored once, when the sweep leaves it (the sums keep the order
  // of a per-layer kp[n] += ...).
  mutable int cur;          // node of s0 (-1: none yet)
  mutable double s0, s1;    // running sums of nodes cur and cur + 1
  SWDK_HD void start() const { cur = -1; s0 = 0.0; s1 = 0.0; }
  SWDK_HD void to_node(int n) const {  // n >= cur: leave the nodes above n
    if (n == cur) return;
    if (cur >= 0) {
      kp[cur] = s0;
      if (n > cur + 1) kp[cur + 1] = s1;
    }
    s0 = (n == cur + 1) ? s1 : 0.0;
    s1 = 0.0;
    cur = n;
  }
  SWDK_HD void finish() const {
    if (!kp || cur < 0) return;
    kp[cur] = s0;
    if (cur + 1 < nz) kp[cur + 1] = s1;
  }
  SWDK_HD void add(int l, double fa, double fr, double xa, double xb, double xr) const {
    if (!kp) return;
    if (nw > 0 && l == 0) return;
    const int lp = (nw > 0) ? l - 1 : l;
    const int n0 = (lp >> 2) + nw;
    const double xbf = xb * fa, xaf = xa * fa, xrf = xr * fr;
    to_node(n0);
    if (l == L - 1) {
      const float2 c = crs[n0];
      const double dadb = c.x, drda = c.y;
      s0 += 4.875 * (xbf + xaf * dadb + xrf * drda * dadb);
    } else {
      const double t = (double)(2 * (lp & 3) + 1) / 8.0;
      {
        const float2 c = crs[n0];
        const double dadb = c.x, drda = c.y;
        s0 += (1.0 - t) * (xbf + xaf * dadb + xrf * drda * dadb);
      }
      {
        const float2 c = crs[n0 + 1];
        const double dadb = c.x, drda = c.y;
        s1 += t * (xbf + xaf * dadb + xrf * drda * dadb);
      }
    }
  }
};

// slot constants: wavenumber, frequency and their reciprocals
struct SlotK {
  double k, k2, ik, ik2, om, om2, iom2;
};

SWDK_HD SlotK slot_consts(double omega, double wvno) {
  SlotK s;
  s.k = wvno;
  s.k2 = wvno * wvno;
  s.ik = 1.0 / wvno;
  s.ik2 = s.ik * s.ik;
  s.om = omega;
  s.om2 = omega * omega;
  s.iom2 = 1.0 / s.om2;
  return s;
}

// exact power-of-two exponent e with 2^(e-1) <= t < 2^e (t > 0 finite) and
// the scale 2^-e
SWDK_HD int pow2_norm(double t, double& scale) {
  int e;
  frexp(t, &e);
  scale = ldexp(1.0, -e);
  return e;
}

// ---------------------------------------------------------------------------
// varsv (sregn96.f90:827-911) for the pure real / pure imaginary vertical
// wavenumbers that cdsqrt of a real argument produces, plus what the energy
// integrals need of the same layer: |r|, 1/|r|, and exp(-r d) (real r, cut
// to 0 beyond r d = 75 as ffunc..h2func do) or cos/sin(|r| d) (imaginary r)
// ---------------------------------------------------------------------------
struct LVars {
  double cosp, rsinp, sinpr, pex, ep, rp, irp, sp;  // P: ep = exp(-rp d) (1 if imaginary), sp = sin(|rp| d)
  double cosq, rsinq, sinqr, svex, eq, rs, irs, sq;
  bool preal, sreal;
};

SWDK_HD void vars_one(double x2, double d, double& cosv, double& rsinv, double& sinvr, double& ex, double& e,
                      double& r, double& ir, double& sv, bool& real) {
  const double tiny = (double)1.0e-5f;
  if (x2 >= 0.0) {  // r real
    ir = (x2 > 0.0) ? rsqrt(x2) : 0.0;
    r = x2 * ir;
    const double pr = r * d;
    e = (pr < 75.0) ? exp(-pr) : 0.0;
    const double fac = (pr < 30.0) ? e * e : 0.0;  // exp(-2 pr)
    cosv = 0.5 + fac * 0.5;
    const double sre = 0.5 - fac * 0.5;
    rsinv = r * sre;
    sinvr = (fabs(pr) < tiny && r < tiny) ? d : sre * ir;
    ex = pr;
    sv = 0.0;
    real = true;
  } else {  // r = i |r|
    ir = rsqrt(-x2);
    r = -x2 * ir;
    double s, c;
    sincos(r * d, &s, &c);
    cosv = c;
    rsinv = -r * s;
    sinvr = (r < tiny) ? d : s * ir;
    ex = 0.0;
    e = 1.0;
    sv = s;
    real = false;
  }
}

SWDK_HD void vars_lean(double x2p, double x2s, double d, int iwat, LVars& v) {
  vars_one(x2p, d, v.cosp, v.rsinp, v.sinpr, v.pex, v.ep, v.rp, v.irp, v.sp, v.preal);
  if (iwat == 1) {  // the S terms of a fluid layer (the energy integrals use only ra there)
    v.cosq = 1.0; v.rsinq = 0.0; v.sinqr = 0.0; v.svex = 0.0; v.eq = 1.0;
    v.rs = 0.0; v.irs = 0.0; v.sq = 0.0; v.sreal = true;
    return;
  }
  vars_one(x2s, d, v.cosq, v.rsinq, v.sinqr, v.svex, v.eq, v.rs, v.irs, v.sq, v.sreal);
}

// ee = cp * CA with CA the dnka matrix of sregn96 (REAL*4 rho, b; CA(i,j)
// = c<i-1><j-1> below), formed entry by entry into the product so that the
// 25 entries are never all held at once
SWDK_HD void dnka_apply(const LVars& v, const RayLayer& y, int iwat, const SlotK& s, const double* cp, double* ee) {
  const double irom2 = y.irf * s.iom2, rom2 = y.rf * s.om2;
  if (iwat == 1) {  // fluid: CA = diag(cosp, ., dfac, ., cosp) with the (1,2)/(2,1) and (4,5)/(5,4) pairs
    const double dfac = (v.pex > 35.0) ? 0.0 : v.ep;  // exp(-ex)
    const double c01 = -v.rsinp * irom2, c10 = -(y.rf * v.sinpr * s.om2);
    ee[0] = cp[0] * v.cosp + cp[1] * c10;
    ee[1] = cp[0] * c01 + cp[1] * v.cosp;
    ee[2] = cp[2] * dfac;
    ee[3] = cp[3] * v.cosp + cp[4] * c10;
    ee[4] = cp[3] * c01 + cp[4] * v.cosp;
    return;
  }
  const double exa = v.pex + v.svex;
  const double a0 = (exa < 60.0) ? v.ep * v.eq : 0.0;  // exp(-exa)
  const double cosp = v.cosp, cossv = v.cosq, rsinp = v.rsinp, rsinsv = v.rsinq, sinpr = v.sinpr,
               sinsvr = v.sinqr;
  const double k = s.k, k2 = s.k2, ik = s.ik, ik2 = s.ik2;
  const double cpcq = cosp * cossv, cpy = cosp * sinsvr, cpz = cosp * rsinsv, cqw = cossv * sinpr,
               cqx = cossv * rsinp;
  const double xy = rsinp * sinsvr, xz = rsinp * rsinsv, wy = sinpr * sinsvr, wz = sinpr * rsinsv;
  const double gam = y.gq * k2 * s.iom2;
  const double gam2 = gam * gam, gamm1 = gam - 1., gamm2 = gamm1 * gamm1;
  const double cqww2 = cqw * k2, cqxw2 = cqx * ik2, gg1 = gam * gamm1;
  const double a0c = 2.0 * (a0 - cpcq);
  const double xz2 = xz * ik2, gxz2 = gam * xz2, g2xz2 = gam2 * xz2;
  const double a0cgg1 = a0c * (gam + gamm1);
  const double wy2 = wy * k2, g2wy2 = gamm2 * wy2, g1wy2 = gamm1 * wy2;
  const double t1 = a0c * gg1 + g2xz2 + g2wy2;
  const double c00 = cpcq - t1;
  const double c22 = a0 + t1 + t1;
  const double c01 = (-cqx + k2 * cpy) * irom2;
  const double c02 = k * (0.5 * a0cgg1 + gxz2 + g1wy2) * irom2;
  const double c03 = (-cqww2 + cpz) * irom2;
  const double c04 = -(k2 * (a0c + wy2) + xz) * (y.irf2 * s.iom2 * s.iom2);
  const double c10 = (-gamm2 * cqw + gam2 * cpz * ik2) * rom2;
  const double c11 = cpcq;
  const double c12 = (gamm1 * cqww2 - gam * cpz) * ik;
  const double c13 = -wz;
  const double c20 = -2.0 * (0.5 * a0cgg1 * gg1 + gam2 * gxz2 + gamm2 * g1wy2) * rom2 * ik;
  const double c21 = (-k * (gam * cqxw2 - gamm1 * cpy)) * 2.0;
  const double c30 = (-gam2 * cqxw2 + gamm2 * cpy) * rom2;
  const double c31 = -xy;
  const double c40 = -(y.rf2 * s.om2 * s.om2) * (gamm2 * (a0c * gam2 + g2wy2) + gam2 * g2xz2) * ik2;
  // rows 2..5 repeat entries: c14 = c03, c23 = -2 c12, c24 = -2 c02,
  // c32 = -c21/2, c33 = c11, c34 = c01, c41 = c30, c42 = -c20/2, c43 = c10, c44 = c00
  const double p0 = cp[0], p1 = cp[1], p2 = cp[2], p3 = cp[3], p4 = cp[4];
  ee[0] = p0 * c00 + p1 * c10 + p2 * c20 + p3 * c30 + p4 * c40;
  ee[1] = p0 * c01 + p1 * c11 + p2 * c21 + p3 * c31 + p4 * c30;
  ee[2] = p0 * c02 + p1 * c12 + p2 * c22 + p3 * (-c21 * 0.5) + p4 * (-c20 * 0.5);
  ee[3] = p0 * c03 + p1 * c13 + p2 * (-2.0 * c12) + p3 * c11 + p4 * c10;
  ee[4] = p0 * c04 + p1 * c03 + p2 * (-2.0 * c02) + p3 * c01 + p4 * c00;
}

// a0 = AA * vv with AA the hska matrix (sregn96.f90:913-987), formed entry
// by entry into the product
SWDK_HD void hska_apply(const LVars& v, const RayLayer& y, int iwat, const SlotK& s, const double* vv, double* a0) {
  const double irom2 = y.irf * s.iom2, rom2 = y.rf * s.om2;
  if (iwat == 1) {
    const double dfac = (v.pex > 35.0) ? 0.0 : v.ep;
    const double a12 = -v.rsinp * irom2, a21 = -(rom2 * v.sinpr);
    a0[0] = dfac * vv[0];
    a0[1] = v.cosp * vv[1] + a12 * vv[2];
    a0[2] = a21 * vv[1] + v.cosp * vv[2];
    a0[3] = dfac * vv[3];
    return;
  }
  // exp(svex - pex), 0 when pex - svex > 70; exp(-pex) / exp(-svex) while
  // both factors are held (below 75)
  double dfac;
  if ((v.pex - v.svex) > 70.0) dfac = 0.0;
  else if (v.pex < 75.0 && v.svex < 75.0) dfac = v.ep * recip(v.eq);
  else dfac = exp(v.svex - v.pex);
  const double cossv = dfac * v.cosq, rsinsv = dfac * v.rsinq, sinsvr = dfac * v.sinqr;
  const double cosp = v.cosp, rsinp = v.rsinp, sinpr = v.sinpr;
  const double k = s.k, k2 = s.k2, ik = s.ik, ik2 = s.ik2;
  const double gam = y.gq * k2 * s.iom2;
  const double gamm1 = gam - 1.0;
  const double dc = cosp - cossv;
  const double A00 = cossv + gam * dc;
  const double A01 = -k * gamm1 * sinpr + gam * rsinsv * ik;
  const double A02 = -(k * dc * irom2);
  const double A03 = (k2 * sinpr - rsinsv) * irom2;
  const double A10 = gam * rsinp * ik - k * gamm1 * sinsvr;
  const double A11 = cosp - gam * dc;
  const double A12 = (-rsinp + k2 * sinsvr) * irom2;
  const double A20 = rom2 * gam * gamm1 * dc * ik;
  const double A21 = rom2 * (-gamm1 * gamm1 * sinpr + gam * gam * rsinsv * ik2);
  const double A30 = rom2 * (gam * gam * rsinp * ik2 - gamm1 * gamm1 * sinsvr);
  // AA(2,4) = -AA(1,3), AA(3,3) = AA(2,2), AA(3,4) = -AA(1,2),
  // AA(4,2) = -AA(3,1), AA(4,3) = -AA(2,1), AA(4,4) = AA(1,1)
  const double v0 = vv[0], v1 = vv[1], v2 = vv[2], v3 = vv[3];
  a0[0] = A00 * v0 + A01 * v1 + A02 * v2 + A03 * v3;
  a0[1] = A10 * v0 + A11 * v1 + A12 * v2 + (-A02) * v3;
  a0[2] = A20 * v0 + A21 * v1 + A11 * v2 + (-A01) * v3;
  a0[3] = A30 * v0 + (-A20) * v1 + (-A10) * v2 + A00 * v3;
}

// half-space start vector of the up pass: evalg's gbr (sregn96.f90:736-760,
// 774-790) for the bottom layer, once per pass
SWDK_HD void halfspace_gbr(const RayLayer& y, int iwat, const SlotK& s, double g[5]) {
  const cx ra = csqrt_real(s.k2 - s.om2 * y.ia2), rb = csqrt_real(s.k2 - s.om2 * y.ib2);
  const double zr = y.zr, om2 = s.om2, wvno = s.k, wvno2 = s.k2;
  double gam = y.zb * wvno / s.om;
  gam = 2.0 * (gam * gam);
  const double gamm1 = gam - 1.0;
  cx gbr[5];
  if (iwat == 0) {
    gbr[0] = (zr * zr * om2 * om2) * (-((gam * gam) * ra * rb) + wvno2 * gamm1 * gamm1);
    gbr[1] = -((zr * (wvno2 * ra)) * om2);
    gbr[2] = -(((zr * (-((gam * ra) * rb) + wvno2 * gamm1)) * om2) * wvno);
    gbr[3] = (zr * (wvno2 * rb)) * om2;
    gbr[4] = wvno2 * (wvno2 - ra * rb);
    const cx den = -((zr * zr * om2 * om2 * wvno2) * ra * rb);
    for (int i = 0; i < 5; ++i) gbr[i] = (0.25 * gbr[i]) / den;
  } else {  // a fluid half-space under the column (jbdry = 0)
    gbr[0] = mkc(0); gbr[1] = mkc(0); gbr[2] = mkc(0);
    gbr[3] = (0.5 * zr * om2) / ra;
    gbr[4] = mkc(-0.5);
  }
  for (int i = 0; i < 5; ++i) g[i] = gbr[i].re;
}

// Eigenfunction values at a layer top: (ur, uz, tz, tr)
struct Eig4 {
  double ur, uz, tz, tr;
};

struct EnergyAcc {
  double sumi0, sumi1, sumi2, sumi3;
};

SWDK_HD double re_mul(cx a, cx b) { return a.re * b.re - a.im * b.im; }
// 1/z of a general complex z: conj(z) / |z|^2
SWDK_HD cx cinv_any(cx z) {
  const double s = recip(z.re * z.re + z.im * z.im);
  return mkc(z.re * s, -z.im * s);
}
// a vertical wavenumber (pure real or pure imaginary) from its magnitude,
// and its reciprocal from the magnitude's reciprocal
SWDK_HD cx rval(bool real, double r) { return real ? mkc(r, 0.0) : mkc(0.0, r); }
SWDK_HD cx rinv(bool real, double ir) { return real ? mkc(ir, 0.0) : mkc(0.0, -ir); }
// exp(-r d): real r -> e, imaginary r -> cos - i sin
SWDK_HD cx rexp(bool real, double e, double c, double s) { return real ? mkc(e, 0.0) : mkc(c, -s); }
// ffunc (sregn96.f90:1319-1335), (1 - exp(-2 r d)) / (2 r) for |r| >= 1e-8:
// real r with e = exp(-r d) (0 when r d >= 40); imaginary r from cos, sin
SWDK_HD cx ffun(bool real, double ir, double e, double c, double s) {
  if (real) return mkc((1.0 - e * e) * 0.5 * ir, 0.0);
  return mkc(s * c * ir, -s * s * ir);
}

// energy() body for one layer (sregn96.f90:1097-1178); writes the raw
// (un-normalised) dcda, dcdb, dcdr of the layer.
//
// intijr (sregn96.f90:1198-1317) is evaluated without forming E and E^-1:
// row r of E (evalg, sregn96.f90:716-734) is (p_r, q_r, s_r p_r, -s_r q_r)
// with s = (+,-,+,-), (p,q) = (k, rb), (ra, k), (g1, g2 rb), (g2 ra, g1),
// k = wvno, g1 = rho om2 (gam-1), g2 = rho om2 gam / k; all six integrals
// used by energy pair rows of equal sign s, so with P = p_i p_j,
// Q = q_i q_j, X = p_i q_j + q_i p_j
//   interior layer: cint = P SA_s + Q SB_s + X SX_s,
//     SA_s = FA (kmpu^2 + km1pd^2) + 2 s GA kmpu km1pd
//     SB_s = FB (kmsu^2 + km1sd^2) - 2 s GB kmsu km1sd
//     SX_s = H1 (kmpu kmsu - km1pd km1sd) + s H2 (km1pd kmsu - kmpu km1sd)
//   half-space:     cint = P km1pd^2/(2ra) - X km1pd km1sd/(ra+rb) + Q km1sd^2/(2rb)
// and the potentials are rows of E^-1 applied to (ur, uz, tz, tr).
SWDK_HD void energy_lean(const RayLayer& y, const LVars& v, int iwat, bool half, const Eig4& u0, const Eig4& u1,
                         const SlotK& s, double c, EnergyAcc& acc, double& dcda, double& dcdb, double& dcdr) {
  const double za = y.za, zb = y.zb, zr = y.zr, zdm = y.d;
  const double k = s.k, k2 = s.k2, ik = s.ik, ik2 = s.ik2;
  const double ra2 = k2 - s.om2 * y.ia2, rb2 = k2 - s.om2 * y.ib2;
  const cx ra = rval(v.preal, v.rp), ira = rinv(v.preal, v.irp);
  const double gam = 2.0 * (zb * zb * k2 * s.iom2);  // 2 (zb wvno / om)^2
  const double gamm1 = gam - 1.0;
  const double rom2 = zr * s.om2, irom2 = y.izr * s.iom2;
  double INT11, INT13 = 0.0, INT22, INT24 = 0.0, INT33 = 0.0, INT44 = 0.0;
  if (iwat == 0) {
    const cx rb = rval(v.sreal, v.rs), irb = rinv(v.sreal, v.irs);
    const double g1 = rom2 * gamm1, g2 = rom2 * gam * ik;
    const double h1 = 0.5 * gam * ik, h2 = -(0.5 * irom2), ga = 0.5 * gamm1, wa = 0.5 * k * irom2;
    const cx km1pd = (h1 * u0.ur + h2 * u0.tz) + (ga * u0.uz - wa * u0.tr) * ira;
    const cx km1sd = (ga * u0.ur - wa * u0.tz) * irb + (h1 * u0.uz + h2 * u0.tr);
    if (!half) {
      const cx kmpu = (h1 * u1.ur + h2 * u1.tz) - (ga * u1.uz - wa * u1.tr) * ira;
      const cx kmsu = (h1 * u1.uz + h2 * u1.tr) - (ga * u1.ur - wa * u1.tz) * irb;
      // FA, GA, FB, GB, H1, H2 (sregn96.f90:1319-1397)
      const double ard = v.preal ? v.rp * zdm : 0.0, brd = v.sreal ? v.rs * zdm : 0.0;
      const cx ea = rexp(v.preal, v.ep, v.cosp, v.sp), eb = rexp(v.sreal, v.eq, v.cosq, v.sq);
      const cx ea40 = (ard < 40.0) ? ea : mkc(0.0), eb40 = (brd < 40.0) ? eb : mkc(0.0);
      const cx FA = (v.rp < 1.0e-08) ? mkc(zdm) : ffun(v.preal, v.irp, ea40.re, v.cosp, v.sp);
      const cx FB = (v.rs < 1.0e-08) ? mkc(zdm) : ffun(v.sreal, v.irs, eb40.re, v.cosq, v.sq);
      const cx GA = ea * zdm, GB = eb * zdm;
      const cx sab = ra + rb;
      const cx H1 = (cabsc(sab) < 1.0e-08) ? mkc(zdm)
                    : (1.0 - ((ard + brd < 40.0) ? ea * eb : mkc(0.0))) * cinv_any(sab);
      const cx dab = ra - rb;
      const cx H2 = (cabsc(dab) < 1.0e-08) ? mkc(zdm) : (eb40 - ea40) * cinv_any(dab);
      const cx pp = kmpu * kmpu + km1pd * km1pd, ss = kmsu * kmsu + km1sd * km1sd;
      const cx pd = kmpu * km1pd, sd = kmsu * km1sd;
      const cx x1 = kmpu * kmsu - km1pd * km1sd, x2 = km1pd * kmsu - kmpu * km1sd;
      const double FApp = re_mul(FA, pp), GApd2 = 2.0 * re_mul(GA, pd), FBss = re_mul(FB, ss),
                   GBsd2 = 2.0 * re_mul(GB, sd);
      const cx H1x = H1 * x1, H2x = H2 * x2;
      const double SAp = FApp + GApd2, SAm = FApp - GApd2;
      const double SBp = FBss - GBsd2, SBm = FBss + GBsd2;
      const double Xp = re_mul(rb, H1x + H2x), Xm = re_mul(ra, H1x - H2x);
      INT11 = k2 * SAp + rb2 * SBp + 2.0 * k * Xp;
      INT13 = k * g1 * SAp + g2 * rb2 * SBp + (k * g2 + g1) * Xp;
      INT33 = g1 * g1 * SAp + g2 * g2 * rb2 * SBp + 2.0 * g1 * g2 * Xp;
      INT22 = ra2 * SAm + k2 * SBm + 2.0 * k * Xm;
      INT24 = g2 * ra2 * SAm + k * g1 * SBm + (g1 + k * g2) * Xm;
      INT44 = g2 * g2 * ra2 * SAm + g1 * g1 * SBm + 2.0 * g1 * g2 * Xm;
    } else {
      const double TA = re_mul(km1pd * km1pd, 0.5 * ira), TB = re_mul(km1sd * km1sd, 0.5 * irb);
      const cx TX = -((km1pd * km1sd) * cinv_any(ra + rb));
      const double Xb = re_mul(rb, TX), Xa = re_mul(ra, TX);
      INT11 = k2 * TA + rb2 * TB + 2.0 * k * Xb;
      INT13 = k * g1 * TA + g2 * rb2 * TB + (k * g2 + g1) * Xb;
      INT33 = g1 * g1 * TA + g2 * g2 * rb2 * TB + 2.0 * g1 * g2 * Xb;
      INT22 = ra2 * TA + k2 * TB + 2.0 * k * Xa;
      INT24 = g2 * ra2 * TA + k * g1 * TB + (g1 + k * g2) * Xa;
      INT44 = g2 * g2 * ra2 * TA + g1 * g1 * TB + 2.0 * g1 * g2 * Xa;
    }
  } else {
    // fluid layer: 2x2 E = [[ra, -ra], [-rho om2, -rho om2]] (sregn96.f90:791-801)
    const double ir = -(0.5 * irom2);
    const cx km1pd = (-0.5 * u0.uz) * ira + ir * u0.tz;
    const double w = -rom2;
    if (!half) {
      const cx kmpu = (0.5 * u1.uz) * ira + ir * u1.tz;
      const double ard = v.preal ? v.rp * zdm : 0.0;
      const cx ea = rexp(v.preal, v.ep, v.cosp, v.sp);
      const cx ea40 = (ard < 40.0) ? ea : mkc(0.0);
      const cx FA = (v.rp < 1.0e-08) ? mkc(zdm) : ffun(v.preal, v.irp, ea40.re, v.cosp, v.sp);
      const cx GA = ea * zdm;
      const cx sq = (kmpu * kmpu + km1pd * km1pd) * FA, cr = 2.0 * (kmpu * km1pd * GA);
      INT11 = ra2 * (sq - cr).re;
      INT22 = w * w * (sq + cr).re;
    } else {
      INT11 = 0.0;
      INT22 = w * w * re_mul(km1pd * km1pd, 0.5 * ira);
    }
  }
  // getmat (sregn96.f90:1531-1583) and the energy sums
  const double rho = zr, ah = za, av = za, eta = 1.0;
  const double TA = zr * za * za, TC = TA, iTC = y.izr * y.ia2;
  if (iwat == 1) {
    const double TN = 0.0, TF = TA - 2. * TN;
    const double a12 = -(k2 - s.om2 * y.ia2) * irom2;
    const double wr = k * irom2;
    const double URUR = INT22 * (wr * wr), UZUZ = INT11;
    const double URDUZ = -(wr * a12 * INT22);
    const double DUZDUZ = a12 * a12 * INT22;
    acc.sumi0 = acc.sumi0 + rho * (URUR + UZUZ);
    acc.sumi1 = acc.sumi1 + TA * URUR;
    acc.sumi2 = acc.sumi2 - TF * URDUZ;
    acc.sumi3 = acc.sumi3 + TC * DUZDUZ;
    const double facah = rho * ah * (URUR - 2. * eta * URDUZ * ik);
    const double facav = rho * av * DUZDUZ * ik2;
    dcda = facah + facav;
    dcdb = 0.0;
    const double facr = -(0.5 * c * c * (URUR + UZUZ));
    dcdr = 0.5 * (av * facav + ah * facah) * y.izr + facr;
  } else {
    const double bv = zb;
    const double TL = zr * zb * zb;
    const double TF = TA - 2. * TL;
    const double a12 = -k, a14 = y.izr * y.ib2, a21 = k * TF * iTC, a23 = iTC;
    const double URUR = INT11, UZUZ = INT22;
    const double DURDUR = a12 * a12 * INT22 + 2. * a12 * a14 * INT24 + a14 * a14 * INT44;
    const double DUZDUZ = a21 * a21 * INT11 + 2. * a21 * a23 * INT13 + a23 * a23 * INT33;
    const double URDUZ = a21 * INT11 + a23 * INT13;
    const double UZDUR = a12 * INT22 + a14 * INT24;
    acc.sumi0 = acc.sumi0 + rho * (URUR + UZUZ);
    acc.sumi1 = acc.sumi1 + TL * UZUZ + TA * URUR;
    acc.sumi2 = acc.sumi2 + TL * UZDUR - TF * URDUZ;
    acc.sumi3 = acc.sumi3 + TL * DURDUR + TC * DUZDUZ;
    const double facah = rho * ah * (URUR - 2. * eta * URDUZ * ik);
    const double facav = rho * av * DUZDUZ * ik2;
    const double facbv = rho * bv * (UZUZ + 2. * UZDUR * ik + DURDUR * ik2 + 4. * eta * URDUZ * ik);
    dcda = facah + facav;
    dcdb = facbv;
    const double facr = -(0.5 * c * c * (URUR + UZUZ));
    dcdr = 0.5 * (av * facav + ah * facah + bv * facbv) * y.izr + facr;
  }
}

// svfunc eigenfunction at a layer top from the compound (cd) and Haskell
// (vv) vectors (sregn96.f90:279-312); if1213 = 1/f1213
SWDK_HD Eig4 eigen_at(const double* cd, const double* vv, double ext, double if1213) {
  const double cd1 = cd[0], cd2 = cd[1], cd3 = cd[2], cd4 = -cd[2], cd5 = cd[3], cd6 = cd[4];
  const double tz1 = -vv[3], tz2 = -vv[2], tz3 = vv[1], tz4 = vv[0];
  const double uu1 = tz2 * cd6 - tz3 * cd5 + tz4 * cd4;
  const double uu2 = -tz1 * cd6 + tz3 * cd3 - tz4 * cd2;
  const double uu3 = tz1 * cd5 - tz2 * cd3 + tz4 * cd1;
  const double uu4 = -tz1 * cd4 + tz2 * cd2 - tz3 * cd1;
  Eig4 u;
  if (ext > -80.0 && ext < 80.0) {
    const double fact = exp(ext) * if1213;
    u.ur = uu1 * fact;
    u.uz = uu2 * fact;
    u.tz = uu3 * fact;
    u.tr = uu4 * fact;
  } else {
    u.ur = 0.0; u.uz = 0.0; u.tz = 0.0; u.tr = 0.0;
  }
  return u;
}

// Depth truncation of a pass.  Below the layer where the S-wave evanescent
// decay sum(Re r_beta d) accumulated from the top exceeds trunc_q, the
// eigenfunctions are below exp(-trunc_q) of their surface amplitude and the
// layers' energy integrals and kernels below exp(-2 trunc_q) of the largest:
// the pass then treats the next layer as the half-space (the up pass's start
// vector there converges to the same surface value to a relative
// exp(-2 trunc_q), the compound vector's subdominant parts decaying by
// exp(-2 q) per evanescent layer) and the layers below it get zero kernels.
// Returns the number of layers the pass uses (L when nothing is cut;
// trunc_q <= 0 disables the cut).
template <class Layer>
SWDK_HD int pass_layers(const Layer* lay, int L, double k2, double om2, double trunc_q) {
  if (!(trunc_q > 0.0)) return L;
  double cum = 0.0;
  for (int m = 0; m < L - 2; ++m) {
    const Layer& y = lay[m];
    if (y.zb > 0.0) {
      const double x2s = k2 - om2 * y.ib2;
      if (x2s > 0.0) cum += x2s * rsqrt(x2s) * y.d;
    }
    if (cum > trunc_q) return m + 2;  // lay[m+1] becomes the half-space
  }
  return L;
}

// The device passes run uncut (0): the slots of a warp are different
// periods of one column and cut at very different depths, so a warp's
// sweeps take as long as its deepest slot's while every slot pays for the
// search (eigen stage 154 ms uncut against 166 ms cut at 40 per step of the
// default workload).  Cutting at 40 changes U and kernels by < 1e-12
// relative (CPU harness test).
constexpr double EIG_TRUNC_Q = 0.0;

// Up-pass storage of a Rayleigh pass with checkpoints: the compound vector
// (and its exponent bookkeeping) is kept only at every RAY_SEG-th layer and
// at the half-space; the down sweep recomputes each segment of RAY_SEG
// layers from its checkpoint into seg[] just before it needs them.  The
// recomputation repeats the up pass's arithmetic exactly, so the values are
// the ones a full per-layer store would hold, with about 2 KB of scratch per
// slot instead of 6 doubles per layer.
#ifndef SWDK_RAY_SEG
#define SWDK_RAY_SEG 16
#endif
constexpr int RAY_SEG = SWDK_RAY_SEG;
constexpr int RAY_NCK = (LMAX + RAY_SEG - 1) / RAY_SEG;
struct RayScratch {
  double ck[RAY_NCK][8];  // layer j*RAY_SEG: cd[5], exponent sum, exr, exi
  double hs[8];           // the half-space start of the (cut) pass
  double seg[RAY_SEG][6];  // the segment being consumed: cd[5], exponent sum
};

// one step of the up pass (sregn96.f90:401-489) after vars_lean of its
// layer: the compound vector cd of layer m from that of layer m+1 (in
// place), with its exponent sum
SWDK_HD void ray_up_apply(const LVars& v, const RayLayer& y, int iw, const SlotK& s, double* cd, double& exr,
                          int& exi) {
  double ee[5];
  dnka_apply(v, y, iw, s, cd, ee);
  double t1 = 0.0;
  for (int i = 0; i < 5; ++i) t1 = fmax(t1, fabs(ee[i]));
  int e = 0;
  double sc = 1.0;
  if (t1 >= 1.e-40) e = pow2_norm(t1, sc);
  for (int i = 0; i < 5; ++i) cd[i] = ee[i] * sc;
  exr = exr + v.pex + v.svex;
  exi += e;
  cd[5] = exr + (double)exi * LN2;
}

SWDK_HD void ray_keep(double* dst, const double* cd, double exr, int exi) {
  for (int i = 0; i < 6; ++i) dst[i] = cd[i];
  dst[6] = exr;
  dst[7] = (double)exi;
}

// One Rayleigh pass (sregn96's svfunc + energy) at (omega, wvno) over the
// column's layer records lay[0..L-1] (top-down, lay[L-1] the half-space),
// depth-truncated by pass_layers.  Returns ugr (flat) and norm = ugr*sumi0;
// the raw layer kernels go to the sink as the top-down sweep produces them.
//
// One loop runs the up pass (layers L-2 .. 0, keeping checkpoints), then
// the top-down sweep (layers 0 .. L-1), which at the first layer of each
// segment recomputes the segment's compound vectors from its checkpoint by
// further up steps.  Every step evaluates its layer's variables (vars_lean:
// square roots, exponentials or sines and cosines) at one place in the
// code, so the kernel holds one copy of that code instead of three (the
// Rayleigh eigen kernel waited on instruction fetch about as often as on
// its FP64 results).  The steps and their arithmetic are those of separate
// up, recompute and down loops.
template <class Sink>
SWDK_HDI void rayleigh_pass(const RayLayer* lay, int Lfull, double omega, double wvno, RayScratch& scr, double& ugr,
                            double& norm, const Sink& sink, double trunc_q = EIG_TRUNC_Q) {
  const SlotK s = slot_consts(omega, wvno);
  const int L = pass_layers(lay, Lfull, s.k2, s.om2, trunc_q);
  // ---- up (sregn96.f90:401-489) start: the half-space ----
  double cd[6];
  {
    const RayLayer& y = lay[L - 1];
    halfspace_gbr(y, (y.zb > 0.0) ? 0 : 1, s, cd);
    cd[5] = 0.0;
  }
  double exr = 0.0;
  int exi = 0;
  ray_keep(scr.hs, cd, exr, exi);
  if ((L - 1) % RAY_SEG == 0) ray_keep(scr.ck[(L - 1) / RAY_SEG], cd, exr, exi);
  // ---- down + svfunc + energy state ----
  double if1213 = 0.0, exe0 = 0.0;
  Eig4 u0 = {0.0, 0.0, 0.0, 0.0};
  double vv[4] = {1.0, 0.0, 0.0, 0.0};
  double dxr = 0.0;
  int dxi = 0;
  EnergyAcc acc = {0.0, 0.0, 0.0, 0.0};
  const double c = omega * s.ik;
  int up = L - 2;        // layer of the next up-pass step (< 0: the up pass is done)
  int dn = 0;            // layer of the next down step
  int sl = -1, sj0 = -1;  // segment recomputation: its next layer sl while sl > sj0
  bool down = false;
  auto begin_down = [&]() {
    sink.start();
    const double* top = scr.ck[0];  // layer 0
    if1213 = -1.0 / top[1];
    exe0 = top[5];
    u0.ur = top[2] / top[1];
    u0.uz = 1.0; u0.tz = 0.0; u0.tr = 0.0;
    if (lay[0].zb <= 0.0) { u0.ur = 0.0; u0.tr = 0.0; }  // fluid top (jwat)
    down = true;
  };
  if (up < 0) begin_down();
#pragma unroll 1  // a layer recursion: unrolling only grows the code
  for (;;) {
    int lm;
    bool upstep;
    if (!down) {
      lm = up;
      upstep = true;
    } else {
      const int j0 = dn - dn % RAY_SEG;  // first layer of dn's segment
      if (sl <= sj0 && dn == j0 && dn < L - 1 && sj0 != j0) {
        // cd of layers j0+1 .. t from the checkpoint at t
        const int t = (j0 + RAY_SEG < L - 1) ? j0 + RAY_SEG : L - 1;
        const double* src = (t == L - 1) ? scr.hs : scr.ck[t / RAY_SEG];
        for (int i = 0; i < 6; ++i) cd[i] = src[i];
        exr = src[6];
        exi = (int)src[7];
        for (int i = 0; i < 6; ++i) scr.seg[t - j0 - 1][i] = cd[i];
        sj0 = j0;
        sl = t - 1;
      }
      upstep = sl > sj0;
      lm = upstep ? sl : dn;
    }
    const RayLayer& y = lay[lm];
    const int iw = (y.zb > 0.0) ? 0 : 1;
    LVars v;
    vars_lean(s.k2 - s.om2 * y.ia2, s.k2 - s.om2 * y.ib2, y.d, iw, v);
    if (upstep) {
      ray_up_apply(v, y, iw, s, cd, exr, exi);
      if (!down) {
        if (up % RAY_SEG == 0) ray_keep(scr.ck[up / RAY_SEG], cd, exr, exi);
        if (--up < 0) begin_down();
      } else {
        for (int i = 0; i < 6; ++i) scr.seg[sl - sj0 - 1][i] = cd[i];
        --sl;
      }
      continue;
    }
    const bool half = (dn == L - 1);
    Eig4 u1 = u0;
    if (!half) {
      double a0[4];
      hska_apply(v, y, iw, s, vv, a0);
      double t1 = fmax(fmax(fabs(a0[0]), fabs(a0[1])), fmax(fabs(a0[2]), fabs(a0[3])));
      int e = 0;
      double sc = 1.0;
      if (t1 >= 1.e-40) e = pow2_norm(t1, sc);
      for (int i = 0; i < 4; ++i) vv[i] = a0[i] * sc;
      dxr = dxr + v.pex;
      dxi += e;
      const double exa1 = dxr + (double)dxi * LN2;
      const double* cd1 = scr.seg[dn - (dn - dn % RAY_SEG)];  // layer dn + 1
      u1 = eigen_at(cd1, vv, exa1 + cd1[5] - exe0, if1213);
    }
    double da, db, dr;
    energy_lean(y, v, iw, half, u0, u1, s, c, acc, da, db, dr);
    sink.add(dn, y.vtp, y.rtp, da, db, dr);
    u0 = u1;
    if (++dn >= L) break;
  }
  sink.finish();
  ugr = (wvno * acc.sumi1 + acc.sumi2) / (omega * acc.sumi0);
  norm = ugr * acc.sumi0;
}

// ---------------------------------------------------------------------------
// One Love pass (slegn96.f90): up, shfunc normalisation, energy.  The up
// pass keeps (uu, tt, exl) only at every RAY_SEG-th layer and the
// half-space; the energy sweep recomputes each segment from its checkpoint
// and applies shfunc's normalisation exp(-ext) on the fly.  Returns ugr and
// the normaliser sumi1.
// ---------------------------------------------------------------------------
struct LoveScratch {
  double ck[RAY_NCK][3];
  double hs[3];
  double seg[RAY_SEG + 1][3];  // layers j0 .. j0 + RAY_SEG of the current segment
};

// one step of slegn96's up pass (slegn96.f90:372-445): (uu, tt) of layer k
// from layer k+1 (s1), power-of-two normalised, and the step's exponent exl
SWDK_HD void love_up_step(const LoveLayer& y, double wvno2, double om2, const double* s1, double* sk) {
  if (!(y.zb > 0.0)) { sk[0] = 0.0; sk[1] = 0.0; sk[2] = 0.0; return; }
  const double dpth = y.d;
  const double x2 = wvno2 - om2 * y.ib2;  // (wvno + xkb)(wvno - xkb)
  double cosq, yl, zl, eexl = 0.0;
  if (x2 < 0.0) {  // wvno < xkb
    const double ir = rsqrt(-x2), rb = -x2 * ir;
    double sq, cq;
    sincos(rb * dpth, &sq, &cq);
    yl = sq * ir; zl = -rb * sq; cosq = cq;
  } else if (x2 == 0.0) {
    cosq = 1.0; yl = dpth; zl = 0.0;
  } else {
    const double ir = rsqrt(x2), rb = x2 * ir, q = rb * dpth;
    eexl = q;
    const double e1 = (q < 18.0) ? exp(-q) : 0.0;
    const double fac = e1 * e1;  // exp(-2q)
    cosq = (1.0 + fac) * 0.5;
    const double sq = (1.0 - fac) * 0.5;
    yl = sq * ir; zl = rb * sq;
  }
  const double a11 = cosq, a22 = cosq, a12 = -(yl * y.imu), a21 = -(zl * y.mu);
  const double amp0 = a11 * s1[0] + a12 * s1[1];
  const double str0 = a21 * s1[0] + a22 * s1[1];
  const double rr = fmax(fabs(amp0), fabs(str0));
  int e = 0;
  double sc = 1.0;
  if (rr >= 1.e-30) e = pow2_norm(rr, sc);
  sk[0] = amp0 * sc;
  sk[1] = str0 * sc;
  sk[2] = (double)e * LN2 + eexl;
}

// the raw up-pass values of layers j0 .. t (t the checkpoint at or below
// j0 + RAY_SEG) into seg[0 .. t - j0]
SWDK_HD void love_fill_segment(const LoveLayer* lay, int L, double wvno2, double om2, LoveScratch& scr, int j0) {
  const int t = (j0 + RAY_SEG < L - 1) ? j0 + RAY_SEG : L - 1;
  const double* src = (t == L - 1) ? scr.hs : scr.ck[t / RAY_SEG];
  for (int i = 0; i < 3; ++i) scr.seg[t - j0][i] = src[i];
#pragma unroll 1
  for (int l = t - 1; l >= j0; --l) love_up_step(lay[l], wvno2, om2, scr.seg[l - j0 + 1], scr.seg[l - j0]);
}

template <class Sink>
SWDK_HDI void love_pass(const LoveLayer* lay, int Lfull, double omega, double wvno, LoveScratch& scr, double& ugr,
                        double& norm, const Sink& sink, double trunc_q = EIG_TRUNC_Q) {
  const double wvno2 = wvno * wvno, om2 = omega * omega, ik = 1.0 / wvno, ik2 = ik * ik;
  const int L = pass_layers(lay, Lfull, wvno2, om2, trunc_q);
  // ---- up (slegn96.f90:372-445), checkpoints only ----
  double sv[3];
  {
    const LoveLayer& y = lay[L - 1];
    if (y.zb > (double)0.01f) {
      const double rb = sqrt(fabs(wvno2 - om2 * y.ib2));
      sv[0] = 1.0;
      sv[1] = -y.mu * rb;
    } else {
      sv[0] = 1.0;
      sv[1] = 0.0;
    }
    sv[2] = 0.0;
  }
  for (int i = 0; i < 3; ++i) scr.hs[i] = sv[i];
  if ((L - 1) % RAY_SEG == 0)
    for (int i = 0; i < 3; ++i) scr.ck[(L - 1) / RAY_SEG][i] = sv[i];
#pragma unroll 1  // a layer recursion: unrolling only grows the code
  for (int k = L - 2; k >= 0; --k) {
    double nv[3];
    love_up_step(lay[k], wvno2, om2, sv, nv);
    for (int i = 0; i < 3; ++i) sv[i] = nv[i];
    if (k % RAY_SEG == 0)
      for (int i = 0; i < 3; ++i) scr.ck[k / RAY_SEG][i] = sv[i];
  }
  // ---- shfunc normalisation (slegn96.f90:212-240): layer k's (uu, tt)
  // are the raw values times exp(-ext), ext summing the exl of the solid
  // layers above; tt(1) = 0.  The amplitude scale umax is uu(1) unless
  // that is zero (a fluid top), then the largest normalised |uu|. ----
  const double top0 = scr.ck[0][0];
  double umax = top0;
  if (top0 == 0.0) {
    double ext = 0.0;
#pragma unroll 1
    for (int k = 1; k < L; ++k) {
      const int j0 = (k - 1) - (k - 1) % RAY_SEG;
      if (k - 1 == j0) love_fill_segment(lay, L, wvno2, om2, scr, j0);
      double u = 0.0;
      if (lay[k].zb > 0.0) {
        ext = ext + scr.seg[k - 1 - j0][2];
        const double fact = (ext < 80.0) ? exp(-ext) : 0.0;
        u = scr.seg[k - j0][0] * fact;
      }
      if (fabs(u) > fabs(umax)) umax = u;
    }
  }
  const double iumax = (fabs(umax) > 0.0) ? 1.0 / umax : 1.0;
  // ---- energy (slegn96.f90:447-576) with uu/tt scaled by 1/umax on the fly ----
  const double c = omega * ik;
  double sumi0 = 0.0, sumi1 = 0.0;
  double ext = 0.0;
  double uu = top0 * iumax, tt = 0.0;
  sink.start();
#pragma unroll 1  // a layer recursion: unrolling only grows the code
  for (int k = 0; k < L; ++k) {
    const int j0 = k - k % RAY_SEG;
    double nuu = 0.0, ntt = 0.0;
    if (k < L - 1) {
      if (k == j0) love_fill_segment(lay, L, wvno2, om2, scr, j0);
      if (lay[k + 1].zb > 0.0) {
        ext = ext + scr.seg[k - j0][2];
        const double fact = (ext < 80.0) ? exp(-ext) : 0.0;
        nuu = scr.seg[k + 1 - j0][0] * fact * iumax;
        ntt = scr.seg[k + 1 - j0][1] * fact * iumax;
      }
    }
    const LoveLayer& y = lay[k];
    const double zb = y.zb;
    if (zb > 0.0) {
      const double drho = y.zr, dpth = y.d, dmu = y.mu;
      const double x2 = wvno2 - om2 * y.ib2;
      double rb = 0.0, irb = 0.0;
      if (x2 != 0.0) {
        irb = rsqrt(fabs(x2));
        rb = fabs(x2) * irb;
      }
      if (rb < 1.0e-10) { rb = 1.0e-10; irb = 1.0e10; }
      double upup, dupdup;
      if (k == L - 1) {
        upup = (0.5 * irb) * uu * uu;
        dupdup = (0.5 * rb) * uu * uu;
      } else {
        const bool real = !(x2 < 0.0);  // nub = rb, or i rb when wvno < xkb
        // ei11 = ei21 = 0.5/wvno, ei12 = -ei22 = 0.5/(wvno dmu nub)
        const double e0 = 0.5 * ik;
        const cx ei12 = rinv(real, 0.5 * ik * y.imu * irb);
        const cx km1dn = mkc(e0 * uu) - ei12 * tt;
        const cx kmup = mkc(e0 * nuu) + ei12 * ntt;
        const double q = rb * dpth;
        cx f, g;
        if (real) {
          const double e1 = (q < 75.0) ? exp(-q) : 0.0;
          const double e2 = (q < 40.0) ? e1 * e1 : 0.0;  // exp(-2 nub d)
          f = mkc((1.0 - e2) * 0.5 * irb, 0.0);
          g = mkc(dpth * e1, 0.0);
        } else {
          double sn, cs;
          sincos(q, &sn, &cs);
          f = mkc(sn * cs * irb, -sn * sn * irb);
          g = mkc(dpth * cs, -dpth * sn);
        }
        const cx f1 = f * (wvno2 * (kmup * kmup + km1dn * km1dn));
        const cx f2 = g * (2.0 * wvno2) * kmup * km1dn;
        upup = (f1 + f2).re;
        const double nub2 = real ? rb * rb : -rb * rb;
        dupdup = nub2 * (f1 - f2).re;
      }
      sumi0 = sumi0 + drho * upup;
      sumi1 = sumi1 + dmu * upup;
      const double VSHH = zb, VSHV = zb;
      const double DCDBH = c * drho * VSHH * upup;
      const double DCDBV = c * drho * VSHV * dupdup * ik2;
      sink.add(k, y.vtp, y.rtp, 0.0, DCDBH + DCDBV,
               0.5 * c * (-c * c * upup + VSHH * VSHH * upup + VSHV * VSHV * dupdup * ik2));
    }
    uu = nuu;
    tt = ntt;
  }
  sink.finish();
  ugr = sumi1 / (c * sumi0);
  norm = sumi1;
}

}  // namespace swdk
