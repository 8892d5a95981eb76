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
#pragma once
#include "swdk_core.cuh"

namespace swdk {

constexpr int LMAX = 320;   // sublayers per column (4*80-3 = 317)
constexpr int NZMAX = 96;   // grid nodes per column
constexpr double LN2 = 0.69314718055994530942;

// flattened eigen model of one column (bldsph), top-down index m
struct EigModel {
  const double *zd, *za, *zb, *zrho, *vtp, *rtp;
  int L;
};

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
  double* kp;         // node accumulator [nz] (null: no kernels wanted)
  const float2* crs;  // (dalpha/dbeta, drho/dalpha) per node
  int L, nw;
  SWDK_HD void add(const EigModel& M, int l, double xa, double xb, double xr) const {
    if (!kp) return;
    int n0, n1 = -1;
    double w0, w1 = 0.0;
    if (nw > 0 && l == 0) return;
    const int lp = (nw > 0) ? l - 1 : l;
    if (l == L - 1) {
      n0 = (lp >> 2) + nw;
      w0 = 4.875;
    } else {
      const double t = (double)(2 * (lp & 3) + 1) / 8.0;
      n0 = (lp >> 2) + nw;
      w0 = 1.0 - t;
      n1 = n0 + 1;
      w1 = t;
    }
    const double fa = M.vtp[l], fr = M.rtp[l];
    const double xbf = xb * fa, xaf = xa * fa, xrf = xr * fr;
    {
      const float2 c = crs[n0];
      const double dadb = c.x, drda = c.y;
      kp[n0] += w0 * (xbf + xaf * dadb + xrf * drda * dadb);
    }
    if (n1 >= 0) {
      const float2 c = crs[n1];
      const double dadb = c.x, drda = c.y;
      kp[n1] += w1 * (xbf + xaf * dadb + xrf * drda * dadb);
    }
  }
};

// ---------------------------------------------------------------------------
// varsv (sregn96.f90:827-911) for the pure real / pure imaginary vertical
// wavenumbers that cdsqrt of a real argument produces
// ---------------------------------------------------------------------------
struct Vars {
  double cosp, cosq, rsinp, rsinq, sinpr, sinqr, pex, svex;
};

SWDK_HD void varsv_real(double x2p, double x2s, double zd, int iwat, Vars& v) {
  const double tiny = (double)1.0e-5f;
  // P
  if (x2p >= 0.0) {  // rp real
    const double rp = sqrt(x2p), pr = rp * zd;
    const double pfac = (pr < 30.) ? exp(-2. * pr) : 0.0;
    v.cosp = 0.5 + pfac * 0.5;
    const double sre = 0.5 - pfac * 0.5;
    v.rsinp = rp * sre;
    v.sinpr = (fabs(pr) < tiny && rp < tiny) ? zd : sre / rp;
    v.pex = pr;
  } else {  // rp = i r
    const double r = sqrt(-x2p), pi = r * zd;
    double sp, cp;
    sincos(pi, &sp, &cp);
    v.cosp = cp;
    v.rsinp = -r * sp;
    v.sinpr = (r < tiny) ? zd : sp / r;
    v.pex = 0.0;
  }
  if (iwat == 1) {
    v.cosq = 1.0; v.rsinq = 0.0; v.sinqr = 0.0; v.svex = 0.0;
    return;
  }
  if (x2s >= 0.0) {
    const double rs = sqrt(x2s), qr = rs * zd;
    const double sfac = (qr < 30.) ? exp(-2. * qr) : 0.0;
    v.cosq = 0.5 + sfac * 0.5;
    const double sre = 0.5 - sfac * 0.5;
    v.rsinq = rs * sre;
    v.sinqr = (fabs(qr) < tiny && rs < tiny) ? zd : sre / rs;
    v.svex = qr;
  } else {
    const double r = sqrt(-x2s), qi = r * zd;
    double sq, cq;
    sincos(qi, &sq, &cq);
    v.cosq = cq;
    v.rsinq = -r * sq;
    v.sinqr = (r < tiny) ? zd : sq / r;
    v.svex = 0.0;
  }
}

// dnka of sregn96 (REAL*4 rho, b); ca[i][j] = CA(i+1,j+1)
SWDK_HD void dnka_r(double ca[5][5], const Vars& v, float rho, float b, int iwat, double wvno, double wvno2,
                    double om2) {
  const double ex = v.pex, exa = v.pex + v.svex;
  if (iwat == 1) {
    for (int i = 0; i < 5; ++i)
      for (int j = 0; j < 5; ++j) ca[i][j] = 0.0;
    const double dfac = (ex > 35.0) ? 0.0 : exp(-ex);
    ca[2][2] = dfac;
    ca[0][0] = v.cosp;
    ca[4][4] = v.cosp;
    ca[0][1] = -v.rsinp / ((double)rho * om2);
    ca[1][0] = -((double)rho * v.sinpr * om2);
    ca[1][1] = v.cosp;
    ca[3][3] = v.cosp;
    ca[3][4] = ca[0][1];
    ca[4][3] = ca[1][0];
    return;
  }
  const double a0 = (exa < 60.0) ? exp(-exa) : 0.0;
  const double cosp = v.cosp, cossv = v.cosq, rsinp = v.rsinp, rsinsv = v.rsinq, sinpr = v.sinpr,
               sinsvr = v.sinqr;
  const double cpcq = cosp * cossv, cpy = cosp * sinsvr, cpz = cosp * rsinsv, cqw = cossv * sinpr,
               cqx = cossv * rsinp;
  const double xy = rsinp * sinsvr, xz = rsinp * rsinsv, wy = sinpr * sinsvr, wz = sinpr * rsinsv;
  const float rho2 = rho * rho;
  const double gam = (double)(2.0f * b * b) * wvno2 / om2;
  const double gam2 = gam * gam, gamm1 = gam - 1., gamm2 = gamm1 * gamm1;
  const double cqww2 = cqw * wvno2, cqxw2 = cqx / wvno2, gg1 = gam * gamm1;
  const double a0c = 2.0 * (a0 - cpcq);
  const double xz2 = xz / wvno2, gxz2 = gam * xz2, g2xz2 = gam2 * xz2;
  const double a0cgg1 = a0c * (gam + gamm1);
  const double wy2 = wy * wvno2, g2wy2 = gamm2 * wy2, g1wy2 = gamm1 * wy2;
  const double rhod = (double)rho, rho2d = (double)rho2;
  const double rom2 = rhod * om2;
  double temp = a0c * gg1 + g2xz2 + g2wy2;
  ca[2][2] = a0 + temp + temp;
  ca[0][0] = cpcq - temp;
  ca[0][1] = (-cqx + wvno2 * cpy) / rom2;
  temp = 0.5 * a0cgg1 + gxz2 + g1wy2;
  ca[0][2] = wvno * temp / rom2;
  ca[0][3] = (-cqww2 + cpz) / rom2;
  temp = wvno2 * (a0c + wy2) + xz;
  ca[0][4] = -temp / (rho2d * om2 * om2);
  ca[1][0] = (-gamm2 * cqw + gam2 * cpz / wvno2) * rhod * om2;
  ca[1][1] = cpcq;
  ca[1][2] = (gamm1 * cqww2 - gam * cpz) / wvno;
  ca[1][3] = -wz;
  ca[1][4] = ca[0][3];
  temp = 0.5 * a0cgg1 * gg1 + gam2 * gxz2 + gamm2 * g1wy2;
  ca[2][0] = -2.0 * temp * rhod * om2 / wvno;
  ca[2][1] = (-wvno * (gam * cqxw2 - gamm1 * cpy)) * 2.0;
  ca[2][3] = -2.0 * ca[1][2];
  ca[2][4] = -2.0 * ca[0][2];
  ca[3][0] = (-gam2 * cqxw2 + gamm2 * cpy) * rhod * om2;
  ca[3][1] = -xy;
  ca[3][2] = -ca[2][1] / 2.0;
  ca[3][3] = ca[1][1];
  ca[3][4] = ca[0][1];
  temp = gamm2 * (a0c * gam2 + g2wy2) + gam2 * g2xz2;
  ca[4][0] = -rho2d * om2 * om2 * temp / wvno2;
  ca[4][1] = ca[3][0];
  ca[4][2] = -ca[2][0] / 2.0;
  ca[4][3] = ca[1][0];
  ca[4][4] = ca[0][0];
}

// hska (sregn96.f90:913-987)
SWDK_HD void hska_r(double AA[4][4], const Vars& v, float rho, float b, int iwat, double wvno, double wvno2,
                    double om2) {
  const double rhod = (double)rho;
  if (iwat == 1) {
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) AA[i][j] = 0.0;
    const double dfac = (v.pex > 35.0) ? 0.0 : exp(-v.pex);
    AA[0][0] = dfac;
    AA[3][3] = dfac;
    AA[1][1] = v.cosp;
    AA[2][2] = v.cosp;
    AA[1][2] = -v.rsinp / (rhod * om2);
    AA[2][1] = -(rhod * om2 * v.sinpr);
    return;
  }
  const double dfac = ((v.pex - v.svex) > 70.0) ? 0.0 : exp(v.svex - v.pex);
  const double cossv = dfac * v.cosq, rsinsv = dfac * v.rsinq, sinsvr = dfac * v.sinqr;
  const double cosp = v.cosp, rsinp = v.rsinp, sinpr = v.sinpr;
  const double gam = (double)(2.0f * b * b) * wvno2 / om2;
  const double gamm1 = gam - 1.0;
  const double rom2 = rhod * om2;
  AA[0][0] = cossv + gam * (cosp - cossv);
  AA[0][1] = -wvno * gamm1 * sinpr + gam * rsinsv / wvno;
  AA[0][2] = -(wvno * (cosp - cossv) / rom2);
  AA[0][3] = (wvno2 * sinpr - rsinsv) / rom2;
  AA[1][0] = gam * rsinp / wvno - wvno * gamm1 * sinsvr;
  AA[1][1] = cosp - gam * (cosp - cossv);
  AA[1][2] = (-rsinp + wvno2 * sinsvr) / rom2;
  AA[1][3] = -AA[0][2];
  AA[2][0] = rom2 * gam * gamm1 * (cosp - cossv) / wvno;
  AA[2][1] = rom2 * (-gamm1 * gamm1 * sinpr + gam * gam * rsinsv / wvno2);
  AA[2][2] = AA[1][1];
  AA[2][3] = -AA[0][1];
  AA[3][0] = rom2 * (gam * gam * rsinp / wvno2 - gamm1 * gamm1 * sinsvr);
  AA[3][1] = -AA[2][0];
  AA[3][2] = -AA[1][0];
  AA[3][3] = AA[0][0];
}

// evalg with jbdry = 0 (sregn96.f90:649-825); solid or fluid layer m
struct EMat {
  cx ra, rb;
  cx e[4][4], ei[4][4];
};

SWDK_HD void evalg_r(const EigModel& M, int m, int iwat, bool allfluid, double wvno, double om, double om2,
                     double wvno2, EMat& E, cx* gbr) {
  const double xka = om / M.za[m];
  const double xkb = (M.zb[m] > 0.0) ? om / M.zb[m] : 0.0;
  E.ra = csqrt_real(wvno2 - xka * xka);
  E.rb = csqrt_real(wvno2 - xkb * xkb);
  double gam = M.zb[m] * wvno / om;
  gam = 2.0 * (gam * gam);
  const double gamm1 = gam - 1.0;
  const cx ra = E.ra, rb = E.rb;
  const double zr = M.zrho[m];
  if (iwat == 0) {
    const double g1 = zr * om2 * gamm1, g2 = zr * om2 * gam;
    E.e[0][0] = mkc(wvno); E.e[0][1] = rb; E.e[0][2] = mkc(wvno); E.e[0][3] = -rb;
    E.e[1][0] = ra; E.e[1][1] = mkc(wvno); E.e[1][2] = -ra; E.e[1][3] = mkc(wvno);
    E.e[2][0] = mkc(g1); E.e[2][1] = g2 * rb / wvno; E.e[2][2] = mkc(g1); E.e[2][3] = -(g2 * rb / wvno);
    E.e[3][0] = g2 * ra / wvno; E.e[3][1] = mkc(g1); E.e[3][2] = -(g2 * ra / wvno); E.e[3][3] = mkc(g1);
    const double h1 = 0.5 * gam / wvno, h2 = -(0.5 / (zr * om2));
    const cx iga = (0.5 * gamm1) / ra, igb = (0.5 * gamm1) / rb;
    const cx wa = (0.5 * wvno) / ((zr * om2) * ra), wb = (0.5 * wvno) / ((zr * om2) * rb);
    E.ei[0][0] = mkc(h1); E.ei[0][1] = -iga; E.ei[0][2] = mkc(h2); E.ei[0][3] = wa;
    E.ei[1][0] = -igb; E.ei[1][1] = mkc(h1); E.ei[1][2] = wb; E.ei[1][3] = mkc(h2);
    E.ei[2][0] = mkc(h1); E.ei[2][1] = iga; E.ei[2][2] = mkc(h2); E.ei[2][3] = -wa;
    E.ei[3][0] = igb; E.ei[3][1] = mkc(h1); E.ei[3][2] = -wb; E.ei[3][3] = mkc(h2);
    if (gbr) {
      gbr[0] = (zr * zr * om2 * om2) * (-((gam * gam) * ra * rb) + wvno2 * gamm1 * gamm1);
      gbr[1] = -((zr * (wvno2 * ra)) * om2);
      gbr[2] = -(((zr * (-((gam * ra) * rb) + wvno2 * gamm1)) * om2) * wvno);
      gbr[3] = (zr * (wvno2 * rb)) * om2;
      gbr[4] = wvno2 * (wvno2 - ra * rb);
      const cx den = -((zr * zr * om2 * om2 * wvno2) * ra * rb);
      for (int i = 0; i < 5; ++i) gbr[i] = (0.25 * gbr[i]) / den;
    }
  } else {
    if (gbr) {
      if (allfluid) {
        gbr[0] = 0.5 / ra;
        gbr[1] = mkc(0.5) / mkc(-(zr * om2));
        gbr[2] = mkc(0); gbr[3] = mkc(0); gbr[4] = mkc(0);
      } else {
        gbr[0] = mkc(0); gbr[1] = mkc(0); gbr[2] = mkc(0);
        gbr[3] = (0.5 * zr * om2) / ra;
        gbr[4] = mkc(-0.5);
      }
    }
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) { E.e[i][j] = mkc(0); E.ei[i][j] = mkc(0); }
    E.e[0][0] = ra; E.e[0][1] = -ra;
    E.e[1][0] = mkc(-(zr * om2)); E.e[1][1] = mkc(-(zr * om2));
    E.ei[0][0] = 0.5 / ra;
    E.ei[0][1] = mkc(-(0.5 / (zr * om2)));
    E.ei[1][0] = -(0.5 / ra);
    E.ei[1][1] = mkc(-(0.5 / (zr * om2)));
  }
}

SWDK_HD cx ffunc_c(cx nub, double dm) {
  if (cabsc(nub) < 1.0e-08) return mkc(dm);
  const cx argcd = nub * dm;
  const cx exqq = (argcd.re < 40.0) ? cexpc(-2.0 * argcd) : mkc(0.0);
  return (1.0 - exqq) / (2.0 * nub);
}
SWDK_HD cx gfunc_c(cx nub, double dm) {
  const cx argcd = nub * dm;
  if (argcd.re < 75) return cexpc(-argcd) * dm;
  return mkc(0.0);
}
SWDK_HD cx h1func_c(cx nua, cx nub, double dm) {
  if (cabsc(nub + nua) < 1.0e-08) return mkc(dm);
  const cx argcd = (nua + nub) * dm;
  const cx exqq = (argcd.re < 40.0) ? cexpc(-argcd) : mkc(0.0);
  return (1.0 - exqq) / (nub + nua);
}
SWDK_HD cx h2func_c(cx nua, cx nub, double dm) {
  if (cabsc(nub - nua) < 1.0e-08) return mkc(dm);
  cx argcd = nua * dm;
  const cx exqp = (argcd.re < 40.0) ? cexpc(-argcd) : mkc(0.0);
  argcd = nub * dm;
  const cx exqq = (argcd.re < 40.0) ? cexpc(-argcd) : mkc(0.0);
  return (exqq - exqp) / (nua - nub);
}

// Eigenfunction values at a layer top: (ur, uz, tz, tr)
struct Eig4 {
  double ur, uz, tz, tr;
};


struct EnergyAcc {
  double sumi0, sumi1, sumi2, sumi3;
};

// energy() body for one layer m (sregn96.f90:1097-1178); writes the raw
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
// exp(-2 ra d), exp(-(ra+rb) d) are products of exp(-ra d), exp(-rb d).
SWDK_HD double re_mul(cx a, cx b) { return a.re * b.re - a.im * b.im; }
SWDK_HD cx cinv(cx a) {  // 1/a for pure real or pure imaginary a
  if (a.im == 0.0) return mkc(1.0 / a.re, 0.0);
  if (a.re == 0.0) return mkc(0.0, -1.0 / a.im);
  return mkc(1.0) / a;
}

SWDK_HD void energy_layer_r(const EigModel& M, int m, int iwat, bool allfluid, const Eig4& u0, const Eig4& u1,
                            double om, double om2, double wvno, double wvno2, double c, EnergyAcc& acc,
                            double& dcda, double& dcdb, double& dcdr) {
  (void)allfluid;
  const int typelyr = (m == M.L - 1) ? 1 : 0;
  const double za = M.za[m], zb = M.zb[m], zr = M.zrho[m], zdm = M.zd[m];
  const double xka = om / za;
  const double xkb = (zb > 0.0) ? om / zb : 0.0;
  const double ra2 = wvno2 - xka * xka, rb2 = wvno2 - xkb * xkb;
  const cx ra = csqrt_real(ra2), rb = csqrt_real(rb2);
  double gam = zb * wvno / om;
  gam = 2.0 * (gam * gam);
  const double gamm1 = gam - 1.0;
  const double rom2 = zr * om2;
  double INT11, INT13 = 0.0, INT22, INT24 = 0.0, INT33 = 0.0, INT44 = 0.0;
  // exp(-ra d), exp(-rb d) with the reference's cut-offs applied by the users
  auto cexp_neg = [](cx r, double d) { return cexpc(mkc(-r.re * d, -r.im * d)); };
  if (iwat == 0) {
    const double g1 = rom2 * gamm1, g2 = rom2 * gam / wvno;
    const double h1 = 0.5 * gam / wvno, h2 = -(0.5 / rom2), ga = 0.5 * gamm1, wa = 0.5 * wvno / rom2;
    const cx ira = cinv(ra), irb = cinv(rb);
    const cx km1pd = (h1 * u0.ur + h2 * u0.tz) + (ga * u0.uz - wa * u0.tr) * ira;
    const cx km1sd = (ga * u0.ur - wa * u0.tz) * irb + (h1 * u0.uz + h2 * u0.tr);
    const double k = wvno, k2 = wvno2;
    // pair coefficients: P (real), Q (real), X = xr * r (r = ra or rb)
    if (typelyr == 0) {
      const cx kmpu = (h1 * u1.ur + h2 * u1.tz) - (ga * u1.uz - wa * u1.tr) * ira;
      const cx kmsu = (h1 * u1.uz + h2 * u1.tr) - (ga * u1.ur - wa * u1.tz) * irb;
      // FA, GA, FB, GB, H1, H2 (sregn96.f90:1319-1397)
      const cx ard = ra * zdm, brd = rb * zdm;
      const cx ea = (ard.re < 75.0) ? cexp_neg(ra, zdm) : mkc(0.0);
      const cx eb = (brd.re < 75.0) ? cexp_neg(rb, zdm) : mkc(0.0);
      const cx ea40 = (ard.re < 40.0) ? ea : mkc(0.0);
      const cx eb40 = (brd.re < 40.0) ? eb : mkc(0.0);
      const cx FA = (cabsc(ra) < 1.0e-08) ? mkc(zdm) : (1.0 - ea40 * ea40) / (2.0 * ra);
      const cx FB = (cabsc(rb) < 1.0e-08) ? mkc(zdm) : (1.0 - eb40 * eb40) / (2.0 * rb);
      const cx GA = ea * zdm, GB = eb * zdm;
      const cx sab = ra + rb;
      const cx H1 = (cabsc(sab) < 1.0e-08) ? mkc(zdm)
                    : (1.0 - ((((ard + brd).re) < 40.0) ? ea * eb : mkc(0.0))) / sab;
      const cx dab = ra - rb;
      const cx H2 = (cabsc(dab) < 1.0e-08) ? mkc(zdm) : (eb40 - ea40) / dab;
      const cx pp = kmpu * kmpu + km1pd * km1pd, ss = kmsu * kmsu + km1sd * km1sd;
      const cx pd = kmpu * km1pd, sd = kmsu * km1sd;
      const cx x1 = kmpu * kmsu - km1pd * km1sd, x2 = km1pd * kmsu - kmpu * km1sd;
      const cx FApp = FA * pp, GApd2 = 2.0 * (GA * pd), FBss = FB * ss, GBsd2 = 2.0 * (GB * sd);
      const cx H1x = H1 * x1, H2x = H2 * x2;
      const cx SAp = FApp + GApd2, SAm = FApp - GApd2;
      const cx SBp = FBss - GBsd2, SBm = FBss + GBsd2;
      const cx SXp = H1x + H2x, SXm = H1x - H2x;
      INT11 = k2 * SAp.re + rb2 * SBp.re + 2.0 * k * re_mul(rb, SXp);
      INT13 = k * g1 * SAp.re + g2 * rb2 * SBp.re + (k * g2 + g1) * re_mul(rb, SXp);
      INT33 = g1 * g1 * SAp.re + g2 * g2 * rb2 * SBp.re + 2.0 * g1 * g2 * re_mul(rb, SXp);
      INT22 = ra2 * SAm.re + k2 * SBm.re + 2.0 * k * re_mul(ra, SXm);
      INT24 = g2 * ra2 * SAm.re + k * g1 * SBm.re + (g1 + k * g2) * re_mul(ra, SXm);
      INT44 = g2 * g2 * ra2 * SAm.re + g1 * g1 * SBm.re + 2.0 * g1 * g2 * re_mul(ra, SXm);
    } else {
      const cx TA = (km1pd * km1pd) / (2.0 * ra), TB = (km1sd * km1sd) / (2.0 * rb);
      const cx TX = -((km1pd * km1sd) / (ra + rb));
      INT11 = k2 * TA.re + rb2 * TB.re + 2.0 * k * re_mul(rb, TX);
      INT13 = k * g1 * TA.re + g2 * rb2 * TB.re + (k * g2 + g1) * re_mul(rb, TX);
      INT33 = g1 * g1 * TA.re + g2 * g2 * rb2 * TB.re + 2.0 * g1 * g2 * re_mul(rb, TX);
      INT22 = ra2 * TA.re + k2 * TB.re + 2.0 * k * re_mul(ra, TX);
      INT24 = g2 * ra2 * TA.re + k * g1 * TB.re + (g1 + k * g2) * re_mul(ra, TX);
      INT44 = g2 * g2 * ra2 * TA.re + g1 * g1 * TB.re + 2.0 * g1 * g2 * re_mul(ra, TX);
    }
  } else {
    // fluid layer: 2x2 E = [[ra, -ra], [-rho om2, -rho om2]] (sregn96.f90:791-801)
    const cx ira = cinv(ra);
    const double ir = -(0.5 / rom2);
    const cx km1pd = (-0.5 * u0.uz) * ira + ir * u0.tz;
    const double w = -rom2;
    if (typelyr == 0) {
      const cx kmpu = (0.5 * u1.uz) * ira + ir * u1.tz;
      const cx ard = ra * zdm;
      const cx ea = (ard.re < 75.0) ? cexp_neg(ra, zdm) : mkc(0.0);
      const cx ea40 = (ard.re < 40.0) ? ea : mkc(0.0);
      const cx FA = (cabsc(ra) < 1.0e-08) ? mkc(zdm) : (1.0 - ea40 * ea40) / (2.0 * ra);
      const cx GA = ea * zdm;
      const cx sq = (kmpu * kmpu + km1pd * km1pd) * FA, cr = 2.0 * (kmpu * km1pd * GA);
      INT11 = ra2 * (sq - cr).re;
      INT22 = w * w * (sq + cr).re;
    } else {
      const cx t = (km1pd * km1pd) / (2.0 * ra);
      INT11 = 0.0;
      INT22 = w * w * t.re;
    }
  }
  // getmat (sregn96.f90:1531-1583) and the energy sums
  const double rho = zr, ah = za, av = za, eta = 1.0;
  const double TA = zr * za * za, TC = zr * za * za;
  if (iwat == 1) {
    const double TN = 0.0, TF = TA - 2. * TN;
    const double a12 = -(wvno * wvno - om * om / (ah * ah)) / (rho * om * om);
    const double wr = wvno / (rho * om2);
    const double URUR = INT22 * (wr * wr), UZUZ = INT11;
    const double URDUZ = -((wvno / (rho * om2)) * a12 * INT22);
    const double DUZDUZ = a12 * a12 * INT22;
    acc.sumi0 = acc.sumi0 + rho * (URUR + UZUZ);
    acc.sumi1 = acc.sumi1 + TA * URUR;
    acc.sumi2 = acc.sumi2 - TF * URDUZ;
    acc.sumi3 = acc.sumi3 + TC * DUZDUZ;
    const double facah = rho * ah * (URUR - 2. * eta * URDUZ / wvno);
    const double facav = rho * av * DUZDUZ / wvno2;
    dcda = facah + facav;
    dcdb = 0.0;
    const double facr = -(0.5 * c * c * (URUR + UZUZ));
    dcdr = 0.5 * (av * facav + ah * facah) / rho + facr;
  } else {
    const double bv = zb;
    const double TL = zr * zb * zb;
    const double TF = TA - 2. * TL;
    const double a12 = -wvno, a14 = 1.0 / TL, a21 = wvno * TF / TC, a23 = 1.0 / TC;
    const double URUR = INT11, UZUZ = INT22;
    const double DURDUR = a12 * a12 * INT22 + 2. * a12 * a14 * INT24 + a14 * a14 * INT44;
    const double DUZDUZ = a21 * a21 * INT11 + 2. * a21 * a23 * INT13 + a23 * a23 * INT33;
    const double URDUZ = a21 * INT11 + a23 * INT13;
    const double UZDUR = a12 * INT22 + a14 * INT24;
    acc.sumi0 = acc.sumi0 + rho * (URUR + UZUZ);
    acc.sumi1 = acc.sumi1 + TL * UZUZ + TA * URUR;
    acc.sumi2 = acc.sumi2 + TL * UZDUR - TF * URDUZ;
    acc.sumi3 = acc.sumi3 + TL * DURDUR + TC * DUZDUZ;
    const double facah = rho * ah * (URUR - 2. * eta * URDUZ / wvno);
    const double facav = rho * av * DUZDUZ / wvno2;
    const double facbv = rho * bv * (UZUZ + 2. * UZDUR / wvno + DURDUR / wvno2 + 4. * eta * URDUZ / wvno);
    dcda = facah + facav;
    dcdb = facbv;
    const double facr = -(0.5 * c * c * (URUR + UZUZ));
    dcdr = 0.5 * (av * facav + ah * facah + bv * facbv) / rho + facr;
  }
}

// svfunc eigenfunction at layer top i from the compound (cd) and Haskell (vv)
// vectors (sregn96.f90:279-312)
SWDK_HD Eig4 eigen_at(const double* cd, const double* vv, double ext, double f1213) {
  const double cd1 = cd[0], cd2 = cd[1], cd3 = cd[2], cd4 = -cd[2], cd5 = cd[3], cd6 = cd[4];
  const double tz1 = -vv[3], tz2 = -vv[2], tz3 = vv[1], tz4 = vv[0];
  const double uu1 = tz2 * cd6 - tz3 * cd5 + tz4 * cd4;
  const double uu2 = -tz1 * cd6 + tz3 * cd3 - tz4 * cd2;
  const double uu3 = tz1 * cd5 - tz2 * cd3 + tz4 * cd1;
  const double uu4 = -tz1 * cd4 + tz2 * cd2 - tz3 * cd1;
  Eig4 u;
  if (ext > -80.0 && ext < 80.0) {
    const double fact = exp(ext);
    u.ur = uu1 * fact / f1213;
    u.uz = uu2 * fact / f1213;
    u.tz = uu3 * fact / f1213;
    u.tr = uu4 * fact / f1213;
  } else {
    u.ur = 0.0; u.uz = 0.0; u.tz = 0.0; u.tr = 0.0;
  }
  return u;
}

// Scratch of one Rayleigh pass: per layer 6 doubles (cd[5], exe), reused for
// the raw layer kernels (dcda, dcdb, dcdr) once the layer has been consumed.
// Returns ugr (flat) and norm = ugr*sumi0; scr[6m+0..2] = raw dcda/dcdb/dcdr.
SWDK_HDI void rayleigh_pass(const EigModel& M, bool allfluid, double omega, double wvno, double* scr, double& ugr,
                            double& norm, const NodeSink& sink) {
  const int L = M.L;
  const double wvno2 = wvno * wvno, om2 = omega * omega;
  // ---- up (sregn96.f90:401-489) ----
  {
    cx gbr[5];
    EMat E;
    const int iw = (M.zb[L - 1] > 0.0) ? 0 : 1;
    evalg_r(M, L - 1, iw, allfluid, wvno, omega, om2, wvno2, E, gbr);
    double* c0 = scr + 6 * (L - 1);
    for (int j = 0; j < 5; ++j) c0[j] = gbr[j].re;
    c0[5] = 0.0;
  }
  double exr = 0.0;
  int exi = 0;
  double ca[5][5];
#pragma unroll 1  // a layer recursion: unrolling only grows the code
  for (int m = L - 2; m >= 0; --m) {
    const double zam = M.za[m], zbm = M.zb[m], zdm = M.zd[m];
    const int iw = (zbm > 0.0) ? 0 : 1;
    const double xka = omega / zam;
    const double xkb = (zbm > 0.0) ? omega / zbm : 0.0;
    Vars v;
    varsv_real(wvno2 - xka * xka, wvno2 - xkb * xkb, zdm, iw, v);
    dnka_r(ca, v, (float)M.zrho[m], (float)zbm, iw, wvno, wvno2, om2);
    const double* cp = scr + 6 * (m + 1);
    double ee[5];
    for (int i = 0; i < 5; ++i) {
      double cr = 0.0;
      for (int j = 0; j < 5; ++j) cr = cr + cp[j] * ca[j][i];
      ee[i] = cr;
    }
    double t1 = 0.0;
    for (int i = 0; i < 5; ++i) t1 = fmax(t1, fabs(ee[i]));
    int e = 0;
    if (t1 >= 1.e-40) e = pow2_exponent(t1);
    double* cm = scr + 6 * m;
    for (int i = 0; i < 5; ++i) cm[i] = ldexp(ee[i], -e);
    exr = exr + v.pex + v.svex;
    exi += e;
    cm[5] = exr + (double)exi * LN2;
  }
  // ---- down + svfunc + energy, top-down ----
  const double f1213 = -scr[1];
  const double exe0 = scr[5];
  Eig4 u0;
  u0.ur = scr[2] / scr[1];
  u0.uz = 1.0; u0.tz = 0.0; u0.tr = 0.0;
  if (M.zb[0] <= 0.0 && !allfluid) { u0.ur = 0.0; u0.tr = 0.0; }  // fluid top (jwat)
  double vv[4] = {1.0, 0.0, 0.0, 0.0};
  double dxr = 0.0;
  int dxi = 0;
  EnergyAcc acc = {0.0, 0.0, 0.0, 0.0};
  const double c = omega / wvno;
  double AA[4][4];
#pragma unroll 1  // a layer recursion: unrolling only grows the code
  for (int m = 0; m < L; ++m) {
    const double zbm = M.zb[m];
    const int iw = (zbm > 0.0) ? 0 : 1;
    Eig4 u1 = u0;
    if (m < L - 1) {
      const double zam = M.za[m], zdm = M.zd[m];
      const double xka = omega / zam;
      const double xkb = (zbm > 0.0) ? omega / zbm : 0.0;
      Vars v;
      varsv_real(wvno2 - xka * xka, wvno2 - xkb * xkb, zdm, iw, v);
      hska_r(AA, v, (float)M.zrho[m], (float)zbm, iw, wvno, wvno2, om2);
      double a0[4];
      for (int i = 0; i < 4; ++i) {
        double cc = 0.0;
        for (int j = 0; j < 4; ++j) cc = cc + AA[i][j] * vv[j];
        a0[i] = cc;
      }
      double t1 = fmax(fmax(fabs(a0[0]), fabs(a0[1])), fmax(fabs(a0[2]), fabs(a0[3])));
      int e = 0;
      if (t1 >= 1.e-40) e = pow2_exponent(t1);
      for (int i = 0; i < 4; ++i) vv[i] = ldexp(a0[i], -e);
      dxr = dxr + v.pex;
      dxi += e;
      const double exa1 = dxr + (double)dxi * LN2;
      const double* cd1 = scr + 6 * (m + 1);
      u1 = eigen_at(cd1, vv, exa1 + cd1[5] - exe0, f1213);
    }
    double da, db, dr;
    energy_layer_r(M, m, iw, allfluid, u0, u1, omega, om2, wvno, wvno2, c, acc, da, db, dr);
    sink.add(M, m, da, db, dr);
    u0 = u1;
  }
  ugr = (wvno * acc.sumi1 + acc.sumi2) / (omega * acc.sumi0);
  norm = ugr * acc.sumi0;
}

// ---------------------------------------------------------------------------
// Love pass (slegn96.f90): up, shfunc normalisation, energy.  scr holds 3
// doubles per layer (uu, tt, exl) then the raw (dcdb, dcdr).  Returns ugr and
// the normaliser sumi1.
// ---------------------------------------------------------------------------
SWDK_HDI void love_pass(const EigModel& M, double omega, double wvno, double* scr, double& ugr, double& norm,
                        const NodeSink& sink) {
  const int L = M.L;
  const double wvno2 = wvno * wvno;
  // ---- up (slegn96.f90:372-445) ----
  {
    double* s0 = scr + 3 * (L - 1);
    if (M.zb[L - 1] > (double)0.01f) {
      const double zb = M.zb[L - 1];
      const double xkb = omega / zb;
      const double rb = sqrt((wvno + xkb) * fabs(wvno - xkb));
      s0[0] = 1.0;
      s0[1] = -(M.zrho[L - 1] * (zb * zb)) * rb;
    } else {
      s0[0] = 1.0;
      s0[1] = 0.0;
    }
    s0[2] = 0.0;
  }
#pragma unroll 1  // a layer recursion: unrolling only grows the code
  for (int k = L - 2; k >= 0; --k) {
    double* sk = scr + 3 * k;
    const double zb = M.zb[k];
    if (!(zb > 0.0)) { sk[0] = 0.0; sk[1] = 0.0; sk[2] = 0.0; continue; }
    const double dpth = M.zd[k];
    const double xkb = omega / zb;
    const double rb = sqrt((wvno + xkb) * fabs(wvno - xkb));
    const double q = rb * dpth;
    const double mu = M.zrho[k] * zb * zb;
    double cosq, yl, zl, eexl = 0.0;
    if (wvno < xkb) {
      double sq, cq;
      sincos(q, &sq, &cq);
      yl = sq / rb; zl = -rb * sq; cosq = cq;
    } else if (wvno == xkb) {
      cosq = 1.0; yl = dpth; zl = 0.0;
    } else {
      eexl = q;
      const double fac = (q < 18.0) ? exp(-2.0 * q) : 0.0;
      cosq = (1.0 + fac) * 0.5;
      const double sq = (1.0 - fac) * 0.5;
      yl = sq / rb; zl = rb * sq;
    }
    const double a11 = cosq, a22 = cosq, a12 = -(yl / mu), a21 = -(zl * mu);
    const double* s1 = scr + 3 * (k + 1);
    const double amp0 = a11 * s1[0] + a12 * s1[1];
    const double str0 = a21 * s1[0] + a22 * s1[1];
    const double rr = fmax(fabs(amp0), fabs(str0));
    int e = 0;
    if (rr >= 1.e-30) e = pow2_exponent(rr);
    sk[0] = ldexp(amp0, -e);
    sk[1] = ldexp(str0, -e);
    sk[2] = (double)e * LN2 + eexl;
  }
  // ---- shfunc normalisation (slegn96.f90:212-240) ----
  double ext = 0.0;
  double umax = scr[0];
  scr[1] = 0.0;  // tt(1) = 0
#pragma unroll 1  // a layer recursion: unrolling only grows the code
  for (int k = 1; k < L; ++k) {
    double* sk = scr + 3 * k;
    if (M.zb[k] > 0.0) {
      ext = ext + scr[3 * (k - 1) + 2];
      const double fact = (ext < 80.0) ? 1. / exp(ext) : 0.0;
      sk[0] = sk[0] * fact;
      sk[1] = sk[1] * fact;
    } else {
      sk[0] = 0.0; sk[1] = 0.0;
    }
    if (fabs(sk[0]) > fabs(umax)) umax = sk[0];
  }
  if (scr[0] != 0.0) umax = scr[0];
  const double iumax = (fabs(umax) > 0.0) ? 1.0 / umax : 1.0;
  // ---- energy (slegn96.f90:447-576) with uu/tt scaled by 1/umax on the fly ----
  const double c = omega / wvno;
  double sumi0 = 0.0, sumi1 = 0.0;
  double prev_uu = scr[0] * iumax, prev_tt = scr[1] * iumax;
#pragma unroll 1  // a layer recursion: unrolling only grows the code
  for (int k = 0; k < L; ++k) {
    const double uu = prev_uu, tt = prev_tt;
    double nuu = 0.0, ntt = 0.0;
    if (k < L - 1) {
      nuu = scr[3 * (k + 1)] * iumax;
      ntt = scr[3 * (k + 1) + 1] * iumax;
    }
    prev_uu = nuu;
    prev_tt = ntt;
    const double zb = M.zb[k];
    if (!(zb > 0.0)) continue;
    const double zr = M.zrho[k];
    const double TN = zr * zb * zb;
    const double drho = zr, dpth = M.zd[k];
    const double xkb = omega / zb;
    double rb = sqrt((wvno + xkb) * fabs(wvno - xkb));
    const double dmu = zr * (zb * zb);
    if (rb < 1.0e-10) rb = 1.0e-10;
    double upup, dupdup;
    if (k == L - 1) {
      upup = (0.5 / rb) * uu * uu;
      dupdup = (0.5 * rb) * uu * uu;
    } else {
      cx nub = mkc(rb, 0.0);
      if (wvno < xkb) nub = mkc(0.0, rb);
      const cx xnub = dmu * nub;
      const cx ei11 = mkc(0.5 / wvno), ei12 = 0.5 / (wvno * xnub), ei21 = mkc(0.5 / wvno),
               ei22 = -(0.5 / (wvno * xnub));
      const cx el11 = mkc(wvno), el12 = mkc(wvno);
      const cx km1dn = ei21 * uu + ei22 * tt;
      const cx kmup = ei11 * nuu + ei12 * ntt;
      const cx f3 = nub * dpth;
      cx exqq = mkc(0.0);
      if (f3.re < 40.0) exqq = cexpc(-2.0 * f3);
      const cx f = (1.0 - exqq) / (2.0 * nub);
      exqq = mkc(0.0);
      if (f3.re < 75.0) exqq = cexpc(-f3);
      const cx g = dpth * exqq;
      const cx f1 = f * (el11 * el11 * kmup * kmup + el12 * el12 * km1dn * km1dn);
      const cx f2 = g * (el11 * el12 + el11 * el12) * kmup * km1dn;
      upup = (f1 + f2).re;
      dupdup = (nub * nub * (f1 - f2)).re;
    }
    sumi0 = sumi0 + drho * upup;
    sumi1 = sumi1 + TN * upup;
    const double VSHH = zb, VSHV = zb;
    const double DCDBH = c * drho * VSHH * upup;
    const double DCDBV = c * drho * VSHV * dupdup / wvno2;
    sink.add(M, k, 0.0, DCDBH + DCDBV, 0.5 * c * (-c * c * upup + VSHH * VSHH * upup + VSHV * VSHV * dupdup / wvno2));
  }
  ugr = sumi1 / (c * sumi0);
  norm = sumi1;
}

// ---------------------------------------------------------------------------
// _ParamConvert (SurfaceWave.cpp:59-101) of x(l) = raw(l)/norm * fac(l)
// into node values out[0..nz-1]; nw leading fluid nodes.
// raw(l) = scr[stride*l + off]
// ---------------------------------------------------------------------------
SWDK_HD double layer_val(const double* scr, int stride, int off, int l, double norm, const double* fac) {
  return (scr[stride * l + off] / norm) * fac[l];
}

SWDK_HDI void param_convert_dev(const double* scr, int stride, int off, double norm, const double* fac, int L, int nz,
                                int nw, double* out) {
  const int n = 4;
  if (nw == 0) {
    for (int i = 0; i < nz; ++i) {
      double tup = 0.0, tdwn = 0.0;
      const int idup = (i - 1) * n, iddw = i * n;
      for (int j = 0; j < n; ++j) {
        const double tmp = (2. * j + 1.0) / (2. * n);
        if (idup + j >= 0) tup += layer_val(scr, stride, off, idup + j, norm, fac) * tmp;
        if (iddw + j < L) tdwn += layer_val(scr, stride, off, iddw + j, norm, fac) * (1.0 - tmp);
        if (iddw == L - 1) tdwn += layer_val(scr, stride, off, L - 1, norm, fac);
      }
      out[i] = 0.0 + (tup + tdwn);
    }
  } else {
    out[0] = layer_val(scr, stride, off, 0, norm, fac);
    for (int i = 1; i < nw; ++i) out[i] = 0.0;
    for (int i = nw; i < nz; ++i) {
      double tup = 0.0, tdwn = 0.0;
      const int idup = (i - nw - 1) * n + 1, iddw = (i - nw) * n + 1;
      for (int j = 0; j < n; ++j) {
        const double tmp = (2. * j + 1.0) / (2. * n);
        if (idup + j >= 1) tup += layer_val(scr, stride, off, idup + j, norm, fac) * tmp;
        if (iddw + j < L) tdwn += layer_val(scr, stride, off, iddw + j, norm, fac) * (1.0 - tmp);
        if (iddw == L - 1) tdwn += layer_val(scr, stride, off, L - 1, norm, fac);
      }
      out[i] = 0.0 + (tup + tdwn);
    }
  }
}

}  // namespace swdk
