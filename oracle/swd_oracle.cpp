// ============================================================================
// CPU ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// A line-by-line C++ restatement of JDSurfG's per-column surface-wave forward
// model.  Only tests/, __graft_entry__.smoke() and bench.py's cpu-baseline leg
// load this library, and only as the checker / timed CPU baseline; the GPU
// product path never calls it.
//
// Restated reference files (paths inside the JDSurfG project):
//   src/SWD/surfdisp96.f   : surfdisp96 (57-370), gtsolh (377-398), getsol
//                            (400-495), sphere (499-571), nevill (575-694),
//                            half (696-708), dltar/dltar1/dltar4 (712-898),
//                            var (901-1018), normc (1022-1047), dnka (1051-1095)
//   src/SWD/sregn96.f90    : bldsph (130-184), svfunc (193-399), up (401-489),
//                            dnka (491-647), evalg (649-825), varsv (827-911),
//                            hska (913-987), down (989-1059), energy
//                            (1061-1196), intijr (1198-1317), ffunc..h2func
//                            (1319-1397), normc (1399-1428), getdcdh
//                            (1430-1529), getmat (1531-1583), sprayl
//                            (1585-1629), sregn96 (1631-1735), sregnpu
//                            (1737-1878)
//   src/SWD/slegn96.f90    : bldsph (107-167), shfunc (179-246), varl
//                            (248-328), hskl (330-351), emat (353-370), up
//                            (372-445), energy (447-629), splove (631-670),
//                            slegn96 (672-783), slegnpu (785-918)
//   src/SWD/surfdisp.cpp   : _flat2sphere (17-51), surfdisp (64-116),
//                            groupvel_l (126-148), groupvel_r (158-174)
//   src/SWD/empirical.cpp  : empirical_relation / empirical_deriv (9-34)
//   src/SWD/SurfaceWave.cpp: get_period_index (14-48), _ParamConvert (59-101),
//                            grid2LayerModel (113-155), get_nt_row (157-167),
//                            disp1D (177-255), kernel1D (266-412), get_2d_map
//                            (420-450), get_1d_kernel (458-502), Frechet row
//                            assembly in frechet_matrix (590-676)
//
// Precision quirks of the Fortran are kept: REAL*4 model/flattened arrays,
// implicitly REAL*4 temporaries in surfdisp96/getsol/gtsolh, sngl() output of
// the root, single-precision constants (0.01 in nevill, 1.0e-5 in varsv,
// -2.275 in bldsph), single-precision pi in sregn96/sregnpu/slegn96/slegnpu,
// Earth radius 6370 in surfdisp96 vs 6371 elsewhere, the T2-valued module
// kernels in the *pu group-kernel formula and the 4.875x half-space weight of
// _ParamConvert.  Complex division follows Fortran's Smith rule.  Build with
// -ffp-contract=off so the arithmetic order is the source order.
//
// Deviations (documented, all on inputs where the reference reads undefined
// memory or exits):
//   * slegn96/slegnpu with a top fluid layer: the reference reads the never
//     written uu(1)/exl(1) of the fluid layer (slegn96.f90:213-231); here they
//     are 0, which leaves every kernel and U unchanged (they are invariant to
//     the eigenfunction scale) whenever the reference's garbage is finite.
//   * get_1d_kernel leaves the water node of the kernel uninitialised
//     (SurfaceWave.cpp:495); here it is 0.
//   * surfdisp() calls exit(1) when a period has no root after the retry
//     (surfdisp.cpp:100-108); here the period gets c=0 and status NO_ROOT.
//   * Columns with nw>=2 leading fluid nodes (vs==0) are merged into one
//     homogeneous fluid layer (surfdisp96 supports exactly one, llw=2); the
//     reference's grid2LayerModel handles only nw<=1 and the two agree there.
//   * groupvel_l sets vp = 1.732*vs (surfdisp.cpp:139), which for a fluid top
//     layer makes surfdisp96 start its scan at c = 0 (undefined); the layer's
//     own vp is used instead.  For solid columns Love roots do not depend on
//     vp, so the results are identical there.
// ============================================================================
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <vector>
#include <string>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ----------------------------------------------------------------------------
// Fortran-style double complex with Smith division (gfortran -fcx-fortran-rules)
// ----------------------------------------------------------------------------
struct cx { double re, im; };
inline cx C(double r, double i = 0.0) { return cx{r, i}; }
inline cx operator+(cx a, cx b) { return cx{a.re + b.re, a.im + b.im}; }
inline cx operator-(cx a, cx b) { return cx{a.re - b.re, a.im - b.im}; }
inline cx operator-(cx a) { return cx{-a.re, -a.im}; }
inline cx operator*(cx a, cx b) { return cx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline cx operator*(double s, cx a) { return cx{s * a.re, s * a.im}; }
inline cx operator*(cx a, double s) { return cx{a.re * s, a.im * s}; }
inline cx operator/(cx a, double s) { return cx{a.re / s, a.im / s}; }
inline cx operator+(cx a, double s) { return cx{a.re + s, a.im}; }
inline cx operator+(double s, cx a) { return cx{s + a.re, a.im}; }
inline cx operator-(double s, cx a) { return cx{s - a.re, -a.im}; }
inline cx operator-(cx a, double s) { return cx{a.re - s, a.im}; }
inline cx operator/(cx a, cx b) {
  if (std::fabs(b.re) >= std::fabs(b.im)) {
    double r = b.im / b.re, den = b.re + b.im * r;
    return cx{(a.re + a.im * r) / den, (a.im - a.re * r) / den};
  } else {
    double r = b.re / b.im, den = b.im + b.re * r;
    return cx{(a.re * r + a.im) / den, (a.im * r - a.re) / den};
  }
}
inline cx operator/(double s, cx b) { return C(s) / b; }
// cdsqrt(dcmplx(x,0)) : principal root, +i for negative x
inline cx csqrt_real(double x) { return x >= 0.0 ? C(std::sqrt(x), 0.0) : C(0.0, std::sqrt(-x)); }
inline cx cexp_(cx z) {
  double e = std::exp(z.re);
  if (z.im == 0.0) return C(e, 0.0);
  return C(e * std::cos(z.im), e * std::sin(z.im));
}
inline double cabs_(cx z) { return std::hypot(z.re, z.im); }
inline cx conj_(cx z) { return cx{z.re, -z.im}; }
inline double dsign1(double x) { return std::copysign(1.0, x); }

// float integer power as gfortran expands x**(-5): 1/((x*x)*(x*x)*x)
inline float powm5f(float x) { float x2 = x * x; float x4 = x2 * x2; float x5 = x4 * x; return 1.0f / x5; }
inline double powm5d(double x) { double x2 = x * x; double x4 = x2 * x2; double x5 = x4 * x; return 1.0 / x5; }

// single-precision pi of sregn96/sregnpu/slegn96/slegnpu
const double PI_F = (double)3.1415926535898f;

// ============================================================================
// surfdisp96.f
// ============================================================================
struct RootOpts {
  int refine;     // 0 = reference nevill (|c1-c2|<=1e-6 c1); 1 = tight Brent
  double rtol;    // relative bracket width for refine==1
  int sngl;       // 1 = round roots to REAL*4 like the reference (cg(k)=sngl(c))
};

struct Sd96 {
  int mmax, llw;
  std::vector<float> d, a, b, rho, rtp, dtp, btp;
  float dhalf = 0.f;
  double del1st = 0.0;  // getsol_module threadprivate state
  long nevals = 0;
  int iterlimit = 0;
};

// sphere (surfdisp96.f:499-571), ar = 6370
void sphere(Sd96& M, int ifunc, int iflag) {
  const int mmax = M.mmax;
  float *d = M.d.data(), *a = M.a.data(), *b = M.b.data(), *rho = M.rho.data();
  float *rtp = M.rtp.data(), *dtp = M.dtp.data(), *btp = M.btp.data();
  const double ar = 6370.0;
  double dr = 0.0, r0 = ar, r1, z0, z1, tmp;
  d[mmax - 1] = 1.0f;
  if (iflag == 0) {
    for (int i = 0; i < mmax; ++i) { dtp[i] = d[i]; rtp[i] = rho[i]; }
    for (int i = 0; i < mmax; ++i) {
      dr = dr + (double)d[i];
      r1 = ar - dr;
      z0 = ar * std::log(ar / r0);
      z1 = ar * std::log(ar / r1);
      d[i] = (float)(z1 - z0);
      tmp = (ar + ar) / (r0 + r1);
      a[i] = (float)((double)a[i] * tmp);
      b[i] = (float)((double)b[i] * tmp);
      btp[i] = (float)tmp;
      r0 = r1;
    }
    M.dhalf = d[mmax - 1];
  } else {
    d[mmax - 1] = M.dhalf;
    for (int i = 0; i < mmax; ++i) {
      if (ifunc == 1) rho[i] = rtp[i] * powm5f(btp[i]);
      else if (ifunc == 2) rho[i] = rtp[i] * std::pow(btp[i], -2.275f);
    }
  }
  d[mmax - 1] = 0.0f;
}

// gtsolh (surfdisp96.f:377-398), all REAL*4
void gtsolh(float a, float b, float& c) {
  c = 0.95f * b;
  for (int i = 0; i < 5; ++i) {
    float gamma = b / a;
    float kappa = c / b;
    float k2 = kappa * kappa;
    float gk = gamma * kappa;
    float gk2 = gk * gk;
    float fac1 = std::sqrt(1.0f - gk2);
    float fac2 = std::sqrt(1.0f - k2);
    float tk = 2.0f - k2;
    float fr = tk * tk - 4.0f * fac1 * fac2;
    float frp = -(4.0f * (2.0f - k2) * kappa) + 4.0f * fac2 * gamma * gamma * kappa / fac1 +
                4.0f * fac1 * kappa / fac2;
    frp = frp / b;
    c = c - fr / frp;
  }
}

// var (surfdisp96.f:901-1018); the dead tail (cosq/y/z rescale) is omitted
struct VarOut { double w, cosp, exa, a0, cpcq, cpy, cpz, cqw, cqx, xy, xz, wy, wz; };
inline VarOut var_(double p, double q, double ra, double rb, double wvno, double xka, double xkb, double dpth) {
  VarOut o;
  double exa = 0.0, a0 = 1.0, pex = 0.0, sex = 0.0;
  double sinp, w = 0, x = 0, cosp = 0, sinq, y = 0, z = 0, cosq = 0, fac;
  if (wvno < xka) {
    sinp = std::sin(p); w = sinp / ra; x = -ra * sinp; cosp = std::cos(p);
  } else if (wvno == xka) {
    cosp = 1.0; w = dpth; x = 0.0;
  } else if (wvno > xka) {
    pex = p; fac = 0.0;
    if (p < 16) fac = std::exp(-2.0 * p);
    cosp = (1.0 + fac) * 0.5; sinp = (1.0 - fac) * 0.5;
    w = sinp / ra; x = ra * sinp;
  }
  if (wvno < xkb) {
    sinq = std::sin(q); y = sinq / rb; z = -rb * sinq; cosq = std::cos(q);
  } else if (wvno == xkb) {
    cosq = 1.0; y = dpth; z = 0.0;
  } else if (wvno > xkb) {
    sex = q; fac = 0.0;
    if (q < 16) fac = std::exp(-2.0 * q);
    cosq = (1.0 + fac) * 0.5; sinq = (1.0 - fac) * 0.5;
    y = sinq / rb; z = rb * sinq;
  }
  exa = pex + sex;
  a0 = 0.0;
  if (exa < 60.0) a0 = std::exp(-exa);
  o.w = w; o.cosp = cosp; o.exa = exa; o.a0 = a0;
  o.cpcq = cosp * cosq; o.cpy = cosp * y; o.cpz = cosp * z; o.cqw = cosq * w; o.cqx = cosq * x;
  o.xy = x * y; o.xz = x * z; o.wy = w * y; o.wz = w * z;
  return o;
}

// normc (surfdisp96.f:1022-1047); returns ex = log(t1)
inline double normc5(double* ee, int n) {
  double t1 = 0.0;
  for (int i = 0; i < n; ++i) if (std::fabs(ee[i]) > t1) t1 = std::fabs(ee[i]);
  if (t1 < 1.e-40) t1 = 1.0;
  for (int i = 0; i < n; ++i) { double t2 = ee[i]; t2 = t2 / t1; ee[i] = t2; }
  return std::log(t1);
}

// dnka (surfdisp96.f:1051-1095); ca[i][j] = ca(i+1,j+1)
inline void dnka_sd(double ca[5][5], double wvno2, double gam, double gammk, double rho, const VarOut& v) {
  const double one = 1.0, two = 2.0;
  double gamm1 = gam - one;
  double twgm1 = gam + gamm1;
  double gmgmk = gam * gammk;
  double gmgm1 = gam * gamm1;
  double gm1sq = gamm1 * gamm1;
  double rho2 = rho * rho;
  double a0pq = v.a0 - v.cpcq;
  ca[0][0] = v.cpcq - two * gmgm1 * a0pq - gmgmk * v.xz - wvno2 * gm1sq * v.wy;
  ca[0][1] = (wvno2 * v.cpy - v.cqx) / rho;
  ca[0][2] = -(twgm1 * a0pq + gammk * v.xz + wvno2 * gamm1 * v.wy) / rho;
  ca[0][3] = (v.cpz - wvno2 * v.cqw) / rho;
  ca[0][4] = -(two * wvno2 * a0pq + v.xz + wvno2 * wvno2 * v.wy) / rho2;
  ca[1][0] = (gmgmk * v.cpz - gm1sq * v.cqw) * rho;
  ca[1][1] = v.cpcq;
  ca[1][2] = gammk * v.cpz - gamm1 * v.cqw;
  ca[1][3] = -v.wz;
  ca[1][4] = ca[0][3];
  ca[3][0] = (gm1sq * v.cpy - gmgmk * v.cqx) * rho;
  ca[3][1] = -v.xy;
  ca[3][2] = gamm1 * v.cpy - gammk * v.cqx;
  ca[3][3] = ca[1][1];
  ca[3][4] = ca[0][1];
  ca[4][0] = -(two * gmgmk * gm1sq * a0pq + gmgmk * gmgmk * v.xz + gm1sq * gm1sq * v.wy) * rho2;
  ca[4][1] = ca[3][0];
  ca[4][2] = -(gammk * gamm1 * twgm1 * a0pq + gam * gammk * gammk * v.xz + gamm1 * gm1sq * v.wy) * rho;
  ca[4][3] = ca[1][0];
  ca[4][4] = ca[0][0];
  double t = -two * wvno2;
  ca[2][0] = t * ca[4][2];
  ca[2][1] = t * ca[3][2];
  ca[2][2] = v.a0 + two * (v.cpcq - ca[0][0]);
  ca[2][3] = t * ca[1][2];
  ca[2][4] = t * ca[0][2];
}

// dltar4 (surfdisp96.f:798-898)
double dltar4(Sd96& M, double wvno, double omga) {
  const int mmax = M.mmax, llw = M.llw;
  const float *d = M.d.data(), *a = M.a.data(), *b = M.b.data(), *rho = M.rho.data();
  double e[5], ee[5], ca[5][5];
  double omega = omga;
  if (omega < 1.0e-4) omega = 1.0e-4;
  double wvno2 = wvno * wvno;
  double xka = omega / (double)a[mmax - 1];
  double xkb = omega / (double)b[mmax - 1];
  double wvnop = wvno + xka, wvnom = std::fabs(wvno - xka);
  double ra = std::sqrt(wvnop * wvnom);
  wvnop = wvno + xkb; wvnom = std::fabs(wvno - xkb);
  double rb = std::sqrt(wvnop * wvnom);
  double t = (double)b[mmax - 1] / omega;
  double gammk = 2.0 * t * t;
  double gam = gammk * wvno2;
  double gamm1 = gam - 1.0;
  double rho1 = (double)rho[mmax - 1];
  e[0] = rho1 * rho1 * (gamm1 * gamm1 - gam * gammk * ra * rb);
  e[1] = -rho1 * ra;
  e[2] = rho1 * (gamm1 - gammk * ra * rb);
  e[3] = rho1 * rb;
  e[4] = wvno2 - ra * rb;
  for (int m = mmax - 2; m >= llw - 1; --m) {
    xka = omega / (double)a[m];
    xkb = omega / (double)b[m];
    t = (double)b[m] / omega;
    gammk = 2.0 * t * t;
    gam = gammk * wvno2;
    wvnop = wvno + xka; wvnom = std::fabs(wvno - xka);
    ra = std::sqrt(wvnop * wvnom);
    wvnop = wvno + xkb; wvnom = std::fabs(wvno - xkb);
    rb = std::sqrt(wvnop * wvnom);
    double dpth = (double)d[m];
    rho1 = (double)rho[m];
    double p = ra * dpth, q = rb * dpth;
    VarOut v = var_(p, q, ra, rb, wvno, xka, xkb, dpth);
    dnka_sd(ca, wvno2, gam, gammk, rho1, v);
    for (int i = 0; i < 5; ++i) {
      double cr = 0.0;
      for (int j = 0; j < 5; ++j) cr = cr + e[j] * ca[j][i];
      ee[i] = cr;
    }
    normc5(ee, 5);
    for (int i = 0; i < 5; ++i) e[i] = ee[i];
  }
  if (llw != 1) {
    xka = omega / (double)a[0];
    wvnop = wvno + xka; wvnom = std::fabs(wvno - xka);
    ra = std::sqrt(wvnop * wvnom);
    double dpth = (double)d[0];
    rho1 = (double)rho[0];
    double p = ra * dpth;
    double znul = 1.0e-05;
    VarOut v = var_(p, znul, ra, znul, wvno, xka, znul, dpth);
    double w0 = -rho1 * v.w;
    return v.cosp * e[0] + w0 * e[1];
  }
  return e[0];
}

// dltar1 (surfdisp96.f:734-794)
double dltar1(Sd96& M, double wvno, double omega) {
  const int mmax = M.mmax, llw = M.llw;
  const float *d = M.d.data(), *b = M.b.data(), *rho = M.rho.data();
  double beta1 = (double)b[mmax - 1];
  double rho1 = (double)rho[mmax - 1];
  double xkb = omega / beta1;
  double wvnop = wvno + xkb, wvnom = std::fabs(wvno - xkb);
  double rb = std::sqrt(wvnop * wvnom);
  double e1 = rho1 * rb;
  double e2 = 1.0 / (beta1 * beta1);
  for (int m = mmax - 2; m >= llw - 1; --m) {
    beta1 = (double)b[m];
    rho1 = (double)rho[m];
    double xmu = rho1 * beta1 * beta1;
    xkb = omega / beta1;
    wvnop = wvno + xkb; wvnom = std::fabs(wvno - xkb);
    rb = std::sqrt(wvnop * wvnom);
    double q = (double)d[m] * rb;
    double sinq, cosq = 0, y = 0, z = 0;
    if (wvno < xkb) {
      sinq = std::sin(q); y = sinq / rb; z = -rb * sinq; cosq = std::cos(q);
    } else if (wvno == xkb) {
      cosq = 1.0; y = (double)d[m]; z = 0.0;
    } else {
      double fac = 0.0;
      if (q < 16) fac = std::exp(-2.0 * q);
      cosq = (1.0 + fac) * 0.5; sinq = (1.0 - fac) * 0.5;
      y = sinq / rb; z = rb * sinq;
    }
    double e10 = e1 * cosq + e2 * xmu * z;
    double e20 = e1 * y / xmu + e2 * cosq;
    double xnor = std::fabs(e10), ynor = std::fabs(e20);
    if (ynor > xnor) xnor = ynor;
    if (xnor < 1.e-40) xnor = 1.0;
    e1 = e10 / xnor;
    e2 = e20 / xnor;
  }
  return e1;
}

inline double dltar(Sd96& M, double wvno, double omega, int kk) {
  M.nevals++;
  if (kk == 1) return dltar1(M, wvno, omega);
  return dltar4(M, wvno, omega);
}

const double TWOPI = 2.0 * 3.141592653589793;

// half (surfdisp96.f:696-708)
inline void half(Sd96& M, double c1, double c2, double& c3, double& del3, double omega, int ifunc) {
  c3 = 0.5 * (c1 + c2);
  double wvno = omega / c3;
  del3 = dltar(M, wvno, omega, ifunc);
}

// nevill (surfdisp96.f:575-694)
void nevill(Sd96& M, double t, double c1, double c2, double del1, double del2, int ifunc, double& cc) {
  double x[20], y[20];
  double omega = TWOPI / t;
  double c3, del3;
  half(M, c1, c2, c3, del3, omega, ifunc);
  int nev = 1, nctrl = 1, m = 1;
  for (;;) {
    nctrl = nctrl + 1;
    if (nctrl >= 100) { M.iterlimit++; break; }
    if (c3 < std::min(c1, c2) || c3 > std::max(c1, c2)) {
      nev = 0;
      half(M, c1, c2, c3, del3, omega, ifunc);
    }
    double s13 = del1 - del3;
    double s32 = del3 - del2;
    if (dsign1(del3) * dsign1(del1) < 0.0) { c2 = c3; del2 = del3; }
    else { c1 = c3; del1 = del3; }
    if (std::fabs(c1 - c2) <= 1.e-6 * c1) break;
    if (dsign1(s13) != dsign1(s32)) nev = 0;
    double ss1 = std::fabs(del1);
    double s1 = (double)0.01f * ss1;
    double ss2 = std::fabs(del2);
    double s2 = (double)0.01f * ss2;
    if (s1 > ss2 || s2 > ss1 || nev == 0) {
      half(M, c1, c2, c3, del3, omega, ifunc);
      nev = 1; m = 1;
    } else {
      if (nev == 2) { x[m] = c3; y[m] = del3; }
      else { x[0] = c1; y[0] = del1; x[1] = c2; y[1] = del2; m = 1; }
      bool bad = false;
      for (int kk = 1; kk <= m; ++kk) {
        int j = m - kk + 1;  // 1-based
        double denom = y[m] - y[j - 1];
        if (std::fabs(denom) < 1.0e-10 * std::fabs(y[m])) { bad = true; break; }
        x[j - 1] = (-y[j - 1] * x[j] + y[m] * x[j - 1]) / denom;
      }
      if (!bad) {
        c3 = x[0];
        double wvno = omega / c3;
        del3 = dltar(M, wvno, omega, ifunc);
        nev = 2;
        m = m + 1;
        if (m > 10) m = 10;
      } else {
        half(M, c1, c2, c3, del3, omega, ifunc);
        nev = 1; m = 1;
      }
    }
  }
  cc = c3;
}

// Tight refinement (not in the reference): Brent's zeroin on the same
// bracket, stopping when the sign-verified bracket is <= 2*(rtol/2)*c.
void brent(Sd96& M, double t, double c1, double c2, double del1, double del2, int ifunc, double rtol, double& cc) {
  double omega = TWOPI / t;
  double a = c1, fa = del1, b = c2, fb = del2, c = a, fc = fa, d = b - a, e = d;
  const double eps = 2.220446049250313e-16;
  for (int it = 0; it < 200; ++it) {
    if (std::signbit(fb) == std::signbit(fc)) { c = a; fc = fa; d = b - a; e = d; }
    if (std::fabs(fc) < std::fabs(fb)) { a = b; b = c; c = a; fa = fb; fb = fc; fc = fa; }
    double tol1 = 2.0 * eps * std::fabs(b) + 0.5 * rtol * std::fabs(b);
    double xm = 0.5 * (c - b);
    if (std::fabs(xm) <= tol1 || fb == 0.0) break;
    if (std::fabs(e) >= tol1 && std::fabs(fa) > std::fabs(fb)) {
      double s = fb / fa, p, q;
      if (a == c) { p = 2.0 * xm * s; q = 1.0 - s; }
      else {
        double qq = fa / fc, r = fb / fc;
        p = s * (2.0 * xm * qq * (qq - r) - (b - a) * (r - 1.0));
        q = (qq - 1.0) * (r - 1.0) * (s - 1.0);
      }
      if (p > 0.0) q = -q;
      p = std::fabs(p);
      if (2.0 * p < std::min(3.0 * xm * q - std::fabs(tol1 * q), std::fabs(e * q))) { e = d; d = p / q; }
      else { d = xm; e = d; }
    } else { d = xm; e = d; }
    a = b; fa = fb;
    if (std::fabs(d) > tol1) b = b + d;
    else b = b + std::copysign(tol1, xm);
    fb = dltar(M, omega / b, omega, ifunc);
  }
  cc = b;
}

// getsol (surfdisp96.f:400-495)
void getsol(Sd96& M, double t1, double& c1, double clow, double dc, double cm, float betmx, int& iret,
            int ifunc, int ifirst, const RootOpts& o) {
  double omega = TWOPI / t1;
  double wvno = omega / c1;
  double del1 = dltar(M, wvno, omega, ifunc);
  if (ifirst == 1) M.del1st = del1;
  double plmn = dsign1(M.del1st) * dsign1(del1);
  int idir = +1;
  if (ifirst == 1) idir = +1;
  else if (plmn >= 0.0) idir = +1;
  else idir = -1;
  double c2, del2;
  for (;;) {
    if (idir > 0) c2 = c1 + dc; else c2 = c1 - dc;
    if (c2 <= clow) { idir = +1; c1 = clow; continue; }
    omega = TWOPI / t1;
    wvno = omega / c2;
    del2 = dltar(M, wvno, omega, ifunc);
    if (dsign1(del1) != dsign1(del2)) break;
    c1 = c2;
    del1 = del2;
    if (c1 < cm) { iret = -1; return; }
    if (c1 >= ((double)betmx + dc)) { iret = -1; return; }
  }
  double cn;
  if (o.refine == 0) nevill(M, t1, c1, c2, del1, del2, ifunc, cn);
  else brent(M, t1, c1, c2, del1, del2, ifunc, o.rtol, cn);
  c1 = cn;
  if (c1 > (double)betmx) { iret = -1; return; }
  iret = 1;
}

// surfdisp96 (surfdisp96.f:57-370)
void surfdisp96_impl(const float* thkm, const float* vpm, const float* vsm, const float* rhom, int nlayer,
                     int iflsph, int iwave, int mode, int igr, int kmax, const double* t, double* cg, int* ierr,
                     const RootOpts& o, long* nevals, int* iterlim) {
  Sd96 M;
  M.mmax = nlayer;
  const int mmax = nlayer;
  M.d.assign(thkm, thkm + mmax); M.a.assign(vpm, vpm + mmax);
  M.b.assign(vsm, vsm + mmax); M.rho.assign(rhom, rhom + mmax);
  M.rtp.assign(mmax, 0.f); M.dtp.assign(mmax, 0.f); M.btp.assign(mmax, 0.f);
  int nsph = iflsph;
  *ierr = 0;
  int idispl = 0, idispr = 0;
  if (iwave == 1) { idispl = kmax; idispr = 0; }
  else if (iwave == 2) { idispl = 0; idispr = kmax; }
  int iverb[2] = {0, 0};
  const float sone0 = 1.500f, ddc0 = 0.005f, h0 = 0.005f;
  M.llw = 1;
  if (M.b[0] <= 0.0f) M.llw = 2;
  const double one = 1.0e-2;
  if (nsph == 1) sphere(M, 0, 0);
  int jmn = 0, jsol = 1;
  float betmx = -1.e20f, betmn = 1.e20f;
  for (int i = 0; i < mmax; ++i) {
    if (M.b[i] > 0.01f && M.b[i] < betmn) { betmn = M.b[i]; jmn = i; jsol = 1; }
    else if (M.b[i] <= 0.01f && M.a[i] < betmn) { betmn = M.a[i]; jmn = i; jsol = 0; }
    if (M.b[i] > betmx) betmx = M.b[i];
  }
  std::vector<double> c(kmax, 0.0), cb(kmax, 0.0);
  for (int ifunc = 1; ifunc <= 2; ++ifunc) {
    if (ifunc == 1 && idispl <= 0) continue;
    if (ifunc == 2 && idispr <= 0) continue;
    if (nsph == 1) sphere(M, ifunc, 1);
    float ddc = ddc0, sone = sone0, h = h0;
    if (sone < 0.01f) sone = 2.0f;
    double onea = (double)sone;
    float cc1;
    if (jsol == 0) cc1 = betmn;
    else gtsolh(M.a[jmn], M.b[jmn], cc1);
    cc1 = 0.95f * cc1;
    cc1 = 0.90f * cc1;
    double cc = (double)cc1;
    double dc = (double)ddc;
    dc = std::fabs(dc);
    double c1 = cc, cm = cc, clow = cc;
    for (int i = 0; i < kmax; ++i) { cb[i] = 0.0; c[i] = 0.0; }
    int ift = 999;
    for (int iq = 1; iq <= mode; ++iq) {
      int is = 1, ie = kmax;
      int k;
      bool failed = false;
      for (k = is; k <= ie; ++k) {
        if (k >= ift) { failed = true; break; }
        double t1 = t[k - 1];
        float t1a, t1b = 0.f;
        if (igr > 0) {
          t1a = (float)(t1 / (double)(1.0f + h));
          t1b = (float)(t1 / (double)(1.0f - h));
          t1 = (double)t1a;
        } else {
          t1a = (float)t1;
        }
        int ifirst = 0;
        if (k == is && iq == 1) { c1 = cc; clow = cc; ifirst = 1; }
        else if (k == is && iq > 1) { c1 = c[is - 1] + one * dc; clow = c1; ifirst = 1; }
        else if (k > is && iq > 1) {
          ifirst = 0;
          clow = c[k - 1] + one * dc;
          c1 = c[k - 2];
          if (c1 < clow) c1 = clow;
        } else if (k > is && iq == 1) {
          ifirst = 0;
          c1 = c[k - 2] - onea * dc;
          clow = cm;
        }
        int iret;
        getsol(M, t1, c1, clow, dc, cm, betmx, iret, ifunc, ifirst, o);
        if (iret == -1) { failed = true; break; }
        c[k - 1] = c1;
        if (igr > 0) {
          t1 = (double)t1b;
          ifirst = 0;
          clow = cb[k - 1] + one * dc;
          c1 = c1 - onea * dc;
          getsol(M, t1, c1, clow, dc, cm, betmx, iret, ifunc, ifirst, o);
          if (iret == -1) c1 = c[k - 1];
          cb[k - 1] = c1;
        } else {
          c1 = 0.0;
        }
        if (o.sngl) {
          float cc0 = (float)c[k - 1];
          float ccc1 = (float)c1;
          if (igr == 0) cg[k - 1] = (double)cc0;
          else {
            float gvel = (1.0f / t1a - 1.0f / t1b) / (1.0f / (t1a * cc0) - 1.0f / (t1b * ccc1));
            cg[k - 1] = (double)gvel;
          }
        } else {
          if (igr == 0) cg[k - 1] = c[k - 1];
          else {
            double ta = (double)t1a, tb = (double)t1b;
            cg[k - 1] = (1.0 / ta - 1.0 / tb) / (1.0 / (ta * c[k - 1]) - 1.0 / (tb * c1));
          }
        }
      }
      if (failed) {
        if (iq <= 1) {
          if (iverb[ifunc - 1] == 0) { iverb[ifunc - 1] = 1; *ierr = 1; }
        }
        ift = k;
        for (int i = k; i <= ie; ++i) cg[i - 1] = 0.0;
      }
    }
  }
  if (nevals) *nevals += M.nevals;
  if (iterlim) *iterlim += M.iterlimit;
}

const RootOpts REF_OPTS = {0, 1e-6, 1};

// ============================================================================
// sregn96.f90
// ============================================================================
struct Ray {
  int mmax;
  std::vector<double> zd, zrho, za, zb, xmu, xlam;
  std::vector<double> ur, uz, tz, tr, dcda, dcdb, dcdr, dcdh;
  std::vector<int> iwat;
  double sumi0, sumi1, sumi2, sumi3, flagr, are, ugr;
  std::vector<double> vtp, dtp, rtp;
  std::vector<double> exe, exa, cd, vv;  // cd(mmax,5), vv(mmax,4) stored [m*5+j]
  bool allfluid;
  cx ra, rb, e[4][4], einv[4][4];
  double uu0[4];
  void alloc(int n) {
    mmax = n;
    zd.assign(n, 0); zrho.assign(n, 0); za.assign(n, 0); zb.assign(n, 0); xmu.assign(n, 0); xlam.assign(n, 0);
    ur.assign(n, 0); uz.assign(n, 0); tz.assign(n, 0); tr.assign(n, 0);
    dcda.assign(n, 0); dcdb.assign(n, 0); dcdr.assign(n, 0); dcdh.assign(n, 0);
    iwat.assign(n, 0); exe.assign(n, 0); exa.assign(n, 0); cd.assign(n * 5, 0); vv.assign(n * 4, 0);
  }
  double& CD(int m, int j) { return cd[m * 5 + j]; }
  double& VV(int m, int j) { return vv[m * 4 + j]; }
};

// bldsph (sregn96.f90:130-184), ar = 6371
void ray_bldsph(Ray& S) {
  const double ar = 6371.0;
  double dr = 0.0, r0 = ar;
  const double expo = (double)(-2.275f);
  for (int i = 0; i < S.mmax; ++i) S.dtp[i] = 0.0;
  for (int i = 0; i < S.mmax; ++i) {
    if (i == S.mmax - 1) dr = dr + 1.0;
    else dr = dr + S.zd[i];
    double r1 = ar - dr;
    double z0 = ar * std::log(ar / r0);
    double z1 = ar * std::log(ar / r1);
    double tmp = (2.0 * ar) / (r0 + r1);
    S.vtp[i] = tmp;
    S.rtp[i] = std::pow(tmp, expo);
    S.dtp[i] = ar / r0;
    S.za[i] = S.za[i] * tmp;
    S.zb[i] = S.zb[i] * tmp;
    S.zrho[i] = S.zrho[i] * S.rtp[i];
    S.zd[i] = z1 - z0;
    r0 = r1;
  }
  S.zd[S.mmax - 1] = 0.0;
}

// evalg with jbdry = 0 (sregn96.f90:649-825); gbr is row inp of gbr(2,5)
void ray_evalg0(Ray& S, int m, cx gbr[5], double wvno, double om, double om2, double wvno2) {
  double xka = om / S.za[m];
  double xkb = (S.zb[m] > 0.0) ? om / S.zb[m] : 0.0;
  S.ra = csqrt_real(wvno2 - xka * xka);
  S.rb = csqrt_real(wvno2 - xkb * xkb);
  double gam = S.zb[m] * wvno / om;
  gam = 2.0 * (gam * gam);
  double gamm1 = gam - 1.0;
  cx ra = S.ra, rb = S.rb;
  double zr = S.zrho[m];
  cx (&E)[4][4] = S.e;
  cx (&EI)[4][4] = S.einv;
  if (S.iwat[m] == 0) {
    E[0][0] = C(wvno); E[0][1] = rb; E[0][2] = C(wvno); E[0][3] = -rb;
    E[1][0] = ra; E[1][1] = C(wvno); E[1][2] = -ra; E[1][3] = C(wvno);
    E[2][0] = C(zr * om2 * gamm1);
    E[2][1] = (zr * om2 * gam) * rb / wvno;
    E[2][2] = C(zr * om2 * gamm1);
    E[2][3] = -((zr * om2 * gam) * rb / wvno);
    E[3][0] = (zr * om2 * gam) * ra / wvno;
    E[3][1] = C(zr * om2 * gamm1);
    E[3][2] = -((zr * om2 * gam) * ra / wvno);
    E[3][3] = C(zr * om2 * gamm1);
    EI[0][0] = C(0.5 * gam / wvno);
    EI[0][1] = -((0.5 * gamm1) / ra);
    EI[0][2] = C(-(0.5 / (zr * om2)));
    EI[0][3] = (0.5 * wvno) / ((zr * om2) * ra);
    EI[1][0] = -((0.5 * gamm1) / rb);
    EI[1][1] = C(0.5 * gam / wvno);
    EI[1][2] = (0.5 * wvno) / ((zr * om2) * rb);
    EI[1][3] = C(-(0.5 / (zr * om2)));
    EI[2][0] = C(0.5 * gam / wvno);
    EI[2][1] = (0.5 * gamm1) / ra;
    EI[2][2] = C(-(0.5 / (zr * om2)));
    EI[2][3] = -((0.5 * wvno) / ((zr * om2) * ra));
    EI[3][0] = (0.5 * gamm1) / rb;
    EI[3][1] = C(0.5 * gam / wvno);
    EI[3][2] = -((0.5 * wvno) / ((zr * om2) * rb));
    EI[3][3] = C(-(0.5 / (zr * om2)));
    if (gbr) {
      gbr[0] = (zr * zr * om2 * om2) * (-((gam * gam) * ra * rb) + wvno2 * gamm1 * gamm1);
      gbr[1] = -((zr * (wvno2 * ra)) * om2);
      gbr[2] = -(((zr * (-((gam * ra) * rb) + wvno2 * gamm1)) * om2) * wvno);
      gbr[3] = (zr * (wvno2 * rb)) * om2;
      gbr[4] = wvno2 * (wvno2 - ra * rb);
      cx den = -((zr * zr * om2 * om2 * wvno2) * ra * rb);
      for (int i = 0; i < 5; ++i) gbr[i] = (0.25 * gbr[i]) / den;
    }
  } else {
    if (gbr) {
      if (S.allfluid) {
        gbr[0] = 0.5 / ra;
        gbr[1] = C(0.5) / C(-(zr * om2));
        gbr[2] = C(0); gbr[3] = C(0); gbr[4] = C(0);
      } else {
        gbr[0] = C(0); gbr[1] = C(0); gbr[2] = C(0);
        gbr[3] = (0.5 * zr * om2) / ra;
        gbr[4] = C(-0.5);
      }
    }
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) { E[i][j] = C(0); EI[i][j] = C(0); }
    E[0][0] = ra; E[0][1] = -ra;
    E[1][0] = C(-(zr * om2)); E[1][1] = C(-(zr * om2));
    EI[0][0] = 0.5 / ra;
    EI[0][1] = C(-(0.5 / (zr * om2)));
    EI[1][0] = -(0.5 / ra);
    EI[1][1] = C(-(0.5 / (zr * om2)));
  }
}

// varsv (sregn96.f90:827-911)
void ray_varsv(cx p, cx q, cx rp, cx rsv, double& cosp, double& cosq, double& rsinp, double& rsinq,
               double& sinpr, double& sinqr, double& pex, double& svex, int iwat, double zd) {
  pex = 0.0; svex = 0.0;
  double pr = p.re, pi = p.im, qr = q.re, qi = q.im;
  pex = pr;
  const double tiny = (double)1.0e-5f;
  cx epp = C(std::cos(pi), std::sin(pi)) / 2.0;
  cx epm = conj_(epp);
  double pfac = (pr < 30.) ? std::exp(-2. * pr) : 0.0;
  cosp = (epp + pfac * epm).re;
  cx sinp = epp - pfac * epm;
  rsinp = (rp * sinp).re;
  if (std::fabs(pr) < tiny && cabs_(rp) < tiny) sinpr = zd;
  else sinpr = (sinp / rp).re;
  if (iwat == 1) {
    cosq = 1.0; rsinq = 0.0; sinqr = 0.0;
  } else {
    svex = qr;
    cx eqp = C(std::cos(qi), std::sin(qi)) / 2.0;
    cx eqm = conj_(eqp);
    double svfac = (qr < 30.) ? std::exp(-2. * qr) : 0.0;
    cosq = (eqp + svfac * eqm).re;
    cx sinq = eqp - svfac * eqm;
    rsinq = (rsv * sinq).re;
    if (std::fabs(qr) < tiny && cabs_(rsv) < tiny) sinqr = zd;
    else sinqr = (sinq / rsv).re;
  }
}

// dnka (sregn96.f90:491-647); rho and b arrive as REAL*4
void ray_dnka(double ca[5][5], double cosp, double rsinp, double sinpr, double cossv, double rsinsv, double sinsvr,
              float rho, float b, int iwat, double ex, double exa, double wvno, double wvno2, double om2) {
  if (iwat == 1) {
    for (int i = 0; i < 5; ++i) for (int j = 0; j < 5; ++j) ca[i][j] = 0.0;
    double dfac = (ex > 35.0) ? 0.0 : std::exp(-ex);
    ca[2][2] = dfac;
    ca[0][0] = cosp;
    ca[4][4] = cosp;
    ca[0][1] = -rsinp / ((double)rho * om2);
    ca[1][0] = -((double)rho * sinpr * om2);
    ca[1][1] = cosp;
    ca[3][3] = cosp;
    ca[3][4] = ca[0][1];
    ca[4][3] = ca[1][0];
    return;
  }
  double a0 = (exa < 60.0) ? std::exp(-exa) : 0.0;
  double cpcq = cosp * cossv, cpy = cosp * sinsvr, cpz = cosp * rsinsv, cqw = cossv * sinpr, cqx = cossv * rsinp;
  double xy = rsinp * sinsvr, xz = rsinp * rsinsv, wy = sinpr * sinsvr, wz = sinpr * rsinsv;
  float rho2 = rho * rho;
  double gam = (double)(2.0f * b * b) * wvno2 / om2;
  double gam2 = gam * gam;
  double gamm1 = gam - 1.;
  double gamm2 = gamm1 * gamm1;
  double cqww2 = cqw * wvno2;
  double cqxw2 = cqx / wvno2;
  double gg1 = gam * gamm1;
  double a0c = 2.0 * (a0 - cpcq);
  double xz2 = xz / wvno2;
  double gxz2 = gam * xz2;
  double g2xz2 = gam2 * xz2;
  double a0cgg1 = a0c * (gam + gamm1);
  double wy2 = wy * wvno2;
  double g2wy2 = gamm2 * wy2;
  double g1wy2 = gamm1 * wy2;
  double rhod = (double)rho, rho2d = (double)rho2;
  double temp = a0c * gg1 + g2xz2 + g2wy2;
  ca[2][2] = a0 + temp + temp;
  ca[0][0] = cpcq - temp;
  ca[0][1] = (-cqx + wvno2 * cpy) / (rhod * om2);
  temp = 0.5 * a0cgg1 + gxz2 + g1wy2;
  ca[0][2] = wvno * temp / (rhod * om2);
  ca[0][3] = (-cqww2 + cpz) / (rhod * om2);
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
void ray_hska(double AA[4][4], double cosp, double rsinp, double sinpr, double tcossv, double trsinsv,
              double tsinsvr, float rho, float b, int iwat, double pex, double svex, double wvno, double wvno2,
              double om2) {
  double rhod = (double)rho;
  if (iwat == 1) {
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) AA[i][j] = 0.0;
    double dfac = (pex > 35.0) ? 0.0 : std::exp(-pex);
    AA[0][0] = dfac;
    AA[3][3] = dfac;
    AA[1][1] = cosp;
    AA[2][2] = cosp;
    AA[1][2] = -rsinp / (rhod * om2);
    AA[2][1] = -(rhod * om2 * sinpr);
    return;
  }
  double dfac = ((pex - svex) > 70.0) ? 0.0 : std::exp(svex - pex);
  double cossv = dfac * tcossv, rsinsv = dfac * trsinsv, sinsvr = dfac * tsinsvr;
  double gam = (double)(2.0f * b * b) * wvno2 / om2;
  double gamm1 = gam - 1.0;
  AA[0][0] = cossv + gam * (cosp - cossv);
  AA[0][1] = -wvno * gamm1 * sinpr + gam * rsinsv / wvno;
  AA[0][2] = -(wvno * (cosp - cossv) / (rhod * om2));
  AA[0][3] = (wvno2 * sinpr - rsinsv) / (rhod * om2);
  AA[1][0] = gam * rsinp / wvno - wvno * gamm1 * sinsvr;
  AA[1][1] = cosp - gam * (cosp - cossv);
  AA[1][2] = (-rsinp + wvno2 * sinsvr) / (rhod * om2);
  AA[1][3] = -AA[0][2];
  AA[2][0] = rhod * om2 * gam * gamm1 * (cosp - cossv) / wvno;
  AA[2][1] = rhod * om2 * (-gamm1 * gamm1 * sinpr + gam * gam * rsinsv / wvno2);
  AA[2][2] = AA[1][1];
  AA[2][3] = -AA[0][1];
  AA[3][0] = rhod * om2 * (gam * gam * rsinp / wvno2 - gamm1 * gamm1 * sinsvr);
  AA[3][1] = -AA[2][0];
  AA[3][2] = -AA[1][0];
  AA[3][3] = AA[0][0];
}

// up (sregn96.f90:401-489)
void ray_up(Ray& S, double omega, double wvno, double& fr) {
  const int mmax = S.mmax;
  double wvno2 = wvno * wvno, om2 = omega * omega;
  cx gbr[5];
  ray_evalg0(S, mmax - 1, gbr, wvno, omega, om2, wvno2);
  for (int j = 0; j < 5; ++j) S.CD(mmax - 1, j) = gbr[j].re;
  S.exe[mmax - 1] = 0.0;
  double exsum = 0.0;
  double ca[5][5], ee[5];
  for (int m = mmax - 2; m >= 0; --m) {
    double xka = omega / S.za[m];
    double xkb = (S.zb[m] > 0.0) ? omega / S.zb[m] : 0.0;
    cx rp = csqrt_real(wvno2 - xka * xka);
    cx rsv = csqrt_real(wvno2 - xkb * xkb);
    cx p = rp * S.zd[m], q = rsv * S.zd[m];
    double cosp, cossv, rsinp, rsinsv, sinpr, sinsvr, pex, svex;
    ray_varsv(p, q, rp, rsv, cosp, cossv, rsinp, rsinsv, sinpr, sinsvr, pex, svex, S.iwat[m], S.zd[m]);
    ray_dnka(ca, cosp, rsinp, sinpr, cossv, rsinsv, sinsvr, (float)S.zrho[m], (float)S.zb[m], S.iwat[m], pex,
             pex + svex, wvno, wvno2, om2);
    for (int i = 0; i < 5; ++i) {
      double cr = 0.0;
      for (int j = 0; j < 5; ++j) cr = cr + S.CD(m + 1, j) * ca[j][i];
      ee[i] = cr;
    }
    double exn = normc5(ee, 5);
    exsum = exsum + pex + svex + exn;
    S.exe[m] = exsum;
    for (int i = 0; i < 5; ++i) S.CD(m, i) = ee[i];
  }
  fr = S.CD(0, 0);
}

// down (sregn96.f90:989-1059)
void ray_down(Ray& S, double omega, double wvno) {
  const int mmax = S.mmax;
  double om2 = omega * omega, wvno2 = wvno * wvno;
  for (int i = 0; i < 4; ++i) S.VV(0, i) = (i == 0) ? 1.0 : 0.0;
  S.exa[0] = 0.0;
  double exsum = 0.0, AA[4][4], aa0[4];
  for (int m = 0; m < mmax - 1; ++m) {
    double xka = omega / S.za[m];
    double xkb = (S.zb[m] > 0.0) ? omega / S.zb[m] : 0.0;
    cx rp = csqrt_real(wvno2 - xka * xka);
    cx rsv = csqrt_real(wvno2 - xkb * xkb);
    cx p = rp * S.zd[m], q = rsv * S.zd[m];
    double cosp, cossv, rsinp, rsinsv, sinpr, sinsvr, pex, svex;
    ray_varsv(p, q, rp, rsv, cosp, cossv, rsinp, rsinsv, sinpr, sinsvr, pex, svex, S.iwat[m], S.zd[m]);
    ray_hska(AA, cosp, rsinp, sinpr, cossv, rsinsv, sinsvr, (float)S.zrho[m], (float)S.zb[m], S.iwat[m], pex, svex,
             wvno, wvno2, om2);
    for (int i = 0; i < 4; ++i) {
      double cc = 0.0;
      for (int j = 0; j < 4; ++j) cc = cc + AA[i][j] * S.VV(m, j);
      aa0[i] = cc;
    }
    double ex2 = normc5(aa0, 4);
    exsum = exsum + pex + ex2;
    S.exa[m + 1] = exsum;
    for (int i = 0; i < 4; ++i) S.VV(m + 1, i) = aa0[i];
  }
}

// svfunc (sregn96.f90:193-399)
void ray_svfunc(Ray& S, double omega, double wvno) {
  double fr;
  ray_up(S, omega, wvno, fr);
  ray_down(S, omega, wvno);
  const int mmax = S.mmax;
  double f1213 = -S.CD(0, 1);
  S.ur[0] = S.CD(0, 2) / S.CD(0, 1);
  S.uz[0] = 1.0; S.tz[0] = 0.0; S.tr[0] = 0.0;
  S.uu0[0] = S.ur[0]; S.uu0[1] = 1.0; S.uu0[2] = fr; S.uu0[3] = fr;
  for (int i = 1; i < mmax; ++i) {
    double cd1 = S.CD(i, 0), cd2 = S.CD(i, 1), cd3 = S.CD(i, 2), cd4 = -S.CD(i, 2), cd5 = S.CD(i, 3), cd6 = S.CD(i, 4);
    double tz1 = -S.VV(i, 3), tz2 = -S.VV(i, 2), tz3 = S.VV(i, 1), tz4 = S.VV(i, 0);
    double uu1 = tz2 * cd6 - tz3 * cd5 + tz4 * cd4;
    double uu2 = -tz1 * cd6 + tz3 * cd3 - tz4 * cd2;
    double uu3 = tz1 * cd5 - tz2 * cd3 + tz4 * cd1;
    double uu4 = -tz1 * cd4 + tz2 * cd2 - tz3 * cd1;
    double ext = S.exa[i] + S.exe[i] - S.exe[0];
    if (ext > -80.0 && ext < 80.0) {
      double fact = std::exp(ext);
      S.ur[i] = uu1 * fact / f1213;
      S.uz[i] = uu2 * fact / f1213;
      S.tz[i] = uu3 * fact / f1213;
      S.tr[i] = uu4 * fact / f1213;
    } else {
      S.ur[i] = 0.0; S.uz[i] = 0.0; S.tz[i] = 0.0; S.tr[i] = 0.0;
    }
  }
  if (!S.allfluid) {
    int jwat = 0;
    for (int i = 0; i < mmax; ++i) { if (S.iwat[i] > 0) jwat = i + 1; else break; }
    for (int i = 0; i < jwat; ++i) { S.ur[i] = 0.0; S.tr[i] = 0.0; }
  }
}

// ffunc .. h2func (sregn96.f90:1319-1397)
cx ffunc(cx nub, double dm) {
  if (cabs_(nub) < 1.0e-08) return C(dm);
  cx argcd = nub * dm;
  cx exqq = (argcd.re < 40.0) ? cexp_(-2.0 * argcd) : C(0.0);
  return (1.0 - exqq) / (2.0 * nub);
}
cx gfunc(cx nub, double dm) {
  cx argcd = nub * dm;
  if (argcd.re < 75) return cexp_(-argcd) * dm;
  return C(0.0);
}
cx h1func(cx nua, cx nub, double dm) {
  if (cabs_(nub + nua) < 1.0e-08) return C(dm);
  cx argcd = (nua + nub) * dm;
  cx exqq = (argcd.re < 40.0) ? cexp_(-argcd) : C(0.0);
  return (1.0 - exqq) / (nub + nua);
}
cx h2func(cx nua, cx nub, double dm) {
  if (cabs_(nub - nua) < 1.0e-08) return C(dm);
  cx argcd = nua * dm;
  cx exqp = (argcd.re < 40.0) ? cexp_(-argcd) : C(0.0);
  argcd = nub * dm;
  cx exqq = (argcd.re < 40.0) ? cexp_(-argcd) : C(0.0);
  return (exqq - exqp) / (nua - nub);
}

// intijr (sregn96.f90:1198-1317); i,j are 1-based like the Fortran
double ray_intijr(Ray& S, int i, int j, int m, int typelyr, double om, double om2, double wvno, double wvno2) {
  ray_evalg0(S, m, nullptr, wvno, om, om2, wvno2);
  cx (&e)[4][4] = S.e;
  cx (&ei)[4][4] = S.einv;
  cx ra = S.ra, rb = S.rb;
  --i; --j;
  cx cint;
  if (S.iwat[m] == 1) {
    if (typelyr < 0) {
      cx kmpu = ei[0][0] * S.uz[m + 1] + ei[0][1] * S.tz[m + 1];
      cint = e[i][0] * e[j][0] * kmpu * kmpu / (2.0 * ra);
    } else if (typelyr == 0) {
      cx km1pd = ei[1][0] * S.uz[m] + ei[1][1] * S.tz[m];
      cx kmpu = ei[0][0] * S.uz[m + 1] + ei[0][1] * S.tz[m + 1];
      cx FA = ffunc(ra, S.zd[m]);
      cx GA = gfunc(ra, S.zd[m]);
      cint = e[i][0] * e[j][0] * kmpu * kmpu * FA + (e[i][0] * e[j][1] + e[i][1] * e[j][0]) * kmpu * km1pd * GA +
             e[i][1] * e[j][1] * km1pd * km1pd * FA;
    } else {
      cx km1pd = ei[1][0] * S.uz[m] + ei[1][1] * S.tz[m];
      cint = e[i][1] * e[j][1] * km1pd * km1pd / (2.0 * ra);
    }
  } else {
    if (typelyr < 0) {
      cx kmpu = ei[0][0] * S.ur[m] + ei[0][1] * S.uz[m] + ei[0][2] * S.tz[m] + ei[0][3] * S.tr[m];
      cx kmsu = ei[1][0] * S.ur[m] + ei[1][1] * S.uz[m] + ei[1][2] * S.tz[m] + ei[1][3] * S.tr[m];
      cint = e[i][0] * e[j][0] * kmpu * kmpu / (2.0 * ra) +
             (e[i][0] * e[j][1] + e[i][1] * e[j][0]) * kmpu * kmsu / (ra + rb) +
             e[i][1] * e[j][1] * kmsu * kmsu / (2.0 * rb);
    } else if (typelyr == 0) {
      cx km1pd = ei[2][0] * S.ur[m] + ei[2][1] * S.uz[m] + ei[2][2] * S.tz[m] + ei[2][3] * S.tr[m];
      cx km1sd = ei[3][0] * S.ur[m] + ei[3][1] * S.uz[m] + ei[3][2] * S.tz[m] + ei[3][3] * S.tr[m];
      cx kmpu = ei[0][0] * S.ur[m + 1] + ei[0][1] * S.uz[m + 1] + ei[0][2] * S.tz[m + 1] + ei[0][3] * S.tr[m + 1];
      cx kmsu = ei[1][0] * S.ur[m + 1] + ei[1][1] * S.uz[m + 1] + ei[1][2] * S.tz[m + 1] + ei[1][3] * S.tr[m + 1];
      cx FA = ffunc(ra, S.zd[m]);
      cx GA = gfunc(ra, S.zd[m]);
      cx FB = ffunc(rb, S.zd[m]);
      cx GB = gfunc(rb, S.zd[m]);
      cx H1 = h1func(ra, rb, S.zd[m]);
      cx H2 = h2func(ra, rb, S.zd[m]);
      cint = e[i][0] * e[j][0] * kmpu * kmpu * FA + e[i][2] * e[j][2] * km1pd * km1pd * FA +
             e[i][1] * e[j][1] * kmsu * kmsu * FB + e[i][3] * e[j][3] * km1sd * km1sd * FB +
             H1 * ((e[i][0] * e[j][1] + e[i][1] * e[j][0]) * kmpu * kmsu +
                   (e[i][2] * e[j][3] + e[i][3] * e[j][2]) * km1pd * km1sd) +
             H2 * ((e[i][0] * e[j][3] + e[i][3] * e[j][0]) * kmpu * km1sd +
                   (e[i][1] * e[j][2] + e[i][2] * e[j][1]) * km1pd * kmsu) +
             GA * (e[i][0] * e[j][2] + e[i][2] * e[j][0]) * kmpu * km1pd +
             GB * (e[i][1] * e[j][3] + e[i][3] * e[j][1]) * kmsu * km1sd;
    } else {
      cx km1pd = ei[2][0] * S.ur[m] + ei[2][1] * S.uz[m] + ei[2][2] * S.tz[m] + ei[2][3] * S.tr[m];
      cx km1sd = ei[3][0] * S.ur[m] + ei[3][1] * S.uz[m] + ei[3][2] * S.tz[m] + ei[3][3] * S.tr[m];
      cint = e[i][2] * e[j][2] * km1pd * km1pd / (2.0 * ra) +
             (e[i][2] * e[j][3] + e[i][3] * e[j][2]) * km1pd * km1sd / (ra + rb) +
             e[i][3] * e[j][3] * km1sd * km1sd / (2.0 * rb);
    }
  }
  return cint.re;
}

// getmat (sregn96.f90:1531-1583)
void ray_getmat(Ray& S, int m, double wvno, double om, double& a12, double& a14, double& a21, double& a23,
                double& ah, double& av, double& bh, double& bv, double& eta, double& rho, double& TA, double& TC,
                double& TF, double& TL, double& TN) {
  if (S.iwat[m] == 1) {
    ah = S.za[m]; av = S.za[m]; bh = 0.0; bv = 0.0; rho = S.zrho[m]; eta = 1.0;
    TL = 0.0; TN = 0.0;
    TC = S.zrho[m] * S.za[m] * S.za[m];
    TA = S.zrho[m] * S.za[m] * S.za[m];
    TF = TA - 2. * TN;
    a12 = -(wvno * wvno - om * om / (ah * ah)) / (rho * om * om);
  } else {
    ah = S.za[m]; av = S.za[m]; bh = S.zb[m]; bv = S.zb[m]; rho = S.zrho[m]; eta = 1.0;
    TL = S.zrho[m] * S.zb[m] * S.zb[m];
    TN = S.zrho[m] * S.zb[m] * S.zb[m];
    TC = S.zrho[m] * S.za[m] * S.za[m];
    TA = S.zrho[m] * S.za[m] * S.za[m];
    TF = TA - 2. * TN;
    a12 = -wvno;
    a14 = 1.0 / TL;
    a21 = wvno * TF / TC;
    a23 = 1.0 / TC;
  }
}

// getdcdh (sregn96.f90:1430-1529)
void ray_getdcdh(Ray& S, double om2, double wvno, double wvno2, double fac) {
  for (int m = 0; m < S.mmax; ++m) {
    double tuz = S.uz[m], ttz = S.tz[m], ttr = S.tr[m], tur;
    if (S.iwat[m] == 1) tur = -wvno * ttz / (S.zrho[m] * om2);
    else tur = S.ur[m];
    double gfac1, gfac2, gfac3, gfac4, gfac5, gfac6;
    if (m == 0) {
      double drho = S.zrho[0] - 0.0, dmu = S.xmu[0] - 0.0, dlm = S.xlam[0] - 0.0;
      double dl2mu = dlm + dmu + dmu;
      double xl2mp = S.xlam[m] + S.xmu[m] + S.xmu[m];
      double duzdzp = (ttz + wvno * S.xlam[m] * tur) / xl2mp;
      double durdzp;
      if (S.iwat[m] == 1) durdzp = wvno * tuz;
      else durdzp = (ttr / S.xmu[m]) - wvno * tuz;
      double drur2 = tur * tur * drho;
      double dlur2 = tur * tur * dl2mu;
      gfac1 = om2 * drho * (tuz * tuz);
      gfac2 = om2 * drur2;
      gfac3 = -wvno2 * dmu * (tuz * tuz);
      gfac4 = -wvno2 * dlur2;
      gfac5 = (xl2mp * (duzdzp * duzdzp));
      gfac6 = (S.xmu[m] * (durdzp * durdzp));
    } else {
      double drho = S.zrho[m] - S.zrho[m - 1];
      double dmu = S.xmu[m] - S.xmu[m - 1];
      double dlm = S.xlam[m] - S.xlam[m - 1];
      double dl2mu = dlm + dmu + dmu;
      double xl2mp = S.xlam[m] + S.xmu[m] + S.xmu[m];
      double xl2mm = S.xlam[m - 1] + S.xmu[m - 1] + S.xmu[m - 1];
      double duzdzp = (ttz + wvno * S.xlam[m] * tur) / xl2mp;
      double durdzp, durdzm, drur2, dlur2, duzdzm;
      if (S.xmu[m] == 0.0) durdzp = wvno * tuz;
      else durdzp = (ttr / S.xmu[m]) - wvno * tuz;
      if (S.xmu[m - 1] == 0.0) durdzm = wvno * tuz;
      else durdzm = (ttr / S.xmu[m - 1]) - wvno * tuz;
      if (S.iwat[m - 1] == 1 && S.iwat[m] == 0) {
        double URB = -wvno * S.tz[m] / (S.zrho[m - 1] * om2);
        drur2 = tur * tur * S.zrho[m] - URB * URB * S.zrho[m - 1];
        dlur2 = tur * tur * xl2mp - URB * URB * xl2mm;
        duzdzm = (ttz + wvno * S.xlam[m - 1] * URB) / S.xlam[m - 1];
      } else if (S.iwat[m - 1] == 1 && S.iwat[m] == 1) {
        double URB = -wvno * S.tz[m] / (S.zrho[m - 1] * om2);
        drur2 = tur * tur * S.zrho[m] - URB * URB * S.zrho[m - 1];
        dlur2 = tur * tur * xl2mp - URB * URB * xl2mm;
        duzdzm = (ttz + wvno * S.xlam[m - 1] * URB) / xl2mm;
      } else {
        drur2 = tur * tur * drho;
        dlur2 = tur * tur * dl2mu;
        duzdzm = (ttz + wvno * S.xlam[m - 1] * tur) / xl2mm;
      }
      gfac1 = om2 * drho * (tuz * tuz);
      gfac2 = om2 * drur2;
      gfac3 = -wvno2 * dmu * (tuz * tuz);
      gfac4 = -wvno2 * dlur2;
      gfac5 = (xl2mp * (duzdzp * duzdzp) - xl2mm * (duzdzm * duzdzm));
      gfac6 = (S.xmu[m] * (durdzp * durdzp) - S.xmu[m - 1] * (durdzm * durdzm));
    }
    double dfac = fac * (gfac1 + gfac2 + gfac3 + gfac4 + gfac5 + gfac6);
    if (std::fabs(dfac) < 1.0e-38) dfac = 0.0;
    S.dcdh[m] = dfac;
  }
}

// energy (sregn96.f90:1061-1196)
void ray_energy(Ray& S, double om, double wvno) {
  const int mmax = S.mmax;
  S.sumi0 = 0.0; S.sumi1 = 0.0; S.sumi2 = 0.0; S.sumi3 = 0.0;
  double c = om / wvno, om2 = om * om, wvno2 = wvno * wvno;
  for (int m = 0; m < mmax; ++m) {
    double a12 = 0, a14 = 0, a21 = 0, a23 = 0, ah, av, bh, bv, eta, rho, TA, TC, TF, TL, TN;
    ray_getmat(S, m, wvno, om, a12, a14, a21, a23, ah, av, bh, bv, eta, rho, TA, TC, TF, TL, TN);
    int typelyr = (m == mmax - 1) ? 1 : 0;
    double INT11 = ray_intijr(S, 1, 1, m, typelyr, om, om2, wvno, wvno2);
    double INT13 = ray_intijr(S, 1, 3, m, typelyr, om, om2, wvno, wvno2);
    double INT22 = ray_intijr(S, 2, 2, m, typelyr, om, om2, wvno, wvno2);
    double INT24 = ray_intijr(S, 2, 4, m, typelyr, om, om2, wvno, wvno2);
    double INT33 = ray_intijr(S, 3, 3, m, typelyr, om, om2, wvno, wvno2);
    double INT44 = ray_intijr(S, 4, 4, m, typelyr, om, om2, wvno, wvno2);
    (void)INT33; (void)bh;
    if (S.iwat[m] == 1) {
      double wr = wvno / (rho * om2);
      double URUR = INT22 * (wr * wr);
      double UZUZ = INT11;
      double URDUZ = -((wvno / (rho * om2)) * a12 * INT22);
      double DUZDUZ = a12 * a12 * INT22;
      S.sumi0 = S.sumi0 + rho * (URUR + UZUZ);
      S.sumi1 = S.sumi1 + TA * URUR;
      S.sumi2 = S.sumi2 - TF * URDUZ;
      S.sumi3 = S.sumi3 + TC * DUZDUZ;
      double facah = rho * ah * (URUR - 2. * eta * URDUZ / wvno);
      double facav = rho * av * DUZDUZ / wvno2;
      S.dcda[m] = facah + facav;
      double facr = -(0.5 * c * c * (URUR + UZUZ));
      S.dcdr[m] = 0.5 * (av * facav + ah * facah) / rho + facr;
      S.ur[m] = -(wvno * S.tz[m] / (rho * om2));
    } else {
      double URUR = INT11;
      double UZUZ = INT22;
      double DURDUR = a12 * a12 * INT22 + 2. * a12 * a14 * INT24 + a14 * a14 * INT44;
      double DUZDUZ = a21 * a21 * INT11 + 2. * a21 * a23 * INT13 + a23 * a23 * INT33;
      double URDUZ = a21 * INT11 + a23 * INT13;
      double UZDUR = a12 * INT22 + a14 * INT24;
      S.sumi0 = S.sumi0 + rho * (URUR + UZUZ);
      S.sumi1 = S.sumi1 + TL * UZUZ + TA * URUR;
      S.sumi2 = S.sumi2 + TL * UZDUR - TF * URDUZ;
      S.sumi3 = S.sumi3 + TL * DURDUR + TC * DUZDUZ;
      double facah = rho * ah * (URUR - 2. * eta * URDUZ / wvno);
      double facav = rho * av * DUZDUZ / wvno2;
      double facbh = 0.0;
      double facbv = rho * bv * (UZUZ + 2. * UZDUR / wvno + DURDUR / wvno2 + 4. * eta * URDUZ / wvno);
      S.dcda[m] = facah + facav;
      S.dcdb[m] = facbv + facbh;
      double facr = -(0.5 * c * c * (URUR + UZUZ));
      S.dcdr[m] = 0.5 * (av * facav + ah * facah + bv * facbv) / rho + facr;
    }
  }
  S.flagr = om2 * S.sumi0 - wvno2 * S.sumi1 - 2.0 * wvno * S.sumi2 - S.sumi3;
  S.ugr = (wvno * S.sumi1 + S.sumi2) / (om * S.sumi0);
  S.are = wvno / (2.0 * om * S.ugr * S.sumi0);
  double fac = S.are * c / wvno2;
  for (int m = 0; m < mmax; ++m) {
    S.dcda[m] = S.dcda[m] / (S.ugr * S.sumi0);
    S.dcdb[m] = S.dcdb[m] / (S.ugr * S.sumi0);
    S.dcdr[m] = S.dcdr[m] / (S.ugr * S.sumi0);
  }
  ray_getdcdh(S, om2, wvno, wvno2, fac);
}

// sprayl (sregn96.f90:1585-1629)
void ray_sprayl(Ray& S, double om, double c, double& csph, double& usph) {
  const double ar = 6371.0;
  double x = c / (2. * ar * om);
  double tm = std::sqrt(1. + x * x);
  double tm3 = tm * tm * tm;
  for (int i = 0; i < S.mmax; ++i) {
    S.dcda[i] = S.dcda[i] * S.vtp[i] / tm3;
    S.dcdb[i] = S.dcdb[i] * S.vtp[i] / tm3;
    S.dcdh[i] = S.dcdh[i] * S.dtp[i] / tm3;
    S.dcdr[i] = S.dcdr[i] * S.rtp[i] / tm3;
  }
  usph = S.ugr * tm;
  csph = c / tm;
}

void ray_setup(Ray& S, const float* thk, const float* vp, const float* vs, const float* rhom, int nlayer,
               int iflsph) {
  S.alloc(nlayer);
  for (int i = 0; i < nlayer; ++i) {
    S.zb[i] = vs[i]; S.za[i] = vp[i]; S.zrho[i] = rhom[i]; S.zd[i] = thk[i];
  }
  S.allfluid = true;
  for (int i = 0; i < nlayer; ++i) {
    if (S.zb[i] > 0.0) { S.allfluid = false; S.iwat[i] = 0; }
    else S.iwat[i] = 1;
  }
  if (iflsph > 0) {
    S.vtp.assign(nlayer, 0); S.dtp.assign(nlayer, 0); S.rtp.assign(nlayer, 0);
    ray_bldsph(S);
  }
  for (int i = 0; i < nlayer; ++i) {
    S.xmu[i] = S.zrho[i] * (S.zb[i] * S.zb[i]);
    S.xlam[i] = S.zrho[i] * (S.za[i] * S.za[i]) - 2 * S.xmu[i];
  }
}

// suffix sums of sregn96.f90:1717-1721 (Fortran sum(x(i+1:mmax)) left to right)
void dcdh_to_thickness(double* x, int mmax) {
  for (int i = 0; i < mmax - 1; ++i) {
    double s = 0.0;
    for (int j = i + 1; j < mmax; ++j) s = s + x[j];
    x[i] = s;
  }
  x[mmax - 1] = 0.0;
}

// ============================================================================
// slegn96.f90
// ============================================================================
struct Love {
  int mmax;
  std::vector<double> zd, zb, zrho, xmu, uu, tt, dcdb, dcdh, dcdr, vtp, dtp, rtp, exl;
  std::vector<int> iwat;
  double cosq, sinq, yl, zl, mu;
  double sumi0, sumi1, sumi2, flagr, ale, ugr;
  void alloc(int n) {
    mmax = n;
    zd.assign(n, 0); zb.assign(n, 0); zrho.assign(n, 0); xmu.assign(n, 0);
    uu.assign(n, 0); tt.assign(n, 0); dcdb.assign(n, 0); dcdh.assign(n, 0); dcdr.assign(n, 0);
    exl.assign(n, 0); iwat.assign(n, 0);
  }
};

// bldsph (slegn96.f90:107-167)
void love_bldsph(Love& S) {
  const double ar = 6371.0;
  double dr = 0.0, r0 = ar;
  S.zd[S.mmax - 1] = 1.0;
  for (int i = 0; i < S.mmax; ++i) {
    dr = dr + S.zd[i];
    double r1 = ar - dr;
    double z0 = ar * std::log(ar / r0);
    double z1 = ar * std::log(ar / r1);
    S.dtp[i] = ar / r0;
    double tmp = (2.0 * ar) / (r0 + r1);
    S.vtp[i] = tmp;
    S.rtp[i] = powm5d(tmp);
    S.zb[i] = S.zb[i] * tmp;
    S.zrho[i] = S.zrho[i] * S.rtp[i];
    S.zd[i] = z1 - z0;
    r0 = r1;
  }
  S.zd[S.mmax - 1] = 0.0;
}

// varl (slegn96.f90:248-328)
void love_varl(Love& S, int m, double& rb, double omega, double wvno, double& xkb, double dpth, double& eexl) {
  xkb = omega / S.zb[m];
  double wvnop = wvno + xkb, wvnom = std::fabs(wvno - xkb);
  rb = std::sqrt(wvnop * wvnom);
  double q = rb * dpth;
  S.mu = S.zrho[m] * S.zb[m] * S.zb[m];
  eexl = 0.0;
  if (wvno < xkb) {
    S.sinq = std::sin(q); S.yl = S.sinq / rb; S.zl = -rb * S.sinq; S.cosq = std::cos(q);
  } else if (wvno == xkb) {
    S.cosq = 1.0; S.yl = dpth; S.zl = 0.0;
  } else if (wvno > xkb) {
    eexl = q;
    double fac = 0.0;
    if (q < 18.0) fac = std::exp(-2.0 * q);
    S.cosq = (1.0 + fac) * 0.5; S.sinq = (1.0 - fac) * 0.5;
    S.yl = S.sinq / rb; S.zl = rb * S.sinq;
  }
}

// up (slegn96.f90:372-445)
void love_up(Love& S, double omega, double wvno, double& fl) {
  const int mmax = S.mmax;
  double rb, xkb, eexl;
  if (S.zb[mmax - 1] > 0.01) {
    love_varl(S, mmax - 1, rb, omega, wvno, xkb, 0.0, eexl);
    S.uu[mmax - 1] = 1.0;
    S.tt[mmax - 1] = -S.xmu[mmax - 1] * rb;
  } else {
    S.uu[mmax - 1] = 1.0;
    S.tt[mmax - 1] = 0.0;
  }
  S.exl[mmax - 1] = 0.0;
  double ttlast = 0.0;
  for (int k = mmax - 2; k >= 0; --k) {
    if (S.iwat[k] == 0) {
      love_varl(S, k, rb, omega, wvno, xkb, S.zd[k], eexl);
      double hl11 = S.cosq, hl12 = S.yl / S.mu, hl21 = S.zl * S.mu, hl22 = S.cosq;
      int k1 = k + 1;
      double a11 = hl11, a22 = hl22, a12 = -hl12, a21 = -hl21;
      double amp0 = a11 * S.uu[k1] + a12 * (S.tt[k1]);
      double str0 = a21 * S.uu[k1] + a22 * (S.tt[k1]);
      double rr = std::fabs(amp0), ss = std::fabs(str0);
      if (ss > rr) rr = ss;
      if (rr < 1.e-30) rr = 1.0;
      S.exl[k] = std::log(rr) + eexl;
      S.uu[k] = amp0 / rr;
      S.tt[k] = str0 / rr;
      ttlast = S.tt[k];
    }
  }
  fl = ttlast;
}

// shfunc (slegn96.f90:179-246); fluid-layer uu/exl are 0 (see header)
void love_shfunc(Love& S, double omega, double wvno) {
  double fl;
  love_up(S, omega, wvno, fl);
  double ext = 0.0;
  double umax = S.uu[0];
  S.tt[0] = 0.0;
  for (int k = 1; k < S.mmax; ++k) {
    if (S.iwat[k] == 0) {
      ext = ext + S.exl[k - 1];
      double fact = 0.0;
      if (ext < 80.0) fact = 1. / std::exp(ext);
      S.uu[k] = S.uu[k] * fact;
      S.tt[k] = S.tt[k] * fact;
    } else {
      S.uu[k] = 0.0; S.tt[k] = 0.0;
    }
    if (std::fabs(S.uu[k]) > std::fabs(umax)) umax = S.uu[k];
  }
  if (S.uu[0] != 0.0) umax = S.uu[0];
  if (std::fabs(umax) > 0.0) {
    for (int k = 0; k < S.mmax; ++k)
      if (S.iwat[k] == 0) { S.uu[k] = S.uu[k] / umax; S.tt[k] = S.tt[k] / umax; }
  }
}

// energy (slegn96.f90:447-629)
void love_energy(Love& S, double omega, double wvno) {
  const int mmax = S.mmax;
  double c = omega / wvno, omega2 = omega * omega, wvno2 = wvno * wvno;
  S.sumi0 = 0.0; S.sumi1 = 0.0; S.sumi2 = 0.0;
  for (int k = 0; k < mmax; ++k) {
    if (S.iwat[k] == 0) {
      double TN = S.zrho[k] * S.zb[k] * S.zb[k];
      double TL = S.zrho[k] * S.zb[k] * S.zb[k];
      double VSHH = S.zb[k], VSHV = S.zb[k];
      int k1 = k + 1;
      double drho = S.zrho[k], dpth = S.zd[k], rb, xkb, eexl;
      love_varl(S, k, rb, omega, wvno, xkb, dpth, eexl);
      double dmu = S.xmu[k];
      if (rb < 1.0e-10) rb = 1.0e-10;
      double upup, dupdup;
      if (k == mmax - 1) {
        upup = (0.5 / rb) * S.uu[mmax - 1] * S.uu[mmax - 1];
        dupdup = (0.5 * rb) * S.uu[mmax - 1] * S.uu[mmax - 1];
      } else {
        cx nub = C(rb, 0.0);
        if (wvno < xkb) nub = C(0.0, rb);
        cx xnub = dmu * nub;
        cx ei11 = C(0.5 / wvno), ei12 = 0.5 / (wvno * xnub), ei21 = C(0.5 / wvno), ei22 = -(0.5 / (wvno * xnub));
        cx el11 = C(wvno), el12 = C(wvno);
        (void)ei21;
        cx km1dn = ei21 * S.uu[k] + ei22 * S.tt[k];
        cx kmup = ei11 * S.uu[k1] + ei12 * S.tt[k1];
        cx f3 = nub * dpth;
        cx exqq = C(0.0);
        if (f3.re < 40.0) exqq = cexp_(-2.0 * f3);
        cx f = (1.0 - exqq) / (2.0 * nub);
        exqq = C(0.0);
        if (f3.re < 75.0) exqq = cexp_(-f3);
        cx g = dpth * exqq;
        cx f1 = f * (el11 * el11 * kmup * kmup + el12 * el12 * km1dn * km1dn);
        cx f2 = g * (el11 * el12 + el11 * el12) * kmup * km1dn;
        upup = (f1 + f2).re;
        dupdup = (nub * nub * (f1 - f2)).re;
      }
      S.sumi0 = S.sumi0 + drho * upup;
      S.sumi1 = S.sumi1 + TN * upup;
      S.sumi2 = S.sumi2 + TL * dupdup;
      double DCDBH = c * drho * VSHH * upup;
      double DCDBV = c * drho * VSHV * dupdup / wvno2;
      S.dcdb[k] = DCDBH + DCDBV;
      double DCDRSH = 0.5 * c * (-c * c * upup + VSHH * VSHH * upup + VSHV * VSHV * dupdup / wvno2);
      S.dcdr[k] = DCDRSH;
    } else {
      S.dcdb[k] = 0.0; S.dcdr[k] = 0.0;
    }
  }
  for (int k = 0; k < mmax; ++k) {
    if (S.iwat[k] == 0) { S.dcdb[k] = S.dcdb[k] / S.sumi1; S.dcdr[k] = S.dcdr[k] / S.sumi1; }
    else { S.dcdb[k] = 0.0; S.dcdr[k] = 0.0; }
  }
  S.flagr = omega2 * S.sumi0 - wvno2 * S.sumi1 - S.sumi2;
  S.ugr = S.sumi1 / (c * S.sumi0);
  S.ale = 0.5 / S.sumi1;
  double fac = S.ale * c / wvno2;
  int llflag = 0;
  for (int k = 0; k < mmax; ++k) {
    if (S.iwat[k] == 0) {
      double drho, dmu, dvdz;
      if (llflag == 0) { drho = S.zrho[k]; dmu = S.xmu[k]; dvdz = 0.0; }
      else {
        drho = S.zrho[k] - S.zrho[k - 1];
        dmu = S.xmu[k] - S.xmu[k - 1];
        dvdz = S.tt[k] * S.tt[k] * (1.0 / S.xmu[k] - 1.0 / S.xmu[k - 1]);
      }
      double dfac = fac * (S.uu[k] * S.uu[k] * (omega2 * drho - wvno2 * dmu) + dvdz);
      S.dcdh[k] = (std::fabs(dfac) < 1.0e-38) ? 0.0 : dfac;
      llflag = llflag + 1;
    } else {
      S.dcdh[k] = 0.0;
    }
  }
}

void love_setup(Love& S, const float* thk, const float* vs, const float* rhom, int nlayer, int iflsph, bool pu) {
  S.alloc(nlayer);
  for (int i = 0; i < nlayer; ++i) { S.zb[i] = vs[i]; S.zrho[i] = rhom[i]; S.zd[i] = thk[i]; }
  for (int i = 0; i < nlayer; ++i) {
    if (pu) S.iwat[i] = (S.zb[i] > 0.0) ? 0 : 1;
    else S.iwat[i] = (S.zb[i] == 0.0) ? 1 : 0;
  }
  if (iflsph > 0) {
    S.vtp.assign(nlayer, 0); S.dtp.assign(nlayer, 0); S.rtp.assign(nlayer, 0);
    love_bldsph(S);
  }
  for (int i = 0; i < nlayer; ++i) S.xmu[i] = S.zrho[i] * (S.zb[i] * S.zb[i]);
}

// ============================================================================
// empirical.cpp, SurfaceWave.cpp column path
// ============================================================================
void empirical_relation(float vsz, float& vpz, float& rhoz) {
  double v = vsz;
  vpz = (float)(0.9409 + 2.0947 * v - 0.8206 * std::pow(v, 2) + 0.2683 * std::pow(v, 3) - 0.0251 * std::pow(v, 4));
  double p = vpz;
  rhoz = (float)(1.6612 * p - 0.4721 * std::pow(p, 2) + 0.0671 * std::pow(p, 3) - 0.0043 * std::pow(p, 4) +
                 0.000106 * std::pow(p, 5));
}
void empirical_deriv(float vp, float vs, float& drda, float& dadb) {
  double p = vp, s = vs;
  drda = (float)(1.6612 - 0.4721 * 2 * p + 0.0671 * 3 * std::pow(p, 2) - 0.0043 * 4 * std::pow(p, 3) +
                 0.000106 * 5 * std::pow(p, 4));
  dadb = (float)(2.0947 - 0.8206 * 2 * s + 0.2683 * 3 * std::pow(s, 2) - 0.0251 * 4 * std::pow(s, 3));
}

// number of leading fluid nodes (vs == 0)
int count_water(const float* vs, int nz) {
  int nw = 0;
  while (nw < nz - 1 && vs[nw] == 0.0f) ++nw;
  return nw;
}

// grid2LayerModel (SurfaceWave.cpp:113-155), generalised to nw>=1 leading
// fluid nodes merged into one layer; identical to the reference for nw<=1.
int grid2layer(const float* dep, const float* vp, const float* vs, const float* rho, int nz, int sublayers, float* rthk,
               float* rvp, float* rvs, float* rrho) {
  int n = sublayers + 1;
  int nw = count_water(vs, nz);
  int rmax, istart;
  if (nw > 0) {
    rmax = (nz - nw) + (nz - nw - 1) * sublayers + 1;
    istart = nw;
    rthk[0] = dep[nw] - dep[0];
    rrho[0] = rho[0];
    rvs[0] = 0.0f;
    rvp[0] = vp[0];
  } else {
    rmax = nz + (nz - 1) * sublayers;
    istart = 0;
  }
  int k = (nw > 0) ? 1 : 0;
  for (int i = istart; i < nz - 1; ++i) {
    float thk = (dep[i + 1] - dep[i]) / n;
    for (int j = 0; j < n; ++j) {
      rthk[k] = thk;
      rvp[k] = (float)(vp[i] + (2 * j + 1) * (vp[i + 1] - vp[i]) / (2.0 * n));
      rvs[k] = (float)(vs[i] + (2 * j + 1) * (vs[i + 1] - vs[i]) / (2.0 * n));
      rrho[k] = (float)(rho[i] + (2 * j + 1) * (rho[i + 1] - rho[i]) / (2.0 * n));
      k++;
    }
  }
  k = rmax - 1;
  rthk[k] = 0.0f;
  rvp[k] = vp[nz - 1];
  rvs[k] = vs[nz - 1];
  rrho[k] = rho[nz - 1];
  return rmax;
}

// _ParamConvert (SurfaceWave.cpp:59-101), generalised like grid2layer
void param_convert(const float* vs, int nz, int sublayer, int rmax, const double* rdcdm, double* dcdm) {
  int n = sublayer + 1;
  int nw = count_water(vs, nz);
  if (nw == 0) {
    for (int i = 0; i < nz; ++i) {
      double tup = 0.0, tdwn = 0.0;
      int idup = (i - 1) * n, iddw = i * n;
      dcdm[i] = 0.0;
      for (int j = 0; j < n; ++j) {
        double tmp = (2. * j + 1.0) / (2. * n);
        if (idup + j >= 0) tup += rdcdm[idup + j] * tmp;
        if (iddw + j < rmax) tdwn += rdcdm[iddw + j] * (1.0 - tmp);
        if (iddw == rmax - 1) tdwn += rdcdm[rmax - 1];
      }
      dcdm[i] += tup + tdwn;
    }
  } else {
    dcdm[0] = rdcdm[0];
    for (int i = 1; i < nw; ++i) dcdm[i] = 0.0;
    for (int i = nw; i < nz; ++i) {
      dcdm[i] = 0.0;
      double tup = 0.0, tdwn = 0.0;
      int idup = (i - nw - 1) * n + 1, iddw = (i - nw) * n + 1;
      for (int j = 0; j < n; ++j) {
        double tmp = (2. * j + 1.0) / (2. * n);
        if (idup + j >= 1) tup += rdcdm[idup + j] * tmp;
        if (iddw + j < rmax) tdwn += rdcdm[iddw + j] * (1.0 - tmp);
        if (iddw == rmax - 1) tdwn += rdcdm[rmax - 1];
      }
      dcdm[i] += tup + tdwn;
    }
  }
}

}  // namespace

// ============================================================================
// C-ABI
// ============================================================================
extern "C" {

// ---- the reference's Fortran C-ABI (swd.hpp:5-96), reference-faithful -----
void surfdisp96_(const float* thkm, const float* vpm, const float* vsm, const float* rhom, int nlayer, int iflsph,
                 int iwave, int mode, int igr, int kmax, const double* t, double* cg, int* ierr) {
  surfdisp96_impl(thkm, vpm, vsm, rhom, nlayer, iflsph, iwave, mode, igr, kmax, t, cg, ierr, REF_OPTS, nullptr,
                  nullptr);
}

void sregn96_(const float* thk, const float* vp, const float* vs, const float* rhom, int nlayer, const double* t,
              double* cp, double* cg, double* dispu, double* dispw, double* stressu, double* stressw, double* dc2da,
              double* dc2db, double* dc2dh, double* dc2dr, int iflsph) {
  Ray S;
  ray_setup(S, thk, vp, vs, rhom, nlayer, iflsph);
  const int mmax = nlayer;
  double twopi = 2.0 * PI_F;
  double omega = twopi / *t;
  double c = *cp;
  S.ugr = c;
  double wvno = omega / c;
  ray_svfunc(S, omega, wvno);
  ray_energy(S, omega, wvno);
  if (std::fabs(c) < 1.0e-36) c = 0.0;
  if (std::fabs(S.ugr) < 1.0e-36) S.ugr = 0.0;
  double csph, usph;
  if (iflsph > 0) ray_sprayl(S, omega, c, csph, usph);
  else { csph = c; usph = S.ugr; }
  dcdh_to_thickness(S.dcdh.data(), mmax);
  for (int i = 0; i < mmax; ++i) {
    dc2da[i] = S.dcda[i]; dc2db[i] = S.dcdb[i]; dc2dr[i] = S.dcdr[i]; dc2dh[i] = S.dcdh[i];
    dispu[i] = S.ur[i]; dispw[i] = S.uz[i]; stressu[i] = S.tr[i]; stressw[i] = S.tz[i];
  }
  *cp = csph;
  *cg = usph;
}

void sregnpu_(const float* thk, const float* vp, const float* vs, const float* rhom, int nlayer, const double* t,
              double* cp, double* cg, double* dispu, double* dispw, double* stressu, double* stressw, double* t1,
              double* cp1, double* t2, double* cp2, double* dc2da, double* dc2db, double* dc2dh, double* dc2dr,
              double* du2da, double* du2db, double* du2dh, double* du2dr, int iflsph) {
  Ray S;
  ray_setup(S, thk, vp, vs, rhom, nlayer, iflsph);
  const int n = nlayer;
  std::vector<double> a1(n), a2(n), b1(n), b2(n), h1(n), h2(n), r1(n), r2(n);
  double twopi = 2.0 * PI_F;
  double omega = twopi / *t, c = *cp, wvno = omega / c;
  ray_svfunc(S, omega, wvno);
  ray_energy(S, omega, wvno);
  double cgv = S.ugr;
  for (int i = 0; i < n; ++i) {
    dc2da[i] = S.dcda[i]; dc2db[i] = S.dcdb[i]; dc2dr[i] = S.dcdr[i]; dc2dh[i] = S.dcdh[i];
    dispu[i] = S.ur[i]; dispw[i] = S.uz[i]; stressu[i] = S.tr[i]; stressw[i] = S.tz[i];
  }
  omega = twopi / *t1; c = *cp1; wvno = omega / c;
  ray_svfunc(S, omega, wvno);
  ray_energy(S, omega, wvno);
  for (int i = 0; i < n; ++i) { a1[i] = S.dcda[i]; b1[i] = S.dcdb[i]; r1[i] = S.dcdr[i]; h1[i] = S.dcdh[i]; }
  omega = twopi / *t2; c = *cp2; wvno = omega / c;
  ray_svfunc(S, omega, wvno);
  ray_energy(S, omega, wvno);
  for (int i = 0; i < n; ++i) { a2[i] = S.dcda[i]; b2[i] = S.dcdb[i]; r2[i] = S.dcdr[i]; h2[i] = S.dcdh[i]; }
  double uc1 = cgv / *cp;
  double dt = (*t2 - *t1);
  double f1 = uc1 * (2.0 - uc1), f2 = uc1 * uc1 * *t;
  for (int i = 0; i < n; ++i) {
    du2da[i] = f1 * S.dcda[i] - f2 * (a2[i] - a1[i]) / dt;
    du2db[i] = f1 * S.dcdb[i] - f2 * (b2[i] - b1[i]) / dt;
    du2dr[i] = f1 * S.dcdr[i] - f2 * (r2[i] - r1[i]) / dt;
    du2dh[i] = f1 * S.dcdh[i] - f2 * (h2[i] - h1[i]) / dt;
  }
  double cpv = *cp;
  if (iflsph > 0) {
    const double ar = 6371.0;
    omega = twopi / *t;
    double x = cpv / (2. * ar * omega);
    double tm = std::sqrt(1. + x * x);
    double y = 0.5 / (ar * omega);
    double tm1 = (y * y) / tm;
    double tm3 = tm * tm * tm;
    for (int i = 0; i < n; ++i) {
      du2da[i] = (tm * du2da[i] + cgv * cpv * dc2da[i] * tm1) * S.vtp[i];
      du2db[i] = (tm * du2db[i] + cgv * cpv * dc2db[i] * tm1) * S.vtp[i];
      du2dr[i] = (tm * du2dr[i] + cgv * cpv * dc2dr[i] * tm1) * S.rtp[i];
      du2dh[i] = (tm * du2dh[i] + cgv * cpv * dc2dh[i] * tm1) * S.dtp[i];
      dc2da[i] = dc2da[i] / tm3 * S.vtp[i];
      dc2db[i] = dc2db[i] / tm3 * S.vtp[i];
      dc2dr[i] = dc2dr[i] / tm3 * S.rtp[i];
      dc2dh[i] = dc2dh[i] / tm3 * S.dtp[i];
    }
    cpv = cpv / tm;
    cgv = cgv * tm;
  }
  dcdh_to_thickness(dc2dh, n);
  dcdh_to_thickness(du2dh, n);
  *cp = cpv;
  *cg = cgv;
}

void slegn96_(const float* thk, const float* vs, const float* rhom, int nlayer, const double* t, double* cp,
              double* cg, double* disp, double* stress, double* dc2db, double* dc2dh, double* dc2dr, int iflsph) {
  Love S;
  love_setup(S, thk, vs, rhom, nlayer, iflsph, false);
  double twopi = 2.0 * PI_F;
  double omega = twopi / *t;
  double c = *cp;
  double wvno = omega / c;
  love_shfunc(S, omega, wvno);
  love_energy(S, omega, wvno);
  double csph, usph;
  if (iflsph > 0) {
    const double a = 6371.0;
    double x = 3.0 * c / (2. * a * omega);
    double tm = std::sqrt(1. + x * x);
    double tm3 = tm * tm * tm;
    for (int i = 0; i < S.mmax; ++i) {
      S.dcdb[i] = S.dcdb[i] * S.vtp[i] / tm3;
      S.dcdh[i] = S.dcdh[i] * S.dtp[i] / tm3;
      S.dcdr[i] = S.dcdr[i] * S.rtp[i] / tm3;
    }
    csph = c / tm;
    usph = S.ugr * tm;
  } else { csph = c; usph = S.ugr; }
  if (std::fabs(S.ugr) < 1.0e-36) S.ugr = 0.0;
  dcdh_to_thickness(S.dcdh.data(), S.mmax);
  for (int i = 0; i < S.mmax; ++i) {
    disp[i] = S.uu[i]; stress[i] = S.uu[i];  // slegn96.f90:770 copies uu into stress
    dc2db[i] = S.dcdb[i]; dc2dr[i] = S.dcdr[i]; dc2dh[i] = S.dcdh[i];
  }
  *cp = csph;
  *cg = usph;
}

void slegnpu_(const float* thk, const float* vs, const float* rhom, int nlayer, const double* t, double* cp,
              double* cg, double* disp, double* stress, double* t1, double* cp1, double* t2, double* cp2,
              double* dc2db, double* dc2dh, double* dc2dr, double* du2db, double* du2dh, double* du2dr, int iflsph) {
  Love S;
  love_setup(S, thk, vs, rhom, nlayer, iflsph, true);
  const int n = nlayer;
  std::vector<double> b1(n), b2(n), h1(n), h2(n), r1(n), r2(n);
  double twopi = 2.0 * PI_F;
  double omega = twopi / *t, c = *cp, wvno = omega / c;
  love_shfunc(S, omega, wvno);
  love_energy(S, omega, wvno);
  double cgv = S.ugr;
  for (int i = 0; i < n; ++i) {
    dc2db[i] = S.dcdb[i]; stress[i] = S.tt[i]; dc2dr[i] = S.dcdr[i]; disp[i] = S.uu[i]; dc2dh[i] = S.dcdh[i];
  }
  omega = twopi / *t1; c = *cp1; wvno = omega / c;
  love_shfunc(S, omega, wvno);
  love_energy(S, omega, wvno);
  for (int i = 0; i < n; ++i) { b1[i] = S.dcdb[i]; r1[i] = S.dcdr[i]; h1[i] = S.dcdh[i]; }
  omega = twopi / *t2; c = *cp2; wvno = omega / c;
  love_shfunc(S, omega, wvno);
  love_energy(S, omega, wvno);
  for (int i = 0; i < n; ++i) { b2[i] = S.dcdb[i]; r2[i] = S.dcdr[i]; h2[i] = S.dcdh[i]; }
  double uc1 = cgv / *cp;
  double dt = (*t2 - *t1);
  double f1 = uc1 * (2.0 - uc1), f2 = uc1 * uc1 * *t;
  for (int i = 0; i < n; ++i) {
    du2db[i] = f1 * S.dcdb[i] - f2 * (b2[i] - b1[i]) / dt;
    du2dr[i] = f1 * S.dcdr[i] - f2 * (r2[i] - r1[i]) / dt;
    du2dh[i] = f1 * S.dcdh[i] - f2 * (h2[i] - h1[i]) / dt;
  }
  double cpv = *cp;
  if (iflsph > 0) {
    const double ar = 6371.0;
    omega = twopi / *t;
    double x = 3.0 * cpv / (2. * ar * omega);
    double tm = std::sqrt(1. + x * x);
    double y = 1.5 / (ar * omega);
    double tm1 = (y * y) / tm;
    double tm3 = tm * tm * tm;
    for (int i = 0; i < n; ++i) {
      du2db[i] = (tm * du2db[i] + cgv * cpv * dc2db[i] * tm1) * S.vtp[i];
      du2dr[i] = (tm * du2dr[i] + cgv * cpv * dc2dr[i] * tm1) * S.rtp[i];
      du2dh[i] = (tm * du2dh[i] + cgv * cpv * dc2dh[i] * tm1) * S.dtp[i];
      dc2db[i] = dc2db[i] / tm3 * S.vtp[i];
      dc2dr[i] = dc2dr[i] / tm3 * S.rtp[i];
      dc2dh[i] = dc2dh[i] / tm3 * S.dtp[i];
    }
    cpv = cpv / tm;
    cgv = cgv * tm;
  }
  dcdh_to_thickness(dc2dh, n);
  dcdh_to_thickness(du2dh, n);
  *cp = cpv;
  *cg = cgv;
}

// ---- oracle extensions ------------------------------------------------------
// surfdisp96 with a selectable refinement: refine=0 reference nevill,
// refine=1 tight Brent with bracket width <= rtol*c; sngl=0 keeps the FP64 root.
void swdo_surfdisp96_ex(const float* thkm, const float* vpm, const float* vsm, const float* rhom, int nlayer,
                        int iflsph, int iwave, int mode, int igr, int kmax, const double* t, double* cg, int* ierr,
                        int refine, double rtol, int sngl, long* nevals, int* iterlim) {
  RootOpts o{refine, rtol, sngl};
  surfdisp96_impl(thkm, vpm, vsm, rhom, nlayer, iflsph, iwave, mode, igr, kmax, t, cg, ierr, o, nevals, iterlim);
}

// a single secular-function value (flat model as given, after the same
// flattening surfdisp96 applies when iflsph=1); for tests of the sign change
double swdo_dltar(const float* thkm, const float* vpm, const float* vsm, const float* rhom, int nlayer, int iflsph,
                  int iwave, double t, double c) {
  Sd96 M;
  M.mmax = nlayer;
  M.d.assign(thkm, thkm + nlayer); M.a.assign(vpm, vpm + nlayer);
  M.b.assign(vsm, vsm + nlayer); M.rho.assign(rhom, rhom + nlayer);
  M.rtp.assign(nlayer, 0.f); M.dtp.assign(nlayer, 0.f); M.btp.assign(nlayer, 0.f);
  M.llw = (M.b[0] <= 0.0f) ? 2 : 1;
  if (iflsph == 1) { sphere(M, 0, 0); sphere(M, iwave, 1); }
  double omega = TWOPI / t;
  return dltar(M, omega / c, omega, iwave);
}

void swdo_gtsolh(float a, float b, float* c) { gtsolh(a, b, *c); }

void swdo_empirical_relation(const float* vs, float* vp, float* rho, int n) {
  for (int i = 0; i < n; ++i) empirical_relation(vs[i], vp[i], rho[i]);
}
void swdo_empirical_deriv(const float* vp, const float* vs, float* drda, float* dadb, int n) {
  for (int i = 0; i < n; ++i) empirical_deriv(vp[i], vs[i], drda[i], dadb[i]);
}
int swdo_grid2layer(const float* dep, const float* vp, const float* vs, const float* rho, int nz, int sublayers,
                    float* rthk, float* rvp, float* rvs, float* rrho) {
  return grid2layer(dep, vp, vs, rho, nz, sublayers, rthk, rvp, rvs, rrho);
}
void swdo_param_convert(const float* vs, int nz, int sublayer, int rmax, const double* rdcdm, double* dcdm) {
  param_convert(vs, nz, sublayer, rmax, rdcdm, dcdm);
}

}  // extern "C"

// ============================================================================
// surfdisp.cpp wrapper and the SurfaceWave.cpp column path
// ============================================================================
namespace {

enum { ST_OK = 0, ST_NO_ROOT = 1, ST_RETRIED = 2, ST_NAN_INPUT = 3 };

// _flat2sphere (surfdisp.cpp:17-51); wtype 0=Rc 1=Rg 2=Lc 3=Lg
double flat2sphere(double t, double c, int wtype) {
  const double ar = 6371.0;
  double omega = 2.0 * M_PI / t;
  double x = ((wtype >= 2) ? 1.5 : 0.5) * c / (ar * omega);
  double tm = std::sqrt(1. + std::pow(x, 2));
  return (wtype == 0 || wtype == 2) ? c / tm : c * tm;
}

// surfdisp (surfdisp.cpp:64-116): retry of failed periods one at a time; the
// reference's exit(1) becomes c=0 with status NO_ROOT.
void surfdisp_w(const float* thk, const float* vp, const float* vs, const float* rho, int nlayer, const double* t,
                double* cg, int kmax, int wtype, int mode, bool sphere, bool keep_flat, const RootOpts& o, long* nev,
                int* iterlim, int* status) {
  int iwave = (wtype >= 2) ? 1 : 2;
  int igr = (wtype == 1 || wtype == 3) ? 1 : 0;
  int ifsph = sphere ? 1 : 0;
  int ierr;
  if (status) for (int i = 0; i < kmax; ++i) status[i] = ST_OK;
  surfdisp96_impl(thk, vp, vs, rho, nlayer, ifsph, iwave, mode + 1, igr, kmax, t, cg, &ierr, o, nev, iterlim);
  if (ierr != 0) {
    for (int i = 0; i < kmax; ++i) {
      if (cg[i] == 0.0 || std::isnan(cg[i])) {
        surfdisp96_impl(thk, vp, vs, rho, nlayer, ifsph, iwave, mode + 1, igr, 1, &t[i], &cg[i], &ierr, o, nev,
                        iterlim);
        if (ierr != 0 || cg[i] == 0.0 || std::isnan(cg[i])) {
          cg[i] = 0.0;
          if (status) status[i] = ST_NO_ROOT;
        } else if (status) {
          status[i] = ST_RETRIED;
        }
      }
    }
  }
  // higher-mode periods beyond a mode's existence end as zeros without ierr
  // (surfdisp96.f:322,358-364): no retry, marked NO_ROOT
  if (status)
    for (int i = 0; i < kmax; ++i)
      if ((cg[i] == 0.0 || std::isnan(cg[i])) && status[i] == ST_OK) status[i] = ST_NO_ROOT;
  if (sphere && !keep_flat)
    for (int i = 0; i < kmax; ++i) cg[i] = flat2sphere(t[i], cg[i], wtype);
}

struct Tables {
  const double* t[4];  // Rc, Rg, Lc, Lg: (ntmax, nmode) column-major, -1 padded
  int ntmax[4], nmode[4];
};

int get_nt_row(const double* col, int ntmax) {
  int n;
  for (n = 0; n < ntmax; ++n) if (col[n] == -1) break;
  return n;
}

struct Opts {
  RootOpts ro;
  int sphere;
};

// Conditioning probe (test hook, not a reference behaviour): kernel1d and
// disp1d hand the eigenfunction routines c*(1+g_cpert) instead of each root
// c (and c1, c2 of the group kernels), so a test can measure how far the
// oracle's own kernels and group velocities move under a rounding-level
// change of their input.  0 (the default) leaves both exactly as the
// reference.
double g_cpert = 0.0;
// A second probe: c1 and c2 of the group kernels (the roots at T(1 +- 0.005))
// moved by g_ulp[0] and g_ulp[1] REAL*4 ulps, each on its own; 0 leaves them.
int g_ulp[2] = {0, 0};

double ulp_step(double c, int n) {
  float f = (float)c;
  for (; n > 0; --n) f = std::nextafter(f, HUGE_VALF);
  for (; n < 0; ++n) f = std::nextafter(f, -HUGE_VALF);
  return (double)f;
}

// kernel1D (SurfaceWave.cpp:266-412); kvs/kvp/krho are (nz, kmax) column-major
void kernel1d(const float* vs, const float* vp, const float* rho, const float* dep, int nz, const Tables& T,
              double* vc, double* vout, double* kvs, double* kvp, double* krho, int* status, const Opts& op,
              long* nev, int* iterlim) {
  const int sublayer = 3;
  int rmax0 = nz + (nz - 1) * sublayer;
  std::vector<float> rvp(rmax0), rvs(rmax0), rthk(rmax0), rrho(rmax0);
  int rmax = grid2layer(dep, vp, vs, rho, nz, sublayer, rthk.data(), rvp.data(), rvs.data(), rrho.data());
  std::vector<double> ur(rmax), uz(rmax), tr(rmax), tz(rmax), dudar(rmax), dudbr(rmax), dudrr(rmax), dudhr(rmax),
      dcdar(rmax), dcdbr(rmax), dcdrr(rmax), dcdhr(rmax);
  bool sphere = op.sphere != 0;
  int iflsph = op.sphere;
  const float *TH = rthk.data(), *VP = rvp.data(), *VS = rvs.data(), *RH = rrho.data();
  int idx = 0;
  for (int w = 0; w < 4; ++w) {
    if (T.ntmax[w] * T.nmode[w] <= 0) continue;
    for (int mode = 0; mode < T.nmode[w]; ++mode) {
      const double* tt = T.t[w] + (size_t)mode * T.ntmax[w];
      int nt = get_nt_row(tt, T.ntmax[w]);
      if (nt == 0) continue;
      if (w == 0 || w == 2) {  // phase: Rc (sregn96) / Lc (slegn96)
        surfdisp_w(TH, VP, VS, RH, rmax, tt, vc + idx, nt, w, mode, sphere, true, op.ro, nev, iterlim,
                   status ? status + idx : nullptr);
        for (int i = 0; i < nt; ++i) {
          int k = i + idx;
          double cg;
          if (vc[k] == 0.0) {  // no root: the reference would have exited
            vout[k] = 0.0;
            for (int iz = 0; iz < nz; ++iz) { kvs[k * nz + iz] = 0; kvp[k * nz + iz] = 0; krho[k * nz + iz] = 0; }
            continue;
          }
          if (g_cpert != 0.0) vc[k] = vc[k] * (1.0 + g_cpert);
          if (w == 0) {
            sregn96_(TH, VP, VS, RH, rmax, &tt[i], vc + k, &cg, ur.data(), uz.data(), tr.data(), tz.data(),
                     dcdar.data(), dcdbr.data(), dcdhr.data(), dcdrr.data(), iflsph);
            param_convert(vs, nz, sublayer, rmax, dcdar.data(), kvp + k * nz);
            param_convert(vs, nz, sublayer, rmax, dcdbr.data(), kvs + k * nz);
            param_convert(vs, nz, sublayer, rmax, dcdrr.data(), krho + k * nz);
          } else {
            slegn96_(TH, VS, RH, rmax, &tt[i], vc + k, &cg, uz.data(), tz.data(), dcdbr.data(), dcdhr.data(),
                     dcdrr.data(), iflsph);
            param_convert(vs, nz, sublayer, rmax, dcdbr.data(), kvs + k * nz);
            param_convert(vs, nz, sublayer, rmax, dcdrr.data(), krho + k * nz);
            for (int iz = 0; iz < nz; ++iz) kvp[k * nz + iz] = 0.;
          }
          vout[k] = vc[k];
        }
      } else {  // group: Rg (sregnpu) / Lg (slegnpu)
        std::vector<double> cp(nt), t1(nt), t2(nt), c1(nt), c2(nt);
        std::vector<int> s0(nt), s1(nt), s2(nt);
        double dt = 0.01;
        for (int i = 0; i < nt; ++i) { t1[i] = tt[i] * (1.0 + 0.5 * dt); t2[i] = tt[i] * (1.0 - 0.5 * dt); }
        int wp = (w == 1) ? 0 : 2;  // the reference calls surfdisp with "Rc"/"Lc"
        surfdisp_w(TH, VP, VS, RH, rmax, tt, cp.data(), nt, wp, mode, sphere, true, op.ro, nev, iterlim, s0.data());
        surfdisp_w(TH, VP, VS, RH, rmax, t1.data(), c1.data(), nt, wp, mode, sphere, true, op.ro, nev, iterlim,
                   s1.data());
        surfdisp_w(TH, VP, VS, RH, rmax, t2.data(), c2.data(), nt, wp, mode, sphere, true, op.ro, nev, iterlim,
                   s2.data());
        for (int i = 0; i < nt; ++i) {
          int k = i + idx;
          if (status) {
            int st = ST_OK;
            if (s0[i] == ST_NO_ROOT || s1[i] == ST_NO_ROOT || s2[i] == ST_NO_ROOT) st = ST_NO_ROOT;
            else if (s0[i] == ST_RETRIED || s1[i] == ST_RETRIED || s2[i] == ST_RETRIED) st = ST_RETRIED;
            status[k] = st;
          }
          if (cp[i] == 0.0 || c1[i] == 0.0 || c2[i] == 0.0) {
            vc[k] = 0.0; vout[k] = 0.0;
            for (int iz = 0; iz < nz; ++iz) { kvs[k * nz + iz] = 0; kvp[k * nz + iz] = 0; krho[k * nz + iz] = 0; }
            continue;
          }
          if (g_cpert != 0.0) {
            cp[i] = cp[i] * (1.0 + g_cpert);
            c1[i] = c1[i] * (1.0 + g_cpert);
            c2[i] = c2[i] * (1.0 + g_cpert);
          }
          if (g_ulp[0]) c1[i] = ulp_step(c1[i], g_ulp[0]);
          if (g_ulp[1]) c2[i] = ulp_step(c2[i], g_ulp[1]);
          if (w == 1) {
            sregnpu_(TH, VP, VS, RH, rmax, &tt[i], &cp[i], vc + k, ur.data(), uz.data(), tr.data(), tz.data(),
                     &t1[i], &c1[i], &t2[i], &c2[i], dcdar.data(), dcdbr.data(), dcdhr.data(), dcdrr.data(),
                     dudar.data(), dudbr.data(), dudhr.data(), dudrr.data(), iflsph);
            param_convert(vs, nz, sublayer, rmax, dudar.data(), kvp + k * nz);
            param_convert(vs, nz, sublayer, rmax, dudbr.data(), kvs + k * nz);
            param_convert(vs, nz, sublayer, rmax, dudrr.data(), krho + k * nz);
          } else {
            slegnpu_(TH, VS, RH, rmax, &tt[i], &cp[i], vc + k, uz.data(), tz.data(), &t1[i], &c1[i], &t2[i],
                     &c2[i], dcdbr.data(), dcdhr.data(), dcdrr.data(), dudbr.data(), dudhr.data(), dudrr.data(),
                     iflsph);
            param_convert(vs, nz, sublayer, rmax, dudbr.data(), kvs + k * nz);
            param_convert(vs, nz, sublayer, rmax, dudrr.data(), krho + k * nz);
            for (int iz = 0; iz < nz; ++iz) kvp[k * nz + iz] = 0.;
          }
          vout[k] = vc[k];
          vc[k] = cp[i];
        }
      }
      idx += nt;
    }
  }
}

// disp1D (SurfaceWave.cpp:177-255) incl. groupvel_r/_l (surfdisp.cpp:126-175)
void disp1d(const float* vs, const float* vp, const float* rho, const float* dep, int nz, const Tables& T, double* vc,
            double* vout, int* status, const Opts& op, long* nev, int* iterlim) {
  const int sublayer = 3;
  int rmax0 = nz + (nz - 1) * sublayer;
  std::vector<float> rvp(rmax0), rvs(rmax0), rthk(rmax0), rrho(rmax0);
  int rmax = grid2layer(dep, vp, vs, rho, nz, sublayer, rthk.data(), rvp.data(), rvs.data(), rrho.data());
  bool sphere = op.sphere != 0;
  int iflsph = op.sphere;
  const float *TH = rthk.data(), *VP = rvp.data(), *VS = rvs.data(), *RH = rrho.data();
  std::vector<double> b0(rmax), b1(rmax), b2(rmax), b3(rmax), b4(rmax), b5(rmax), b6(rmax), b7(rmax);
  int idx = 0;
  for (int w = 0; w < 4; ++w) {
    if (T.ntmax[w] * T.nmode[w] <= 0) continue;
    for (int mode = 0; mode < T.nmode[w]; ++mode) {
      const double* tt = T.t[w] + (size_t)mode * T.ntmax[w];
      int nt = get_nt_row(tt, T.ntmax[w]);
      if (nt == 0) continue;
      int wp = (w <= 1) ? 0 : 2;
      surfdisp_w(TH, VP, VS, RH, rmax, tt, vc + idx, nt, wp, mode, sphere, false, op.ro, nev, iterlim,
                 status ? status + idx : nullptr);
      if (w == 0 || w == 2) {
        for (int i = 0; i < nt; ++i) vout[idx + i] = vc[idx + i];
      } else {
        std::vector<double> cp(nt);
        std::vector<float> vpl(rmax);
        const float* VPu = VP;
        (void)vpl;  // groupvel_l's vp = 1.732 vs only matters for fluid layers (start value); the layer vp is used
        std::vector<int> sg(nt);
        surfdisp_w(TH, VPu, VS, RH, rmax, tt, cp.data(), nt, wp, mode, sphere, true, op.ro, nev, iterlim, sg.data());
        for (int i = 0; i < nt; ++i) {
          double* cgp = vout + idx + i;
          if (cp[i] == 0.0) { *cgp = 0.0; continue; }
          if (g_cpert != 0.0) cp[i] = cp[i] * (1.0 + g_cpert);
          if (w == 1)
            sregn96_(TH, VP, VS, RH, rmax, tt + i, &cp[i], cgp, b0.data(), b1.data(), b2.data(), b3.data(),
                     b4.data(), b5.data(), b6.data(), b7.data(), iflsph);
          else
            slegn96_(TH, VS, RH, rmax, tt + i, &cp[i], cgp, b0.data(), b1.data(), b2.data(), b3.data(), b4.data(),
                     iflsph);
          if (status && sg[i] != ST_OK && status[idx + i] == ST_OK) status[idx + i] = sg[i];
        }
      }
      idx += nt;
    }
  }
}

int total_kmax(const Tables& T) {
  int kmax = 0;
  for (int w = 0; w < 4; ++w)
    for (int m = 0; m < T.nmode[w]; ++m) kmax += get_nt_row(T.t[w] + (size_t)m * T.ntmax[w], T.ntmax[w]);
  return kmax;
}

}  // namespace

extern "C" {

// the conditioning probe of kernel1d (0 = off)
void swdo_set_eigen_cpert(double rel) { g_cpert = rel; }
// the group-root probe of kernel1d (0, 0 = off)
void swdo_set_group_ulp(int u1, int u2) { g_ulp[0] = u1; g_ulp[1] = u2; }

// get_1d_kernel (SurfaceWave.cpp:458-502) over ncol columns with OpenMP.
//   vs: (ncol, nz) column-major float; vp_in/rho_in optional explicit node
//   vp/rho (NULL -> Brocher); depth[nz]; period tables as in SurfTime.
//   vc, vout: (ncol, kmax); kernel: (ncol, nz, kmax); status: (ncol, kmax)
//   refine/rtol/sngl select the root refinement; sphere=1 as the reference.
// Returns kmax.
int swdo_get_1d_kernel(int ncol, int nz, const float* vs, const float* vp_in, const float* rho_in, const float* depth,
                       const double* tRc, int ntRc, int nmRc, const double* tRg, int ntRg, int nmRg,
                       const double* tLc, int ntLc, int nmLc, const double* tLg, int ntLg, int nmLg, double* vc,
                       double* vout, double* kernel, int* status, int refine, double rtol, int sngl, int sphere,
                       int nthreads, long* nevals_out) {
  Tables T{{tRc, tRg, tLc, tLg}, {ntRc, ntRg, ntLc, ntLg}, {nmRc, nmRg, nmLc, nmLg}};
  int kmax = total_kmax(T);
  Opts op{{refine, rtol, sngl}, sphere};
  long nev_total = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : nev_total)
  for (int n = 0; n < ncol; ++n) {
    std::vector<float> v(nz), vpp(nz), rh(nz), dep(nz);
    for (int k = 0; k < nz; ++k) {
      v[k] = vs[n + (size_t)ncol * k];
      dep[k] = depth[k];
      if (vp_in) { vpp[k] = vp_in[n + (size_t)ncol * k]; rh[k] = rho_in[n + (size_t)ncol * k]; }
      else empirical_relation(v[k], vpp[k], rh[k]);
    }
    std::vector<double> kvs((size_t)nz * kmax, 0.0), kvp((size_t)nz * kmax, 0.0), krho((size_t)nz * kmax, 0.0);
    std::vector<double> cp(kmax, 0.0), cg(kmax, 0.0);
    std::vector<int> st(kmax, 0);
    long nev = 0;
    int itl = 0;
    kernel1d(v.data(), vpp.data(), rh.data(), dep.data(), nz, T, cp.data(), cg.data(), kvs.data(), kvp.data(),
             krho.data(), st.data(), op, &nev, &itl);
    nev_total += nev;
    for (int ii = 0; ii < kmax; ++ii) {
      vc[n + (size_t)ncol * ii] = cp[ii];
      vout[n + (size_t)ncol * ii] = cg[ii];
      if (status) status[n + (size_t)ncol * ii] = st[ii];
      for (int jj = 0; jj < nz; ++jj) {
        size_t o = n + (size_t)ncol * (jj + (size_t)nz * ii);
        if (v[jj] == 0.0f && jj == 0) { kernel[o] = 0.0; continue; }
        if (v[jj] == 0.0f) { kernel[o] = 0.0; continue; }  // merged fluid nodes (nw>=2)
        float drda, dadb;
        empirical_deriv(vpp[jj], v[jj], drda, dadb);
        kernel[o] = kvs[jj + (size_t)nz * ii] + kvp[jj + (size_t)nz * ii] * dadb +
                    krho[jj + (size_t)nz * ii] * drda * dadb;
      }
    }
  }
  if (nevals_out) *nevals_out = nev_total;
  return kmax;
}

// get_2d_map (SurfaceWave.cpp:420-450) over ncol columns with OpenMP.
int swdo_get_2d_map(int ncol, int nz, const float* vs, const float* vp_in, const float* rho_in, const float* depth,
                    const double* tRc, int ntRc, int nmRc, const double* tRg, int ntRg, int nmRg, const double* tLc,
                    int ntLc, int nmLc, const double* tLg, int ntLg, int nmLg, double* vc, double* vout, int* status,
                    int refine, double rtol, int sngl, int sphere, int nthreads, long* nevals_out) {
  Tables T{{tRc, tRg, tLc, tLg}, {ntRc, ntRg, ntLc, ntLg}, {nmRc, nmRg, nmLc, nmLg}};
  int kmax = total_kmax(T);
  Opts op{{refine, rtol, sngl}, sphere};
  long nev_total = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : nev_total)
  for (int n = 0; n < ncol; ++n) {
    std::vector<float> v(nz), vpp(nz), rh(nz), dep(nz);
    for (int k = 0; k < nz; ++k) {
      v[k] = vs[n + (size_t)ncol * k];
      dep[k] = depth[k];
      if (vp_in) { vpp[k] = vp_in[n + (size_t)ncol * k]; rh[k] = rho_in[n + (size_t)ncol * k]; }
      else empirical_relation(v[k], vpp[k], rh[k]);
    }
    std::vector<double> cp(kmax, 0.0), cg(kmax, 0.0);
    std::vector<int> st(kmax, 0);
    long nev = 0;
    int itl = 0;
    disp1d(v.data(), vpp.data(), rh.data(), dep.data(), nz, T, cp.data(), cg.data(), st.data(), op, &nev, &itl);
    nev_total += nev;
    for (int ii = 0; ii < kmax; ++ii) {
      vc[n + (size_t)ncol * ii] = cp[ii];
      vout[n + (size_t)ncol * ii] = cg[ii];
      if (status) status[n + (size_t)ncol * ii] = st[ii];
    }
  }
  if (nevals_out) *nevals_out = nev_total;
  return kmax;
}

// surfdisp() restated (surfdisp.cpp:64-116) with wtype 0..3 = Rc,Rg,Lc,Lg
void swdo_surfdisp(const float* thk, const float* vp, const float* vs, const float* rho, int nlayer, const double* t,
                   double* cg, int kmax, int wtype, int mode, int sphere, int keep_flat, int refine, double rtol,
                   int sngl, int* status) {
  RootOpts o{refine, rtol, sngl};
  surfdisp_w(thk, vp, vs, rho, nlayer, t, cg, kmax, wtype, mode, sphere != 0, keep_flat != 0, o, nullptr, nullptr,
             status);
}

// Frechet row assembly (SurfaceWave.cpp:590-676) for nrows receivers.
//   kernel: (nx*ny, nz, kmax) column-major double; row_slot[r] = period index
//   of row r; fdm: nrows x (nx, ny) column-major float ray-path weights.
//   Writes per row nnz[r], and the compacted indices/values at row_off[r]
//   (row_off is an exclusive prefix computed by the caller, capacity n per
//   row when row_off==NULL -> r*n).  Returns the total nonzeros.
long swdo_frechet_rows(int nx, int ny, int nz, int kmax, const double* kernel, int nrows, const int* row_slot,
                       const float* fdm, int* nnz, int* indices, float* values) {
  const int n = (nx - 2) * (ny - 2) * (nz - 1);
  const size_t ncol = (size_t)nx * ny;
  long total = 0;
  std::vector<float> frechet(n);
  for (int r = 0; r < nrows; ++r) {
    const float* f = fdm + (size_t)r * ncol;
    int idx = row_slot[r];
    int c = 0;
    for (int iz = 0; iz < nz - 1; ++iz)
      for (int iy = 0; iy < ny - 2; ++iy)
        for (int ix = 0; ix < nx - 2; ++ix) {
          size_t ii = (size_t)(iy + 1) * nx + ix + 1;
          frechet[c] = (float)((double)f[(ix + 1) + (size_t)nx * (iy + 1)] *
                               kernel[ii + ncol * (iz + (size_t)nz * idx)]);
          c += 1;
        }
    int cnt = 0;
    int* oi = indices + (size_t)r * n;
    float* ov = values + (size_t)r * n;
    for (int j = 0; j < n; ++j) {
      float tmp = frechet[j];
      if (std::fabs(tmp) > 0.0) { oi[cnt] = j; ov[cnt] = tmp; cnt += 1; }
    }
    nnz[r] = cnt;
    total += cnt;
  }
  return total;
}

}  // extern "C"

extern "C" {
// kernel1D (SurfaceWave.cpp:266-412) for one column: kvs/kvp/krho are
// (nz, kmax) column-major node kernels before the empirical chain rule.
int swdo_kernel1d(const float* vs, const float* vp, const float* rho, const float* dep, int nz, const double* tRc,
                  int ntRc, int nmRc, const double* tRg, int ntRg, int nmRg, const double* tLc, int ntLc, int nmLc,
                  const double* tLg, int ntLg, int nmLg, double* vc, double* vout, double* kvs, double* kvp,
                  double* krho, int* status, int refine, double rtol, int sngl, int sphere) {
  Tables T{{tRc, tRg, tLc, tLg}, {ntRc, ntRg, ntLc, ntLg}, {nmRc, nmRg, nmLc, nmLg}};
  Opts op{{refine, rtol, sngl}, sphere};
  long nev = 0;
  int itl = 0;
  kernel1d(vs, vp, rho, dep, nz, T, vc, vout, kvs, kvp, krho, status, op, &nev, &itl);
  return total_kmax(T);
}
}
