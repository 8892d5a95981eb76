// extern "C" entry points over the reference's own C++ wrapper functions
// (src/SWD/surfdisp.cpp, src/SWD/empirical.cpp, compiled unchanged into
// oracle/_ref/), so tests can compare the oracle's restatement of those
// wrappers with the reference code itself.  Test infrastructure only.
#include <string>
void surfdisp(const float*, const float*, const float*, const float*, int, const double*, double*, int,
              const std::string&, int, bool, bool);
void groupvel_l(const float*, const float*, const float*, int, const double*, double*, int, int, bool);
void groupvel_r(const float*, const float*, const float*, const float*, int, const double*, double*, int, int, bool);
void empirical_relation(float vsz, float& vpz, float& rhoz);
void empirical_deriv(float vp, float vs, float& drda, float& dadb);

extern "C" {
void ref_surfdisp(const float* thk, const float* vp, const float* vs, const float* rho, int nlayer, const double* t,
                  double* cg, int kmax, int wtype, int mode, int sphere, int keep_flat) {
  static const char* names[4] = {"Rc", "Rg", "Lc", "Lg"};
  surfdisp(thk, vp, vs, rho, nlayer, t, cg, kmax, std::string(names[wtype]), mode, sphere != 0, keep_flat != 0);
}
void ref_groupvel_r(const float* thk, const float* vp, const float* vs, const float* rho, int nlayer, const double* t,
                    double* cg, int kmax, int mode, int sphere) {
  groupvel_r(thk, vp, vs, rho, nlayer, t, cg, kmax, mode, sphere != 0);
}
void ref_groupvel_l(const float* thk, const float* vs, const float* rho, int nlayer, const double* t, double* cg,
                    int kmax, int mode, int sphere) {
  groupvel_l(thk, vs, rho, nlayer, t, cg, kmax, mode, sphere != 0);
}
void ref_empirical_relation(const float* vs, float* vp, float* rho, int n) {
  for (int i = 0; i < n; ++i) empirical_relation(vs[i], vp[i], rho[i]);
}
void ref_empirical_deriv(const float* vp, const float* vs, float* drda, float* dadb, int n) {
  for (int i = 0; i < n; ++i) empirical_deriv(vp[i], vs[i], drda[i], dadb[i]);
}
}
