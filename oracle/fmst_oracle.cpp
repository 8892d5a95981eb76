// CPU oracle for the fast-marching traveltime path -- TEST INFRASTRUCTURE ONLY.
//
// Restates, in C++, the reference's FMST module as the inversion loops call
// it (src/SWD/SurfaceWave.cpp:510-541 travel_time, :551-676 frechet_matrix):
//   src/SWD/fmst.f90:9-82     fmst_init      (grid set-up: gdx=gdz=8, sgdl=8,
//                                             asgr=1, fom=1, snb=0.5, earth=6371)
//   src/SWD/fmst.f90:84-106   fmst_finalize
//   src/SWD/fmst.f90:108-332  fmst_travel    (exported as fmst_run: source-grid
//                                             refinement, two FMM passes, srtimes)
//   src/SWD/fmst.f90:334-348  fmst_reset     (group-velocity grid for the rays)
//   src/SWD/fmst.f90:350-976  fmst_raypath   (ray tracing, B-spline Frechet
//                                             weights, traveltime along the ray)
//   src/SWD/fmm.f90:138-332   travel         (narrow-band fast marching)
//   src/SWD/fmm.f90:345-430   fouds1, :437-610 fouds2 (first / mixed-order
//                                             upwind updates on the sphere)
//   src/SWD/fmm.f90:618-770   addtree, downtree, updtree (binary heap)
//   src/SWD/fmm.f90:776-870   gridder        (cubic B-spline dicing)
//   src/SWD/fmm.f90:877-944   bsplrefine     (refined source grid)
//   src/SWD/fmm.f90:951-1078  srtimes        (receiver traveltimes)
//   src/SWD/fmm.f90:1662-1683 bilinear
//   src/shared/spherical.cpp:9-27 delsph     (as oracle_delsph)
// All arithmetic is REAL*4 in the order the Fortran states it (x**2 = x*x,
// x**3 = (x*x)*x, no contraction: built with -ffp-contract=off); sin is the
// C library's sinf, as gfortran calls it for REAL*4.
//
// Deviations, all on inputs where the reference has no defined behaviour:
//   * a source or receiver outside the grid (the reference prints and STOPs)
//     makes fmst_run / fmst_raypath return with ttime = NaN;
//   * a narrow band larger than the reference's heap (snb*nnx*nnz entries,
//     which the reference overruns silently) aborts the pair with NaN;
//   * a ray that does not reach the source within nnx*nnz steps (the
//     reference then reads an undefined point count) gives tsyn = NaN.
// The per-thread state mirrors the reference's OpenMP threadprivate module
// variables, so pairs can run on OpenMP threads as travel_time does.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr float PI_SP = 3.1415926535898f;  // fmm.f90:24, REAL(sp) parameter

struct A2f {  // REAL(sp) array (1:d1, 1:d2), column-major
    std::vector<float> a;
    int ld = 0, d2 = 0;
    void alloc(int n1, int n2) { a.assign((size_t)n1 * n2, 0.0f); ld = n1; d2 = n2; }
    float& operator()(int i, int j) { return a[(size_t)(i - 1) + (size_t)(j - 1) * ld]; }
};
struct A2i {
    std::vector<int> a;
    int ld = 0, d2 = 0;
    void alloc(int n1, int n2) { a.assign((size_t)n1 * n2, 0); ld = n1; d2 = n2; }
    int& operator()(int i, int j) { return a[(size_t)(i - 1) + (size_t)(j - 1) * ld]; }
    void fill(int v) { std::fill(a.begin(), a.end(), v); }
};

inline float sq(float x) { return x * x; }
inline float cube(float x) { return (x * x) * x; }

struct Fmst {
    int nvx = 0, nvz = 0, nnx = 0, nnz = 0, fom = 1, gdx = 8, gdz = 8;
    int vnl = 0, vnr = 0, vnt = 0, vnb = 0, nrnx = 0, nrnz = 0, sgdl = 8, rbint = 0;
    int nnxr = 0, nnzr = 0, asgr = 1;
    A2i nsts, nstsr;
    float gox = 0, goz = 0, dnx = 0, dnz = 0, dvx = 0, dvz = 0, snb = 0.5f, earth = 6371.0f;
    float goxd = 0, gozd = 0, dvxd = 0, dvzd = 0, dnxd = 0, dnzd = 0;
    float drnx = 0, drnz = 0, gorx = 0, gorz = 0, dnxr = 0, dnzr = 0, goxr = 0, gozr = 0;
    std::vector<float> velv;  // (0:nvz+1, 0:nvx+1)
    A2f veln, velnb, ttn, ttnr, velnew;
    int ntr = 0;
    std::vector<int> bpx, bpz;  // btg(1:maxbt)%px, %pz
    bool failed = false;

    float& vv(int i, int j) { return velv[(size_t)i + (size_t)j * (nvz + 2)]; }

    // fmst.f90:9-82
    void init(int nx, int ny, float goxdf, float gozdf, float dvxdf, float dvzdf) {
        gdx = 8; gdz = 8; asgr = 1; sgdl = 8; earth = 6371.0f; fom = 1; snb = 0.5f;
        nvx = nx - 2; nvz = ny - 2;
        goxd = goxdf - dvxdf; gozd = gozdf + dvzdf;
        dvxd = dvxdf; dvzd = dvzdf;
        velv.assign((size_t)(nvz + 2) * (nvx + 2), 0.0f);
        dvx = dvxd * PI_SP / 180.0f;
        dvz = dvzd * PI_SP / 180.0f;
        gox = (90.0f - goxd) * PI_SP / 180.0f;
        goz = gozd * PI_SP / 180.0f;
        nnx = (nvx - 1) * gdx + 1;
        nnz = (nvz - 1) * gdz + 1;
        dnx = dvx / (float)gdx;
        dnz = dvz / (float)gdz;
        dnxd = dvxd / (float)gdx;
        dnzd = dvzd / (float)gdz;
        veln.alloc(nnz, nnx);
        ttn.alloc(nnz, nnx);
        rbint = 0;
        nsts.alloc(nnz, nnx);
        int maxbt = (int)std::lround(snb * (float)(nnx * nnz));
        bpx.assign(maxbt + 1, 0);
        bpz.assign(maxbt + 1, 0);
        velnb.alloc(nnz, nnx);
        failed = false;
    }

    // fmm.f90:776-870
    void gridder(const double* pv) {
        for (int i = 0; i <= nvz + 1; ++i)
            for (int j = 0; j <= nvx + 1; ++j) vv(i, j) = (float)pv[(size_t)i * (nvx + 2) + j];
        std::vector<float> ui((size_t)(gdx + 1) * 4), vi((size_t)(gdz + 1) * 4);
        auto U = [&](int i, int k) -> float& { return ui[(size_t)(i - 1) + (size_t)(k - 1) * (gdx + 1)]; };
        auto V = [&](int i, int k) -> float& { return vi[(size_t)(i - 1) + (size_t)(k - 1) * (gdz + 1)]; };
        for (int i = 1; i <= gdx + 1; ++i) {
            float u = (float)gdx;
            u = (float)(i - 1) / u;
            U(i, 1) = cube(1.0f - u) / 6.0f;
            U(i, 2) = (4.0f - 6.0f * sq(u) + 3.0f * cube(u)) / 6.0f;
            U(i, 3) = (1.0f + 3.0f * u + 3.0f * sq(u) - 3.0f * cube(u)) / 6.0f;
            U(i, 4) = cube(u) / 6.0f;
        }
        for (int i = 1; i <= gdz + 1; ++i) {
            float u = (float)gdz;
            u = (float)(i - 1) / u;
            V(i, 1) = cube(1.0f - u) / 6.0f;
            V(i, 2) = (4.0f - 6.0f * sq(u) + 3.0f * cube(u)) / 6.0f;
            V(i, 3) = (1.0f + 3.0f * u + 3.0f * sq(u) - 3.0f * cube(u)) / 6.0f;
            V(i, 4) = cube(u) / 6.0f;
        }
        for (int i = 1; i <= nvz - 1; ++i) {
            int conz = (i == nvz - 1) ? gdz + 1 : gdz;
            for (int j = 1; j <= nvx - 1; ++j) {
                int conx = (j == nvx - 1) ? gdx + 1 : gdx;
                for (int l = 1; l <= conz; ++l) {
                    int stz = gdz * (i - 1) + l;
                    for (int m = 1; m <= conx; ++m) {
                        int stx = gdx * (j - 1) + m;
                        float sumi = 0.0f;
                        for (int i1 = 1; i1 <= 4; ++i1) {
                            float sumj = 0.0f;
                            for (int j1 = 1; j1 <= 4; ++j1) sumj = sumj + U(m, j1) * vv(i - 2 + i1, j - 2 + j1);
                            sumi = sumi + V(l, i1) * sumj;
                        }
                        veln(stz, stx) = sumi;
                    }
                }
            }
        }
    }

    // fmm.f90:877-944
    void bsplrefine() {
        int nrxr = gdx * sgdl, nrzr = gdz * sgdl;
        std::vector<float> ui((size_t)(nrxr + 1) * 4), vi((size_t)(nrzr + 1) * 4);
        for (int j = 1; j <= nrxr + 1; ++j) {  // ui(j,i,:) depends on j only
            float u = (float)nrxr;
            u = (float)(j - 1) / u;
            float* p = &ui[(size_t)(j - 1) * 4];
            p[0] = cube(1.0f - u) / 6.0f;
            p[1] = (4.0f - 6.0f * sq(u) + 3.0f * cube(u)) / 6.0f;
            p[2] = (1.0f + 3.0f * u + 3.0f * sq(u) - 3.0f * cube(u)) / 6.0f;
            p[3] = cube(u) / 6.0f;
        }
        for (int i = 1; i <= nrzr + 1; ++i) {  // vi(j,i,:) depends on i only
            float v = (float)nrzr;
            v = (float)(i - 1) / v;
            float* p = &vi[(size_t)(i - 1) * 4];
            p[0] = cube(1.0f - v) / 6.0f;
            p[1] = (4.0f - 6.0f * sq(v) + 3.0f * cube(v)) / 6.0f;
            p[2] = (1.0f + 3.0f * v + 3.0f * sq(v) - 3.0f * cube(v)) / 6.0f;
            p[3] = cube(v) / 6.0f;
        }
        int origx = (vnl - 1) * sgdl + 1, origz = (vnt - 1) * sgdl + 1;
        for (int i = 1; i <= nvz - 1; ++i) {
            int conz = (i == nvz - 1) ? nrzr + 1 : nrzr;
            for (int j = 1; j <= nvx - 1; ++j) {
                int conx = (j == nvx - 1) ? nrxr + 1 : nrxr;
                for (int k = 1; k <= conz; ++k) {
                    int st1 = gdz * (i - 1) + (k - 1) / sgdl + 1;
                    if (st1 < vnt || st1 > vnb) continue;
                    st1 = nrzr * (i - 1) + k;
                    for (int l = 1; l <= conx; ++l) {
                        int st2 = gdx * (j - 1) + (l - 1) / sgdl + 1;
                        if (st2 < vnl || st2 > vnr) continue;
                        st2 = nrxr * (j - 1) + l;
                        float sum[4];
                        for (int i1 = 1; i1 <= 4; ++i1) {
                            sum[i1 - 1] = 0.0f;
                            for (int j1 = 1; j1 <= 4; ++j1)
                                sum[i1 - 1] = sum[i1 - 1] + ui[(size_t)(l - 1) * 4 + j1 - 1] * vv(i - 2 + i1, j - 2 + j1);
                            sum[i1 - 1] = vi[(size_t)(k - 1) * 4 + i1 - 1] * sum[i1 - 1];
                        }
                        int idm1 = st1 - origz + 1, idm2 = st2 - origx + 1;
                        if (idm1 < 1 || idm1 > nnz) continue;
                        if (idm2 < 1 || idm2 > nnx) continue;
                        veln(idm1, idm2) = sum[0] + sum[1] + sum[2] + sum[3];
                    }
                }
            }
        }
    }

    // fmm.f90:1662-1683
    float bilinear(const float nv[2][2], float dsx, float dsz) const {
        float biv = 0.0f;
        for (int i = 1; i <= 2; ++i)
            for (int j = 1; j <= 2; ++j) {
                float produ = (1.0f - std::fabs(((float)(i - 1) * dnx - dsx) / dnx)) *
                              (1.0f - std::fabs(((float)(j - 1) * dnz - dsz) / dnz));
                biv = biv + nv[i - 1][j - 1] * produ;
            }
        return biv;
    }

    // fmm.f90:618-647
    void addtree(int iz, int ix) {
        ntr = ntr + 1;
        if (ntr >= (int)bpx.size()) { failed = true; ntr = (int)bpx.size() - 1; return; }
        nsts(iz, ix) = ntr;
        bpx[ntr] = ix;
        bpz[ntr] = iz;
        int tpc = ntr, tpp = tpc / 2;
        while (tpp > 0) {
            if (ttn(iz, ix) < ttn(bpz[tpp], bpx[tpp])) {
                nsts(iz, ix) = tpp;
                nsts(bpz[tpp], bpx[tpp]) = tpc;
                std::swap(bpx[tpc], bpx[tpp]);
                std::swap(bpz[tpc], bpz[tpp]);
                tpc = tpp;
                tpp = tpc / 2;
            } else {
                tpp = 0;
            }
        }
    }

    // fmm.f90:657-736
    void downtree() {
        if (ntr == 1) { ntr = ntr - 1; return; }
        nsts(bpz[ntr], bpx[ntr]) = 1;
        bpx[1] = bpx[ntr];
        bpz[1] = bpz[ntr];
        ntr = ntr - 1;
        int tpp = 1, tpc = 2 * tpp;
        while (tpc < ntr) {
            float rd1 = ttn(bpz[tpc], bpx[tpc]);
            float rd2 = ttn(bpz[tpc + 1], bpx[tpc + 1]);
            if (rd1 > rd2) tpc = tpc + 1;
            rd1 = ttn(bpz[tpc], bpx[tpc]);
            rd2 = ttn(bpz[tpp], bpx[tpp]);
            if (rd1 < rd2) {
                nsts(bpz[tpp], bpx[tpp]) = tpc;
                nsts(bpz[tpc], bpx[tpc]) = tpp;
                std::swap(bpx[tpc], bpx[tpp]);
                std::swap(bpz[tpc], bpz[tpp]);
                tpp = tpc;
                tpc = 2 * tpp;
            } else {
                tpc = ntr + 1;
            }
        }
        if (tpc == ntr) {
            float rd1 = ttn(bpz[tpc], bpx[tpc]);
            float rd2 = ttn(bpz[tpp], bpx[tpp]);
            if (rd1 < rd2) {
                nsts(bpz[tpp], bpx[tpp]) = tpc;
                nsts(bpz[tpc], bpx[tpc]) = tpp;
                std::swap(bpx[tpc], bpx[tpp]);
                std::swap(bpz[tpc], bpz[tpp]);
            }
        }
    }

    // fmm.f90:744-770
    void updtree(int iz, int ix) {
        int tpc = nsts(iz, ix), tpp = tpc / 2;
        while (tpp > 0) {
            if (ttn(iz, ix) < ttn(bpz[tpp], bpx[tpp])) {
                nsts(iz, ix) = tpp;
                nsts(bpz[tpp], bpx[tpp]) = tpc;
                std::swap(bpx[tpc], bpx[tpp]);
                std::swap(bpz[tpc], bpz[tpp]);
                tpc = tpp;
                tpp = tpc / 2;
            } else {
                tpp = 0;
            }
        }
    }

    // fmm.f90:345-430 (fom = 0; fmst_init always selects fom = 1)
    void fouds1(int iz, int ix) {
        int tsw1 = 0;
        float travm = 0.0f;
        float slown = 1.0f / veln(iz, ix);
        float ri = earth;
        float risti = ri * std::sin(gox + (float)(ix - 1) * dnx);
        for (int j = ix - 1; j <= ix + 1; j += 2)
            for (int k = iz - 1; k <= iz + 1; k += 2) {
                if (j < 1 || j > nnx || k < 1 || k > nnz) continue;
                int swsol = 0;
                float a = 0, b = 0, c = 0, tref = 0;
                if (nsts(iz, j) == 0) {
                    swsol = 1;
                    if (nsts(k, ix) == 0) {
                        float u = ri * dnx, v = risti * dnz;
                        float em = ttn(k, ix) - ttn(iz, j);
                        a = sq(u) + sq(v);
                        b = -2.0f * sq(u) * em;
                        c = sq(u) * (sq(em) - sq(v) * sq(slown));
                        tref = ttn(iz, j);
                    } else {
                        a = 1.0f; b = 0.0f;
                        c = -sq(slown) * sq(ri) * sq(dnx);
                        tref = ttn(iz, j);
                    }
                } else if (nsts(k, ix) == 0) {
                    swsol = 1;
                    a = 1.0f; b = 0.0f;
                    c = -sq(slown * risti * dnz);
                    tref = ttn(k, ix);
                }
                if (swsol == 1) {
                    float rd1 = sq(b) - 4.0f * a * c;
                    if (rd1 < 0.0f) rd1 = 0.0f;
                    float tdsh = (-b + std::sqrt(rd1)) / (2.0f * a);
                    float trav = tref + tdsh;
                    if (tsw1 == 1) travm = std::fmin(trav, travm);
                    else { travm = trav; tsw1 = 1; }
                }
            }
        ttn(iz, ix) = travm;
    }

    // fmm.f90:437-610
    void fouds2(int iz, int ix) {
        int tsw1 = 0;
        float travm = 0.0f;
        float slown = 1.0f / veln(iz, ix);
        float ri = earth;
        float risti = ri * std::sin(gox + (float)(ix - 1) * dnx);
        for (int j = ix - 1; j <= ix + 1; j += 2) {
            if (j < 1 || j > nnx) continue;
            int swj = -1, j2;
            if (j == ix - 1) {
                j2 = j - 1;
                if (j2 >= 1 && nsts(iz, j2) == 0) swj = 0;
            } else {
                j2 = j + 1;
                if (j2 <= nnx && nsts(iz, j2) == 0) swj = 0;
            }
            if (nsts(iz, j) == 0 && swj == 0) {
                swj = -1;
                if (ttn(iz, j) > ttn(iz, j2)) swj = 0;
            } else {
                swj = -1;
            }
            for (int k = iz - 1; k <= iz + 1; k += 2) {
                if (k < 1 || k > nnz) continue;
                int swk = -1, k2;
                if (k == iz - 1) {
                    k2 = k - 1;
                    if (k2 >= 1 && nsts(k2, ix) == 0) swk = 0;
                } else {
                    k2 = k + 1;
                    if (k2 <= nnz && nsts(k2, ix) == 0) swk = 0;
                }
                if (nsts(k, ix) == 0 && swk == 0) {
                    swk = -1;
                    if (ttn(k, ix) > ttn(k2, ix)) swk = 0;
                } else {
                    swk = -1;
                }
                int swsol = 0;
                float a = 0, b = 0, c = 0, tref = 0, tdiv = 1.0f;
                if (swj == 0) {
                    swsol = 1;
                    if (swk == 0) {
                        float u = 2.0f * ri * dnx, v = 2.0f * risti * dnz;
                        float em = 4.0f * ttn(iz, j) - ttn(iz, j2) - 4.0f * ttn(k, ix);
                        em = em + ttn(k2, ix);
                        a = sq(v) + sq(u);
                        b = 2.0f * em * sq(u);
                        c = sq(u) * (sq(em) - sq(slown) * sq(v));
                        tref = 4.0f * ttn(iz, j) - ttn(iz, j2);
                        tdiv = 3.0f;
                    } else if (nsts(k, ix) == 0) {
                        float u = risti * dnz, v = 2.0f * ri * dnx;
                        float em = 3.0f * ttn(k, ix) - 4.0f * ttn(iz, j) + ttn(iz, j2);
                        a = sq(v) + 9.0f * sq(u);
                        b = 6.0f * em * sq(u);
                        c = sq(u) * (sq(em) - sq(slown) * sq(v));
                        tref = ttn(k, ix);
                        tdiv = 1.0f;
                    } else {
                        float u = 2.0f * ri * dnx;
                        a = 1.0f; b = 0.0f;
                        c = -sq(u) * sq(slown);
                        tref = 4.0f * ttn(iz, j) - ttn(iz, j2);
                        tdiv = 3.0f;
                    }
                } else if (nsts(iz, j) == 0) {
                    swsol = 1;
                    if (swk == 0) {
                        float u = ri * dnx, v = 2.0f * risti * dnz;
                        float em = 3.0f * ttn(iz, j) - 4.0f * ttn(k, ix) + ttn(k2, ix);
                        a = sq(v) + 9.0f * sq(u);
                        b = 6.0f * em * sq(u);
                        c = sq(u) * (sq(em) - sq(v) * sq(slown));
                        tref = ttn(iz, j);
                        tdiv = 1.0f;
                    } else if (nsts(k, ix) == 0) {
                        float u = ri * dnx, v = risti * dnz;
                        float em = ttn(k, ix) - ttn(iz, j);
                        a = sq(u) + sq(v);
                        b = -2.0f * sq(u) * em;
                        c = sq(u) * (sq(em) - sq(v) * sq(slown));
                        tref = ttn(iz, j);
                        tdiv = 1.0f;
                    } else {
                        a = 1.0f; b = 0.0f;
                        c = -sq(slown) * sq(ri) * sq(dnx);
                        tref = ttn(iz, j);
                        tdiv = 1.0f;
                    }
                } else {
                    if (swk == 0) {
                        swsol = 1;
                        float u = 2.0f * risti * dnz;
                        a = 1.0f; b = 0.0f;
                        c = -sq(u) * sq(slown);
                        tref = 4.0f * ttn(k, ix) - ttn(k2, ix);
                        tdiv = 3.0f;
                    } else if (nsts(k, ix) == 0) {
                        swsol = 1;
                        a = 1.0f; b = 0.0f;
                        c = -sq(slown) * sq(risti) * sq(dnz);
                        tref = ttn(k, ix);
                        tdiv = 1.0f;
                    }
                }
                if (swsol == 1) {
                    float rd1 = sq(b) - 4.0f * a * c;
                    if (rd1 < 0.0f) rd1 = 0.0f;
                    float tdsh = (-b + std::sqrt(rd1)) / (2.0f * a);
                    float trav = (tref + tdsh) / tdiv;
                    if (tsw1 == 1) travm = std::fmin(trav, travm);
                    else { travm = trav; tsw1 = 1; }
                }
            }
        }
        ttn(iz, ix) = travm;
    }

    void update(int iz, int ix) { if (fom == 0) fouds1(iz, ix); else fouds2(iz, ix); }

    // fmm.f90:138-332
    void travel(float scx, float scz, int urg) {
        int isx = (int)((scx - gox) / dnx) + 1;
        int isz = (int)((scz - goz) / dnz) + 1;
        if (isx < 1 || isx > nnx || isz < 1 || isz > nnz) { failed = true; return; }
        if (isx == nnx) isx = isx - 1;
        if (isz == nnz) isz = isz - 1;
        if (urg != 2) nsts.fill(-1);
        ntr = 0;
        if (urg == 2) {
            for (int i = 1; i <= nnx; ++i)
                for (int j = 1; j <= nnz; ++j)
                    if (nsts(j, i) > 0) addtree(j, i);
        } else {
            float vss[2][2];
            for (int i = 1; i <= 2; ++i)
                for (int j = 1; j <= 2; ++j) vss[i - 1][j - 1] = veln(isz - 1 + j, isx - 1 + i);
            float dsx = (scx - gox) - (float)(isx - 1) * dnx;
            float dsz = (scz - goz) - (float)(isz - 1) * dnz;
            float vsrc = bilinear(vss, dsx, dsz);
            for (int i = 1; i <= 2; ++i)
                for (int j = 1; j <= 2; ++j) {
                    float ds = std::sqrt(sq(dsx - (float)(i - 1) * dnx) + sq(dsz - (float)(j - 1) * dnz));
                    ttn(isz - 1 + j, isx - 1 + i) = 2.0f * ds / (vss[i - 1][j - 1] + vsrc);
                    addtree(isz - 1 + j, isx - 1 + i);
                }
        }
        while (ntr > 0 && !failed) {
            if (urg == 1) {
                int ix = bpx[1], iz = bpz[1], swrg = 0;
                if (ix == 1 && vnl != 1) swrg = 1;
                if (ix == nnx && vnr != nnx) swrg = 1;
                if (iz == 1 && vnt != 1) swrg = 1;
                if (iz == nnz && vnb != nnz) swrg = 1;
                if (swrg == 1) { nsts(iz, ix) = 0; break; }
            }
            int ix = bpx[1], iz = bpz[1];
            nsts(iz, ix) = 0;
            downtree();
            for (int i = ix - 1; i <= ix + 1; i += 2) {
                if (i < 1 || i > nnx) continue;
                if (nsts(iz, i) == -1) { update(iz, i); addtree(iz, i); }
                else if (nsts(iz, i) > 0) { update(iz, i); updtree(iz, i); }
            }
            for (int i = iz - 1; i <= iz + 1; i += 2) {
                if (i < 1 || i > nnz) continue;
                if (nsts(i, ix) == -1) { update(i, ix); addtree(i, ix); }
                else if (nsts(i, ix) > 0) { update(i, ix); updtree(i, ix); }
            }
        }
    }

    // fmm.f90:951-1078
    float srtimes(float scx, float scz, float rcx1, float rcz1) {
        int irx = (int)((rcx1 - gox) / dnx) + 1;
        int irz = (int)((rcz1 - goz) / dnz) + 1;
        int sw = 0;
        if (irx < 1 || irx > nnx || irz < 1 || irz > nnz) return NAN;
        if (irx == nnx) irx = irx - 1;
        if (irz == nnz) irz = irz - 1;
        int isx = (int)((scx - gox) / dnx) + 1;
        int isz = (int)((scz - goz) / dnz) + 1;
        float dpl = dnx * earth;
        float rd1 = dnz * earth * std::sin(gox);
        if (rd1 < dpl) dpl = rd1;
        rd1 = dnz * earth * std::sin(gox + (float)(nnx - 1) * dnx);
        if (rd1 < dpl) dpl = rd1;
        float sred = sq((scx - rcx1) * earth);
        sred = sred + sq((scz - rcz1) * earth * std::sin(rcx1));
        sred = std::sqrt(sred);
        if (sred < dpl) sw = 1;
        if (isx == irx && isz == irz) sw = 1;
        float trr;
        if (sw == 1) {
            float vss[2][2];
            for (int k = 1; k <= 2; ++k)
                for (int l = 1; l <= 2; ++l) vss[k - 1][l - 1] = veln(isz - 1 + l, isx - 1 + k);
            float drx = (scx - gox) - (float)(isx - 1) * dnx;
            float drz = (scz - goz) - (float)(isz - 1) * dnz;
            float vels = bilinear(vss, drx, drz);
            for (int k = 1; k <= 2; ++k)
                for (int l = 1; l <= 2; ++l) vss[k - 1][l - 1] = veln(irz - 1 + l, irx - 1 + k);
            drx = (rcx1 - gox) - (float)(irx - 1) * dnx;
            drz = (rcz1 - goz) - (float)(irz - 1) * dnz;
            float velr = bilinear(vss, drx, drz);
            trr = 2.0f * sred / (vels + velr);
        } else {
            float drx = (rcx1 - gox) - (float)(irx - 1) * dnx;
            float drz = (rcz1 - goz) - (float)(irz - 1) * dnz;
            trr = 0.0f;
            for (int k = 1; k <= 2; ++k)
                for (int l = 1; l <= 2; ++l) {
                    float produ = (1.0f - std::fabs(((float)(l - 1) * dnz - drz) / dnz)) *
                                  (1.0f - std::fabs(((float)(k - 1) * dnx - drx) / dnx));
                    trr = trr + ttn(irz - 1 + l, irx - 1 + k) * produ;
                }
        }
        return trr;
    }

    // fmst.f90:108-332
    void run(const double* velf, float srcx, float srcz, const float* rcx, const float* rcz, int nr, float* ttime) {
        const int sgs = 8;
        failed = false;
        gridder(velf);
        float x = srcx, z = srcz;
        int nnxb, nnzb;
        float dnxb, dnzb, goxb, gozb;
        // asgr == 1 always (fmst_init)
        for (int j = 1; j <= nnx; ++j)
            for (int k = 1; k <= nnz; ++k) velnb(k, j) = veln(k, j);
        nnxb = nnx; nnzb = nnz; dnxb = dnx; dnzb = dnz; goxb = gox; gozb = goz;
        int isx = (int)((x - gox) / dnx) + 1;
        int isz = (int)((z - goz) / dnz) + 1;
        if (isx < 1 || isx > nnx || isz < 1 || isz > nnz) {
            for (int i = 0; i < nr; ++i) ttime[i] = NAN;
            failed = true;
            return;
        }
        if (isx == nnx) isx = isx - 1;
        if (isz == nnz) isz = isz - 1;
        vnl = isx - sgs; if (vnl < 1) vnl = 1;
        vnr = isx + sgs; if (vnr > nnx) vnr = nnx;
        vnt = isz - sgs; if (vnt < 1) vnt = 1;
        vnb = isz + sgs; if (vnb > nnz) vnb = nnz;
        nrnx = (vnr - vnl) * sgdl + 1;
        nrnz = (vnb - vnt) * sgdl + 1;
        drnx = dvx / (float)(gdx * sgdl);
        drnz = dvz / (float)(gdz * sgdl);
        gorx = gox + dnx * (float)(vnl - 1);
        gorz = goz + dnz * (float)(vnt - 1);
        nnx = nrnx; nnz = nrnz; dnx = drnx; dnz = drnz; gox = gorx; goz = gorz;
        if (nnx > nnxb || nnz > nnzb) {
            int idm1 = std::max(nnx, nnxb), idm2 = std::max(nnz, nnzb);
            veln.alloc(idm2, idm1);
            ttn.alloc(idm2, idm1);
            nsts.alloc(idm2, idm1);
            int maxbt = (int)std::lround(snb * (float)(idm1 * idm2));
            bpx.assign(maxbt + 1, 0);
            bpz.assign(maxbt + 1, 0);
        }
        bsplrefine();
        travel(x, z, 1);
        // ttnr = ttn, nstsr = nsts (whole arrays, reference realloc-on-assignment)
        ttnr = ttn;
        nstsr = nsts;
        int ogx = vnl, ogz = vnt, grdfx = sgdl, grdfz = sgdl;
        nsts.fill(-1);
        for (int k = 1; k <= nnz; k += grdfz) {
            int idm1 = ogz + (k - 1) / grdfz;
            for (int l = 1; l <= nnx; l += grdfx) {
                int idm2 = ogx + (l - 1) / grdfx;
                nsts(idm1, idm2) = nstsr(k, l);
                if (nsts(idm1, idm2) >= 0) ttn(idm1, idm2) = ttnr(k, l);
            }
        }
        nnxr = nnx; nnzr = nnz; goxr = gox; gozr = goz; dnxr = dnx; dnzr = dnz;
        nnx = nnxb; nnz = nnzb; dnx = dnxb; dnz = dnzb; gox = goxb; goz = gozb;
        for (int j = 1; j <= nnx; ++j)
            for (int k = 1; k <= nnz; ++k) veln(k, j) = velnb(k, j);
        for (int k = 1; k <= nnx; ++k)
            for (int l = 1; l <= nnz; ++l)
                if (nsts(l, k) == 0) {
                    if (l - 1 >= 1 && nsts(l - 1, k) == -1) nsts(l, k) = 1;
                    if (l + 1 <= nnz && nsts(l + 1, k) == -1) nsts(l, k) = 1;
                    if (k - 1 >= 1 && nsts(l, k - 1) == -1) nsts(l, k) = 1;
                    if (k + 1 <= nnx && nsts(l, k + 1) == -1) nsts(l, k) = 1;
                }
        travel(x, z, 2);
        for (int i = 0; i < nr; ++i) ttime[i] = failed ? NAN : srtimes(x, z, rcx[i], rcz[i]);
    }

    // fmst.f90:334-348
    void reset(const double* velin) {
        A2f temp = veln;
        gridder(velin);
        velnew.alloc(nnz, nnx);
        for (int j = 1; j <= nnx; ++j)
            for (int k = 1; k <= nnz; ++k) velnew(k, j) = veln(k, j);
        veln = temp;
    }

    float vel_at(float px, float pz, int ipx, int ipz) {
        // bilinear velnew at (px, pz) from cell (ipx, ipz) (fmst.f90:794-805 and its repeats)
        float drx = (px - gox) - (float)(ipx - 1) * dnx;
        float drz = (pz - goz) - (float)(ipz - 1) * dnz;
        float vel = 0.0f;
        for (int l = 1; l <= 2; ++l)
            for (int m = 1; m <= 2; ++m) {
                float produ = (1.0f - std::fabs(((float)(m - 1) * dnz - drz) / dnz));
                produ = produ * (1.0f - std::fabs(((float)(l - 1) * dnx - drx) / dnx));
                if (ipz - 1 + m <= nnz && ipx - 1 + l <= nnx) vel = vel + velnew(ipz - 1 + m, ipx - 1 + l) * produ;
            }
        return vel;
    }

    static void basis(float v, float* vi) {
        vi[0] = cube(1.0f - v) / 6.0f;
        vi[1] = (4.0f - 6.0f * sq(v) + 3.0f * cube(v)) / 6.0f;
        vi[2] = (1.0f + 3.0f * v + 3.0f * sq(v) - 3.0f * cube(v)) / 6.0f;
        vi[3] = cube(v) / 6.0f;
    }

    // fmst.f90:350-976
    float raypath(float scx, float scz, float surfrcx, float surfrcz, float* fdm);
};

thread_local Fmst S;

}  // namespace

extern "C" float oracle_delsph(float colatrad1, float lonrad1, float colatrad2, float lonrad2) {
    // src/shared/spherical.cpp:9-27: double expressions stored into floats
    float R = 6371.0f;
    float dlat = colatrad2 - colatrad1;
    float dlon = lonrad2 - lonrad1;
    float lat1 = (float)(M_PI * 0.5 - colatrad1);
    float lat2 = (float)(M_PI * 0.5 - colatrad2);
    float a = (float)(std::sin(dlat * 0.5) * std::sin(dlat * 0.5) +
                      std::sin(dlon * 0.5) * std::sin(dlon * 0.5) * std::cos((double)lat1) * std::cos((double)lat2));
    float c = (float)(2.0 * std::atan2(std::sqrt((double)a), std::sqrt((double)(1 - a))));
    return R * c;
}

float Fmst::raypath(float scx, float scz, float surfrcx, float surfrcz, float* fdm) {
    const int maxrp = nnx * nnz;
    std::vector<float> rgx(maxrp + 3), rgz(maxrp + 3);  // 1-based rgx(1:maxrp+2)
    std::vector<float> fdm0((size_t)(nvz + 2) * (nvx + 2), 0.0f);  // fdm0(0:nvz+1, 0:nvx+1)
    auto F0 = [&](int i, int j) -> float& { return fdm0[(size_t)i + (size_t)j * (nvz + 2)]; };
    int isx, isz;
    if (asgr == 1) {
        isx = (int)((scx - goxr) / dnxr) + 1;
        isz = (int)((scz - gozr) / dnzr) + 1;
    } else {
        isx = (int)((scx - gox) / dnx) + 1;
        isz = (int)((scz - goz) / dnz) + 1;
    }
    float dpl = dnx * earth;
    float rd1 = dnz * earth * std::sin(gox);
    if (rd1 < dpl) dpl = rd1;
    rd1 = dnz * earth * std::sin(gox + (float)(nnx - 1) * dnx);
    if (rd1 < dpl) dpl = rd1;
    dpl = 0.5f * dpl;
    int ipx = (int)((surfrcx - gox) / dnx) + 1;
    int ipz = (int)((surfrcz - goz) / dnz) + 1;
    int sw = 0, nrp = -1;
    if (ipx < 1 || ipx >= nnx || ipz < 1 || ipz >= nnz) {
        for (int j = 0; j <= nvz + 1; ++j)
            for (int k = 0; k <= nvx + 1; ++k) fdm[(size_t)k + (size_t)j * (nvx + 2)] = 0.0f;
        return NAN;
    }
    rgx[1] = surfrcx;
    rgz[1] = surfrcz;
    float sred = sq((scx - rgx[1]) * earth);
    sred = sred + sq((scz - rgz[1]) * earth * std::sin(rgx[1]));
    sred = std::sqrt(sred);
    if (sred < 2.0f * dpl) { rgx[2] = scx; rgz[2] = scz; nrp = 2; sw = 1; }
    int ipxr = 0, ipzr = 0, igref;
    if (asgr == 1) {
        ipxr = (int)((surfrcx - goxr) / dnxr) + 1;
        ipzr = (int)((surfrcz - gozr) / dnzr) + 1;
        igref = 1;
        if (ipxr < 1 || ipxr >= nnxr) igref = 0;
        if (ipzr < 1 || ipzr >= nnzr) igref = 0;
        if (igref == 1) {
            if (nstsr(ipzr, ipxr) != 0 || nstsr(ipzr + 1, ipxr) != 0) igref = 0;
            if (nstsr(ipzr, ipxr + 1) != 0 || nstsr(ipzr + 1, ipxr + 1) != 0) igref = 0;
        }
    } else {
        igref = 0;
    }
    if (sw == 0) {
        if (asgr == 1) {
            if (igref == 1 && ipxr == isx && ipzr == isz) { rgx[2] = scx; rgz[2] = scz; nrp = 2; sw = 1; }
        } else if (ipx == isx && ipz == isz) {
            rgx[2] = scx; rgz[2] = scz; nrp = 2; sw = 1;
        }
    }
    for (int j = 1; j <= maxrp; ++j) {
        if (sw == 1) break;
        float dtx, dtz;
        if (igref == 1) {
            dtx = ttnr(ipzr, ipxr + 1) - ttnr(ipzr, ipxr);
            dtx = dtx + ttnr(ipzr + 1, ipxr + 1) - ttnr(ipzr + 1, ipxr);
            dtx = dtx / (2.0f * earth * dnxr);
            dtz = ttnr(ipzr + 1, ipxr) - ttnr(ipzr, ipxr);
            dtz = dtz + ttnr(ipzr + 1, ipxr + 1) - ttnr(ipzr, ipxr + 1);
            dtz = dtz / (2.0f * earth * std::sin(rgx[j]) * dnzr);
        } else {
            dtx = ttn(ipz, ipx + 1) - ttn(ipz, ipx);
            dtx = dtx + ttn(ipz + 1, ipx + 1) - ttn(ipz + 1, ipx);
            dtx = dtx / (2.0f * earth * dnx);
            dtz = ttn(ipz + 1, ipx) - ttn(ipz, ipx);
            dtz = dtz + ttn(ipz + 1, ipx + 1) - ttn(ipz, ipx + 1);
            dtz = dtz / (2.0f * earth * std::sin(rgx[j]) * dnz);
        }
        rd1 = std::sqrt(sq(dtx) + sq(dtz));
        rgx[j + 1] = rgx[j] - dpl * dtx / (earth * rd1);
        rgz[j + 1] = rgz[j] - dpl * dtz / (earth * std::sin(rgx[j]) * rd1);
        int ipxo = ipx, ipzo = ipz;
        if (asgr == 1) {
            ipxr = (int)((rgx[j + 1] - goxr) / dnxr) + 1;
            ipzr = (int)((rgz[j + 1] - gozr) / dnzr) + 1;
            igref = 1;
            if (ipxr < 1 || ipxr >= nnxr) igref = 0;
            if (ipzr < 1 || ipzr >= nnzr) igref = 0;
            if (igref == 1) {
                if (nstsr(ipzr, ipxr) != 0 || nstsr(ipzr + 1, ipxr) != 0) igref = 0;
                if (nstsr(ipzr, ipxr + 1) != 0 || nstsr(ipzr + 1, ipxr + 1) != 0) igref = 0;
            }
            ipx = (int)((rgx[j + 1] - gox) / dnx) + 1;
            ipz = (int)((rgz[j + 1] - goz) / dnz) + 1;
        } else {
            ipx = (int)((rgx[j + 1] - gox) / dnx) + 1;
            ipz = (int)((rgz[j + 1] - goz) / dnz) + 1;
            igref = 0;
        }
        sred = sq((scx - rgx[j + 1]) * earth);
        sred = sred + sq((scz - rgz[j + 1]) * earth * std::sin(rgx[j + 1]));
        sred = std::sqrt(sred);
        sw = 0;
        if (sred < 2.0f * dpl) { rgx[j + 2] = scx; rgz[j + 2] = scz; nrp = j + 2; sw = 1; }
        if (sw == 0) {
            if (asgr == 1) {
                if (igref == 1 && ipxr == isx && ipzr == isz) { rgx[j + 2] = scx; rgz[j + 2] = scz; nrp = j + 2; sw = 1; }
            } else if (ipx == isx && ipz == isz) {
                rgx[j + 2] = scx; rgz[j + 2] = scz; nrp = j + 2; sw = 1;
            }
        }
        if (ipx < 1) { rgx[j + 1] = gox; ipx = 1; rbint = 1; }
        if (ipx >= nnx) { rgx[j + 1] = gox + (float)(nnx - 1) * dnx; ipx = nnx - 1; rbint = 1; }
        if (ipz < 1) { rgz[j + 1] = goz; ipz = 1; rbint = 1; }
        if (ipz >= nnz) { rgz[j + 1] = goz + (float)(nnz - 1) * dnz; ipz = nnz - 1; rbint = 1; }
        // Frechet derivatives (fmst.f90:734-906)
        int ivx = (ipx - 1) / gdx + 1, ivz = (ipz - 1) / gdz + 1;
        int ivxo = (ipxo - 1) / gdx + 1, ivzo = (ipzo - 1) / gdz + 1;
        int nhp = 0, chp[4];
        float vrat[4];
        if (ivx != ivxo) {
            nhp = nhp + 1;
            float xi = (ivx > ivxo) ? gox + (float)(ivx - 1) * dvx : gox + (float)ivx * dvx;
            vrat[nhp - 1] = (xi - rgx[j]) / (rgx[j + 1] - rgx[j]);
            chp[nhp - 1] = 1;
        }
        if (ivz != ivzo) {
            nhp = nhp + 1;
            float zi = (ivz > ivzo) ? goz + (float)(ivz - 1) * dvz : goz + (float)ivz * dvz;
            float r = (zi - rgz[j]) / (rgz[j + 1] - rgz[j]);
            if (nhp == 1) { vrat[nhp - 1] = r; chp[nhp - 1] = 2; }
            else if (r >= vrat[nhp - 2]) { vrat[nhp - 1] = r; chp[nhp - 1] = 2; }
            else {
                vrat[nhp - 1] = vrat[nhp - 2]; chp[nhp - 1] = chp[nhp - 2];
                vrat[nhp - 2] = r; chp[nhp - 2] = 2;
            }
        }
        nhp = nhp + 1;
        vrat[nhp - 1] = 1.0f;
        chp[nhp - 1] = 0;
        float vel = vel_at(rgx[j], rgz[j], ipxo, ipzo);
        float vi[4], wi[4], vio[4], wio[4];
        basis(((rgx[j] - gox) - (float)(ivxo - 1) * dvx) / dvx, vi);
        basis(((rgz[j] - goz) - (float)(ivzo - 1) * dvz) / dvz, wi);
        int ivxt = ivxo, ivzt = ivzo;
        for (int k = 1; k <= nhp; ++k) {
            float velo = vel;
            for (int q = 0; q < 4; ++q) { vio[q] = vi[q]; wio[q] = wi[q]; }
            if (k > 1) {
                if (chp[k - 2] == 1) ivxt = ivx;
                else if (chp[k - 2] == 2) ivzt = ivz;
            }
            float rigz = rgz[j] + vrat[k - 1] * (rgz[j + 1] - rgz[j]);
            float rigx = rgx[j] + vrat[k - 1] * (rgx[j + 1] - rgx[j]);
            int ipxt = (int)((rigx - gox) / dnx) + 1;
            int ipzt = (int)((rigz - goz) / dnz) + 1;
            vel = vel_at(rigx, rigz, ipxt, ipzt);
            basis(((rigx - gox) - (float)(ivxt - 1) * dvx) / dvx, vi);
            basis(((rigz - goz) - (float)(ivzt - 1) * dvz) / dvz, wi);
            float dinc = (k == 1) ? vrat[k - 1] * dpl : (vrat[k - 1] - vrat[k - 2]) * dpl;
            for (int l = 1; l <= 4; ++l)
                for (int m = 1; m <= 4; ++m) {
                    float r1 = vi[m - 1] * wi[l - 1] / sq(vel);
                    float r2 = vio[m - 1] * wio[l - 1] / sq(velo);
                    r1 = -(r1 + r2) * dinc / 2.0f;
                    r2 = F0(ivzt - 2 + l, ivxt - 2 + m);
                    F0(ivzt - 2 + l, ivxt - 2 + m) = r1 + r2;
                }
        }
    }
    float tsyn = 0.0f;
    if (nrp < 0) {
        tsyn = NAN;
    } else {
        for (int j = 1; j <= nrp - 1; ++j) {
            float dinc = oracle_delsph(rgx[j], rgz[j], rgx[j + 1], rgz[j + 1]);
            int ipxo = (int)((rgx[j] - gox) / dnx) + 1;
            int ipzo = (int)((rgz[j] - goz) / dnz) + 1;
            float velo = vel_at(rgx[j], rgz[j], ipxo, ipzo);
            ipxo = (int)((rgx[j + 1] - gox) / dnx) + 1;
            ipzo = (int)((rgz[j + 1] - goz) / dnz) + 1;
            float vel = vel_at(rgx[j + 1], rgz[j + 1], ipxo, ipzo);
            tsyn = tsyn + dinc * 0.5f * (1.0f / vel + 1.0f / velo);
        }
    }
    // fdm = transpose(fdm0): fdm(0:nvx+1, 0:nvz+1) column-major
    for (int j = 0; j <= nvz + 1; ++j)
        for (int k = 0; k <= nvx + 1; ++k) fdm[(size_t)k + (size_t)j * (nvx + 2)] = F0(j, k);
    return tsyn;
}

// ---------------------------------------------------------------------------
// The reference's C entry points (src/SWD/SurfaceWave.hpp:8-50)
extern "C" void fmst_init(int nx, int ny, float goxdf, float gozdf, float dvxdf, float dvzdf) {
    S.init(nx, ny, goxdf, gozdf, dvxdf, dvzdf);
}
extern "C" void fmst_finalize() { S = Fmst(); }
extern "C" void fmst_run(const double* velf, float srcx, float srcz, const float* rcx, const float* rcz, int nr,
                         float* ttime) {
    S.run(velf, srcx, srcz, rcx, rcz, nr, ttime);
}
extern "C" void fmst_reset(const double* velin) { S.reset(velin); }
extern "C" float fmst_raypath(float scx, float scz, float rcx, float rcz, float* fdm) {
    return S.raypath(scx, scz, rcx, rcz, fdm);
}

// Coarse traveltime field and node status of the last fmst_run on this
// thread ((nnz, nnx) column-major), for tests.
extern "C" int oracle_fmst_field(float* ttn, int32_t* nsts, int cap) {
    int n = S.nnx * S.nnz;
    if (n > cap) return -1;
    for (int ix = 1; ix <= S.nnx; ++ix)
        for (int iz = 1; iz <= S.nnz; ++iz) {
            ttn[(size_t)(iz - 1) + (size_t)(ix - 1) * S.nnz] = S.ttn(iz, ix);
            nsts[(size_t)(iz - 1) + (size_t)(ix - 1) * S.nnz] = S.nsts(iz, ix);
        }
    return n;
}

// The per-pair loop of SurfTime::travel_time (SurfaceWave.cpp:510-541) and,
// with want_fdm, of frechet_matrix (:583-672), over OpenMP threads:
// pair p uses phase map vc + slot[p]*ncol and group map vout + slot[p]*ncol,
// its receivers rcv_ptr[p]..rcv_ptr[p+1]-1; group[p] != 0 (Rg/Lg) replaces
// the receiver time by the ray's time.  fdm (if not null) receives the
// (nx, ny) weights of every receiver, in receiver order.
extern "C" void oracle_fmst_pairs(int nx, int ny, float goxd, float gozd, float dvxd, float dvzd, int npairs,
                                  const int32_t* slot, const float* srcx, const float* srcz, const int64_t* rcv_ptr,
                                  const float* rcx, const float* rcz, const int32_t* group, const double* vc,
                                  const double* vout, float* ttime, float* fdm, int nthreads) {
    const size_t ncol = (size_t)nx * ny;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
    for (int p = 0; p < npairs; ++p) {
        int64_t r0 = rcv_ptr[p], nr = rcv_ptr[p + 1] - r0;
        fmst_init(nx, ny, goxd, gozd, dvxd, dvzd);
        fmst_run(vc + (size_t)slot[p] * ncol, srcx[p], srcz[p], rcx + r0, rcz + r0, (int)nr, ttime + r0);
        fmst_reset(vout + (size_t)slot[p] * ncol);
        std::vector<float> tmp(ncol);
        for (int64_t i = 0; i < nr; ++i) {
            if (!fdm && !group[p]) continue;
            float* f = fdm ? fdm + (size_t)(r0 + i) * ncol : tmp.data();
            float t = fmst_raypath(srcx[p], srcz[p], rcx[r0 + i], rcz[r0 + i], f);
            if (group[p]) ttime[r0 + i] = t;
        }
        fmst_finalize();
    }
}
