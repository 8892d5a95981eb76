// Test harness: the GPU's fast-marching code (jdsurfg_b200/csrc/
// swdk_fmst_march.cuh: refined source grid, narrow-band march with the
// reference's heap, receiver times) compiled for the host, one pair after
// another, so tests can compare it with the oracle on the CPU.  Built by
// tests/test_fmst_march_host.py with -ffp-contract=off.
#include <vector>

#include "swdk_fmst_march.cuh"

using namespace swdk_fmst_march;

// mode 0: the window march one lane runs; 1: the neighbours one by one from
// their own stencils (the per-lane work of the four-lane march).
// Receiver times (srtimes) of every pair, and for pair `field_pair` its
// propagation-grid times and statuses ((nnz, nnx) column-major).  vc is
// (kmax, nx*ny); returns the largest narrow band, or -1 on overflow.
extern "C" int fm_host_pairs(int mode, int nx, int ny, float goxd, float gozd, float dvxd, float dvzd, int npairs,
                             const int32_t* slot, const float* srcx, const float* srcz, const int64_t* rcv_ptr,
                             const float* rcx, const float* rcz, const double* vc, float* ttime, int field_pair,
                             float* field_t, int32_t* field_s) {
    const Grid G = make_grid(nx, ny, goxd, gozd, dvxd, dvzd);
    std::vector<float> risti_c, risti_r;
    make_risti(G, risti_c, risti_r);
    const size_t N = (size_t)G.nnx * G.nnz, ncol = (size_t)nx * ny;
    const int cap = (int)std::lround(0.5f * (float)(G.nnx * G.nnz));
    std::vector<FNode> coarse(N), fine((size_t)RMAX * RMAX);
    std::vector<FHeap> heap(cap + 2), fheap(RCAP + 1);
    std::vector<float> rvel((size_t)RMAX * RMAX), rslw((size_t)RMAX * RMAX), veln(N), slwn(N);
    PairGeo geo;
    unsigned int cnt[2] = {0, 0};
    int band = 0;
    for (int p = 0; p < npairs; ++p) {
        const double* map = vc + (size_t)slot[p] * ncol;
        for (int stx = 1; stx <= G.nnx; ++stx)
            for (int stz = 1; stz <= G.nnz; ++stz) {
                const size_t i = (stz - 1) + (size_t)(stx - 1) * G.nnz;
                veln[i] = dice_node(map, G, stz, stx);
                slwn[i] = 1.0f / veln[i];
            }
        geo = pair_geometry(G, srcx[p], srcz[p]);
        for (int64_t r = rcv_ptr[p]; r < rcv_ptr[p + 1]; ++r) ttime[r] = NAN;
        if (geo.status) continue;
        for (int idm2 = 1; idm2 <= geo.nrnx; ++idm2)
            for (int idm1 = 1; idm1 <= geo.nrnz; ++idm1) {
                const size_t i = (idm1 - 1) + (size_t)(idm2 - 1) * RMAX;
                rvel[i] = refine_node(map, G, geo, idm1, idm2);
                rslw[i] = 1.0f / rvel[i];
            }
        for (auto& n : coarse) n = FNode{0.0f, -1};
        Scratch S;
        S.coarse = coarse.data();
        S.heap = heap.data();
        S.fine = fine.data();
        S.rvel = rvel.data();
        S.rslw = rslw.data();
        S.fheap = fheap.data();
        S.geo = &geo;
        S.N = N;
        S.cap = cap;
        S.hstride = cap + 2;
        const int32_t zero = 0;
        cnt[0] = cnt[1] = 0;
        march_pair(G, 0, 0, srcx + p, srcz + p, &zero, slwn.data(), risti_c.data(), risti_r.data(), S, cnt, nullptr,
                   0, mode, 0, 1u);
        if (cnt[0]) return -1;
        band = std::max(band, (int)cnt[1]);
        RayIn in;
        in.coarse = coarse.data();
        in.fine = fine.data();
        in.veln = veln.data();
        in.velg = veln.data();
        for (int64_t r = rcv_ptr[p]; r < rcv_ptr[p + 1]; ++r)
            ttime[r] = srtimes(G, in, geo, srcx[p], srcz[p], rcx[r], rcz[r], sinf(rcx[r]));
        if (p == field_pair)
            for (size_t i = 0; i < N; ++i) {
                field_t[i] = coarse[i].t;
                field_s[i] = coarse[i].s;
            }
    }
    return band;
}

struct LibcSin {  // the C library's sinf, as the reference calls it
    float operator()(float x) const { return sinf(x); }
};
struct RoundedSin {  // sin in double rounded to float, as the device computes it
    float operator()(float x) const { return (float)sin((double)x); }
};

// Receiver times and ray-path weights of every pair (the GPU's srtimes and
// raypath after the march), with the sine of moving ray points from the C
// library (sine = 0) or rounded from double (sine = 1).  vc, vout are
// (kmax, nx*ny); fdm, if not null, gets (nx, ny) per receiver.  Returns 0,
// or the first nonzero ray status.
extern "C" int fm_host_rays(int sine, int nx, int ny, float goxd, float gozd, float dvxd, float dvzd, int npairs,
                            const int32_t* slot, const float* srcx, const float* srcz, const int32_t* group,
                            const int64_t* rcv_ptr, const float* rcx, const float* rcz, const double* vc,
                            const double* vout, float* ttime, float* fdm) {
    const Grid G = make_grid(nx, ny, goxd, gozd, dvxd, dvzd);
    std::vector<float> risti_c, risti_r;
    make_risti(G, risti_c, risti_r);
    const size_t N = (size_t)G.nnx * G.nnz, ncol = (size_t)nx * ny;
    const int cap = (int)std::lround(0.5f * (float)(G.nnx * G.nnz));
    std::vector<FNode> coarse(N), fine((size_t)RMAX * RMAX);
    std::vector<FHeap> heap(cap + 2), fheap(RCAP + 1);
    std::vector<float> rvel((size_t)RMAX * RMAX), rslw((size_t)RMAX * RMAX), veln(N), slwn(N), velg(N);
    unsigned int cnt[2] = {0, 0};
    for (int p = 0; p < npairs; ++p) {
        const double* map = vc + (size_t)slot[p] * ncol;
        const double* gmap = vout + (size_t)slot[p] * ncol;
        for (int stx = 1; stx <= G.nnx; ++stx)
            for (int stz = 1; stz <= G.nnz; ++stz) {
                const size_t i = (stz - 1) + (size_t)(stx - 1) * G.nnz;
                veln[i] = dice_node(map, G, stz, stx);
                slwn[i] = 1.0f / veln[i];
                velg[i] = dice_node(gmap, G, stz, stx);
            }
        PairGeo geo = pair_geometry(G, srcx[p], srcz[p]);
        if (geo.status) return geo.status;
        for (int idm2 = 1; idm2 <= geo.nrnx; ++idm2)
            for (int idm1 = 1; idm1 <= geo.nrnz; ++idm1) {
                const size_t i = (idm1 - 1) + (size_t)(idm2 - 1) * RMAX;
                rvel[i] = refine_node(map, G, geo, idm1, idm2);
                rslw[i] = 1.0f / rvel[i];
            }
        for (auto& n : coarse) n = FNode{0.0f, -1};
        Scratch S;
        S.coarse = coarse.data();
        S.heap = heap.data();
        S.fine = fine.data();
        S.rvel = rvel.data();
        S.rslw = rslw.data();
        S.fheap = fheap.data();
        S.geo = &geo;
        S.N = N;
        S.cap = cap;
        S.hstride = cap + 2;
        const int32_t zero = 0;
        cnt[0] = cnt[1] = 0;
        march_pair(G, 0, 0, srcx + p, srcz + p, &zero, slwn.data(), risti_c.data(), risti_r.data(), S, cnt, nullptr,
                   0, 0, 0, 1u);
        if (cnt[0]) return SWDK_FMST_BAND_OVERFLOW;
        RayIn in;
        in.coarse = coarse.data();
        in.fine = fine.data();
        in.veln = veln.data();
        in.velg = velg.data();
        for (int64_t r = rcv_ptr[p]; r < rcv_ptr[p + 1]; ++r) {
            const float sr = sinf(rcx[r]);
            float t = srtimes(G, in, geo, srcx[p], srcz[p], rcx[r], rcz[r], sr);
            float* f = fdm ? fdm + (size_t)r * ncol : nullptr;
            if (f)
                for (size_t i = 0; i < ncol; ++i) f[i] = 0.0f;
            if (f || group[p]) {
                int st = 0;
                const float tr = sine == 0 ? raypath(G, in, geo, srcx[p], srcz[p], rcx[r], rcz[r], sr, f, &st, LibcSin{})
                                           : raypath(G, in, geo, srcx[p], srcz[p], rcx[r], rcz[r], sr, f, &st,
                                                     RoundedSin{});
                if (st) return st;
                if (group[p]) t = tr;
            }
            ttime[r] = t;
        }
    }
    return 0;
}
