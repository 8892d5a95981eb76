// Fast marching of one station pair: the grid constants, the refined
// source grid, the narrow-band march with the reference's binary heap and
// the mixed-order update (src/SWD/fmst.f90:108-310, src/SWD/fmm.f90:138-770).
// Included by swdk_fmst.cu, where each marching lane runs march_pair for one
// pair; the same code also compiles as plain C++ (FM_HD empty) so the tests
// can run it on the CPU against the oracle.  Its REAL*4 arithmetic follows
// the Fortran's operation order and must be compiled without contraction
// (nvcc -fmad=false, g++ -ffp-contract=off).
#pragma once
#include <stdint.h>

#include <cmath>

#if defined(__CUDACC__)
#define FM_HD __device__
#define FM_INLINE __forceinline__
#else
#define FM_HD
#define FM_INLINE inline
#include <cstring>
#include <algorithm>
using std::max;
using std::min;
inline int __float_as_int(float x) { int i; std::memcpy(&i, &x, 4); return i; }
inline float __double2float_rn(double x) { return (float)x; }
inline float __int_as_float(int i) { float x; std::memcpy(&x, &i, 4); return x; }
struct float4 { float x, y, z, w; };
#endif

#ifndef SWDK_FMST_SOURCE_OUTSIDE
#define SWDK_FMST_SOURCE_OUTSIDE 1
#define SWDK_FMST_RECEIVER_OUTSIDE 2
#define SWDK_FMST_BAND_OVERFLOW 3
#define SWDK_FMST_RAY_UNFINISHED 4
#endif

namespace swdk_fmst_march {

FM_HD FM_INLINE void fm_atomic_max(unsigned int* a, unsigned int v) {
#if defined(__CUDA_ARCH__)
    atomicMax(a, v);
#else
    if (v > *a) *a = v;
#endif
}
FM_HD FM_INLINE void fm_atomic_add(unsigned int* a, unsigned int v) {
#if defined(__CUDA_ARCH__)
    atomicAdd(a, v);
#else
    *a += v;
#endif
}


constexpr int GDX = 8, GDZ = 8;   // grid dicing (fmst.f90:30-31)
constexpr int SGDL = 8;           // source grid dicing level (fmst.f90:33)
constexpr int SGS = 8;            // refined box half-width in nodes (fmst.f90:140)
constexpr float EARTH = 6371.0f;  // fmst.f90:34
constexpr float PI_SP = 3.1415926535898f;
constexpr int RMAX = 2 * SGS * SGDL + 1;   // refined grid nodes per side (129)
constexpr int RCAP = (RMAX * RMAX + 1) / 2; // refined heap (snb * nodes)

struct FNode {  // node status (-1 far, 0 alive, >0 heap position) and time
    float t;
    int s;
};
struct FHeap {  // heap entry: node time and node coordinates (iz-1) | (ix-1) << 16
    float key;
    int node;
};

// Per-pair geometry (fmst.f90:145-200)
struct PairGeo {
    int isx, isz;           // source cell on the propagation grid
    int vnl, vnr, vnt, vnb; // refined box bounds
    int nrnx, nrnz;         // refined grid size
    float gorx, gorz;       // refined grid origin
    int status;             // 0 ok, SWDK_FMST_* otherwise
    int ntr_max;            // largest narrow band seen
};

struct Grid {  // constants of the propagation grid (fmst_init)
    int nx, ny, nvx, nvz, nnx, nnz;
    float gox, goz, dvx, dvz, dnx, dnz, drnx, drnz;
    float dpl;  // min(dnx*earth, dnz*earth*sin(gox), dnz*earth*sin(gox+(nnx-1)*dnx)) (fmm.f90:1011-1015)
};

FM_HD FM_INLINE float sq(float x) { return x * x; }
FM_HD FM_INLINE float cube(float x) { return (x * x) * x; }

// B-spline basis at u (fmm.f90:818-821, fmst.f90:806-813)
FM_HD FM_INLINE void basis(float u, float* b) {
    b[0] = cube(1.0f - u) / 6.0f;
    b[1] = (4.0f - 6.0f * sq(u) + 3.0f * cube(u)) / 6.0f;
    b[2] = (1.0f + 3.0f * u + 3.0f * sq(u) - 3.0f * cube(u)) / 6.0f;
    b[3] = cube(u) / 6.0f;
}

FM_HD FM_INLINE float velv(const double* map, int nx, int i, int j) {
    // velv(i, j) = real(pv(i*(nvx+2)+j+1)) (fmm.f90:808)
    return __double2float_rn(map[(size_t)i * nx + j]);
}

// One propagation-grid node of the diced map (fmm.f90:823-863): cell (i, j)
// and sub-node (l, m) of node (stz, stx).
FM_HD float dice_node(const double* map, const Grid& G, int stz, int stx) {
    int i = (stz - 1) / GDZ + 1;
    if (i > G.nvz - 1) i = G.nvz - 1;
    int l = stz - GDZ * (i - 1);
    int j = (stx - 1) / GDX + 1;
    if (j > G.nvx - 1) j = G.nvx - 1;
    int m = stx - GDX * (j - 1);
    float ui[4], vi[4];
    basis((float)(m - 1) / (float)GDX, ui);
    basis((float)(l - 1) / (float)GDZ, vi);
    float sumi = 0.0f;
#pragma unroll
    for (int i1 = 0; i1 < 4; ++i1) {
        float sumj = 0.0f;
#pragma unroll
        for (int j1 = 0; j1 < 4; ++j1) sumj = sumj + ui[j1] * velv(map, G.nx, i - 1 + i1, j - 1 + j1);
        sumi = sumi + vi[i1] * sumj;
    }
    return sumi;
}

FM_HD PairGeo pair_geometry(const Grid& G, float x, float z) {
    PairGeo g{};
    g.isx = (int)((x - G.gox) / G.dnx) + 1;
    g.isz = (int)((z - G.goz) / G.dnz) + 1;
    if (g.isx < 1 || g.isx > G.nnx || g.isz < 1 || g.isz > G.nnz) {
        g.status = SWDK_FMST_SOURCE_OUTSIDE;
        return g;
    }
    if (g.isx == G.nnx) g.isx -= 1;
    if (g.isz == G.nnz) g.isz -= 1;
    g.vnl = max(g.isx - SGS, 1);
    g.vnr = min(g.isx + SGS, G.nnx);
    g.vnt = max(g.isz - SGS, 1);
    g.vnb = min(g.isz + SGS, G.nnz);
    g.nrnx = (g.vnr - g.vnl) * SGDL + 1;
    g.nrnz = (g.vnb - g.vnt) * SGDL + 1;
    g.gorx = G.gox + G.dnx * (float)(g.vnl - 1);
    g.gorz = G.goz + G.dnz * (float)(g.vnt - 1);
    return g;
}

// One grid (refined or propagation) of one pair during fast marching.
struct March {
    FNode* nd;            // nodes, (iz, ix) at (iz-1) + (ix-1)*ld
    const float* slw;     // slowness 1/v, same layout (fouds2's slown)
    const float* risti;   // earth*sin(gox+(ix-1)*dnx), ix = 1..nnx
    FHeap* heap;          // heap[1..cap]
    int ld, nnx, nnz, cap, ntr, ntr_max;
    float dnx, dnz;
    bool overflow;

    FM_HD FM_INLINE int idx(int iz, int ix) const { return (iz - 1) + (ix - 1) * ld; }
    static FM_HD FM_INLINE int pack(int iz, int ix) { return (iz - 1) | ((ix - 1) << 16); }
    FM_HD FM_INLINE int lin(int pk) const { return (pk & 0xFFFF) + (pk >> 16) * ld; }

    // fmm.f90:618-647 (the moving entry is written once, at its final slot)
    FM_HD void addtree(int pk, float key) {
        if (ntr >= cap) { overflow = true; return; }
        int tpc = ++ntr;
        ntr_max = max(ntr_max, ntr);
        int tpp = tpc / 2;
        while (tpp > 0) {
            FHeap h = heap[tpp];
            if (key < h.key) {
                nd[lin(h.node)].s = tpc;
                heap[tpc] = h;
                tpc = tpp;
                tpp = tpc / 2;
            } else {
                break;
            }
        }
        heap[tpc] = FHeap{key, pk};
        nd[lin(pk)].s = tpc;
    }

    // fmm.f90:744-770, after the node's time changed to key
    FM_HD void updtree(int pk, int n, float key) {
        int tpc = nd[n].s;
        int tpp = tpc / 2;
        while (tpp > 0) {
            FHeap h = heap[tpp];
            if (key < h.key) {
                nd[lin(h.node)].s = tpc;
                heap[tpc] = h;
                tpc = tpp;
                tpp = tpc / 2;
            } else {
                break;
            }
        }
        heap[tpc] = FHeap{key, pk};
        nd[n].s = tpc;
    }

    // fmm.f90:657-736
    FM_HD void downtree() {
        if (ntr == 1) { ntr = 0; return; }
        const FHeap last = heap[ntr];
        ntr = ntr - 1;
        int tpp = 1, tpc = 2;
        while (tpc < ntr) {
            const float4 cc = *reinterpret_cast<const float4*>(&heap[tpc]);  // children tpc, tpc+1
            FHeap c{cc.x, __float_as_int(cc.y)};
            if (cc.x > cc.z) { c = FHeap{cc.z, __float_as_int(cc.w)}; tpc = tpc + 1; }
            if (c.key < last.key) {
                heap[tpp] = c;
                nd[lin(c.node)].s = tpp;
                tpp = tpc;
                tpc = 2 * tpp;
            } else {
                tpc = ntr + 1;
            }
        }
        if (tpc == ntr) {
            FHeap c = heap[tpc];
            if (c.key < last.key) {
                heap[tpp] = c;
                nd[lin(c.node)].s = tpp;
                tpp = tpc;
            }
        }
        heap[tpp] = last;
        nd[lin(last.node)].s = tpp;
    }

    FM_HD FM_INLINE float risti_at(int ix) const { return risti[ix - 1]; }

    // The refined pass stops before accepting a node on a side of the refined
    // grid (fmm.f90:232-254).  The reference tests the right and bottom sides
    // as `vnr /= nnx`, `vnb /= nnz` while nnx, nnz hold the refined grid's
    // sizes (fmst.f90:206-207 set them before travel is called), so those two
    // sides always stop it.
    FM_HD FM_INLINE bool at_refined_side(const PairGeo& g, int iz, int ix) const {
        return (ix == 1 && g.vnl != 1) || (ix == nnx && g.vnr != nnx) || (iz == 1 && g.vnt != 1) ||
               (iz == nnz && g.vnb != nnz);
    }

    // The 25 nodes the four neighbours' stencils read: the axes to distance
    // 3 and the off-axis nodes with |dz|, |dx| <= 2 and |dz| + |dx| <= 3.
    static FM_HD FM_INLINE bool in_window(int dz, int dx) {
        const int adz = dz < 0 ? -dz : dz, adx = dx < 0 ? -dx : dx;
        if (dz == 0 && dx == 0) return false;  // the accepted node itself
        return (dz == 0 && adx <= 3) || (dx == 0 && adz <= 3) || (adz + adx <= 3 && adz <= 2 && adx <= 2);
    }

    // Node (iz+dz, ix+dx) for the window around an accepted node; nodes off
    // the grid read as status -2, which no test for "alive" (== 0) accepts.
    FM_HD FM_INLINE FNode wload(int iz, int ix, int dz, int dx) const {
        const int z = iz + dz, x = ix + dx;
        if (z < 1 || z > nnz || x < 1 || x > nnx) return FNode{0.0f, -2};
        return nd[idx(z, x)];
    }

    // One candidate time of fouds2 (fmm.f90:576-586): the root of
    // a t^2 + b t + c = 0, then (tref + t) / tdiv.  The one-sided stencils have
    // a = 1, b = 0, where rd1 = -(4c) and the division by 2a = 2 is the exact
    // product with 0.5; tdiv = 1 needs no division: the same IEEE results.
    static FM_HD FM_INLINE float root2(float a, float b, float c, float tref, float tdiv) {
        float rd1 = sq(b) - 4.0f * a * c;
        if (rd1 < 0.0f) rd1 = 0.0f;
        const float tdsh = (-b + sqrtf(rd1)) / (2.0f * a);
        return (tdiv == 1.0f) ? tref + tdsh : (tref + tdsh) / tdiv;
    }
    static FM_HD FM_INLINE float root1(float c, float tref, bool third) {
        float rd1 = 0.0f - 4.0f * c;
        if (rd1 < 0.0f) rd1 = 0.0f;
        const float tdsh = sqrtf(rd1) * 0.5f;
        return third ? (tref + tdsh) / 3.0f : tref + tdsh;
    }

    // fmm.f90:437-610 (mixed-order scheme, fom = 1) for the neighbour at
    // offset (CZ, CX) of the accepted node, from the window w[dz+3][dx+3];
    // (iz, ix) are the neighbour's coordinates, slown its slowness.
    //
    // The reference takes the minimum over the four quadrants (j, k) of one
    // candidate each.  A quadrant's candidate is two-sided when both its x
    // side (j: first or second order available) and its z side (k) are, and
    // otherwise one-sided -- a value that depends on j alone (or k alone).  So
    // the two-sided candidates are evaluated per quadrant, each one-sided
    // candidate once, and only if some in-range quadrant would produce it: the
    // same set of candidates, hence the same minimum.
    template <int CZ, int CX>
    FM_HD FM_INLINE float fouds2w(const FNode (&w)[7][7], int iz, int ix, float slown, float risti) const {
        const float ri = EARTH;
        // x sides (sj = -1, +1) and z sides (sk = -1, +1): 0 none, 1 first order, 2 second order
        int X[2], Z[2];
        bool jr[2], kr[2];
        FNode nj[2], nj2[2], nk[2], nk2[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int sj = 2 * q - 1;
            jr[q] = ix + sj >= 1 && ix + sj <= nnx;
            nj[q] = w[CZ + 3][CX + sj + 3];
            nj2[q] = w[CZ + 3][CX + 2 * sj + 3];
            X[q] = (jr[q] && nj[q].s == 0) ? ((nj2[q].s == 0 && nj[q].t > nj2[q].t) ? 2 : 1) : 0;
            const int sk = sj;
            kr[q] = iz + sk >= 1 && iz + sk <= nnz;
            nk[q] = w[CZ + sk + 3][CX + 3];
            nk2[q] = w[CZ + 2 * sk + 3][CX + 3];
            Z[q] = (kr[q] && nk[q].s == 0) ? ((nk2[q].s == 0 && nk[q].t > nk2[q].t) ? 2 : 1) : 0;
        }
        const bool xnone = (kr[0] && Z[0] == 0) || (kr[1] && Z[1] == 0);  // some quadrant has no z side
        const bool znone = (jr[0] && X[0] == 0) || (jr[1] && X[1] == 0);  // some quadrant has no x side
        bool any = false;
        float travm = 0.0f;
        auto take = [&](float trav) {
            travm = any ? fminf(trav, travm) : trav;
            any = true;
        };
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            if (X[a] == 0) continue;
            const float tj = nj[a].t, tj2 = nj2[a].t;
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                if (!kr[b] || Z[b] == 0) continue;
                const float tk = nk[b].t, tk2 = nk2[b].t;
                if (X[a] == 2 && Z[b] == 2) {
                    const float u = 2.0f * ri * dnx, v = 2.0f * risti * dnz;
                    float em = 4.0f * tj - tj2 - 4.0f * tk;
                    em = em + tk2;
                    take(root2(sq(v) + sq(u), 2.0f * em * sq(u), sq(u) * (sq(em) - sq(slown) * sq(v)),
                               4.0f * tj - tj2, 3.0f));
                } else if (X[a] == 2) {  // second order in x, first in z
                    const float u = risti * dnz, v = 2.0f * ri * dnx;
                    const float em = 3.0f * tk - 4.0f * tj + tj2;
                    take(root2(sq(v) + 9.0f * sq(u), 6.0f * em * sq(u), sq(u) * (sq(em) - sq(slown) * sq(v)), tk,
                               1.0f));
                } else if (Z[b] == 2) {  // first order in x, second in z
                    const float u = ri * dnx, v = 2.0f * risti * dnz;
                    const float em = 3.0f * tj - 4.0f * tk + tk2;
                    take(root2(sq(v) + 9.0f * sq(u), 6.0f * em * sq(u), sq(u) * (sq(em) - sq(v) * sq(slown)), tj,
                               1.0f));
                } else {  // first order in both
                    const float u = ri * dnx, v = risti * dnz;
                    const float em = tk - tj;
                    take(root2(sq(u) + sq(v), -2.0f * sq(u) * em, sq(u) * (sq(em) - sq(v) * sq(slown)), tj, 1.0f));
                }
            }
            if (xnone) {  // one-sided in x
                if (X[a] == 2) {
                    const float u = 2.0f * ri * dnx;
                    take(root1(-sq(u) * sq(slown), 4.0f * tj - tj2, true));
                } else {
                    take(root1(-sq(slown) * sq(ri) * sq(dnx), tj, false));
                }
            }
        }
        if (znone) {
#pragma unroll
            for (int b = 0; b < 2; ++b) {  // one-sided in z
                if (!kr[b] || Z[b] == 0) continue;
                if (Z[b] == 2) {
                    const float u = 2.0f * risti * dnz;
                    take(root1(-sq(u) * sq(slown), 4.0f * nk[b].t - nk2[b].t, true));
                } else {
                    take(root1(-sq(slown) * sq(risti) * sq(dnz), nk[b].t, false));
                }
            }
        }
        return travm;
    }

    // one neighbour's heap update (fmm.f90:262-320) with its new time
    FM_HD FM_INLINE void apply(int iz, int ix, int s, float t) {
        const int n = idx(iz, ix);
        if (s == -1) {
            nd[n].t = t;
            addtree(pack(iz, ix), t);
        } else if (s > 0) {
            nd[n].t = t;
            updtree(pack(iz, ix), n, t);
        }
    }

    // Trial time of the neighbour at offset (dz, dx) of the accepted node
    // (iz, ix) whose time is tacc: fouds2 from the neighbour's own 8-node
    // stencil (the accepted node, alive, is one of them).  Returns the
    // neighbour's status before the update (-2 off the grid, 0 alive: no
    // update) and, for far or close neighbours, its new time in *t.
    FM_HD FM_INLINE int solve_neighbour(int iz, int ix, float tacc, int dz, int dx, float* t) const {
        const int z = iz + dz, x = ix + dx;
        if (z < 1 || z > nnz || x < 1 || x > nnx) return -2;
        const int n = idx(z, x);
        // the neighbour's status, its stencil and slowness in one round of loads
        const int s = nd[n].s;
        const float sl = slw[n];
        FNode w[7][7];
        w[3][2] = wload(z, x, 0, -1);
        w[3][4] = wload(z, x, 0, 1);
        w[3][1] = wload(z, x, 0, -2);
        w[3][5] = wload(z, x, 0, 2);
        w[2][3] = wload(z, x, -1, 0);
        w[4][3] = wload(z, x, 1, 0);
        w[1][3] = wload(z, x, -2, 0);
        w[5][3] = wload(z, x, 2, 0);
        // the accepted node, seen from the neighbour (constant indices keep w in registers)
        if (dx == -1) w[3][4] = FNode{tacc, 0};
        else if (dx == 1) w[3][2] = FNode{tacc, 0};
        else if (dz == -1) w[4][3] = FNode{tacc, 0};
        else w[2][3] = FNode{tacc, 0};
        if (s == -1 || s > 0) *t = fouds2w<0, 0>(w, z, x, sl, risti_at(x));
        return s;
    }

    // The same march as march() with the neighbours solved one by one from
    // their own stencils (the per-lane work of march_coop), sequentially.
    FM_HD void march_nb(bool refined, const PairGeo& g) {
        while (ntr > 0 && !overflow) {
            const FHeap root = heap[1];
            const int iz = (root.node & 0xFFFF) + 1, ix = (root.node >> 16) + 1;
            const int node = idx(iz, ix);
            if (refined && at_refined_side(g, iz, ix)) { nd[node].s = 0; return; }
            nd[node].s = 0;
            float t[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            int st[4];
            st[0] = solve_neighbour(iz, ix, root.key, 0, -1, &t[0]);
            st[1] = solve_neighbour(iz, ix, root.key, 0, 1, &t[1]);
            st[2] = solve_neighbour(iz, ix, root.key, -1, 0, &t[2]);
            st[3] = solve_neighbour(iz, ix, root.key, 1, 0, &t[3]);
            downtree();
            apply(iz, ix - 1, st[0], t[0]);
            apply(iz, ix + 1, st[1], t[1]);
            apply(iz - 1, ix, st[2], t[2]);
            apply(iz + 1, ix, st[3], t[3]);
        }
    }

#if defined(__CUDA_ARCH__)
    // march() by the lanes of a group (lane g4 of the group, mask gmask): the
    // lanes base .. base+3 solve the trial times of the neighbours x-1, x+1,
    // z-1, z+1; lane 0 of the group owns the heap, sifts it down meanwhile
    // and applies the four updates in the reference's order.  base = 0: lane
    // 0 also solves x-1 (groups of four lanes); base = 1: lane 0 only keeps
    // the heap, so its sift-down overlaps the solves (groups of eight lanes,
    // five of them active).  Every lane runs this with the same March state;
    // only lane 0's heap fields are live.
    __device__ void march_coop(bool refined, const PairGeo& g, int g4, unsigned gmask, int base) {
        const int lead = __ffs(gmask) - 1;
        const int q = g4 - base;  // neighbour this lane solves (0..3), or none
        const int dz = q == 2 ? -1 : (q == 3 ? 1 : 0), dx = q == 0 ? -1 : (q == 1 ? 1 : 0);
        for (;;) {
            int go = 0, pk = 0;
            float tacc = 0.0f;
            if (g4 == 0 && ntr > 0 && !overflow) {
                const FHeap root = heap[1];
                const int iz = (root.node & 0xFFFF) + 1, ix = (root.node >> 16) + 1;
                nd[idx(iz, ix)].s = 0;
                go = (refined && at_refined_side(g, iz, ix)) ? 0 : 1;
                pk = root.node;
                tacc = root.key;
            }
            go = __shfl_sync(gmask, go, lead);
            if (!go) break;
            pk = __shfl_sync(gmask, pk, lead);
            tacc = __shfl_sync(gmask, tacc, lead);
            __syncwarp(gmask);
            const int iz = (pk & 0xFFFF) + 1, ix = (pk >> 16) + 1;
            float t = 0.0f;
            int s = -2;
            if (q >= 0 && q < 4) s = solve_neighbour(iz, ix, tacc, dz, dx, &t);
            if (g4 == 0) downtree();
            const int s0 = __shfl_sync(gmask, s, lead + base), s1 = __shfl_sync(gmask, s, lead + base + 1),
                      s2 = __shfl_sync(gmask, s, lead + base + 2), s3 = __shfl_sync(gmask, s, lead + base + 3);
            const float t0 = __shfl_sync(gmask, t, lead + base), t1 = __shfl_sync(gmask, t, lead + base + 1),
                        t2 = __shfl_sync(gmask, t, lead + base + 2), t3 = __shfl_sync(gmask, t, lead + base + 3);
            if (g4 == 0) {
                apply(iz, ix - 1, s0, t0);
                apply(iz, ix + 1, s1, t1);
                apply(iz - 1, ix, s2, t2);
                apply(iz + 1, ix, s3, t3);
            }
            __syncwarp(gmask);
        }
        __syncwarp(gmask);
    }
#endif

    // fmm.f90:224-324: march until the heap is empty or, in the refined pass,
    // the node about to be accepted lies on a side of the refined grid.  The
    // reference tests the right and bottom sides as `vnr /= nnx`, `vnb /= nnz`
    // while nnx, nnz hold the refined grid's sizes (fmst.f90:206-207 set them
    // before travel is called), so those two sides always stop the pass.
    //
    // The four neighbours' trial times (fouds2) read only alive nodes, and
    // none of the neighbours' heap updates makes a node alive or changes an
    // alive node's time; the statuses the updates change only move between
    // far and close.  So the 25-node window around the accepted node is
    // loaded once (before the sift-down, to overlap the two), all four trial
    // times are solved from it, and the heap is then updated in the
    // reference's order (x-1, x+1, z-1, z+1): the same arithmetic and the
    // same heap, with one round of loads per accepted node.
    FM_HD void march(bool refined, const PairGeo& g) {
        while (ntr > 0 && !overflow) {
            const FHeap root = heap[1];  // the accepted node and its time
            const int iz = (root.node & 0xFFFF) + 1, ix = (root.node >> 16) + 1;
            const int node = idx(iz, ix);
            if (refined && at_refined_side(g, iz, ix)) { nd[node].s = 0; return; }
            nd[node].s = 0;
            FNode w[7][7];
            if (iz > 3 && iz + 3 <= nnz && ix > 3 && ix + 3 <= nnx) {  // the window lies inside the grid
#pragma unroll
                for (int dz = -3; dz <= 3; ++dz)
#pragma unroll
                    for (int dx = -3; dx <= 3; ++dx)
                        if (in_window(dz, dx)) w[dz + 3][dx + 3] = nd[node + dz + dx * ld];
            } else {
#pragma unroll
                for (int dz = -3; dz <= 3; ++dz)
#pragma unroll
                    for (int dx = -3; dx <= 3; ++dx)
                        if (in_window(dz, dx)) w[dz + 3][dx + 3] = wload(iz, ix, dz, dx);
            }
            w[3][3] = FNode{root.key, 0};  // the accepted node, now alive
            const int s0 = w[3][2].s, s1 = w[3][4].s, s2 = w[2][3].s, s3 = w[4][3].s;
            // slowness of the neighbours still to update, r*sin(colatitude) of their columns
            const float v0 = (s0 == -1 || s0 > 0) ? slw[node - ld] : 1.0f;
            const float v1 = (s1 == -1 || s1 > 0) ? slw[node + ld] : 1.0f;
            const float v2 = (s2 == -1 || s2 > 0) ? slw[node - 1] : 1.0f;
            const float v3 = (s3 == -1 || s3 > 0) ? slw[node + 1] : 1.0f;
            const float rm = ix > 1 ? risti_at(ix - 1) : 0.0f, rc = risti_at(ix),
                        rp = ix < nnx ? risti_at(ix + 1) : 0.0f;
            downtree();
            float t0 = 0.0f, t1 = 0.0f, t2 = 0.0f, t3 = 0.0f;
            if (s0 == -1 || s0 > 0) t0 = fouds2w<0, -1>(w, iz, ix - 1, v0, rm);
            if (s1 == -1 || s1 > 0) t1 = fouds2w<0, 1>(w, iz, ix + 1, v1, rp);
            if (s2 == -1 || s2 > 0) t2 = fouds2w<-1, 0>(w, iz - 1, ix, v2, rc);
            if (s3 == -1 || s3 > 0) t3 = fouds2w<1, 0>(w, iz + 1, ix, v3, rc);
            if (ix - 1 >= 1) apply(iz, ix - 1, s0, t0);
            if (ix + 1 <= nnx) apply(iz, ix + 1, s1, t1);
            if (iz - 1 >= 1) apply(iz - 1, ix, s2, t2);
            if (iz + 1 <= nnz) apply(iz + 1, ix, s3, t3);
        }
    }
};

// fmm.f90:1662-1683
FM_HD FM_INLINE float bilinear(const float nv[2][2], float dsx, float dsz, float dnx, float dnz) {
    float biv = 0.0f;
#pragma unroll
    for (int i = 1; i <= 2; ++i)
#pragma unroll
        for (int j = 1; j <= 2; ++j) {
            float produ = (1.0f - fabsf(((float)(i - 1) * dnx - dsx) / dnx)) *
                          (1.0f - fabsf(((float)(j - 1) * dnz - dsz) / dnz));
            biv = biv + nv[i - 1][j - 1] * produ;
        }
    return biv;
}

struct Scratch {  // device arrays of one chunk of pairs
    FNode* coarse;   // P * N
    FHeap* heap;     // P * hstride (cap + 1 rounded up to even: 16-byte aligned child pairs)
    FNode* fine;     // P * RMAX * RMAX
    float* rvel;     // P * RMAX * RMAX velocities of the refined grids
    float* rslw;     // P * RMAX * RMAX their slowness
    FHeap* fheap;    // P * (RCAP + 1)
    PairGeo* geo;    // P
    size_t N;
    int cap, hstride;
};

FM_HD void march_pair(const Grid& G, int p, int gp, const float* __restrict__ srcx,
                           const float* __restrict__ srcz, const int32_t* __restrict__ pslot,
                           const float* __restrict__ slwn, const float* __restrict__ risti_c,
                           const float* __restrict__ risti_r, const Scratch& S, unsigned int* __restrict__ n_overflow,
                           FHeap* hp, int smem_cap, int mode, int g4, unsigned gmask) {
    // mode 0: one lane, window march; 1: one lane, neighbours one by one;
    // 2: the four lanes g4 = 0..3 of mask gmask march the pair together
    // (lane 0 writes the grids and owns the heap); 3: five lanes, lane 0 only
    // owns the heap and lanes 1..4 solve.
    PairGeo g = S.geo[p];
    if (g.status) return;
    const bool lead = g4 == 0;
    auto group_sync = [&]() {
#if defined(__CUDA_ARCH__)
        if (mode >= 2) __syncwarp(gmask);
#endif
    };
    auto run = [&](March& M, bool refined) {
        if (mode == 1) M.march_nb(refined, g);
#if defined(__CUDA_ARCH__)
        else if (mode == 2 || mode == 3) M.march_coop(refined, g, g4, gmask, mode == 3 ? 1 : 0);
#endif
        else M.march(refined, g);
    };
    const float x = srcx[gp], z = srcz[gp];
    FNode* fine = S.fine + (size_t)p * RMAX * RMAX;

    // refined source grid pass (urg = 1): fmm.f90:170-205 start, then march
    March R;
    R.nd = fine;
    R.slw = S.rslw + (size_t)p * RMAX * RMAX;
    const float* rvel = S.rvel + (size_t)p * RMAX * RMAX;
    R.risti = risti_r + (size_t)(g.vnl - 1) * RMAX;
    R.heap = hp ? hp : S.fheap + (size_t)p * (RCAP + 1);
    R.ld = RMAX;
    R.nnx = g.nrnx;
    R.nnz = g.nrnz;
    R.cap = hp ? min(smem_cap, RCAP) : RCAP;
    R.ntr = 0;
    R.ntr_max = 0;
    R.dnx = G.drnx;
    R.dnz = G.drnz;
    R.overflow = false;
    if (lead) {
        for (int ix = 1; ix <= g.nrnx; ++ix)
            for (int iz = 1; iz <= g.nrnz; ++iz) R.nd[R.idx(iz, ix)] = FNode{0.0f, -1};
        int isx = (int)((x - g.gorx) / G.drnx) + 1;
        int isz = (int)((z - g.gorz) / G.drnz) + 1;
        if (isx == g.nrnx) isx -= 1;
        if (isz == g.nrnz) isz -= 1;
        isx = min(max(isx, 1), g.nrnx - 1);
        isz = min(max(isz, 1), g.nrnz - 1);
        float vss[2][2];
        for (int i = 1; i <= 2; ++i)
            for (int j = 1; j <= 2; ++j) vss[i - 1][j - 1] = rvel[R.idx(isz - 1 + j, isx - 1 + i)];
        float dsx = (x - g.gorx) - (float)(isx - 1) * G.drnx;
        float dsz = (z - g.gorz) - (float)(isz - 1) * G.drnz;
        float vsrc = bilinear(vss, dsx, dsz, G.drnx, G.drnz);
        for (int i = 1; i <= 2; ++i)
            for (int j = 1; j <= 2; ++j) {
                float ds = sqrtf(sq(dsx - (float)(i - 1) * G.drnx) + sq(dsz - (float)(j - 1) * G.drnz));
                float t = 2.0f * ds / (vss[i - 1][j - 1] + vsrc);
                R.nd[R.idx(isz - 1 + j, isx - 1 + i)].t = t;
                R.addtree(March::pack(isz - 1 + j, isx - 1 + i), t);
            }
    }
    group_sync();
    run(R, true);

    // resample onto the propagation grid (fmst.f90:240-252); the grid's
    // statuses were set to far by k_fmst_clear
    March C;
    C.nd = S.coarse + (size_t)p * S.N;
    C.slw = slwn + (size_t)pslot[gp] * S.N;
    C.risti = risti_c;
    C.heap = hp ? hp : S.heap + (size_t)p * S.hstride;
    C.ld = G.nnz;
    C.nnx = G.nnx;
    C.nnz = G.nnz;
    C.cap = hp ? smem_cap : S.cap;
    C.ntr = 0;
    C.ntr_max = 0;
    C.dnx = G.dnx;
    C.dnz = G.dnz;
    C.overflow = false;
    if (lead) {
        for (int k = 1; k <= g.nrnz; k += SGDL) {
            const int idm1 = g.vnt + (k - 1) / SGDL;
            for (int l = 1; l <= g.nrnx; l += SGDL) {
                const int idm2 = g.vnl + (l - 1) / SGDL;
                const FNode f = fine[R.idx(k, l)];
                FNode& c = C.nd[C.idx(idm1, idm2)];
                c.s = f.s;
                if (f.s >= 0) c.t = f.t;
            }
        }
        // narrow-band completion (fmst.f90:275-296), only the box can hold alive nodes
        for (int k = g.vnl; k <= g.vnr; ++k)
            for (int l = g.vnt; l <= g.vnb; ++l) {
                FNode& c = C.nd[C.idx(l, k)];
                if (c.s != 0) continue;
                if (l - 1 >= 1 && C.nd[C.idx(l - 1, k)].s == -1) c.s = 1;
                if (l + 1 <= G.nnz && C.nd[C.idx(l + 1, k)].s == -1) c.s = 1;
                if (k - 1 >= 1 && C.nd[C.idx(l, k - 1)].s == -1) c.s = 1;
                if (k + 1 <= G.nnx && C.nd[C.idx(l, k + 1)].s == -1) c.s = 1;
            }
        // second pass (urg = 2): the narrow band from the resampled grid, in the
        // reference's scan order (fmm.f90:188-195)
        for (int i = g.vnl; i <= g.vnr; ++i)
            for (int j = g.vnt; j <= g.vnb; ++j) {
                const int n = C.idx(j, i);
                if (C.nd[n].s > 0) C.addtree(March::pack(j, i), C.nd[n].t);
            }
    }
    group_sync();
    run(C, false);
    if (!lead) return;
    g.ntr_max = C.ntr_max;
    fm_atomic_max(n_overflow + 1, (unsigned int)C.ntr_max);
    if (R.overflow || C.overflow) {
        g.status = SWDK_FMST_BAND_OVERFLOW;
        fm_atomic_add(n_overflow, 1u);
    }
    S.geo[p] = g;
}


// Velocity of node (idm1, idm2) of a pair's refined source grid
// (fmm.f90:877-944 bsplrefine): the node is fine-fine node (st1, st2) of the
// B-spline cell (i, j) that contains it.
FM_HD FM_INLINE float refine_node(const double* map, const Grid& G, const PairGeo& g, int idm1, int idm2) {
    const int nrxr = GDX * SGDL, nrzr = GDZ * SGDL;
    const int origx = (g.vnl - 1) * SGDL + 1, origz = (g.vnt - 1) * SGDL + 1;
    const int st1 = idm1 + origz - 1, st2 = idm2 + origx - 1;
    int i = (st1 - 1) / nrzr + 1;
    if (i > G.nvz - 1) i = G.nvz - 1;
    const int k = st1 - nrzr * (i - 1);
    int j = (st2 - 1) / nrxr + 1;
    if (j > G.nvx - 1) j = G.nvx - 1;
    const int l = st2 - nrxr * (j - 1);
    float ui[4], vi[4];
    basis((float)(l - 1) / (float)nrxr, ui);
    basis((float)(k - 1) / (float)nrzr, vi);
    float sum[4];
#pragma unroll
    for (int i1 = 0; i1 < 4; ++i1) {
        sum[i1] = 0.0f;
#pragma unroll
        for (int j1 = 0; j1 < 4; ++j1) sum[i1] = sum[i1] + ui[j1] * velv(map, G.nx, i - 1 + i1, j - 1 + j1);
        sum[i1] = vi[i1] * sum[i1];
    }
    return sum[0] + sum[1] + sum[2] + sum[3];
}

struct RayIn {
    const FNode* coarse;  // the pair's propagation grid after marching
    const FNode* fine;    // its refined grid
    const float* veln;    // phase velocities (srtimes)
    const float* velg;    // group velocities (rays)
};

// bilinear velocity of the group grid at (px, pz) from cell (ipx, ipz) (fmst.f90:794-805)
FM_HD FM_INLINE float vel_at(const Grid& G, const float* velg, float px, float pz, int ipx, int ipz) {
    float drx = (px - G.gox) - (float)(ipx - 1) * G.dnx;
    float drz = (pz - G.goz) - (float)(ipz - 1) * G.dnz;
    float vel = 0.0f;
#pragma unroll
    for (int l = 1; l <= 2; ++l)
#pragma unroll
        for (int m = 1; m <= 2; ++m) {
            float produ = (1.0f - fabsf(((float)(m - 1) * G.dnz - drz) / G.dnz));
            produ = produ * (1.0f - fabsf(((float)(l - 1) * G.dnx - drx) / G.dnx));
            int iz = ipz - 1 + m, ix = ipx - 1 + l;
            if (iz <= G.nnz && ix <= G.nnx && iz >= 1 && ix >= 1)
                vel = vel + velg[(iz - 1) + (size_t)(ix - 1) * G.nnz] * produ;
        }
    return vel;
}

// fmm.f90:951-1078
FM_HD float srtimes(const Grid& G, const RayIn& in, const PairGeo& g, float scx, float scz, float rcx1,
                         float rcz1, float sin_rcx1) {
    int irx = (int)((rcx1 - G.gox) / G.dnx) + 1;
    int irz = (int)((rcz1 - G.goz) / G.dnz) + 1;
    if (irx == G.nnx) irx -= 1;
    if (irz == G.nnz) irz -= 1;
    int sw = 0;
    float sred = sq((scx - rcx1) * EARTH);
    sred = sred + sq((scz - rcz1) * EARTH * sin_rcx1);
    sred = sqrtf(sred);
    if (sred < G.dpl) sw = 1;
    if (g.isx == irx && g.isz == irz) sw = 1;
    auto T = [&](int iz, int ix) { return in.coarse[(iz - 1) + (size_t)(ix - 1) * G.nnz].t; };
    auto V = [&](int iz, int ix) { return in.veln[(iz - 1) + (size_t)(ix - 1) * G.nnz]; };
    if (sw == 1) {
        float vss[2][2];
        for (int k = 1; k <= 2; ++k)
            for (int l = 1; l <= 2; ++l) vss[k - 1][l - 1] = V(g.isz - 1 + l, g.isx - 1 + k);
        float drx = (scx - G.gox) - (float)(g.isx - 1) * G.dnx;
        float drz = (scz - G.goz) - (float)(g.isz - 1) * G.dnz;
        float vels = bilinear(vss, drx, drz, G.dnx, G.dnz);
        for (int k = 1; k <= 2; ++k)
            for (int l = 1; l <= 2; ++l) vss[k - 1][l - 1] = V(irz - 1 + l, irx - 1 + k);
        drx = (rcx1 - G.gox) - (float)(irx - 1) * G.dnx;
        drz = (rcz1 - G.goz) - (float)(irz - 1) * G.dnz;
        float velr = bilinear(vss, drx, drz, G.dnx, G.dnz);
        return 2.0f * sred / (vels + velr);
    }
    float drx = (rcx1 - G.gox) - (float)(irx - 1) * G.dnx;
    float drz = (rcz1 - G.goz) - (float)(irz - 1) * G.dnz;
    float trr = 0.0f;
    for (int k = 1; k <= 2; ++k)
        for (int l = 1; l <= 2; ++l) {
            float produ = (1.0f - fabsf(((float)(l - 1) * G.dnz - drz) / G.dnz)) *
                          (1.0f - fabsf(((float)(k - 1) * G.dnx - drx) / G.dnx));
            trr = trr + T(irz - 1 + l, irx - 1 + k) * produ;
        }
    return trr;
}


// src/shared/spherical.cpp:9-27
FM_HD FM_INLINE float delsph(float colatrad1, float lonrad1, float colatrad2, float lonrad2) {
    const float R = 6371.0f;
    float dlat = colatrad2 - colatrad1;
    float dlon = lonrad2 - lonrad1;
    float lat1 = __double2float_rn(M_PI * 0.5 - (double)colatrad1);
    float lat2 = __double2float_rn(M_PI * 0.5 - (double)colatrad2);
    double s1 = sin((double)dlat * 0.5), s2 = sin((double)dlon * 0.5);
    float a = __double2float_rn(s1 * s1 + s2 * s2 * cos((double)lat1) * cos((double)lat2));
    float c = __double2float_rn(2.0 * atan2(sqrt((double)a), sqrt((double)(1.0f - a))));
    return R * c;
}

// fmst.f90:350-976 for one receiver: returns tsyn; fdm (if not null) gets the
// (nx, ny) column-major weights, accumulated in the reference's order.
// sin_f(x) gives sin(colatitude) of a ray point (the reference: the C
// library's sinf); sin_rcx is that of the receiver.
template <class Sin>
FM_HD float raypath(const Grid& G, const RayIn& in, const PairGeo& g, float scx, float scz, float rcx, float rcz,
                    float sin_rcx, float* fdm, int* status, Sin sin_f) {
    const float dpl = 0.5f * G.dpl;
    const float dnxr = G.drnx, dnzr = G.drnz, goxr = g.gorx, gozr = g.gorz;
    const int nnxr = g.nrnx, nnzr = g.nrnz;
    auto TT = [&](int iz, int ix) { return in.coarse[(iz - 1) + (size_t)(ix - 1) * G.nnz].t; };
    auto TR = [&](int iz, int ix) { return in.fine[(iz - 1) + (size_t)(ix - 1) * RMAX].t; };
    auto SR = [&](int iz, int ix) { return in.fine[(iz - 1) + (size_t)(ix - 1) * RMAX].s; };
    const int isx = (int)((scx - goxr) / dnxr) + 1;
    const int isz = (int)((scz - gozr) / dnzr) + 1;
    int ipx = (int)((rcx - G.gox) / G.dnx) + 1;
    int ipz = (int)((rcz - G.goz) / G.dnz) + 1;
    if (ipx < 1 || ipx >= G.nnx || ipz < 1 || ipz >= G.nnz) {
        *status = SWDK_FMST_RECEIVER_OUTSIDE;
        return __int_as_float(0x7fc00000);
    }
    float px = rcx, pz = rcz;  // rgx(j), rgz(j)
    float sin_px = sin_rcx;
    int sw = 0;
    float sred = sq((scx - px) * EARTH);
    sred = sred + sq((scz - pz) * EARTH * sin_px);
    sred = sqrtf(sred);
    if (sred < 2.0f * dpl) sw = 1;
    auto in_refined = [&](float qx, float qz, int& ixr, int& izr) {
        ixr = (int)((qx - goxr) / dnxr) + 1;
        izr = (int)((qz - gozr) / dnzr) + 1;
        if (ixr < 1 || ixr >= nnxr || izr < 1 || izr >= nnzr) return 0;
        if (SR(izr, ixr) != 0 || SR(izr + 1, ixr) != 0) return 0;
        if (SR(izr, ixr + 1) != 0 || SR(izr + 1, ixr + 1) != 0) return 0;
        return 1;
    };
    int ipxr, ipzr;
    int igref = in_refined(rcx, rcz, ipxr, ipzr);
    if (sw == 0 && igref == 1 && ipxr == isx && ipzr == isz) sw = 1;
    float tsyn = 0.0f;
    // traveltime along the ray (fmst.f90:916-946), accumulated segment by
    // segment once both ends are final
    auto seg_time = [&](float ax, float az, float bx, float bz) {
        float dinc = delsph(ax, az, bx, bz);
        int ipxo = (int)((ax - G.gox) / G.dnx) + 1, ipzo = (int)((az - G.goz) / G.dnz) + 1;
        float velo = vel_at(G, in.velg, ax, az, ipxo, ipzo);
        ipxo = (int)((bx - G.gox) / G.dnx) + 1;
        ipzo = (int)((bz - G.goz) / G.dnz) + 1;
        float vel = vel_at(G, in.velg, bx, bz, ipxo, ipzo);
        tsyn = tsyn + dinc * 0.5f * (1.0f / vel + 1.0f / velo);
    };
    if (sw == 1) {
        seg_time(px, pz, scx, scz);
        return tsyn;
    }
    const long maxrp = (long)G.nnx * G.nnz;
    for (long j = 1; j <= maxrp; ++j) {
        float dtx, dtz;
        if (igref == 1) {
            dtx = TR(ipzr, ipxr + 1) - TR(ipzr, ipxr);
            dtx = dtx + TR(ipzr + 1, ipxr + 1) - TR(ipzr + 1, ipxr);
            dtx = dtx / (2.0f * EARTH * dnxr);
            dtz = TR(ipzr + 1, ipxr) - TR(ipzr, ipxr);
            dtz = dtz + TR(ipzr + 1, ipxr + 1) - TR(ipzr, ipxr + 1);
            dtz = dtz / (2.0f * EARTH * sin_px * dnzr);
        } else {
            dtx = TT(ipz, ipx + 1) - TT(ipz, ipx);
            dtx = dtx + TT(ipz + 1, ipx + 1) - TT(ipz + 1, ipx);
            dtx = dtx / (2.0f * EARTH * G.dnx);
            dtz = TT(ipz + 1, ipx) - TT(ipz, ipx);
            dtz = dtz + TT(ipz + 1, ipx + 1) - TT(ipz, ipx + 1);
            dtz = dtz / (2.0f * EARTH * sin_px * G.dnz);
        }
        const float rd1 = sqrtf(sq(dtx) + sq(dtz));
        float nx_ = px - dpl * dtx / (EARTH * rd1);
        float nz_ = pz - dpl * dtz / (EARTH * sin_px * rd1);
        const int ipxo = ipx, ipzo = ipz;
        igref = in_refined(nx_, nz_, ipxr, ipzr);
        ipx = (int)((nx_ - G.gox) / G.dnx) + 1;
        ipz = (int)((nz_ - G.goz) / G.dnz) + 1;
        const float sin_n = sin_f(nx_);
        sred = sq((scx - nx_) * EARTH);
        sred = sred + sq((scz - nz_) * EARTH * sin_n);
        sred = sqrtf(sred);
        sw = 0;
        if (sred < 2.0f * dpl) sw = 1;
        if (sw == 0 && igref == 1 && ipxr == isx && ipzr == isz) sw = 1;
        float sin_next = sin_n;
        if (ipx < 1) { nx_ = G.gox; ipx = 1; sin_next = sin_f(nx_); }
        if (ipx >= G.nnx) { nx_ = G.gox + (float)(G.nnx - 1) * G.dnx; ipx = G.nnx - 1; sin_next = sin_f(nx_); }
        if (ipz < 1) { nz_ = G.goz; ipz = 1; }
        if (ipz >= G.nnz) { nz_ = G.goz + (float)(G.nnz - 1) * G.dnz; ipz = G.nnz - 1; }
        // the clamped point's refined-grid flag stays as computed above (fmst.f90:616-665)
        if (fdm) {
            // Frechet weights of segment (px,pz) -> (nx_,nz_) (fmst.f90:734-906)
            const int ivx = (ipx - 1) / GDX + 1, ivz = (ipz - 1) / GDZ + 1;
            const int ivxo = (ipxo - 1) / GDX + 1, ivzo = (ipzo - 1) / GDZ + 1;
            int nhp = 0, chp[3];
            float vrat[3];
            if (ivx != ivxo) {
                nhp = nhp + 1;
                float xi = (ivx > ivxo) ? G.gox + (float)(ivx - 1) * G.dvx : G.gox + (float)ivx * G.dvx;
                vrat[nhp - 1] = (xi - px) / (nx_ - px);
                chp[nhp - 1] = 1;
            }
            if (ivz != ivzo) {
                nhp = nhp + 1;
                float zi = (ivz > ivzo) ? G.goz + (float)(ivz - 1) * G.dvz : G.goz + (float)ivz * G.dvz;
                float r = (zi - pz) / (nz_ - pz);
                if (nhp == 1) { vrat[0] = r; chp[0] = 2; }
                else if (r >= vrat[nhp - 2]) { vrat[nhp - 1] = r; chp[nhp - 1] = 2; }
                else {
                    vrat[nhp - 1] = vrat[nhp - 2];
                    chp[nhp - 1] = chp[nhp - 2];
                    vrat[nhp - 2] = r;
                    chp[nhp - 2] = 2;
                }
            }
            nhp = nhp + 1;
            vrat[nhp - 1] = 1.0f;
            chp[nhp - 1] = 0;
            float vel = vel_at(G, in.velg, px, pz, ipxo, ipzo);
            float vi[4], wi[4], vio[4], wio[4];
            basis(((px - G.gox) - (float)(ivxo - 1) * G.dvx) / G.dvx, vi);
            basis(((pz - G.goz) - (float)(ivzo - 1) * G.dvz) / G.dvz, wi);
            int ivxt = ivxo, ivzt = ivzo;
            for (int k = 1; k <= nhp; ++k) {
                const float velo = vel;
#pragma unroll
                for (int q = 0; q < 4; ++q) { vio[q] = vi[q]; wio[q] = wi[q]; }
                if (k > 1) {
                    if (chp[k - 2] == 1) ivxt = ivx;
                    else if (chp[k - 2] == 2) ivzt = ivz;
                }
                const float rigz = pz + vrat[k - 1] * (nz_ - pz);
                const float rigx = px + vrat[k - 1] * (nx_ - px);
                const int ipxt = (int)((rigx - G.gox) / G.dnx) + 1;
                const int ipzt = (int)((rigz - G.goz) / G.dnz) + 1;
                vel = vel_at(G, in.velg, rigx, rigz, ipxt, ipzt);
                basis(((rigx - G.gox) - (float)(ivxt - 1) * G.dvx) / G.dvx, vi);
                basis(((rigz - G.goz) - (float)(ivzt - 1) * G.dvz) / G.dvz, wi);
                const float dinc = (k == 1) ? vrat[k - 1] * dpl : (vrat[k - 1] - vrat[k - 2]) * dpl;
                if (ivzt < 1 || ivzt > G.nvz - 1 || ivxt < 1 || ivxt > G.nvx - 1) continue;  // cannot happen
#pragma unroll
                for (int l = 1; l <= 4; ++l)
#pragma unroll
                    for (int m = 1; m <= 4; ++m) {
                        float r1 = vi[m - 1] * wi[l - 1] / sq(vel);
                        float r2 = vio[m - 1] * wio[l - 1] / sq(velo);
                        r1 = -(r1 + r2) * dinc / 2.0f;
                        float* f = fdm + (size_t)(ivxt - 2 + m) + (size_t)(ivzt - 2 + l) * G.nx;
                        *f = r1 + *f;
                    }
            }
        }
        seg_time(px, pz, nx_, nz_);
        px = nx_;
        pz = nz_;
        sin_px = sin_next;
        if (sw == 1) {
            seg_time(px, pz, scx, scz);
            return tsyn;
        }
    }
    *status = SWDK_FMST_RAY_UNFINISHED;
    return __int_as_float(0x7fc00000);
}

// fmst_init (fmst.f90:27-64) on the host, REAL*4 throughout.
inline Grid make_grid(int nx, int ny, float goxdf, float gozdf, float dvxdf, float dvzdf) {
    Grid G{};
    G.nx = nx;
    G.ny = ny;
    G.nvx = nx - 2;
    G.nvz = ny - 2;
    const float goxd = goxdf - dvxdf, gozd = gozdf + dvzdf;
    G.dvx = dvxdf * PI_SP / 180.0f;
    G.dvz = dvzdf * PI_SP / 180.0f;
    G.gox = (90.0f - goxd) * PI_SP / 180.0f;
    G.goz = gozd * PI_SP / 180.0f;
    G.nnx = (G.nvx - 1) * GDX + 1;
    G.nnz = (G.nvz - 1) * GDZ + 1;
    G.dnx = G.dvx / (float)GDX;
    G.dnz = G.dvz / (float)GDZ;
    G.drnx = G.dvx / (float)(GDX * SGDL);
    G.drnz = G.dvz / (float)(GDZ * SGDL);
    // half the smallest cell side, as srtimes and fmst_raypath compute it (fmm.f90:1011-1015)
    volatile float dpl = G.dnx * EARTH;
    volatile float rd1 = G.dnz * EARTH * sinf(G.gox);
    if (rd1 < dpl) dpl = rd1;
    rd1 = G.dnz * EARTH * sinf(G.gox + (float)(G.nnx - 1) * G.dnx);
    if (rd1 < dpl) dpl = rd1;
    G.dpl = dpl;
    return G;
}

// r*sin(colatitude) (fouds2's risti, fmm.f90:468) of every column of the
// propagation grid and of every refined grid a source can open (left bound
// vnl = 1..nnx), with the C library's sinf as the reference calls it.
template <class Vec>
inline void make_risti(const Grid& G, Vec& risti_c, Vec& risti_r) {
    risti_c.resize(G.nnx);
    for (int ix = 1; ix <= G.nnx; ++ix) {
        volatile float arg = G.gox + (float)(ix - 1) * G.dnx;
        risti_c[ix - 1] = EARTH * sinf(arg);
    }
    risti_r.assign((size_t)G.nnx * RMAX, 0.0f);
    for (int vnl = 1; vnl <= G.nnx; ++vnl) {
        volatile float gorx = G.gox + G.dnx * (float)(vnl - 1);
        for (int ix = 1; ix <= RMAX; ++ix) {
            volatile float arg = gorx + (float)(ix - 1) * G.drnx;
            risti_r[(size_t)(vnl - 1) * RMAX + ix - 1] = EARTH * sinf(arg);
        }
    }
}

}  // namespace swdk_fmst_march
