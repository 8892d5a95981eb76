// Fast-marching traveltimes, ray paths and ray-path Frechet weights for
// batches of station pairs on the GPU.
//
// Replaces the per-pair FMST calls of SurfTime::travel_time
// (src/SWD/SurfaceWave.cpp:510-541) and SurfTime::frechet_matrix (:583-672):
// fmst_init / fmst_run / fmst_reset / fmst_raypath / fmst_finalize
// (src/SWD/fmst.f90, src/SWD/fmm.f90).  Each station pair is an independent
// fast-marching problem; the batch runs every pair of an inversion iteration
// at once:
//   k_fmst_grid     cubic B-spline dicing (fmm.f90:776-870 gridder) of the
//                   phase and group maps of every period slot the batch uses,
//                   one thread per propagation-grid node;
//   k_fmst_refvel   the refined source grid's velocities (fmm.f90:877-944
//                   bsplrefine), one thread per refined node and pair;
//   k_fmst_travel   the two fast-marching passes of fmst_run
//                   (fmst.f90:108-310: refined source grid, resampling onto
//                   the propagation grid, narrow-band completion, second pass;
//                   fmm.f90:138-332 travel, :437-610 fouds2, :618-770 the
//                   binary heap), one thread per pair;
//   k_fmst_rays     srtimes (fmm.f90:951-1078) and fmst_raypath
//                   (fmst.f90:350-976), one thread per receiver.
// The heap is the reference's binary tree with the same sift rules, so nodes
// are accepted in the same order; entries carry their node's time so a sift
// reads one 16-byte pair of children instead of two indirections.  All
// arithmetic is REAL*4 in the Fortran's order: this file is compiled with
// -fmad=false (no contraction), IEEE division and square root.  The fouds2
// factors r*sin(colatitude) come from the host's sinf in tables (the
// reference calls the C library's sinf); the ray tracer's sines, which depend
// on the ray, are sin() in double rounded to float.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "swdk.h"
#include "swdk_fmst_march.cuh"

namespace {

using namespace swdk_fmst_march;

__global__ void k_fmst_grid(Grid G, int nslot, const int32_t* __restrict__ slots, const double* __restrict__ vc,
                            const double* __restrict__ vout, float* __restrict__ veln, float* __restrict__ slwn,
                            float* __restrict__ velg) {
    const size_t N = (size_t)G.nnx * G.nnz, ncol = (size_t)G.nx * G.ny;
    const size_t total = N * nslot;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        int s = (int)(q / N);
        size_t n = q - (size_t)s * N;
        int stz = (int)(n % G.nnz) + 1, stx = (int)(n / G.nnz) + 1;
        size_t off = (size_t)slots[s] * ncol;
        const float v = dice_node(vc + off, G, stz, stx);
        veln[q] = v;
        slwn[q] = 1.0f / v;  // fouds2's slown (fmm.f90:466)
        velg[q] = dice_node(vout + off, G, stz, stx);
    }
}

// Refined source-grid velocities (fmm.f90:877-944); node (idm1, idm2) of the
// refined grid is fine-fine node (st1, st2) of the cell that contains it.
__global__ void k_fmst_refvel(Grid G, int npair, const int32_t* __restrict__ cp, const float* __restrict__ srcx,
                              const float* __restrict__ srcz, const int32_t* __restrict__ pslot,
                              const int32_t* __restrict__ slots, const double* __restrict__ vc,
                              float* __restrict__ rvel, float* __restrict__ rslw, PairGeo* __restrict__ geo) {
    const int p = blockIdx.y;  // pair of the chunk; cp[p] is its index in the batch
    if (p >= npair) return;
    const int gp = cp[p];
    const PairGeo g = pair_geometry(G, srcx[gp], srcz[gp]);
    if (blockIdx.x == 0 && threadIdx.x == 0) geo[p] = g;
    if (g.status) return;
    const double* map = vc + (size_t)slots[pslot[gp]] * G.nx * G.ny;
    float* out = rvel + (size_t)p * RMAX * RMAX;
    float* outs = rslw + (size_t)p * RMAX * RMAX;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < g.nrnx * g.nrnz; q += gridDim.x * blockDim.x) {
        const int idm1 = q % g.nrnz + 1, idm2 = q / g.nrnz + 1;
        const float v = refine_node(map, G, g, idm1, idm2);
        out[(idm1 - 1) + (size_t)(idm2 - 1) * RMAX] = v;
        outs[(idm1 - 1) + (size_t)(idm2 - 1) * RMAX] = 1.0f / v;
    }
}

// fmst.f90:108-310: each warp marches `lanes / per` pairs at a time, `per`
// lanes per pair (1: one lane solves all four neighbours of an accepted
// node; 4: four lanes solve one each, lane 0 of the four owns the heap; 8:
// lane 0 owns the heap and lanes 1-4 solve), and
// loops over the pairs; the grid holds the number of warps per SM that keeps
// the marching fronts in L1.
__global__ void __launch_bounds__(128) k_fmst_travel(Grid G, int npair, int lanes, int per,
                                                     const int32_t* __restrict__ cp, const float* __restrict__ srcx,
                                                     const float* __restrict__ srcz, const int32_t* __restrict__ pslot,
                                                     const float* __restrict__ slwn, const float* __restrict__ risti_c,
                                                     const float* __restrict__ risti_r, Scratch S,
                                                     unsigned int* __restrict__ n_overflow, int smem_cap) {
    extern __shared__ __align__(16) FHeap sheap[];
    const int lane = threadIdx.x & 31;
    if (lane >= lanes) return;
    const int ppw = lanes / per, slot = lane / per;
    const int g4 = lane % per;        // lane within the pair's group
    if (per == 8 && g4 > 4) return;   // groups of eight use five lanes
    const unsigned gmask = per == 1 ? (1u << lane) : per == 4 ? (0xFu << (lane & ~3)) : (0x1Fu << (lane & ~7));
    // with smem_cap > 0 each pair's heap (1..smem_cap) lives in shared memory;
    // a band that outgrows it flags the pair for a second pass with the full
    // heap in global memory
    FHeap* hp = smem_cap > 0 ? sheap + (size_t)(((threadIdx.x >> 5) * ppw + slot) * ((smem_cap + 2) & ~1)) : nullptr;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;; warp += nwarps) {
        const int p = warp * ppw + slot;
        if (p >= npair) return;  // the same for the lanes of one pair
        march_pair(G, p, cp[p], srcx, srcz, pslot, slwn, risti_c, risti_r, S, n_overflow, hp, smem_cap,
                   per == 1 ? 0 : per == 4 ? 2 : 3, g4, gmask);
    }
}

// statuses of the chunk's propagation grids to far
__global__ void k_fmst_clear(FNode* __restrict__ nd, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        nd[i] = FNode{0.0f, -1};
}

// sin(colatitude) of a moving ray point on the device: sin in double,
// rounded to float (the C library's sinf, which the reference calls, is off
// by one ulp from that for about 1 % of arguments)
struct DeviceSin {
    __device__ float operator()(float x) const { return __double2float_rn(sin((double)x)); }
};

__global__ void k_fmst_rays(Grid G, int nrc, const int32_t* __restrict__ cr, const int32_t* __restrict__ crq,
                            const int32_t* __restrict__ cp, const float* __restrict__ srcx,
                            const float* __restrict__ srcz,
                            const int32_t* __restrict__ pslot, const int32_t* __restrict__ group,
                            const float* __restrict__ rcx, const float* __restrict__ rcz,
                            const float* __restrict__ sinr, const float* __restrict__ veln,
                            const float* __restrict__ velg, Scratch S, float* __restrict__ ttime,
                            float* __restrict__ fdm, int32_t* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrc) return;
    const int r = cr[i];    // receiver index in the batch
    const int pl = crq[i];  // its pair within the chunk
    const int p = cp[pl];   // and in the batch
    const PairGeo g = S.geo[pl];
    int st = g.status;
    float t = __int_as_float(0x7fc00000);
    float* f = fdm ? fdm + (size_t)r * G.nx * G.ny : nullptr;
    if (st == 0) {
        RayIn in;
        in.coarse = S.coarse + (size_t)pl * S.N;
        in.fine = S.fine + (size_t)pl * RMAX * RMAX;
        in.veln = veln + (size_t)pslot[p] * S.N;
        in.velg = velg + (size_t)pslot[p] * S.N;
        const float x = rcx[r], z = rcz[r];
        int irx = (int)((x - G.gox) / G.dnx) + 1, irz = (int)((z - G.goz) / G.dnz) + 1;
        if (irx < 1 || irx > G.nnx || irz < 1 || irz > G.nnz) {
            st = SWDK_FMST_RECEIVER_OUTSIDE;
        } else {
            t = srtimes(G, in, g, srcx[p], srcz[p], x, z, sinr[r]);
            if (f || group[p]) {
                float tr = raypath(G, in, g, srcx[p], srcz[p], x, z, sinr[r], f, &st, DeviceSin{});
                if (group[p]) t = tr;
            }
        }
    }
    ttime[r] = st ? __int_as_float(0x7fc00000) : t;
    status[r] = st;
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side

struct swdk_fmst {
    int device = 0;
    Grid G{};
    std::string err;
    std::vector<float> risti_c, risti_r;  // host tables
    float* d_risti_c = nullptr;
    float* d_risti_r = nullptr;
    // per-call buffers, grown on demand
    void* d_meta = nullptr;
    size_t meta_bytes = 0;
    void* h_meta = nullptr;  // pinned staging
    size_t h_meta_bytes = 0;
    cudaEvent_t meta_done = nullptr;
    float* d_grids = nullptr;
    size_t grid_bytes = 0;
    void* d_scratch = nullptr;
    size_t scratch_bytes = 0;
    unsigned int* d_overflow = nullptr;
    size_t budget = (size_t)16 << 30;
    // marching layout (measured on B200 with the 3040-pair, 33 x 36 survey):
    // 8 lanes per warp as two pairs of four lanes, 12 warps per SM, heaps of
    // 1.5 (nnx + nnz) entries in shared memory
    int lanes = 8;
    int warps_per_sm = 12; // resident marching warps per SM (0: one warp per pair group)
    int smem_heap = -1;    // heap entries per pair in shared memory (0: global heap, -1: automatic)
    int per = 4;           // lanes per pair (1 or 4)
    int nsm = 148;
    double ms_last = 0.0;
    int max_band = 0, overflow_pairs = 0;  // of the last call
    void* h_list = nullptr;                // pinned chunk lists
    size_t h_list_bytes = 0;
    void* d_list = nullptr;
    size_t list_bytes = 0;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
};

static int fail(swdk_fmst* f, const char* what, cudaError_t e) {
    f->err = std::string(what) + ": " + cudaGetErrorString(e);
    return SWDK_E_CUDA;
}

extern "C" int swdk_fmst_create(swdk_fmst** out, int device, const swdk_fmst_grid* grid) {
    if (!out || !grid) return SWDK_E_ARG;
    *out = nullptr;
    if (grid->nx < 4 || grid->ny < 4 || !(grid->dvxd > 0.0f) || !(grid->dvzd > 0.0f)) return SWDK_E_ARG;
    swdk_fmst* f = new swdk_fmst();
    f->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) { delete f; return SWDK_E_CUDA; }
    cudaDeviceGetAttribute(&f->nsm, cudaDevAttrMultiProcessorCount, device);
    cudaFuncSetAttribute(k_fmst_travel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    // fmst_init (fmst.f90:27-64) and the r*sin(colatitude) tables
    f->G = make_grid(grid->nx, grid->ny, grid->goxd, grid->gozd, grid->dvxd, grid->dvzd);
    make_risti(f->G, f->risti_c, f->risti_r);
    if ((e = cudaMalloc(&f->d_risti_c, f->risti_c.size() * 4)) != cudaSuccess ||
        (e = cudaMalloc(&f->d_risti_r, f->risti_r.size() * 4)) != cudaSuccess ||
        (e = cudaMemcpy(f->d_risti_c, f->risti_c.data(), f->risti_c.size() * 4, cudaMemcpyHostToDevice)) !=
            cudaSuccess ||
        (e = cudaMemcpy(f->d_risti_r, f->risti_r.data(), f->risti_r.size() * 4, cudaMemcpyHostToDevice)) !=
            cudaSuccess ||
        (e = cudaMalloc(&f->d_overflow, 2 * sizeof(unsigned int))) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&f->meta_done, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreate(&f->t0)) != cudaSuccess || (e = cudaEventCreate(&f->t1)) != cudaSuccess) {
        swdk_fmst_destroy(f);
        return SWDK_E_CUDA;
    }
    *out = f;
    return SWDK_OK;
}

extern "C" void swdk_fmst_destroy(swdk_fmst* f) {
    if (!f) return;
    cudaSetDevice(f->device);
    cudaDeviceSynchronize();
    cudaFree(f->d_risti_c);
    cudaFree(f->d_risti_r);
    cudaFree(f->d_meta);
    cudaFree(f->d_grids);
    cudaFree(f->d_scratch);
    cudaFree(f->d_overflow);
    if (f->h_meta) cudaFreeHost(f->h_meta);
    if (f->h_list) cudaFreeHost(f->h_list);
    cudaFree(f->d_list);
    if (f->meta_done) cudaEventDestroy(f->meta_done);
    if (f->t0) cudaEventDestroy(f->t0);
    if (f->t1) cudaEventDestroy(f->t1);
    delete f;
}

extern "C" const char* swdk_fmst_last_error(const swdk_fmst* f) { return f ? f->err.c_str() : "null handle"; }

extern "C" int swdk_fmst_set_options(swdk_fmst* f, size_t scratch_budget_bytes, int lanes_per_warp,
                                     int warps_per_sm, int smem_heap_entries, int lanes_per_pair) {
    if (!f || lanes_per_warp < 1 || lanes_per_warp > 32 || warps_per_sm < 0 || warps_per_sm > 64 ||
        smem_heap_entries < -1 || (lanes_per_pair != 1 && lanes_per_pair != 4 && lanes_per_pair != 8) ||
        lanes_per_warp % lanes_per_pair ||
        (size_t)(lanes_per_warp / lanes_per_pair) * ((smem_heap_entries + 2) & ~1) * sizeof(FHeap) > 200 * 1024)
        return SWDK_E_ARG;
    f->smem_heap = smem_heap_entries;
    f->per = lanes_per_pair;
    if (scratch_budget_bytes) f->budget = scratch_budget_bytes;
    f->lanes = lanes_per_warp;
    f->warps_per_sm = warps_per_sm;
    return SWDK_OK;
}

extern "C" int swdk_fmst_info(const swdk_fmst* f, int* nnx, int* nnz, double* ms_last, int* max_band,
                              int* overflow_pairs) {
    if (!f) return SWDK_E_ARG;
    if (nnx) *nnx = f->G.nnx;
    if (nnz) *nnz = f->G.nnz;
    if (ms_last) *ms_last = f->ms_last;
    if (max_band) *max_band = f->max_band;
    if (overflow_pairs) *overflow_pairs = f->overflow_pairs;
    return SWDK_OK;
}

static int grow(swdk_fmst* f, void** p, size_t* have, size_t need) {
    if (*have >= need) return SWDK_OK;
    cudaFree(*p);
    *p = nullptr;
    *have = 0;
    cudaError_t e = cudaMalloc(p, need);
    if (e != cudaSuccess) return fail(f, "cudaMalloc", e);
    *have = need;
    return SWDK_OK;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// makes the handle's device current for the scope of a call and restores the
// caller's current device on every return path
struct DeviceScope {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceScope(int device) {
        err = cudaGetDevice(&prev);
        if (err == cudaSuccess && prev != device) err = cudaSetDevice(device);
        else if (err == cudaSuccess) prev = -1;  // already current: nothing to restore
    }
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

extern "C" int swdk_fmst_pairs(swdk_fmst* f, int npairs, const int32_t* slot, const float* srcx, const float* srcz,
                               const int32_t* group, const int64_t* rcv_ptr, const float* rcx, const float* rcz,
                               const double* d_vc, const double* d_vout, int kmax, float* d_ttime, float* d_fdm,
                               int32_t* d_status, void* stream) {
    if (!f || npairs < 0 || !slot || !srcx || !srcz || !group || !rcv_ptr || !rcx || !rcz || !d_vc || !d_vout ||
        !d_ttime || !d_status || kmax < 1)
        return SWDK_E_ARG;
    if (npairs == 0) return SWDK_OK;
    DeviceScope dev(f->device);
    if (dev.err != cudaSuccess) return fail(f, "cudaSetDevice", dev.err);
    cudaStream_t st = (cudaStream_t)stream;
    const Grid& G = f->G;
    const int64_t nrcv = rcv_ptr[npairs];
    if (rcv_ptr[0] != 0 || nrcv < 0 || nrcv > INT32_MAX) return SWDK_E_ARG;
    for (int p = 0; p < npairs; ++p)
        if (slot[p] < 0 || slot[p] >= kmax || rcv_ptr[p + 1] < rcv_ptr[p]) return SWDK_E_ARG;
    // distinct period slots (compact index per pair)
    std::vector<int32_t> used, pslot(npairs);
    {
        std::vector<int32_t> map(kmax, -1);
        for (int p = 0; p < npairs; ++p) {
            if (map[slot[p]] < 0) { map[slot[p]] = (int32_t)used.size(); used.push_back(slot[p]); }
            pslot[p] = map[slot[p]];
        }
    }
    // metadata: one pinned staging buffer, one copy
    const size_t o_used = 0, o_pslot = align256(o_used + used.size() * 4), o_srcx = align256(o_pslot + npairs * 4),
                 o_srcz = align256(o_srcx + npairs * 4), o_group = align256(o_srcz + npairs * 4),
                 o_rcx = align256(o_group + npairs * 4), o_rcz = align256(o_rcx + nrcv * 4),
                 o_sinr = align256(o_rcz + nrcv * 4), meta = align256(o_sinr + nrcv * 4);
    cudaError_t e;
    if ((e = cudaEventSynchronize(f->meta_done)) != cudaSuccess) return fail(f, "event", e);
    if (f->h_meta_bytes < meta) {
        if (f->h_meta) cudaFreeHost(f->h_meta);
        f->h_meta = nullptr;
        f->h_meta_bytes = 0;
        if ((e = cudaMallocHost(&f->h_meta, meta)) != cudaSuccess) return fail(f, "cudaMallocHost", e);
        f->h_meta_bytes = meta;
    }
    if (int rc = grow(f, &f->d_meta, &f->meta_bytes, meta)) return rc;
    char* h = (char*)f->h_meta;
    std::memcpy(h + o_used, used.data(), used.size() * 4);
    std::memcpy(h + o_pslot, pslot.data(), npairs * 4);
    std::memcpy(h + o_srcx, srcx, npairs * 4);
    std::memcpy(h + o_srcz, srcz, npairs * 4);
    std::memcpy(h + o_group, group, npairs * 4);
    std::memcpy(h + o_rcx, rcx, nrcv * 4);
    std::memcpy(h + o_rcz, rcz, nrcv * 4);
    {  // sin(colatitude) of each receiver with the C library's sinf, as the reference
        float* sr = (float*)(h + o_sinr);
        for (int64_t r = 0; r < nrcv; ++r) sr[r] = sinf(rcx[r]);
    }
    if ((e = cudaMemcpyAsync(f->d_meta, f->h_meta, meta, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return fail(f, "metadata copy", e);
    cudaEventRecord(f->meta_done, st);
    char* d = (char*)f->d_meta;
    const int32_t* d_used = (const int32_t*)(d + o_used);
    const int32_t* d_pslot = (const int32_t*)(d + o_pslot);
    const float* d_srcx = (const float*)(d + o_srcx);
    const float* d_srcz = (const float*)(d + o_srcz);
    const int32_t* d_group = (const int32_t*)(d + o_group);
    const float* d_rcx = (const float*)(d + o_rcx);
    const float* d_rcz = (const float*)(d + o_rcz);
    const float* d_sinr = (const float*)(d + o_sinr);

    f->max_band = 0;
    f->overflow_pairs = 0;
    cudaEventRecord(f->t0, st);

    // diced phase and group grids of the slots in use
    const size_t N = (size_t)G.nnx * G.nnz;
    void* gptr = f->d_grids;
    if (int rc = grow(f, &gptr, &f->grid_bytes, 3 * N * used.size() * 4)) return rc;
    f->d_grids = (float*)gptr;
    float* veln = f->d_grids;
    float* velg = f->d_grids + N * used.size();
    float* slwn = f->d_grids + 2 * N * used.size();
    {
        size_t total = N * used.size();
        int blocks = (int)std::min<size_t>((total + 255) / 256, (size_t)f->nsm * 16);
        k_fmst_grid<<<blocks, 256, 0, st>>>(G, (int)used.size(), d_used, d_vc, d_vout, veln, slwn, velg);
    }
    if (d_fdm) cudaMemsetAsync(d_fdm, 0, (size_t)nrcv * G.nx * G.ny * 4, st);

    // Chunks of pairs within the scratch budget: a first pass with a heap
    // sized for ordinary fronts (or in shared memory), then the reference's
    // full heap for every pair whose narrow band outgrew it.  A chunk is a
    // list of pairs and of their receivers, so the second pass runs all its
    // pairs together.
    const size_t full_cap = (size_t)std::lround(0.5f * (float)(G.nnx * G.nnz));
    std::vector<int> todo(npairs);
    for (int p = 0; p < npairs; ++p) todo[p] = p;
    // automatic shared-memory heap: 1.5 (nnx + nnz) entries (a narrow band
    // is a front across the grid), within 160 KB of shared memory per SM
    int smem_heap = f->smem_heap;
    if (smem_heap < 0) {
        const int pairs_per_sm = std::max(1, (f->warps_per_sm > 0 ? f->warps_per_sm : 16) * (f->lanes / f->per));
        smem_heap = (int)std::min<size_t>((size_t)(1.5 * (G.nnx + G.nnz)), (160u << 10) / (8u * pairs_per_sm) - 2);
        if (smem_heap < 256) smem_heap = 0;
    }
    for (int pass = 0; pass < 2 && !todo.empty(); ++pass) {
        const bool smem = pass == 0 && smem_heap > 0;
        const size_t cap = smem ? std::min(full_cap, (size_t)smem_heap)
                                : pass == 0 ? std::min(full_cap, (size_t)8 * (G.nnx + G.nnz) + 1024) : full_cap;
        const size_t hstride = (cap + 2) & ~(size_t)1;
        const size_t per = align256(N * sizeof(FNode)) + align256(hstride * sizeof(FHeap)) +
                           align256((size_t)RMAX * RMAX * sizeof(FNode)) + 2 * align256((size_t)RMAX * RMAX * 4) +
                           align256((size_t)(RCAP + 1) * sizeof(FHeap)) + align256(sizeof(PairGeo));
        const int P = (int)std::max<size_t>(1, std::min<size_t>({todo.size(), f->budget / per, (size_t)65535}));
        if (int rc = grow(f, &f->d_scratch, &f->scratch_bytes, per * P + 4096)) return rc;
        std::vector<int> overflowed;
        for (size_t i = 0; i < todo.size(); i += P) {
            const int np = (int)std::min<size_t>(P, todo.size() - i);
            // chunk lists: pairs (cp), receivers (cr) and each receiver's pair in the chunk (crq)
            int64_t nrc = 0;
            for (int q = 0; q < np; ++q) nrc += rcv_ptr[todo[i + q] + 1] - rcv_ptr[todo[i + q]];
            const size_t lbytes = align256((size_t)np * 4) + 2 * align256((size_t)nrc * 4);
            if (f->h_list_bytes < lbytes) {
                if (f->h_list) cudaFreeHost(f->h_list);
                f->h_list = nullptr;
                f->h_list_bytes = 0;
                if ((e = cudaMallocHost(&f->h_list, lbytes)) != cudaSuccess) return fail(f, "cudaMallocHost", e);
                f->h_list_bytes = lbytes;
            }
            if (int rc = grow(f, &f->d_list, &f->list_bytes, lbytes)) return rc;
            int32_t* hcp = (int32_t*)f->h_list;
            int32_t* hcr = (int32_t*)((char*)f->h_list + align256((size_t)np * 4));
            int32_t* hcq = (int32_t*)((char*)hcr + align256((size_t)nrc * 4));
            {
                int64_t k = 0;
                for (int q = 0; q < np; ++q) {
                    const int gp = todo[i + q];
                    hcp[q] = gp;
                    for (int64_t r = rcv_ptr[gp]; r < rcv_ptr[gp + 1]; ++r, ++k) {
                        hcr[k] = (int32_t)r;
                        hcq[k] = q;
                    }
                }
            }
            if ((e = cudaMemcpyAsync(f->d_list, f->h_list, lbytes, cudaMemcpyHostToDevice, st)) != cudaSuccess)
                return fail(f, "chunk list copy", e);
            const int32_t* dcp = (const int32_t*)f->d_list;
            const int32_t* dcr = (const int32_t*)((const char*)f->d_list + align256((size_t)np * 4));
            const int32_t* dcq = (const int32_t*)((const char*)dcr + align256((size_t)nrc * 4));

            char* base = (char*)f->d_scratch;
            Scratch S;
            S.N = N;
            S.cap = (int)cap;
            S.hstride = (int)hstride;
            S.coarse = (FNode*)base;
            base += align256(N * sizeof(FNode) * np);
            S.heap = (FHeap*)base;
            base += align256(hstride * sizeof(FHeap) * np);
            S.fine = (FNode*)base;
            base += align256((size_t)RMAX * RMAX * sizeof(FNode) * np);
            S.rvel = (float*)base;
            base += align256((size_t)RMAX * RMAX * 4 * np);
            S.rslw = (float*)base;
            base += align256((size_t)RMAX * RMAX * 4 * np);
            S.fheap = (FHeap*)base;
            base += align256((size_t)(RCAP + 1) * sizeof(FHeap) * np);
            S.geo = (PairGeo*)base;
            cudaMemsetAsync(f->d_overflow, 0, 2 * sizeof(unsigned int), st);
            {
                size_t n = N * np;
                int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)f->nsm * 16);
                k_fmst_clear<<<blocks, 256, 0, st>>>(S.coarse, n);
            }
            k_fmst_refvel<<<dim3(8, np), 256, 0, st>>>(G, np, dcp, d_srcx, d_srcz, d_pslot, d_used, d_vc, S.rvel,
                                                      S.rslw, S.geo);
            {
                const int lanes = f->lanes, ppw = lanes / f->per;
                int warps = (np + ppw - 1) / ppw;
                if (f->warps_per_sm > 0) warps = std::min(warps, f->warps_per_sm * f->nsm);
                const size_t shm = smem ? (size_t)ppw * hstride * sizeof(FHeap) : 0;
                // shared memory only as large as the resident warps need; the rest stays L1
                int carve = 0;
                if (shm) {
                    const int wps = f->warps_per_sm > 0 ? f->warps_per_sm : 32;
                    carve = (int)std::min<size_t>(100, (shm * wps * 100 + 228 * 1024 - 1) / (228 * 1024));
                }
                cudaFuncSetAttribute(k_fmst_travel, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
                k_fmst_travel<<<warps, 32, shm, st>>>(G, np, lanes, f->per, dcp, d_srcx, d_srcz, d_pslot, slwn,
                                                      f->d_risti_c,
                                                      f->d_risti_r, S, f->d_overflow, smem ? (int)cap : 0);
            }
            if (nrc > 0)
                k_fmst_rays<<<(int)((nrc + 127) / 128), 128, 0, st>>>(G, (int)nrc, dcr, dcq, dcp, d_srcx, d_srcz,
                                                                     d_pslot, d_group, d_rcx, d_rcz, d_sinr, veln,
                                                                     velg, S, d_ttime, d_fdm, d_status);
            if ((e = cudaGetLastError()) != cudaSuccess) return fail(f, "launch", e);
            unsigned int cnt[2] = {0, 0};
            if ((e = cudaMemcpyAsync(cnt, f->d_overflow, sizeof(cnt), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
                (e = cudaStreamSynchronize(st)) != cudaSuccess)
                return fail(f, "chunk", e);
            f->max_band = std::max(f->max_band, (int)cnt[1]);
            if (cnt[0]) {
                f->overflow_pairs += (int)cnt[0];
                std::vector<PairGeo> geo(np);
                if ((e = cudaMemcpy(geo.data(), S.geo, np * sizeof(PairGeo), cudaMemcpyDeviceToHost)) != cudaSuccess)
                    return fail(f, "chunk status", e);
                for (int q = 0; q < np; ++q)
                    if (geo[q].status == SWDK_FMST_BAND_OVERFLOW) overflowed.push_back(todo[i + q]);
            }
        }
        if (pass == 0 && cap == full_cap) break;  // nothing larger to fall back to
        todo.swap(overflowed);
    }
    cudaEventRecord(f->t1, st);
    if ((e = cudaEventSynchronize(f->t1)) != cudaSuccess) return fail(f, "fmst", e);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, f->t0, f->t1);
    f->ms_last = ms;
    return SWDK_OK;
}
