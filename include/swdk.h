/*
 * swdk.h -- C-ABI of the B200 surface-wave dispersion and depth-kernel
 * engine (libswdk.so).  Plain pointers and sizes only.
 *
 * It replaces, for one call over a whole 3-D model, the per-column OpenMP
 * loops of JDSurfG's SurfTime class and the Fortran calls they make:
 *
 *   swdk_get_1d_kernel   <- SurfTime::get_1d_kernel
 *                           (src/SWD/SurfaceWave.hpp:103,
 *                            src/SWD/SurfaceWave.cpp:458-502), i.e. kernel1D
 *                           (SurfaceWave.cpp:266-412) per column with
 *                           surfdisp96_/sregn96_/sregnpu_/slegn96_/slegnpu_
 *                           (src/SWD/swd.hpp:5-96)
 *   swdk_get_2d_map      <- SurfTime::get_2d_map
 *                           (SurfaceWave.hpp:102, SurfaceWave.cpp:420-450),
 *                           i.e. disp1D (SurfaceWave.cpp:177-255)
 *   swdk_set_periods     <- the SurfTime members tRc/tRg/tLc/tLg
 *                           (SurfaceWave.hpp:86-88), (ntmax, nmode)
 *                           column-major with -1 padding as io.cpp fills them
 *   swdk_set_depth       <- SurfTime::set_model's depth (SurfaceWave.cpp:678-686)
 *   swdk_surfdisp96_batch<- surfdisp96_ (swd.hpp:78-81) over many layered
 *                           models with one period list
 *   swdk_frechet_rows    <- the row assembly of SurfTime::frechet_matrix
 *                           (SurfaceWave.cpp:630-660)
 *
 * Array layouts are Eigen's column-major ones used by the reference:
 *   vs, vp, rho      : (nx, ny, nz)       float,  element (ix,iy,iz) at ix + nx*(iy + ny*iz)
 *   vc, vout, status : (nx*ny, kmax)      double/int32, column n = ix + nx*iy
 *   kernel           : (nx*ny, nz, kmax)  double
 * kmax = total number of periods over Rc, Rg, Lc, Lg and their modes, in
 * the reference's slot order (SurfaceWave.cpp:14-48).
 *
 * Return value: 0 on success, a negative SWDK_E* code otherwise.  Per-slot
 * outcomes are in `status` (SWDK_ST_*).  A context is used from one host
 * thread at a time; calls on different contexts are independent.
 */
#ifndef SWDK_H_
#define SWDK_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* error codes */
#define SWDK_OK 0
#define SWDK_E_ARG (-1)       /* bad argument (NULL, size out of range)      */
#define SWDK_E_CUDA (-2)      /* a CUDA runtime call failed                  */
#define SWDK_E_NOPERIODS (-3) /* swdk_set_periods not called / no periods    */
#define SWDK_E_NODEPTH (-4)   /* swdk_set_depth not called or nz mismatch    */
#define SWDK_E_LIMIT (-5)     /* model beyond the compiled limits            */

/* per-slot status */
#define SWDK_ST_OK 0
#define SWDK_ST_NO_ROOT 1    /* no root after the single-period retry; the
                                reference calls exit(1) (surfdisp.cpp:100-108) */
#define SWDK_ST_RETRIED 2    /* found by that retry (surfdisp.cpp:94-99)     */
#define SWDK_ST_NAN_INPUT 3  /* column has non-finite or invalid values     */
#define SWDK_ST_ITER_LIMIT 4 /* refinement hit its iteration cap            */

/* root refinement */
#define SWDK_REFINE_REFERENCE 0 /* surfdisp96 nevill: |c1-c2| <= 1e-6*c1     */
#define SWDK_REFINE_TIGHT 1     /* Brent on the same bracket, width <= rtol*c */

/* compiled limits */
#define SWDK_MAX_NZ 80          /* grid nodes per column                   */
#define SWDK_MAX_LAYERS 320     /* sublayers per column (4*nz-3)           */
#define SWDK_MAX_PERIODS 128    /* periods per (wave type, mode) list      */

typedef struct swdk_config {
  int device;      /* CUDA device ordinal (default 0)                         */
  int refine;      /* SWDK_REFINE_* (default SWDK_REFINE_TIGHT)                */
  double rtol;     /* bracket width for SWDK_REFINE_TIGHT (default 1e-10)     */
  int sngl;        /* 1: roots rounded to REAL*4 as surfdisp96 does (default) */
  int sphere;      /* 1: spherical earth as SurfTime (default); 0: flat       */
  int block_roots; /* blocks of the persistent root kernel, 0 = occupancy
                      default (swdk_autotune sets it)                       */
  int split_cols;  /* calls with at least this many columns run as two
                      concurrent column halves on child contexts; <= 0
                      (default) = never.  Host-memory calls stream their
                      outputs back behind the eigen stage's column chunks
                      either way.                                           */
  int node_layers; /* 1 (default): the root search rebuilds each column's
                      flattened sublayers from its grid nodes and one
                      per-depth table (the same arithmetic as the layer
                      tables, 1 KB per column instead of 8 KB, so the working
                      set stays in L2); 0: it reads the full layer tables.
                      Columns with fluid nodes always use the tables.       */
} swdk_config;

typedef struct swdk_stats {
  int64_t secular_evals; /* secular-function evaluations of the last call    */
  int64_t layer_evals_rayleigh; /* sum over Rayleigh evaluations of the layers
                                   propagated (dltar4, surfdisp96.f:798-898) */
  int64_t layer_evals_love;     /* same for Love (dltar1, surfdisp96.f:734-794) */
  int32_t nchains;       /* distinct (wave, period list) root chains per column */
  int32_t nslots;        /* kmax of the last call                            */
  float ms_prep, ms_roots, ms_eigen; /* device time of the last call's stages */
  int64_t proposals_accepted;  /* learned brackets confirmed by the FP64 sign change */
  int64_t proposals_rejected;  /* learned brackets that fell back to the plain scan  */
  float ms_proposal;           /* device time of feature extraction + inference  */
  int32_t kernel_launches;     /* kernels this library launched for the call       */
  int64_t evals_by_phase[6];   /* secular evaluations by phase: [0] the scan of a
                                  mode's first period (getsol, surfdisp96.f:400-495),
                                  [1] scans of later periods, group passes and
                                  dropped proposals, [2] the learned cell's two ends,
                                  [3] walks from a learned cell, [4] the refinement
                                  (nevill / Brent), [5] single-period retries
                                  (surfdisp.cpp:94-109)                          */
} swdk_stats;

typedef struct swdk_ctx swdk_ctx;

/* Fills *cfg with the defaults listed above. */
int swdk_config_default(swdk_config* cfg);

/* Creates a context on cfg->device (cfg may be NULL for defaults). */
int swdk_create(swdk_ctx** ctx, const swdk_config* cfg);
void swdk_destroy(swdk_ctx* ctx);

/* Period tables of SurfTime (tRc, tRg, tLc, tLg); a table may be NULL with
 * ntmax = nmode = 0.  Each is (ntmax, nmode) column-major, -1 padded. */
int swdk_set_periods(swdk_ctx* ctx, const double* tRc, int ntRc, int nmRc, const double* tRg, int ntRg, int nmRg,
                     const double* tLc, int ntLc, int nmLc, const double* tLg, int ntLg, int nmLg);

/* Node depths (km) of the model grid, as SurfTime::depth. */
int swdk_set_depth(swdk_ctx* ctx, const float* depth, int nz);

/* kmax of the current period tables (number of slots per column). */
int swdk_kmax(const swdk_ctx* ctx);

/* SurfTime::get_1d_kernel over an (nx, ny, nz) model in HOST memory.
 * vp and rho may be NULL: then they follow from vs by the Brocher relations
 * like the reference; when given, they are used as node values (fluid
 * nodes: vs = 0) and the chain rule still uses the Brocher derivatives as
 * SurfaceWave.cpp:491-500 does.  status may be NULL. */
int swdk_get_1d_kernel(swdk_ctx* ctx, int nx, int ny, int nz, const float* vs, const float* vp, const float* rho,
                       double* vc, double* vout, double* kernel, int32_t* status);

/* SurfTime::get_2d_map: dispersion only (phase; group from the energy
 * integrals for Rg/Lg as groupvel_r/_l do). */
int swdk_get_2d_map(swdk_ctx* ctx, int nx, int ny, int nz, const float* vs, const float* vp, const float* rho,
                    double* vc, double* vout, int32_t* status);

/* The same two calls on DEVICE pointers (current device of the context),
 * enqueued on `stream` (a cudaStream_t, NULL = the context's stream); they
 * return once the work is enqueued. */
int swdk_get_1d_kernel_device(swdk_ctx* ctx, int nx, int ny, int nz, const float* d_vs, const float* d_vp,
                              const float* d_rho, double* d_vc, double* d_vout, double* d_kernel, int32_t* d_status,
                              void* stream);
int swdk_get_2d_map_device(swdk_ctx* ctx, int nx, int ny, int nz, const float* d_vs, const float* d_vp,
                           const float* d_rho, double* d_vc, double* d_vout, int32_t* d_status, void* stream);

/* surfdisp96_ over nmodel layered models of nlayer layers each (HOST
 * memory).  thk/vp/vs/rho are (nlayer, nmodel) column-major (model m's
 * layers contiguous), t has kmax periods, cg is (kmax, nmodel), ierr has
 * nmodel entries.  iflsph/iwave/mode/igr have surfdisp96's meaning
 * (iwave 1 Love 2 Rayleigh, mode 1 = fundamental, igr 0 phase). */
int swdk_surfdisp96_batch(swdk_ctx* ctx, int nmodel, int nlayer, const float* thk, const float* vp, const float* vs,
                          const float* rho, int iflsph, int iwave, int mode, int igr, int kmax, const double* t,
                          double* cg, int32_t* ierr);

/* Frechet rows of SurfTime::frechet_matrix from a DEVICE kernel
 * (nx*ny, nz, kmax) double: for each of nrows receivers r with period slot
 * row_slot[r] and ray weights fdm[r] ((nx, ny) float column-major), row r
 * is float(fdm(ix+1,iy+1) * kernel(ii, iz, slot)) over the interior cells
 * j = iz*(nx-2)*(ny-2) + iy*(nx-2) + ix, iz < nz-1, nonzeros kept in
 * ascending j.  Device outputs: nnz[nrows], and indices/values with row r
 * at r*(nx-2)*(ny-2)*(nz-1) (capacity per row).  Enqueued on `stream`. */
int swdk_frechet_rows_device(swdk_ctx* ctx, int nx, int ny, int nz, int kmax, const double* d_kernel, int nrows,
                             const int32_t* d_row_slot, const float* d_fdm, int32_t* d_nnz, int32_t* d_indices,
                             float* d_values, void* stream);

/* The same rows as CSR: d_rowptr[nrows+1] (int64, device) and the
 * compacted indices/values of all rows in row order (capacity entries
 * available).  Two passes: counts and their prefix sum, then the rows; the
 * total number of nonzeros is returned in *nnz_total (the call waits for the
 * count), SWDK_E_LIMIT if it exceeds capacity (call again with enough). */
int swdk_frechet_csr_device(swdk_ctx* ctx, int nx, int ny, int nz, int kmax, const double* d_kernel, int nrows,
                            const int32_t* d_row_slot, const float* d_fdm, int64_t* d_rowptr, int32_t* d_indices,
                            float* d_values, int64_t capacity, int64_t* nnz_total, void* stream);

/* surfdisp96_ for callers that cannot allocate device memory.
 *
 * No counterpart in the reference: it is swdk_surfdisp96_batch on device
 * pointers with no context and no allocation of any kind.  It is for host
 * programs that own every byte of device memory themselves -- an inversion
 * driver with a fixed, pre-reserved memory budget, or a framework whose
 * allocator must stay the only one -- and so cannot let a library call
 * cudaMalloc (or cudaFree, which also waits for the whole device) while an
 * iteration is running.
 *
 * Inputs/outputs are the caller's DEVICE memory on `device`: thk/vp/vs/rho
 * are (nlayer, nmodel) column-major floats, t has kmax doubles, cg receives
 * (kmax, nmodel) doubles (model m's periods contiguous) and ierr nmodel ints,
 * with surfdisp96's meaning; refine/rtol/sngl as in swdk_config.  The work is
 * enqueued on `stream` (a cudaStream_t; NULL = legacy default stream).
 *
 * Scratch: a file-scope __device__ array of SWDK_NOALLOC_SCRATCH_BYTES that
 * every GPU loading the library holds until the process exits.  A call needs
 * 32*nlayer*nmodel + 12*mode*kmax*nmodel bytes (plus alignment and 32 bytes
 * per model); larger calls return SWDK_E_LIMIT and do nothing.  The first
 * call on each device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current, so make that first call
 * before any stream capture.  The address is kept for the life of the
 * process: cudaDeviceReset on a device after its first call here is not
 * supported (the library's module, and with it the array, is reloaded at a
 * new address).  A CUDA error already pending on the calling thread is
 * reported as SWDK_E_CUDA before anything is launched, and left pending for
 * the caller.  All calls on one device share the array and
 * it keeps the last call's contents: calls whose GPU work overlaps (other
 * streams, other host threads) race and corrupt each other's results, so
 * serialise them.  The previously current device is restored on return. */
#define SWDK_NOALLOC_SCRATCH_BYTES (64u << 20)
int swdk_surfdisp96_noalloc(int device, int nmodel, int nlayer, const float* d_thk, const float* d_vp,
                            const float* d_vs, const float* d_rho, int iflsph, int iwave, int mode, int igr, int kmax,
                            const double* d_t, double* d_cg, int32_t* d_ierr, int refine, double rtol, int sngl,
                            void* stream);

/* ---- learned bracket proposal (no counterpart in the reference) ----------
 * A small MLP per wave type proposes each root's phase velocity c and a
 * bracket half-width; the FP64 period equation must change sign across the
 * bracket with the mode's polarity, otherwise the reference's plain scan
 * runs.  Only the tight refinement uses proposals; roots are unchanged, the
 * number of secular-function evaluations drops. */
typedef struct swdk_mlp swdk_mlp;
int swdk_mlp_create(swdk_mlp** out, int device, uint64_t seed);
void swdk_mlp_destroy(swdk_mlp* mlp);
int64_t swdk_mlp_num_params(const swdk_mlp* mlp);
int swdk_mlp_get_params(swdk_mlp* mlp, float* host, int64_t n);
int swdk_mlp_set_params(swdk_mlp* mlp, const float* host, int64_t n);
int swdk_mlp_get_grads(swdk_mlp* mlp, float* host, int64_t n);
/* d_x: (M, 320) bf16 features; d_out: (M, 2) float (mu, log sigma) */
int swdk_mlp_forward(swdk_mlp* mlp, const void* d_x, int M, float* d_out, void* stream);
/* Fused inference (all layers of a 128-row tile in one persistent tcgen05
 * kernel) straight to bracket proposals: d_prop[r] = (3.5 + mu, clamp(kappa *
 * sigma, 2e-5 c, 0.2)) as float2 for r < nrows.  d_xtiles holds the rows as
 * 128-row tile images of 320 bf16 in the 128-byte-swizzled K-major layout
 * (tile t, K-block kb of 64 columns, row r, column c at byte
 * t*81920 + kb*16384 + r*128 + (((c%64)/8 ^ r%8) * 16) + (c%8)*2), rows padded
 * to a multiple of 128.  Asynchronous on `stream`; a timed-out wait sets the
 * flag read by swdk_mlp_error_flag. */
int swdk_mlp_propose(swdk_mlp* mlp, const void* d_xtiles, int nrows, double kappa, void* d_prop, void* stream);
/* forward + Gaussian NLL + backward; Adam step when lr > 0 */
int swdk_mlp_train_step(swdk_mlp* mlp, const void* d_x, const float* d_y, int M, float lr, float* loss_out,
                        void* stream);
int swdk_mlp_save(swdk_mlp* mlp, const char* path);
int swdk_mlp_load(swdk_mlp* mlp, const char* path);
int swdk_mlp_error_flag(swdk_mlp* mlp, int* flag);
const char* swdk_mlp_last_error(const swdk_mlp* mlp);
/* C = A * B^T on the tensor cores: A (M, K), B (N, K) bf16 device, C (M, N)
 * float; M % 128 == 0, N % 64 == 0, K % 64 == 0. */
int swdk_gemm_bf16_tn(int M, int N, int K, const void* d_a, const void* d_b, float* d_c, int* d_err, void* stream);

/* Attach proposal networks (either may be NULL); kappa_* scales the
 * predicted sigma into the bracket half-width of that wave type.  From the
 * second period of a mode on, the bracket is centred on the previous
 * period's root plus the predicted change, c(k-1) + mu(k) - mu(k-1).  The
 * first period of a Rayleigh chain's first mode jumps to the cell of the
 * network's own estimate, the stretch below it checked at every fourth
 * point of the scan grid; the first period of Love chains and of higher
 * modes keeps the plain scan.  NULL/NULL disables proposals.  The networks
 * must outlive their use by this context. */
int swdk_set_proposal(swdk_ctx* ctx, swdk_mlp* rayleigh, swdk_mlp* love, double kappa_rayleigh, double kappa_love);

/* Testing aid (no counterpart in the reference): every proposed phase
 * velocity is moved by shift_km_s (|shift| <= 10) before the search; 0, the
 * default, leaves the network's proposals as they are.  A constant shift
 * leaves the anchored brackets of later periods unchanged and moves only
 * the first-period jump, whose roots must not move.  Drops a captured
 * graph. */
int swdk_set_proposal_shift(swdk_ctx* ctx, double shift_km_s);

/* Training support: root search only (all root chains of get_1d_kernel)
 * on device models, then per-slot metadata, the roots and their status, and
 * features/targets for chosen rows (row = slot * nx*ny + column). */
int swdk_roots_device(swdk_ctx* ctx, int nx, int ny, int nz, const float* d_vs, const float* d_vp, const float* d_rho,
                      void* stream);
int swdk_root_slots(swdk_ctx* ctx, int* nslots, int32_t* wave, int32_t* mode, double* period);
int swdk_last_roots(swdk_ctx* ctx, double* h_c, int32_t* h_status);
int swdk_training_rows(swdk_ctx* ctx, const int64_t* d_rows, int n, void* d_x, float* d_y, void* stream);

/* The reciprocal the secular functions use for 1/alpha, 1/beta, 1/rho and
 * 1/(rho beta^2) (hardware estimate + two Newton-Raphson steps), applied to
 * n device doubles; exported for its accuracy test. */
int swdk_recip_device(const double* d_x, double* d_r, int n, void* stream);

/* One call of the device path captured as a CUDA graph and replayed.
 * path: 0 get_1d_kernel, 1 get_2d_map, 2 root search only.  Capture first
 * runs the call once eagerly (buffers, plans, depth upload, proposal
 * networks), then records it on the context's stream; the graph keeps the
 * given device pointers, so a replay recomputes from their current
 * contents.  swdk_set_periods/set_depth/set_proposal and swdk_autotune drop
 * the graph.  Replays update no statistics. */
int swdk_graph_capture(swdk_ctx* ctx, int path, int nx, int ny, int nz, const float* d_vs, const float* d_vp,
                       const float* d_rho, double* d_vc, double* d_vout, double* d_kernel, int32_t* d_status);
int swdk_graph_launch(swdk_ctx* ctx, void* stream);

/* Many models in one CUDA graph (uneven batches: different grids, depth
 * vectors, period tables, modes).  Each model has its own context (its
 * plans and buffers) and call; the graph forks one branch per context off a
 * main stream and joins them, so small models run concurrently.  The
 * contexts must be distinct and on one device.  As swdk_graph_capture, it
 * first runs every call once eagerly.  A NULL stream launches on the
 * graph's own stream. */
typedef struct swdk_call {
  int path; /* 0 get_1d_kernel, 1 get_2d_map, 2 root search only */
  int nx, ny, nz;
  const float *d_vs, *d_vp, *d_rho;
  double *d_vc, *d_vout, *d_kernel;
  int32_t* d_status;
} swdk_call;
typedef struct swdk_graph swdk_graph;
int swdk_batch_graph_create(int n, swdk_ctx* const* ctxs, const swdk_call* calls, swdk_graph** out);
int swdk_batch_graph_launch(swdk_graph* graph, void* stream);
void swdk_batch_graph_destroy(swdk_graph* graph);

/* Ragged batch: the models of one inversion iteration (each context with
 * its own period tables and depth vector, each call with its own grid and
 * device buffers, as for swdk_batch_graph_create) computed by ONE
 * persistent root-search launch over every (model, chain, column), one
 * retry launch and one eigen launch per wave type over every (model,
 * column), after each model's column preparation and proposals.  Every call
 * has the same path and every context the same device, refine, rtol, sngl
 * and sphere.  The object keeps its own device buffers (layer models, roots)
 * and a graph of one pass.  New (uneven batches); no reference counterpart:
 * the reference runs get_1d_kernel model by model (SurfaceWave.cpp:458-502).
 *   swdk_ragged_run    : one pass enqueued on stream (NULL: the object's own
 *                        stream, waited for), statistics by swdk_ragged_stats;
 *   swdk_ragged_launch : the pass as a CUDA graph (captured on the first
 *                        call after one eager pass); inputs may change in
 *                        place between launches. */
typedef struct swdk_ragged swdk_ragged;
int swdk_ragged_create(int n, swdk_ctx* const* ctxs, const swdk_call* calls, swdk_ragged** out);
int swdk_ragged_run(swdk_ragged* batch, void* stream);
int swdk_ragged_launch(swdk_ragged* batch, void* stream);
int swdk_ragged_stats(swdk_ragged* batch, swdk_stats* out);
void swdk_ragged_destroy(swdk_ragged* batch);

/* Autotuner of the persistent root-search kernel: times the root search on
 * the given device model for 1..k resident blocks per SM (k = occupancy
 * limit) and one oversubscribed grid, keeps the fastest in the context and
 * returns it in *blocks (may be NULL). */
int swdk_autotune(swdk_ctx* ctx, int nx, int ny, int nz, const float* d_vs, const float* d_vp, const float* d_rho,
                  int* blocks);

/* The Frechet rows as the reference's row-file byte stream, built on the
 * device (replaces the record loop of SurfTime::frechet_matrix,
 * SurfaceWave.cpp:596-603, 641-659): d_out receives int32 m_header, int32 n,
 * then per row r int32 row id (d_row_ids[r], or row_id0 + r when d_row_ids
 * is NULL), int32 nnz, int32 idx[nnz], float32 val[nnz] from the CSR rows
 * (d_rowptr has m+1 entries, nnz_total = d_rowptr[m]).  The stream needs
 * 2 + 2*m + 2*nnz_total words; a smaller out_words returns SWDK_E_LIMIT. */
int swdk_frechet_records_device(int64_t m, int32_t m_header, int32_t n, const int32_t* d_row_ids, int32_t row_id0,
                                const int64_t* d_rowptr, const int32_t* d_indices, const float* d_values,
                                int64_t nnz_total, int32_t* d_out, int64_t out_words, void* stream);

/* LSMR's matrix products on the device with the CSR rows of
 * swdk_frechet_csr_device (replaces myaprod_csr, src/shared/parallel.cpp:
 * 31-115, used by LSMR in src/shared/lsmrModule_csr.f90): mode 1 y += A x,
 * mode 2 x += A^T y; A is m x n with int64 row pointers, int32 column
 * indices and FP32 values, x and y are FP64 device vectors.  Asynchronous
 * on `stream` (NULL: the legacy default stream).  Mode 2 accumulates with
 * atomics, so its summation order (last bits) varies between calls. */
int swdk_aprod_csr(int mode, int64_t m, int64_t n, const int64_t* d_rowptr, const int32_t* d_indices,
                   const float* d_values, double* d_x, double* d_y, void* stream);

/* LSMR on the device (replaces the solve of csr_matrix::lsmr_solver,
 * src/shared/csr_matrix.cpp, running src/shared/lsmrModule_csr.f90):
 * min ||A x - b||^2 + damp^2 ||x||^2 by Fong & Saunders' iteration with FP64
 * device vectors and every scalar recurrence on the device; the host reads
 * the state back every 16 iterations.  A (m x n) and its transpose (n x m,
 * each row a column of A with its entries in row order) are device CSR with
 * int64 row pointers, int32 indices and FP32 values, owned by the caller and
 * kept alive while the handle is used.  d_b (m) and d_x (n) are FP64 device
 * vectors.  istop as in the reference module: 1 ||r|| small, 2 ||A^T r||
 * small, 3 cond(A) above conlim, 4-6 the same at machine precision, 7 the
 * iteration limit; 0 when b or A^T b is zero (x = 0).  Local
 * reorthogonalization is not implemented.  The solve is the same bits on
 * every run. */
typedef struct swdk_lsmr swdk_lsmr;
typedef struct swdk_lsmr_info {
  int istop, itn;
  double normA, condA, normr, normAr, normx;
} swdk_lsmr_info;
int swdk_lsmr_create(int device, int64_t m, int64_t n, const int64_t* d_rowptr, const int32_t* d_indices,
                     const float* d_values, const int64_t* d_trowptr, const int32_t* d_tindices,
                     const float* d_tvalues, swdk_lsmr** out);
int swdk_lsmr_solve(swdk_lsmr* solver, const double* d_b, double* d_x, double damp, double atol, double btol,
                    double conlim, int itnlim, swdk_lsmr_info* info, void* stream);
void swdk_lsmr_destroy(swdk_lsmr* solver);

/* Statistics of the last get_1d_kernel / get_2d_map / surfdisp96 call. */
int swdk_get_stats(swdk_ctx* ctx, swdk_stats* out);

/* Human-readable text of the last error on this context. */
const char* swdk_last_error(const swdk_ctx* ctx);

/* ------------------------------------------------------------------------
 * Fast-marching traveltimes and ray-path Frechet weights (FMST)
 *
 * Replaces the per-pair calls fmst_init / fmst_run / fmst_reset /
 * fmst_raypath / fmst_finalize (src/SWD/SurfaceWave.hpp:8-50, implemented in
 * src/SWD/fmst.f90 and src/SWD/fmm.f90) that SurfTime::travel_time
 * (src/SWD/SurfaceWave.cpp:510-541) and SurfTime::frechet_matrix
 * (:583-672) make for every station pair, with one batched call over all
 * pairs of an inversion iteration.  Same algorithm and REAL*4 arithmetic:
 * propagation grid diced 8x from the (nx, ny) model grid, a refined grid
 * (8x finer, 8 nodes around the source) marched first, the mixed-order
 * narrow-band fast marching with the reference's binary heap, bilinear
 * receiver times, and rays traced back down the traveltime gradient with
 * cubic B-spline Frechet weights and the group-velocity traveltime.
 * ------------------------------------------------------------------------ */
typedef struct swdk_fmst swdk_fmst;

/* fmst_init's arguments (fmst.f90:9): model grid nx (latitude) x ny
 * (longitude) nodes, upper-left corner latitude goxd and longitude gozd and
 * spacings dvxd, dvzd, all in degrees (SurfTime's lat0, lon0, dlat, dlon). */
typedef struct swdk_fmst_grid {
    int nx, ny;
    float goxd, gozd, dvxd, dvzd;
} swdk_fmst_grid;

/* per-receiver status of swdk_fmst_pairs (the reference prints and STOPs
 * for the first three; its ray loop then reads an undefined point count) */
#define SWDK_FMST_SOURCE_OUTSIDE 1    /* fmst.f90:159-167 */
#define SWDK_FMST_RECEIVER_OUTSIDE 2  /* fmm.f90:1000-1007, fmst.f90:497-504 */
#define SWDK_FMST_BAND_OVERFLOW 3     /* narrow band above snb*nnx*nnz nodes */
#define SWDK_FMST_RAY_UNFINISHED 4    /* ray did not reach the source in nnx*nnz steps */

/* Handle for one model grid on `device`: the grid constants (REAL*4, as
 * fmst_init computes them) and the host-computed r*sin(colatitude) tables
 * of the propagation grid and of every refined source grid. */
int swdk_fmst_create(swdk_fmst** out, int device, const swdk_fmst_grid* grid);
void swdk_fmst_destroy(swdk_fmst* fmst);
const char* swdk_fmst_last_error(const swdk_fmst* fmst);

/* Scratch budget for the per-pair marching grids (bytes; 0 keeps the
 * current, 16 GiB by default), marching lanes per warp (1..32, a multiple of
 * lanes_per_pair; default 8), resident marching warps per SM (0..64, default
 * 12; 0 = one warp per group of pairs, all at once), heap entries per pair
 * kept in shared memory (-1 = automatic, the default: 1.5 (nnx + nnz); 0 =
 * heap in global memory; a pair whose band outgrows it is marched again with
 * the full heap) and lanes per pair (1: one lane solves the four neighbours
 * of each accepted node; 4, the default: four lanes solve one each; 8: a
 * fifth lane keeps the heap meanwhile).  None of them changes a result. */
int swdk_fmst_set_options(swdk_fmst* fmst, size_t scratch_budget_bytes, int lanes_per_warp, int warps_per_sm,
                          int smem_heap_entries, int lanes_per_pair);

/* Propagation grid size; of the last swdk_fmst_pairs: device time, the
 * largest narrow band (heap entries) and the pairs whose band outgrew the
 * first pass's heap and were marched again with the reference's full heap.
 * Any pointer may be NULL. */
int swdk_fmst_info(const swdk_fmst* fmst, int* nnx, int* nnz, double* ms_last, int* max_band, int* overflow_pairs);

/* All station pairs of one iteration.  HOST arrays (StationPair fields,
 * SurfaceWave.hpp:53-82): pair p has period slot slot[p] (get_period_index,
 * 0..kmax-1), source colatitude/longitude srcx[p], srcz[p] in radians,
 * group[p] != 0 for Rg/Lg data, and receivers rcv_ptr[p]..rcv_ptr[p+1]-1 of
 * rcx/rcz (radians).  DEVICE arrays: d_vc, d_vout are the phase and used
 * velocity maps (nx*ny, kmax) column-major (vc and vout of get_2d_map /
 * get_1d_kernel); outputs d_ttime[nrcv] (data[p.counter+i]: the receiver
 * time of fmst_run, or for Rg/Lg pairs the ray's group traveltime), d_status
 * [nrcv] (SWDK_FMST_*, NaN times where nonzero) and, if d_fdm is not NULL,
 * the ray-path weights of every receiver as (nx, ny) column-major floats at
 * d_fdm + r*nx*ny (fmst_raypath's fdm, the input of
 * swdk_frechet_csr_device).  Without d_fdm only Rg/Lg receivers trace rays,
 * as travel_time does.  Runs on `stream`; returns when the results are
 * complete. */
int swdk_fmst_pairs(swdk_fmst* fmst, int npairs, const int32_t* slot, const float* srcx, const float* srcz,
                    const int32_t* group, const int64_t* rcv_ptr, const float* rcx, const float* rcz,
                    const double* d_vc, const double* d_vout, int kmax, float* d_ttime, float* d_fdm,
                    int32_t* d_status, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SWDK_H_ */
