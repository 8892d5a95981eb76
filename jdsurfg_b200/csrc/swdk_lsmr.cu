// LSMR on the device over the Frechet rows (the damped least-squares solve
// of every inversion iteration; the reference runs src/shared/
// lsmrModule_csr.f90 through csr_matrix::lsmr_solver, with the matrix
// products of myaprod_csr, src/shared/parallel.cpp:31-115).
//
// The iteration is Fong & Saunders, "LSMR: An iterative algorithm for sparse
// least-squares problems", SIAM J. Sci. Comput. 33 (2011): Golub-Kahan
// bidiagonalization, the QR factorization of the lower bidiagonal matrix
// with the damping rotation, the second QR factorization that minimizes
// ||A^T r||, and the paper's estimates of ||r||, ||A^T r||, ||A||, cond(A)
// for the stopping rules (istop as in the reference's module).  Every
// scalar of the recurrences lives in device memory and is updated by a
// one-thread kernel, so an iteration is a fixed sequence of launches with
// no host round trip; the host reads the state back every LS_CHECK
// iterations.  Once a stopping rule fires, every kernel of the iteration
// returns at once, so the iterations queued behind it change nothing.
//
// A^T y uses the transposed matrix (built by the caller, each row of it a
// column of A with its entries in row order) and the same row kernel as
// A x, and the norms are two-stage sums over a fixed grid: the whole solve
// is the same bits on every run.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>

#include "swdk.h"

namespace {

constexpr int LS_PART = 296;    // blocks of the partial sums (two per SM of a B200)
constexpr int LS_THREADS = 256;
constexpr int LS_CHECK = 16;    // iterations queued between two reads of the state

struct LsmrState {
  // bidiagonalization and the two QR factorizations
  double alpha, beta, alpha_bar, zeta_bar, rho_prev, rho_bar_prev, c_bar, s_bar;
  // ||r|| estimate
  double beta_dd, beta_dot, rho_dot_prev, tau_tilde_prev, theta_tilde, zeta_prev, damp_sum;
  // ||A||, cond(A)
  double normA2, rho_bar_max, rho_bar_min;
  double normb, normr, normAr, normA, condA, normx;
  double damp, atol, btol, ctol;
  double c_hbar, c_x, c_h;  // this iteration's vector coefficients
  int itn, itnlim, istop, done;
};

// y = s*y + A x over the rows of A, one warp per row; s = -alpha (which 0),
// -beta (1) or 1 (2: y += A x).  (s*y) and the sum are rounded separately,
// as a scaling followed by an accumulating product would be.
__global__ void k_ls_spmv(int64_t m, const int64_t* __restrict__ rowptr, const int32_t* __restrict__ idx,
                          const float* __restrict__ val, const double* __restrict__ x, double* __restrict__ y,
                          const LsmrState* __restrict__ st, int which) {
  if (st->done || (which == 1 && !(st->beta > 0.0))) return;
  const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= m) return;
  double acc = 0.0;
  for (int64_t j = rowptr[r] + lane; j < rowptr[r + 1]; j += 32) acc += (double)val[j] * x[idx[j]];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0) {
    const double s = which == 0 ? -st->alpha : which == 1 ? -st->beta : 1.0;
    y[r] = __dadd_rn(which == 2 ? y[r] : __dmul_rn(s, y[r]), acc);
  }
}

// block sum of a fixed-order strided sum of squares: part[blockIdx.x]
__device__ void block_sum_store(double v, double* part) {
  __shared__ double sh[LS_THREADS];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = LS_THREADS / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// partial sums of a[i]^2 (skipped when `need` is false in the state)
__global__ void k_ls_partial(int64_t n, const double* __restrict__ a, double* __restrict__ part,
                             const LsmrState* __restrict__ st, int which) {
  if (st->done || (which == 1 && !(st->beta > 0.0))) return;
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += a[i] * a[i];
  block_sum_store(s, part);
}

// the norm from the partial sums: which 0 -> beta, 1 -> alpha (only after a
// step with beta > 0), 3 -> beta of the start (normb as well)
__global__ void k_ls_norm(const double* __restrict__ part, LsmrState* __restrict__ st, int which) {
  if (st->done || (which == 1 && !(st->beta > 0.0))) return;
  __shared__ double sh[512];
  double v = 0.0;
  for (int i = threadIdx.x; i < LS_PART; i += blockDim.x) v += part[i];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double nrm = sqrt(sh[0]);
    if (which == 1) st->alpha = nrm;
    else st->beta = nrm;
    if (which == 3) st->normb = nrm;
  }
}

// a /= beta (which 0) or alpha (1), when positive
__global__ void k_ls_div(int64_t n, double* __restrict__ a, const LsmrState* __restrict__ st, int which) {
  if (st->done || !(st->beta > 0.0)) return;
  const double d = which == 0 ? st->beta : st->alpha;
  if (!(d > 0.0)) return;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = a[i] / d;
}

// the state after the start vectors: beta u = b, alpha v = A^T u
__global__ void k_ls_start(LsmrState* st, double damp, double atol, double btol, double ctol, int itnlim) {
  LsmrState& s = *st;
  const double alpha = s.alpha, beta = s.beta;
  s.damp = damp; s.atol = atol; s.btol = btol; s.ctol = ctol; s.itnlim = itnlim;
  s.itn = 0; s.istop = 0;
  s.normr = beta; s.normAr = alpha * beta; s.normA = 0.0; s.condA = 1.0; s.normx = 0.0;
  s.done = (alpha * beta == 0.0) ? 1 : 0;
  s.alpha_bar = alpha; s.zeta_bar = alpha * beta;
  s.rho_prev = 1.0; s.rho_bar_prev = 1.0; s.c_bar = 1.0; s.s_bar = 0.0;
  s.beta_dd = beta; s.beta_dot = 0.0;
  s.rho_dot_prev = 1.0; s.tau_tilde_prev = 0.0; s.theta_tilde = 0.0; s.zeta_prev = 0.0;
  s.damp_sum = 0.0;
  s.normA2 = alpha * alpha;
  s.rho_bar_max = 0.0; s.rho_bar_min = 1e300;
}

// one iteration's scalar recurrences (after alpha, beta of the step)
__global__ void k_ls_scalar(LsmrState* st) {
  LsmrState& s = *st;
  if (s.done) return;
  s.itn += 1;
  const double alpha = s.alpha, beta = s.beta, damp = s.damp;
  // damping rotation on (alpha_bar, damp)
  const double alpha_hat = hypot(s.alpha_bar, damp);
  const double c_hat = s.alpha_bar / alpha_hat, s_hat = damp / alpha_hat;
  // first QR rotation
  const double rho = hypot(alpha_hat, beta);
  const double c = alpha_hat / rho, sn = beta / rho;
  const double theta_next = sn * alpha;
  s.alpha_bar = c * alpha;
  // second QR rotation
  const double theta_bar = s.s_bar * rho;
  const double rho_bar = hypot(s.c_bar * rho, theta_next);
  const double c_bar = s.c_bar * rho / rho_bar, s_bar = theta_next / rho_bar;
  s.c_bar = c_bar;
  s.s_bar = s_bar;
  const double zeta = c_bar * s.zeta_bar;
  s.zeta_bar = -s_bar * s.zeta_bar;
  // search directions and solution
  s.c_hbar = -(theta_bar * rho) / (s.rho_prev * s.rho_bar_prev);
  s.c_x = zeta / (rho * rho_bar);
  s.c_h = -(theta_next / rho);
  // ||r||: the rotations applied to the right-hand side (beta_1, 0, ...)
  const double beta_acute = c_hat * s.beta_dd;
  const double beta_check = -s_hat * s.beta_dd;
  const double beta_hat = c * beta_acute;
  s.beta_dd = -sn * beta_acute;
  const double rho_tilde = hypot(s.rho_dot_prev, theta_bar);
  const double c_t = s.rho_dot_prev / rho_tilde, s_t = theta_bar / rho_tilde;
  const double theta_tilde_old = s.theta_tilde;
  s.theta_tilde = s_t * rho_bar;
  const double rho_dot = c_t * rho_bar;
  s.beta_dot = -s_t * s.beta_dot + c_t * beta_hat;
  s.tau_tilde_prev = (s.zeta_prev - theta_tilde_old * s.tau_tilde_prev) / rho_tilde;
  const double tau_dot = (zeta - s.theta_tilde * s.tau_tilde_prev) / rho_dot;
  s.damp_sum += beta_check * beta_check;
  const double d = s.beta_dot - tau_dot;
  s.normr = sqrt(s.damp_sum + d * d + s.beta_dd * s.beta_dd);
  // ||A|| and cond(A)
  s.normA2 += beta * beta;
  s.normA = sqrt(s.normA2);
  s.normA2 += alpha * alpha;
  s.rho_bar_max = fmax(s.rho_bar_max, s.rho_bar_prev);
  if (s.itn > 1) s.rho_bar_min = fmin(s.rho_bar_min, s.rho_bar_prev);
  s.condA = fmax(s.rho_bar_max, rho_bar) / fmin(s.rho_bar_min, rho_bar);
  s.normAr = fabs(s.zeta_bar);
  s.rho_prev = rho;
  s.rho_bar_prev = rho_bar;
  s.rho_dot_prev = rho_dot;
  s.zeta_prev = zeta;
}

// h_bar = c_hbar h_bar + h; x += c_x h_bar; h = c_h h + v; partial sums of x^2
__global__ void k_ls_vec(int64_t n, double* __restrict__ x, double* __restrict__ h, double* __restrict__ hbar,
                         const double* __restrict__ v, double* __restrict__ part, const LsmrState* __restrict__ st) {
  if (st->done) return;
  const double ch = st->c_hbar, cx = st->c_x, chh = st->c_h;
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double hb = __dadd_rn(__dmul_rn(hbar[i], ch), h[i]);
    hbar[i] = hb;
    const double xi = __dadd_rn(x[i], __dmul_rn(cx, hb));
    x[i] = xi;
    h[i] = __dadd_rn(__dmul_rn(h[i], chh), v[i]);
    s += xi * xi;
  }
  block_sum_store(s, part);
}

// ||x|| and the stopping rules (the reference module's istop)
__global__ void k_ls_tests(const double* __restrict__ part, LsmrState* st) {
  if (st->done) return;
  __shared__ double sh[512];
  double v = 0.0;
  for (int i = threadIdx.x; i < LS_PART; i += blockDim.x) v += part[i];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  LsmrState& s = *st;
  s.normx = sqrt(sh[0]);
  const double test1 = s.normr / s.normb;
  const double test2 = (s.normA * s.normr > 0.0) ? s.normAr / (s.normA * s.normr) : INFINITY;
  const double test3 = 1.0 / s.condA;
  const double t1 = test1 / (1.0 + s.normA * s.normx / s.normb);
  const double rtol = s.btol + s.atol * s.normA * s.normx / s.normb;
  int istop = 0;
  if (s.itn >= s.itnlim) istop = 7;
  if (1.0 + test3 <= 1.0) istop = 6;
  if (1.0 + test2 <= 1.0) istop = 5;
  if (1.0 + t1 <= 1.0) istop = 4;
  if (test3 <= s.ctol) istop = 3;
  if (test2 <= s.atol) istop = 2;
  if (test1 <= rtol) istop = 1;
  s.istop = istop;
  s.done = istop > 0;
}

}  // namespace

struct swdk_lsmr {
  int device = 0;
  int64_t m = 0, n = 0;
  const int64_t* rowptr = nullptr;
  const int32_t* idx = nullptr;
  const float* val = nullptr;
  const int64_t* trowptr = nullptr;
  const int32_t* tidx = nullptr;
  const float* tval = nullptr;
  double *u = nullptr, *v = nullptr, *h = nullptr, *hbar = nullptr, *part = nullptr;
  LsmrState* st = nullptr;
  LsmrState* hst = nullptr;  // pinned copy read back every LS_CHECK iterations
};

namespace {

// restores the caller's current device on return
struct LsDeviceScope {
  int prev = -1;
  explicit LsDeviceScope(int d) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    cudaSetDevice(d);
  }
  ~LsDeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

void ls_free(swdk_lsmr* s) {
  for (double* p : {s->u, s->v, s->h, s->hbar, s->part})
    if (p) cudaFree(p);
  if (s->st) cudaFree(s->st);
  if (s->hst) cudaFreeHost(s->hst);
}

unsigned int ls_blocks(int64_t n, int per) { return (unsigned int)((n + per - 1) / per); }

}  // namespace

extern "C" {

int swdk_lsmr_create(int device, int64_t m, int64_t n, const int64_t* d_rowptr, const int32_t* d_indices,
                     const float* d_values, const int64_t* d_trowptr, const int32_t* d_tindices,
                     const float* d_tvalues, swdk_lsmr** out) {
  if (!out) return SWDK_E_ARG;
  *out = nullptr;
  if (device < 0 || m <= 0 || n <= 0 || !d_rowptr || !d_trowptr || m > 0x7fffffffLL * 8 || n > 0x7fffffffLL * 8)
    return SWDK_E_ARG;
  LsDeviceScope scope(device);
  swdk_lsmr* s = new (std::nothrow) swdk_lsmr();
  if (!s) return SWDK_E_CUDA;
  s->device = device;
  s->m = m; s->n = n;
  s->rowptr = d_rowptr; s->idx = d_indices; s->val = d_values;
  s->trowptr = d_trowptr; s->tidx = d_tindices; s->tval = d_tvalues;
  cudaError_t e = cudaMalloc(&s->u, (size_t)m * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&s->v, (size_t)n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&s->h, (size_t)n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&s->hbar, (size_t)n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&s->part, LS_PART * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&s->st, sizeof(LsmrState));
  if (e == cudaSuccess) e = cudaMallocHost(&s->hst, sizeof(LsmrState));
  if (e != cudaSuccess) {
    ls_free(s);
    delete s;
    return SWDK_E_CUDA;
  }
  *out = s;
  return SWDK_OK;
}

int swdk_lsmr_solve(swdk_lsmr* s, const double* d_b, double* d_x, double damp, double atol, double btol,
                    double conlim, int itnlim, swdk_lsmr_info* info, void* stream) {
  if (!s || !d_b || !d_x || itnlim < 0) return SWDK_E_ARG;
  LsDeviceScope scope(s->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t m = s->m, n = s->n;
  const unsigned int gm = ls_blocks(m * 32, LS_THREADS), gn = ls_blocks(n * 32, LS_THREADS);
  const unsigned int em = ls_blocks(m, LS_THREADS), en = ls_blocks(n, LS_THREADS);
  const double ctol = conlim > 0.0 ? 1.0 / conlim : 0.0;
  // start: beta u = b, alpha v = A^T u, x = 0, h = v, h_bar = 0
  cudaMemsetAsync(s->st, 0, sizeof(LsmrState), st);
  cudaMemcpyAsync(s->u, d_b, (size_t)m * sizeof(double), cudaMemcpyDeviceToDevice, st);
  cudaMemsetAsync(s->v, 0, (size_t)n * sizeof(double), st);
  cudaMemsetAsync(d_x, 0, (size_t)n * sizeof(double), st);
  cudaMemsetAsync(s->hbar, 0, (size_t)n * sizeof(double), st);
  k_ls_partial<<<LS_PART, LS_THREADS, 0, st>>>(m, s->u, s->part, s->st, 0);
  k_ls_norm<<<1, 512, 0, st>>>(s->part, s->st, 3);
  k_ls_div<<<em, LS_THREADS, 0, st>>>(m, s->u, s->st, 0);
  k_ls_spmv<<<gn, LS_THREADS, 0, st>>>(n, s->trowptr, s->tidx, s->tval, s->u, s->v, s->st, 2);
  k_ls_partial<<<LS_PART, LS_THREADS, 0, st>>>(n, s->v, s->part, s->st, 1);
  k_ls_norm<<<1, 512, 0, st>>>(s->part, s->st, 1);
  k_ls_div<<<en, LS_THREADS, 0, st>>>(n, s->v, s->st, 1);
  k_ls_start<<<1, 1, 0, st>>>(s->st, damp, atol, btol, ctol, itnlim);
  cudaMemcpyAsync(s->h, s->v, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st);
  if (cudaGetLastError() != cudaSuccess) return SWDK_E_CUDA;
  for (int it = 0;; ++it) {
    if (it % LS_CHECK == 0) {
      if (cudaMemcpyAsync(s->hst, s->st, sizeof(LsmrState), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess)
        return SWDK_E_CUDA;
      if (s->hst->done || s->hst->itn >= itnlim) break;
    }
    // beta u = A v - alpha u
    k_ls_spmv<<<gm, LS_THREADS, 0, st>>>(m, s->rowptr, s->idx, s->val, s->v, s->u, s->st, 0);
    k_ls_partial<<<LS_PART, LS_THREADS, 0, st>>>(m, s->u, s->part, s->st, 0);
    k_ls_norm<<<1, 512, 0, st>>>(s->part, s->st, 0);
    k_ls_div<<<em, LS_THREADS, 0, st>>>(m, s->u, s->st, 0);
    // alpha v = A^T u - beta v
    k_ls_spmv<<<gn, LS_THREADS, 0, st>>>(n, s->trowptr, s->tidx, s->tval, s->u, s->v, s->st, 1);
    k_ls_partial<<<LS_PART, LS_THREADS, 0, st>>>(n, s->v, s->part, s->st, 1);
    k_ls_norm<<<1, 512, 0, st>>>(s->part, s->st, 1);
    k_ls_div<<<en, LS_THREADS, 0, st>>>(n, s->v, s->st, 1);
    k_ls_scalar<<<1, 1, 0, st>>>(s->st);
    k_ls_vec<<<LS_PART, LS_THREADS, 0, st>>>(n, d_x, s->h, s->hbar, s->v, s->part, s->st);
    k_ls_tests<<<1, 512, 0, st>>>(s->part, s->st);
    if (cudaGetLastError() != cudaSuccess) return SWDK_E_CUDA;
  }
  if (info) {
    const LsmrState& h = *s->hst;
    info->istop = h.istop;
    info->itn = h.itn;
    info->normA = h.normA;
    info->condA = h.condA;
    info->normr = h.normr;
    info->normAr = h.normAr;
    info->normx = h.normx;
  }
  return SWDK_OK;
}

void swdk_lsmr_destroy(swdk_lsmr* s) {
  if (!s) return;
  {
    LsDeviceScope scope(s->device);
    ls_free(s);
  }
  delete s;
}

}  // extern "C"
