"""LSMR on the GPU over the assembled sensitivity rows.

The reference solves the damped least-squares system of every inversion
iteration with LSMR (csr_matrix::lsmr_solver, src/shared/csr_matrix.cpp,
running src/shared/lsmrModule_csr.f90 in FP32 with OpenMP matrix products).
Here the matrix stays on the device as the CSR rows swdk_frechet_csr_device
produced (FP32 values, int32 columns, int64 row pointers), with its
transpose built once on the device; the vectors are FP64.  lsmr() runs the
whole iteration in libswdk (swdk_lsmr_solve: row-kernel products of A and
of its transpose, fixed-grid norms, the scalar recurrences in device
memory), so the solve is the same bits on every run; lsmr_stepwise() is the
same iteration driven step by step from the host.

The iteration follows Fong & Saunders, "LSMR: An iterative algorithm for
sparse least-squares problems", SIAM J. Sci. Comput. 33 (2011): Golub-Kahan
bidiagonalization, a first QR factorization of the lower bidiagonal matrix
(with the damping rotation), a second QR factorization giving the
minimization of ||A^T r||, and the paper's estimates of ||r||, ||A^T r||,
||A|| and cond(A) for the stopping rules.  istop has the meaning of the
reference's module:
  1 ||r|| small enough (b-compatible system), 2 ||A^T r|| small (least
  squares), 3 cond(A) above conlim, 4-6 the same three at machine
  precision, 7 iteration limit.
Local reorthogonalization (the reference's localSize) is not implemented.
"""
import ctypes as C
import math

from .engine import SwdkError, lib, torch_stream


class DeviceCSR:
    """m x n matrix as device CSR (torch tensors): rowptr int64 (m+1),
    indices int32, values float32.

    deterministic=True (the default) keeps the transposed matrix too (built
    once on the device, a column's entries in row order), so A^T y is a row
    product like A x: the same sums in the same order on every call.  With
    False, A^T y scatters with FP64 atomics (the reference's myaprod_csr uses
    an OpenMP atomic the same way) and its last bits vary between calls."""

    def __init__(self, rowptr, indices, values, m, n, deterministic=True):
        self.rowptr, self.indices, self.values, self.m, self.n = rowptr, indices, values, m, n
        L = lib()
        L.swdk_aprod_csr.argtypes = [C.c_int, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p]
        self.t = self.transpose() if deterministic else None

    def solver(self):
        """The matrix's swdk_lsmr handle (its work vectors), created on first
        use and kept for the matrix's lifetime."""
        if getattr(self, "_solver", None) is None:
            import weakref
            L = _bind()
            h = C.c_void_p()
            t = self.t
            rc = L.swdk_lsmr_create(self.rowptr.device.index, self.m, self.n, self.rowptr.data_ptr(),
                                    self.indices.data_ptr(), self.values.data_ptr(), t.rowptr.data_ptr(),
                                    t.indices.data_ptr(), t.values.data_ptr(), C.byref(h))
            if rc != 0:
                raise SwdkError(f"swdk_lsmr_create failed ({rc})")
            self._solver = h
            weakref.finalize(self, L.swdk_lsmr_destroy, h)
        return self._solver

    def transpose(self):
        """The n x m transpose as device CSR, each row (a column of A) with its
        entries in increasing row order."""
        import torch
        dev = self.rowptr.device
        counts = torch.diff(self.rowptr)
        rows = torch.repeat_interleave(torch.arange(self.m, dtype=torch.int32, device=dev), counts)
        perm = torch.argsort(self.indices, stable=True)
        colptr = torch.zeros(self.n + 1, dtype=torch.int64, device=dev)
        colptr[1:] = torch.cumsum(torch.bincount(self.indices, minlength=self.n), 0)
        return DeviceCSR(colptr, rows[perm].contiguous(), self.values[perm].contiguous(), self.n, self.m,
                         deterministic=False)

    def aprod(self, mode, x, y):
        """mode 1: y += A x; mode 2: x += A^T y (x, y FP64 device tensors)."""
        import torch
        if mode == 2 and self.t is not None:
            self.t.aprod(1, y, x)
            return
        st = torch.cuda.current_stream(x.device).cuda_stream
        rc = lib().swdk_aprod_csr(mode, self.m, self.n, self.rowptr.data_ptr(), self.indices.data_ptr(),
                                  self.values.data_ptr(), x.data_ptr(), y.data_ptr(), st)
        if rc != 0:
            raise SwdkError(f"swdk_aprod_csr failed ({rc})")


class _Info(C.Structure):
    _fields_ = [("istop", C.c_int), ("itn", C.c_int), ("normA", C.c_double), ("condA", C.c_double),
                ("normr", C.c_double), ("normAr", C.c_double), ("normx", C.c_double)]


def _bind():
    L = lib()
    if not getattr(L, "_lsmr_bound", False):
        vp = C.c_void_p
        L.swdk_lsmr_create.argtypes = [C.c_int, C.c_int64, C.c_int64, vp, vp, vp, vp, vp, vp, C.POINTER(vp)]
        L.swdk_lsmr_solve.argtypes = [vp, vp, vp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                      C.POINTER(_Info), vp]
        L.swdk_lsmr_destroy.argtypes = [vp]
        L.swdk_lsmr_destroy.restype = None
        L._lsmr_bound = True
    return L


def lsmr(A, b, damp=0.0, atol=1e-6, btol=1e-6, conlim=1e8, itnlim=None):
    """Solve min ||A x - b||^2 + damp^2 ||x||^2.  A: DeviceCSR with its
    transpose (deterministic=True); b: FP64 device tensor (m).  The whole
    iteration runs on the device (swdk_lsmr_solve: the scalar recurrences in
    device memory, the host reading them every 16 iterations), on torch's
    current stream.  Returns x (device) and dict(istop, itn, normA, condA,
    normr, normAr, normx)."""
    import torch
    if A.t is None:
        return lsmr_stepwise(A, b, damp, atol, btol, conlim, itnlim)
    L = _bind()
    m, n = A.m, A.n
    itnlim = min(m, n) if itnlim is None else itnlim
    x = torch.empty(n, dtype=torch.float64, device=b.device)
    b = b.contiguous()
    info = _Info()
    st = C.c_void_p(torch_stream(b.device))
    rc = L.swdk_lsmr_solve(A.solver(), C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), damp, atol, btol, conlim,
                           itnlim, C.byref(info), st)
    if rc != 0:
        raise SwdkError(f"swdk_lsmr_solve failed ({rc})")
    return x, dict(istop=info.istop, itn=info.itn, normA=info.normA, condA=info.condA, normr=info.normr,
                   normAr=info.normAr, normx=info.normx)


def lsmr_stepwise(A, b, damp=0.0, atol=1e-6, btol=1e-6, conlim=1e8, itnlim=None):
    """The same iteration step by step from the host: the two products by
    libswdk, the vector updates as torch operations and the scalar
    recurrences in Python (two norm reads per iteration).  Kept as the
    readable statement of what swdk_lsmr_solve does on the device; used
    when A has no transpose."""
    import torch
    m, n = A.m, A.n
    dev = b.device
    itnlim = min(m, n) if itnlim is None else itnlim
    ctol = 1.0 / conlim if conlim > 0 else 0.0
    x = torch.zeros(n, dtype=torch.float64, device=dev)

    # Golub-Kahan start: beta_1 u_1 = b, alpha_1 v_1 = A^T u_1
    u = b.clone()
    beta = float(torch.linalg.vector_norm(u))
    v = torch.zeros(n, dtype=torch.float64, device=dev)
    alpha = 0.0
    if beta > 0.0:
        u /= beta
        A.aprod(2, v, u)
        alpha = float(torch.linalg.vector_norm(v))
    if alpha > 0.0:
        v /= alpha
    normb = beta
    info = dict(istop=0, itn=0, normA=0.0, condA=1.0, normr=beta, normAr=alpha * beta, normx=0.0)
    if alpha * beta == 0.0:
        return x, info

    # state of the two QR factorizations
    alpha_bar, zeta_bar = alpha, alpha * beta      # first column of the damped bidiagonal, rhs of the 2nd QR
    rho_prev, rho_bar_prev, c_bar, s_bar = 1.0, 1.0, 1.0, 0.0
    h = v.clone()
    h_bar = torch.zeros(n, dtype=torch.float64, device=dev)
    # residual-norm recurrences (Fong & Saunders, section 3.4)
    beta_dd, beta_dot = beta, 0.0
    rho_dot_prev, tau_tilde_prev, theta_tilde, zeta_prev = 1.0, 0.0, 0.0, 0.0
    damp_sum = 0.0
    normA2 = alpha * alpha
    rho_bar_max, rho_bar_min = 0.0, 1e300
    istop, itn = 0, 0
    normr = beta
    while itn < itnlim:
        itn += 1
        # bidiagonalization: beta u <- A v - alpha u ; alpha v <- A^T u - beta v
        u *= -alpha
        A.aprod(1, v, u)
        beta = float(torch.linalg.vector_norm(u))
        if beta > 0.0:
            u /= beta
            v *= -beta
            A.aprod(2, v, u)
            alpha = float(torch.linalg.vector_norm(v))
            if alpha > 0.0:
                v /= alpha
        # damping rotation on (alpha_bar, damp)
        alpha_hat = math.hypot(alpha_bar, damp)
        c_hat, s_hat = alpha_bar / alpha_hat, damp / alpha_hat
        # first QR rotation: (alpha_hat, beta)
        rho = math.hypot(alpha_hat, beta)
        c, s = alpha_hat / rho, beta / rho
        theta_next = s * alpha
        alpha_bar = c * alpha
        # second QR rotation
        theta_bar = s_bar * rho
        rho_bar = math.hypot(c_bar * rho, theta_next)
        c_bar, s_bar = c_bar * rho / rho_bar, theta_next / rho_bar
        zeta = c_bar * zeta_bar
        zeta_bar = -s_bar * zeta_bar
        # search directions and solution
        h_bar.mul_(-(theta_bar * rho) / (rho_prev * rho_bar_prev)).add_(h)
        x.add_(h_bar, alpha=zeta / (rho * rho_bar))
        h.mul_(-(theta_next / rho)).add_(v)
        # ||r||: rotations applied to the right-hand side (beta_1, 0, ...)
        beta_acute = c_hat * beta_dd
        beta_check = -s_hat * beta_dd
        beta_hat = c * beta_acute
        beta_dd = -s * beta_acute
        rho_tilde = math.hypot(rho_dot_prev, theta_bar)
        c_t, s_t = rho_dot_prev / rho_tilde, theta_bar / rho_tilde
        theta_tilde_old = theta_tilde
        theta_tilde = s_t * rho_bar
        rho_dot = c_t * rho_bar
        beta_dot = -s_t * beta_dot + c_t * beta_hat
        tau_tilde_prev = (zeta_prev - theta_tilde_old * tau_tilde_prev) / rho_tilde
        tau_dot = (zeta - theta_tilde * tau_tilde_prev) / rho_dot
        damp_sum += beta_check * beta_check
        normr = math.sqrt(damp_sum + (beta_dot - tau_dot) ** 2 + beta_dd ** 2)
        # ||A|| and cond(A) estimates
        normA2 += beta * beta
        normA = math.sqrt(normA2)
        normA2 += alpha * alpha
        rho_bar_max = max(rho_bar_max, rho_bar_prev)
        if itn > 1:
            rho_bar_min = min(rho_bar_min, rho_bar_prev)
        condA = max(rho_bar_max, rho_bar) / min(rho_bar_min, rho_bar)
        normAr = abs(zeta_bar)
        normx = float(torch.linalg.vector_norm(x))
        # roll the recurrences
        rho_prev, rho_bar_prev, rho_dot_prev, zeta_prev = rho, rho_bar, rho_dot, zeta
        # stopping rules
        test1 = normr / normb
        test2 = normAr / (normA * normr) if normA * normr > 0.0 else math.inf
        test3 = 1.0 / condA
        t1 = test1 / (1.0 + normA * normx / normb)
        rtol = btol + atol * normA * normx / normb
        if itn >= itnlim:
            istop = 7
        if 1.0 + test3 <= 1.0:
            istop = 6
        if 1.0 + test2 <= 1.0:
            istop = 5
        if 1.0 + t1 <= 1.0:
            istop = 4
        if test3 <= ctol:
            istop = 3
        if test2 <= atol:
            istop = 2
        if test1 <= rtol:
            istop = 1
        info.update(istop=istop, itn=itn, normA=normA, condA=condA, normr=normr, normAr=normAr, normx=normx)
        if istop > 0:
            break
    return x, info
