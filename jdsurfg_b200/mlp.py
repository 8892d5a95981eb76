"""ctypes binding of the learned bracket proposal network (swdk_mlp_* in
libswdk.so): training, inference and checkpoints on the GPU."""
import ctypes as C

import numpy as np

from .engine import SwdkError, lib as _lib, torch_stream

IN_DIM, HIDDEN, OUT_PHYS = 320, 256, 64


def _bind():
    L = _lib()
    if getattr(L, "_mlp_bound", False):
        return L
    vp = C.c_void_p
    L.swdk_mlp_create.argtypes = [C.POINTER(vp), C.c_int, C.c_uint64]
    L.swdk_mlp_destroy.argtypes = [vp]
    L.swdk_mlp_destroy.restype = None
    L.swdk_mlp_num_params.argtypes = [vp]
    L.swdk_mlp_num_params.restype = C.c_int64
    L.swdk_mlp_get_params.argtypes = [vp, vp, C.c_int64]
    L.swdk_mlp_set_params.argtypes = [vp, vp, C.c_int64]
    L.swdk_mlp_get_grads.argtypes = [vp, vp, C.c_int64]
    L.swdk_mlp_forward.argtypes = [vp, vp, C.c_int, vp, vp]
    L.swdk_mlp_propose.argtypes = [vp, vp, C.c_int, C.c_double, vp, vp]
    L.swdk_mlp_error_flag.argtypes = [vp, C.POINTER(C.c_int)]
    L.swdk_mlp_train_step.argtypes = [vp, vp, vp, C.c_int, C.c_float, C.POINTER(C.c_float), vp]
    L.swdk_mlp_save.argtypes = [vp, C.c_char_p]
    L.swdk_mlp_load.argtypes = [vp, C.c_char_p]
    L.swdk_mlp_last_error.argtypes = [vp]
    L.swdk_mlp_last_error.restype = C.c_char_p
    L.swdk_gemm_bf16_tn.argtypes = [C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp]
    L._mlp_bound = True
    return L


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


class MLP:
    """The proposal network on one GPU (FP32 masters, BF16 tensor-core GEMMs)."""

    def __init__(self, device=0, seed=1234):
        L = _bind()
        h = C.c_void_p()
        rc = L.swdk_mlp_create(C.byref(h), device, seed)
        if rc != 0:
            raise SwdkError(f"swdk_mlp_create failed ({rc})")
        self._h = h
        self.n = L.swdk_mlp_num_params(h)

    def close(self):
        if getattr(self, "_h", None):
            _bind().swdk_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != 0:
            raise SwdkError(f"{what} failed ({rc}): {_bind().swdk_mlp_last_error(self._h).decode()}")

    def params(self):
        out = np.empty(self.n, np.float32)
        self._check(_bind().swdk_mlp_get_params(self._h, out.ctypes.data_as(C.c_void_p), self.n), "get_params")
        return out

    def set_params(self, w):
        w = np.ascontiguousarray(w, np.float32)
        self._check(_bind().swdk_mlp_set_params(self._h, w.ctypes.data_as(C.c_void_p), self.n), "set_params")

    def grads(self):
        out = np.empty(self.n, np.float32)
        self._check(_bind().swdk_mlp_get_grads(self._h, out.ctypes.data_as(C.c_void_p), self.n), "get_grads")
        return out

    def forward(self, x_bf16, out=None):
        """x_bf16: torch bfloat16 (M, 320) on the device -> (M, 2) float32."""
        import torch
        M = x_bf16.shape[0]
        if out is None:
            out = torch.empty((M, 2), dtype=torch.float32, device=x_bf16.device)
        self._check(_bind().swdk_mlp_forward(self._h, _p(x_bf16), M, _p(out), None), "forward")
        return out

    def propose(self, x_tiles, nrows, kappa, prop):
        """Fused inference on tile-image features straight to (c, half-width)
        per row (prop: (nrows, 2) float32), on torch's current stream."""
        import torch
        st = C.c_void_p(torch_stream(prop.device))
        self._check(_bind().swdk_mlp_propose(self._h, _p(x_tiles), nrows, kappa, _p(prop), st), "propose")
        return prop

    def error_flag(self):
        f = C.c_int(0)
        self._check(_bind().swdk_mlp_error_flag(self._h, C.byref(f)), "error_flag")
        return f.value

    def train_step(self, x_bf16, y, lr):
        loss = C.c_float(0.0)
        self._check(_bind().swdk_mlp_train_step(self._h, _p(x_bf16), _p(y), x_bf16.shape[0], lr, C.byref(loss), None),
                    "train_step")
        return loss.value

    def save(self, path):
        self._check(_bind().swdk_mlp_save(self._h, path.encode()), "save")

    def load(self, path):
        self._check(_bind().swdk_mlp_load(self._h, path.encode()), "load")


def layout():
    """Offsets of (W, b) per layer in the flat parameter vector."""
    kin = [IN_DIM, HIDDEN, HIDDEN, HIDDEN, HIDDEN]
    nout = [HIDDEN, HIDDEN, HIDDEN, HIDDEN, OUT_PHYS]
    off, out = 0, []
    for k, n in zip(kin, nout):
        out.append((off, n, k, off + n * k))
        off += n * k + n
    return out


def gemm_bf16_tn(a, b, c, err):
    """c = a @ b.T with the tcgen05 GEMM (device torch tensors)."""
    M, K = a.shape
    N = b.shape[0]
    rc = _bind().swdk_gemm_bf16_tn(M, N, K, _p(a), _p(b), _p(c), _p(err), None)
    if rc != 0:
        raise SwdkError(f"swdk_gemm_bf16_tn failed ({rc})")
