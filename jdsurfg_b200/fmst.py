"""ctypes binding of the fast-marching part of libswdk.so (swdk_fmst_*).

FMST replaces the per-pair calls fmst_init / fmst_run / fmst_reset /
fmst_raypath / fmst_finalize (JDSurfG src/SWD/SurfaceWave.hpp:8-50,
src/SWD/fmst.f90, src/SWD/fmm.f90) with one batched device call over all
station pairs of an iteration.  Pairs are given as the fields of the
reference's StationPair (src/SWD/SurfaceWave.hpp:53-82), flattened:

    slot[p]     period slot of pair p (SurfTime::get_period_index)
    srcx, srcz  source colatitude and longitude, radians (float32)
    group[p]    1 for Rg/Lg data, 0 for Rc/Lc
    rcv_ptr     receivers of pair p are rcv_ptr[p] .. rcv_ptr[p+1]-1 (int64)
    rcx, rcz    receiver colatitude and longitude, radians (float32)

Velocity maps are the device (kmax, nx*ny) float64 tensors vc / vout that
Engine.get_2d_map_device / get_1d_kernel_device fill.
"""
import ctypes as C

import numpy as np

from .engine import SwdkError, _p, lib

FMST_SOURCE_OUTSIDE, FMST_RECEIVER_OUTSIDE, FMST_BAND_OVERFLOW, FMST_RAY_UNFINISHED = 1, 2, 3, 4


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("goxd", C.c_float), ("gozd", C.c_float), ("dvxd", C.c_float),
                ("dvzd", C.c_float)]


def _bind():
    L = lib()
    if getattr(L, "_fmst_bound", False):
        return L
    vp = C.c_void_p
    L.swdk_fmst_create.argtypes = [C.POINTER(vp), C.c_int, C.POINTER(Grid)]
    L.swdk_fmst_destroy.argtypes = [vp]
    L.swdk_fmst_destroy.restype = None
    L.swdk_fmst_last_error.argtypes = [vp]
    L.swdk_fmst_last_error.restype = C.c_char_p
    L.swdk_fmst_set_options.argtypes = [vp, C.c_size_t, C.c_int, C.c_int, C.c_int, C.c_int]
    L.swdk_fmst_info.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double),
                                 C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.swdk_fmst_pairs.argtypes = [vp, C.c_int] + [vp] * 9 + [C.c_int] + [vp] * 4
    L._fmst_bound = True
    return L


def _a(x, dt):
    return np.ascontiguousarray(np.asarray(x), dtype=dt)


class FMST:
    """Fast marching on one model grid (fmst_init's arguments: nx latitude x
    ny longitude nodes, upper-left corner lat0/lon0 and spacing in degrees)."""

    def __init__(self, nx, ny, lat0, lon0, dlat, dlon, device=0):
        L = _bind()
        self.nx, self.ny = nx, ny
        h = C.c_void_p()
        g = Grid(nx, ny, lat0, lon0, dlat, dlon)
        rc = L.swdk_fmst_create(C.byref(h), device, C.byref(g))
        if rc != 0:
            raise SwdkError(f"swdk_fmst_create failed ({rc})")
        self._h = h
        a, b = C.c_int(0), C.c_int(0)
        L.swdk_fmst_info(self._h, C.byref(a), C.byref(b), None, None, None)
        self.nnx, self.nnz = a.value, b.value

    def close(self):
        if getattr(self, "_h", None):
            _bind().swdk_fmst_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_options(self, scratch_budget_bytes=0, lanes_per_warp=8, warps_per_sm=12, smem_heap=-1, lanes_per_pair=4):
        """Marching layout (none of it changes a result): see swdk_fmst_set_options."""
        rc = _bind().swdk_fmst_set_options(self._h, scratch_budget_bytes, lanes_per_warp, warps_per_sm, smem_heap,
                                           lanes_per_pair)
        if rc != 0:
            raise SwdkError(f"swdk_fmst_set_options failed ({rc})")

    def last_ms(self):
        return self.last_info()["ms"]

    def last_info(self):
        """Device ms, largest narrow band and re-marched pairs of the last call."""
        ms, band, ov = C.c_double(0.0), C.c_int(0), C.c_int(0)
        _bind().swdk_fmst_info(self._h, None, None, C.byref(ms), C.byref(band), C.byref(ov))
        return dict(ms=ms.value, max_band=band.value, overflow_pairs=ov.value)

    def pairs(self, pairs, vc, vout, want_fdm=False, stream=None):
        """Traveltimes of every receiver (and with want_fdm the ray-path
        weights, (nrcv, ny, nx) float32 == (nx, ny) column-major per row) as
        device tensors; status per receiver (FMST_*)."""
        import torch
        L = _bind()
        slot, srcx, srcz = _a(pairs["slot"], np.int32), _a(pairs["srcx"], np.float32), _a(pairs["srcz"], np.float32)
        group, rptr = _a(pairs["group"], np.int32), _a(pairs["rcv_ptr"], np.int64)
        rcx, rcz = _a(pairs["rcx"], np.float32), _a(pairs["rcz"], np.float32)
        nrcv = int(rptr[-1])
        dev = vc.device
        tt = torch.empty(nrcv, dtype=torch.float32, device=dev)
        st = torch.empty(nrcv, dtype=torch.int32, device=dev)
        fdm = torch.empty((nrcv, self.ny, self.nx), dtype=torch.float32, device=dev) if want_fdm else None
        if stream is None:
            stream = torch.cuda.current_stream(dev).cuda_stream
        rc = L.swdk_fmst_pairs(self._h, len(slot), _p(slot), _p(srcx), _p(srcz), _p(group), _p(rptr), _p(rcx),
                               _p(rcz), _p(vc), _p(vout), vc.shape[0], _p(tt), _p(fdm), _p(st), stream)
        if rc != 0:
            raise SwdkError(f"swdk_fmst_pairs failed ({rc}): {L.swdk_fmst_last_error(self._h).decode()}")
        return dict(ttime=tt, status=st, fdm=fdm)
