"""ctypes binding of libswdk.so: the SurfTime-facing calls of the GPU engine.

The method names follow the reference class they replace (JDSurfG
src/SWD/SurfaceWave.hpp: SurfTime::get_1d_kernel, get_2d_map, set_model and
the period tables tRc/tRg/tLc/tLg).  Arrays use the reference's Eigen
column-major layouts, exposed to numpy as C-order arrays with the axes
reversed:

    vs, vp, rho        : (nz, ncol)        float32   == Eigen fmat3(nx, ny, nz)
    vc, vout, status   : (kmax, ncol)      float64 / int32 == dmat2(nx*ny, kmax)
    kernel             : (kmax, nz, ncol)  float64   == dmat3(nx*ny, nz, kmax)

There is no CPU fallback: constructing an Engine without the built library or
without a CUDA device raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libswdk.so")

ST_OK, ST_NO_ROOT, ST_RETRIED, ST_NAN_INPUT, ST_ITER_LIMIT = 0, 1, 2, 3, 4
REFINE = {"reference": 0, "tight": 1}


class Config(C.Structure):
    _fields_ = [("device", C.c_int), ("refine", C.c_int), ("rtol", C.c_double), ("sngl", C.c_int),
                ("sphere", C.c_int), ("block_roots", C.c_int), ("split_cols", C.c_int), ("node_layers", C.c_int)]


class Call(C.Structure):
    """swdk_call: one model's device call inside a batch graph."""
    _fields_ = [("path", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("d_vs", C.c_void_p), ("d_vp", C.c_void_p), ("d_rho", C.c_void_p),
                ("d_vc", C.c_void_p), ("d_vout", C.c_void_p), ("d_kernel", C.c_void_p), ("d_status", C.c_void_p)]


class Stats(C.Structure):
    _fields_ = [("secular_evals", C.c_int64), ("layer_evals_rayleigh", C.c_int64), ("layer_evals_love", C.c_int64),
                ("nchains", C.c_int32), ("nslots", C.c_int32),
                ("ms_prep", C.c_float), ("ms_roots", C.c_float), ("ms_eigen", C.c_float),
                ("proposals_accepted", C.c_int64), ("proposals_rejected", C.c_int64), ("ms_proposal", C.c_float),
                ("kernel_launches", C.c_int32), ("evals_by_phase", C.c_int64 * 6)]

EVAL_PHASES = ("scan_first_period", "scan", "learned_cell", "walk", "refine", "retry")


def stats_dict(s):
    """A swdk_stats structure as a dict."""
    return dict(secular_evals=s.secular_evals, layer_evals_rayleigh=s.layer_evals_rayleigh,
                layer_evals_love=s.layer_evals_love, nchains=s.nchains, nslots=s.nslots, ms_prep=s.ms_prep,
                ms_roots=s.ms_roots, ms_eigen=s.ms_eigen, proposals_accepted=s.proposals_accepted,
                proposals_rejected=s.proposals_rejected, ms_proposal=s.ms_proposal,
                kernel_launches=s.kernel_launches,
                evals_by_phase=dict(zip(EVAL_PHASES, [int(x) for x in s.evals_by_phase])))


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run jdsurfg_b200/build.py (or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.swdk_config_default.argtypes = [C.POINTER(Config)]
        L.swdk_create.argtypes = [C.POINTER(vp), C.POINTER(Config)]
        L.swdk_destroy.argtypes = [vp]
        L.swdk_destroy.restype = None
        L.swdk_set_periods.argtypes = [vp] + [vp, C.c_int, C.c_int] * 4
        L.swdk_set_depth.argtypes = [vp, vp, C.c_int]
        L.swdk_kmax.argtypes = [vp]
        L.swdk_get_1d_kernel.argtypes = [vp, C.c_int, C.c_int, C.c_int] + [vp] * 7
        L.swdk_get_2d_map.argtypes = [vp, C.c_int, C.c_int, C.c_int] + [vp] * 6
        L.swdk_get_1d_kernel_device.argtypes = [vp, C.c_int, C.c_int, C.c_int] + [vp] * 8
        L.swdk_get_2d_map_device.argtypes = [vp, C.c_int, C.c_int, C.c_int] + [vp] * 7
        L.swdk_surfdisp96_batch.argtypes = [vp, C.c_int, C.c_int, vp, vp, vp, vp, C.c_int, C.c_int, C.c_int,
                                            C.c_int, C.c_int, vp, vp, vp]
        L.swdk_frechet_rows_device.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, C.c_int, vp, vp, vp,
                                               vp, vp, vp]
        L.swdk_get_stats.argtypes = [vp, C.POINTER(Stats)]
        L.swdk_set_proposal.argtypes = [vp, vp, vp, C.c_double, C.c_double]
        L.swdk_set_proposal_shift.argtypes = [vp, C.c_double]
        L.swdk_roots_device.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp]
        L.swdk_root_slots.argtypes = [vp, C.POINTER(C.c_int), vp, vp, vp]
        L.swdk_last_roots.argtypes = [vp, vp, vp]
        L.swdk_training_rows.argtypes = [vp, vp, C.c_int, vp, vp, vp]
        L.swdk_graph_capture.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int] + [vp] * 7
        L.swdk_graph_launch.argtypes = [vp, vp]
        L.swdk_autotune.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp, vp, vp, C.POINTER(C.c_int)]
        L.swdk_frechet_csr_device.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, C.c_int, vp, vp, vp, vp, vp,
                                              C.c_int64, C.POINTER(C.c_int64), vp]
        L.swdk_batch_graph_create.argtypes = [C.c_int, vp, vp, C.POINTER(vp)]
        L.swdk_batch_graph_launch.argtypes = [vp, vp]
        L.swdk_batch_graph_destroy.argtypes = [vp]
        L.swdk_batch_graph_destroy.restype = None
        L.swdk_ragged_create.argtypes = [C.c_int, vp, vp, C.POINTER(vp)]
        L.swdk_ragged_run.argtypes = [vp, vp]
        L.swdk_ragged_launch.argtypes = [vp, vp]
        L.swdk_ragged_stats.argtypes = [vp, C.POINTER(Stats)]
        L.swdk_ragged_destroy.argtypes = [vp]
        L.swdk_ragged_destroy.restype = None
        L.swdk_last_error.argtypes = [vp]
        L.swdk_last_error.restype = C.c_char_p
        _LIB = L
    return _LIB


def torch_stream(device):
    """Handle of torch's current stream on `device` for the entry points
    whose NULL stream means the context's own stream: torch's default stream
    (handle 0) is passed as cudaStreamLegacy (0x1), the legacy default
    stream it stands for."""
    import torch
    h = torch.cuda.current_stream(device).cuda_stream
    return h if h else 1


def _p(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


class SwdkError(RuntimeError):
    pass


class Engine:
    """One GPU context (device buffers, plans, stream) of libswdk."""

    def __init__(self, device=0, refine="tight", rtol=1e-10, sngl=True, sphere=True, block_roots=0, split_cols=0,
                 node_layers=True):
        L = lib()
        cfg = Config()
        L.swdk_config_default(C.byref(cfg))
        cfg.device = device
        cfg.refine = REFINE[refine] if isinstance(refine, str) else int(refine)
        cfg.rtol = rtol
        cfg.sngl = 1 if sngl else 0
        cfg.sphere = 1 if sphere else 0
        cfg.block_roots = block_roots
        cfg.split_cols = split_cols
        cfg.node_layers = 1 if node_layers else 0
        h = C.c_void_p()
        rc = L.swdk_create(C.byref(h), C.byref(cfg))
        if rc != 0:
            raise SwdkError(f"swdk_create failed ({rc}); a CUDA device is required")
        self._h = h
        self.cfg = cfg
        self._keep = []

    def close(self):
        if getattr(self, "_h", None):
            lib().swdk_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != 0:
            msg = lib().swdk_last_error(self._h).decode()
            raise SwdkError(f"{what} failed ({rc}): {msg}")

    # -- SurfTime state -------------------------------------------------------
    def set_periods(self, tables):
        """tables: [tRc, tRg, tLc, tLg], each (ntmax, nmode) array with -1
        padding or None."""
        args = []
        keep = []
        for t in tables:
            if t is None:
                args += [None, 0, 0]
            else:
                t = np.asfortranarray(np.asarray(t, np.float64))
                if t.ndim == 1:
                    t = t[:, None]
                keep.append(t)
                args += [_p(t), t.shape[0], t.shape[1]]
        self._check(lib().swdk_set_periods(self._h, *args), "swdk_set_periods")
        self.kmax = lib().swdk_kmax(self._h)

    def set_depth(self, depth):
        d = _f32(depth)
        self._check(lib().swdk_set_depth(self._h, _p(d), len(d)), "swdk_set_depth")
        self.nz = len(d)

    def setup(self, case):
        self.set_depth(case["depth"])
        self.set_periods(case["tables"])

    # -- host-memory calls ----------------------------------------------------
    def get_1d_kernel(self, vs, vp=None, rho=None, nx=None, ny=1):
        vs, vp, rho = _f32(vs), _f32(vp), _f32(rho)
        nz, ncol = vs.shape
        nx = ncol if nx is None else nx
        ny = ncol // nx
        vc = np.empty((self.kmax, ncol))
        vout = np.empty((self.kmax, ncol))
        ker = np.empty((self.kmax, nz, ncol))
        st = np.empty((self.kmax, ncol), np.int32)
        self._check(lib().swdk_get_1d_kernel(self._h, nx, ny, nz, _p(vs), _p(vp), _p(rho), _p(vc), _p(vout), _p(ker),
                                             _p(st)), "swdk_get_1d_kernel")
        return dict(vc=vc, vout=vout, kernel=ker, status=st)

    def get_2d_map(self, vs, vp=None, rho=None, nx=None, ny=1):
        vs, vp, rho = _f32(vs), _f32(vp), _f32(rho)
        nz, ncol = vs.shape
        nx = ncol if nx is None else nx
        ny = ncol // nx
        vc = np.empty((self.kmax, ncol))
        vout = np.empty((self.kmax, ncol))
        st = np.empty((self.kmax, ncol), np.int32)
        self._check(lib().swdk_get_2d_map(self._h, nx, ny, nz, _p(vs), _p(vp), _p(rho), _p(vc), _p(vout), _p(st)),
                    "swdk_get_2d_map")
        return dict(vc=vc, vout=vout, status=st)

    def run_case(self, case, path="kernel"):
        self.setup(case)
        f = self.get_1d_kernel if path == "kernel" else self.get_2d_map
        return f(case["vs"], case["vp"], case["rho"], nx=case["nx"], ny=case["ny"])

    # -- device-memory calls (torch tensors or raw pointers) ------------------
    def get_1d_kernel_device(self, nx, ny, nz, vs, vp, rho, vc, vout, kernel, status, stream=None):
        self._check(lib().swdk_get_1d_kernel_device(self._h, nx, ny, nz, _p(vs), _p(vp), _p(rho), _p(vc), _p(vout),
                                                    _p(kernel), _p(status), stream), "swdk_get_1d_kernel_device")

    def get_2d_map_device(self, nx, ny, nz, vs, vp, rho, vc, vout, status, stream=None):
        self._check(lib().swdk_get_2d_map_device(self._h, nx, ny, nz, _p(vs), _p(vp), _p(rho), _p(vc), _p(vout),
                                                 _p(status), stream), "swdk_get_2d_map_device")

    def surfdisp96_batch(self, thk, vp, vs, rho, iflsph, iwave, mode, igr, t):
        """surfdisp96_ over models given as (nmodel, nlayer) arrays."""
        thk, vp, vs, rho = _f32(thk), _f32(vp), _f32(vs), _f32(rho)
        nmodel, nlayer = thk.shape
        t = np.ascontiguousarray(t, np.float64)
        cg = np.empty((nmodel, len(t)))
        ierr = np.empty(nmodel, np.int32)
        self._check(lib().swdk_surfdisp96_batch(self._h, nmodel, nlayer, _p(thk), _p(vp), _p(vs), _p(rho), iflsph,
                                                iwave, mode, igr, len(t), _p(t), _p(cg), _p(ierr)),
                    "swdk_surfdisp96_batch")
        return cg, ierr

    def frechet_rows_device(self, nx, ny, nz, kmax, kernel, row_slot, fdm, nnz, indices, values, stream=None):
        self._check(lib().swdk_frechet_rows_device(self._h, nx, ny, nz, kmax, _p(kernel), len(row_slot), _p(row_slot),
                                                   _p(fdm), _p(nnz), _p(indices), _p(values), stream),
                    "swdk_frechet_rows_device")

    # -- learned bracket proposals -------------------------------------------
    def set_proposal(self, rayleigh=None, love=None, kappa_rayleigh=4.0, kappa_love=4.0):
        """Attach proposal networks (jdsurfg_b200.mlp.MLP or None each)."""
        self._nets = (rayleigh, love)
        hr = rayleigh._h if rayleigh is not None else None
        hl = love._h if love is not None else None
        self._check(lib().swdk_set_proposal(self._h, hr, hl, kappa_rayleigh, kappa_love), "swdk_set_proposal")

    def set_proposal_shift(self, shift_km_s):
        """Testing aid: move every proposed phase velocity by shift_km_s
        (only the first period's jump moves; the roots must not)."""
        self._check(lib().swdk_set_proposal_shift(self._h, float(shift_km_s)), "swdk_set_proposal_shift")

    def roots_device(self, nx, ny, nz, vs, vp=None, rho=None, stream=None):
        """Root search of every get_1d_kernel root slot on device models."""
        self._check(lib().swdk_roots_device(self._h, nx, ny, nz, _p(vs), _p(vp), _p(rho), stream),
                    "swdk_roots_device")

    def root_slots(self):
        """(wave, mode, period) per root slot (wave 2 Rayleigh, 1 Love; mode 0-based)."""
        n = C.c_int(0)
        self._check(lib().swdk_root_slots(self._h, C.byref(n), None, None, None), "swdk_root_slots")
        w = np.empty(n.value, np.int32)
        m = np.empty(n.value, np.int32)
        t = np.empty(n.value, np.float64)
        self._check(lib().swdk_root_slots(self._h, C.byref(n), _p(w), _p(m), _p(t)), "swdk_root_slots")
        return w, m, t

    def last_roots(self, ncol):
        """Roots (nslot, ncol) and their status of the last root search."""
        w, _, _ = self.root_slots()
        c = np.empty((len(w), ncol))
        st = np.empty((len(w), ncol), np.int32)
        self._check(lib().swdk_last_roots(self._h, _p(c), _p(st)), "swdk_last_roots")
        return c, st

    def training_rows(self, rows, x, y=None, stream=None):
        """Features (bf16 (n, 320)) and targets (c - 3.5) of rows slot*ncol+col
        after roots_device; rows is an int64 device tensor."""
        self._check(lib().swdk_training_rows(self._h, _p(rows), rows.shape[0], _p(x), _p(y), stream),
                    "swdk_training_rows")

    def frechet_csr_device(self, nx, ny, nz, kmax, kernel, row_slot, fdm, rowptr, indices, values, stream=None):
        """Frechet rows as CSR on the device; returns the number of nonzeros.
        With indices None only the row pointer and the count are produced."""
        tot = C.c_int64(0)
        cap = 0 if indices is None else indices.numel()
        rc = lib().swdk_frechet_csr_device(self._h, nx, ny, nz, kmax, _p(kernel), len(row_slot), _p(row_slot),
                                           _p(fdm), _p(rowptr), _p(indices), _p(values), cap, C.byref(tot), stream)
        if indices is None and rc == -5:  # SWDK_E_LIMIT: counted, nothing written
            return tot.value
        self._check(rc, "swdk_frechet_csr_device")
        return tot.value

    # -- CUDA graph of one device call, autotuner ------------------------------
    PATHS = {"kernel": 0, "map": 1, "roots": 2}

    def graph_capture(self, path, nx, ny, nz, vs, vp, rho, vc=None, vout=None, kernel=None, status=None):
        self._check(lib().swdk_graph_capture(self._h, self.PATHS[path], nx, ny, nz, _p(vs), _p(vp), _p(rho), _p(vc),
                                             _p(vout), _p(kernel), _p(status)), "swdk_graph_capture")

    def graph_launch(self, stream=None):
        self._check(lib().swdk_graph_launch(self._h, stream), "swdk_graph_launch")

    def autotune(self, nx, ny, nz, vs, vp=None, rho=None):
        b = C.c_int(0)
        self._check(lib().swdk_autotune(self._h, nx, ny, nz, _p(vs), _p(vp), _p(rho), C.byref(b)), "swdk_autotune")
        return b.value

    def stats(self):
        s = Stats()
        self._check(lib().swdk_get_stats(self._h, C.byref(s)), "swdk_get_stats")
        return stats_dict(s)
