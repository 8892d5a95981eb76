"""ctypes access to the CPU oracle (oracle/libswd_oracle.so).

Test infrastructure only: tests use it as the checker; bench.py uses it for
the timed CPU baseline.  Nothing in the product path imports this module.
"""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
_LIB = None
_REF = None


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def build():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def lib():
    global _LIB
    if _LIB is None:
        so = os.path.join(ORACLE_DIR, "libswd_oracle.so")
        if not os.path.exists(so):
            build()
        _LIB = C.CDLL(so)
        _LIB.swdo_dltar.restype = C.c_double
        _LIB.swdo_frechet_rows.restype = C.c_long
    return _LIB


def ref_cxx():
    """The reference's own surfdisp.cpp/empirical.cpp (oracle/_ref), or None."""
    global _REF
    if _REF is None:
        so = os.path.join(ORACLE_DIR, "_ref", "libswd_refcxx.so")
        if not os.path.exists(so):
            return None
        _REF = C.CDLL(so)
    return _REF


def reference_dir():
    """The reference checkout, or None: the environment variable
    JDSURFG_REFERENCE, else the default oracle/Makefile's recipe uses."""
    ref = os.environ.get("JDSURFG_REFERENCE")
    if not ref:
        try:
            ref = subprocess.run(["make", "-s", "-C", ORACLE_DIR, "--eval",
                                  "print-var: ; @echo $(JDSURFG_REFERENCE)", "print-var"], check=True,
                                 capture_output=True, text=True).stdout.strip()
        except Exception:
            ref = None
    return ref if ref and os.path.isdir(ref) else None


def load_swd_model():
    d = np.loadtxt(os.path.join(ROOT, "tests", "golden", "swd_model.txt"), skiprows=1).astype(np.float32)
    return [np.ascontiguousarray(d[:, i]) for i in range(4)]  # z, vs, vp, rho


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def surfdisp96(thk, vp, vs, rho, iflsph, iwave, mode, igr, t, refine=0, rtol=1e-10, sngl=1):
    thk, vp, vs, rho = f32(thk), f32(vp), f32(vs), f32(rho)
    t = np.ascontiguousarray(t, np.float64)
    cg = np.zeros(len(t))
    ierr, nev, itl = C.c_int(0), C.c_long(0), C.c_int(0)
    lib().swdo_surfdisp96_ex(_ptr(thk), _ptr(vp), _ptr(vs), _ptr(rho), len(thk), iflsph, iwave, mode, igr, len(t),
                             _ptr(t), _ptr(cg), C.byref(ierr), refine, C.c_double(rtol), sngl, C.byref(nev),
                             C.byref(itl))
    return cg, ierr.value, nev.value


def surfdisp(thk, vp, vs, rho, t, wtype, mode=0, sphere=1, keep_flat=1, refine=0, rtol=1e-10, sngl=1):
    thk, vp, vs, rho = f32(thk), f32(vp), f32(vs), f32(rho)
    t = np.ascontiguousarray(t, np.float64)
    cg = np.zeros(len(t))
    st = np.zeros(len(t), np.int32)
    lib().swdo_surfdisp(_ptr(thk), _ptr(vp), _ptr(vs), _ptr(rho), len(thk), _ptr(t), _ptr(cg), len(t), wtype, mode,
                        sphere, keep_flat, refine, C.c_double(rtol), sngl, _ptr(st))
    return cg, st


def dltar(thk, vp, vs, rho, iflsph, iwave, t, c):
    thk, vp, vs, rho = f32(thk), f32(vp), f32(vs), f32(rho)
    return lib().swdo_dltar(_ptr(thk), _ptr(vp), _ptr(vs), _ptr(rho), len(thk), iflsph, iwave, C.c_double(t),
                            C.c_double(c))


def sregn96(thk, vp, vs, rho, t, cp, iflsph=1):
    thk, vp, vs, rho = f32(thk), f32(vp), f32(vs), f32(rho)
    n = len(thk)
    b = [np.zeros(n) for _ in range(8)]
    tt, cpv, cg = C.c_double(t), C.c_double(cp), C.c_double(0)
    lib().sregn96_(_ptr(thk), _ptr(vp), _ptr(vs), _ptr(rho), n, C.byref(tt), C.byref(cpv), C.byref(cg),
                   *[_ptr(x) for x in b], iflsph)
    keys = ["ur", "uz", "tr", "tz", "dcda", "dcdb", "dcdh", "dcdr"]
    out = dict(zip(keys, b))
    out["c"] = cpv.value
    out["u"] = cg.value
    return out


def slegn96(thk, vs, rho, t, cp, iflsph=1):
    thk, vs, rho = f32(thk), f32(vs), f32(rho)
    n = len(thk)
    b = [np.zeros(n) for _ in range(5)]
    tt, cpv, cg = C.c_double(t), C.c_double(cp), C.c_double(0)
    lib().slegn96_(_ptr(thk), _ptr(vs), _ptr(rho), n, C.byref(tt), C.byref(cpv), C.byref(cg),
                   *[_ptr(x) for x in b], iflsph)
    keys = ["uu", "tt", "dcdb", "dcdh", "dcdr"]
    out = dict(zip(keys, b))
    out["c"] = cpv.value
    out["u"] = cg.value
    return out


def grid2layer(z, vp, vs, rho, sublayers=3):
    nz = len(z)
    L = nz + (nz - 1) * sublayers
    th, a, b, r = [np.zeros(L, np.float32) for _ in range(4)]
    L = lib().swdo_grid2layer(_ptr(f32(z)), _ptr(f32(vp)), _ptr(f32(vs)), _ptr(f32(rho)), nz, sublayers, _ptr(th),
                              _ptr(a), _ptr(b), _ptr(r))
    return th[:L], a[:L], b[:L], r[:L]


def _table_args(tables):
    args, keep = [], []
    for w in range(4):
        t = tables[w]
        if t is None:
            args += [None, 0, 0]
        else:
            t = np.asfortranarray(np.asarray(t, np.float64))
            keep.append(t)
            args += [_ptr(t), t.shape[0], t.shape[1]]
    return args, keep


def _kmax(tables):
    from jdsurfg_b200.synth import kmax_of
    return kmax_of([None if t is None else np.asarray(t) for t in tables])


def kernel1d(vs, vp, rho, dep, tables, refine=1, rtol=1e-12, sngl=0, sphere=1):
    """One column through kernel1D; returns node kernels before the chain rule."""
    nz = len(dep)
    targs, keep = _table_args(tables)
    kmax = _kmax(tables)
    vc, vo = np.zeros(kmax), np.zeros(kmax)
    kvs, kvp, kr = np.zeros(kmax * nz), np.zeros(kmax * nz), np.zeros(kmax * nz)
    st = np.zeros(kmax, np.int32)
    lib().swdo_kernel1d(_ptr(f32(vs)), _ptr(f32(vp)), _ptr(f32(rho)), _ptr(f32(dep)), nz, *targs, _ptr(vc), _ptr(vo),
                        _ptr(kvs), _ptr(kvp), _ptr(kr), _ptr(st), refine, C.c_double(rtol), sngl, sphere)
    sh = (kmax, nz)
    return dict(vc=vc, vout=vo, kvs=kvs.reshape(sh), kvp=kvp.reshape(sh), krho=kr.reshape(sh), status=st)


def get_1d_kernel(case, refine=1, rtol=1e-10, sngl=1, sphere=1, nthreads=0, cols=None):
    from jdsurfg_b200.synth import subset_columns
    if cols is not None:
        case = subset_columns(case, cols)
    vs = case["vs"]
    nz, ncol = vs.shape
    targs, keep = _table_args(case["tables"])
    kmax = _kmax(case["tables"])
    vc, vo = np.zeros((kmax, ncol)), np.zeros((kmax, ncol))
    ker = np.zeros((kmax, nz, ncol))
    st = np.zeros((kmax, ncol), np.int32)
    nev = C.c_long(0)
    lib().swdo_get_1d_kernel(ncol, nz, _ptr(vs), _ptr(case["vp"]), _ptr(case["rho"]), _ptr(case["depth"]), *targs,
                             _ptr(vc), _ptr(vo), _ptr(ker), _ptr(st), refine, C.c_double(rtol), sngl, sphere,
                             nthreads, C.byref(nev))
    return dict(vc=vc, vout=vo, kernel=ker, status=st, nevals=nev.value)


def kernel_spread(case, cols, rel=1e-15, steps=(-3, -1, 1, 3)):
    """Conditioning of the oracle's own kernel path at the given columns:
    get_1d_kernel with every phase velocity handed to sregn96/slegn96 (and
    c1, c2 of the group kernels) moved by s*rel relative, s in `steps`.
    Returns (kernel spread, U spread): per (slot, column) the largest change
    of the node kernel relative to the slot's largest |kernel|, and the
    largest change of vout (km/s), over the steps."""
    base = get_1d_kernel(case, cols=cols)
    scale = np.abs(base["kernel"]).max(axis=1) + 1e-30
    ks = np.zeros_like(scale)
    us = np.zeros_like(scale)
    try:
        for st in steps:
            lib().swdo_set_eigen_cpert(C.c_double(st * rel))
            r = get_1d_kernel(case, cols=cols)
            ks = np.maximum(ks, np.abs(r["kernel"] - base["kernel"]).max(axis=1) / scale)
            us = np.maximum(us, np.abs(r["vout"] - base["vout"]))
    finally:
        lib().swdo_set_eigen_cpert(C.c_double(0.0))
    return ks, us


def kernel_at(case, col, rel):
    """get_1d_kernel of one column with every phase velocity handed to the
    eigenfunction routines moved by the relative amount `rel`: the oracle's
    kernels at another implementation's root when the two roots differ by
    rel (one REAL*4 ulp after sngl())."""
    try:
        lib().swdo_set_eigen_cpert(C.c_double(rel))
        return get_1d_kernel(case, cols=np.array([col]))
    finally:
        lib().swdo_set_eigen_cpert(C.c_double(0.0))


def group_root_spread(case, cols):
    """Sensitivity of the oracle's group kernels to the REAL*4 rounding of
    their hidden roots c1, c2 at T(1 +- 0.005): the largest kernel change
    (relative to the slot's largest |kernel|) per (slot, column) when c1 or
    c2 alone moves by one REAL*4 ulp either way.  sregnpu/slegnpu difference
    the phase kernels at c1 and c2 over a 1 % period step, so a one-ulp
    change of one of them moves the group kernel about 100 times as much as
    the same change of c; phase slots do not move."""
    base = get_1d_kernel(case, cols=cols)
    scale = np.abs(base["kernel"]).max(axis=1) + 1e-30
    ks = np.zeros_like(scale)
    try:
        for u in ((-1, 0), (1, 0), (0, -1), (0, 1)):
            lib().swdo_set_group_ulp(u[0], u[1])
            r = get_1d_kernel(case, cols=cols)
            ks = np.maximum(ks, np.abs(r["kernel"] - base["kernel"]).max(axis=1) / scale)
    finally:
        lib().swdo_set_group_ulp(0, 0)
    return ks


def map_spread(case, cols, rel=1e-15, steps=(-3, -1, 1, 3)):
    """The same conditioning probe for get_2d_map: the largest change of vout
    (km/s) per (slot, column) when the phase velocity handed to
    sregn96/slegn96 moves by s*rel relative."""
    base = get_2d_map(case, cols=cols)
    us = np.zeros_like(base["vout"])
    try:
        for st in steps:
            lib().swdo_set_eigen_cpert(C.c_double(st * rel))
            r = get_2d_map(case, cols=cols)
            us = np.maximum(us, np.abs(r["vout"] - base["vout"]))
    finally:
        lib().swdo_set_eigen_cpert(C.c_double(0.0))
    return us


def get_2d_map(case, refine=1, rtol=1e-10, sngl=1, sphere=1, nthreads=0, cols=None):
    from jdsurfg_b200.synth import subset_columns
    if cols is not None:
        case = subset_columns(case, cols)
    vs = case["vs"]
    nz, ncol = vs.shape
    targs, keep = _table_args(case["tables"])
    kmax = _kmax(case["tables"])
    vc, vo = np.zeros((kmax, ncol)), np.zeros((kmax, ncol))
    st = np.zeros((kmax, ncol), np.int32)
    nev = C.c_long(0)
    lib().swdo_get_2d_map(ncol, nz, _ptr(vs), _ptr(case["vp"]), _ptr(case["rho"]), _ptr(case["depth"]), *targs,
                          _ptr(vc), _ptr(vo), _ptr(st), refine, C.c_double(rtol), sngl, sphere, nthreads,
                          C.byref(nev))
    return dict(vc=vc, vout=vo, status=st, nevals=nev.value)


def frechet_rows(nx, ny, nz, kernel, row_slot, fdm):
    """Frechet rows (SurfaceWave.cpp:590-676): list of (indices, values)."""
    kmax = kernel.shape[0]
    kernel = np.ascontiguousarray(kernel, np.float64)
    row_slot = np.ascontiguousarray(row_slot, np.int32)
    fdm = np.ascontiguousarray(fdm, np.float32)
    nrows = len(row_slot)
    n = (nx - 2) * (ny - 2) * (nz - 1)
    nnz = np.zeros(nrows, np.int32)
    idx = np.zeros(nrows * n, np.int32)
    val = np.zeros(nrows * n, np.float32)
    lib().swdo_frechet_rows(nx, ny, nz, kmax, _ptr(kernel), nrows, _ptr(row_slot), _ptr(fdm), _ptr(nnz), _ptr(idx),
                            _ptr(val))
    rows = []
    for r in range(nrows):
        rows.append((idx[r * n:r * n + nnz[r]].copy(), val[r * n:r * n + nnz[r]].copy()))
    return rows


def group_u_spread(case, col, group_wave, periods, k, rel=1e-15, steps=(-3, -1, 1, 3)):
    """Conditioning of the reference's kernel-path group velocity: the range
    of sregnpu_/slegnpu_'s U (flat) at period periods[k] when the phase
    velocity input moves by a few `rel` relative steps.  group_wave: "Rg" or
    "Lg".  Returns (U at the root, max |U(c(1+s*rel)) - U(c)|)."""
    from jdsurfg_b200 import synth
    vs = case["vs"][:, col]
    if case["vp"] is None:
        vp, rho = synth.brocher(vs)
    else:
        vp, rho = case["vp"][:, col], case["rho"][:, col]
    th, a, b, r = grid2layer(case["depth"], vp, vs, rho)
    iw = 2 if group_wave == "Rg" else 1
    T = np.asarray(periods, np.float64)
    c0 = surfdisp96(th, a, b, r, 1, iw, 1, 0, T, refine=1)[0][k]
    c1 = surfdisp96(th, a, b, r, 1, iw, 1, 0, T * 1.005, refine=1)[0][k]
    c2 = surfdisp96(th, a, b, r, 1, iw, 1, 0, T * 0.995, refine=1)[0][k]
    n = len(th)
    th, a, b, r = f32(th), f32(a), f32(b), f32(r)
    out = []
    for s in (0,) + tuple(steps):
        bufs = [np.zeros(n) for _ in range(12)]
        tt, cp, cg = C.c_double(T[k]), C.c_double(c0 * (1 + s * rel)), C.c_double(0)
        t1, cc1, t2, cc2 = C.c_double(T[k] * 1.005), C.c_double(c1), C.c_double(T[k] * 0.995), C.c_double(c2)
        if iw == 2:
            lib().sregnpu_(_ptr(th), _ptr(a), _ptr(b), _ptr(r), n, C.byref(tt), C.byref(cp), C.byref(cg),
                           *[_ptr(x) for x in bufs[:4]], C.byref(t1), C.byref(cc1), C.byref(t2), C.byref(cc2),
                           *[_ptr(x) for x in bufs[4:]], 1)
        else:
            lib().slegnpu_(_ptr(th), _ptr(b), _ptr(r), n, C.byref(tt), C.byref(cp), C.byref(cg),
                           *[_ptr(x) for x in bufs[:2]], C.byref(t1), C.byref(cc1), C.byref(t2), C.byref(cc2),
                           *[_ptr(x) for x in bufs[2:8]], 1)
        out.append(cg.value)
    return out[0], max(abs(u - out[0]) for u in out[1:])


# ---------------------------------------------------------------------------
# Fast-marching traveltimes and ray-path weights (oracle/fmst_oracle.cpp)

def delsph(a, b, c, d):
    f = lib().oracle_delsph
    f.restype = C.c_float
    f.argtypes = [C.c_float] * 4
    return f(a, b, c, d)


def ref_delsph(a, b, c, d):
    """The reference's own src/shared/spherical.cpp delsph (oracle/_ref), or None."""
    r = ref_cxx()
    if r is None:
        return None
    r.delsph.restype = C.c_float
    r.delsph.argtypes = [C.c_float] * 4
    return r.delsph(a, b, c, d)


def fmst_pairs(grid, pairs, vc, vout, want_fdm=False, nthreads=0):
    """The per-pair loop of SurfTime::travel_time (want_fdm=False) or
    frechet_matrix (want_fdm=True).  grid = (nx, ny, goxd, gozd, dvxd, dvzd);
    pairs = dict(slot, srcx, srcz, rcv_ptr, rcx, rcz, group); vc, vout =
    (kmax, nx*ny) float64 maps.  Returns ttime (nrcv) and fdm (nrcv, ny, nx)
    float32 (None unless want_fdm)."""
    nx, ny, goxd, gozd, dvxd, dvzd = grid
    slot = np.ascontiguousarray(pairs["slot"], np.int32)
    srcx, srcz = f32(pairs["srcx"]), f32(pairs["srcz"])
    rptr = np.ascontiguousarray(pairs["rcv_ptr"], np.int64)
    rcx, rcz = f32(pairs["rcx"]), f32(pairs["rcz"])
    group = np.ascontiguousarray(pairs["group"], np.int32)
    vc = np.ascontiguousarray(vc, np.float64)
    vout = np.ascontiguousarray(vout, np.float64)
    nrcv = int(rptr[-1])
    tt = np.zeros(nrcv, np.float32)
    fdm = np.zeros((nrcv, ny, nx), np.float32) if want_fdm else None
    nthreads = nthreads or os.cpu_count()
    lib().oracle_fmst_pairs(nx, ny, C.c_float(goxd), C.c_float(gozd), C.c_float(dvxd), C.c_float(dvzd), len(slot),
                            _ptr(slot), _ptr(srcx), _ptr(srcz), _ptr(rptr), _ptr(rcx), _ptr(rcz), _ptr(group),
                            _ptr(vc), _ptr(vout), _ptr(tt), _ptr(fdm), nthreads)
    return tt, fdm


def fmst_field(grid, vmap, srcx, srcz):
    """Coarse traveltime field and node status after one fmst_run
    ((nnz, nnx) arrays, column-major flattened as [ix][iz])."""
    nx, ny, goxd, gozd, dvxd, dvzd = grid
    L = lib()
    L.fmst_init(nx, ny, C.c_float(goxd), C.c_float(gozd), C.c_float(dvxd), C.c_float(dvzd))
    rc = np.array([srcx], np.float32)
    rz = np.array([srcz], np.float32)
    tt = np.zeros(1, np.float32)
    L.fmst_run(_ptr(np.ascontiguousarray(vmap, np.float64)), C.c_float(srcx), C.c_float(srcz), _ptr(rc), _ptr(rz), 1,
               _ptr(tt))
    nnx, nnz = (nx - 3) * 8 + 1, (ny - 3) * 8 + 1
    t = np.zeros(nnx * nnz, np.float32)
    s = np.zeros(nnx * nnz, np.int32)
    L.oracle_fmst_field(_ptr(t), _ptr(s), nnx * nnz)
    L.fmst_finalize()
    return t.reshape(nnx, nnz), s.reshape(nnx, nnz)
