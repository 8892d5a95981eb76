"""The GPU's fast-marching code compiled for the CPU (tests/
fmst_march_host.cpp includes jdsurfg_b200/csrc/swdk_fmst_march.cuh): its
propagation-grid times and statuses and its receiver times must equal the
oracle's restatement of fmst.f90 / fmm.f90 bit for bit.  This checks the
marching logic (window solve, heap, refined grid, resampling) and the ray
tracer without a GPU; tests/test_gpu_fmst.py checks the device build."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import oracle_lib as O
from jdsurfg_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "fmst_march_host.cpp")
HDR = os.path.join(ROOT, "jdsurfg_b200", "csrc", "swdk_fmst_march.cuh")
OUT = os.path.join(ROOT, "tests", "_build", "libfm_host.so")


def _lib():
    if not os.path.exists(OUT) or max(os.path.getmtime(SRC), os.path.getmtime(HDR)) > os.path.getmtime(OUT):
        os.makedirs(os.path.dirname(OUT), exist_ok=True)
        subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-strict-aliasing", "-shared", "-fPIC",
                        "-I" + os.path.dirname(HDR), SRC, "-o", OUT], check=True)
    return C.CDLL(OUT)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _run(grid, pairs, vc, field_pair=0, mode=0):
    L = _lib()
    nx, ny, goxd, gozd, dvxd, dvzd = grid
    slot = np.ascontiguousarray(pairs["slot"], np.int32)
    srcx, srcz = np.ascontiguousarray(pairs["srcx"], np.float32), np.ascontiguousarray(pairs["srcz"], np.float32)
    rptr = np.ascontiguousarray(pairs["rcv_ptr"], np.int64)
    rcx, rcz = np.ascontiguousarray(pairs["rcx"], np.float32), np.ascontiguousarray(pairs["rcz"], np.float32)
    vc = np.ascontiguousarray(vc, np.float64)
    nnx, nnz = (nx - 3) * 8 + 1, (ny - 3) * 8 + 1
    tt = np.zeros(int(rptr[-1]), np.float32)
    ft = np.zeros(nnx * nnz, np.float32)
    fs = np.zeros(nnx * nnz, np.int32)
    L.fm_host_pairs.restype = C.c_int
    band = L.fm_host_pairs(mode, nx, ny, C.c_float(goxd), C.c_float(gozd), C.c_float(dvxd), C.c_float(dvzd), len(slot),
                           _p(slot), _p(srcx), _p(srcz), _p(rptr), _p(rcx), _p(rcz), _p(vc), _p(tt), field_pair,
                           _p(ft), _p(fs))
    return tt, ft.reshape(nnx, nnz), fs.reshape(nnx, nnz), band


def _survey(**kw):
    s = synth.make_survey("example", **kw)
    slot, group = synth.survey_slots(s)
    p = s["pairs"]
    pairs = dict(slot=slot, srcx=p["srcx"], srcz=p["srcz"], group=np.zeros_like(group), rcv_ptr=p["rcv_ptr"],
                 rcx=p["rcx"], rcz=p["rcz"])
    return s, pairs


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("kw", [dict(nx=14, ny=16, nstation=10, nperiod=2, seed=11),
                                dict(nstation=6, nperiod=1, seed=4)])
def test_gpu_marching_code_matches_oracle(kw, mode):
    """mode 0: the one-lane window march; mode 1: each neighbour solved from
    its own stencil, the per-lane work of the four-lane march."""
    s, pairs = _survey(**kw)
    m = O.get_2d_map(s["case"])
    tt, ft, fs, band = _run(s["grid"], pairs, m["vc"], field_pair=1, mode=mode)
    assert band > 0
    ref, _ = O.fmst_pairs(s["grid"], pairs, m["vc"], m["vout"])
    assert np.array_equal(tt, ref)
    rt, rs = O.fmst_field(s["grid"], m["vc"][pairs["slot"][1]], float(pairs["srcx"][1]), float(pairs["srcz"][1]))
    assert np.array_equal(fs == 0, rs == 0) and (fs == 0).all()
    assert np.array_equal(ft, rt)


def _edge_pairs(grid, d2r=np.float32(np.pi / 180)):
    """Sources on propagation-grid nodes (a homogeneous model then gives
    exactly equal times in symmetric directions, so the heap's order among
    ties decides the result) and next to each side and corner of the grid
    (the refined source grid then reaches the model's sides)."""
    nx, ny, lat0, lon0, dl, _ = grid
    # the propagation grid spans model nodes 1 .. nx-2 (lat) and 1 .. ny-2 (lon)
    lat_lo, lat_hi = lat0 - (nx - 2) * dl, lat0 - dl
    lon_lo, lon_hi = lon0 + dl, lon0 + (ny - 2) * dl
    e = 0.02 * dl
    srcs = [(lat0 - 5 * dl, lon0 + 6 * dl), (lat0 - 5 * dl - dl / 8, lon0 + 6 * dl + dl / 8),
            (lat_hi - e, lon0 + 5 * dl), (lat_lo + e, lon0 + 5 * dl), (lat0 - 4 * dl, lon_lo + e),
            (lat0 - 4 * dl, lon_hi - e), (lat_hi - e, lon_lo + e), (lat_lo + e, lon_hi - e)]
    rng = np.random.default_rng(3)
    rlat = np.concatenate([rng.uniform(lat_lo + e, lat_hi - e, 10), [lat_lo + e, lat_hi - e, lat0 - 5 * dl]])
    rlon = np.concatenate([rng.uniform(lon_lo + e, lon_hi - e, 10), [lon_hi - e, lon_lo + e, lon0 + 6 * dl]])
    col = lambda lat: np.float32((np.float32(90.0) - np.float32(lat)) * d2r)
    lon = lambda x: np.float32(np.float32(x) * d2r)
    pairs = dict(slot=np.zeros(len(srcs), np.int32), srcx=np.array([col(a) for a, _ in srcs], np.float32),
                 srcz=np.array([lon(b) for _, b in srcs], np.float32), group=np.zeros(len(srcs), np.int32),
                 rcv_ptr=np.arange(len(srcs) + 1, dtype=np.int64) * len(rlat),
                 rcx=np.tile([col(a) for a in rlat], len(srcs)).astype(np.float32),
                 rcz=np.tile([lon(b) for b in rlon], len(srcs)).astype(np.float32))
    return pairs


@pytest.mark.parametrize("mode", [0, 1])
def test_ties_and_grid_sides_match_oracle(mode):
    grid = (14, 16, 40.0, 100.0, 0.3, 0.3)
    nx, ny = grid[:2]
    pairs = _edge_pairs(grid)
    for v in (np.full((1, nx * ny), 3.0), 3.0 + 0.3 * np.sin(np.arange(nx * ny))[None, :]):
        tt, _, _, band = _run(grid, pairs, v, field_pair=0, mode=mode)
        assert band > 0
        ref, _ = O.fmst_pairs(grid, pairs, v, v)
        assert not np.isnan(ref).any()
        assert np.array_equal(tt, ref)
        for p in (0, 1, 2, 6):
            _, ft, fs, _ = _run(grid, pairs, v, field_pair=p, mode=mode)
            rt, rs = O.fmst_field(grid, v[0], float(pairs["srcx"][p]), float(pairs["srcz"][p]))
            assert np.array_equal(ft, rt) and (fs == 0).all()


def _rays(grid, pairs, vc, vout, sine):
    L = _lib()
    nx, ny, goxd, gozd, dvxd, dvzd = grid
    a32 = lambda k: np.ascontiguousarray(pairs[k], np.int32)
    f32 = lambda k: np.ascontiguousarray(pairs[k], np.float32)
    slot, group, rptr = a32("slot"), a32("group"), np.ascontiguousarray(pairs["rcv_ptr"], np.int64)
    srcx, srcz, rcx, rcz = f32("srcx"), f32("srcz"), f32("rcx"), f32("rcz")
    vc, vout = np.ascontiguousarray(vc, np.float64), np.ascontiguousarray(vout, np.float64)
    nrcv = int(rptr[-1])
    tt = np.zeros(nrcv, np.float32)
    fdm = np.zeros((nrcv, ny, nx), np.float32)
    L.fm_host_rays.restype = C.c_int
    rc = L.fm_host_rays(sine, nx, ny, C.c_float(goxd), C.c_float(gozd), C.c_float(dvxd), C.c_float(dvzd), len(slot),
                        _p(slot), _p(srcx), _p(srcz), _p(group), _p(rptr), _p(rcx), _p(rcz), _p(vc), _p(vout),
                        _p(tt), _p(fdm))
    assert rc == 0
    return tt, fdm


def test_gpu_ray_code_matches_oracle_up_to_the_sine():
    """The GPU's ray tracer (srtimes, raypath with its Frechet weights and the
    group traveltime along the ray) on the CPU: with the C library's sinf for
    the ray points, as the reference and the oracle use, its times and
    weights are the oracle's bit for bit; with the device's sine (double,
    rounded) they stay within the tolerances tests/test_gpu_fmst.py states
    for the GPU (2e-6 of a ray time, 1e-4 of a row's largest weight)."""
    s = synth.make_survey("example", nx=14, ny=16, nstation=10, nperiod=2, seed=11)
    slot, group = synth.survey_slots(s)
    p = s["pairs"]
    pairs = dict(slot=slot, srcx=p["srcx"], srcz=p["srcz"], group=group, rcv_ptr=p["rcv_ptr"], rcx=p["rcx"],
                 rcz=p["rcz"])
    m = O.get_2d_map(s["case"])
    ref_t, ref_f = O.fmst_pairs(s["grid"], pairs, m["vc"], m["vout"], want_fdm=True)
    t0, f0 = _rays(s["grid"], pairs, m["vc"], m["vout"], sine=0)
    assert np.array_equal(t0, ref_t) and np.array_equal(f0, ref_f)
    t1, f1 = _rays(s["grid"], pairs, m["vc"], m["vout"], sine=1)
    grp = np.repeat(group, np.diff(p["rcv_ptr"])).astype(bool)
    assert np.array_equal(t1[~grp], ref_t[~grp])
    assert np.max(np.abs(t1[grp] - ref_t[grp]) / ref_t[grp]) <= 2e-6
    scale = np.abs(ref_f).reshape(len(ref_t), -1).max(axis=1)
    assert np.max(np.abs(f1 - ref_f).reshape(len(ref_t), -1).max(axis=1) / scale) <= 1e-4
