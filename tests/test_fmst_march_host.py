"""The GPU's fast-marching code compiled for the CPU (tests/
fmst_march_host.cpp includes jdsurfg_b200/csrc/swdk_fmst_march.cuh): its
propagation-grid times and statuses and its receiver times must equal the
oracle's restatement of fmst.f90 / fmm.f90 bit for bit.  This checks the
marching logic (window solve, heap, refined grid, resampling) without a
GPU; tests/test_gpu_fmst.py checks the device build."""
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
