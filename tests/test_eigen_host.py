"""The GPU's eigenfunction / energy-integral passes compiled for the CPU
(tests/eigen_host.cpp includes jdsurfg_b200/csrc/swdk_eigen.cuh): group
velocity and raw layer kernels of the Rayleigh and Love passes against the
oracle's sregn96 / slegn96 (restatements of sregn96.f90 / slegn96.f90) at
the oracle's own roots, on flat layer models of the bench's depth grid, the
reference's test model and a model with a water layer.  This checks the
passes' arithmetic without a GPU; tests/test_gpu_parity.py checks the device
build end to end."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import oracle_lib as O
from jdsurfg_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "eigen_host.cpp")
CSRC = os.path.join(ROOT, "jdsurfg_b200", "csrc")
HDRS = [os.path.join(CSRC, h) for h in ("swdk_eigen.cuh", "swdk_core.cuh")]
OUT = os.path.join(ROOT, "tests", "_build", "libeig_host.so")

# relative to the largest |kernel| of the pass; group velocity relative
TOL_K = 1e-9
TOL_U = 1e-11


def _lib():
    if not os.path.exists(OUT) or max(os.path.getmtime(f) for f in [SRC] + HDRS) > os.path.getmtime(OUT):
        os.makedirs(os.path.dirname(OUT), exist_ok=True)
        cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
        subprocess.run(["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-I" + CSRC, "-I" + cuda_inc, SRC, "-o", OUT],
                       check=True)
    L = C.CDLL(OUT)
    L.eig_host_pass.restype = C.c_int
    return L


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def host_pass(wave, thk, vp, vs, rho, t, c, sphere=0, trunc_q=0.0):
    f = lambda a: np.ascontiguousarray(a, np.float32)
    thk, vp, vs, rho = f(thk), f(vp), f(vs), f(rho)
    L = len(thk)
    ugr, norm = C.c_double(0), C.c_double(0)
    da, db, dr = np.zeros(L), np.zeros(L), np.zeros(L)
    rc = _lib().eig_host_pass(wave, L, _p(thk), _p(vp), _p(vs), _p(rho), sphere, C.c_double(t), C.c_double(c),
                              C.c_double(trunc_q), C.byref(ugr), C.byref(norm), _p(da), _p(db), _p(dr))
    assert rc == 0
    return ugr.value, norm.value, da, db, dr


def _models():
    """Flat layer models: columns of the bench's 64-node grid (one with the
    low-velocity zone), the reference's kernel-test model and a water layer
    over the first column."""
    out = []
    case = synth.make_config("large", nx=4, ny=4, seed=77)
    for col in (0, 5, 11):
        vs = case["vs"][:, col]
        vp, rho = synth.brocher(vs)
        out.append(O.grid2layer(case["depth"], vp, vs, rho))
    z, vs, vp, rho = O.load_swd_model()
    out.append(O.grid2layer(z, vp, vs, rho))
    th, a, b, r = out[0]
    out.append((np.concatenate([[2.0], th]).astype(np.float32), np.concatenate([[1.5], a]).astype(np.float32),
                np.concatenate([[0.0], b]).astype(np.float32), np.concatenate([[1.03], r]).astype(np.float32)))
    return out


PERIODS = np.array([1.0, 2.5, 6.0, 15.0, 40.0, 80.0])


@pytest.mark.parametrize("wave", [2, 1], ids=["rayleigh", "love"])
def test_eigen_passes_match_oracle_flat(wave):
    worst_k = worst_u = 0.0
    n = 0
    for mi, (th, a, b, r) in enumerate(_models()):
        for mode in (1, 2):
            cg, ierr, _ = O.surfdisp96(th, a, b, r, 0, wave, mode, 0, PERIODS, refine=1, rtol=1e-12, sngl=0)
            for t, c in zip(PERIODS, cg):
                if c == 0.0:
                    continue
                ugr, norm, da, db, dr = host_pass(wave, th, a, b, r, t, c)
                if wave == 2:
                    ref = O.sregn96(th, a, b, r, t, c, iflsph=0)
                    got = np.concatenate([da, db, dr]) / norm
                    exp = np.concatenate([ref["dcda"], ref["dcdb"], ref["dcdr"]])
                else:
                    ref = O.slegn96(th, b, r, t, c, iflsph=0)
                    got = np.concatenate([db, dr]) / norm
                    exp = np.concatenate([ref["dcdb"], ref["dcdr"]])
                ek = np.abs(got - exp).max() / np.abs(exp).max()
                eu = abs(ugr - ref["u"]) / abs(ref["u"])
                worst_k, worst_u = max(worst_k, ek), max(worst_u, eu)
                n += 1
                assert ek <= TOL_K, (mi, mode, t, c, ek)
                assert eu <= TOL_U, (mi, mode, t, c, eu)
    assert n >= 40
    print(f"{n} passes: max kernel rel err {worst_k:.2e}, max |dU|/U {worst_u:.2e}")


@pytest.mark.parametrize("wave", [2, 1], ids=["rayleigh", "love"])
def test_depth_truncation_changes_nothing_measurable(wave):
    """The device passes cut the layers below exp(-40) of the S-wave decay
    from the top (swdk_eigen.cuh pass_layers): against the full-depth pass,
    group velocity and kernels agree to rounding (1e-12), and short periods cut
    layers."""
    worst = 0.0
    cut = 0
    for th, a, b, r in _models()[:3]:
        cg, _, _ = O.surfdisp96(th, a, b, r, 1, wave, 1, 0, PERIODS, refine=1, rtol=1e-12, sngl=0)
        for t, c in zip(PERIODS, cg):
            u0, n0, a0, b0, r0 = host_pass(wave, th, a, b, r, t, c, sphere=1, trunc_q=0.0)
            u1, n1, a1, b1, r1 = host_pass(wave, th, a, b, r, t, c, sphere=1, trunc_q=40.0)
            k0 = np.concatenate([a0, b0, r0]) / n0
            k1 = np.concatenate([a1, b1, r1]) / n1
            worst = max(worst, np.abs(k1 - k0).max() / np.abs(k0).max(), abs(u1 - u0) / abs(u0))
            cut += int((np.concatenate([a1, b1, r1]) == 0).sum() > (np.concatenate([a0, b0, r0]) == 0).sum())
    print(f"truncated vs full: max rel diff {worst:.2e}, {cut} passes cut")
    assert worst <= 1e-12
    assert cut >= 3


@pytest.mark.parametrize("wave", [2, 1], ids=["rayleigh", "love"])
def test_node_sums_equal_per_layer_accumulation(wave):
    """The kernel's node sums (NodeSink: the two nodes of the current
    interval held while the sweep passes them, each stored once) equal a
    per-layer kp[n] += w * (...) accumulation bit for bit, with and without
    a merged fluid layer and with the depth truncation cutting the sweep."""
    L_ = _lib()
    L_.eig_host_nodesums.restype = C.c_int
    rng = np.random.default_rng(5)
    f = lambda a: np.ascontiguousarray(a, np.float32)
    nchecked = 0
    for mi, (th, a, b, r) in enumerate(_models()[:3] + _models()[4:]):
        L = len(th)
        nw = 1 if mi == 3 else 0
        nz = (L + 3) // 4 if nw == 0 else (L - 2) // 4 + 1 + nw
        crs = f(rng.uniform(0.5, 2.0, 2 * nz))
        cg, _, _ = O.surfdisp96(th, a, b, r, 0, wave, 1, 0, PERIODS, refine=1, rtol=1e-12, sngl=0)
        for t, c in zip(PERIODS, cg):
            if c == 0.0:
                continue
            for q in (0.0, 40.0):
                kp, kref = np.zeros(nz), np.zeros(nz)
                rc = L_.eig_host_nodesums(wave, L, _p(f(th)), _p(f(a)), _p(f(b)), _p(f(r)), nw, nz, _p(crs),
                                          C.c_double(t), C.c_double(c), C.c_double(q), _p(kp), _p(kref))
                assert rc == 0
                np.testing.assert_array_equal(kp.view(np.int64), kref.view(np.int64))
                nchecked += 1
    assert nchecked >= 20
