"""The root search's chain state machine compiled for the CPU
(tests/chain_host.cpp includes jdsurfg_b200/csrc/swdk_core.cuh) with
planted bracket proposals: wherever a proposal puts the first period's
cell of a Rayleigh chain (on the root, far above it, below it, beyond the
largest shear velocity) and whatever it proposes for the later periods, the
roots and statuses are the plain scan's bits.  On the root the first
period needs a fraction of the plain scan's evaluations; far above it a
checked grid point finds the sign change and the scan resumes below it
(counted as a fallback).  The GPU tests check the same on the device with
the trained networks (tests/test_gpu_learned.py)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import oracle_lib as O
from jdsurfg_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "chain_host.cpp")
HDR = os.path.join(ROOT, "jdsurfg_b200", "csrc", "swdk_core.cuh")
OUT = os.path.join(ROOT, "tests", "_build", "libchain_host.so")


def _lib():
    if not os.path.exists(OUT) or max(os.path.getmtime(SRC), os.path.getmtime(HDR)) > os.path.getmtime(OUT):
        os.makedirs(os.path.dirname(OUT), exist_ok=True)
        cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
        subprocess.run(["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-I" + os.path.dirname(HDR),
                        "-I" + cuda_inc, SRC, "-o", OUT], check=True)
    L = C.CDLL(OUT)
    L.chain_host_run.restype = C.c_int
    return L


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _models(n, seed=2024):
    """Flat layer models of the default grid's columns (4 sublayers per node
    interval), their periods, scan start and largest shear velocity."""
    case = synth.make_config("large", seed=seed)
    z = np.asarray(case["depth"], np.float64)
    per = np.ascontiguousarray(case["tables"][0][:, 0], np.float64)
    out = []
    for col in range(n):
        vs = np.asarray(case["vs"][:, col], np.float32)
        vp, rho = synth.brocher(vs)
        thk, a, b, r = (np.ascontiguousarray(x, np.float32) for x in O.grid2layer(z, vp, vs, rho))
        cc = 0.95 * 0.90 * 0.92 * float(b.min())  # below every root of the chain
        out.append((thk, a, b, r, cc, np.float32(b.max())))
    return per, out


def _run(model, per, iwave, prop=None):
    thk, a, b, r, cc, betmx = model
    n = len(per)
    roots = np.zeros(n)
    st = np.zeros(n, np.int32)
    ev, ok, fail = C.c_longlong(0), C.c_int(0), C.c_int(0)
    pr = None if prop is None else np.ascontiguousarray(prop, np.float32)
    ierr = _lib().chain_host_run(len(thk), _p(thk), _p(a), _p(b), _p(r), iwave, n, _p(per), 1, C.c_double(cc),
                                 C.c_float(betmx), _p(pr), _p(roots), _p(st), C.byref(ev), C.byref(ok),
                                 C.byref(fail))
    assert ierr >= 0
    return roots, st, ev.value, ok.value, fail.value


def _proposals(roots, first_shift, later_noise, rng):
    """(c, half-width) per period: the plain roots, moved by first_shift at
    the first period and by seeded noise of later_noise km/s after it."""
    c = roots + rng.normal(0.0, later_noise, len(roots)) if later_noise else roots.copy()
    c[0] = roots[0] + first_shift
    return np.stack([c, np.full(len(roots), 0.02)], axis=1).astype(np.float32)


@pytest.mark.parametrize("first_shift,later_noise", [(0.0, 0.0), (0.15, 0.0), (-0.15, 0.0), (0.03, 0.01),
                                                     (0.6, 0.0), (-0.04, 0.05), (2.5, 0.0)])
def test_planted_proposals_keep_the_plain_roots(first_shift, later_noise):
    per, models = _models(12)
    rng = np.random.default_rng(7)
    ev_plain = ev_prop = fails = 0
    for m in models:
        rp, sp, ep, _, _ = _run(m, per, 2)
        assert (sp == 0).all()
        rl, sl, el, ok, fail = _run(m, per, 2, _proposals(rp, first_shift, later_noise, rng))
        np.testing.assert_array_equal(rl, rp)
        np.testing.assert_array_equal(sl, sp)
        ev_plain += ep
        ev_prop += el
        fails += fail
    print(f"first-period shift {first_shift:+.2f} km/s, later noise {later_noise}: evaluations {ev_plain} plain, "
          f"{ev_prop} with proposals, {fails} fallbacks")
    if first_shift == 0.0 and later_noise == 0.0:
        assert ev_prop < 0.7 * ev_plain
    if 0.15 <= first_shift <= 0.6:  # above the root: caught by a checked point
        assert fails >= len(models) // 2
    if first_shift > 2.0:  # beyond the largest shear velocity: no jump, no fallback
        assert fails == 0


def test_love_chains_keep_the_first_period_scan():
    """Love chains take proposals from the second period on only: a first-
    period proposal on the root saves nothing there, and roots stay equal."""
    per, models = _models(6, seed=11)
    rng = np.random.default_rng(3)
    for m in models:
        rp, sp, ep, _, _ = _run(m, per, 1)
        exact = _proposals(rp, 0.0, 0.0, rng)
        rl, sl, el, _, _ = _run(m, per, 1, exact)
        far = _proposals(rp, 0.3, 0.0, rng)
        rf, sf, ef, _, _ = _run(m, per, 1, far)
        np.testing.assert_array_equal(rl, rp)
        np.testing.assert_array_equal(rf, rp)
        np.testing.assert_array_equal(sl, sp)
        assert el == ef  # the first period's proposal is not used
