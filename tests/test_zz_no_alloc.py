"""The allocation-free entry point swdk_surfdisp96_noalloc.

Some host programs manage all device memory themselves -- an inversion
driver running inside a fixed, pre-reserved memory budget, or a framework
whose own allocator must stay the only one -- and cannot let a library call
cudaMalloc or cudaFree (which also waits for the whole device) in the middle
of an iteration.  swdk_surfdisp96_noalloc serves them: inputs and outputs are
the caller's device buffers and all scratch is a fixed static device array.

This file is collected last so that a failure here cannot hide the results
of the other tests; it also passes when run alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from jdsurfg_b200 import Engine
from jdsurfg_b200.engine import lib

pytestmark = pytest.mark.gpu

TOL_C = 1e-6  # km/s against the oracle, as the other parity tests


def _models(n, L, seed):
    rng = np.random.default_rng(seed)
    thk = np.full((n, L), 0.55, np.float32)
    thk[:, -1] = 0
    vs = (np.linspace(2.5, 4.6, L)[None, :] * (1 + 0.04 * rng.standard_normal((n, L)))).astype(np.float32)
    vp = (1.75 * vs).astype(np.float32)
    rho = (0.32 * vp + 0.77).astype(np.float32)
    return thk, vp, vs, rho


def _noalloc(thk, vp, vs, rho, iwave, mode, t, refine=1):
    import torch
    dev = torch.device("cuda", 0)
    n, L = thk.shape
    d = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (thk, vp, vs, rho)]
    dt = torch.from_numpy(np.ascontiguousarray(t, np.float64)).to(dev)
    cg = torch.full((n, len(t)), -7.0, dtype=torch.float64, device=dev)  # stale values must be overwritten
    ierr = torch.full((n,), -7, dtype=torch.int32, device=dev)
    L_ = lib()
    L_.swdk_surfdisp96_noalloc.argtypes = [C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 4 + [C.c_int] * 5 + [
        C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_void_p]
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = L_.swdk_surfdisp96_noalloc(0, n, L, *[C.c_void_p(x.data_ptr()) for x in d], 1, iwave, mode, 0, len(t),
                                    C.c_void_p(dt.data_ptr()), C.c_void_p(cg.data_ptr()),
                                    C.c_void_p(ierr.data_ptr()), refine, 1e-10, 1, C.c_void_p(stream))
    torch.cuda.synchronize()
    return rc, cg.cpu().numpy(), ierr.cpu().numpy()


def _oracle(thk, vp, vs, rho, iwave, mode, t):
    """surfdisp96_ of every model by the CPU oracle (tight refinement, sngl output)."""
    cg = np.zeros((thk.shape[0], len(t)))
    ierr = np.zeros(thk.shape[0], np.int32)
    for i in range(thk.shape[0]):
        cg[i], ierr[i], _ = O.surfdisp96(thk[i], vp[i], vs[i], rho[i], 1, iwave, mode, 0, t, refine=1, rtol=1e-10,
                                         sngl=1)
    return cg, ierr


def test_noalloc_matches_batch_entry_point_and_oracle_twice():
    # first call: Rayleigh, two modes; one model with a NaN layer
    thk, vp, vs, rho = _models(96, 61, seed=1)
    vs[17, 9] = np.nan
    t = np.geomspace(2.0, 50.0, 14)
    rc, cg, ierr = _noalloc(thk, vp, vs, rho, 2, 2, t)
    assert rc == 0
    ref, rerr = Engine(refine=1).surfdisp96_batch(thk, vp, vs, rho, 1, 2, 2, 0, t)
    # the same chain code as the batch entry point: identical results
    np.testing.assert_array_equal(cg, ref)
    np.testing.assert_array_equal(ierr, rerr)
    # the NaN model: ierr set, every period zero
    assert ierr[17] == 1 and (cg[17] == 0.0).all()
    ok = np.ones(len(thk), bool)
    ok[17] = False
    oc, oerr = _oracle(thk[ok], vp[ok], vs[ok], rho[ok], 2, 2, t)
    np.testing.assert_array_equal(ierr[ok], oerr)
    assert np.abs(cg[ok] - oc).max() <= TOL_C
    # second call in a row, different sizes and wave type: nothing stale
    thk, vp, vs, rho = _models(40, 37, seed=2)
    t = np.geomspace(3.0, 30.0, 9)
    rc, cg, ierr = _noalloc(thk, vp, vs, rho, 1, 1, t)
    assert rc == 0
    ref, rerr = Engine(refine=1).surfdisp96_batch(thk, vp, vs, rho, 1, 1, 1, 0, t)
    np.testing.assert_array_equal(cg, ref)
    np.testing.assert_array_equal(ierr, rerr)
    oc, oerr = _oracle(thk, vp, vs, rho, 1, 1, t)
    np.testing.assert_array_equal(ierr, oerr)
    assert np.abs(cg - oc).max() <= TOL_C


def test_noalloc_rejects_calls_beyond_its_scratch():
    # 32*nlayer*nmodel alone exceeds the 64 MiB scratch: rejected, nothing run
    thk, vp, vs, rho = _models(8192, 300, seed=3)
    rc, cg, _ = _noalloc(thk, vp, vs, rho, 2, 1, np.array([5.0, 10.0]))
    assert rc == -5  # SWDK_E_LIMIT
    assert (cg == -7.0).all()
