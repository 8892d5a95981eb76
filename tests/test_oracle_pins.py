"""Pins of the CPU oracle (the checker) against the reference's own test,
the reference's own C++ wrapper code, analytic known answers and physics
identities.  CPU only."""
import os

import numpy as np
import pytest
from scipy.optimize import brentq

import oracle_lib as O
from jdsurfg_b200 import synth

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_halfspace_rayleigh_root_analytic():
    # homogeneous half-space: the Rayleigh root of (2-k^2)^2 = 4 sqrt(1-g^2k^2) sqrt(1-k^2)
    a, b = 6.0, 3.5
    thk, vp, vs, rho = [2.0, 0.0], [a, a], [b, b], [2.75, 2.75]
    t = np.array([2.0, 10.0, 50.0])
    c, ierr, _ = O.surfdisp96(thk, vp, vs, rho, 0, 2, 1, 0, t, refine=1, rtol=1e-12, sngl=0)
    f = lambda cr: (2 - (cr / b) ** 2) ** 2 - 4 * np.sqrt(1 - (cr / a) ** 2) * np.sqrt(1 - (cr / b) ** 2)
    cr = brentq(f, 0.5 * b, 0.999 * b, xtol=1e-15)
    assert ierr == 0
    assert np.abs(c - cr).max() < 1e-10
    # the reference's own stop (|c1-c2| <= 1e-6 c1, surfdisp96.f:634) is ~1e-6 relative
    c0, _, _ = O.surfdisp96(thk, vp, vs, rho, 0, 2, 1, 0, t, refine=0, sngl=0)
    assert np.abs(c0 - cr).max() < 1e-6 * cr


def test_love_layer_over_halfspace_analytic():
    H, b1, b2, r1, r2 = 10.0, 3.0, 4.0, 2.5, 3.0  # float-exact values
    thk, vs, rho = [H, 0.0], [b1, b2], [r1, r2]
    vp = [5.5, 7.0]
    t = np.array([2.0, 5.0, 10.0, 30.0, 60.0])
    c, ierr, _ = O.surfdisp96(thk, vp, vs, rho, 0, 1, 1, 0, t, refine=1, rtol=1e-12, sngl=0)
    mu1, mu2 = r1 * b1 * b1, r2 * b2 * b2
    for T, cv in zip(t, c):
        w = 2 * np.pi / T
        f = lambda cc: np.tan(w * H * np.sqrt(1 / b1 ** 2 - 1 / cc ** 2)) - mu2 * np.sqrt(1 / cc ** 2 - 1 / b2 ** 2) / (
            mu1 * np.sqrt(1 / b1 ** 2 - 1 / cc ** 2))
        s1p = np.pi / 2 / (w * H)
        hi = 1 / np.sqrt(1 / b1 ** 2 - s1p ** 2) if 1 / b1 ** 2 - s1p ** 2 > 0 else b2
        cr = brentq(f, b1 * (1 + 1e-12), min(hi * (1 - 1e-12), b2 * (1 - 1e-12)), xtol=1e-15)
        assert abs(cv - cr) < 1e-9, (T, cv, cr)


def _layered(seed=3, L=40):
    rng = np.random.default_rng(seed)
    thk = np.full(L, 0.5, np.float32)
    thk[-1] = 0
    vs = (np.linspace(2.5, 4.5, L) * (1 + 0.03 * rng.standard_normal(L))).astype(np.float32)
    vp = (1.75 * vs).astype(np.float32)
    rho = (0.32 * vp + 0.77).astype(np.float32)
    return thk, vp, vs, rho


@pytest.mark.skipif(O.ref_cxx() is None, reason="oracle/_ref (reference C++ wrapper) not built")
def test_wrapper_matches_reference_cpp():
    """The oracle's restatement of surfdisp()/groupvel_*() against the
    reference's own surfdisp.cpp compiled unchanged (oracle/_ref)."""
    import ctypes as C
    ref = O.ref_cxx()
    thk, vp, vs, rho = _layered()
    L = len(thk)
    t = np.geomspace(2, 60, 20)
    p = O._ptr
    for wt in range(4):
        for keep in (0, 1):
            for mode in (0, 1):
                a = np.zeros(20)
                ref.ref_surfdisp(p(thk), p(vp), p(vs), p(rho), L, p(t), p(a), 20, wt, mode, 1, keep)
                b, _ = O.surfdisp(thk, vp, vs, rho, t, wt, mode=mode, sphere=1, keep_flat=keep, refine=0)
                assert np.array_equal(a, b), (wt, keep, mode)
    a = np.zeros(20)
    ref.ref_groupvel_r(p(thk), p(vp), p(vs), p(rho), L, p(t), p(a), 20, 0, 1)
    b = np.zeros(20)
    cp, _ = O.surfdisp(thk, vp, vs, rho, t, 0, keep_flat=1, refine=0)
    for i in range(20):
        b[i] = O.sregn96(thk, vp, vs, rho, t[i], cp[i])["u"]
    assert np.array_equal(a, b)
    vsr = np.linspace(0.0, 4.8, 97).astype(np.float32)
    v1, r1 = np.zeros(97, np.float32), np.zeros(97, np.float32)
    ref.ref_empirical_relation(p(vsr), p(v1), p(r1), 97)
    import ctypes
    v2, r2 = np.zeros(97, np.float32), np.zeros(97, np.float32)
    O.lib().swdo_empirical_relation(p(vsr), p(v2), p(r2), 97)
    assert np.array_equal(v1, v2) and np.array_equal(r1, r2)


def _fd_node_kernels(z, vs, vp, rho, t, wt, par, dv=0.01):
    nz = len(z)
    fd = np.zeros((len(t), nz))
    for iz in range(nz):
        arr = {"vs": vs.copy(), "vp": vp.copy(), "rho": rho.copy()}
        v0 = arr[par][iz]
        out = []
        for s in (-0.5, 0.5):
            arr[par][iz] = v0 * (1 + s * dv)
            th, a, b, r = O.grid2layer(z, arr["vp"], arr["vs"], arr["rho"])
            c, _ = O.surfdisp(th, a, b, r, t, wt, sphere=1, keep_flat=0, refine=1, rtol=1e-13, sngl=0)
            out.append(c)
        fd[:, iz] = (out[1] - out[0]) / (v0 * dv)
    return fd


@pytest.mark.parametrize("wt,tol", [(0, 2e-4), (1, 1.5e-2), (2, 2e-4), (3, 1.5e-2)])
def test_reference_fd_kernel_check(wt, tol):
    """test/swd/main.cpp of the reference: analytic node kernels against central
    differences of surfdisp (+-0.5 % per node) on the reference's model.txt.
    Phase kernels agree to ~2e-5, group kernels to ~0.5 % (surfdisp's numerical
    group velocity and sregnpu's period stencil differ)."""
    z, vs, vp, rho = O.load_swd_model()
    t = 4.0 + 2.0 * np.arange(0, 19, 3)
    tabs = [None] * 4
    tabs[wt] = t[:, None]
    r = O.kernel1d(vs, vp, rho, z, tabs, refine=1, rtol=1e-13, sngl=0)
    pars = [("vs", r["kvs"]), ("rho", r["krho"])] + ([("vp", r["kvp"])] if wt < 2 else [])
    for par, K in pars:
        fd = _fd_node_kernels(z, vs, vp, rho, t, wt, par)
        rel = np.abs(K[:, :-1] - fd[:, :-1]).max(axis=1) / np.abs(fd[:, :-1]).max(axis=1)
        assert rel.max() < tol, (par, rel)


def test_flat_kernel_homogeneity_identities():
    """Flat-earth layer kernels obey exact scaling identities: scaling all
    velocities and thicknesses by s scales c by s, so
    sum(a dc/da + b dc/db) + sum(h dc/dh_i) = c; scaling density leaves c
    unchanged, so sum(rho dc/drho) = 0.  (dc/dh here is per layer thickness.)"""
    thk, vp, vs, rho = _layered(5)
    for T in (3.0, 12.0, 40.0):
        cp, _, _ = O.surfdisp96(thk, vp, vs, rho, 0, 2, 1, 0, np.array([T]), refine=1, rtol=1e-13, sngl=0)
        r = O.sregn96(thk, vp, vs, rho, T, cp[0], iflsph=0)
        c = r["c"]
        s_v = np.sum(vp * r["dcda"] + vs * r["dcdb"])
        s_h = np.sum(thk[:-1] * r["dcdh"][:-1])
        assert abs(s_v + s_h - c) < 2e-6 * c, (T, s_v + s_h, c)
        assert abs(np.sum(rho * r["dcdr"])) < 2e-6 * c
        cp, _, _ = O.surfdisp96(thk, vp, vs, rho, 0, 1, 1, 0, np.array([T]), refine=1, rtol=1e-13, sngl=0)
        r = O.slegn96(thk, vs, rho, T, cp[0], iflsph=0)
        c = r["c"]
        s_v = np.sum(vs * r["dcdb"])
        s_h = np.sum(thk[:-1] * r["dcdh"][:-1])
        assert abs(s_v + s_h - c) < 2e-6 * c, (T, s_v + s_h, c)
        assert abs(np.sum(rho * r["dcdr"])) < 2e-6 * c


def test_energy_group_velocity_matches_dispersion_derivative():
    """U from the energy integrals (sregn96/slegn96 ugr) against U = dw/dk of
    the tight FP64 dispersion curve (flat earth)."""
    thk, vp, vs, rho = _layered(9)
    for iwave in (1, 2):
        for T in (4.0, 15.0, 45.0):
            h = 1e-4
            ts = np.array([T * (1 - h), T, T * (1 + h)])
            c, _, _ = O.surfdisp96(thk, vp, vs, rho, 0, iwave, 1, 0, ts, refine=1, rtol=1e-14, sngl=0)
            w = 2 * np.pi / ts
            k = w / c
            U_fd = (w[2] - w[0]) / (k[2] - k[0])
            if iwave == 2:
                U = O.sregn96(thk, vp, vs, rho, T, c[1], iflsph=0)["u"]
            else:
                U = O.slegn96(thk, vs, rho, T, c[1], iflsph=0)["u"]
            # the eigenfunction routines use single-precision pi in omega
            assert abs(U - U_fd) < 2e-6 * U, (iwave, T, U, U_fd)


def test_golden_regression():
    """The oracle still reproduces its frozen outputs (tests/golden)."""
    g = np.load(os.path.join(GOLD, "oracle_golden.npz"))
    z, vs, vp, rho = O.load_swd_model()
    t = 4.0 + 2.0 * np.arange(19)
    for refine, tag in ((0, "faithful"), (1, "tight")):
        for wt, name in enumerate(["Rc", "Rg", "Lc", "Lg"]):
            tabs = [None] * 4
            tabs[wt] = t[:, None]
            r = O.kernel1d(vs, vp, rho, z, tabs, refine=refine)
            for key in ("vc", "vout", "kvs", "kvp", "krho"):
                np.testing.assert_array_equal(r[key], g[f"model_{tag}_{name}_{key}"])


def test_frechet_rows_layout():
    """Row layout of SurfaceWave.cpp:630-659: j = iz*(nx-2)(ny-2) + iy*(nx-2) + ix
    over interior cells, ascending, float(fdm*kernel) kept where nonzero."""
    nx, ny, nz, kmax = 5, 4, 3, 2
    rng = np.random.default_rng(0)
    ker = rng.standard_normal((kmax, nz, nx * ny))
    fdm = np.zeros((2, ny, nx), np.float32)
    fdm[0, 1, 2] = 0.5
    fdm[1, 2, 1] = -1.0
    fdm[1, 2, 3] = 1e-30
    rows = O.frechet_rows(nx, ny, nz, ker, [1, 0], fdm.reshape(2, -1))
    idx, val = rows[0]
    assert list(idx) == [(iz * (ny - 2) * (nx - 2) + 0 * (nx - 2) + 1) for iz in range(nz - 1)]
    np.testing.assert_array_equal(val, (0.5 * ker[1, :nz - 1, 1 * nx + 2]).astype(np.float32))
    idx, val = rows[1]
    assert len(idx) == 2 * (nz - 1)


def test_frechet_file_round_trip():
    """The reference's row-file layout (SurfaceWave.cpp:596-603, 641-659) from
    CSR rows of the oracle, read back record by record."""
    import tempfile, os
    from jdsurfg_b200.frechet_file import write_frechet, read_frechet
    rng = np.random.default_rng(4)
    nx, ny, nz, kmax = 6, 5, 4, 3
    kernel = rng.standard_normal((kmax, nz, nx * ny))
    kernel[:, :, ::7] = 0.0
    row_slot = np.array([0, 2, 1, 2], np.int32)
    fdm = rng.standard_normal((len(row_slot), nx * ny)).astype(np.float32)
    fdm[1, :] = 0.0  # a row without entries
    rows = O.frechet_rows(nx, ny, nz, kernel, row_slot, fdm)
    rowptr = np.concatenate([[0], np.cumsum([len(i) for i, _ in rows])])
    idx = np.concatenate([i for i, _ in rows]) if rowptr[-1] else np.zeros(0, np.int32)
    val = np.concatenate([v for _, v in rows]) if rowptr[-1] else np.zeros(0, np.float32)
    n = (nx - 2) * (ny - 2) * (nz - 1)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "frechet.0")
        write_frechet(p, 17, n, np.arange(10, 10 + len(rows)), rowptr, idx, val)
        assert os.path.getsize(p) == 8 + sum(8 + 8 * len(i) for i, _ in rows)
        m, n2, back = read_frechet(p)
    assert (m, n2) == (17, n)
    for r, ((i0, v0), (rid, i1, v1)) in enumerate(zip(rows, back)):
        assert rid == 10 + r
        assert np.array_equal(i0, i1) and np.array_equal(v0, v1)
        assert np.all(np.diff(i1) > 0) and np.all(np.abs(v1) > 0)
    assert len(back[1][1]) == 0


def test_group_root_probe_moves_only_group_slots():
    """oracle_lib.group_root_spread moves the hidden roots c1, c2 of the
    group kernels (sregnpu/slegnpu) by one REAL*4 ulp: phase slots stay
    exactly, group slots move, and the probe leaves the oracle unchanged."""
    case = synth.make_config("tiny", seed=3)
    cols = np.arange(2)
    base = O.get_1d_kernel(case, cols=cols)
    kg = O.group_root_spread(case, cols)
    nt = kg.shape[0] // 4  # Rc, Rg, Lc, Lg, mode 0
    ok = base["status"] != 1
    assert np.all(kg[:nt][ok[:nt]] == 0.0) and np.all(kg[2 * nt:3 * nt][ok[2 * nt:3 * nt]] == 0.0)
    assert np.all(kg[nt:2 * nt][ok[nt:2 * nt]] > 0.0) and np.all(kg[3 * nt:][ok[3 * nt:]] > 0.0)
    again = O.get_1d_kernel(case, cols=cols)
    np.testing.assert_array_equal(again["kernel"], base["kernel"])
