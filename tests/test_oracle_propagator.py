"""An independent pin of the oracle's multilayer root search: Rayleigh and
Love dispersion of the reference's own test model (test/swd/model.txt,
layered as grid2LayerModel layers it) solved here by a different method --
the motion-stress vector propagated through each layer with the matrix
exponential of the layer's first-order system (Aki & Richards, Quantitative
Seismology, eqs. 7.28 and 7.24), the two free-surface solutions kept
orthonormal layer by layer, and the mode condition that some combination
of them decays in the half-space.  It shares no formulation with the
delta-matrix recursion of surfdisp96 (dltar4 / dltar1) that the oracle
restates, yet must find the same roots.  CPU only."""
import numpy as np
import pytest
from scipy.linalg import expm
from scipy.optimize import brentq

import oracle_lib as O


def _psv(k, w, a, b, rho):
    """d/dz (ux, uz, tzx, tzz) for a homogeneous layer (A&R eq. 7.28)."""
    mu = rho * b * b
    lam = rho * a * a - 2.0 * mu
    l2m = lam + 2.0 * mu
    zeta = 4.0 * mu * (lam + mu) / l2m
    return np.array([[0.0, k, 1.0 / mu, 0.0],
                     [-k * lam / l2m, 0.0, 0.0, 1.0 / l2m],
                     [k * k * zeta - w * w * rho, 0.0, 0.0, k * lam / l2m],
                     [0.0, -w * w * rho, -k, 0.0]])


def _sh(k, w, b, rho):
    """d/dz (uy, tzy) for a homogeneous layer (A&R eq. 7.24)."""
    mu = rho * b * b
    return np.array([[0.0, 1.0 / mu], [k * k * mu - w * w * rho, 0.0]])


def _orth(F):
    """Orthonormal basis of span(F) related to F by a triangular factor of
    positive determinant (so the sign of the mode condition is kept)."""
    Q, R = np.linalg.qr(F)
    return Q * np.sign(np.diag(R))


def _rayleigh_D(c, T, thk, a, b, rho):
    w = 2.0 * np.pi / T
    k = w / c
    F = np.array([[1.0, 0.0], [0.0, 1.0], [0.0, 0.0], [0.0, 0.0]])  # free surface: no traction
    for h, ai, bi, ri in zip(thk[:-1], a[:-1], b[:-1], rho[:-1]):
        F = _orth(expm(_psv(k, w, ai, bi, ri) * h) @ F)
    A = _psv(k, w, a[-1], b[-1], rho[-1])
    na = np.sqrt(k * k - (w / a[-1]) ** 2)
    nb = np.sqrt(k * k - (w / b[-1]) ** 2)
    # Pg's kernel is the pair of solutions decaying with depth: some surface
    # solution decays iff Pg F loses rank; its displacement rows carry the
    # growing P and S components independently (na nb < k^2)
    Pg = (A + na * np.eye(4)) @ (A + nb * np.eye(4))
    return np.linalg.det((Pg @ F)[:2, :])


def _love_D(c, T, thk, b, rho):
    w = 2.0 * np.pi / T
    k = w / c
    f = np.array([1.0, 0.0])
    for h, bi, ri in zip(thk[:-1], b[:-1], rho[:-1]):
        f = expm(_sh(k, w, bi, ri) * h) @ f
        f = f / np.linalg.norm(f)
    A = _sh(k, w, b[-1], rho[-1])
    nb = np.sqrt(k * k - (w / b[-1]) ** 2)
    return ((A + nb * np.eye(2)) @ f)[0]  # the growing component's displacement


def _first_root(D, lo, hi, step):
    x0, f0 = lo, D(lo)
    x = lo + step
    while x < hi:
        f = D(x)
        if np.sign(f) != np.sign(f0):
            return brentq(D, x0, x, xtol=1e-13, rtol=1e-15)
        x0, f0 = x, f
        x += step
    raise AssertionError("no root")


def _model():
    z, vs, vp, rho = O.load_swd_model()
    thk, a, b, r = O.grid2layer(z, vp, vs, rho)
    return [np.asarray(x, np.float64) for x in (thk, a, b, r)], [np.asarray(x, np.float32) for x in (thk, a, b, r)]


def test_propagator_matrices_and_halfspace_root():
    # the layer matrices have the textbook vertical wavenumbers as eigenvalues
    k, w, a, b, rho = 0.9, 2.0, 6.0, 3.5, 2.7
    ev = np.sort(np.linalg.eigvals(_psv(k, w, a, b, rho)).real)
    na, nb = np.sqrt(k * k - (w / a) ** 2), np.sqrt(k * k - (w / b) ** 2)
    np.testing.assert_allclose(ev, np.sort([-na, -nb, nb, na]), rtol=1e-12)
    np.testing.assert_allclose(np.sort(np.linalg.eigvals(_sh(k, w, b, rho)).real), [-nb, nb], rtol=1e-12)
    # a homogeneous half-space under a layer of the same material: the
    # analytic Rayleigh root
    thk, av, bv, rv = [np.array(x) for x in ([2.0, 0.0], [a, a], [b, b], [rho, rho])]
    f = lambda cr: (2 - (cr / b) ** 2) ** 2 - 4 * np.sqrt(1 - (cr / a) ** 2) * np.sqrt(1 - (cr / b) ** 2)
    cr = brentq(f, 0.5 * b, 0.999 * b, xtol=1e-15)
    cp = _first_root(lambda c: _rayleigh_D(c, 10.0, thk, av, bv, rv), 0.8 * b, 0.9999 * b, 0.01)
    assert abs(cp - cr) < 1e-10


@pytest.mark.parametrize("T", [2.0, 5.0, 10.0, 20.0, 40.0])
def test_rayleigh_roots_of_the_reference_test_model(T):
    (thk, a, b, r), (thk32, a32, b32, r32) = _model()
    c, ierr, _ = O.surfdisp96(thk32, a32, b32, r32, 0, 2, 1, 0, np.array([T]), refine=1, rtol=1e-12, sngl=0)
    assert ierr == 0
    cp = _first_root(lambda x: _rayleigh_D(x, T, thk, a, b, r), 0.8 * b.min(), 0.99999 * b[-1], 0.004)
    assert abs(cp - c[0]) < 1e-11, (T, cp, c[0])


@pytest.mark.parametrize("T", [2.0, 5.0, 10.0, 20.0, 40.0])
def test_love_roots_of_the_reference_test_model(T):
    (thk, a, b, r), (thk32, a32, b32, r32) = _model()
    c, ierr, _ = O.surfdisp96(thk32, a32, b32, r32, 0, 1, 1, 0, np.array([T]), refine=1, rtol=1e-12, sngl=0)
    assert ierr == 0
    cp = _first_root(lambda x: _love_D(x, T, thk, b, r), b.min() * (1 + 1e-9), 0.99999 * b[-1], 0.004)
    assert abs(cp - c[0]) < 1e-11, (T, cp, c[0])


def _nth_root(D, lo, hi, step, n):
    x0, f0 = lo, D(lo)
    x, found = lo + step, 0
    while x < hi:
        f = D(x)
        if np.sign(f) != np.sign(f0):
            found += 1
            if found == n:
                return brentq(D, x0, x, xtol=1e-13, rtol=1e-15)
        x0, f0 = x, f
        x += step
    raise AssertionError("no root")


@pytest.mark.parametrize("T", [2.0, 5.0, 10.0])
@pytest.mark.parametrize("iwave", [1, 2])
def test_first_overtone_of_the_reference_test_model(T, iwave):
    """surfdisp96's second mode (its scan continued from the mode below) is
    the propagator's second root."""
    (thk, a, b, r), (thk32, a32, b32, r32) = _model()
    c, ierr, _ = O.surfdisp96(thk32, a32, b32, r32, 0, iwave, 2, 0, np.array([T]), refine=1, rtol=1e-12, sngl=0)
    assert ierr == 0
    if iwave == 2:
        D, lo = (lambda x: _rayleigh_D(x, T, thk, a, b, r)), 0.8 * b.min()
    else:
        D, lo = (lambda x: _love_D(x, T, thk, b, r)), b.min() * (1 + 1e-9)
    cp = _nth_root(D, lo, 0.99999 * b[-1], 0.002, 2)
    assert abs(cp - c[0]) < 1e-11, (T, iwave, cp, c[0])
