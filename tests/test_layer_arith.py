"""The root search rebuilds each flattened sublayer from its two grid nodes
(LayerView::sub_layer in jdsurfg_b200/csrc/swdk_core.cuh) with one
single-precision add: v0 + d/8, d = (2j+1)(v1 - v0) in REAL*4.  The model
preparation forms the same sum in double and rounds it to REAL*4.  d/8 is
exact in REAL*4, so both are the correctly rounded REAL*4 sum; this pins
that identity on random, near-equal, far-apart and tie-prone values
(tests/test_gpu_layers.py checks the rebuilt layers against the tables on
the GPU)."""
import numpy as np


def _both(a, b, j):
    w = np.float32(2 * j + 1)
    d = (w * (b - a)).astype(np.float32)
    ref = (a.astype(np.float64) + d.astype(np.float64) * 0.125).astype(np.float32)
    new = (a + np.float32(0.125) * d).astype(np.float32)
    return ref, new


def test_single_add_equals_double_then_round():
    rng = np.random.default_rng(20)
    n = 2_000_000
    cases = [
        (rng.uniform(0.0, 10.0, n), rng.uniform(0.0, 10.0, n)),                  # velocities, densities
        (rng.uniform(1.0, 9.0, n), None),                                         # near-equal nodes
        (rng.uniform(0.0, 1.0e3, n), rng.uniform(0.0, 1.0e-3, n)),               # far-apart magnitudes
        (rng.integers(0, 2 ** 20, n) * 2.0 ** -10, rng.integers(0, 2 ** 20, n) * 2.0 ** -10),  # exact ties
        (rng.uniform(1.0e-3, 1.0e-2, n), rng.uniform(1.0, 10.0, n)),
    ]
    for a, b in cases:
        a = np.asarray(a, np.float32)
        b = (a * (1 + rng.normal(0.0, 1e-6, n))).astype(np.float32) if b is None else np.asarray(b, np.float32)
        for j in range(4):
            ref, new = _both(a, b, j)
            assert np.array_equal(ref.view(np.uint32), new.view(np.uint32)), j
    # neighbouring floats
    a = np.nextafter(rng.uniform(1.0, 8.0, n).astype(np.float32), np.float32(10.0))
    b = np.nextafter(a, np.float32(0.0))
    for j in range(4):
        ref, new = _both(a, b, j)
        assert np.array_equal(ref.view(np.uint32), new.view(np.uint32)), j
