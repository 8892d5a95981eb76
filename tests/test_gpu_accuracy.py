"""Accuracy report on the 256x256x64, 60-period grid with phase AND group
velocity of Rayleigh and Love (mode 0): max and RMS |dc|, |dU| and kernel
relative error of the GPU path against the all-FP64 oracle.

The reference's group velocity in the kernel path (sregnpu/slegnpu energy
integrals) is ill-conditioned at a few (column, period) points: moving the
phase velocity input by 1e-15 relative moves U by up to 1e-4 km/s there.
Two correct FP64 implementations then disagree by that much.  A slot whose
|dU| exceeds 1e-6 km/s therefore passes only if the oracle's own U moves by
at least |dU| under such a perturbation (sregnpu_/slegnpu_ called directly);
its kernel, and the phase kernel of the same period, are held to the same
rule with a looser factor.
"""
import numpy as np
import pytest

import oracle_lib as O
from jdsurfg_b200 import Engine, synth

pytestmark = pytest.mark.gpu

TOL_C, TOL_U, TOL_K = 1e-6, 1e-6, 1e-5


def test_accuracy_report_phase_and_group():
    full = synth.make_config("mixed", seed=2024)
    ncol = 96
    case = synth.subset_columns(full, np.arange(ncol))
    ref = O.get_1d_kernel(case, refine=1, rtol=1e-10)
    eng = Engine(device=0)
    eng.setup(case)
    g = eng.get_1d_kernel(case["vs"], case["vp"], case["rho"], nx=case["nx"], ny=case["ny"])
    eng.close()
    assert np.array_equal(g["status"], ref["status"])
    ok = ref["status"] == 0
    dc = np.abs(g["vc"] - ref["vc"])
    du = np.abs(g["vout"] - ref["vout"])
    scale = np.abs(ref["kernel"]).max(axis=1, keepdims=True) + 1e-30
    kr = (np.abs(g["kernel"] - ref["kernel"]) / scale).max(axis=1)
    print(f"|dc| max {dc[ok].max():.3g} rms {np.sqrt(np.mean(dc[ok] ** 2)):.3g}; "
          f"|dU| max {du[ok].max():.3g} rms {np.sqrt(np.mean(du[ok] ** 2)):.3g}; "
          f"kernel rel max {kr[ok].max():.3g} rms {np.sqrt(np.mean(kr[ok] ** 2)):.3g}")
    assert dc[ok].max() <= TOL_C
    periods = np.geomspace(1.0, 80.0, 60)
    bad = np.argwhere(ok & ((du > TOL_U) | (kr > TOL_K)))
    assert len(bad) <= max(3, ok.sum() // 1000), f"{len(bad)} slots outside tolerance"
    for s, col in bad:
        wave = ("Rc", "Rg", "Lc", "Lg")[s // 60]
        assert dc[s, col] <= TOL_C
        # the eigenfunctions (and so phase kernels too) share the group slot's
        # conditioning at the same period and phase velocity
        probe = "Rg" if wave in ("Rc", "Rg") else "Lg"
        _, spread = O.group_u_spread(case, int(col), probe, periods, int(s % 60))
        print(f"slot {s} column {col}: |dU| {du[s, col]:.3g}, kernel {kr[s, col]:.3g}, oracle U spread "
              f"under 1e-15 changes of c: {spread:.3g}")
        assert du[s, col] <= max(TOL_U, 2 * spread)
        assert kr[s, col] <= max(TOL_K, 10 * spread)
