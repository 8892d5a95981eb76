"""Accuracy report of the GPU path against the all-FP64 oracle on 2048
seeded random columns of two grids:

* the 256x256x64 grid at 60 periods 1-80 s with phase AND group velocity of
  Rayleigh and Love (mode 0), and
* the 128x128x48 production grid at 40 periods 1-60 s, Rayleigh and Love
  modes 0-1, phase and group, with water layers and low-velocity zones.

Per grid it prints max and RMS |dc|, |dU| and the kernel error (relative to
the slot's largest |kernel|).  Tolerances: |dc|, |dU| <= 1e-6 km/s, kernel
<= 1e-5.

Kernels are compared at the same phase velocity.  Where the GPU's root and
the oracle's round to different REAL*4 values (one ulp, |dc| ~ 2e-7 km/s,
within the root tolerance) the oracle's kernel is recomputed at the GPU's
root before comparing: a kernel at a short period moves by up to a few
percent under a one-ulp change of c, in the reference as here.

Exemptions are in matching units.  The reference's kernel path is
ill-conditioned at a few (column, period) points: moving the phase velocity
handed to sregn96/sregnpu/slegn96/slegnpu by 1e-15 relative then moves U by
up to 1e-4 km/s and the kernel by up to 1e-3 of its largest value, so two
correct FP64 implementations disagree by that much.  A slot outside the
tolerance passes only if the oracle's own U (km/s) and kernel (relative)
move by comparable amounts under such changes (oracle_lib.kernel_spread):
|dU| <= max(1e-6, 2 * U spread) and kernel error <= max(1e-5, 10 * kernel
spread).  A group slot can also differ because its T(1 +- 0.005) roots,
which the outputs do not show, round one REAL*4 ulp apart: sregnpu and
slegnpu difference the phase kernels at those roots over a 1 % period step,
so one ulp of either moves the group kernel by up to ~1e-4 of its largest
value.  Such a slot passes if the oracle's U moves as far under one ulp
(2^-24) of all its roots and its kernel as far under one ulp of all of them
or of one hidden root alone (oracle_lib.group_root_spread).  The numbers of
exempted slots are printed.
"""
import numpy as np
import pytest

import oracle_lib as O
from jdsurfg_b200 import Engine, synth

pytestmark = pytest.mark.gpu

TOL_C, TOL_U, TOL_K = 1e-6, 1e-6, 1e-5
NCOL = 2048


def _report(name, seed):
    full = synth.make_config(name, seed=seed)
    ncol_full = full["nx"] * full["ny"]
    cols = np.sort(np.random.default_rng(seed + 1).choice(ncol_full, NCOL, replace=False))
    case = synth.subset_columns(full, cols)
    ref = O.get_1d_kernel(case, refine=1, rtol=1e-10)
    eng = Engine(device=0)
    eng.setup(case)
    g = eng.get_1d_kernel(case["vs"], case["vp"], case["rho"], nx=case["nx"], ny=case["ny"])
    eng.close()
    np.testing.assert_array_equal(g["status"], ref["status"])
    ok = (ref["status"] == 0) | (ref["status"] == 2)
    dc = np.abs(g["vc"] - ref["vc"])
    du = np.abs(g["vout"] - ref["vout"])
    scale = np.abs(ref["kernel"]).max(axis=1) + 1e-30
    kr = np.abs(g["kernel"] - ref["kernel"]).max(axis=1) / scale
    assert dc[ok].max() <= TOL_C, f"{name}: max |dc| {dc[ok].max():.3g}"
    # slots whose roots differ by a REAL*4 ulp: the oracle's group velocity
    # and kernel at the GPU's root
    nsame_c = 0
    for s, col in np.argwhere(ok & ((kr > TOL_K) | (du > TOL_U)) & (dc > 0)):
        rel = g["vc"][s, col] / ref["vc"][s, col] - 1.0
        r2 = O.kernel_at(case, int(col), rel)
        kr[s, col] = np.abs(g["kernel"][s, :, col] - r2["kernel"][s, :, 0]).max() / scale[s, col]
        du[s, col] = abs(g["vout"][s, col] - r2["vout"][s, 0])
        nsame_c += 1
    bad = ok & ((du > TOL_U) | (kr > TOL_K))
    bcols = np.nonzero(bad.any(axis=0))[0]
    nexempt = nround = 0
    if len(bcols):
        ks, us = O.kernel_spread(case, bcols)
        # the same under one REAL*4 ulp of the roots handed to the eigen
        # routines: all of them (2^-24 relative), and the group slots' hidden
        # T(1 +- 0.005) roots one at a time (they are not in the outputs)
        ks24, us24 = O.kernel_spread(case, bcols, rel=2.0 ** -24, steps=(-1, 1))
        kg = O.group_root_spread(case, bcols)
        for j, col in enumerate(bcols):
            for s in np.nonzero(bad[:, col])[0]:
                print(f"{name} slot {s} column {cols[col]}: |dc| {dc[s, col]:.3g}, |dU| {du[s, col]:.3g} "
                      f"(oracle U spread {us[s, j]:.3g}, {us24[s, j]:.3g} per ulp), kernel {kr[s, col]:.3g} "
                      f"(oracle kernel spread {ks[s, j]:.3g}, {ks24[s, j]:.3g} per ulp, {kg[s, j]:.3g} per ulp "
                      f"of a hidden group root)")
                if du[s, col] <= max(TOL_U, 2.0 * us[s, j]) and kr[s, col] <= max(TOL_K, 10.0 * ks[s, j]):
                    nexempt += 1
                    continue
                assert du[s, col] <= max(TOL_U, 2.0 * us24[s, j])
                assert kr[s, col] <= max(TOL_K, 2.0 * max(ks24[s, j], kg[s, j]))
                nround += 1
    rms = lambda x: float(np.sqrt(np.mean(x[ok] ** 2)))
    line = (f"{name}: {NCOL} columns x {ref['vc'].shape[0]} slots ({int(ok.sum())} with a root): "
            f"|dc| max {dc[ok].max():.3g} rms {rms(dc):.3g} km/s; |dU| max {du[ok].max():.3g} rms {rms(du):.3g} km/s; "
            f"kernel rel max {kr[ok].max():.3g} rms {rms(kr):.3g}; {nsame_c} kernels compared at the GPU's root "
            f"(roots one REAL*4 ulp apart); {nexempt} slots exempted by the oracle's own conditioning, {nround} by "
            f"its sensitivity to one REAL*4 ulp of the roots")
    print(line)
    return nexempt + nround, int(ok.sum())


def test_accuracy_256x256x64_phase_and_group():
    nexempt, n = _report("mixed", 2024)
    assert nexempt <= n // 1000


def test_accuracy_production_modes_water():
    nexempt, n = _report("production", 4048)
    assert nexempt <= n // 1000


def test_group_map_production_1024_columns():
    """get_2d_map (SurfaceWave.cpp:420-450): phase and group maps of Rayleigh
    and Love modes 0-1 (group velocity from sregn96/slegn96 at the phase
    root, disp1D) on 1024 random columns of the production grid."""
    full = synth.make_config("production", seed=777)
    cols = np.sort(np.random.default_rng(778).choice(full["nx"] * full["ny"], 1024, replace=False))
    case = synth.subset_columns(full, cols)
    ref = O.get_2d_map(case, refine=1, rtol=1e-10)
    eng = Engine(device=0)
    eng.setup(case)
    g = eng.get_2d_map(case["vs"], case["vp"], case["rho"], nx=case["nx"], ny=case["ny"])
    eng.close()
    np.testing.assert_array_equal(g["status"], ref["status"])
    ok = (ref["status"] == 0) | (ref["status"] == 2)
    dc = np.abs(g["vc"] - ref["vc"])
    du = np.abs(g["vout"] - ref["vout"])
    assert dc[ok].max() <= TOL_C
    bad = ok & (du > TOL_U)
    bcols = np.nonzero(bad.any(axis=0))[0]
    if len(bcols):
        us = O.map_spread(case, bcols)
        for j, col in enumerate(bcols):
            for s in np.nonzero(bad[:, col])[0]:
                print(f"map slot {s} column {cols[col]}: |dU| {du[s, col]:.3g} (oracle U spread {us[s, j]:.3g})")
                assert du[s, col] <= max(TOL_U, 2.0 * us[s, j])
    print(f"get_2d_map production: {ok.sum()} slots, |dc| max {dc[ok].max():.3g}, |dU| max {du[ok].max():.3g} "
          f"rms {np.sqrt(np.mean(du[ok] ** 2)):.3g} km/s, {int(bad.sum())} exempted")
    assert bad.sum() <= ok.sum() // 1000
