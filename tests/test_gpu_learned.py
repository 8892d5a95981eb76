"""The learned bracket proposal on the GPU.

The proposal only chooses where the scan looks first; every root is still
located by an FP64 sign change of the period equation on the reference's
scan grid and refined from the same grid cell.  So the learned path has to
reproduce the plain path's roots (and hence status and kernels) exactly,
while needing fewer secular-function evaluations -- that reduction is what
the trained network gains, and these tests report and bound it.
"""
import numpy as np
import pytest

from jdsurfg_b200 import Engine, synth
from jdsurfg_b200 import learn

pytestmark = pytest.mark.gpu


def _run(case, nets_dir=None, random_nets=False, kappa=None):
    eng = Engine(device=0, refine="tight")
    keep = None
    if nets_dir:
        keep = learn.load_proposals(eng, nets_dir, kappa=kappa)
    elif random_nets:
        from jdsurfg_b200.mlp import MLP
        keep = (MLP(device=0, seed=99), MLP(device=0, seed=98))
        eng.set_proposal(keep[0], keep[1], 4.0, 4.0)
    eng.setup(case)
    out = eng.get_1d_kernel(case["vs"], case["vp"], case["rho"], nx=case["nx"], ny=case["ny"])
    st = eng.stats()
    eng.close()
    return out, st


@pytest.mark.parametrize("name,ncols", [("large", 2048), ("production", 1024)])
def test_learned_matches_plain_and_saves_evaluations(name, ncols):
    case = synth.subset_columns(synth.make_config(name, seed=2024), np.arange(ncols))
    plain, sp = _run(case)
    lrn, sl = _run(case, nets_dir=learn.WEIGHTS)
    assert np.array_equal(plain["status"], lrn["status"])
    assert np.abs(plain["vc"] - lrn["vc"]).max() <= 1e-6
    assert np.abs(plain["vout"] - lrn["vout"]).max() <= 1e-6
    scale = np.abs(plain["kernel"]).max(axis=1, keepdims=True) + 1e-30
    assert (np.abs(plain["kernel"] - lrn["kernel"]) / scale).max() <= 1e-5
    gain = sp["secular_evals"] / sl["secular_evals"]
    used = sl["proposals_accepted"] / max(1, sl["proposals_accepted"] + sl["proposals_rejected"])
    print(f"{name}: secular evaluations plain {sp['secular_evals']} learned {sl['secular_evals']} "
          f"(x{gain:.2f}); proposals used {sl['proposals_accepted']}, fell back {sl['proposals_rejected']}")
    assert sl["proposals_accepted"] > 0
    assert used > 0.95
    assert gain > 1.25


def test_untrained_network_cannot_change_roots():
    """Random weights propose nonsense; the FP64 sign checks must catch it."""
    case = synth.subset_columns(synth.make_config("production", seed=7), np.arange(512))
    plain, _ = _run(case)
    junk, sj = _run(case, random_nets=True)
    assert np.array_equal(plain["status"], junk["status"])
    assert np.abs(plain["vc"] - junk["vc"]).max() <= 1e-6
    assert np.abs(plain["vout"] - junk["vout"]).max() <= 1e-6


def test_training_rows_and_targets():
    import torch
    case = synth.subset_columns(synth.make_config("large", seed=11), np.arange(256))
    eng = Engine(device=0, refine="tight")
    eng.setup(case)
    dev = torch.device("cuda", 0)
    vs = torch.from_numpy(case["vs"]).to(dev)
    eng.roots_device(case["nx"], case["ny"], case["nz"], vs)
    c, st = eng.last_roots(256)
    wave, mode, period = eng.root_slots()
    assert c.shape == (len(wave), 256) and set(np.unique(wave)) <= {1, 2}
    rows = torch.tensor([0, 5, 300, len(wave) * 256 - 1, -3, len(wave) * 256], dtype=torch.int64, device=dev)
    x = torch.full((6, 320), 7.0, dtype=torch.bfloat16, device=dev)
    y = torch.full((6,), 7.0, dtype=torch.float32, device=dev)
    eng.training_rows(rows, x, y)
    torch.cuda.synchronize()
    xr, yr = x.float().cpu().numpy(), y.cpu().numpy()
    flat = c.ravel()
    for i, r in enumerate([0, 5, 300, len(wave) * 256 - 1]):
        assert abs(yr[i] - (flat[r] - 3.5)) < 1e-6
        s, col = divmod(r, 256)
        assert abs(xr[i, 0] - case["vs"][0, col] / 4.5) < 1e-2
        assert abs(xr[i, 256] - np.log(period[s]) / np.log(100.0)) < 1e-2
        assert xr[i, 258:].max() == 0.0
    # out-of-range rows give zero features and targets
    assert np.all(xr[4:] == 0.0) and np.all(yr[4:] == 0.0)
    eng.close()


@pytest.mark.parametrize("shift", [0.15, -0.15, 0.03, -0.6])
def test_shifted_first_period_proposals_keep_the_roots(shift):
    """A constant shift of every proposed phase velocity leaves the anchored
    brackets of later periods (c(k-1) + mu(k) - mu(k-1)) as they are and
    moves only the first period's jump: above the root, a checked point
    finds the sign change and the scan resumes from the checked point below
    it; below the root, the scan goes on up from the cell.  The roots, and
    so status, U and kernels, stay the plain scan's bits."""
    case = synth.subset_columns(synth.make_config("large", seed=2024), np.arange(1024))
    plain, _ = _run(case)
    base, sb = _run(case, nets_dir=learn.WEIGHTS)
    eng = Engine(device=0, refine="tight")
    keep = learn.load_proposals(eng, learn.WEIGHTS)
    eng.set_proposal_shift(shift)
    eng.setup(case)
    out = eng.get_1d_kernel(case["vs"], case["vp"], case["rho"], nx=case["nx"], ny=case["ny"])
    st = eng.stats()
    eng.close()
    del keep
    for k in ("vc", "vout", "status", "kernel"):
        np.testing.assert_array_equal(out[k], plain[k], err_msg=k)
    # the shift did move the first-period search
    print(f"shift {shift:+.2f} km/s: secular evaluations {sb['secular_evals']} -> {st['secular_evals']}, "
          f"proposals fell back {sb['proposals_rejected']} -> {st['proposals_rejected']}")
    assert st["secular_evals"] != sb["secular_evals"]
    if shift >= 0.15:
        assert st["proposals_rejected"] > sb["proposals_rejected"]
