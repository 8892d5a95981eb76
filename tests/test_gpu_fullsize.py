"""The default workload at its full size (256 x 256 columns, 64 nodes, 60
periods, Rayleigh and Love mode 0 phase with kernels; 7.9 M slots) through
properties that do not depend on size, since the oracle cannot run all of
it in a test:

* the learned and the plain path give the same bits (roots, status,
  kernels) and the learned path needs fewer secular evaluations;
* the CUDA-graph replay gives the bits of the eager call;
* every slot has a root, every output is finite, and every phase velocity
  lies inside the models' velocity range;
* 48 random columns equal the oracle (|dc| <= 1e-6 km/s, kernels <= 1e-5
  of their largest value) or, where the kernel differs, the oracle moves as
  far under a 1e-15 change of its roots (tests/test_gpu_accuracy.py has the
  full account of that conditioning)."""
import numpy as np
import pytest

import oracle_lib as O
from jdsurfg_b200 import Engine, learn, synth

pytestmark = pytest.mark.gpu


def _device_call(eng, case, torch, dev):
    nx, ny, nz = case["nx"], case["ny"], len(case["depth"])
    t = lambda a: None if a is None else torch.from_numpy(a).to(dev)
    vs, vp, rho = t(case["vs"]), t(case["vp"]), t(case["rho"])
    kmax, ncol = eng.kmax, nx * ny
    vc = torch.empty((kmax, ncol), dtype=torch.float64, device=dev)
    vout = torch.empty_like(vc)
    st = torch.empty((kmax, ncol), dtype=torch.int32, device=dev)
    ker = torch.empty((kmax, nz, ncol), dtype=torch.float64, device=dev)
    return (vs, vp, rho), (vc, vout, ker, st)


def test_default_workload_full_size():
    import torch
    dev = torch.device("cuda", 0)
    case = synth.make_config("large", seed=2024)
    nx, ny, nz = case["nx"], case["ny"], len(case["depth"])
    outs, stats = [], []
    for learned in (False, True):
        eng = Engine(device=0)
        keep = learn.load_proposals(eng) if learned else None
        eng.setup(case)
        (vs, vp, rho), (vc, vout, ker, st) = _device_call(eng, case, torch, dev)
        eng.get_1d_kernel_device(nx, ny, nz, vs, vp, rho, vc, vout, ker, st)
        torch.cuda.synchronize()
        stats.append(eng.stats())
        outs.append([a.cpu().numpy() for a in (vc, vout, ker, st)])
        if learned:
            # graph replay of the same call into fresh outputs
            (vs, vp, rho), (vc2, vout2, ker2, st2) = _device_call(eng, case, torch, dev)
            eng.graph_capture("kernel", nx, ny, nz, vs, vp, rho, vc2, vout2, ker2, st2)
            eng.graph_launch()
            torch.cuda.synchronize()
            for a, b in zip(outs[-1], (vc2, vout2, ker2, st2)):
                assert np.array_equal(a, b.cpu().numpy())
        eng.close()
        del keep
    (pvc, pvo, pk, pst), (lvc, lvo, lk, lst) = outs
    assert np.array_equal(pvc, lvc) and np.array_equal(pst, lst) and np.array_equal(pk, lk)
    assert stats[1]["secular_evals"] < stats[0]["secular_evals"]
    assert np.all(lst != 1) and np.all(lvc > 0.0)
    assert np.all(np.isfinite(lvc)) and np.all(np.isfinite(lvo)) and np.all(np.isfinite(lk))
    # inside the model's shear-velocity range (2.5-4.7 km/s +- 8 %, flattened)
    assert lvc.min() > 1.5 and lvc.max() < 6.0
    cols = np.sort(np.random.default_rng(9).choice(nx * ny, 48, replace=False))
    sub = synth.subset_columns(case, cols)
    ref = O.get_1d_kernel(sub, refine=1, rtol=1e-10)
    assert np.array_equal(ref["status"], lst[:, cols])
    assert np.abs(ref["vc"] - lvc[:, cols]).max() <= 1e-6
    scale = np.abs(ref["kernel"]).max(axis=1) + 1e-30
    kr = np.abs(ref["kernel"] - lk[:, :, cols]).max(axis=1) / scale
    bad = np.argwhere(kr > 1e-5)
    if len(bad):
        ks, _ = O.kernel_spread(sub, np.unique(bad[:, 1]))
        jj = {c: i for i, c in enumerate(np.unique(bad[:, 1]))}
        for s, j in bad:
            assert kr[s, j] <= 10.0 * ks[s, jj[j]], (s, cols[j], kr[s, j])
    print(f"full size: {lvc.size} slots; evaluations plain {stats[0]['secular_evals']} learned "
          f"{stats[1]['secular_evals']}; graph replay identical; 48 sampled columns: max |dc| "
          f"{np.abs(ref['vc'] - lvc[:, cols]).max():.2e} km/s, max kernel rel err {kr.max():.2e}")
