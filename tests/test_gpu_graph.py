"""CUDA-graph replay of the device path and the root-kernel autotuner: the
replayed graph must give exactly the eager call's results, also after the
input model is overwritten in place, and tuning must not change any result."""
import numpy as np
import pytest

from jdsurfg_b200 import Engine, learn, synth

pytestmark = pytest.mark.gpu


def _dev(case, torch, dev):
    t = lambda a: None if a is None else torch.from_numpy(a).to(dev)
    return t(case["vs"]), t(case["vp"]), t(case["rho"])


def _eager(eng, case, torch, dev, path):
    nx, ny, nz = case["nx"], case["ny"], case["nz"]
    vs, vp, rho = _dev(case, torch, dev)
    kmax, ncol = eng.kmax, nx * ny
    vc = torch.empty((kmax, ncol), dtype=torch.float64, device=dev)
    vout = torch.empty_like(vc)
    st = torch.empty((kmax, ncol), dtype=torch.int32, device=dev)
    if path == "kernel":
        ker = torch.empty((kmax, nz, ncol), dtype=torch.float64, device=dev)
        eng.get_1d_kernel_device(nx, ny, nz, vs, vp, rho, vc, vout, ker, st)
    else:
        ker = None
        eng.get_2d_map_device(nx, ny, nz, vs, vp, rho, vc, vout, st)
    torch.cuda.synchronize()
    return vc.cpu().numpy(), vout.cpu().numpy(), st.cpu().numpy(), None if ker is None else ker.cpu().numpy()


@pytest.mark.parametrize("path,learned", [("kernel", True), ("map", False)])
def test_graph_replay_matches_eager(path, learned):
    import torch
    dev = torch.device("cuda", 0)
    a = synth.subset_columns(synth.make_config("production", seed=2024), np.arange(512))
    b = synth.subset_columns(synth.make_config("production", seed=77), np.arange(512))
    eng = Engine(device=0)
    nets = learn.load_proposals(eng) if learned else None
    eng.setup(a)
    ref_a = _eager(eng, a, torch, dev, path)
    ref_b = _eager(eng, b, torch, dev, path)
    nx, ny, nz = a["nx"], a["ny"], a["nz"]
    vs, vp, rho = _dev(a, torch, dev)
    kmax, ncol = eng.kmax, nx * ny
    vc = torch.zeros((kmax, ncol), dtype=torch.float64, device=dev)
    vout = torch.zeros_like(vc)
    st = torch.zeros((kmax, ncol), dtype=torch.int32, device=dev)
    ker = torch.zeros((kmax, nz, ncol), dtype=torch.float64, device=dev) if path == "kernel" else None
    eng.graph_capture(path, nx, ny, nz, vs, vp, rho, vc, vout, ker, st)
    for case, ref in ((a, ref_a), (b, ref_b), (a, ref_a)):
        vs2, vp2, rho2 = _dev(case, torch, dev)
        vs.copy_(vs2)
        vp.copy_(vp2)
        rho.copy_(rho2)
        vc.zero_()
        torch.cuda.synchronize()
        eng.graph_launch(torch.cuda.current_stream(dev).cuda_stream)
        torch.cuda.synchronize()
        assert np.array_equal(vc.cpu().numpy(), ref[0])
        assert np.array_equal(vout.cpu().numpy(), ref[1])
        assert np.array_equal(st.cpu().numpy(), ref[2])
        if ker is not None:
            assert np.array_equal(ker.cpu().numpy(), ref[3])
    eng.close()


def test_autotune_keeps_results():
    import torch
    dev = torch.device("cuda", 0)
    a = synth.subset_columns(synth.make_config("large", seed=2024), np.arange(2048))
    eng = Engine(device=0)
    eng.setup(a)
    ref = _eager(eng, a, torch, dev, "map")
    vs, vp, rho = _dev(a, torch, dev)
    blocks = eng.autotune(a["nx"], a["ny"], a["nz"], vs, vp, rho)
    assert blocks >= 1
    got = _eager(eng, a, torch, dev, "map")
    for x, y in zip(ref[:3], got[:3]):
        assert np.array_equal(x, y)
    eng.close()


@pytest.mark.parametrize("path", ["kernel", "map"])
def test_column_halves_equal_one_piece(path):
    """Calls split as two concurrent column halves on child contexts
    (split_cols 8192; by default only host-memory calls split) give the bits
    of the one-piece call, for device and host calls."""
    import torch
    dev = torch.device("cuda", 0)
    a = synth.subset_columns(synth.make_config("production", seed=2024), np.arange(9000))
    outs = []
    for split in (-1, 8192):
        eng = Engine(device=0, split_cols=split)
        keep = learn.load_proposals(eng)
        eng.setup(a)
        dvc = _eager(eng, a, torch, dev, path)
        host = eng.get_1d_kernel(a["vs"], a["vp"], a["rho"], nx=a["nx"]) if path == "kernel" else \
            eng.get_2d_map(a["vs"], a["vp"], a["rho"], nx=a["nx"])
        st = eng.stats()
        outs.append((dvc, host, st))
        eng.close()
    (d1, h1, s1), (d2, h2, s2) = outs
    for x, y in zip(d1, d2):
        if x is not None:
            assert np.array_equal(x, y)
    for k in h1:
        assert np.array_equal(h1[k], h2[k]), k
    assert np.array_equal(d1[0], h2["vc"])
    assert s1["secular_evals"] == s2["secular_evals"] and s1["proposals_accepted"] == s2["proposals_accepted"]
