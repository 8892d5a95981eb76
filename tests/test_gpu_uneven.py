"""Uneven batch (many models of different grids, depths, periods, wave types
and modes in one CUDA-graph launch) against the oracle, against each model's
own eager call, and its depth kernels as CSR Frechet rows."""
import numpy as np
import pytest

import oracle_lib as O
from jdsurfg_b200 import synth
from jdsurfg_b200.batch import UnevenBatch

pytestmark = pytest.mark.gpu

TOL_C, TOL_K = 1e-6, 1e-5


def test_uneven_batch_graph_matches_oracle_and_eager():
    cases = synth.make_uneven_batch(6, seed=3, small=True)
    assert len({(c["nx"], c["ny"], c["nz"]) for c in cases}) > 1
    B = UnevenBatch(cases, learned=True)
    B.launch()
    got = [B.outputs(i) for i in range(len(cases))]
    for i, case in enumerate(cases):
        cols = np.arange(min(48, case["nx"] * case["ny"]))
        ref = O.get_1d_kernel(case, refine=1, cols=cols)
        g = {k: v[..., cols] for k, v in got[i].items()}
        assert np.array_equal(g["status"], ref["status"]), i
        ok = ref["status"] != 1
        assert np.abs(g["vc"] - ref["vc"])[ok].max() <= TOL_C
        assert np.abs(g["vout"] - ref["vout"])[ok].max() <= TOL_C
        scale = np.abs(ref["kernel"]).max(axis=1, keepdims=True) + 1e-30
        assert (np.abs(g["kernel"] - ref["kernel"]) / scale).max() <= TOL_K
    # a second launch and each model's eager call give the same bits
    B.launch()
    for i in range(len(cases)):
        again = B.outputs(i)
        B.run_eager(i)
        eager = B.outputs(i)
        for k in got[i]:
            assert np.array_equal(got[i][k], again[k]) and np.array_equal(got[i][k], eager[k]), (i, k)
    B.close()


def test_uneven_batch_csr_rows_match_oracle_layout():
    import torch
    cases = synth.make_uneven_batch(3, seed=8, small=True)
    B = UnevenBatch(cases, learned=False)
    B.launch()
    for i, case in enumerate(cases):
        nx, ny, nz = case["nx"], case["ny"], case["nz"]
        eng = B.engines[i]
        kmax = eng.kmax
        rng = np.random.default_rng(i)
        nrows = 37
        row_slot = rng.integers(0, kmax, nrows).astype(np.int32)
        fdm = (rng.standard_normal((nrows, nx * ny)) * (rng.random((nrows, nx * ny)) < 0.3)).astype(np.float32)
        dev = B.dev
        ker = B.bufs[i]["ker"]
        rowptr = torch.empty(nrows + 1, dtype=torch.int64, device=dev)
        cap = nrows * (nx - 2) * (ny - 2) * (nz - 1)
        idx = torch.empty(cap, dtype=torch.int32, device=dev)
        val = torch.empty(cap, dtype=torch.float32, device=dev)
        tot = eng.frechet_csr_device(nx, ny, nz, kmax, ker, torch.from_numpy(row_slot).to(dev),
                                     torch.from_numpy(fdm).to(dev), rowptr, idx, val)
        torch.cuda.synchronize()
        rows = O.frechet_rows(nx, ny, nz, ker.cpu().numpy(), row_slot, fdm)
        rp = rowptr.cpu().numpy()
        assert tot == rp[-1] == sum(len(a) for a, _ in rows)
        ii, vv = idx.cpu().numpy(), val.cpu().numpy()
        for r, (a, v) in enumerate(rows):
            assert np.array_equal(ii[rp[r]:rp[r + 1]], a)
            assert np.array_equal(vv[rp[r]:rp[r + 1]], v)
        # too little capacity is refused with the count reported
        with pytest.raises(Exception):
            eng.frechet_csr_device(nx, ny, nz, kmax, ker, torch.from_numpy(row_slot).to(dev),
                                   torch.from_numpy(fdm).to(dev), rowptr, idx[:max(0, tot - 1)], val)
    B.close()
