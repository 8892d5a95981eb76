"""LSMR on the device (jdsurfg_b200/lsmr.py) with libswdk's CSR products:
the products against scipy's sparse matrix, and the solver against scipy's
LSMR run on the same FP32-valued matrix in FP64."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(m, n, density, seed):
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    A = sp.random(m, n, density=density, format="csr", random_state=seed, dtype=np.float64)
    A.data = (A.data - 0.5).astype(np.float32).astype(np.float64)  # FP32 values, as the Frechet rows
    A.sort_indices()
    b = A @ rng.standard_normal(n) + 1e-3 * rng.standard_normal(m)
    return A, b


def _device(A, deterministic=True):
    import torch
    from jdsurfg_b200.lsmr import DeviceCSR
    d = torch.device("cuda", 0)
    return DeviceCSR(torch.from_numpy(A.indptr.astype(np.int64)).to(d),
                     torch.from_numpy(A.indices.astype(np.int32)).to(d),
                     torch.from_numpy(A.data.astype(np.float32)).to(d), A.shape[0], A.shape[1],
                     deterministic=deterministic)


def test_csr_products_match_scipy():
    import torch
    A, _ = _problem(3000, 2000, 0.01, 1)
    D = _device(A)
    rng = np.random.default_rng(2)
    x = rng.standard_normal(2000)
    y0 = rng.standard_normal(3000)
    xd = torch.from_numpy(x).cuda()
    yd = torch.from_numpy(y0.copy()).cuda()
    D.aprod(1, xd, yd)
    assert np.allclose(yd.cpu().numpy(), y0 + A @ x, rtol=1e-12, atol=1e-12)
    x0 = rng.standard_normal(2000)
    xd = torch.from_numpy(x0.copy()).cuda()
    D.aprod(2, xd, torch.from_numpy(y0).cuda())
    assert np.allclose(xd.cpu().numpy(), x0 + A.T @ y0, rtol=1e-11, atol=1e-11)
    # the scattering product (FP64 atomics) agrees to rounding
    xa = torch.from_numpy(x0.copy()).cuda()
    _device(A, deterministic=False).aprod(2, xa, torch.from_numpy(y0).cuda())
    assert np.allclose(xa.cpu().numpy(), xd.cpu().numpy(), rtol=1e-12, atol=1e-12)


def test_transpose_product_is_deterministic_and_matches_row_order():
    """A^T y through the device transpose: the same bits on every call, and
    the transpose holds A's entries column by column in row order."""
    import torch
    A, _ = _problem(4000, 1500, 0.02, 5)
    D = _device(A)
    T = A.T.tocsr()
    T.sort_indices()
    assert np.array_equal(D.t.rowptr.cpu().numpy(), T.indptr)
    assert np.array_equal(D.t.indices.cpu().numpy(), T.indices)
    assert np.array_equal(D.t.values.cpu().numpy(), T.data.astype(np.float32))
    y = torch.from_numpy(np.random.default_rng(6).standard_normal(4000)).cuda()
    outs = []
    for _ in range(3):
        x = torch.zeros(1500, dtype=torch.float64, device="cuda")
        D.aprod(2, x, y)
        outs.append(x.cpu().numpy())
    assert all(np.array_equal(outs[0].view(np.int64), o.view(np.int64)) for o in outs[1:])


@pytest.mark.parametrize("damp", [0.0, 0.3])
def test_lsmr_matches_scipy(damp):
    import torch
    from scipy.sparse.linalg import lsmr as sp_lsmr
    from jdsurfg_b200.lsmr import lsmr
    A, b = _problem(2500, 1200, 0.02, 3)
    D = _device(A)
    x, info = lsmr(D, torch.from_numpy(b).cuda(), damp=damp, atol=1e-10, btol=1e-10, itnlim=300)
    ref = sp_lsmr(A, b, damp=damp, atol=1e-10, btol=1e-10, maxiter=300)
    xr = ref[0]
    assert info["istop"] == ref[1]
    assert abs(info["itn"] - ref[2]) <= 2
    assert np.linalg.norm(x.cpu().numpy() - xr) <= 1e-6 * np.linalg.norm(xr)
    assert abs(info["normr"] - ref[3]) <= 1e-6 * max(1.0, ref[3])
    # the normal equations of the damped problem hold at the solution
    xs = x.cpu().numpy()
    g = A.T @ (A @ xs - b) + damp ** 2 * xs
    assert np.linalg.norm(g) <= 1e-6 * np.linalg.norm(A.T @ b)


def test_device_solve_matches_stepwise_and_is_deterministic():
    """swdk_lsmr_solve (everything on the device) against the host-driven
    iteration with the same formulas: the same stop, the same iteration
    count, the solutions within 1e-10; and the same bits on a second run."""
    import torch
    from jdsurfg_b200.lsmr import lsmr, lsmr_stepwise
    A, b = _problem(3000, 1400, 0.02, 8)
    D = _device(A)
    bd = torch.from_numpy(b).cuda()
    x1, i1 = lsmr(D, bd, damp=0.05, atol=1e-9, btol=1e-9, itnlim=200)
    x2, i2 = lsmr(D, bd, damp=0.05, atol=1e-9, btol=1e-9, itnlim=200)
    xs, isw = lsmr_stepwise(D, bd, damp=0.05, atol=1e-9, btol=1e-9, itnlim=200)
    a1, a2, as_ = x1.cpu().numpy(), x2.cpu().numpy(), xs.cpu().numpy()
    assert np.array_equal(a1.view(np.int64), a2.view(np.int64)) and i1 == i2
    assert i1["istop"] == isw["istop"] and abs(i1["itn"] - isw["itn"]) <= 1
    assert np.linalg.norm(a1 - as_) <= 1e-10 * np.linalg.norm(as_)
    assert abs(i1["normr"] - isw["normr"]) <= 1e-10 * max(1.0, isw["normr"])


def test_device_solve_iteration_limit_and_zero_rhs():
    import torch
    from jdsurfg_b200.lsmr import lsmr
    A, b = _problem(2000, 900, 0.02, 9)
    D = _device(A)
    x, info = lsmr(D, torch.from_numpy(b).cuda(), atol=0.0, btol=0.0, conlim=0.0, itnlim=5)
    assert info["istop"] == 7 and info["itn"] == 5
    x0, i0 = lsmr(D, torch.zeros(2000, dtype=torch.float64, device="cuda"))
    assert i0["istop"] == 0 and i0["itn"] == 0 and float(x0.abs().max()) == 0.0
