"""The proposal network's hand-written kernels on the GPU: the tcgen05 GEMM
against torch, and forward/backward gradients against an FP64 CPU MLP."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (256, 256, 320), (1024, 256, 256), (256, 320, 1024)])
def test_tcgen05_gemm_matches_torch(M, N, K):
    import torch
    from jdsurfg_b200.mlp import gemm_bf16_tn
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    a = torch.randn(M, K, device="cuda", generator=g).bfloat16()
    b = torch.randn(N, K, device="cuda", generator=g).bfloat16()
    c = torch.full((M, N), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    gemm_bf16_tn(a, b, c, err)
    torch.cuda.synchronize()
    ref = a.double() @ b.double().T
    assert int(err.item()) == 0
    assert torch.isfinite(c).all()
    rel = ((c.double() - ref).abs().max() / ref.abs().max()).item()
    assert rel < 1e-5, rel


def _np_mlp_loss_grads(w, x, y):
    """FP64 reference of the network, its Gaussian NLL and gradients."""
    from math import sqrt
    from scipy.special import erf
    from jdsurfg_b200.mlp import layout
    L = layout()
    acts, pre = [x], []
    h = x
    for i, (wo, n, k, bo) in enumerate(L):
        W = w[wo:wo + n * k].reshape(n, k)
        b = w[bo:bo + n]
        z = h @ W.T + b
        pre.append(z)
        if i < len(L) - 1:
            h = 0.5 * z * (1.0 + erf(z / sqrt(2.0)))
            acts.append(h)
    out = pre[-1]
    M = len(y)
    mu, ls = out[:, 0], np.clip(out[:, 1], -12, 4)
    e = (y - mu) * np.exp(-ls)
    loss = np.mean(0.5 * e * e + ls)
    dz = np.zeros_like(out)
    dz[:, 0] = -e * np.exp(-ls) / M
    dz[:, 1] = (1 - e * e) / M
    g = np.zeros_like(w)
    for i in range(len(L) - 1, -1, -1):
        wo, n, k, bo = L[i]
        W = w[wo:wo + n * k].reshape(n, k)
        g[wo:wo + n * k] = (dz.T @ acts[i]).ravel()
        g[bo:bo + n] = dz.sum(0)
        if i > 0:
            dh = dz @ W
            z = pre[i - 1]
            cdf = 0.5 * (1 + erf(z / sqrt(2.0)))
            pdf = np.exp(-0.5 * z * z) / sqrt(2 * np.pi)
            dz = dh * (cdf + z * pdf)
    return loss, g


def test_mlp_gradients_match_fp64_cpu():
    import torch
    from jdsurfg_b200.mlp import MLP, layout
    net = MLP(seed=7)
    w = net.params().astype(np.float64)
    # weights as the GPU sees them (bf16)
    wb = torch.from_numpy(w.astype(np.float32)).bfloat16().double().numpy()
    rng = np.random.default_rng(0)
    M = 200
    x = np.zeros((M, 320), np.float32)
    x[:, :258] = rng.standard_normal((M, 258)).astype(np.float32) * 0.5
    y = rng.standard_normal(M).astype(np.float32) * 0.3
    xb = torch.from_numpy(x).cuda().bfloat16()
    yt = torch.from_numpy(y).cuda()
    loss = net.train_step(xb, yt, 0.0)
    g = net.grads().astype(np.float64)
    lref, gref = _np_mlp_loss_grads(wb, xb.double().cpu().numpy(), y.astype(np.float64))
    assert abs(loss - lref) < 1e-2 * max(1.0, abs(lref)), (loss, lref)
    for i, (wo, n, k, bo) in enumerate(layout()):
        a, b = g[wo:wo + n * k], gref[wo:wo + n * k]
        cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30)
        rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-30)
        # BF16 activations and operands between layers: ~1 % agreement
        assert cos > 0.999 and rel < 0.05, (i, cos, rel)


def test_mlp_learns_and_checkpoints(tmp_path):
    import torch
    from jdsurfg_b200.mlp import MLP
    net = MLP(seed=3)
    rng = np.random.default_rng(1)
    M = 1024
    x = np.zeros((M, 320), np.float32)
    x[:, :258] = rng.standard_normal((M, 258)).astype(np.float32) * 0.5
    y = (x[:, :8].sum(1) * 0.2).astype(np.float32)
    xb = torch.from_numpy(x).cuda().bfloat16()
    yt = torch.from_numpy(y).cuda()
    first = net.train_step(xb, yt, 1e-3)
    for _ in range(300):
        last = net.train_step(xb, yt, 1e-3)
    assert last < first - 1.0, (first, last)
    out1 = net.forward(xb).cpu().numpy()
    path = str(tmp_path / "mlp.bin")
    net.save(path)
    net2 = MLP(seed=99)
    net2.load(path)
    out2 = net2.forward(xb).cpu().numpy()
    np.testing.assert_array_equal(out1, out2)


def _tile_image(x):
    """(M, 320) bf16 rows -> the 128-row swizzled tile images swdk_mlp_propose reads."""
    import torch
    M = x.shape[0]
    T = (M + 127) // 128
    xp = torch.zeros((T * 128, 320), dtype=torch.bfloat16, device=x.device)
    xp[:M] = x
    # (T, 128 rows, 5 K-blocks, 8 chunks, 8 elems) -> (T, kb, r, swizzled chunk, e)
    v = xp.view(T, 128, 5, 8, 8).permute(0, 2, 1, 3, 4).contiguous()
    out = torch.empty_like(v)
    r = torch.arange(128, device=x.device)
    for j in range(8):
        out[:, :, r, (j ^ (r % 8)), :] = v[:, :, r, j, :]
    return out.reshape(-1)


def test_fused_proposal_matches_training_forward():
    """k_mlp_propose (all layers of a tile in one tcgen05 kernel, activations in
    shared memory) against the training path's layer-by-layer forward, with a
    ragged last tile."""
    import torch
    from jdsurfg_b200.mlp import MLP
    net = MLP(device=0, seed=3)
    g = torch.Generator(device="cuda").manual_seed(11)
    M = 128 * 37 + 45
    x = (0.5 * torch.randn(M, 320, device="cuda", generator=g)).bfloat16()
    x[:, 258:] = 0
    torch.cuda.synchronize()
    ref = net.forward(x).double()
    kappa = 2.5
    c_ref = 3.5 + ref[:, 0]
    hw_ref = kappa * torch.exp(torch.clamp(ref[:, 1], -12.0, 2.0))
    hw_ref = torch.maximum(hw_ref, 2e-5 * c_ref).clamp(max=0.2)
    xt = _tile_image(x)
    prop = torch.full((M, 2), float("nan"), device="cuda")
    net.propose(xt, M, kappa, prop)
    torch.cuda.synchronize()
    assert net.error_flag() == 0
    p = prop.double()
    assert torch.isfinite(p).all()
    assert (p[:, 0] - c_ref).abs().max().item() < 1e-5
    assert ((p[:, 1] - hw_ref).abs() / hw_ref).max().item() < 1e-4
