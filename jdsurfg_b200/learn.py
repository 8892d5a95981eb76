"""Training of the learned bracket proposal (GPU only).

The plain GPU solver produces the training set: seeded synthetic models of
the production generator (jdsurfg_b200/synth.py) on both depth grids the
engine is run on (48 nodes to 87.5 km and 64 nodes to 127.5 km), root
search with ``Engine.roots_device`` over every root slot of get_1d_kernel,
and (features, c - 3.5 km/s) rows of converged roots drawn at random.  One
network per wave type (Rayleigh, Love) is trained with the hand-written
tcgen05 forward/backward and Adam kernels of libswdk (``MLP.train_step``),
minimising the Gaussian negative log-likelihood of the root given the
predicted mean and log sigma.  kappa, the factor from sigma to the bracket
half-width, is set from a held-out split so that the bracket covers the
requested fraction of roots.  The engine centres each bracket on the
previous period's root plus the predicted change, c(k-1) + mu(k) - mu(k-1),
so kappa is calibrated on that anchored error, over complete period chains
of held-out models.

The proposal never decides a root: the engine evaluates the FP64 period
equation at both bracket ends and runs the reference's plain scan whenever
the sign pattern is not the mode's (surfdisp96.f:432-451).

    python -m jdsurfg_b200.learn --out jdsurfg_b200/weights
"""
import argparse
import json
import os
import time

import numpy as np

from . import synth
from .engine import Engine, ST_OK
from .mlp import MLP, IN_DIM

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "weights")
WAVE_NAMES = {2: "rayleigh", 1: "love"}

# training geometries: (generator, grid) with seeds disjoint from the
# benchmark (2024 + rank) and test (2024, 7, 11, ...) seeds
GEOMETRIES = (("production", 128, 128), ("large", 128, 128))
TRAIN_SEEDS = (91001, 91002, 91003, 91004)
CALIB_SEEDS = (92001,)


def _torch():
    import torch
    return torch


def generate(rows_per_wave=1_000_000, device=0, seeds=TRAIN_SEEDS, geometries=GEOMETRIES, log=print):
    """Rows of converged roots from the plain GPU solver.

    Returns {wave: (x bf16 (n, 320), y float32 (n,))} on the device and a
    summary dict."""
    torch = _torch()
    dev = torch.device("cuda", device)
    eng = Engine(device=device, refine="tight")
    parts = {2: [], 1: []}
    per_run = max(1, len(seeds) * len(geometries))
    info = dict(runs=[])
    for seed in seeds:
        for gi, (name, nx, ny) in enumerate(geometries):
            case = synth.make_config(name, seed=seed + 100 * gi, nx=nx, ny=ny)
            eng.setup(case)
            ncol = nx * ny
            vs = torch.from_numpy(case["vs"]).to(dev)
            vp = torch.from_numpy(case["vp"]).to(dev) if case["vp"] is not None else None
            rho = torch.from_numpy(case["rho"]).to(dev) if case["rho"] is not None else None
            t0 = time.time()
            eng.roots_device(nx, ny, case["nz"], vs, vp, rho)
            c, st = eng.last_roots(ncol)
            wave, mode, period = eng.root_slots()
            ok = (st == ST_OK) & np.isfinite(c) & (c > 0)
            rng = np.random.default_rng(seed * 7 + gi)
            for w in (2, 1):
                cand = np.flatnonzero((ok & (wave[:, None] == w)).ravel())
                if cand.size == 0:
                    continue
                take = min(cand.size, rows_per_wave // per_run)
                rows = np.sort(rng.choice(cand, size=take, replace=False)).astype(np.int64)
                r_d = torch.from_numpy(rows).to(dev)
                x = torch.empty((take, IN_DIM), dtype=torch.bfloat16, device=dev)
                y = torch.empty(take, dtype=torch.float32, device=dev)
                eng.training_rows(r_d, x, y)
                parts[w].append((x, y))
            torch.cuda.synchronize(dev)
            info["runs"].append(dict(geometry=name, seed=seed + 100 * gi, ncol=ncol, nslot=len(wave),
                                     ok_frac=float(ok.mean()), seconds=round(time.time() - t0, 2)))
            log(f"  generated {name} seed {seed + 100 * gi}: {len(wave)} slots x {ncol} columns, "
                f"{ok.mean():.4f} converged, {time.time() - t0:.1f} s")
    eng.close()
    data = {}
    for w, lst in parts.items():
        if lst:
            data[w] = (torch.cat([a for a, _ in lst]), torch.cat([b for _, b in lst]))
    return data, info


def train(x, y, device=0, steps=6000, batch=4096, lr=1.0e-3, lr_end=1.0e-5, seed=1234, log=print):
    """Adam on the Gaussian NLL with a cosine learning-rate schedule."""
    torch = _torch()
    net = MLP(device=device, seed=seed)
    n = x.shape[0]
    gen = torch.Generator(device=x.device)
    gen.manual_seed(seed)
    hist = []
    t0 = time.time()
    for s in range(steps):
        idx = torch.randint(0, n, (batch,), device=x.device, generator=gen)
        a = lr_end + 0.5 * (lr - lr_end) * (1.0 + np.cos(np.pi * s / steps))
        loss = net.train_step(x[idx].contiguous(), y[idx].contiguous(), a)
        if s % 500 == 0 or s == steps - 1:
            hist.append((s, float(loss)))
            log(f"    step {s:6d} lr {a:.2e} nll {loss:.4f}  ({time.time() - t0:.1f} s)")
    return net, hist


def evaluate(net, x, y, batch=65536):
    """Held-out residuals: (mu - y, sigma) as numpy arrays."""
    torch = _torch()
    mus, sig = [], []
    for a in range(0, x.shape[0], batch):
        o = net.forward(x[a:a + batch].contiguous())
        mus.append((o[:, 0] - y[a:a + batch]).double().cpu().numpy())
        sig.append(torch.exp(o[:, 1].double()).cpu().numpy())
    return np.concatenate(mus), np.concatenate(sig)


def calibrate(res, sig, coverage=0.995):
    """kappa such that |mu - c| <= kappa * sigma on `coverage` of the rows."""
    z = np.abs(res) / np.maximum(sig, 1e-12)
    return float(np.quantile(z, coverage))


def chain_position(wave, mode, period):
    """0-based period index of every root slot within its (chain, mode) block:
    root slots run chain by chain, mode by mode, periods increasing."""
    k = np.zeros(len(wave), np.int64)
    for i in range(1, len(wave)):
        same = wave[i] == wave[i - 1] and mode[i] == mode[i - 1] and period[i] > period[i - 1]
        k[i] = k[i - 1] + 1 if same else 0
    return k


def predict_all(eng, nets, ncol, wave, chunk=262144):
    """(mu, sigma) of every root row (slot * ncol + col) after roots_device."""
    torch = _torch()
    dev = torch.device("cuda", eng.cfg.device)
    nrow = len(wave) * ncol
    mu = np.zeros(nrow, np.float64)
    sig = np.zeros(nrow, np.float64)
    x = torch.empty((chunk, IN_DIM), dtype=torch.bfloat16, device=dev)
    for a in range(0, nrow, chunk):
        n = min(chunk, nrow - a)
        rows = torch.arange(a, a + n, dtype=torch.int64, device=dev)
        eng.training_rows(rows, x[:n])
        w = wave[(np.arange(a, a + n) // ncol)]
        for wv, name in ((2, "rayleigh"), (1, "love")):
            sel = np.flatnonzero(w == wv)
            if sel.size == 0 or name not in nets:
                continue
            o = nets[name].forward(x[torch.from_numpy(sel).to(dev)].contiguous()).double().cpu().numpy()
            mu[a + sel] = o[:, 0]
            sig[a + sel] = np.exp(np.clip(o[:, 1], -12.0, 2.0))
    return mu, sig


def calibrate_anchored(nets, device=0, coverage=0.995, seeds=CALIB_SEEDS, geometries=GEOMETRIES, log=print):
    """kappa per wave type for the anchored bracket c(k-1) + mu(k) - mu(k-1)
    (the engine's form), from complete chains of held-out models."""
    torch = _torch()
    dev = torch.device("cuda", device)
    eng = Engine(device=device, refine="tight")
    z = {2: [], 1: []}
    err = {2: [], 1: []}
    for seed in seeds:
        for gi, (name, nx, ny) in enumerate(geometries):
            case = synth.make_config(name, seed=seed + 100 * gi, nx=nx, ny=ny)
            eng.setup(case)
            ncol = nx * ny
            vs = torch.from_numpy(case["vs"]).to(dev)
            vp = torch.from_numpy(case["vp"]).to(dev) if case["vp"] is not None else None
            rho = torch.from_numpy(case["rho"]).to(dev) if case["rho"] is not None else None
            eng.roots_device(nx, ny, case["nz"], vs, vp, rho)
            c, st = eng.last_roots(ncol)
            wave, mode, period = eng.root_slots()
            kpos = chain_position(wave, mode, period)
            mu, sig = predict_all(eng, nets, ncol, wave)
            mu = mu.reshape(len(wave), ncol)
            sig = sig.reshape(len(wave), ncol)
            for s in np.flatnonzero(kpos > 0):
                ok = (st[s] == ST_OK) & (st[s - 1] == ST_OK)
                e = (mu[s, ok] - mu[s - 1, ok]) - (c[s, ok] - c[s - 1, ok])
                z[wave[s]].append(np.abs(e) / np.maximum(sig[s, ok], 1e-12))
                err[wave[s]].append(np.abs(e))
    eng.close()
    out = {}
    for w, name in ((2, "rayleigh"), (1, "love")):
        if not z[w]:
            continue
        zz = np.concatenate(z[w])
        ee = np.concatenate(err[w])
        out[name] = dict(kappa=float(np.quantile(zz, coverage)), rows=int(zz.size),
                         anchored_p50=float(np.median(ee)), anchored_p99=float(np.quantile(ee, 0.99)))
        log(f"  anchored {name}: {zz.size} rows, |error| p50 {out[name]['anchored_p50']:.5f} "
            f"p99 {out[name]['anchored_p99']:.5f} km/s, kappa {out[name]['kappa']:.2f}")
    return out


def train_proposals(out=WEIGHTS, device=0, rows_per_wave=1_000_000, steps=6000, batch=4096, coverage=0.995,
                    log=print):
    torch = _torch()
    os.makedirs(out, exist_ok=True)
    t0 = time.time()
    data, info = generate(rows_per_wave=rows_per_wave, device=device, log=log)
    meta = dict(generator=info, rows={}, kappa={}, heldout={}, steps=steps, batch=batch, coverage=coverage)
    nets = {}
    for w, (x, y) in data.items():
        name = WAVE_NAMES[w]
        n = x.shape[0]
        perm = torch.randperm(n, device=x.device, generator=torch.Generator(device=x.device).manual_seed(5))
        nho = max(1024, n // 20)
        ho, tr = perm[:nho], perm[nho:]
        log(f"  training {name}: {tr.numel()} rows, {nho} held out")
        net, hist = train(x[tr], y[tr], device=device, steps=steps, batch=batch, log=log)
        res, sig = evaluate(net, x[ho], y[ho])
        kappa = calibrate(res, sig, coverage)
        hw = np.clip(kappa * sig, 2e-5 * (3.5 + y[ho].double().cpu().numpy()), 0.2)
        meta["rows"][name] = int(n)
        meta["kappa"][name] = kappa
        meta["heldout"][name] = dict(rms_km_s=float(np.sqrt(np.mean(res ** 2))),
                                     p50_abs=float(np.median(np.abs(res))),
                                     p99_abs=float(np.quantile(np.abs(res), 0.99)),
                                     median_halfwidth=float(np.median(hw)),
                                     covered=float(np.mean(np.abs(res) <= hw)), loss=hist[-1][1])
        net.save(os.path.join(out, f"{name}.mlp"))
        log(f"  {name}: held-out rms {meta['heldout'][name]['rms_km_s']:.4f} km/s, kappa {kappa:.2f}, "
            f"median half-width {meta['heldout'][name]['median_halfwidth']:.4f} km/s")
        nets[name] = net
    del data
    meta["anchored"] = calibrate_anchored(nets, device=device, coverage=coverage, log=log)
    meta["engine_kappa"] = {k: v["kappa"] for k, v in meta["anchored"].items()}
    for net in nets.values():
        net.close()
    meta["seconds"] = round(time.time() - t0, 1)
    with open(os.path.join(out, "proposal.json"), "w") as f:
        json.dump(meta, f, indent=1)
    return meta


def load_proposals(engine, weights=WEIGHTS, device=None, kappa=None):
    """Attach the trained networks in `weights` to an Engine; returns them
    (keep them alive as long as the engine uses them)."""
    with open(os.path.join(weights, "proposal.json")) as f:
        meta = json.load(f)
    dev = engine.cfg.device if device is None else device
    nets = {}
    for name in ("rayleigh", "love"):
        p = os.path.join(weights, f"{name}.mlp")
        if os.path.exists(p):
            net = MLP(device=dev)
            net.load(p)
            nets[name] = net
    ek = meta["engine_kappa"]
    kr = kappa if kappa else ek.get("rayleigh", 4.0)
    kl = kappa if kappa else ek.get("love", 4.0)
    engine.set_proposal(nets.get("rayleigh"), nets.get("love"), kr, kl)
    return nets, meta


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--rows", type=int, default=1_000_000, help="training rows per wave type")
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--coverage", type=float, default=0.995)
    a = ap.parse_args()
    meta = train_proposals(a.out, a.device, a.rows, a.steps, a.batch, a.coverage)
    print(json.dumps({k: meta[k] for k in ("rows", "kappa", "heldout", "engine_kappa", "seconds")}))


if __name__ == "__main__":
    main()
