#!/usr/bin/env python
"""Throughput of SurfTime::get_1d_kernel (dispersion + depth kernels for every
column, period and mode of a 3-D model) on B200, learned-bracket path against
the plain GPU scan.

A step is one get_1d_kernel call over the whole workload.  The default
workload ("large") is the 256x256-column model with 64 nodes, 60 periods
1-80 s, Rayleigh and Love fundamental-mode phase velocity and dc/dvs
kernels, LVZ in 20 % of the columns (seeded synthetic models).  The learned
bracket proposal (jdsurfg_b200/weights) is on; the same steps are then timed
with it off ("plain" in the line).  value = column-period-mode slots per
second with inputs resident in HBM; e2e = the same through the host-memory
C-ABI call with pinned host buffers, host<->device copies inside the timed
region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl swdk|reference]

Under torchrun each rank computes its own grid (different seed): weak
scaling, no collective on the data path.  --impl reference times the CPU
oracle (a line-by-line restatement of the reference's Fortran/C++ path; the
reference's Fortran cannot be compiled here) on the host cores, on a bounded
sample of the same workload.
"""
import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "dispersion+kernel column-periods/s, learned vs plain GPU at |Δc|≤1e-6 km/s"
UNIT = "column-period-modes/s"
# Algorithmic FP64 flops per layer per secular evaluation (FMA = 2), hand count
# of surfdisp96.f dltar4/var/dnka/normc (798-1095) and dltar1 (734-794);
# divisions, square roots and exp/sin/cos are not counted.
F_SEC_RAYLEIGH = 161
F_SEC_LOVE = 19
# Algorithmic FP64 flops per layer of one eigenfunction pass (FMA = 2), hand
# count of the formulation in jdsurfg_b200/csrc/swdk_eigen.cuh for a solid
# layer with real vertical wavenumbers: Rayleigh = up sweep (varsv terms 22,
# dnka product 139, normalisation 9) + down sweep (varsv terms 22, hska
# product 78, normalisation and exponents 9, svfunc eigenfunction 25, energy
# integrals and getmat 354, _ParamConvert/chain-rule sink 17); Love = up 24 +
# shfunc 3 + energy and sink 105.  Divisions, square roots and exp/sin/cos
# are not counted.  A phase slot is one pass, a group slot three
# (sregnpu/slegnpu at T, T(1+0.005), T(1-0.005)).
F_EIG_RAYLEIGH = 675
F_EIG_LOVE = 132
# proposal network multiply-adds per row: 320x256 + 3 x 256x256 + 256x64
MLP_MACS_PER_ROW = 320 * 256 + 3 * 256 * 256 + 256 * 64


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="swdk", choices=["swdk", "reference"])
    ap.add_argument("--workload", default="large",
                    choices=["production", "large", "small", "tiny", "uneven", "fmst", "lsmr"])
    ap.add_argument("--proposal", default="learned", choices=["learned", "none"])
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-scan comparison timing")
    ap.add_argument("--no-graph", action="store_true", help="time eager calls instead of CUDA-graph replays")
    ap.add_argument("--ncols", type=int, default=0, help="use only the first N columns (profiling)")
    ap.add_argument("--refine", default="tight", choices=["tight", "reference"])
    ap.add_argument("--split-cols", type=int, default=0,
                    help="column count from which a call runs as two concurrent halves (0, the default: never)")
    ap.add_argument("--roots-blocks", type=int, default=0, help="fixed root-search grid (0: default/autotuned)")
    ap.add_argument("--no-node-layers", action="store_true",
                    help="root search reads the full layer tables instead of rebuilding sublayers from the nodes")
    ap.add_argument("--path", default="kernel", choices=["kernel", "map"],
                    help="kernel: get_1d_kernel (dispersion + depth kernels); map: get_2d_map (phase and group maps "
                         "of travel_time's line-search steps)")
    ap.add_argument("--uneven-mode", default="ragged", choices=["ragged", "branches"],
                    help="uneven workload: one ragged launch per kernel, or a graph branch per model")
    ap.add_argument("--sharded", action="store_true",
                    help="strong scaling: ONE model split by columns over the ranks (allocate_tasks), each step "
                         "computing the rank's block and all-gathering the vc/vout/status maps with NCCL")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU time of the baseline sample")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def workload(args, rank):
    from jdsurfg_b200 import synth
    case = synth.make_config(args.workload, seed=2024 + rank)
    if args.ncols:
        n = min(args.ncols, case["nx"] * case["ny"])
        case = synth.subset_columns(case, np.arange(n))
    return case


WORKLOAD_TEXT = {
    "large": "256x256 columns x 64 nodes, 60 periods 1-80 s, Rayleigh+Love mode 0 phase, dc/dvs kernels",
    "production": "128x128 columns x 48 nodes, 40 periods 1-60 s, Rayleigh+Love modes 0-1 phase+group, water",
    "small": "16x16 columns x 20 nodes, 25 periods 2-40 s, Rayleigh mode 0 phase+group",
    "tiny": "4x3 columns x 12 nodes, 6 periods, all wave types",
    "uneven": "48 models, grids 32x32..200x200, 24..80 nodes, 15..60 periods in 1..100 s, 1-2 of Rc/Rg/Lc/Lg, "
              "modes 0..2, one CUDA graph",
}


def case_desc(args, case, kmax):
    return {"workload": args.workload, "what": WORKLOAD_TEXT[args.workload], "nx": case["nx"], "ny": case["ny"],
            "nz": case["nz"], "kmax": kmax, "columns": case["nx"] * case["ny"], "refine": args.refine,
            "proposal": args.proposal, "root_tolerance_km_s": 1e-6, "path": getattr(args, "path", "kernel"),
            "l2": "flushed between steps (256 MiB write)", "sphere": True}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        self.p = None
        if shutil.which("nvidia-smi"):
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() in ("active", "1"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                pass
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def fp64_peak_tflops(torch, dev):
    """Measured FP64 throughput of this GPU: cuBLAS float64 GEMM, best of 5."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    return best


def build_oracle_native():
    """The CPU baseline: the oracle built for this host (-march=native)."""
    d = tempfile.mkdtemp(prefix="swdo_")
    so = os.path.join(d, "libswd_oracle_native.so")
    src = os.path.join(ROOT, "oracle", "swd_oracle.cpp")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    try:
        subprocess.run([cxx, "-O3", "-march=native", "-fopenmp", "-fPIC", "-std=c++17", "-ffp-contract=off", "-shared",
                        "-o", so, src], check=True, capture_output=True)
        return so, "g++ -O3 -march=native -fopenmp"
    except Exception:
        return os.path.join(ROOT, "oracle", "libswd_oracle.so"), "g++ -O3 -fopenmp (portable build)"


def cpu_baseline(case, args, target_s):
    """The oracle port on all host threads over a bounded column sample."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import ctypes as C
    import oracle_lib as O
    so, how = build_oracle_native()
    O._LIB = C.CDLL(so)
    O._LIB.swdo_dltar.restype = C.c_double
    O._LIB.swdo_frechet_rows.restype = C.c_long
    cores = os.cpu_count() or 1
    ncol = case["nx"] * case["ny"]
    refine = 0  # the reference's own algorithm: surfdisp96's scan + nevill refinement
    n = min(ncol, max(cores, 8))
    fn = O.get_2d_map if getattr(args, "path", "kernel") == "map" else O.get_1d_kernel
    t0 = time.perf_counter()
    r = fn(case, refine=refine, nthreads=cores, cols=np.arange(n))
    dt = time.perf_counter() - t0
    kmax = r["vc"].shape[0]
    per_col = dt / n
    n2 = int(min(ncol, max(n, target_s / max(per_col, 1e-9))))
    n2 = max(cores, (n2 // cores) * cores) if n2 >= cores else n2
    n2 = min(n2, ncol)
    t0 = time.perf_counter()
    r = fn(case, refine=refine, nthreads=cores, cols=np.arange(n2))
    dt = time.perf_counter() - t0
    return {"value": n2 * kmax / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{n2} of {ncol} columns x {kmax} slots ({dt:.1f} s, {how}, OpenMP over columns, "
                      f"reference-faithful refinement)"}, n2, dt


FMST_METRIC = "fast-marching receivers/s (traveltime + ray-path Frechet weights, all station pairs)"
FMST_UNIT = "receivers/s"


def fmst_survey(rank=0):
    from jdsurfg_b200 import synth
    s = synth.make_survey("example", seed=7 + rank)
    slot, group = synth.survey_slots(s)
    p = s["pairs"]
    pairs = dict(slot=slot, srcx=p["srcx"], srcz=p["srcz"], group=group, rcv_ptr=p["rcv_ptr"], rcx=p["rcx"],
                 rcz=p["rcz"])
    return s, pairs


def fmst_config(s, pairs):
    nx, ny = s["grid"][:2]
    return {"workload": "fmst", "what": "station pairs shaped like the reference's example: 33x36 grid at 0.3 deg, "
                                        "41 nodes, 19 periods 4-40 s, Rayleigh phase+group, 80 stations, "
                                        "propagation grid 241x265 (8x dicing) plus 129x129 refined source grid",
            "pairs": int(len(pairs["slot"])), "receivers": int(pairs["rcv_ptr"][-1]), "nx": nx, "ny": ny}


def fmst_cpu_baseline(s, pairs, vc, vout, seconds):
    """The oracle's per-pair loop (travel_time / frechet_matrix restated) on
    every host core over the first pairs, sized to about `seconds`."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    cores = os.cpu_count() or 1
    rp = pairs["rcv_ptr"]

    def sub(n):
        return dict(slot=pairs["slot"][:n], srcx=pairs["srcx"][:n], srcz=pairs["srcz"][:n], group=pairs["group"][:n],
                    rcv_ptr=rp[:n + 1], rcx=pairs["rcx"], rcz=pairs["rcz"])
    n = min(len(pairs["slot"]), 4 * cores)
    t0 = time.perf_counter()
    O.fmst_pairs(s["grid"], sub(n), vc, vout, want_fdm=True, nthreads=cores)
    dt = time.perf_counter() - t0
    n2 = int(min(len(pairs["slot"]), max(n, n * seconds / max(dt, 1e-3))))
    t0 = time.perf_counter()
    O.fmst_pairs(s["grid"], sub(n2), vc, vout, want_fdm=True, nthreads=cores)
    dt = time.perf_counter() - t0
    return {"value": int(rp[n2]) / dt, "unit": FMST_UNIT, "cores": cores, "kind": "port",
            "sample": f"first {n2} of {len(pairs['slot'])} pairs ({int(rp[n2])} receivers), rays and weights for "
                      f"every receiver, OpenMP over pairs as SurfaceWave.cpp:583-672"}, n2


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    if args.workload == "fmst":
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib as O
        s, pairs = fmst_survey(0)
        m = O.get_2d_map(s["case"])
        per_step_s = max(2.0, 60.0 / max(1, args.steps + args.warmup))
        cb, n2 = fmst_cpu_baseline(s, pairs, m["vc"], m["vout"], per_step_s)
        line = {"impl": "reference", "metric": FMST_METRIC, "value": cb["value"], "unit": FMST_UNIT,
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * int(pairs["rcv_ptr"][-1]) / cb["value"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded generator, jdsurfg_b200/synth.py make_survey)",
                "config": dict(fmst_config(s, pairs), l2="flushed between steps (256 MiB write)"), "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": FMST_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0
    case = workload(args, 0)
    from jdsurfg_b200 import synth
    kmax = synth.kmax_of(case["tables"])
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    for _ in range(max(0, args.warmup)):
        pass
    per_step_s = max(2.0, 60.0 / max(1, args.steps + args.warmup))
    cb, n2, _ = cpu_baseline(case, args, per_step_s)
    import oracle_lib as O
    refine = 0  # reference-faithful: surfdisp96's own scan + nevill refinement
    cols = np.arange(n2)
    fn = O.get_2d_map if args.path == "map" else O.get_1d_kernel
    for _ in range(args.warmup):
        fn(case, refine=refine, nthreads=cb["cores"], cols=cols[:max(1, n2 // 4)])
    t0 = time.perf_counter()
    for _ in range(args.steps):
        fn(case, refine=refine, nthreads=cb["cores"], cols=cols)
    dt = time.perf_counter() - t0
    value = args.steps * n2 * kmax / dt
    cb["value"] = value
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, jdsurfg_b200/synth.py)", "config": case_desc(args, case, kmax),
            "cpu_baseline": cb, "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


LSMR_METRIC = "LSMR iterations/s over the Frechet rows (A x and A^T y per iteration)"
LSMR_UNIT = "iterations/s"


def lsmr_matrix(torch, dev, seed=11):
    """A sparse matrix shaped like the example survey's Frechet rows: 42879
    receiver rows over a 33x36 grid of 30 nodes (35640 cells); each row a
    ray band of 128 consecutive grid columns times the 30 depths (3840
    nonzeros, 165 M in all), FP32 values.  Built on the device."""
    from jdsurfg_b200.lsmr import DeviceCSR
    m, nxy, nz, w = 42879, 33 * 36, 30, 128
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    start = torch.randint(0, nxy - w, (m,), generator=g, device=dev)
    cols = start[:, None] + torch.arange(w, device=dev)[None, :]
    idx = (cols[:, :, None] * nz + torch.arange(nz, device=dev)[None, None, :]).reshape(-1).to(torch.int32)
    rowptr = torch.arange(m + 1, device=dev, dtype=torch.int64) * (w * nz)
    val = (torch.randn(m * w * nz, generator=g, device=dev) * 1e-3).to(torch.float32)
    A = DeviceCSR(rowptr, idx, val, m, nxy * nz)
    xt = torch.randn(nxy * nz, generator=g, device=dev, dtype=torch.float64)
    b = torch.zeros(m, dtype=torch.float64, device=dev)
    A.aprod(1, xt, b)
    b += 1e-4 * torch.randn(m, generator=g, device=dev, dtype=torch.float64)
    return A, b


def run_lsmr(args, torch, dev, rank, world, pg):
    """One step = K LSMR iterations (SurfTime's damped least-squares solve,
    lsmrModule_csr.f90) on the device over a Frechet-shaped CSR matrix;
    value = iterations/s.  e2e = the same solve with b from and x to pinned
    host memory."""
    from jdsurfg_b200.lsmr import lsmr
    K = 50
    A, b = lsmr_matrix(torch, dev, seed=11 + rank)
    nnz = int(A.indices.numel())
    for _ in range(args.warmup):
        lsmr(A, b, damp=0.1, atol=0.0, btol=0.0, conlim=0.0, itnlim=K)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev.index)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    its = 0
    for _ in range(args.steps):
        x, info = lsmr(A, b, damp=0.1, atol=0.0, btol=0.0, conlim=0.0, itnlim=K)
        its += info["itn"]  # the solve may stop at machine precision before K
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    its_step = its / args.steps
    if pg:
        t = torch.tensor([ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    # e2e: b from pinned host memory, x back to pinned host memory
    hb = b.cpu().pin_memory()
    hx = torch.empty(A.n, dtype=torch.float64).pin_memory()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    its_e2e = 0
    for _ in range(args.steps):
        xd, inf = lsmr(A, hb.to(dev, non_blocking=True), damp=0.1, atol=0.0, btol=0.0, conlim=0.0, itnlim=K)
        hx.copy_(xd)
        its_e2e += inf["itn"]
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / its_e2e  # seconds per iteration
    # algorithmic bytes per iteration: A (int32 index + FP32 value per
    # nonzero) read by A x and its transpose by A^T y, both row-pointer
    # arrays, and the FP64 vectors read and written once each
    per_it = 2 * nnz * 8 + (A.m + A.n + 2) * 8 + 4 * (A.m + A.n) * 8
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fp:
            peaks = json.load(fp)
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs") or 6650.0
    achieved = per_it * its_step / (ms * 1e-3) / 1e9
    if rank == 0:
        cb = None
        if not args.no_cpu_baseline:
            cb = lsmr_cpu_baseline(A, b, args.cpu_seconds)
        line = {"metric": LSMR_METRIC, "value": world * its_step / (ms * 1e-3), "unit": LSMR_UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64 vectors, f32 matrix values",
                "data": "synthetic Frechet-shaped CSR (bench.py lsmr_matrix)",
                "config": {"workload": "lsmr", "rows": A.m, "cols": A.n, "nonzeros": nnz, "iteration_limit": K,
                           "iterations_per_step": its_step,
                           "damp": 0.1, "solver": "swdk_lsmr_solve: products of A and of its device transpose, "
                                                  "norms and scalar recurrences on the device",
                           "l2": "inputs (1.3 GB of CSR per product) larger than L2"},
                "clocks": clk,
                "e2e": {"value": world / e2e_s, "unit": LSMR_UNIT, "h2d_bytes_per_step": int(A.m * 8),
                        "d2h_bytes_per_step": int(A.n * 8)},
                "gpu_launches": None,
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                             "traffic": None, "bytes_per_iteration": per_it,
                             "note": "per iteration two SpMV over the 165 M nonzeros, four fixed-grid norm "
                                     "reductions and the one-thread recurrences; the host reads the state every "
                                     "16 iterations"},
                "cpu_baseline": cb, "istop": info["istop"], "itn": info["itn"]}
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def lsmr_cpu_baseline(A, b, seconds):
    """scipy's LSMR (FP64, one thread) on the same matrix copied to the host,
    for as many iterations as fit the time budget."""
    import scipy.sparse as sp
    from scipy.sparse.linalg import lsmr as sp_lsmr
    M = sp.csr_matrix((A.values.cpu().numpy().astype(np.float64), A.indices.cpu().numpy(), A.rowptr.cpu().numpy()),
                      shape=(A.m, A.n))
    bb = b.cpu().numpy()
    t0 = time.perf_counter()
    sp_lsmr(M, bb, damp=0.1, atol=0.0, btol=0.0, conlim=0.0, maxiter=2)
    per = (time.perf_counter() - t0) / 2
    k = max(2, int(seconds / max(per, 1e-6)))
    k = min(k, 200)
    t0 = time.perf_counter()
    done = sp_lsmr(M, bb, damp=0.1, atol=0.0, btol=0.0, conlim=0.0, maxiter=k)[2]
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": LSMR_UNIT, "cores": 1, "kind": "port",
            "sample": f"scipy.sparse.linalg.lsmr, {done} iterations on the same matrix in FP64 (the reference runs "
                      "lsmrModule_csr.f90 in FP32 with OpenMP products; no Fortran compiler here)"}


def run_fmst(args, torch, dev, rank, world, pg):
    """One step = fast marching, receiver times, rays and ray-path Frechet
    weights of every station pair of the example-shaped survey, with the
    phase/group maps (from the GPU engine) resident in HBM; e2e = the whole
    SurfTime.frechet_matrix (dispersion kernels, fast marching, CSR rows)
    from the host model to the host data vector."""
    from jdsurfg_b200 import Engine
    from jdsurfg_b200.fmst import FMST
    from jdsurfg_b200.surftime import SurfTime
    s, pairs = fmst_survey(rank)
    case = s["case"]
    nx, ny = s["grid"][:2]
    nz = len(case["depth"])
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream
    eng = Engine(device=dev.index)
    eng.setup(case)
    vs = torch.from_numpy(case["vs"]).to(dev)
    vc = torch.empty((eng.kmax, nx * ny), dtype=torch.float64, device=dev)
    vout = torch.empty_like(vc)
    ker = torch.empty((eng.kmax, nz, nx * ny), dtype=torch.float64, device=dev)
    st = torch.empty((eng.kmax, nx * ny), dtype=torch.int32, device=dev)
    eng.get_1d_kernel_device(nx, ny, nz, vs, None, None, vc, vout, ker, st, stream=sp)
    torch.cuda.synchronize()
    f = FMST(*s["grid"], device=dev.index)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        flush.fill_(1)
        r = f.pairs(pairs, vc, vout, want_fdm=True, stream=sp)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev.index)
    ms, dev_ms = 0.0, 0.0
    for _ in range(args.steps):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = f.pairs(pairs, vc, vout, want_fdm=True, stream=sp)
        e1.record(stream)
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
        dev_ms += f.last_info()["ms"]
    clk = clocks.stop()
    info = f.last_info()
    ok = int((r["status"] == 0).sum().item())
    if pg:
        t = torch.tensor([ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    nrcv = int(pairs["rcv_ptr"][-1])
    # e2e through the public API: host model in, host data out
    stt = SurfTime(device=dev.index)
    stt.set_model(case["depth"], *s["grid"][2:], nx, ny)
    stt.set_data(s["tables"], s["kmax_per_mode"], s["pairs"])
    stt.frechet_matrix(case["vs"])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        data, nnz = stt.frechet_matrix(case["vs"])
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / args.steps
    stt.close()
    # algorithmic bytes of the marching kernel per pair: the propagation grid
    # (8-byte time+status per node) written and read once, its slowness read
    # once, and the same for the 129x129 refined grid
    N = f.nnx * f.nnz
    alg = len(pairs["slot"]) * (N * 20 + 129 * 129 * 20)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fp:
            peaks = json.load(fp)
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs") or 6650.0
    achieved = alg / (dev_ms / args.steps * 1e-3) / 1e9
    if rank == 0:
        cb = None
        if not args.no_cpu_baseline:
            cb, _ = fmst_cpu_baseline(s, pairs, vc.cpu().numpy(), vout.cpu().numpy(), args.cpu_seconds)
        line = {"metric": FMST_METRIC, "value": world * nrcv / (ms / args.steps * 1e-3), "unit": FMST_UNIT,
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded generator, jdsurfg_b200/synth.py make_survey)",
                "config": dict(fmst_config(s, pairs), l2="flushed between steps (256 MiB write)"),
                "detail": {"max_band": info["max_band"], "receivers_ok": ok},
                "clocks": clk,
                "e2e": {"value": world * nrcv / e2e_s, "unit": FMST_UNIT,
                        "h2d_bytes_per_step": int(case["vs"].nbytes), "d2h_bytes_per_step": int(nrcv * 4),
                        "what": "SurfTime.frechet_matrix: host model -> get_1d_kernel, fast marching, rays, "
                                "CSR rows on the device -> host data vector", "nonzeros": int(nnz)},
                "gpu_launches": 5 * args.steps,
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                             "frac": achieved / hbm, "traffic": None,
                             "note": "the marching is one dependent chain per pair (heap order); latency-bound, "
                                     "the HBM fraction only states how far from bandwidth it is"},
                "cpu_baseline": cb}
        print(json.dumps(line), flush=True)
    f.close()
    eng.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def run_uneven(args, torch, dev, rank, world, pg):
    """One step = one CUDA-graph launch over the 48-model uneven batch."""
    from jdsurfg_b200 import synth
    from jdsurfg_b200.batch import UnevenBatch
    cases = synth.make_uneven_batch(48, seed=5150 + rank)
    B = UnevenBatch(cases, learned=(args.proposal == "learned"), mode=args.uneven_mode)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    B.capture()
    probe = None
    if args.uneven_mode == "ragged":
        B.run()  # one eager pass: stage times and evaluation counts
        probe = B.stats()
    for _ in range(args.warmup):
        flush.fill_(1)
        B.launch(stream.cuda_stream)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev.index)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        flush.fill_(1)
        B.launch(stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    if pg:
        t = torch.tensor([ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    units = B.units
    if probe is not None:
        launches = probe["kernel_launches"]
    else:
        launches = sum(e.stats()["kernel_launches"] for e in B.engines)  # per model, from the eager pass
    kb = sum(c["nx"] * c["ny"] * c["nz"] * e.kmax * 8 for c, e in zip(cases, B.engines))
    roofline = None
    if probe is not None and probe["ms_roots"] > 0:
        peak = fp64_peak_tflops(torch, dev)
        fl = probe["layer_evals_rayleigh"] * F_SEC_RAYLEIGH + probe["layer_evals_love"] * F_SEC_LOVE
        ach = fl / (probe["ms_roots"] * 1e-3) / 1e12
        roofline = {"kernel": "k_roots_queue+k_retry (one ragged launch each)", "bound": "fp64", "achieved": ach,
                    "peak": peak, "unit": "TFLOP/s", "frac": ach / peak, "traffic": None,
                    "work": "secular evaluations done (learned path) x layers x flops per layer",
                    "peak_source": "measured in this run: cuBLAS float64 GEMM 8192^3",
                    "stage_ms": {k: probe[k] for k in ("ms_prep", "ms_proposal", "ms_roots", "ms_eigen")},
                    "evals_per_slot_by_phase": {k: v / units for k, v in probe["evals_by_phase"].items()}}
    if rank == 0:
        line = {"metric": METRIC, "value": world * units / (ms / args.steps * 1e-3), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded generator, jdsurfg_b200/synth.py make_uneven_batch)",
                "config": {"workload": "uneven", "what": WORKLOAD_TEXT["uneven"], "models": len(cases),
                           "slots_per_step": units, "kernel_bytes": kb, "proposal": args.proposal,
                           "timed_as": ("one CUDA graph launch per step: per-model column preparation and "
                                        "proposals, one persistent root search over every (model, chain, column), "
                                        "one retry launch, one eigen launch per wave type over every (model, column)")
                           if args.uneven_mode == "ragged" else
                           "one CUDA graph launch per step (a branch per model)",
                           "l2": "flushed between steps (256 MiB write)"},
                "clocks": clk, "e2e": None, "gpu_launches": launches * args.steps, "roofline": roofline,
                "cpu_baseline": None}
        print(json.dumps(line), flush=True)
    B.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def run_sharded(args, torch, dev, rank, world, pg):
    """Strong scaling of get_1d_kernel over the ranks: every rank holds the
    same model (the workload's seed 2024 grid) in HBM, computes its column
    block (jdsurfg_b200/shard.py, the reference's allocate_tasks split) and
    the maps are all-gathered on the devices; depth kernels stay with the
    rank that computed them.  value = all slots of the one model / step time
    (max over ranks)."""
    from jdsurfg_b200 import Engine, learn
    from jdsurfg_b200.shard import ShardedSurfTime, column_block
    case = workload(args, 0)
    eng = Engine(device=dev.index, refine=args.refine)
    if args.proposal == "learned":
        learn.load_proposals(eng)
    eng.setup(case)
    ncol, kmax = case["nx"] * case["ny"], eng.kmax
    units = ncol * kmax
    sh = ShardedSurfTime(rank, world, engine=eng)
    t = lambda a: None if a is None else torch.from_numpy(a).to(dev)
    vs, vp, rho = t(case["vs"]), t(case["vp"]), t(case["rho"])
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step():
        flush.fill_(1)
        return sh.get_1d_kernel_device(vs, vp, rho, stream=sptr)

    for _ in range(args.warmup):
        r = step()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev.index)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        r = step()
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    if pg:
        tt = torch.tensor([ms], device=dev)
        pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        ms = float(tt.item())
    c0, c1 = column_block(ncol, world, rank)
    gather_bytes = 3 * kmax * (-(-ncol // world)) * 8 * world
    launches = eng.stats()["kernel_launches"] * args.steps
    if rank == 0:
        line = {"metric": METRIC, "value": units / (ms / args.steps * 1e-3), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded generator, jdsurfg_b200/synth.py)",
                "config": dict(case_desc(args, case, kmax), sharded=True,
                               timed_as="per step: the rank's column block through get_1d_kernel_device, then the "
                                        "NCCL all-gather of the vc/vout/status maps (device tensors)",
                               columns_rank0=c1 - c0, all_gather_bytes_per_step=gather_bytes),
                "clocks": clk, "e2e": None, "gpu_launches": launches, "roofline": None, "cpu_baseline": None}
        print(json.dumps(line), flush=True)
    eng.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    if args.workload == "uneven":
        return run_uneven(args, torch, dev, rank, world, pg)
    if args.workload == "fmst":
        return run_fmst(args, torch, dev, rank, world, pg)
    if args.workload == "lsmr":
        return run_lsmr(args, torch, dev, rank, world, pg)
    if args.sharded:
        return run_sharded(args, torch, dev, rank, world, pg)
    from jdsurfg_b200 import Engine
    case = workload(args, rank)
    eng = Engine(device=local, refine=args.refine, split_cols=args.split_cols, block_roots=args.roots_blocks,
                 node_layers=not args.no_node_layers)
    nets = None
    from jdsurfg_b200 import learn
    eng_nets_on = [args.proposal == "learned"]  # whether the timed engine has the proposal attached
    if args.proposal == "learned":
        nets, _ = learn.load_proposals(eng)
    eng.setup(case)
    nx, ny, nz = case["nx"], case["ny"], case["nz"]
    ncol, kmax = nx * ny, eng.kmax
    units = ncol * kmax
    vs = torch.from_numpy(case["vs"]).to(dev)
    vp = None if case["vp"] is None else torch.from_numpy(case["vp"]).to(dev)
    rho = None if case["rho"] is None else torch.from_numpy(case["rho"]).to(dev)
    vc = torch.empty((kmax, ncol), dtype=torch.float64, device=dev)
    vout = torch.empty_like(vc)
    mapped = args.path == "map"
    ker = None if mapped else torch.empty((kmax, nz, ncol), dtype=torch.float64, device=dev)
    st = torch.empty((kmax, ncol), dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    # one explicit stream for the flush, the engine's work and the timing
    # events (a NULL stream handle would mean the engine's own stream)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream

    def call(e):
        if mapped:
            e.get_2d_map_device(nx, ny, nz, vs, vp, rho, vc, vout, st, stream=sptr)
        else:
            e.get_1d_kernel_device(nx, ny, nz, vs, vp, rho, vc, vout, ker, st, stream=sptr)

    def step():
        flush.fill_(1)
        call(eng)

    roots_blocks = eng.autotune(nx, ny, nz, vs, vp, rho) if not args.no_graph and not args.roots_blocks else None
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    STAT_KEYS = ("ms_roots", "ms_proposal", "ms_eigen", "ms_prep", "secular_evals", "layer_evals_rayleigh",
                 "layer_evals_love", "proposals_accepted", "proposals_rejected", "kernel_launches")

    def timed(nsteps):
        """device time of nsteps steps (max over ranks) and stage stats per step x nsteps.
        The per-stage figures come from one eager probe call (CUDA events inside the
        engine); the timed steps replay the captured CUDA graph of that call."""
        step()
        launches = eng.stats()["kernel_launches"]
        # stage breakdown from one call of an unsplit engine with the same
        # settings (the timed call runs as two overlapping column halves,
        # whose stage times do not add up)
        probe_eng = Engine(device=local, refine=args.refine, split_cols=-1, node_layers=not args.no_node_layers)
        if eng_nets_on[0]:
            learn.load_proposals(probe_eng)
        probe_eng.setup(case)
        call(probe_eng)
        probe = probe_eng.stats()
        probe_eng.close()
        acc = {k: probe[k] * nsteps for k in STAT_KEYS}
        acc["kernel_launches"] = launches * nsteps
        acc["evals_by_phase"] = probe["evals_by_phase"]
        use_graph = not args.no_graph
        if use_graph:
            eng.graph_capture(args.path, nx, ny, nz, vs, vp, rho, vc, vout, ker, st)
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(nsteps):
            if use_graph:
                flush.fill_(1)
                eng.graph_launch(sptr)
            else:
                step()
        e1.record(stream)
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if pg:
            t = torch.tensor([ms], device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            ms = float(t.item())
        return ms, acc

    clocks = ClockSampler(local)
    ms, acc = timed(args.steps)
    clk = clocks.stop()
    ms_per_step = ms / args.steps
    value = world * units / (ms_per_step * 1e-3)
    roots_ms, lr, ll, evals = acc["ms_roots"], acc["layer_evals_rayleigh"], acc["layer_evals_love"], acc["secular_evals"]
    stats = eng.stats()
    status = np.bincount(st.cpu().numpy().ravel(), minlength=5).tolist()
    vc_learned = vc.cpu().numpy() if args.proposal == "learned" and not args.no_plain else None

    plain = None
    alg_lr, alg_ll = lr, ll  # algorithmic layer-evaluations: the plain method's count
    if args.proposal == "learned" and not args.no_plain:
        eng.set_proposal(None, None)
        eng_nets_on[0] = False
        for _ in range(1):
            step()
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        pms, pacc = timed(args.steps)
        dmax = float(np.abs(vc.cpu().numpy() - vc_learned).max())
        alg_lr, alg_ll = pacc["layer_evals_rayleigh"], pacc["layer_evals_love"]
        plain = {"value": world * units / (pms / args.steps * 1e-3), "ms_per_step": pms / args.steps,
                 "ms_roots": pacc["ms_roots"] / args.steps,
                 "evals_per_slot": pacc["secular_evals"] / args.steps / units,
                 "learned_speedup": (pms / args.steps) / ms_per_step,
                 "learned_roots_speedup": pacc["ms_roots"] / max(1e-9, roots_ms + acc["ms_proposal"]),
                 "learned_eval_reduction": pacc["secular_evals"] / max(1, evals),
                 "evals_per_slot_by_phase": {k: v / units for k, v in pacc["evals_by_phase"].items()},
                 "max_abs_dc_learned_vs_plain_km_s": dmax}
        nets, _ = learn.load_proposals(eng)  # the e2e leg runs the learned path again
        eng_nets_on[0] = True

    # e2e: host-memory C-ABI call, pinned buffers, copies in the timed region
    e2e = None
    if not args.no_e2e:
        pin = lambda shape, dt: torch.empty(shape, dtype=dt, pin_memory=True).numpy()
        h_vs = pin(case["vs"].shape, torch.float32)
        h_vs[...] = case["vs"]
        h_vp = h_rho = None
        if case["vp"] is not None:
            h_vp = pin(case["vp"].shape, torch.float32)
            h_vp[...] = case["vp"]
            h_rho = pin(case["rho"].shape, torch.float32)
            h_rho[...] = case["rho"]
        h_vc, h_vout = pin((kmax, ncol), torch.float64), pin((kmax, ncol), torch.float64)
        h_ker = None if mapped else pin((kmax, nz, ncol), torch.float64)
        h_st = pin((kmax, ncol), torch.int32)
        import ctypes as C
        from jdsurfg_b200.engine import lib, _p

        def host_step():
            if mapped:
                rc = lib().swdk_get_2d_map(eng._h, nx, ny, nz, _p(h_vs), _p(h_vp), _p(h_rho), _p(h_vc), _p(h_vout),
                                           _p(h_st))
            else:
                rc = lib().swdk_get_1d_kernel(eng._h, nx, ny, nz, _p(h_vs), _p(h_vp), _p(h_rho), _p(h_vc),
                                              _p(h_vout), _p(h_ker), _p(h_st))
            assert rc == 0, rc

        host_step()
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            flush.fill_(1)
            host_step()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        if pg:
            t = torch.tensor([dt], device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            dt = float(t.item())
        h2d = h_vs.nbytes + (0 if h_vp is None else h_vp.nbytes + h_rho.nbytes)
        d2h = h_vc.nbytes + h_vout.nbytes + (0 if h_ker is None else h_ker.nbytes) + h_st.nbytes
        e2e = {"value": world * units * args.steps / dt, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h)}

    # roofline of the dominant kernels: the root search (k_roots_queue +
    # k_retry; FP64 secular functions) and the proposal network (tcgen05 GEMMs)
    peak = fp64_peak_tflops(torch, dev)
    flops = alg_lr * F_SEC_RAYLEIGH + alg_ll * F_SEC_LOVE
    achieved = flops / (roots_ms * 1e-3) / 1e12 if roots_ms > 0 else 0.0
    roofline = {"kernel": "k_roots_queue+k_retry", "bound": "fp64", "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": achieved / peak if peak else None, "traffic": None,
                "peak_source": "measured in this run: cuBLAS float64 GEMM 8192^3 (MEASURED_PEAKS.json has no FP64 figure)",
                "flops_per_layer_eval": {"rayleigh": F_SEC_RAYLEIGH, "love": F_SEC_LOVE},
                "work": "plain-method secular evaluations x layers x flops per layer (the learned "
                        "path's saved evaluations show up as a shorter duration)",
                "share_of_step": roots_ms / ms if ms else None}
    # the eigen stage (k_eigen): passes x layers x F_EIG over its measured
    # stage time, and the write-out bandwidth of its outputs
    from jdsurfg_b200 import synth as _synth
    passes = {"rayleigh": 0, "love": 0}
    for w, tab in enumerate(case["tables"]):
        if tab is None:
            continue
        nslot = _synth.kmax_of([tab if i == w else None for i in range(4)])
        # kernel path: one pass per phase slot, three per group slot; map
        # path: one pass per group slot (disp1D's sregn96/slegn96 for U)
        per = (1 if w in (1, 3) else 0) if mapped else (3 if w in (1, 3) else 1)
        passes["rayleigh" if w < 2 else "love"] += nslot * per
    L = 4 * nz - 3
    eig_flops = ncol * L * (passes["rayleigh"] * F_EIG_RAYLEIGH + passes["love"] * F_EIG_LOVE) * args.steps
    eig_s = acc["ms_eigen"] * 1e-3
    out_bytes = (ncol * kmax * ((0 if mapped else nz) + 2) * 8 + ncol * kmax * 4) * args.steps  # kernel, vc, vout, status
    if eig_s > 0:
        ach_e = eig_flops / eig_s / 1e12
        roofline["eigen"] = {"kernel": "k_eigen", "bound": "fp64", "achieved": ach_e, "peak": peak, "unit": "TFLOP/s",
                             "frac": ach_e / peak if peak else None, "traffic": None,
                             "flops_per_layer_pass": {"rayleigh": F_EIG_RAYLEIGH, "love": F_EIG_LOVE},
                             "passes_per_column": passes, "layers": L,
                             "writeout_gbs": out_bytes / eig_s / 1e9,
                             "writeout_bytes_per_step": out_bytes // args.steps,
                             "share_of_step": acc["ms_eigen"] / ms}
    if args.proposal == "learned" and acc["ms_proposal"] > 0:
        peaks = {}
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
                peaks = json.load(f)
        except Exception:
            pass
        bf16_peak = peaks.get("bf16_tflops") or 1590.0
        rows = units  # one proposal row per root slot
        gflops = 2.0 * rows * MLP_MACS_PER_ROW * args.steps
        ach = gflops / (acc["ms_proposal"] * 1e-3) / 1e12
        roofline["proposal"] = {"kernel": "k_features+k_mlp_propose", "bound": "tensor", "achieved": ach,
                                "peak": bf16_peak, "unit": "TFLOP/s", "frac": ach / bf16_peak,
                                "peak_source": "MEASURED_PEAKS.json bf16_tflops" if peaks.get("bf16_tflops")
                                else "fallback 1590 TFLOP/s",
                                "share_of_step": acc["ms_proposal"] / ms}

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb, _, _ = cpu_baseline(case, args, args.cpu_seconds)
        except Exception as ex:  # the baseline is reported, never required
            cb = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {ex}"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded generator, jdsurfg_b200/synth.py); no public dataset exists for this path",
                "config": case_desc(args, case, kmax),
                "timing": {"timed_as": "eager calls" if args.no_graph else
                           "CUDA-graph replays of one get_1d_kernel_device call",
                           "roots_blocks_autotuned": roots_blocks}, "clocks": clk, "e2e": e2e,
                "gpu_launches": int(acc["kernel_launches"]), "roofline": roofline, "cpu_baseline": cb,
                "plain": plain,
                "detail": {"secular_evals_per_step": evals / args.steps,
                           "evals_per_slot": evals / args.steps / units,
                           "evals_per_slot_by_phase": {k: v / units for k, v in acc["evals_by_phase"].items()},
                           "proposals_used": acc["proposals_accepted"] / args.steps,
                           "proposals_fell_back": acc["proposals_rejected"] / args.steps,
                           "ms_prep": acc["ms_prep"] / args.steps, "ms_proposal": acc["ms_proposal"] / args.steps,
                           "ms_roots": roots_ms / args.steps, "ms_eigen": acc["ms_eigen"] / args.steps,
                           "status_counts": status}}
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
