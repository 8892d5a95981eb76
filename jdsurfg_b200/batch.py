"""Uneven batches: many independent models (different grids, depth vectors,
period tables, wave types and modes) computed by one CUDA-graph launch.

Each model keeps its own Engine (period tables, depth vector, plans).  Two
ways to run them:

* "ragged" (default, swdk_ragged_*): every model's column preparation and
  proposals, then ONE persistent root-search launch over all (model, chain,
  column) items, one retry launch and one eigen launch per wave type over
  all (model, column) blocks, captured as one graph;
* "branches" (swdk_batch_graph_create): the graph forks one branch of each
  model's own pipeline off a main stream, so models run side by side.

The learned proposal networks are loaded once and shared by all models.
"""
import ctypes as C

import numpy as np

from .engine import Call, Engine, SwdkError, lib


class UnevenBatch:
    def __init__(self, cases, device=0, learned=True, path="kernel", mode="ragged"):
        import torch
        from . import learn
        if mode not in ("ragged", "branches"):
            raise ValueError(mode)
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.path = path
        self.mode = mode
        self.ragged = None
        self.cases = cases
        self.engines, self.bufs = [], []
        self.nets = None
        kr = kl = None
        for i, case in enumerate(cases):
            eng = Engine(device=device)
            if learned:
                if self.nets is None:
                    self.nets, meta = learn.load_proposals(eng)
                    kr, kl = meta["engine_kappa"]["rayleigh"], meta["engine_kappa"]["love"]
                else:
                    eng.set_proposal(self.nets.get("rayleigh"), self.nets.get("love"), kr, kl)
            eng.setup(case)
            nx, ny, nz = case["nx"], case["ny"], case["nz"]
            kmax, ncol = eng.kmax, nx * ny
            t = lambda a: None if a is None else torch.from_numpy(a).to(self.dev)
            b = dict(vs=t(case["vs"]), vp=t(case["vp"]), rho=t(case["rho"]),
                     vc=torch.zeros((kmax, ncol), dtype=torch.float64, device=self.dev),
                     st=torch.zeros((kmax, ncol), dtype=torch.int32, device=self.dev))
            b["vout"] = torch.zeros_like(b["vc"])
            b["ker"] = (torch.zeros((kmax, nz, ncol), dtype=torch.float64, device=self.dev) if path == "kernel"
                        else None)
            self.engines.append(eng)
            self.bufs.append(b)
        self.graph = None

    @property
    def units(self):
        """column-period-mode slots of one launch"""
        return sum(c["nx"] * c["ny"] * e.kmax for c, e in zip(self.cases, self.engines))

    def _call(self, i):
        c, b = self.cases[i], self.bufs[i]
        p = lambda x: None if x is None else x.data_ptr()
        return Call(0 if self.path == "kernel" else 1, c["nx"], c["ny"], c["nz"], p(b["vs"]), p(b["vp"]),
                    p(b["rho"]), p(b["vc"]), p(b["vout"]), p(b["ker"]), p(b["st"]))

    def _ragged(self):
        if self.ragged is None:
            n = len(self.engines)
            calls = (Call * n)(*[self._call(i) for i in range(n)])
            ctxs = (C.c_void_p * n)(*[e._h.value for e in self.engines])
            r = C.c_void_p()
            rc = lib().swdk_ragged_create(n, ctxs, calls, C.byref(r))
            if rc != 0:
                raise SwdkError(f"swdk_ragged_create failed ({rc}): "
                                f"{lib().swdk_last_error(self.engines[0]._h).decode()}")
            self.ragged = r
        return self.ragged

    def run(self, stream=None):
        """One eager pass of the ragged batch (statistics in stats())."""
        rc = lib().swdk_ragged_run(self._ragged(), stream)
        if rc != 0:
            raise SwdkError(f"swdk_ragged_run failed ({rc}): {lib().swdk_last_error(self.engines[0]._h).decode()}")

    def stats(self):
        from .engine import Stats, stats_dict
        s = Stats()
        rc = lib().swdk_ragged_stats(self._ragged(), C.byref(s))
        if rc != 0:
            raise SwdkError(f"swdk_ragged_stats failed ({rc})")
        return stats_dict(s)

    def capture(self):
        if self.mode == "ragged":
            self._ragged()
            return
        n = len(self.engines)
        calls = (Call * n)(*[self._call(i) for i in range(n)])
        ctxs = (C.c_void_p * n)(*[e._h.value for e in self.engines])
        g = C.c_void_p()
        rc = lib().swdk_batch_graph_create(n, ctxs, calls, C.byref(g))
        if rc != 0:
            raise SwdkError(f"swdk_batch_graph_create failed ({rc}): {lib().swdk_last_error(self.engines[0]._h).decode()}")
        self.graph = g

    def launch(self, stream=None):
        if self.mode == "ragged":
            rc = lib().swdk_ragged_launch(self._ragged(), stream)
            if rc != 0:
                raise SwdkError(f"swdk_ragged_launch failed ({rc}): "
                                f"{lib().swdk_last_error(self.engines[0]._h).decode()}")
            return
        if self.graph is None:
            self.capture()
        rc = lib().swdk_batch_graph_launch(self.graph, stream)
        if rc != 0:
            raise SwdkError(f"swdk_batch_graph_launch failed ({rc})")

    def run_eager(self, i, stream=None):
        """Model i through its own device call (for comparison)."""
        c, b, eng = self.cases[i], self.bufs[i], self.engines[i]
        if self.path == "kernel":
            eng.get_1d_kernel_device(c["nx"], c["ny"], c["nz"], b["vs"], b["vp"], b["rho"], b["vc"], b["vout"], b["ker"],
                                     b["st"], stream=stream)
        else:
            eng.get_2d_map_device(c["nx"], c["ny"], c["nz"], b["vs"], b["vp"], b["rho"], b["vc"], b["vout"], b["st"],
                                  stream=stream)

    def outputs(self, i):
        self.torch.cuda.synchronize(self.dev)
        b = self.bufs[i]
        out = dict(vc=b["vc"].cpu().numpy(), vout=b["vout"].cpu().numpy(), status=b["st"].cpu().numpy())
        if b["ker"] is not None:
            out["kernel"] = b["ker"].cpu().numpy()
        return out

    def close(self):
        if self.graph is not None:
            lib().swdk_batch_graph_destroy(self.graph)
            self.graph = None
        if self.ragged is not None:
            lib().swdk_ragged_destroy(self.ragged)
            self.ragged = None
        for e in self.engines:
            e.close()
        self.engines = []
