"""Column sharding of the SurfTime path over ranks (one process per GPU).

Every (column, wave, mode) of the model is independent (the reference's
OpenMP loop over columns, SurfaceWave.cpp:469), so ranks take contiguous
column blocks with no exchange on the data path.  The one exchange the
inversion needs downstream is the dispersion maps: fast marching of every
period runs on the full nx x ny map, so vc/vout are all-gathered; the
depth kernels stay where
they were computed, next to the Frechet-row assembly that consumes them.

Blocks follow the reference's own task split (allocate_tasks,
src/shared/parallel.cpp:3-19): the first ntasks % nprocs ranks get one
extra column.

The per-block computation is injected (`compute`), so the host logic --
block bounds, padding, gather and reassembly -- is tested on CPU with gloo
ranks; on GPUs the default computes with the rank's Engine.
"""
import numpy as np


def column_block(ncol, world, rank):
    """[start, end) of rank's columns, the reference's allocate_tasks split."""
    sub = ncol // world
    extra = ncol - world * sub
    if rank < extra:
        start = rank * (sub + 1)
        return start, start + sub + 1
    start = extra + rank * sub
    return start, start + sub


class ShardedSurfTime:
    """get_2d_map / get_1d_kernel of one model split by columns across the
    ranks of a torch.distributed process group."""

    def __init__(self, rank, world, group=None, engine=None, compute=None):
        self.rank, self.world, self.group = rank, world, group
        self.engine = engine
        self.compute = compute

    def _block(self, arr, c0, c1):
        return None if arr is None else np.ascontiguousarray(arr[:, c0:c1])

    def _local(self, path, vs, vp, rho, c0, c1):
        vs_b, vp_b, rho_b = self._block(vs, c0, c1), self._block(vp, c0, c1), self._block(rho, c0, c1)
        if self.compute is not None:
            return self.compute(path, vs_b, vp_b, rho_b)
        f = self.engine.get_1d_kernel if path == "kernel" else self.engine.get_2d_map
        return f(vs_b, vp_b, rho_b, nx=c1 - c0, ny=1)

    def _gather_maps(self, vc, vout, st, ncol):
        """All-gather (kmax, block) maps into (kmax, ncol) on every rank."""
        import torch
        import torch.distributed as dist
        kmax = vc.shape[0]
        bmax = -(-ncol // self.world)  # the largest block
        pack = np.zeros((3, kmax, bmax), np.float64)
        n = vc.shape[1]
        pack[0, :, :n] = vc
        pack[1, :, :n] = vout
        pack[2, :, :n] = st
        t = torch.from_numpy(pack)
        if dist.get_backend(self.group) == "nccl":
            t = t.cuda()
        outs = [torch.empty_like(t) for _ in range(self.world)]
        dist.all_gather(outs, t, group=self.group)
        full = np.zeros((3, kmax, ncol), np.float64)
        for r, o in enumerate(outs):
            c0, c1 = column_block(ncol, self.world, r)
            full[:, :, c0:c1] = o.cpu().numpy()[:, :, :c1 - c0]
        return full[0], full[1], full[2].astype(np.int32)

    def get_2d_map(self, vs, vp=None, rho=None):
        """Full (kmax, ncol) vc, vout, status on every rank."""
        ncol = vs.shape[1]
        c0, c1 = column_block(ncol, self.world, self.rank)
        r = self._local("map", vs, vp, rho, c0, c1)
        vc, vout, st = self._gather_maps(r["vc"], r["vout"], r["status"], ncol)
        return dict(vc=vc, vout=vout, status=st)

    def get_1d_kernel(self, vs, vp=None, rho=None):
        """Full vc/vout/status maps on every rank; the kernel block of this
        rank's columns [c0, c1) stays local."""
        ncol = vs.shape[1]
        c0, c1 = column_block(ncol, self.world, self.rank)
        r = self._local("kernel", vs, vp, rho, c0, c1)
        vc, vout, st = self._gather_maps(r["vc"], r["vout"], r["status"], ncol)
        return dict(vc=vc, vout=vout, status=st, kernel=r["kernel"], columns=(c0, c1))
