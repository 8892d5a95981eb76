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

Station pairs shard the same way for fast marching: frechet_matrix gives
each worker a contiguous block of pairs (allocate_tasks over pairs,
SurfaceWave.cpp:583-600), each writes its own row file and the files are
merged in rank order (merge_csr_files); the traveltimes of all pairs are
all-gathered.  Every rank needs the whole vc/vout maps for that, which the
column gather provides.

The per-block computations are injected (`compute`, `march`), so the host
logic -- block bounds, padding, gather and reassembly -- is tested on CPU
with gloo ranks; on GPUs the defaults compute with the rank's Engine and
FMST.  The *_device methods keep everything on the GPU: the block is
computed from the device-resident model and the maps are gathered by one
NCCL all-gather into device tensors.
"""
import numpy as np

from .engine import torch_stream


def column_block(ncol, world, rank):
    """[start, end) of rank's columns, the reference's allocate_tasks split."""
    sub = ncol // world
    extra = ncol - world * sub
    if rank < extra:
        start = rank * (sub + 1)
        return start, start + sub + 1
    start = extra + rank * sub
    return start, start + sub


def pair_subset(pairs, p0, p1):
    """Pairs [p0, p1) with their receivers, receiver offsets from 0."""
    rp = np.asarray(pairs["rcv_ptr"], np.int64)
    r0, r1 = int(rp[p0]), int(rp[p1])
    out = {k: np.asarray(pairs[k])[p0:p1] for k in ("slot", "srcx", "srcz", "group")}
    out["rcv_ptr"] = rp[p0:p1 + 1] - r0
    out["rcx"] = np.asarray(pairs["rcx"])[r0:r1]
    out["rcz"] = np.asarray(pairs["rcz"])[r0:r1]
    return out


class ShardedSurfTime:
    """get_2d_map / get_1d_kernel of one model split by columns, and the
    station pairs' fast marching split by pairs, across the ranks of a
    torch.distributed process group."""

    def __init__(self, rank, world, group=None, engine=None, compute=None, fmst=None, march=None):
        self.rank, self.world, self.group = rank, world, group
        self.engine = engine
        self.compute = compute
        self.fmst = fmst
        self.march = march

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

    # -- device-resident path: maps gathered by the collective on the GPU ----
    def _local_device(self, path, vs, vp, rho, c0, c1, stream=None):
        """This rank's column block [c0, c1) of a device-resident model (nz,
        ncol): vc, vout, status (kmax, c1-c0) and, for path "kernel", the
        kernel block (kmax, nz, c1-c0), as tensors on vs's device."""
        import torch
        blk = lambda a: None if a is None else a[:, c0:c1].contiguous()
        vs_b, vp_b, rho_b = blk(vs), blk(vp), blk(rho)
        if stream is None and vs.is_cuda:  # order the engine's work with torch's (the gather reads its outputs)
            stream = torch_stream(vs.device)
        if self.compute is not None:
            np_ = lambda a: None if a is None else a.cpu().numpy()
            r = self.compute(path, np_(vs_b), np_(vp_b), np_(rho_b))
            out = {k: torch.as_tensor(r[k], device=vs.device) for k in ("vc", "vout", "status")}
            if path == "kernel":
                out["kernel"] = torch.as_tensor(r["kernel"], device=vs.device)
            return out
        nz, n = vs_b.shape
        kmax = self.engine.kmax
        dev = vs.device
        vc = torch.empty((kmax, n), dtype=torch.float64, device=dev)
        vout = torch.empty_like(vc)
        st = torch.empty((kmax, n), dtype=torch.int32, device=dev)
        if path == "kernel":
            ker = torch.empty((kmax, nz, n), dtype=torch.float64, device=dev)
            self.engine.get_1d_kernel_device(n, 1, nz, vs_b, vp_b, rho_b, vc, vout, ker, st, stream=stream)
            return dict(vc=vc, vout=vout, status=st, kernel=ker)
        self.engine.get_2d_map_device(n, 1, nz, vs_b, vp_b, rho_b, vc, vout, st, stream=stream)
        return dict(vc=vc, vout=vout, status=st)

    def _gather_maps_device(self, vc, vout, st, ncol):
        """All-gather the (kmax, block) maps of every rank into (kmax, ncol)
        tensors on this rank's device: one collective over a (3, kmax, bmax)
        FP64 pack per rank (status as exact small integers), no host copy."""
        import torch
        import torch.distributed as dist
        kmax, n = vc.shape
        if self.world == 1 and not dist.is_initialized():  # one process, nothing to exchange
            return vc, vout, st
        bmax = -(-ncol // self.world)  # the largest block (allocate_tasks)
        pack = torch.zeros((3, kmax, bmax), dtype=torch.float64, device=vc.device)
        pack[0, :, :n] = vc
        pack[1, :, :n] = vout
        pack[2, :, :n] = st.to(torch.float64)
        if dist.get_backend(self.group) == "nccl":
            out = torch.empty((self.world, 3, kmax, bmax), dtype=torch.float64, device=vc.device)
            dist.all_gather_into_tensor(out, pack, group=self.group)
            parts = list(out.unbind(0))
        else:
            parts = [torch.empty_like(pack) for _ in range(self.world)]
            dist.all_gather(parts, pack, group=self.group)
        full = torch.empty((3, kmax, ncol), dtype=torch.float64, device=vc.device)
        for r, o in enumerate(parts):
            c0, c1 = column_block(ncol, self.world, r)
            full[:, :, c0:c1] = o[:, :, :c1 - c0]
        return full[0], full[1], full[2].to(torch.int32)

    def get_1d_kernel_device(self, vs, vp=None, rho=None, stream=None):
        """get_1d_kernel of a device-resident model (nz, ncol) tensors, each
        rank computing its column block: the full vc/vout/status maps on
        every rank's device, the kernel block of this rank's columns."""
        ncol = vs.shape[1]
        c0, c1 = column_block(ncol, self.world, self.rank)
        r = self._local_device("kernel", vs, vp, rho, c0, c1, stream)
        vc, vout, st = self._gather_maps_device(r["vc"], r["vout"], r["status"], ncol)
        return dict(vc=vc, vout=vout, status=st, kernel=r["kernel"], columns=(c0, c1))

    def get_2d_map_device(self, vs, vp=None, rho=None, stream=None):
        """get_2d_map of a device-resident model: full maps on every rank."""
        ncol = vs.shape[1]
        c0, c1 = column_block(ncol, self.world, self.rank)
        r = self._local_device("map", vs, vp, rho, c0, c1, stream)
        vc, vout, st = self._gather_maps_device(r["vc"], r["vout"], r["status"], ncol)
        return dict(vc=vc, vout=vout, status=st)

    # -- fast marching over a block of the station pairs ---------------------
    def _march(self, sub, vc, vout, want_fdm):
        if self.march is not None:
            return self.march(sub, vc, vout, want_fdm)
        import torch
        dev = torch.device("cuda", torch.cuda.current_device())
        r = self.fmst.pairs(sub, torch.as_tensor(vc, device=dev), torch.as_tensor(vout, device=dev),
                            want_fdm=want_fdm)
        return (r["ttime"].cpu().numpy(), None if r["fdm"] is None else r["fdm"].cpu().numpy())

    def _gather_times(self, tt, nrcv, rp):
        """All-gather each rank's receiver times into the full data vector."""
        import torch
        import torch.distributed as dist
        npairs = len(rp) - 1
        rmax = max(int(rp[column_block(npairs, self.world, r)[1]] - rp[column_block(npairs, self.world, r)[0]])
                   for r in range(self.world))
        pad = np.full(rmax, np.nan, np.float32)
        pad[:len(tt)] = tt
        t = torch.from_numpy(pad)
        if dist.get_backend(self.group) == "nccl":
            t = t.cuda()
        outs = [torch.empty_like(t) for _ in range(self.world)]
        dist.all_gather(outs, t, group=self.group)
        data = np.empty(nrcv, np.float32)
        for r, o in enumerate(outs):
            p0, p1 = column_block(npairs, self.world, r)
            a, b = int(rp[p0]), int(rp[p1])
            data[a:b] = o.cpu().numpy()[:b - a]
        return data

    def travel_time(self, pairs, vc, vout):
        """SurfaceWave.cpp:510-541 over this rank's block of pairs; the full
        data vector on every rank."""
        rp = np.asarray(pairs["rcv_ptr"], np.int64)
        p0, p1 = column_block(len(rp) - 1, self.world, self.rank)
        tt, _ = self._march(pair_subset(pairs, p0, p1), vc, vout, False)
        return self._gather_times(tt, int(rp[-1]), rp)

    def frechet_pairs(self, pairs, vc, vout):
        """This rank's pairs [p0, p1): receiver times and ray-path weights
        (rows of frechet_matrix before the depth kernel multiplies them), and
        the full data vector on every rank."""
        rp = np.asarray(pairs["rcv_ptr"], np.int64)
        p0, p1 = column_block(len(rp) - 1, self.world, self.rank)
        tt, fdm = self._march(pair_subset(pairs, p0, p1), vc, vout, True)
        return dict(data=self._gather_times(tt, int(rp[-1]), rp), fdm=fdm, pairs=(p0, p1),
                    receivers=(int(rp[p0]), int(rp[p1])))

