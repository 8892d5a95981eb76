"""SurfTime on the GPU: the surface-wave data class of JDSurfG
(src/SWD/SurfaceWave.hpp:84-116) with every per-column and per-pair loop
replaced by batched device calls.

    read_swd_data(path)         io.cpp:29-250 (period tables, station pairs,
                                observed times from distance / velocity)
    set_model(dep, lat0, lon0, dlat, dlon)   SurfaceWave.cpp:678-686
    get_period_index(...)       SurfaceWave.cpp:14-48
    travel_time(vs)             SurfaceWave.cpp:510-541: get_2d_map, then the
                                FMST pairs (receiver times; ray times for
                                Rg/Lg)
    frechet_matrix(vs, file)    SurfaceWave.cpp:551-676: get_1d_kernel, FMST
                                pairs with ray-path weights, CSR rows on the
                                device, the reference's row file
    compute_grad(vs)            SurfaceWave.cpp:697-782: the same rows times
                                the residuals, summed on the device
    write_syn(dsyn, file)       SurfaceWave.cpp:785-815

vs is (nz, nx*ny) float32 (Eigen fmat3(nx, ny, nz) memory order).
"""
import math

import numpy as np

from . import frechet_file
from .engine import Engine
from .fmst import FMST

WAVES = ("Rc", "Rg", "Lc", "Lg")
DEG2RAD = np.float32(math.pi / 180.0)


def _floats(line):
    out = []
    for tok in line.split():
        try:
            out.append(float(tok))
        except ValueError:
            break
    return out


def read_swd_data(path):
    """Parse the reference's surface-wave data file (io.cpp:29-250).

    Returns dict(tables=[tRc, tRg, tLc, tLg] ((nt, nmode) float64, -1 padded,
    or None), kmax_per_mode=[...], pairs=dict(wavetype, mode, period_idx,
    srcx, srcz, rcv_ptr, rcx, rcz, counter), obst, dist).  Coordinates become
    colatitude/longitude in radians in float32 as the reference computes them
    ((90 - lat) * DEG2RAD, lon * DEG2RAD with DEG2RAD = float(pi/180)).  A
    period line shorter than its mode's count is padded with -1 (the
    reference's strtof would read 0 there)."""
    with open(path) as f:
        lines = f.read().splitlines()
    pos = 0
    tables, kmaxes = [], []
    for _ in range(4):
        head = _floats(lines[pos])
        pos += 1
        nmode = int(head[0]) if head else 0
        km = [int(v) for v in head[1:1 + nmode]]
        kmaxes.append(km)
        if nmode == 0:
            tables.append(None)
            continue
        nt = max(km)
        t = np.full((nt, nmode), -1.0)
        for im in range(nmode):
            vals = _floats(lines[pos])
            pos += 1
            n = min(km[im], len(vals))
            t[:n, im] = np.float32(vals[:n])  # strtof
        tables.append(t)
    wt, modes, pidx, srcx, srcz, rptr, rcx, rcz, obst, dist = [], [], [], [], [], [0], [], [], [], []
    while pos < len(lines):
        line = lines[pos]
        pos += 1
        if not line.strip() or not line.lstrip().startswith("#"):
            continue
        v = line.lstrip()[1:].split()
        lat, lon = np.float32(v[0]), np.float32(v[1])
        mode, period, wavetp, veltp = int(v[2]), int(v[3]), int(v[4]), int(v[5])
        name = {(2, 0): "Rc", (2, 1): "Rg", (1, 0): "Lc"}.get((wavetp, veltp), "Lg")
        sx = np.float32((np.float32(90.0) - lat) * DEG2RAD)
        sz = np.float32(lon * DEG2RAD)
        n = 0
        while pos < len(lines) and not lines[pos].lstrip().startswith("#"):
            vals = _floats(lines[pos])
            pos += 1
            if len(vals) < 3:
                continue
            rx = np.float32((np.float32(90.0) - np.float32(vals[0])) * DEG2RAD)
            rz = np.float32(np.float32(vals[1]) * DEG2RAD)
            rcx.append(rx)
            rcz.append(rz)
            d = _delsph(sx, sz, rx, rz)
            dist.append(d)
            obst.append(np.float32(d / np.float32(vals[2])))
            n += 1
        wt.append(name)
        modes.append(mode)
        pidx.append(period - 1)
        srcx.append(sx)
        srcz.append(sz)
        rptr.append(rptr[-1] + n)
    pairs = dict(wavetype=wt, mode=np.array(modes, np.int32), period_idx=np.array(pidx, np.int32),
                 srcx=np.array(srcx, np.float32), srcz=np.array(srcz, np.float32),
                 rcv_ptr=np.array(rptr, np.int64), rcx=np.array(rcx, np.float32), rcz=np.array(rcz, np.float32))
    pairs["counter"] = pairs["rcv_ptr"][:-1].copy()
    return dict(tables=tables, kmax_per_mode=kmaxes, pairs=pairs, obst=np.array(obst, np.float32),
                dist=np.array(dist, np.float32))


def _delsph(a, b, c, d):
    """src/shared/spherical.cpp:9-27 (double expressions stored into floats)."""
    dlat, dlon = np.float32(c - a), np.float32(d - b)
    lat1 = np.float32(math.pi * 0.5 - float(a))
    lat2 = np.float32(math.pi * 0.5 - float(c))
    s1, s2 = math.sin(float(dlat) * 0.5), math.sin(float(dlon) * 0.5)
    aa = np.float32(s1 * s1 + s2 * s2 * math.cos(float(lat1)) * math.cos(float(lat2)))
    cc = np.float32(2.0 * math.atan2(math.sqrt(float(aa)), math.sqrt(float(np.float32(1.0) - aa))))
    return np.float32(np.float32(6371.0) * cc)


def write_syn(outfile, pairs, tables, sta_dist, obst, dsyn):
    """SurfTime::write_syn (SurfaceWave.cpp:785-815): one line per datum,
    "dist obs syn evlat evlon stlat stlon period mode wavetype", the floats
    in printf's %f, coordinates back to degrees as the reference converts
    them (REAL*4 values of double expressions)."""
    rad2deg = 180.0 / math.pi
    T = {"Rc": tables[0], "Rg": tables[1], "Lc": tables[2], "Lg": tables[3]}
    with open(outfile, "w") as f:
        c = 0
        for k, w in enumerate(pairs["wavetype"]):
            elat = np.float32((math.pi * 0.5 - float(pairs["srcx"][k])) * rad2deg)
            elon = np.float32(float(pairs["srcz"][k]) * rad2deg)
            per = np.float32(T[w][pairs["period_idx"][k], pairs["mode"][k]])
            for i in range(int(pairs["rcv_ptr"][k]), int(pairs["rcv_ptr"][k + 1])):
                slat = np.float32((math.pi * 0.5 - float(pairs["rcx"][i])) * rad2deg)
                slon = np.float32(float(pairs["rcz"][i]) * rad2deg)
                f.write(f"{float(sta_dist[c]):f} {float(obst[c]):f} {float(dsyn[c]):f} ")
                f.write(f"{float(elat):f} {float(elon):f} {float(slat):f} {float(slon):f} ")
                f.write(f"{float(per):f} {int(pairs['mode'][k])} {w}\n")
                c += 1


def period_offsets(kmax_per_mode):
    """Slot offset of each (wave, mode) in get_period_index order."""
    off, base = {}, 0
    for w, km in zip(WAVES, kmax_per_mode):
        for m, k in enumerate(km):
            off[(w, m)] = base
            base += k
    return off, base


class SurfTime:
    """The reference's SurfTime on one GPU (see module docstring)."""

    def __init__(self, device=0, engine=None, proposals=True):
        self.device = device
        self.engine = engine if engine is not None else Engine(device=device)
        self._nets = None
        if proposals and engine is None:
            from . import learn
            self._nets = learn.load_proposals(self.engine)
        self.fmst = None
        # one explicit stream for the engine, fast marching and the row
        # assembly: a NULL stream would mean the engine's own stream to the
        # engine but the legacy stream to the others
        import torch
        self.stream = torch.cuda.Stream(torch.device("cuda", device))

    # -- data and model --------------------------------------------------------
    def read_swd_data(self, path):
        d = read_swd_data(path)
        self.set_data(d["tables"], d["kmax_per_mode"], d["pairs"], d["obst"], d["dist"])

    def set_data(self, tables, kmax_per_mode, pairs, obst=None, dist=None):
        self.tables, self.kmax_per_mode, self.pairs = tables, kmax_per_mode, pairs
        self.offsets, self.kmax = period_offsets(kmax_per_mode)
        nr = int(pairs["rcv_ptr"][-1])
        self.obst = np.zeros(nr, np.float32) if obst is None else np.asarray(obst, np.float32)
        self.sta_dist = np.zeros(nr, np.float32) if dist is None else np.asarray(dist, np.float32)
        self.slot = np.array([self.get_period_index(int(pi), int(m), w) for pi, m, w in
                              zip(pairs["period_idx"], pairs["mode"], pairs["wavetype"])], np.int32)
        self.group = np.array([1 if w in ("Rg", "Lg") else 0 for w in pairs["wavetype"]], np.int32)
        if hasattr(self, "depth"):
            self.engine.set_depth(self.depth)
        self.engine.set_periods(tables)
        assert self.engine.kmax == self.kmax, (self.engine.kmax, self.kmax)

    def set_model(self, dep, lat0, lon0, dlat, dlon, nx, ny):
        self.depth = np.asarray(dep, np.float32)
        self.lat0, self.lon0, self.dlat, self.dlon = float(lat0), float(lon0), float(dlat), float(dlon)
        self.nx, self.ny = nx, ny
        self.engine.set_depth(self.depth)
        if self.fmst is not None:
            self.fmst.close()
        self.fmst = FMST(nx, ny, self.lat0, self.lon0, self.dlat, self.dlon, device=self.device)

    def get_period_index(self, period_idx, mode, wavetype):
        return self.offsets[(wavetype, mode)] + period_idx

    def _pairs(self):
        p = self.pairs
        return dict(slot=self.slot, srcx=p["srcx"], srcz=p["srcz"], group=self.group, rcv_ptr=p["rcv_ptr"],
                    rcx=p["rcx"], rcz=p["rcz"])

    def _vs_device(self, vs):
        import torch
        dev = torch.device("cuda", self.device)
        vs = torch.as_tensor(np.ascontiguousarray(vs, np.float32)).to(dev, non_blocking=False)
        return vs, dev

    # -- the inversion loop's calls ------------------------------------------
    def travel_time(self, vs, return_device=False):
        """SurfaceWave.cpp:510-541 -> data (float32, one per receiver)."""
        import torch
        with torch.cuda.stream(self.stream):
            return self._travel_time(vs, return_device)

    def _travel_time(self, vs, return_device):
        import torch
        vs_d, dev = self._vs_device(vs)
        nz, ncol = vs_d.shape
        vc = torch.empty((self.kmax, ncol), dtype=torch.float64, device=dev)
        vout = torch.empty_like(vc)
        st = torch.empty((self.kmax, ncol), dtype=torch.int32, device=dev)
        sp = self.stream.cuda_stream
        self.engine.get_2d_map_device(self.nx, self.ny, nz, vs_d, None, None, vc, vout, st, stream=sp)
        r = self.fmst.pairs(self._pairs(), vc, vout, stream=sp)
        if return_device:
            return r
        return r["ttime"].cpu().numpy()

    def _rows(self, vs):
        import torch
        vs_d, dev = self._vs_device(vs)
        nz, ncol = vs_d.shape
        vc = torch.empty((self.kmax, ncol), dtype=torch.float64, device=dev)
        vout = torch.empty_like(vc)
        ker = torch.empty((self.kmax, nz, ncol), dtype=torch.float64, device=dev)
        st = torch.empty((self.kmax, ncol), dtype=torch.int32, device=dev)
        sp = self.stream.cuda_stream
        self.engine.get_1d_kernel_device(self.nx, self.ny, nz, vs_d, None, None, vc, vout, ker, st, stream=sp)
        r = self.fmst.pairs(self._pairs(), vc, vout, want_fdm=True, stream=sp)
        nrcv = r["ttime"].shape[0]
        row_slot = torch.as_tensor(np.repeat(self.slot, np.diff(self.pairs["rcv_ptr"]))).to(dev)
        rowptr = torch.empty(nrcv + 1, dtype=torch.int64, device=dev)
        nnz = self.engine.frechet_csr_device(self.nx, self.ny, nz, self.kmax, ker, row_slot, r["fdm"], rowptr, None,
                                             None, stream=sp)
        idx = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
        val = torch.empty(max(nnz, 1), dtype=torch.float32, device=dev)
        self.engine.frechet_csr_device(self.nx, self.ny, nz, self.kmax, ker, row_slot, r["fdm"], rowptr, idx, val,
                                       stream=sp)
        del ker
        n = (self.nx - 2) * (self.ny - 2) * (nz - 1)
        return r, rowptr, idx[:nnz], val[:nnz], n

    def frechet_matrix(self, vs, outfile=None, return_device=False):
        """SurfaceWave.cpp:551-676 -> (data, nonzeros); with outfile, writes the
        reference's row file (header m, n; rows in data order)."""
        import torch
        with torch.cuda.stream(self.stream):
            r, rowptr, idx, val, n = self._rows(vs)
            self.stream.synchronize()
        data = r["ttime"].cpu().numpy()
        nnz = int(idx.shape[0])
        if outfile is not None:  # the record stream is built on the device and written in one piece
            frechet_file.write_frechet_device(outfile, len(data), n, rowptr, idx, val, row_id0=0,
                                              stream=self.stream.cuda_stream)
        if return_device:
            return data, nnz, dict(rowptr=rowptr, indices=idx, values=val, n=n, fmst=r)
        return data, nnz

    def compute_grad(self, vs):
        """SurfaceWave.cpp:697-782 -> (data, grad): grad = sum over rows of
        row * (t - obs), times vs at the interior nodes (FP64 sums on the
        device, returned as float32)."""
        import torch
        from .lsmr import DeviceCSR
        with torch.cuda.stream(self.stream):
            r, rowptr, idx, val, n = self._rows(vs)
            dev = rowptr.device
            data = r["ttime"]
            res = (data.double() - torch.as_tensor(self.obst, device=dev).double())
            A = DeviceCSR(rowptr, idx, val, data.shape[0], n)
            g = torch.zeros(n, dtype=torch.float64, device=dev)
            A.aprod(2, g, res)
            self.stream.synchronize()
        nz = len(self.depth)
        vs3 = np.asarray(vs, np.float32).reshape(nz, self.ny, self.nx)[:nz - 1, 1:-1, 1:-1].reshape(-1)
        grad = g.cpu().numpy() * vs3
        return data.cpu().numpy(), grad.astype(np.float32)

    def write_syn(self, dsyn, outfile):
        """SurfaceWave.cpp:785-815 (see write_syn below)."""
        write_syn(outfile, self.pairs, self.tables, self.sta_dist, self.obst, dsyn)

    def close(self):
        if self.fmst is not None:
            self.fmst.close()
            self.fmst = None
        self.engine.close()
