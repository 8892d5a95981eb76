"""Column sharding across ranks (jdsurfg_b200/shard.py) with world_size 2 on
CPU: gloo process group, the oracle computing each rank's column block; the
all-gathered maps must equal the single-process result exactly, and each
rank keeps exactly its own kernel columns."""
import os
import socket

import numpy as np
import pytest

import oracle_lib as O
from jdsurfg_b200 import synth
from jdsurfg_b200.shard import column_block


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_column_block_matches_reference_split():
    # allocate_tasks (src/shared/parallel.cpp:3-19): first ntasks % nprocs ranks get one more
    for ncol, world in [(10, 3), (12, 4), (5, 8), (1, 2), (7, 1)]:
        blocks = [column_block(ncol, world, r) for r in range(world)]
        assert blocks[0][0] == 0 and blocks[-1][1] == ncol
        for (a0, a1), (b0, b1) in zip(blocks, blocks[1:]):
            assert a1 == b0
        sizes = [b - a for a, b in blocks]
        assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from jdsurfg_b200.shard import ShardedSurfTime
    case = synth.make_config("tiny", seed=5, nx=5, ny=3)

    def compute(path, vs, vp, rho):
        c = dict(case, vs=vs, vp=vp, rho=rho, nx=vs.shape[1], ny=1)
        f = O.get_1d_kernel if path == "kernel" else O.get_2d_map
        return f(c, nthreads=1)

    sh = ShardedSurfTime(rank, world, compute=compute)
    m = sh.get_2d_map(case["vs"], case["vp"], case["rho"])
    k = sh.get_1d_kernel(case["vs"], case["vp"], case["rho"])
    # the tensor path (device tensors on GPUs; CPU tensors over gloo here)
    import torch
    t = lambda a: None if a is None else torch.from_numpy(a)
    kd = sh.get_1d_kernel_device(t(case["vs"]), t(case["vp"]), t(case["rho"]))
    md = sh.get_2d_map_device(t(case["vs"]), t(case["vp"]), t(case["rho"]))
    np.savez(os.path.join(out_dir, f"rank{rank}.npz"), vc=m["vc"], vout=m["vout"], status=m["status"],
             kvc=k["vc"], kernel=k["kernel"], c0=k["columns"][0], c1=k["columns"][1],
             dvc=kd["vc"].numpy(), dvout=kd["vout"].numpy(), dstatus=kd["status"].numpy(),
             dkernel=kd["kernel"].numpy(), mvc=md["vc"].numpy(), mvout=md["vout"].numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_maps_equal_single_process(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    case = synth.make_config("tiny", seed=5, nx=5, ny=3)
    full_map = O.get_2d_map(case, nthreads=1)
    full_ker = O.get_1d_kernel(case, nthreads=1)
    for r in range(world):
        d = np.load(tmp_path / f"rank{r}.npz")
        assert np.array_equal(d["vc"], full_map["vc"])
        assert np.array_equal(d["vout"], full_map["vout"])
        assert np.array_equal(d["status"], full_map["status"])
        assert np.array_equal(d["kvc"], full_ker["vc"])
        c0, c1 = int(d["c0"]), int(d["c1"])
        assert (c0, c1) == column_block(15, world, r)
        assert np.array_equal(d["kernel"], full_ker["kernel"][:, :, c0:c1])
        assert np.array_equal(d["dvc"], full_ker["vc"]) and np.array_equal(d["dvout"], full_ker["vout"])
        assert np.array_equal(d["dstatus"], full_ker["status"])
        assert np.array_equal(d["dkernel"], full_ker["kernel"][:, :, c0:c1])
        assert np.array_equal(d["mvc"], full_map["vc"]) and np.array_equal(d["mvout"], full_map["vout"])


def _rank_pairs(rank, world, port, out_dir):
    """Fast marching split by station pairs: each rank marches its block
    (the oracle stands in for the device), writes its part of the row file,
    and all-gathers the data vector."""
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from jdsurfg_b200 import frechet_file
    from jdsurfg_b200.shard import ShardedSurfTime
    s, pairs = _survey()
    case = s["case"]
    ker = O.get_1d_kernel(case, nthreads=1)

    def march(sub, vc, vout, want_fdm):
        return O.fmst_pairs(s["grid"], sub, vc, vout, want_fdm=want_fdm, nthreads=1)

    sh = ShardedSurfTime(rank, world, march=march)
    tt = sh.travel_time(pairs, ker["vc"], ker["vout"])
    r = sh.frechet_pairs(pairs, ker["vc"], ker["vout"])
    nx, ny = s["grid"][:2]
    nz = len(case["depth"])
    r0, r1 = r["receivers"]
    slot = np.repeat(pairs["slot"], np.diff(pairs["rcv_ptr"]))[r0:r1].astype(np.int32)
    rows = O.frechet_rows(nx, ny, nz, ker["kernel"], slot, r["fdm"].reshape(r1 - r0, -1))
    rowptr = np.concatenate([[0], np.cumsum([len(a) for a, _ in rows])])
    idx = np.concatenate([a for a, _ in rows]) if rows else np.zeros(0, np.int32)
    val = np.concatenate([v for _, v in rows]) if rows else np.zeros(0, np.float32)
    frechet_file.write_frechet(os.path.join(out_dir, f"rows.bin.{rank}"), int(pairs["rcv_ptr"][-1]),
                               (nx - 2) * (ny - 2) * (nz - 1), np.arange(r0, r1), rowptr, idx, val)
    np.savez(os.path.join(out_dir, f"pairs{rank}.npz"), tt=tt, data=r["data"])
    dist.barrier()
    dist.destroy_process_group()


def _survey():
    s = synth.make_survey("example", nx=12, ny=13, nstation=7, nperiod=2, seed=9)
    slot, group = synth.survey_slots(s)
    p = s["pairs"]
    pairs = dict(slot=slot, srcx=p["srcx"], srcz=p["srcz"], group=group, rcv_ptr=p["rcv_ptr"], rcx=p["rcx"],
                 rcz=p["rcz"])
    return s, pairs


def test_sharded_pairs_and_row_files_equal_single_process(tmp_path):
    import torch.multiprocessing as mp
    from jdsurfg_b200 import frechet_file
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_pairs, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    s, pairs = _survey()
    case = s["case"]
    ker = O.get_1d_kernel(case, nthreads=1)
    m2 = O.get_2d_map(case, nthreads=1)
    ref_tt, _ = O.fmst_pairs(s["grid"], pairs, ker["vc"], ker["vout"], nthreads=1)
    ref_t, ref_f = O.fmst_pairs(s["grid"], pairs, ker["vc"], ker["vout"], want_fdm=True, nthreads=1)
    for r in range(world):
        d = np.load(tmp_path / f"pairs{r}.npz")
        assert np.array_equal(d["tt"], ref_tt) and np.array_equal(d["data"], ref_t)
    # the merged per-rank files equal the single-process rows, in data order
    out = str(tmp_path / "rows.bin")
    frechet_file.merge_frechet([f"{out}.{r}" for r in range(world)], out)
    m, n, got = frechet_file.read_frechet(out)
    nx, ny = s["grid"][:2]
    nz = len(case["depth"])
    slot = np.repeat(pairs["slot"], np.diff(pairs["rcv_ptr"])).astype(np.int32)
    rows = O.frechet_rows(nx, ny, nz, ker["kernel"], slot, ref_f.reshape(len(ref_t), -1))
    assert m == len(ref_t) and n == (nx - 2) * (ny - 2) * (nz - 1) and len(got) == len(rows)
    for k, ((rid, gi, gv), (ri, rv)) in enumerate(zip(got, rows)):
        assert rid == k and np.array_equal(gi, ri) and np.array_equal(gv, rv)
    assert m2["vc"].shape == ker["vc"].shape
