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
    np.savez(os.path.join(out_dir, f"rank{rank}.npz"), vc=m["vc"], vout=m["vout"], status=m["status"],
             kvc=k["vc"], kernel=k["kernel"], c0=k["columns"][0], c1=k["columns"][1])
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
