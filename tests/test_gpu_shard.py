"""The engine-backed column sharding (jdsurfg_b200/shard.py) on one GPU:
a one-rank NCCL process group runs ShardedSurfTime's host and device paths,
including the NCCL all-gather of the maps, and both must equal the
unsharded engine call bit for bit.  (The split over two ranks is tested on
CPU with gloo in tests/test_shard_gloo.py; this run has one GPU.)"""
import datetime
import socket

import numpy as np
import pytest

from jdsurfg_b200 import Engine, synth
from jdsurfg_b200.shard import ShardedSurfTime

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_sharded_engine_one_rank_equals_unsharded():
    import torch
    import torch.distributed as dist
    case = synth.make_config("production", seed=31, nx=24, ny=20)
    eng = Engine(device=0)
    eng.setup(case)
    ref = eng.get_1d_kernel(case["vs"], case["vp"], case["rho"], nx=case["nx"], ny=case["ny"])
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        sh = ShardedSurfTime(0, 1, engine=eng)
        h = sh.get_1d_kernel(case["vs"], case["vp"], case["rho"])
        dev = torch.device("cuda", 0)
        t = lambda a: torch.from_numpy(a).to(dev)
        d = sh.get_1d_kernel_device(t(case["vs"]), t(case["vp"]), t(case["rho"]))
        m = sh.get_2d_map_device(t(case["vs"]), t(case["vp"]), t(case["rho"]))
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
    for k in ("vc", "vout", "status", "kernel"):
        np.testing.assert_array_equal(h[k], ref[k])
        np.testing.assert_array_equal(d[k].cpu().numpy(), ref[k])
    mref = eng.get_2d_map(case["vs"], case["vp"], case["rho"], nx=case["nx"], ny=case["ny"])
    eng.close()
    for k in ("vc", "vout", "status"):
        np.testing.assert_array_equal(m[k].cpu().numpy(), mref[k])
