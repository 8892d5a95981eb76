"""Host-side pieces of the learned proposal: committed weights and the
root-slot bookkeeping used to calibrate the anchored bracket."""
import json
import os

import numpy as np

from jdsurfg_b200 import learn


def test_committed_weights_metadata():
    with open(os.path.join(learn.WEIGHTS, "proposal.json")) as f:
        meta = json.load(f)
    assert meta["rows"]["rayleigh"] >= 1_000_000 and meta["rows"]["love"] >= 1_000_000
    assert set(meta["engine_kappa"]) == {"rayleigh", "love"}
    for name in ("rayleigh", "love"):
        p = os.path.join(learn.WEIGHTS, f"{name}.mlp")
        with open(p, "rb") as f:
            assert int.from_bytes(f.read(4), "little") == 0x4D4C5053  # checkpoint magic


def test_chain_position_segments_chains_and_modes():
    # two chains: Rayleigh modes 0-1 over 3 periods, then Love mode 0 over 2
    wave = np.array([2, 2, 2, 2, 2, 2, 1, 1])
    mode = np.array([0, 0, 0, 1, 1, 1, 0, 0])
    per = np.array([1.0, 2.0, 3.0, 1.0, 2.0, 3.0, 1.5, 4.0])
    assert learn.chain_position(wave, mode, per).tolist() == [0, 1, 2, 0, 1, 2, 0, 1]
    # a second chain of the same wave and mode starts where the period drops
    assert learn.chain_position(np.array([2, 2, 2]), np.array([0, 0, 0]), np.array([1.0, 2.0, 1.01])).tolist() == [0, 1, 0]
