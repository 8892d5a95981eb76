"""The root search's two layer sources give the same bits: sublayers
rebuilt from the grid nodes and the depth grid's flattening table
(swdk_config.node_layers = 1, the default) against the full layer tables
(node_layers = 0), on grids with and without fluid nodes (fluid columns use
the tables in both)."""
import numpy as np
import pytest

from jdsurfg_b200 import Engine, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["production", "large"])
def test_node_layers_bit_identical_to_tables(name):
    case = synth.make_config(name, seed=91, nx=24, ny=20)
    out = []
    for nodes in (True, False):
        eng = Engine(device=0, node_layers=nodes)
        eng.setup(case)
        out.append(eng.get_1d_kernel(case["vs"], case["vp"], case["rho"], nx=case["nx"], ny=case["ny"]))
        eng.close()
    for k in ("vc", "vout", "status", "kernel"):
        np.testing.assert_array_equal(out[0][k], out[1][k], err_msg=k)
