"""Writes the committed golden fixtures under tests/golden/.

1. swd_model.txt: the reference's own kernel-test model (test/swd/model.txt of
   JDSurfG: 41 nodes, depth/vs/vp/rho), copied verbatim as data.
2. oracle_golden.npz: outputs of the CPU oracle (reference-faithful and tight
   modes) on that model and on small seeded synthetic columns, frozen so later
   changes to the oracle are caught.

Run from the repository root with the reference checkout named by the
environment variable JDSURFG_REFERENCE (default: /root/reference):
    python tests/golden/make_fixtures.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def main():
    ref = os.environ.get("JDSURFG_REFERENCE", "/root/reference")
    src = os.path.join(ref, "test", "swd", "model.txt")
    with open(src) as f:
        txt = f.read()
    with open(os.path.join(HERE, "swd_model.txt"), "w") as f:
        f.write(txt)

    import oracle_lib as O
    from jdsurfg_b200 import synth

    z, vs, vp, rho = O.load_swd_model()
    t = 4.0 + 2.0 * np.arange(19)
    out = {}
    for refine, tag in ((0, "faithful"), (1, "tight")):
        for wt, name in enumerate(["Rc", "Rg", "Lc", "Lg"]):
            tabs = [None] * 4
            tabs[wt] = t[:, None]
            r = O.kernel1d(vs, vp, rho, z, tabs, refine=refine)
            out[f"model_{tag}_{name}_vc"] = r["vc"]
            out[f"model_{tag}_{name}_vout"] = r["vout"]
            out[f"model_{tag}_{name}_kvs"] = r["kvs"]
            out[f"model_{tag}_{name}_kvp"] = r["kvp"]
            out[f"model_{tag}_{name}_krho"] = r["krho"]
    case = synth.make_config("tiny", seed=7)
    for refine, tag in ((0, "faithful"), (1, "tight")):
        r = O.get_1d_kernel(case, refine=refine)
        out[f"tiny_{tag}_vc"] = r["vc"]
        out[f"tiny_{tag}_vout"] = r["vout"]
        out[f"tiny_{tag}_kernel"] = r["kernel"]
        out[f"tiny_{tag}_status"] = r["status"]
    np.savez_compressed(os.path.join(HERE, "oracle_golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
