"""Writes tests/golden/fmst_golden.npz: the CPU oracle's fast-marching
receiver times, ray times and ray-path weights (oracle/fmst_oracle.cpp, the
restatement of src/SWD/fmst.f90 and fmm.f90) on a small seeded survey,
frozen so later changes to the oracle are caught.  The reference has no
numeric fixtures for this path.

Run from the repository root:
    python tests/golden/make_fmst_fixtures.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def case():
    from jdsurfg_b200 import synth
    s = synth.make_survey("example", nx=14, ny=16, nstation=10, nperiod=2, seed=11)
    slot, group = synth.survey_slots(s)
    p = s["pairs"]
    pairs = dict(slot=slot, srcx=p["srcx"], srcz=p["srcz"], group=group, rcv_ptr=p["rcv_ptr"], rcx=p["rcx"],
                 rcz=p["rcz"])
    return s, pairs


def main():
    import oracle_lib as O
    s, pairs = case()
    m = O.get_2d_map(s["case"])
    tt, fdm = O.fmst_pairs(s["grid"], pairs, m["vc"], m["vout"], want_fdm=True, nthreads=1)
    np.savez_compressed(os.path.join(HERE, "fmst_golden.npz"), vc=m["vc"], vout=m["vout"], ttime=tt, fdm=fdm,
                        **{k: np.asarray(v) for k, v in pairs.items()})
    print(len(tt), "receivers")


if __name__ == "__main__":
    main()
