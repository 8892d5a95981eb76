"""CPU checks of the fast-marching path: the oracle pinned against the
reference's own compiled code (delsph), against analytic traveltimes in a
homogeneous model and against its frozen outputs; the data-file reader and
the period-slot map of SurfTime."""
import os

import numpy as np
import pytest

import oracle_lib as O
from jdsurfg_b200 import surftime, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# the reference's example data file, read when a reference checkout is
# present (JDSURFG_REFERENCE, or oracle/Makefile's default); skipped otherwise
_REF = O.reference_dir()
EXAMPLE = os.path.join(_REF, "example", "surfdataSC.dat") if _REF else ""


def test_delsph_matches_reference_build():
    if O.ref_cxx() is None:
        pytest.skip("oracle/_ref not built (reference sources absent)")
    rng = np.random.default_rng(0)
    for _ in range(2000):
        a = rng.uniform(0.2, 2.9, 4).astype(np.float32)
        a[1::2] = rng.uniform(-3.0, 3.0, 2)
        args = [float(v) for v in a]
        assert np.float32(O.delsph(*args)) == np.float32(O.ref_delsph(*args))
        assert np.float32(surftime._delsph(*a)) == np.float32(O.ref_delsph(*args))


def _homogeneous(v=3.0):
    nx, ny, lat0, lon0, d = 14, 16, 40.0, 100.0, 0.3
    grid = (nx, ny, lat0, lon0, d, d)
    vmap = np.full((1, nx * ny), v)
    d2r = np.float32(np.pi / 180)
    rng = np.random.default_rng(3)
    srcx, srcz = np.float32((90 - 38.3) * d2r), np.float32(102.1 * d2r)
    lat = rng.uniform(40 - 3.4, 40 - 0.4, 24)
    lon = rng.uniform(100.4, 104.0, 24)
    rcx = ((90 - lat) * d2r).astype(np.float32)
    rcz = (lon * d2r).astype(np.float32)
    pairs = dict(slot=[0], srcx=[srcx], srcz=[srcz], rcv_ptr=[0, 24], rcx=rcx, rcz=rcz, group=[0])
    dist = np.array([O.delsph(float(srcx), float(srcz), float(a), float(b)) for a, b in zip(rcx, rcz)])
    return grid, vmap, pairs, dist


def test_homogeneous_model_traveltimes():
    """Fast-marching receiver times and ray times in a homogeneous 3 km/s
    model against great-circle distance / velocity: the mixed-order scheme on
    the 8x diced grid is within 0.5 %, the ray integral within 0.3 %."""
    grid, vmap, pairs, dist = _homogeneous(3.0)
    tt, _ = O.fmst_pairs(grid, pairs, vmap, vmap)
    assert np.max(np.abs(tt - dist / 3.0) / (dist / 3.0)) < 5e-3
    pairs["group"] = [1]
    tg, fdm = O.fmst_pairs(grid, pairs, vmap, vmap, want_fdm=True)
    assert np.max(np.abs(tg - dist / 3.0) / (dist / 3.0)) < 3e-3
    # ray weights are -ds/v^2 spread by B-spline weights that sum to one:
    # sum(w) * v is minus the traveltime of the traced segments (the last
    # step into the source carries no weight), within 6 %
    s = -fdm.reshape(len(tg), -1).sum(axis=1) * 3.0
    assert np.all(s > 0.94 * tg) and np.all(s <= tg * 1.0001)


def test_velocity_scaling():
    """Times scale as 1/v exactly when every velocity is scaled by a power
    of two (all REAL*4 operations then scale exactly)."""
    grid, vmap, pairs, _ = _homogeneous(3.0)
    rng = np.random.default_rng(5)
    v = vmap * (1.0 + 0.1 * rng.standard_normal(vmap.shape))
    t1, _ = O.fmst_pairs(grid, pairs, v, v)
    t2, _ = O.fmst_pairs(grid, pairs, 2.0 * v, 2.0 * v)
    assert np.array_equal(t1, 2.0 * t2)


def test_oracle_matches_golden_fixture():
    g = np.load(os.path.join(ROOT, "tests", "golden", "fmst_golden.npz"))
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_fmst_fixtures as M
    s, pairs = M.case()
    for k in pairs:
        assert np.array_equal(np.asarray(pairs[k]), g[k]), k
    tt, fdm = O.fmst_pairs(s["grid"], pairs, g["vc"], g["vout"], want_fdm=True, nthreads=1)
    assert np.array_equal(tt, g["ttime"])
    assert np.array_equal(fdm, g["fdm"])


def test_threads_do_not_change_oracle_results():
    s = synth.make_survey("example", nx=14, ny=16, nstation=12, nperiod=2, seed=2)
    slot, group = synth.survey_slots(s)
    p = s["pairs"]
    pairs = dict(slot=slot, srcx=p["srcx"], srcz=p["srcz"], group=group, rcv_ptr=p["rcv_ptr"], rcx=p["rcx"],
                 rcz=p["rcz"])
    m = O.get_2d_map(s["case"], nthreads=1)
    a = O.fmst_pairs(s["grid"], pairs, m["vc"], m["vout"], want_fdm=True, nthreads=1)
    b = O.fmst_pairs(s["grid"], pairs, m["vc"], m["vout"], want_fdm=True, nthreads=4)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def _write_data(path, tables, srcs):
    with open(path, "w") as f:
        for t in tables:
            if t is None:
                f.write("0\t\t # none\n")
                continue
            f.write(f"{t.shape[1]} " + " ".join(str(int((t[:, m] != -1).sum())) for m in range(t.shape[1])) + "\n")
            for m in range(t.shape[1]):
                f.write(" ".join(f"{x:g}" for x in t[:, m] if x != -1) + " \n")
        for (lat, lon, mode, per, wt, vt), rcv in srcs:
            f.write(f"# {lat} {lon} {mode} {per} {wt} {vt}\n")
            for a, b, v in rcv:
                f.write(f"{a} {b} {v}\n")


def test_read_swd_data_and_period_slots(tmp_path):
    tR = np.array([[4.0, 5.0], [6.0, 7.0], [8.0, -1.0]])
    tL = np.array([[10.0], [12.0]])
    tables = [tR, tR.copy(), tL, None]
    srcs = [((31.5, 102.0, 1, 2, 2, 0), [(32.0, 103.0, 3.1), (30.5, 101.5, 3.05)]),
            ((30.0, 101.0, 0, 1, 1, 0), [(31.0, 102.5, 3.4)]),
            ((30.2, 101.2, 0, 3, 2, 1), [(31.1, 102.2, 2.9), (31.4, 101.9, 2.8), (30.9, 102.6, 2.95)])]
    path = tmp_path / "surfdata.dat"
    _write_data(path, tables, srcs)
    d = surftime.read_swd_data(str(path))
    assert d["kmax_per_mode"] == [[3, 2], [3, 2], [2], []]
    assert np.array_equal(d["tables"][0], tR) and d["tables"][3] is None
    p = d["pairs"]
    assert p["wavetype"] == ["Rc", "Lc", "Rg"]
    assert list(p["rcv_ptr"]) == [0, 2, 3, 6] and list(p["period_idx"]) == [1, 0, 2]
    d2r = np.float32(np.pi / 180)
    assert p["srcx"][0] == np.float32((np.float32(90.0) - np.float32(31.5)) * d2r)
    assert p["rcz"][3] == np.float32(np.float32(102.2) * d2r)
    assert np.allclose(d["obst"], d["dist"] / np.array([3.1, 3.05, 3.4, 2.9, 2.8, 2.95], np.float32), rtol=1e-6)
    # get_period_index (SurfaceWave.cpp:14-48): Rc modes, Rg modes, Lc, Lg
    off, kmax = surftime.period_offsets(d["kmax_per_mode"])
    assert kmax == 12 and off[("Rc", 1)] == 3 and off[("Rg", 0)] == 5 and off[("Rg", 1)] == 8
    assert off[("Lc", 0)] == 10


def test_read_reference_example_file():
    """The reference's example data set parses (shapes only; read here, never
    shipped)."""
    if not os.path.exists(EXAMPLE):
        pytest.skip("reference example absent")
    d = surftime.read_swd_data(EXAMPLE)
    p = d["pairs"]
    nsrc = sum(1 for line in open(EXAMPLE) if line.lstrip().startswith("#"))
    assert len(p["srcx"]) == nsrc
    assert d["kmax_per_mode"][0] == [19] and d["kmax_per_mode"][1] == [19]
    assert d["tables"][2] is None and d["tables"][3] is None
    assert int(p["rcv_ptr"][-1]) == len(d["obst"]) > 10 * nsrc
    assert set(p["wavetype"]) <= {"Rc", "Rg"}


def test_write_syn_round_trip(tmp_path):
    """write_syn (SurfaceWave.cpp:785-815) after read_swd_data: one line per
    datum with distance, observed and synthetic times, event and station
    coordinates back in degrees, period, mode and wave type."""
    tR = np.array([[4.0], [6.0]])
    srcs = [((31.5, 102.0, 0, 2, 2, 1), [(32.0, 103.0, 3.1), (30.5, 101.5, 3.05)]),
            ((30.0, 101.0, 0, 1, 2, 0), [(31.0, 102.5, 3.4)])]
    path = tmp_path / "surfdata.dat"
    _write_data(path, [tR, tR.copy(), None, None], srcs)
    d = surftime.read_swd_data(str(path))
    dsyn = np.array([10.5, 20.25, 30.125], np.float32)
    out = tmp_path / "syn.dat"
    surftime.write_syn(str(out), d["pairs"], d["tables"], d["dist"], d["obst"], dsyn)
    lines = [l.split() for l in open(out).read().splitlines()]
    assert len(lines) == 3 and [l[-1] for l in lines] == ["Rg", "Rg", "Rc"]
    assert [float(l[2]) for l in lines] == [10.5, 20.25, 30.125]
    assert [float(l[7]) for l in lines] == [6.0, 6.0, 4.0] and [int(l[8]) for l in lines] == [0, 0, 0]
    assert abs(float(lines[0][3]) - 31.5) < 1e-4 and abs(float(lines[0][4]) - 102.0) < 1e-4
    assert abs(float(lines[1][5]) - 30.5) < 1e-4 and abs(float(lines[1][6]) - 101.5) < 1e-4
    assert np.allclose([float(l[0]) for l in lines], d["dist"], rtol=1e-6)
    assert np.allclose([float(l[1]) for l in lines], d["obst"], rtol=1e-6)
