"""Seeded synthetic layered-earth models for the benchmark configurations.

There is no public dataset for this path: every configuration is generated
here from a fixed seed, with the shapes, depth grids, velocity ranges and
period sets of the benchmark configurations.  The same generator feeds the
GPU runs and the CPU oracle.

Layout of a case (all numpy, matching the reference's Eigen column-major
containers): ``vs`` is (nz, ncol) float32 C-order, i.e. an Eigen
``fmat3(nx, ny, nz)`` in memory with column index n = ix + nx*iy; ``vp``/``rho``
are either None (vp/rho from the Brocher relations, as
SurfTime::get_1d_kernel does, SurfaceWave.cpp:476-480) or explicit arrays of
the same shape; each period table ``tables[w]`` (w = Rc, Rg, Lc, Lg) is an
(ntmax, nmode) float64 array with -1 padding like SurfTime::tRc, or None.
"""
import numpy as np

WAVES = ("Rc", "Rg", "Lc", "Lg")


def brocher(vs):
    """Brocher (2005) vp(vs), rho(vp) in float32 (empirical.cpp:9-18)."""
    v = vs.astype(np.float64)
    vp = (0.9409 + 2.0947 * v - 0.8206 * v ** 2 + 0.2683 * v ** 3 - 0.0251 * v ** 4).astype(np.float32)
    p = vp.astype(np.float64)
    rho = (1.6612 * p - 0.4721 * p ** 2 + 0.0671 * p ** 3 - 0.0043 * p ** 4 + 0.000106 * p ** 5).astype(np.float32)
    return vp, rho


def _corr_field(rng, nx, ny, nz, lh, lv):
    from scipy.ndimage import gaussian_filter
    w = rng.standard_normal((nz, ny, nx))
    f = gaussian_filter(w, sigma=(lv, lh, lh), mode="wrap")
    f /= max(np.abs(f).max(), 1e-30)
    return f


def _table(periods, nmode):
    periods = np.asarray(periods, np.float64)
    return np.ascontiguousarray(np.repeat(periods[:, None], nmode, axis=1))


def make_case(nx, ny, depth, vs_top, vs_bot, amp, periods, waves, nmode, seed, lvz_frac=0.0, water_frac=0.0,
              explicit_vp=None, lh=4.0, lv=3.0):
    rng = np.random.default_rng(seed)
    depth = np.asarray(depth, np.float32)
    nz = len(depth)
    frac = (depth - depth[0]) / (depth[-1] - depth[0])
    base = vs_top + (vs_bot - vs_top) * frac
    field = _corr_field(rng, nx, ny, nz, lh, lv)
    vs = (base[:, None, None] * (1.0 + amp * field)).astype(np.float32)
    ncol = nx * ny
    vs = vs.reshape(nz, ncol)
    if lvz_frac > 0:
        cols = rng.random(ncol) < lvz_frac
        zmask = (depth >= 15.0) & (depth <= 25.0)
        vs[np.ix_(zmask, cols)] *= np.float32(0.9)
    vp = rho = None
    if explicit_vp is not None or water_frac > 0:
        if explicit_vp is not None:
            vp = (np.float32(explicit_vp) * vs).astype(np.float32)
            _, rho = brocher(vs)
            rho = brocher_rho(vp)
        else:
            vp, rho = brocher(vs)
    if water_frac > 0:
        wcols = np.nonzero(rng.random(ncol) < water_frac)[0]
        nw = rng.integers(1, 4, size=len(wcols))
        for c, k in zip(wcols, nw):
            vs[:k, c] = 0.0
            vp[:k, c] = 1.5
            rho[:k, c] = 1.03
    tables = [None] * 4
    for w in waves:
        tables[WAVES.index(w)] = _table(periods, nmode)
    return dict(nx=nx, ny=ny, nz=nz, depth=depth, vs=np.ascontiguousarray(vs),
                vp=None if vp is None else np.ascontiguousarray(vp),
                rho=None if rho is None else np.ascontiguousarray(rho), tables=tables)


def brocher_rho(vp):
    p = vp.astype(np.float64)
    return (1.6612 * p - 0.4721 * p ** 2 + 0.0671 * p ** 3 - 0.0043 * p ** 4 + 0.000106 * p ** 5).astype(np.float32)


def depth_grid(nz_fine, dz_fine, nz_total, dz_coarse):
    fine = np.arange(nz_fine) * dz_fine
    coarse = fine[-1] + dz_coarse * np.arange(1, nz_total - nz_fine + 1)
    return np.concatenate([fine, coarse]).astype(np.float32)


def make_config(name, seed=2024, nx=None, ny=None):
    """Named configurations.

    tiny  : 4x3 columns, nz=12 (2 km), Rc/Rg/Lc/Lg mode 0, 6 periods -- unit tests
    small : 16x16, nz=20 nodes every 2 km (0..38 km), vs 2.8->4.6 +-5 %
            (correlation 4 columns / 3 nodes), vp = 1.732 vs, rho = Brocher(vp),
            25 log-spaced periods 2-40 s, Rayleigh mode 0 phase + group
    production : 128x128, nz=48 (1 km to 20 km, then 2.5 km), vs 2.5->4.7
            +-8 %, LVZ -10 % at 15-25 km in 20 % of columns, 1-3 fluid nodes
            (vp 1.5, vs 0, rho 1.03) in 10 % of columns, 40 log-spaced
            periods 1-60 s, Rayleigh and Love, modes 0-1, phase and group
    large : 256x256, nz=64 (1 km to 20 km, then 2.5 km), vs 2.5->4.7 +-8 %,
            LVZ in 20 % of columns, 60 log-spaced periods 1-80 s, Rayleigh and
            Love mode 0 phase
    mixed : the large grid with Rc, Rg, Lc and Lg mode 0 (phase and group),
            the mixed-precision accuracy case
    """
    if name == "tiny":
        depth = np.arange(12, dtype=np.float32) * 2.0
        return make_case(nx or 4, ny or 3, depth, 2.6, 4.4, 0.05, np.geomspace(3.0, 30.0, 6), WAVES, 1, seed)
    if name == "small":
        depth = np.arange(20, dtype=np.float32) * 2.0
        return make_case(nx or 16, ny or 16, depth, 2.8, 4.6, 0.05, np.geomspace(2.0, 40.0, 25), ("Rc", "Rg"), 1,
                         seed, explicit_vp=1.732)
    if name == "production":
        depth = depth_grid(21, 1.0, 48, 2.5)
        return make_case(nx or 128, ny or 128, depth, 2.5, 4.7, 0.08, np.geomspace(1.0, 60.0, 40), WAVES, 2, seed,
                         lvz_frac=0.2, water_frac=0.1)
    if name == "mixed":  # the large grid with phase and group of Rayleigh and Love mode 0
        depth = depth_grid(21, 1.0, 64, 2.5)
        return make_case(nx or 256, ny or 256, depth, 2.5, 4.7, 0.08, np.geomspace(1.0, 80.0, 60), WAVES, 1,
                         seed, lvz_frac=0.2)
    if name == "large":
        depth = depth_grid(21, 1.0, 64, 2.5)
        return make_case(nx or 256, ny or 256, depth, 2.5, 4.7, 0.08, np.geomspace(1.0, 80.0, 60), ("Rc", "Lc"), 1,
                         seed, lvz_frac=0.2)
    raise ValueError(name)


def kmax_of(tables):
    k = 0
    for t in tables:
        if t is None:
            continue
        for m in range(t.shape[1]):
            col = t[:, m]
            n = 0
            while n < len(col) and col[n] != -1:
                n += 1
            k += n
    return k


def subset_columns(case, cols):
    """A case restricted to the given column indices (nx = len(cols), ny = 1)."""
    cols = np.asarray(cols)
    out = dict(case)
    out["nx"], out["ny"] = len(cols), 1
    out["vs"] = np.ascontiguousarray(case["vs"][:, cols])
    out["vp"] = None if case["vp"] is None else np.ascontiguousarray(case["vp"][:, cols])
    out["rho"] = None if case["rho"] is None else np.ascontiguousarray(case["rho"][:, cols])
    return out


def make_uneven_batch(nmodels=48, seed=5150, small=False, max_kernel_bytes=2 << 30):
    """Independent models of one inversion iteration with uneven shapes:
    grids 32x32..200x200 columns, 24..80 nodes (1 km to 20 km, then 2.5 km),
    15..60 log-spaced periods inside 1..100 s, one or two of Rc/Rg/Lc/Lg,
    modes 0..2; LVZ in 20 % and fluid nodes in 10 % of the columns of each
    model.  small=True shrinks grids (8..20) and nodes (24..40) for tests.
    The period count is lowered where a model's kernel would exceed
    max_kernel_bytes."""
    rng = np.random.default_rng(seed)
    cases = []
    for i in range(nmodels):
        lo, hi = (8, 21) if small else (32, 201)
        nx, ny = (int(v) for v in rng.integers(lo, hi, 2))
        nz = int(rng.integers(24, 41 if small else 81))
        depth = depth_grid(21, 1.0, nz, 2.5)
        nt = int(rng.integers(15, 61))
        tmin = float(np.exp(rng.uniform(np.log(1.0), np.log(5.0))))
        tmax = float(np.exp(rng.uniform(np.log(30.0), np.log(100.0))))
        k = int(rng.integers(1, 3))
        waves = tuple(sorted((str(w) for w in rng.choice(WAVES, size=k, replace=False)), key=WAVES.index))
        nmode = int(rng.integers(1, 4))
        per_slot = nx * ny * nz * 8
        nt = max(15, min(nt, max_kernel_bytes // max(1, per_slot * k * nmode)))
        periods = np.geomspace(tmin, tmax, nt)
        c = make_case(nx, ny, depth, 2.5, 4.7, 0.08, periods, waves, nmode, seed * 1000 + i, lvz_frac=0.2,
                      water_frac=0.1)
        c["waves"], c["nmode"] = waves, nmode
        cases.append(c)
    return cases


def make_survey(name="example", seed=7, nx=None, ny=None, nstation=None, nperiod=None, waves=("Rc", "Rg")):
    """Seeded station pairs on a model grid, for the fast-marching path.

    The reference's own data set cannot ship, so its shapes stand in:
    example : 33 x 36 grid at 0.3 deg from (35.3 N, 99.7 E), 41 nodes every
              2 km, 19 periods 4-40 s, Rayleigh phase and group, 80 stations
              inside the grid; every station is a source for each (wave,
              period) and records at ~18 % of the others (about 14
              receivers per pair, ~3000 pairs, ~44 000 traveltimes)
    production : the 128 x 128 production grid at 0.1 deg, 40 periods, 150
              stations, the same fraction of receivers.
    Returns dict(case=..., grid=(nx, ny, lat0, lon0, dlat, dlon), tables,
    kmax_per_mode, pairs) with pairs as SurfTime holds them (colatitude and
    longitude in radians, float32)."""
    rng = np.random.default_rng(seed)
    if name == "example":
        nx, ny = nx or 33, ny or 36
        lat0, lon0, d = 35.3, 99.7, 0.3
        depth = (np.arange(41) * 2.0).astype(np.float32)
        periods = np.arange(4.0, 41.0, 2.0)[: nperiod or 19]
        nstation = nstation or 80
        case = make_case(nx, ny, depth, 2.5, 4.6, 0.06, periods, waves, 1, seed)
    elif name == "production":
        nx, ny = nx or 128, ny or 128
        lat0, lon0, d = 40.0, 100.0, 0.1
        base = make_config("production", seed=seed, nx=nx, ny=ny)
        periods = np.geomspace(1.0, 60.0, 40)[: nperiod or 40]
        nstation = nstation or 150
        case = make_case(nx, ny, base["depth"], 2.5, 4.7, 0.08, periods, waves, 1, seed, lvz_frac=0.2)
    else:
        raise ValueError(name)
    # stations strictly inside the propagation grid (one model cell from each side)
    lat = lat0 - d * rng.uniform(1.5, nx - 2.5, nstation)
    lon = lon0 + d * rng.uniform(1.5, ny - 2.5, nstation)
    d2r = np.float32(np.pi / 180.0)
    colat = ((np.float32(90.0) - lat.astype(np.float32)) * d2r).astype(np.float32)
    lonr = (lon.astype(np.float32) * d2r).astype(np.float32)
    wt, modes, pidx, srcx, srcz, rptr, rcx, rcz = [], [], [], [], [], [0], [], []
    for w in waves:
        for ip in range(len(periods)):
            for s in range(nstation):
                others = np.flatnonzero(rng.random(nstation) < 0.18)
                others = others[others != s]
                if len(others) == 0:
                    continue
                wt.append(w)
                modes.append(0)
                pidx.append(ip)
                srcx.append(colat[s])
                srcz.append(lonr[s])
                rcx.extend(colat[others])
                rcz.extend(lonr[others])
                rptr.append(rptr[-1] + len(others))
    pairs = dict(wavetype=wt, mode=np.array(modes, np.int32), period_idx=np.array(pidx, np.int32),
                 srcx=np.array(srcx, np.float32), srcz=np.array(srcz, np.float32),
                 rcv_ptr=np.array(rptr, np.int64), rcx=np.array(rcx, np.float32), rcz=np.array(rcz, np.float32))
    pairs["counter"] = pairs["rcv_ptr"][:-1].copy()
    kmax_per_mode = [[len(periods)] if (case["tables"][i] is not None) else [] for i in range(4)]
    return dict(case=case, grid=(nx, ny, lat0, lon0, d, d), tables=case["tables"], kmax_per_mode=kmax_per_mode,
                pairs=pairs)


def survey_slots(survey):
    """(slot, group) per pair in get_period_index order."""
    off, base = {}, 0
    for w, km in zip(WAVES, survey["kmax_per_mode"]):
        for m, k in enumerate(km):
            off[(w, m)] = base
            base += k
    p = survey["pairs"]
    slot = np.array([off[(w, int(m))] + int(i) for w, m, i in zip(p["wavetype"], p["mode"], p["period_idx"])],
                    np.int32)
    group = np.array([1 if w in ("Rg", "Lg") else 0 for w in p["wavetype"]], np.int32)
    return slot, group
