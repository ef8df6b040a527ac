"""The seeded synthetic inputs follow the benchmark configurations' shapes, sizes and value
distributions: the heat shell, the insert stress batches, the batched grids, the served request
stream, and (on a small domain) the Gray-Scott scene."""
import numpy as np

from openfpm_data_b200 import workloads as W


def test_heat_shell():
    ps = W.heat_shell()
    assert ps.size == (128, 128, 128) and ps.bck == [0.0]
    d2 = ((ps.coords - 64) ** 2).sum(1)
    assert d2.min() >= 20 ** 2 and d2.max() <= 32 ** 2
    # the whole shell: every lattice point with 20 <= r <= 32
    ax = np.arange(128) - 64
    dd = ax[:, None, None] ** 2 + ax[None, :, None] ** 2 + ax[None, None, :] ** 2
    assert len(ps.coords) == int(((dd >= 400) & (dd <= 1024)).sum())
    u = ps.values[0]
    assert u.dtype == np.float32 and u.min() >= 0.0 and u.max() < 1.0 and abs(float(u.mean()) - 0.5) < 0.01


def test_insert_batch():
    pts, fv, iv = W.insert_batch(0)
    n = 2_000_000
    assert pts.shape == (n, 3) and fv.shape == (n,) and iv.shape == (n,)
    assert fv.dtype == np.float32 and iv.dtype == np.int32
    assert pts.min() >= 0 and pts.max() <= 1023
    # 30 % of the points repeat an earlier draw exactly
    lin = pts[:, 0] + 1024 * (pts[:, 1] + 1024 * pts[:, 2])
    nuniq = len(np.unique(lin))
    assert n - nuniq >= int(0.3 * n) - 1
    # clustered: the spread around the nearest of the 64 fixed centres is about sigma = 24
    cen = np.random.default_rng(np.random.SeedSequence(2).spawn(1)[0]).uniform(0, 1024, size=(64, 3))
    s = pts[:20000].astype(np.float64)
    d = np.sqrt(((s[:, None, :] - cen[None, :, :]) ** 2).sum(2)).min(1)
    assert 20.0 < float(np.median(d)) / np.sqrt(2.366) < 28.0  # median of a 3-D normal radius: 1.538 sigma
    # another iteration draws other points around the same centres
    pts1, _, _ = W.insert_batch(1)
    assert not np.array_equal(pts, pts1)


def test_batch_grids():
    edges, radii, seeds = W.batch_grids()
    assert len(edges) == len(radii) == len(seeds) == 256
    assert (edges % 8 == 0).all() and edges.min() >= 32 and edges.max() <= 384
    frac = radii / edges
    assert frac.min() >= 0.25 and frac.max() <= 0.5
    # log-uniform: about half of the edges below the geometric mean of the range
    gm = np.sqrt(32 * 384)
    assert 0.4 < float((edges < gm).mean()) < 0.6


def test_request_stream():
    reqs = W.requests()
    n = len(reqs)
    assert abs(n - 120_000) < 5 * np.sqrt(120_000)  # Poisson count over 60 s at 2000 / s
    t = np.array([r.t_arrival for r in reqs])
    assert (np.diff(t) > 0).all() and t[-1] <= 60.0
    assert abs(float(np.diff(t).mean()) - 1 / 2000) < 0.05 / 2000
    kinds = np.array([r.kind == "heat" for r in reqs])
    assert 0.49 < float(kinds.mean()) < 0.51
    edges = np.array([r.edge for r in reqs])
    assert (edges % 8 == 0).all() and edges.min() >= 32 and edges.max() <= 256
    steps = np.array([r.steps for r in reqs])
    assert steps.min() >= 50 and steps.max() <= 500
    nb = np.array([len(r.radii) for r in reqs])
    assert nb.min() >= 1 and nb.max() <= 8
    r0 = reqs[0]
    assert (r0.radii >= 0.1 * r0.edge).all() and (r0.radii <= 0.3 * r0.edge).all()


def test_gray_scott_scene_small():
    ps = W.gray_scott(size=64, nballs=4, rmin=6.0, rmax=12.0)
    u, v = ps.values
    assert ps.bck == [1.0, 0.0] and u.dtype == np.float32 and v.dtype == np.float32
    # u = 1, v = 0 outside the seeded cubes; inside u = 0.5 and v = 0.25 within 1 %
    seeded = v > 0
    assert (u[~seeded] == 1.0).all() and (v[~seeded] == 0.0).all()
    assert seeded.any()
    assert np.abs(u[seeded] / 0.5 - 1).max() <= 0.0100001 and np.abs(v[seeded] / 0.25 - 1).max() <= 0.0100001
