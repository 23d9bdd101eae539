"""The rain-squall model on the host (css_b200.rain, entropy_rain.f90) and
its coupling to the device builder and the open top.

CPU: the draws follow Random_Exponential (truncated to (0.3, 4)) and
Place_Cell; Temporal_Structure's two forms; Update_Rain_Squalls ages,
advects (with the periodic phi wrap), kills squalls that leave the theta
range and replaces dead ones with fresh draws starting now.  GPU: a run
with the rain model updating every ufreq/10 steps against the oracle driven
by the same squall lists (five updates), at the FP64 step bar.  The
downflow lanes (Build_Downflow_Lanes): the device field against the
oracle's, alone and with squalls added, and a run with lanes and squalls
against the oracle."""
import math

import numpy as np
import pytest

from css_b200 import problem, rain
from oracle import oracle as O


def setup(seed=4, n=16):
    p, prof, v0, dt, _ = problem.build((48, 48, 64), decomp=(2, 2, 4))
    p.top_inout, p.do_entropy_rain, p.delta_s, p.ufreq = 1, 1, 0.01, 20
    r = rain.RainSqualls(p, prof, nsqualls=n, meandur=20 * dt, meansize=0.05, rhotopin=0.1, stopin=-1e-3,
                         utopin=-0.02, seed=seed)
    return p, prof, v0, dt, r


def test_draws_follow_the_reference_distributions():
    p, prof, v0, dt, r = setup()
    x = r.random_exponential(20000)
    assert x.min() > 0.3 and x.max() < 4.0
    a, b = 0.3, 4.0
    mean = ((a + 1) * math.exp(-a) - (b + 1) * math.exp(-b)) / (math.exp(-a) - math.exp(-b))
    assert abs(x.mean() - mean) < 0.02
    th, ph = np.array([r.place_cell() for _ in range(4000)]).T
    assert th.min() >= p.th1 and th.max() <= p.th2 and ph.min() >= p.phi1 and ph.max() <= p.phi2
    assert abs(th.mean() - 0.5 * (p.th1 + p.th2)) < 0.05 * (p.th2 - p.th1)
    par = r.generate(50)
    k = par[:, rain.DUR] / r.meandur
    for col, mean_ in ((rain.SIZE, r.meansize), (rain.VEL, r.meanvel), (rain.DELS, r.meands)):
        assert np.allclose(par[:, col], mean_ * k)  # rainstats 1: one draw scales every property


def test_temporal_structure():
    p, prof, v0, dt, r = setup()
    r.start[0], r.par[0, rain.DUR], r.sigma_t[0] = 1.0, 10.0, 2.0
    r.temporal_structure(0, 2.0)
    assert r.scaling[0] == pytest.approx(math.sin(0.5 * math.pi * 0.5) ** 2)
    r.temporal_structure(0, 5.0)
    assert r.scaling[0] == 1.0
    r.temporal_structure(0, 10.0)  # t - t0 >= dur - sigma: the written form, sin(pi/2 (dur - t - t0)/sigma)^2
    assert r.scaling[0] == pytest.approx(math.sin(0.5 * math.pi * (10.0 - 10.0 - 1.0) / 2.0) ** 2)
    r.tstruct = 1
    r.temporal_structure(0, 5.0)
    assert r.scaling[0] == 1.0
    r.temporal_structure(0, 11.5)
    assert r.scaling[0] == 0.0


def test_update_advects_wraps_kills_and_replaces():
    p, prof, v0, dt, r = setup(n=4)
    t = 5.0
    W, V = 0.3, 2.0
    w_top, v_top = np.full((p.nphi, p.nth), W), np.full((p.nphi, p.nth), V)
    r.start[:] = t - 1.0
    r.par[:, rain.DUR] = 100.0
    r.par[0, rain.THETA], r.par[0, rain.PHI] = 1.5, 0.5
    r.par[1, rain.THETA], r.par[1, rain.PHI] = 1.5, p.phi2 - 1e-3  # wraps across phi2
    r.par[2, rain.THETA] = p.th2 - 1e-4                             # leaves the theta range
    r.start[3], r.par[3, rain.DUR] = 0.0, 1.0                      # dead: replaced untouched
    old3 = r.par[3].copy()
    for k in range(4):
        r.find_position(k)
    built = r.update(t, 0.01, w_top, v_top)
    assert built[0, 0] == pytest.approx(1.5 + 0.01 * W / p.r2) and built[0, 1] == pytest.approx(0.5 + 0.01 * V / p.r2)
    want = p.phi1 + (p.phi2 - 1e-3 + 0.01 * V / p.r2 - p.phi2)
    assert built[1, 1] == pytest.approx(want)
    assert np.array_equal(built[3, :3], old3[[rain.THETA, rain.PHI, rain.SIZE]])
    for k in (2, 3):  # replaced after the build, starting now with zero scaling
        assert r.start[k] == t and r.scaling[k] == 0.0
    assert r.start[0] == t - 1.0 and r.start[1] == t - 1.0
    assert r.loct[0] == max(min(math.floor((r.par[0, rain.THETA] - p.th1) / r.dth) + 1, p.nth), 1)


@pytest.mark.gpu
def test_rain_run_parity(gpu_available):
    from css_b200.context import Simulation
    p, prof, v0, dt, r = setup()
    rng = np.random.default_rng(2)
    v = v0.copy()
    v[1:4] = 1e-2 * rng.standard_normal(v[1:4].shape)
    sim, orc = Simulation(p, prof), O.Oracle(p, prof)
    dt = min(dt, list(orc.step_size(v, 0.4).values())[0])
    sim.upload(v)
    for o in (sim, orc):
        o.set_clock(0, 0.0, dt)
    every = p.ufreq // 10
    o_state = v
    for step in range(1, 11):
        sim.step_rk4(dt, 1)
        o_state = orc.step(o_state, dt, 1)
        if step % every == 0:
            _, t_end = orc.clock()
            built = r.update(t_end - dt, dt, o_state[1, -1], o_state[2, -1])
            sim.build_squalls(built)
            orc.build_squalls(built)
            for a, b in zip(sim.rain_fields(), orc.rain_fields()):
                assert np.abs(a - b).max() <= 1e-13 * max(np.abs(b).max(), 1e-300)
    assert np.abs(orc.rain_fields()[0]).max() > 0.0
    g = sim.download()
    errs = [float(np.abs(g[i] - o_state[i]).max() / np.abs(o_state[i]).max()) for i in range(5)]
    assert max(errs) < 1e-10, errs


@pytest.mark.gpu
def test_advance_drives_the_device(gpu_available):
    from css_b200.context import Simulation
    p, prof, v0, dt, r = setup(seed=8)
    sim = Simulation(p, prof)
    sim.upload(v0)
    sim.set_clock(0, 0.0, dt)
    rain.advance(sim, r, dt, 6, p.ufreq)
    assert sim.clock()[0] == 6
    dvel, dent = sim.rain_fields()
    assert np.isfinite(sim.download()).all()
    assert np.abs(dvel).max() > 0.0 and np.abs(dent).max() > 0.0
    with pytest.raises(ValueError):
        rain.advance(sim, r, dt, 1, 5)


def lane_cells(p, n, seed, lo=0.2, hi=1.0):
    rng = np.random.default_rng(seed)
    return np.stack([rng.uniform(p.phi1, p.phi2, n), rng.uniform(p.th1, p.th2, n), rng.uniform(lo, hi, n)], axis=1)


@pytest.mark.gpu
@pytest.mark.parametrize("scale", [1.0, 1e-4])
def test_lanes_match_oracle(gpu_available, scale):
    """css_build_lanes against orc_build_lanes (1e-12 of the largest value):
    with full scalings the lane field's maximum exceeds 1 and is normalised
    away, with small ones it is kept (max(x, 1)).  Squalls added on top
    match the oracle's too."""
    from css_b200.context import Simulation
    p, prof, v0, dt, r = setup()
    sim, orc = Simulation(p, prof), O.Oracle(p, prof)
    cells = lane_cells(p, 9, 7)
    cells[:, 2] *= scale
    for o in (sim, orc):
        o.build_lanes(cells, 0.05, -0.02, -1e-3)
    got, want = sim.rain_fields(), orc.rain_fields()
    for a, b in zip(got, want):
        assert np.abs(b).max() > 0.0
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
    if scale == 1.0:
        assert np.abs(want[0]).max() == pytest.approx(0.02, rel=1e-12)  # normalised: meanvel at the peak
    r.scaling[:] = 0.5
    built = r.squalls()
    sim.add_squalls(built)
    orc.add_squalls(built)
    for a, b in zip(sim.rain_fields(), orc.rain_fields()):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def top_mean(p, v):
    """theta profiles of u_theta, u_phi over phi and the top block's radii."""
    size_top = p.nr // p.nnr
    return (v[1, p.nr - size_top:].sum(axis=(0, 1)) / (size_top * p.nphi),
            v[2, p.nr - size_top:].sum(axis=(0, 1)) / (size_top * p.nphi))


@pytest.mark.gpu
def test_rain_run_with_lanes_parity(gpu_available):
    """Ten steps with the rain model updating every ufreq/10 steps, lanes
    first and the squalls added, against the oracle driven by the same cell
    and squall lists, at the FP64 step bar."""
    from css_b200.context import Simulation
    p, prof, v0, dt, r = setup(seed=6)
    cc = rain.ConvectionCells(p, 8, meansize=0.05, stopin=-1e-3, utopin=-0.02, seed=9)
    rng = np.random.default_rng(5)
    v = v0.copy()
    v[1:4] = 1e-2 * rng.standard_normal(v[1:4].shape)
    sim, orc = Simulation(p, prof), O.Oracle(p, prof)
    dt = min(dt, list(orc.step_size(v, 0.4).values())[0])
    sim.upload(v)
    for o in (sim, orc):
        o.set_clock(0, 0.0, dt)
    every = p.ufreq // 10
    o_state = v
    for step in range(1, 11):
        sim.step_rk4(dt, 1)
        o_state = orc.step(o_state, dt, 1)
        if step % every == 0:
            _, t_end = orc.clock()
            cells = cc.update(t_end - dt, dt, *top_mean(p, o_state))
            cells[:, 2] = 0.3 + 0.7 * cells[:, 2]  # lanes that show in a short run
            built = r.update(t_end - dt, dt, o_state[1, -1], o_state[2, -1])
            for o in (sim, orc):
                o.build_lanes(cells, cc.meansize, cc.meanvel, cc.meands)
                o.add_squalls(built)
            for a, b in zip(sim.rain_fields(), orc.rain_fields()):
                assert np.abs(a - b).max() <= 1e-12 * max(np.abs(b).max(), 1e-300)
    g = sim.download()
    errs = [float(np.abs(g[i] - o_state[i]).max() / np.abs(o_state[i]).max()) for i in range(5)]
    assert max(errs) < 1e-10, errs


@pytest.mark.gpu
def test_advance_with_lanes_drives_the_device(gpu_available):
    """rain.advance with convection cells: lanes first, the squalls added,
    every ufreq/10 steps; the lane field is in the rain fields."""
    from css_b200.context import Simulation
    p, prof, v0, dt, r = setup(seed=3)
    cc = rain.ConvectionCells(p, 6, meansize=0.05, stopin=-1e-3, utopin=-0.02, seed=2)
    sim = Simulation(p, prof)
    sim.upload(v0)
    sim.set_clock(0, 0.0, dt)
    rain.advance(sim, r, dt, 4, p.ufreq, lanes=cc)
    dvel, dent = sim.rain_fields()
    assert np.isfinite(sim.download()).all()
    # the same cells and squalls rebuilt by hand give the same fields
    sim.build_lanes(cc.cells(), cc.meansize, cc.meanvel, cc.meands)
    lanes_only = sim.rain_fields()[0]
    assert np.abs(lanes_only).max() > 0.0
    assert np.isfinite(dvel).all() and np.isfinite(dent).all()
