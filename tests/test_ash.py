"""The ASH inflow reader (css_b200.ash; ash_inflow.f90:18-186, interp.f90:
103-176) and its run driver.

CPU: a synthetic file in the reference's direct-access layout reads back
(times relative to record 6's, cos(theta) from field 2's first column);
Interp2d as written reproduces constants everywhere and fields linear in
theta at interior points of a uniform old grid, and its phi stencil takes
the points k-1, k, k+2, k+3; the wall taper moves u_theta's energy into the
entropy field; slices shift once sim_time reaches the third slice.  GPU: a
run crossing a slice boundary against the oracle fed the same slices."""
import math

import numpy as np
import pytest

from css_b200 import ash, problem
from oracle import oracle as O


def make_file(tmp_path, p, nslice=6, ashnth=40, ashnphi=48, seed=1):
    rng = np.random.default_rng(seed)
    th_old = np.linspace(p.th1, p.th2, ashnth)
    costheta = np.cos(th_old)
    slices = 1e-3 * rng.standard_normal((nslice, 5, ashnth, ashnphi))
    times = 1000.0 + 10.0 * np.arange(nslice)
    path = str(tmp_path / "ash_inflow_data")
    ash.write_ash_file(path, slices, costheta, times)
    return path, slices.astype(np.float32).astype(np.float64), costheta, times, ashnth, ashnphi


def setup(tmp_path):
    p, prof, v0, dt, _ = problem.build((48, 48, 64), decomp=(2, 2, 4))
    p.bot_inout, p.bottom_specified, p.ufreq = 1, 1, 3
    return p, prof, v0, dt


def test_reader_layout_and_times(tmp_path):
    p, prof, v0, dt = setup(tmp_path)
    path, slices, costheta, times, ant, anp = make_file(tmp_path, p)
    a = ash.AshInflow(path, ant, anp, p, rhor1=2.0, pr1=3.0)
    rec = a.record(5 * 2 + 3)  # slice 2, field 3
    assert np.array_equal(rec[:, 1:], slices[2, 2])
    assert np.allclose(a.record(2)[:, 0], costheta.astype(np.float32))
    assert np.allclose(a.times, times[:4].astype(np.float32) - np.float32(times[1]))
    assert a.slices.shape == (4, 4, p.nphi, p.nth)


def test_interp2d_constants_and_linear_theta():
    p, prof, v0, dt, _ = problem.build((48, 48, 64), decomp=(2, 2, 4))
    ox = (p.phi2 - p.phi1) / 40 * np.arange(40) + p.phi1
    oy = np.linspace(p.th1 - 0.05, p.th2 + 0.05, 36)
    nx = (p.phi2 - p.phi1) / p.nphi * np.arange(p.nphi) + p.phi1
    ny = (p.th2 - p.th1) / (p.nth - 1) * np.arange(p.nth) + p.th1
    c = ash.interp2d(np.full((36, 40), 2.5), ox, oy, nx, ny)
    assert np.allclose(c, 2.5, rtol=0, atol=1e-14)
    lin = ash.interp2d(np.repeat((3.0 * oy + 1.0)[:, None], 40, axis=1), ox, oy, nx, ny)
    # the y stencil starts one point low (no +1), so the curve is evaluated
    # at mu = (y - oy[k-1]) / dy between oy[k-1] and oy[k]
    dy = oy[36 // 2 - 1] - oy[36 // 2 - 2]
    k = np.maximum(np.floor((ny - oy[0]) / dy).astype(int), 1)
    want = 3.0 * ny + 1.0
    inner = (k >= 2) & (k <= 33)
    assert np.allclose(lin[:, inner], want[inner][None, :], rtol=0, atol=1e-12)


def test_interp2d_phi_stencil_as_written():
    ox = np.arange(10, dtype=float)
    oy = np.arange(6, dtype=float)
    arr = np.zeros((6, 10))
    arr[:, 5] = 1.0  # only x = 5 is nonzero
    # x = 3.5: cell k = 4 (1-based), stencil columns k-1, k, k+2, k+3 = 3, 4, 6, 7 (1-based) = x 2, 3, 5, 6
    out = ash.interp2d(arr, ox, oy, np.array([3.5]), np.array([2.0]))
    mu = (3.5 - 3.0) / (5.0 - 3.0)
    want = ash.catmull_rom(0.0, 0.0, 1.0, 0.0, mu)
    assert out[0, 0] == pytest.approx(want)


def test_taper_and_shift(tmp_path):
    p, prof, v0, dt = setup(tmp_path)
    path, slices, costheta, times, ant, anp = make_file(tmp_path, p)
    a = ash.AshInflow(path, ant, anp, p, rhor1=2.0, pr1=3.0)
    full = np.ones((5, p.nphi, p.nth))
    full[1] = 0.5
    f = a.taper(full)
    assert np.all(f[1][:, 0] == 0.0) and np.all(f[1][:, -1] == 0.0) and np.all(f[1][:, 20] == 0.5)
    cv = p.cp / p.gamma
    assert f[3][0, 0] == pytest.approx(1.0 + cv * 2.0 / 3.0 * 0.25)
    t2 = a.times[2]
    assert not a.shift_if_due(t2 - 1e-9)
    old = a.slices.copy()
    assert a.shift_if_due(t2)
    assert np.array_equal(a.slices[:3], old[1:]) and a.iashtime == 4
    assert a.times[3] == pytest.approx(float(np.float32(times[4])) - float(np.float32(times[1])))


@pytest.mark.gpu
def test_ash_run_parity(tmp_path, gpu_available):
    from css_b200.context import Simulation
    p, prof, v0, dt = setup(tmp_path)
    path, slices, costheta, times, ant, anp = make_file(tmp_path, p)
    a = ash.AshInflow(path, ant, anp, p, rhor1=2.0, pr1=3.0)
    rng = np.random.default_rng(3)
    v = v0.copy()
    v[1:4] = 1e-2 * rng.standard_normal(v[1:4].shape)
    sim, orc = Simulation(p, prof), O.Oracle(p, prof)
    dt = min(dt, list(orc.step_size(v, 0.4).values())[0])
    sim.upload(v)
    sim.inout_init()
    orc.inout_init(v)
    t0 = a.times[2] - 2.5 * dt  # the third step starts past the third slice
    for o in (sim, orc):
        o.set_clock(0, t0, dt)
        o.set_ash_slices(a.slices, a.times, 1.0)
    b = ash.AshInflow(path, ant, anp, p, rhor1=2.0, pr1=3.0)
    o_state = v
    for _ in range(6):
        ash.advance(sim, a, dt, 1)
        _, t = orc.clock()
        if b.shift_if_due(t):
            orc.set_ash_slices(b.slices, b.times, orc.inout_state()["ash_fen_mod"])
        o_state = orc.step(o_state, dt, 1)
    assert a.iashtime == 4 and b.iashtime == 4
    g = sim.download()
    errs = [float(np.abs(g[i] - o_state[i]).max() / np.abs(o_state[i]).max()) for i in range(5)]
    assert max(errs) < 1e-10, errs
    gs, os_ = sim.inout_state(), orc.inout_state()
    assert abs(gs["ash_fen_mod"] - os_["ash_fen_mod"]) <= 1e-12 * abs(os_["ash_fen_mod"])
