"""Open radial boundaries: Top_Inflow_Outflow / Bottom_Inflow_Outflow
(rhs_mpi.f90:1857-2067) with entropy rain (entropy_rain.f90:423-523) and the
prescribed ASH bottom (ash_inflow.f90:188-219, step_rk4.f90:495-518).

The reference has no tests or outputs for these routines, so the oracle's
restatement is pinned on properties that follow from the routines as
written:

- blocks away from the open faces see exactly the closed run's RHS;
- on a state at rest (u_r = 0 everywhere, w = v = 0 on the top plane) the
  closed and open tops share every term except the density closure, the
  thermal damping and the relaxation, so the entropy and density tendencies
  differ on the top plane by the relaxation plus the damping alone;
- the rain and ASH forcings enter linearly: switching them on changes the
  face plane by exactly (mdvel + dvel) taur, dent taur, and tau tconst
  ashvars(mu) (a Catmull-Rom curve through the slices);
- the squall fields equal a numpy restatement of Build_Gaussian_Squalls;
- the clock and the mass total follow Program CSS2's loop and the RHS's
  ufreq cadence.

GPU: the CUDA path against the oracle at the FP64 bar (RHS 1e-12, five steps
1e-10) for each open configuration, and the rejections."""
import math

import numpy as np
import pytest

from css_b200 import problem
from oracle import oracle as O


def build(dims=(48, 48, 64), decomp=(2, 2, 4), **flags):
    p, prof, v0, dt, _ = problem.build(dims, decomp=decomp)
    for k, val in flags.items():
        setattr(p, k, val)
    return p, prof, v0, dt


def stirred(v0, seed, amp=1e-2):
    rng = np.random.default_rng(seed)
    v = v0.copy()
    v[1:4] = amp * rng.standard_normal(v[1:4].shape)
    return v


def test_oracle_open_faces_are_local():
    p, prof, v0, dt = build((60, 32, 64), (3, 2, 4))
    v = stirred(v0, 3)
    q = p.copy()
    q.top_inout = q.bot_inout = 1
    oc, oo = O.Oracle(p, prof), O.Oracle(q, prof)
    for o in (oc, oo):
        o.inout_init(v)
        o.set_clock(1, 0.0, dt)
    dc, do = oc.rhs(v, 2)[1], oo.rhs(v, 2)[1]
    mid = slice(20, 40)  # the middle radial block touches no physical face
    assert np.array_equal(dc[:, mid], do[:, mid])
    assert not np.array_equal(dc[:, :20], do[:, :20]) and not np.array_equal(dc[:, 40:], do[:, 40:])


def resting(v0, p):
    v = v0.copy()
    v[3] = 0.0
    v[1:3, -1] = 0.0
    return v


def temperature(p, v):
    g, cv = p.gamma, p.cp / p.gamma
    return (1.0 / (cv * (g - 1.0))) * v[0] ** (g - 1.0) * np.exp(v[4] / cv)


def test_oracle_top_relaxation_on_a_resting_state():
    p, prof, v0, dt = build(delta_s=0.01)
    v = resting(v0, p)
    q = p.copy()
    q.top_inout = 1
    oc, oo = O.Oracle(p, prof), O.Oracle(q, prof)
    oo.set_clock(1, 0.0, dt)
    dc, do = oc.rhs(v, 2)[1], oo.rhs(v, 2)[1]
    pr = prof.reshape(-1, p.nr)
    sr, dr, rhor = pr[6], pr[2], pr[5]
    cv = p.cp / p.gamma
    t = temperature(p, v)[-1]
    s_t, s_b = v[4, -1], v[4, -2]
    tau = math.sqrt((p.gamma - 1.0) * p.cp * p.t0) / dr[-1] / 20.0
    relax = tau * (s_b - s_t) + tau * (sr[0] + p.delta_s - s_t.sum() / s_t.size)
    damp = (p.t0 - t) / (p.damping_time * (p.gamma - 2.0) * t)
    want_ds = relax + cv * damp
    want_drho = -v[0, -1] * damp
    scale = np.abs(dc[4]).max()
    assert np.abs((do[4, -1] - dc[4, -1]) - want_ds).max() <= 1e-12 * scale
    assert np.abs((do[0, -1] - dc[0, -1]) - want_drho).max() <= 1e-12 * np.abs(dc[0]).max()
    assert np.array_equal(do[4, :-1], dc[4, :-1]) and np.array_equal(do[0, :-1], dc[0, :-1])
    assert np.abs(want_ds).max() > 1e-3 * scale


def test_oracle_rain_forcing_is_linear():
    p, prof, v0, dt = build(top_inout=1, do_entropy_rain=1, delta_s=0.01)
    v = stirred(v0, 5)
    o = O.Oracle(p, prof)
    o.set_clock(1, 0.0, dt)
    rng = np.random.default_rng(9)
    zero = np.zeros((p.nphi, p.nth))
    o.set_rain_fields(zero, zero)
    da = o.rhs(v, 2)[1]
    dvel, dent = 1e-2 * rng.standard_normal((p.nphi, p.nth)), 1e-3 * rng.standard_normal((p.nphi, p.nth))
    o.set_rain_fields(dvel, dent)
    db = o.rhs(v, 2)[1]
    pr = prof.reshape(-1, p.nr)
    dr, r = pr[2], pr[1]
    th, _, _, _ = problem.angles(p)
    tau_w = v[0, -1] * np.sin(th)[None, :]
    dmd = -(tau_w * dvel).sum() / tau_w.sum()
    r0 = p.nr // p.nnr * (p.nnr - 1)
    q4 = ((r[-1] - r[r0]) / (p.r2 - r[r0])) ** 4
    taur = math.sqrt((p.gamma - 1.0) * p.cp * p.t0) * q4 / dr[-1] / 2.0
    diff = db - da
    assert np.abs(diff[3, -1] - (dmd + dvel) * taur).max() <= 1e-12 * np.abs(da[3]).max()
    assert np.abs(diff[4, -1] - dent * taur).max() <= 1e-12 * np.abs(da[4]).max()
    assert np.array_equal(db[:, :-1], da[:, :-1]) and np.array_equal(db[:3, -1], da[:3, -1])


def catmull_rom(s, mu):
    a3 = s[1]
    a0 = -0.5 * s[0] + 1.5 * a3 - 1.5 * s[2] + 0.5 * s[3]
    a1 = s[0] - 2.5 * a3 + 2.0 * s[2] - 0.5 * s[3]
    a2 = -0.5 * s[0] + 0.5 * s[2]
    return a0 * mu ** 3 + a1 * mu ** 2 + a2 * mu + a3


def ash_case(p, seed=13):
    rng = np.random.default_rng(seed)
    slices = 1e-3 * rng.standard_normal((4, 4, p.nphi, p.nth))
    times = np.array([1.9e5, 2.0e5, 2.1e5, 2.2e5])
    return slices, times


def test_oracle_ash_forcing_is_a_catmull_rom_curve():
    p, prof, v0, dt = build(bot_inout=1, bottom_specified=1)
    v = stirred(v0, 7)
    o = O.Oracle(p, prof)
    o.inout_init(v)
    slices, times = ash_case(p)
    t = 2.037e5  # mu = 0.37, tconst = 1
    o.set_clock(1, t, dt)
    o.set_ash_slices(np.zeros_like(slices), times, 1.3)
    da = o.rhs(v, 2)[1]
    o.set_ash_slices(slices, times, 1.3)
    db = o.rhs(v, 2)[1]
    mu = (t - times[1]) / (times[2] - times[1])
    ash = catmull_rom(slices, mu)  # (4 fields, nphi, nth)
    dr = prof.reshape(-1, p.nr)[2]
    tau = math.sqrt((p.gamma - 1.0) * p.cp * p.t0) / (20.0 * dr[0])
    diff = db - da
    for k, f in ((3, 0), (1, 1), (2, 2)):
        assert np.abs(diff[k, 0] - tau * ash[f]).max() <= 1e-12 * np.abs(da[k]).max()
    assert np.abs(diff[4, 0] - tau * 1.3 * ash[3]).max() <= 1e-12 * np.abs(da[4]).max()
    assert np.array_equal(db[:, 1:], da[:, 1:]) and np.array_equal(db[0, 0], da[0, 0])


def squalls_numpy(p, sq, sstruct=1):
    """Build_Gaussian_Squalls / Build_Polynomial_Squalls restated with numpy
    over the top blocks."""
    th, ph, dth, dphi = problem.angles(p)
    nth, nphi = p.nth, p.nphi
    tb = np.array_split(np.arange(nth), p.nnt)
    pb = np.array_split(np.arange(nphi), p.nnp)
    dens = np.zeros((nphi, nth))
    dvel, dent = np.zeros_like(dens), np.zeros_like(dens)
    terms = []
    for t_idx in tb:
        for p_idx in pb:
            myth1, myth2, mynth = t_idx[0] + 1, t_idx[-1] + 1, len(t_idx)
            myp1, myp2, mynp = p_idx[0] + 1, p_idx[-1] + 1, len(p_idx)
            T, P = np.meshgrid(th[t_idx], ph[p_idx])
            for k, (t0, p0, size, scal, vel, dels) in enumerate(sq):
                lct = min(max(math.floor((t0 - p.th1) / dth) + 1, 1), nth)
                lcp = min(max(math.floor((p0 - p.phi1) / dphi) + 1, 1), nphi)
                if not (lct + mynth >= myth1 and lct - mynth <= myth2):
                    continue
                shifts = []
                if lcp + mynp >= myp1 and lcp - mynp <= myp2:
                    shifts.append(0.0)
                if lcp + mynp > nphi and myp1 == 1:
                    shifts.append(p.phi2 - p.phi1)
                if lcp - mynp < 1 and myp2 == nphi:
                    shifts.append(-(p.phi2 - p.phi1))
                for sh in shifts:
                    x2 = ((T - t0) ** 2 + (P - p0 + sh) ** 2) * (p.r2 / size) ** 2
                    if sstruct == 1:
                        val = np.where(-x2 > -11.5, scal * np.exp(-x2), 0.0)
                    else:
                        x = np.sqrt(np.minimum(x2, 1.0))
                        val = np.where(x2 <= 1.0, scal * (1 - 18 * x ** 2 + 32 * x ** 3 - 15 * x ** 4), 0.0)
                    terms.append((np.ix_(p_idx, t_idx), val, vel, dels))
    for ix, val, vel, dels in terms:
        dens[ix] += np.abs(val)
    dens = 1.0 / (dens + 1.0)
    for ix, val, vel, dels in terms:
        dvel[ix] += vel * val * dens[ix]
        dent[ix] += dels * val * dens[ix]
    return dvel, dent


def squall_list(p, n=12, seed=21):
    rng = np.random.default_rng(seed)
    sq = np.empty((n, 6))
    sq[:, 0] = rng.uniform(p.th1, p.th2, n)
    sq[:, 1] = rng.uniform(p.phi1, p.phi2, n)
    sq[:, 1][:2] = [p.phi1 + 0.01, p.phi2 - 0.01]  # two squalls across the periodic seam
    sq[:, 2] = rng.uniform(0.02, 0.08, n)
    sq[:, 3] = rng.uniform(0.2, 1.0, n)
    sq[:, 4] = rng.uniform(-0.02, 0.0, n)
    sq[:, 5] = rng.uniform(-1e-3, 0.0, n)
    return sq


@pytest.mark.parametrize("sstruct", [1, 0])
def test_oracle_squalls_match_numpy(sstruct):
    p, prof, v0, dt = build(top_inout=1, do_entropy_rain=1)
    o = O.Oracle(p, prof)
    sq = squall_list(p)
    o.build_squalls(sq, sstruct)
    dvel, dent = o.rain_fields()
    wv, we = squalls_numpy(p, sq, sstruct)
    assert np.abs(dvel - wv).max() <= 1e-14 * np.abs(wv).max()
    assert np.abs(dent - we).max() <= 1e-14 * np.abs(we).max()
    assert np.abs(wv).max() > 0 and np.abs(wv[:, :]).min() == 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("sstruct", [1, 0])
def test_squall_builder_parity(sstruct, gpu_available):
    from css_b200.context import Simulation
    p, prof, v0, dt = build(top_inout=1, do_entropy_rain=1)
    sim, orc = Simulation(p, prof), O.Oracle(p, prof)
    sq = squall_list(p, n=40, seed=sstruct + 3)
    sim.build_squalls(sq, sstruct)
    orc.build_squalls(sq, sstruct)
    for a, b in zip(sim.rain_fields(), orc.rain_fields()):
        assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()


def test_oracle_clock_and_mass_total():
    p, prof, v0, dt = build(bot_inout=1, ufreq=1)
    o = O.Oracle(p, prof)
    o.inout_init(v0)
    s0 = o.inout_state()
    assert abs(s0["mtot"] - s0["m0"]) <= 1e-13 * s0["m0"]
    o.set_clock(0, 0.5, dt)
    v1 = o.step(v0, dt, 1)
    assert o.clock() == (1, 0.5 + dt)
    assert o.inout_state()["mtot"] == s0["mtot"]  # refreshed from the step's start state
    o.step(v1, dt, 1)
    o2 = O.Oracle(p, prof)
    o2.inout_init(v1)
    assert o.inout_state()["mtot"] == o2.inout_state()["mtot"]


def test_initial_perturbation_taper_follows_the_open_faces():
    """mhdsph_mpi.f90:679-714: the entropy perturbation vanishes on a closed
    radial face and is left free on an open one."""
    for top, bot in ((False, False), (True, False), (False, True), (True, True)):
        p, prof, v0, dt, _ = problem.build((32, 32, 64), decomp=(2, 2, 4), top_inout=top, bot_inout=bot)
        sr = prof.reshape(-1, p.nr)[6]
        pert = np.abs(v0[4] / sr[:, None, None] - 1.0)
        mid = slice(8, 24)
        assert (pert[-1][:, mid].max() > 1e-7) == top, (top, bot)
        assert (pert[0][:, mid].max() > 1e-7) == bot, (top, bot)
        assert p.top_inout == int(top) and p.bot_inout == int(bot)


def test_open_from_checkpoint():
    """startbio / starttio: the opened face's u_r copies the neighbouring
    plane scaled by vamp with zero plane mean; an opened top also copies s."""
    p, prof, v0, dt, _ = problem.build((32, 32, 64), decomp=(2, 2, 4))
    v = stirred(v0, 11)
    o = problem.open_from_checkpoint(v, bottom=True, top=True, vamp=0.5)
    for face, inner in ((0, 1), (-1, -2)):
        want = 0.5 * v[3, inner] - (0.5 * v[3, inner]).mean()
        assert np.allclose(o[3, face], want, rtol=0, atol=1e-15)
        assert abs(o[3, face].mean()) < 1e-15
    assert np.array_equal(o[4, -1], v[4, -2]) and np.array_equal(o[4, 0], v[4, 0])
    assert np.array_equal(o[:, 1:-1], v[:, 1:-1]) and np.array_equal(o[:3], v[:3])
    assert np.array_equal(problem.open_from_checkpoint(v), v)


def test_oracle_rejections():
    p, prof, v0, dt = build(bot_inout=1)
    for flags in (dict(magnetic=1), dict(laplacian=1), dict(do_radheat=1), dict(precision=1),
                  dict(bot_inout=0, bottom_specified=1), dict(do_entropy_rain=1)):
        q = p.copy()
        for k, val in flags.items():
            setattr(q, k, val)
        with pytest.raises(RuntimeError):
            O.Oracle(q, prof)


# ---------------------------------------------------------------------------
# GPU parity
# ---------------------------------------------------------------------------
CONFIGS = {
    "top": dict(top_inout=1, delta_s=0.01),
    "bottom": dict(bot_inout=1),
    "both": dict(top_inout=1, bot_inout=1),
    "top-rain": dict(top_inout=1, do_entropy_rain=1, delta_s=0.01),
    "bottom-ash": dict(bot_inout=1, bottom_specified=1, ufreq=2),
    "both-rk3-tvd": dict(top_inout=1, bot_inout=1, time_stepper=3),
}


def setup_pair(name):
    from css_b200.context import Simulation
    p, prof, v0, dt = build(**CONFIGS[name])
    p.ufreq = p.ufreq or 100
    v = stirred(v0, sum(map(ord, name)))
    sim, orc = Simulation(p, prof), O.Oracle(p, prof)
    sim.upload(v)
    sim.inout_init()
    orc.inout_init(v)
    t0 = 2.01e5 if p.bottom_specified else 0.0
    for o in (sim, orc):
        o.set_clock(1, t0, dt)
        if p.do_entropy_rain:
            o.build_squalls(squall_list(p))
        if p.bottom_specified:
            slices, times = ash_case(p)
            o.set_ash_slices(slices, times, 1.3)
    dt = min(dt, list(orc.step_size(v, 0.4).values())[0])
    return p, prof, v, dt, sim, orc


def fieldwise(a, b):
    return [float(np.abs(a[i] - b[i]).max() / max(np.abs(b[i]).max(), 1e-300)) for i in range(a.shape[0])]


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CONFIGS))
def test_open_boundary_parity(name, gpu_available):
    from test_variants import check
    p, prof, v, dt, sim, orc = setup_pair(name)
    for call in (1, 2):
        _, dg = sim.rhs(v, call)
        _, do = orc.rhs(v, call)
        check(p, prof, v, dg, do)
    gs, os_ = sim.inout_state(), orc.inout_state()
    for k in ("m0", "vol", "mtot"):
        assert abs(gs[k] - os_[k]) <= 1e-13 * abs(os_[k]), (k, gs[k], os_[k])
    if p.do_entropy_rain:
        for a, b in zip(sim.rain_fields(), orc.rain_fields()):
            assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()
    sim.upload(v)
    g = v
    o = v
    for _ in range(5):  # step by step, so the clocks are compared every step
        sim.step_rk4(dt, 1)
        o = orc.step(o, dt, 1)
        assert sim.clock()[0] == orc.clock()[0] and sim.clock()[1] == orc.clock()[1]
    g = sim.download()
    errs = fieldwise(g, o)
    assert max(errs) < 1e-10, errs
    assert np.isfinite(g).all()
    gs, os_ = sim.inout_state(), orc.inout_state()
    for k in ("mtot", "ash_fen_mod"):
        assert abs(gs[k] - os_[k]) <= 1e-12 * max(abs(os_[k]), 1e-300), (k, gs[k], os_[k])


@pytest.mark.gpu
def test_open_boundary_rejections(gpu_available):
    from css_b200._lib import CssError
    from css_b200.context import Simulation
    from css_b200.ensemble import Ensemble
    p, prof, v0, dt = build(top_inout=1)
    for flags in (dict(precision=1), dict(laplacian=1), dict(do_entropy_rain=1, top_inout=0)):
        q = p.copy()
        for k, val in flags.items():
            setattr(q, k, val)
        with pytest.raises(CssError):
            Simulation(q, prof)
    sim = Simulation(p, prof)
    with pytest.raises(CssError):
        Ensemble([sim])
    q = p.copy()
    q.top_inout, q.bot_inout, q.bottom_specified = 0, 1, 1
    s2 = Simulation(q, prof)
    s2.upload(v0)
    slices, times = ash_case(q)
    s2.set_ash_slices(slices, times, 1.0)
    s2.set_clock(0, times[2], dt)  # past the third slice: the caller must shift first
    with pytest.raises(CssError):
        s2.step_rk4(dt, 1)
    closed = Simulation(build()[0], prof)
    with pytest.raises(CssError):
        closed.inout_init()
    fresh = Simulation(p, prof)  # open top, clock never set: deltat 0
    with pytest.raises(CssError):
        fresh.rhs(v0, 2)
    fresh.set_clock(1, 0.0, dt)
    assert np.isfinite(fresh.rhs(v0, 2)[1]).all()
