"""Diagnostics of the current state: Scalar_Output (report_mpi.f90:173-262),
Compute_Step_Size (rhs_mpi.f90:92-275), Shell_Average_Output
(report_mpi.f90:783-1094) and the folded FFT spectrum of
CSS-IDL/spectral_analysis_new.pro:16-25.

The CPU tests pin the oracle against independent numpy statements of the
same formulas (numpy's FFT with the IDL folding written out index by index,
sums and extrema with numpy reductions).  The GPU tests hold the device
diagnostics to the oracle at 1e-12 (relative to the largest magnitude of
each output row); sums differ only in their order."""
import math

import numpy as np
import pytest

from css_b200 import problem
from css_b200.params import PROF_NAMES
from oracle import oracle as O


def rel(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


def stirred(dims, magnetic=False, seed=5, decomp=(2, 2, 4)):
    """A seeded state with velocities of a few percent of the sound speed."""
    p, prof, v0, dt, info = problem.build(dims, magnetic=magnetic, decomp=decomp)
    rng = np.random.default_rng(seed)
    v = v0.copy()
    nr, nphi, nth = p.nr, p.nphi, p.nth
    it = np.arange(nth)[None, None, :]
    ip = np.arange(nphi)[None, :, None]
    for k, m in ((1, 2), (2, 3), (3, 5)):
        v[k] = 1e-2 * (np.sin(2 * math.pi * m * ip / nphi + 0.3 * k) * np.cos(math.pi * it / (nth - 1))
                       + 0.3 * rng.standard_normal((nr, nphi, nth)))
    return p, prof, v


def prof_row(p, prof, name):
    return np.asarray(prof).reshape(len(PROF_NAMES), p.nr)[PROF_NAMES.index(name)]


def temperature(p, v):
    gamm1 = p.gamma - 1.0
    cv = p.cp / p.gamma
    return v[0] ** gamm1 * np.exp(v[4] / cv) / cv / gamm1


def idl_spectrum(p, field):
    """spectral_analysis_new.pro:16-25 for one snapshot, field (nr, nphi, nth)."""
    theta, _, _, _ = problem.angles(p)
    nth, nphi = p.nth, p.nphi
    apod = 1.0 - np.cos(math.pi * (theta - theta.min()) / (theta.max() - theta.min())) ** 64
    out = np.zeros((p.nr, nphi // 2))
    for ir in range(p.nr):
        tdat = field[ir].T * apod[:, None]                 # (nth, nphi), theta first as in IDL
        tmp = np.fft.fft2(tdat) / (nth * nphi)             # IDL forward FFT divides by N
        cube = np.zeros((nth // 2, nphi // 2))
        cube[0, 0] = tmp[0, 0].real
        rev = tmp[nth // 2:, nphi // 2:][::-1, ::-1]       # reverse(reverse(tmp[nth/2:*,nphi/2:*],1),2)
        cube[1:, 1:] = (tmp[1:nth // 2, 1:nphi // 2] + rev[:nth // 2 - 1, :nphi // 2 - 1]).real
        out[ir] = cube.sum(axis=0) / (nth / 2.0)
    return out


# ---------------------------------------------------------------------------
# CPU: the oracle against numpy
# ---------------------------------------------------------------------------
def test_oracle_spectrum_matches_numpy_fft_fold():
    p, prof, v = stirred((24, 32, 64))
    orc = O.Oracle(p, prof)
    ke = 0.5 * v[0] * (v[1] ** 2 + v[2] ** 2 + v[3] ** 2)
    assert rel(orc.spectrum(v, 0), idl_spectrum(p, ke)) < 1e-12
    assert rel(orc.spectrum(v, 2 + 4), idl_spectrum(p, v[4])) < 1e-12


def test_oracle_spectrum_of_one_phi_mode_has_one_line():
    p, prof, v = stirred((24, 32, 64))
    ip = np.arange(p.nphi)[None, :, None]
    v[4] = np.cos(2 * math.pi * 3 * ip / p.nphi) * (1.0 + 0.0 * v[4])
    s = O.Oracle(p, prof).spectrum(v, 2 + 4)
    mask = np.ones(p.nphi // 2, bool)
    mask[3] = False
    assert np.abs(s[:, mask]).max() < 1e-13 * np.abs(s[:, 3]).max()
    assert np.abs(s[:, 3]).min() > 0.0


def test_oracle_shell_averages_match_numpy():
    p, prof, v = stirred((24, 32, 64))
    orc = O.Oracle(p, prof)
    q = [1, 2, 3, 4, 5, 6, 7, 8, 16, 17, 18]
    got = orc.shell_averages(v, q)
    T = temperature(p, v)
    gamm1, cv = p.gamma - 1.0, p.cp / p.gamma
    mean = lambda f: f.reshape(p.nr, -1).mean(axis=1)
    ke = 0.5 * v[0] * (v[1] ** 2 + v[2] ** 2 + v[3] ** 2)
    ub, tb, pb = mean(v[3]), mean(T), gamm1 * cv * mean(v[0] * T)
    du = v[3] - ub[:, None, None]
    want = {1: mean(v[0]), 2: mean(T), 3: mean(v[4]), 4: gamm1 * cv * mean(v[0] * T), 5: mean(v[3]),
            6: mean(v[1]), 7: mean(v[2]), 8: mean(ke), 16: p.cp * mean(du * v[0] * (T - tb[:, None, None])),
            17: mean(ke * du), 18: mean((gamm1 * cv * v[0] * T - pb[:, None, None]) * du)}
    for i, qq in enumerate(q):
        assert rel(got[i], want[qq]) < 1e-12, qq


def test_oracle_shell_average_dsdr_is_the_radial_derivative():
    p, prof, v = stirred((24, 32, 64))
    orc = O.Oracle(p, prof)
    got = orc.shell_averages(v, [9, 15], k0=np.full(p.nr, 2.5))
    # Compute_Derivatives' face datum: dsdr1/dxdr(1), dsdr2/dxdr(nr) with the
    # constant-flux gradient of the SLaplacian background (mhdsph_mpi.f90:573-582)
    ks, dxdr = prof_row(p, prof, "ks"), prof_row(p, prof, "dxdr")
    d1 = -p.lumr1 / (4 * math.pi) / (ks[0] * p.r1 ** 2) if (p.slaplacian and not p.bottom_constant_temp) else 0.0
    d2 = -p.lumr2 / (4 * math.pi) / (ks[-1] * p.r2 ** 2) if (p.slaplacian and not p.top_constant_temp) else 0.0
    lo = np.full((p.nphi, p.nth), d1 / dxdr[0])
    hi = np.full((p.nphi, p.nth), d2 / dxdr[-1])
    dsdr = orc.deriv(0, 1, v[4], lo, hi, bdry=orc_lbcr_s(p))
    if p.non_uniform:
        dsdr = dsdr * prof_row(p, prof, "dxdr")[:, None, None]
    want = dsdr.reshape(p.nr, -1).mean(axis=1)
    assert rel(got[0], want) < 1e-12
    assert rel(got[1], (-ks * want if p.slaplacian else 0.0) + 2.5) < 1e-12


def orc_lbcr_s(p):
    tt, bt = p.top_constant_temp, p.bottom_constant_temp
    return 1 if (tt and bt) else 2 if (tt and not bt) else 3 if (bt and not tt) else 4


def test_oracle_scalars_and_step_size_match_numpy():
    p, prof, v = stirred((24, 32, 64))
    orc = O.Oracle(p, prof)
    sc = orc.scalars(v)
    n = v[0].size
    rho, w, vp, u = v[0], v[1], v[2], v[3]
    gamm1, cv = p.gamma - 1.0, p.cp / p.gamma
    T = temperature(p, v)
    usq = w ** 2 + vp ** 2 + u ** 2
    want = {"kinener": (rho * usq).sum() / (2 * n), "cke": (rho * u ** 2).sum() / (2 * n),
            "drke": (rho * vp ** 2).sum() / (2 * n),
            "umach": math.sqrt((usq / (usq + T * gamm1 * p.cp)).max())}
    want["mcke"] = want["cke"] + (rho * w ** 2).sum() / (2 * n)
    for k, val in want.items():
        assert abs(sc[k] - val) <= 1e-12 * abs(val), k
    st = orc.step_size(v, 0.4)
    theta, _, _, _ = problem.angles(p)
    r = prof_row(p, prof, "r_ind")[:, None, None]
    dr = prof_row(p, prof, "dr_ind")[:, None, None]
    sn = np.sin(theta)[None, None, :]
    dth = (p.th2 - p.th1) / (p.nth - 1)
    dphi = (p.phi2 - p.phi1) / p.nphi
    dxmin = np.minimum(dr, r * np.minimum(dth, sn * dphi))
    ut = u ** 2 + vp ** 2 + w ** 2 + gamm1 * p.cp * p.xi_cs ** 2 * T
    assert abs(st["dtmax"] - 0.4 * min(1e4, (dxmin / np.sqrt(ut)).min())) <= 1e-13 * st["dtmax"]
    wv = r ** 2 * sn * dr * dth * dphi
    e = (wv * rho * (cv * T + 0.5 * (u ** 2 + w ** 2 + vp ** 2))).sum()
    lt = (wv * r * rho * np.sqrt(w ** 2 + sn ** 2 * (vp + r * sn * p.omega_0) ** 2)).sum()
    assert abs(st["Etot"] - e) <= 1e-12 * abs(e)
    assert abs(st["Ltot"] - lt) <= 1e-12 * abs(lt)
    assert abs(st["mtot"] - (wv * rho).sum()) <= 1e-12 * (wv * rho).sum()
    assert abs(st["mrsint"] - (wv * r * sn ** 2 * rho).sum()) <= 1e-12 * (wv * r * sn ** 2 * rho).sum()


def test_oracle_magnetic_diagnostics_match_numpy():
    p, prof, v = stirred((24, 32, 64), magnetic=True)
    orc = O.Oracle(p, prof)
    b = orc.curl_b(v[5:8])
    bt, bp, br = b
    bsq = br ** 2 + bt ** 2 + bp ** 2
    got = orc.shell_averages(v, [10, 11, 12, 13, 14])
    mean = lambda f: f.reshape(p.nr, -1).mean(axis=1)
    for g, w in zip(got, [mean(br), mean(bt), mean(bp), mean(0.125 * bsq / math.pi), mean(np.sqrt(br ** 2 + bt ** 2))]):
        assert rel(g, w) < 1e-12
    sc = orc.scalars(v)
    assert abs(sc["magener"] - bsq.sum() / (8 * math.pi * bsq.size)) <= 1e-12 * sc["magener"]
    assert abs(sc["bmax"] - np.sqrt(bsq).max() * 2 * math.sqrt(2 * math.pi)) <= 1e-13 * sc["bmax"]
    assert rel(orc.spectrum(v, 1), idl_spectrum(p, 0.125 * bsq / math.pi)) < 1e-12


def test_oracle_rejects_unsupported_quantities():
    p, prof, v = stirred((24, 32, 64))
    orc = O.Oracle(p, prof)
    for q in ([19], [0], [10]):
        with pytest.raises(RuntimeError):
            orc.shell_averages(v, q)


# ---------------------------------------------------------------------------
# GPU: the device diagnostics against the oracle
# ---------------------------------------------------------------------------
ALL_HYDRO = list(range(1, 10)) + list(range(15, 19))


def summand_scales(p, prof, v, orc):
    """Error scale of the averages whose summands cancel.  ds/dr (and F_ks)
    of a near-isentropic state is a small difference of large entropies, so
    its rounding scales with the derivative's input: max|s| dnum max(dxdr).
    The fluxes about the means: their largest |summand|."""
    ks, dxdr = prof_row(p, prof, "ks"), prof_row(p, prof, "dxdr")
    d1 = -p.lumr1 / (4 * math.pi) / (ks[0] * p.r1 ** 2) if (p.slaplacian and not p.bottom_constant_temp) else 0.0
    d2 = -p.lumr2 / (4 * math.pi) / (ks[-1] * p.r2 ** 2) if (p.slaplacian and not p.top_constant_temp) else 0.0
    lo = np.full((p.nphi, p.nth), d1 / dxdr[0])
    hi = np.full((p.nphi, p.nth), d2 / dxdr[-1])
    dsdr = orc.deriv(0, 1, v[4], lo, hi, bdry=orc_lbcr_s(p))
    if p.non_uniform:
        dsdr = dsdr * dxdr[:, None, None]
    amean = lambda f: np.abs(f).reshape(p.nr, -1).max(axis=1)
    T = temperature(p, v)
    gamm1, cv = p.gamma - 1.0, p.cp / p.gamma
    ke = 0.5 * v[0] * (v[1] ** 2 + v[2] ** 2 + v[3] ** 2)
    au = np.abs(v[3]) + np.abs(v[3]).reshape(p.nr, -1).mean(axis=1)[:, None, None]
    x = prof_row(p, prof, "x_ind")
    dscale = np.abs(v[4]).max() * (p.nr - 1) / (x[-1] - x[0]) * (np.abs(dxdr).max() if p.non_uniform else 1.0)
    return {9: dscale, 15: np.abs(ks).max() * dscale,
            16: p.cp * amean(au * v[0] * 2 * T).max(), 17: amean(ke * au).max(),
            18: amean(2 * gamm1 * cv * v[0] * T * au).max()}


@pytest.mark.gpu
@pytest.mark.parametrize("magnetic", [False, True])
def test_device_diagnostics_match_oracle(gpu_available, magnetic):
    from css_b200.context import Simulation
    dims = (32, 64, 128) if not magnetic else (24, 32, 64)
    p, prof, v = stirred(dims, magnetic=magnetic)
    sim = Simulation(p, prof)
    orc = O.Oracle(p, prof)
    sim.upload(v)
    q = ALL_HYDRO + ([10, 11, 12, 13, 14] if magnetic else [])
    k0 = np.linspace(1.0, 2.0, p.nr)
    g, o = sim.shell_averages(q, k0), orc.shell_averages(v, q, k0)
    # an average whose terms cancel is held to 1e-12 of the scale of those
    # terms (summand_scales), every other output to 1e-12 of its own size
    scale = summand_scales(p, prof, v, orc)
    for i, qq in enumerate(q):
        err = np.abs(g[i] - o[i]).max()
        assert err <= 1e-12 * max(scale.get(qq, 0.0), np.abs(o[i]).max()), (qq, err, scale.get(qq))
    gs, os_ = sim.scalars(), orc.scalars(v)
    for k in os_:
        assert abs(gs[k] - os_[k]) <= 1e-12 * max(abs(os_[k]), 1e-300), k
    gz, oz = sim.step_size(0.4), orc.step_size(v, 0.4)
    for k in oz:
        assert abs(gz[k] - oz[k]) <= 1e-12 * abs(oz[k]), k
    for kind in [0, 2, 6] + ([1] if magnetic else []):
        gsp, osp = sim.spectrum(kind), orc.spectrum(v, kind)
        assert rel(gsp, osp) < 1e-12, (kind, rel(gsp, osp))
    # the state is untouched and a step still matches after the diagnostics
    assert np.array_equal(sim.download(), v)


@pytest.mark.gpu
def test_device_diagnostics_reject_bad_requests(gpu_available):
    from css_b200._lib import CssError
    from css_b200.context import Simulation
    p, prof, v = stirred((24, 32, 64))
    sim = Simulation(p, prof)
    sim.upload(v)
    for q in ([19], [0], [12]):
        with pytest.raises(CssError):
            sim.shell_averages(q)
    with pytest.raises(CssError):
        sim.spectrum(1)
