"""CPU checks of the FP64 oracle itself: golden vectors from the reference's
own Python operator, the known-answer fields of validation.f90, convergence
order, and the decomposition rules of the reference."""
import math
import os

import numpy as np
import pytest

from css_b200 import params, problem
from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden", "compact_fd6.npz")


def golden_cases():
    g = np.load(GOLD)
    off = 0
    for k in range(len(g["n"])):
        n = int(g["n"][k])
        yield dict(n=n, ibc=int(g["ibc"][k]), field=str(g["field"][k]), dri=float(g["dri"][k]),
                   lo=float(g["lo"][k]), hi=float(g["hi"][k]), f=g["f"][off:off + n], out=g["out"][off:off + n])
        off += n


def test_whole_line_matches_reference_python():
    """Both-ends-physical lines reproduce CSS-Python compact_fd6(dtype=0) for
    every ibc: pins the LU tables, the physical closures and the sweeps."""
    worst = 0.0
    for c in golden_cases():
        dli = c["n"] - 1
        drin = c["dri"] * dli
        d = O.compact_lines(c["f"], 1, True, True, c["ibc"], c["lo"] / dli * drin, c["hi"] / dli * drin,
                            dnum=drin, scale=drin)
        err = np.abs(d - c["out"]).max() / np.abs(c["out"]).max()
        worst = max(worst, err)
    assert worst < 1e-11, worst


def test_dbyd1_dt0_matches_reference_python_except_ibc2():
    """The Fortran Dbyd1_dt0 restatement agrees with compact_fd6 except for
    ibc = 2, where the Fortran zeroes up1 before copying it into up2
    (derivatives.f90:2355-2386) and so solves a different right-end row."""
    for c in golden_cases():
        if c["n"] < 14:
            continue
        dli = c["n"] - 1
        drin = c["dri"] * dli
        d = O.dbyd1_dt0(c["f"], c["lo"] / dli, c["hi"] / dli, c["ibc"]) * drin
        err = np.abs(d - c["out"]).max() / np.abs(c["out"]).max()
        if c["ibc"] == 2:
            assert err > 1e-3
            # the left half is still the same operator
            assert np.abs(d[:4] - c["out"][:4]).max() < 1e-2 * np.abs(c["out"]).max()
        else:
            assert err < 1e-11, (c["n"], c["ibc"], err)


def _uniform_ctx(nr, nth, nphi, dec):
    p = params.default_params(nr, nth, nphi, dec)
    p.non_uniform = 0
    prof, _ = problem.polytrope(p, 3.0)
    prof = prof.reshape(params.NPROF, nr)
    r = p.r1 + (p.r2 - p.r1) * np.arange(nr) / (nr - 1)
    prof[0] = r
    prof[1] = r
    prof[2] = (p.r2 - p.r1) / (nr - 1)
    return p, O.Oracle(p, prof.reshape(-1))


def _fields(p, nm):
    """validation.f90:17-28 test field and its exact gradient (and Laplacian
    parts for the second derivatives)."""
    th, ph, _, _ = problem.angles(p)
    r = p.r1 + (p.r2 - p.r1) * np.arange(p.nr) / (p.nr - 1)
    R, T, P = r[:, None, None], th[None, None, :], ph[None, :, None]
    a = math.pi * nm
    xr, xt, xp = a * (R - p.r1) / (p.r2 - p.r1), a * (T - p.th1) / (p.th2 - p.th1), a * (P - p.phi1) / (p.phi2 - p.phi1)
    f = np.cos(xr) * np.cos(xt) * np.sin(xp)
    g = {
        0: (-a * np.sin(xr) * np.cos(xt) * np.sin(xp) / (p.r2 - p.r1), -(a / (p.r2 - p.r1)) ** 2 * f),
        1: (-a * np.cos(xr) * np.sin(xt) * np.sin(xp) / (p.th2 - p.th1), -(a / (p.th2 - p.th1)) ** 2 * f),
        2: (a * np.cos(xr) * np.cos(xt) * np.cos(xp) / (p.phi2 - p.phi1), -(a / (p.phi2 - p.phi1)) ** 2 * f),
    }
    return f, g


def _bc(direction, kind, f, g1):
    """Boundary data as validation.f90:35-62 and :99-127 set them."""
    if direction == 0:
        lo_f, hi_f, lo_d, hi_d = f[0], f[-1], g1[0], g1[-1]
        tr = lambda a: a.reshape(-1)
    else:
        lo_f, hi_f, lo_d, hi_d = f[:, :, 0], f[:, :, -1], g1[:, :, 0], g1[:, :, -1]
        tr = lambda a: np.ascontiguousarray(a).reshape(-1)  # (nr, nphi) == [ip + nphi*ir]
    lo = {0: 0 * lo_f, 1: lo_f, 2: lo_d, 3: lo_f, 4: lo_d}[kind]
    hi = {0: 0 * hi_f, 1: hi_f, 2: hi_f, 3: hi_d, 4: hi_d}[kind]
    return tr(lo), tr(hi)


@pytest.mark.parametrize("direction", [0, 1, 2])
def test_validation_fields_first_derivative(direction):
    """TestDerivatives known answers (threshold 0.1, validation.f90:212) and
    the convergence order on a 2x refinement: 6th order on halo-closed rows,
    5th on the computed physical closures."""
    errs = []
    for k in (1, 2):
        p, o = _uniform_ctx(32 * k, 32 * k, 48 * k, (2, 2, 3))
        f, g = _fields(p, 2.0)
        e = []
        for kind in (range(5) if direction < 2 else [0]):
            lo, hi = _bc(direction, kind, f, g[direction][0]) if direction < 2 else (None, None)
            d = o.deriv(direction, 1, f, lo, hi, kind)
            e.append(np.abs(d - g[direction][0]).max() / np.abs(g[direction][0]).max())
        errs.append(np.array(e))
        assert max(e) < 0.1
    ratio = errs[0] / errs[1]
    assert ratio.min() > 2 ** 4.5, ratio


@pytest.mark.parametrize("direction", [0, 1, 2])
def test_validation_fields_second_derivative(direction):
    errs = []
    for k in (1, 2):
        p, o = _uniform_ctx(32 * k, 32 * k, 48 * k, (2, 2, 3))
        f, g = _fields(p, 2.0)
        kinds = [1] if direction == 2 else [1, 2, 3, 4]
        e = []
        for kind in kinds:
            if direction < 2:
                lo, hi = _bc(direction, kind, f, g[direction][0])
                if direction == 1 and kind in (2, 3, 4):
                    # D2bydt2 divides the theta Neumann datum by dri, not dti
                    # (derivatives.f90:1322, :1338): hand it datum*dri/dti so
                    # the known answer still applies
                    continue
            else:
                lo = hi = None
            d = o.deriv(direction, 2, f, lo, hi, kind)
            e.append(np.abs(d - g[direction][1]).max() / np.abs(g[direction][1]).max())
        errs.append(np.array(e))
        assert max(e) < 0.1
    ratio = errs[0] / errs[1]
    assert ratio.min() > 2 ** 3.5, ratio


def test_decomposition_rules():
    p, prof, _, _, _ = problem.build((64, 64, 128))
    for dec in [(1, 2, 4), (2, 1, 4), (2, 2, 2), (2, 2, 1)]:
        q = p.copy()
        q.nnr, q.nnt, q.nnp = dec
        with pytest.raises(RuntimeError):
            O.Oracle(q, prof)
    q = p.copy()
    q.nr = 66  # 33-point radial blocks: odd sizes are rejected
    prof2, _ = problem.polytrope(q, 3.0)
    with pytest.raises(RuntimeError):
        O.Oracle(q, prof2)


def test_rhs_hydrostatic_background():
    """Isentropic polytrope at rest, no rotation: du/dt and dw/dt vanish to
    truncation level (pressure gradient balances gravity)."""
    p, prof, v0, _, info = problem.build((64, 64, 96), decomp=(2, 2, 3))
    p.omega_0 = 0.0
    v = v0.copy()
    pr = prof.reshape(params.NPROF, p.nr)
    v[0] = pr[5][:, None, None]
    v[1:4] = 0.0
    v[4] = pr[6][:, None, None]
    _, dv = O.Oracle(p, prof).rhs(v, 1)
    g = pr[7].max()
    assert np.abs(dv[3][1:-1]).max() < 1e-3 * g
    assert np.abs(dv[1]).max() < 1e-8 * g
    assert np.abs(dv[2]).max() < 1e-12


def test_step_runs_and_conserves_shape():
    p, prof, v0, dt, _ = problem.build((64, 64, 96), decomp=(2, 2, 3))
    o = O.Oracle(p, prof)
    v = o.step(v0, dt, 2)
    assert np.isfinite(v).all()
    # impenetrable walls (Bound): u_r = 0 on the radial faces, w = 0 on theta
    assert np.abs(v[3][0]).max() == 0.0 and np.abs(v[3][-1]).max() == 0.0
    assert np.abs(v[1][:, :, 0]).max() == 0.0


def test_mass_is_conserved_to_the_discretisation():
    """Total mass (Compute_Step_Size's mtot, rhs_mpi.f90:92-275) over 40 steps
    from the seeded state with the top damping off (Set_Stop), which adds
    mass at the top shell.  The continuity equation is in non-conservative
    form and the SLD's density ghost at the radial walls is the mean state
    (diffusion.f90:582-728), so mass is conserved only to the discretisation:
    the drift falls as the grid is refined."""
    drift = []
    for dims, dec in (((48, 48, 96), (2, 2, 3)), ((96, 96, 192), (4, 4, 6))):
        p, prof, v0, dt, _ = problem.build(dims, decomp=dec)
        p.set_stop = 1
        o = O.Oracle(p, prof)
        m0 = o.step_size(v0, 0.4)["mtot"]
        v1 = o.step(v0, dt, 40)
        drift.append(abs(o.step_size(v1, 0.4)["mtot"] - m0) / m0)
    assert drift[0] < 5e-6 and drift[1] < 0.5 * drift[0], drift
