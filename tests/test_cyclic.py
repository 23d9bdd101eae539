"""The cyclic phi derivative, an extension beside the reference's
block-closed Dbydp / D2bydp2 (derivatives.f90:1480-1684): every whole phi
line solved as one periodic compact system (Sherman-Morrison).

The oracle's restatement is pinned on dense solves of the circulant system
and on sixth-order convergence; the device entry point css_dbydp_cyclic is
held to the oracle at the FP64 derivative bar (1e-12); and on a smooth
periodic field the cyclic and the reference's blocked operators agree to
truncation level, the cyclic one being the more accurate."""
import math

import numpy as np
import pytest

from css_b200 import problem
from oracle import oracle as O


def circulant(n, order):
    a = 1.0 / 3.0 if order == 1 else 2.0 / 11.0
    A = np.eye(n)
    R = np.zeros((n, n))
    for j in range(n):
        A[j, (j - 1) % n] = a
        A[j, (j + 1) % n] = a
        if order == 1:
            R[j, (j + 1) % n] += 7 / 9; R[j, (j - 1) % n] -= 7 / 9
            R[j, (j + 2) % n] += 1 / 36; R[j, (j - 2) % n] -= 1 / 36
        else:
            R[j, (j + 1) % n] += 12 / 11; R[j, (j - 1) % n] += 12 / 11
            R[j, (j + 2) % n] += 3 / 44; R[j, (j - 2) % n] += 3 / 44
            R[j, j] -= 2 * 12 / 11 + 2 * 3 / 44
    return A, R


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("n", [5, 12, 97])
def test_oracle_equals_dense_circulant_solve(order, n):
    rng = np.random.default_rng(n + order)
    x = rng.standard_normal((4, n))
    A, R = circulant(n, order)
    want = np.linalg.solve(A, R @ x.T).T * 3.0 ** order
    got = O.cyclic_lines(x, order, 3.0)
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()


@pytest.mark.parametrize("order", [1, 2])
def test_oracle_sixth_order(order):
    errs = []
    for n in (32, 64, 128):
        ph = 2 * math.pi * np.arange(n) / n
        d = O.cyclic_lines(np.sin(3 * ph), order, n / (2 * math.pi))
        exact = 3 * np.cos(3 * ph) if order == 1 else -9 * np.sin(3 * ph)
        errs.append(np.abs(d - exact).max())
    rates = [math.log2(errs[i] / errs[i + 1]) for i in range(2)]
    assert min(rates) > 5.8, rates


def smooth_periodic_field(p):
    theta, phi, _, _ = problem.angles(p)
    r = np.linspace(p.r1, p.r2, p.nr)
    u = 2 * math.pi * (phi - p.phi1) / (p.phi2 - p.phi1)
    return (1.0 + 0.1 * r[:, None, None]) * (np.sin(3 * u)[None, :, None] + 0.3 * np.cos(u)[None, :, None]) * \
        np.sin(theta)[None, None, :], u, (p.phi2 - p.phi1) / (2 * math.pi)


@pytest.mark.parametrize("order", [1, 2])
def test_cyclic_and_blocked_agree_to_truncation(order):
    p, prof, v0, dt, _ = problem.build("hydro-64x64x128")
    f, u, L = smooth_periodic_field(p)
    theta, _, _, _ = problem.angles(p)
    g = (1.0 + 0.1 * np.linspace(p.r1, p.r2, p.nr))[:, None, None] * np.sin(theta)[None, None, :]
    if order == 1:
        exact = g * (3 * np.cos(3 * u) - 0.3 * np.sin(u))[None, :, None] / L
    else:
        exact = g * (-9 * np.sin(3 * u) - 0.3 * np.cos(u))[None, :, None] / L ** 2
    cyc = O.dbydp_cyclic(p, f, order)
    blk = O.Oracle(p, prof).deriv(2, order, f, None, None, 0)
    scale = np.abs(exact).max()
    e_cyc = np.abs(cyc - exact).max() / scale
    e_blk = np.abs(blk - exact).max() / scale
    assert e_cyc < 1e-7 and e_blk < 1e-5, (e_cyc, e_blk)
    assert e_cyc <= e_blk
    assert np.abs(cyc - blk).max() / scale < 2 * e_blk


@pytest.mark.gpu
@pytest.mark.parametrize("order", [1, 2])
def test_device_matches_oracle(order, gpu_available):
    from css_b200.context import Simulation
    for name in ("hydro-64x64x128", (40, 40, 60)):
        p, prof, v0, dt, _ = problem.build(name) if isinstance(name, str) else problem.build(name, decomp=(2, 2, 3))
        rng = np.random.default_rng(order)
        f = v0[4] + 1e-3 * rng.standard_normal(v0[4].shape)
        sim = Simulation(p, prof)
        g = sim.dbydp_cyclic(f, order)
        sim.close()
        o = O.dbydp_cyclic(p, f, order)
        assert np.abs(g - o).max() <= 1e-12 * np.abs(o).max(), (name, np.abs(g - o).max() / np.abs(o).max())
