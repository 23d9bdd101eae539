"""css_deriv_pencils, the reference's per-pencil derivative calls batched:
Dbydr's pencils are (theta, r) planes of one phi, Dbydt's and Dbydp's
(theta, phi) planes of one radius.  Each pencil's derivative is the same
plane of the whole-field derivative bit for bit (the same kernels on the
same values, each pencil at its own phi index or radius: D2bydt2 scales
its Neumann datum by the radial block's spacing), for both orders, boundary variants from var (<= 0 a bdry,
>= 1 the run's tables), physical-face data per pencil, pencils in any
order and repeated, and more pencils than one pass holds."""
import numpy as np
import pytest

from css_b200 import problem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def run():
    from css_b200.context import Simulation
    p, prof, v0, dt, _ = problem.build((48, 48, 64), decomp=(2, 2, 4))
    sim = Simulation(p, prof)
    yield p, sim
    sim.close()


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("var", [-1, -2, 0, 4])
def test_r_pencils_match_whole_field(gpu_available, run, order, var):
    p, sim = run
    rng = np.random.default_rng(order + 10 * (var + 3))
    F = rng.standard_normal((p.nr, p.nphi, p.nth))
    lo, hi = rng.standard_normal((p.nphi, p.nth)), rng.standard_normal((p.nphi, p.nth))
    ips = [5, 0, 63, 17, 17, 40] + list(range(p.nphi))  # repeated, unordered, more than one pass
    x = np.stack([F[:, ip, :] for ip in ips])
    got = sim.deriv_pencils(0, order, x, ips, lo[ips], hi[ips], var)
    if var <= 0:
        whole = sim.deriv(0, order, F, lo, hi, -var)
    else:  # the named whole-field routine takes var the same way
        import ctypes
        from css_b200 import _lib
        dp = ctypes.POINTER(ctypes.c_double)
        whole = np.empty_like(F)
        fn = _lib.lib().css_dbydr if order == 1 else _lib.lib().css_d2bydr2
        _lib.check(fn(sim.h, F.ctypes.data_as(dp), whole.ctypes.data_as(dp), lo.ctypes.data_as(dp),
                      hi.ctypes.data_as(dp), var))
    for k, ip in enumerate(ips):
        assert np.array_equal(got[k], whole[:, ip, :]), (k, ip)


@pytest.mark.parametrize("direction", [1, 2])
@pytest.mark.parametrize("order", [1, 2])
def test_theta_phi_pencils_match_whole_field(gpu_available, run, direction, order):
    p, sim = run
    rng = np.random.default_rng(7 * direction + order)
    F = rng.standard_normal((p.nr, p.nphi, p.nth))
    lo, hi = rng.standard_normal((p.nr, p.nphi)), rng.standard_normal((p.nr, p.nphi))
    irs = [47, 3, 3, 20] + list(range(p.nr))
    x = np.stack([F[ir] for ir in irs])
    if direction == 1:
        got = sim.deriv_pencils(1, order, x, irs, lo[irs], hi[irs], -2)
        whole = sim.deriv(1, order, F, lo, hi, 2)
    else:
        got = sim.deriv_pencils(2, order, x, irs, var=0)
        whole = sim.deriv(2, order, F)
    for k, ir in enumerate(irs):
        assert np.array_equal(got[k], whole[ir]), (k, ir)


def test_pencils_refuse_bad_arguments(gpu_available, run):
    from css_b200._lib import CssError
    p, sim = run
    x = np.zeros((2, p.nr, p.nth))
    with pytest.raises(CssError):
        sim.deriv_pencils(0, 3, x)
    with pytest.raises(CssError):
        sim.deriv_pencils(0, 1, x, var=13)
    with pytest.raises(CssError):
        sim.deriv_pencils(0, 1, x, index=[0, p.nphi])
