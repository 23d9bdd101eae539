"""The two-pass RK4 stage (k_thph + k_rstage, css_fused.cuh) against the
oracle and against the four-kernel stage, over the boundary and physics
options of test_variants on 32^3 virtual blocks (64x64x128 at 2x2x4, the
block shape the fused kernels serve): 3 RK4 steps of a stirred state.
Fused and four-kernel stages differ only in the order in which the
density-theta term joins the tendency sums, so they agree to rounding;
both sit within the FP64 bar of the oracle."""
import numpy as np
import pytest

from css_b200 import problem
from oracle import oracle as O
from test_variants import VARIANTS, check

pytestmark = pytest.mark.gpu

CASES = ["default", "no-slip-both", "constant-flux-top", "theta-u-fixed", "uniform-r", "sld-prandtl",
         "no-mass-diffusion", "no-viscous-heating", "reduced-sound-speed", "mhd-default", "mhd-perfect-conductor",
         "mhd-no-slip"]
EXTRA = {"default": {}, "mhd-default": dict(_magnetic=True),
         "mhd-no-slip": dict(_magnetic=True, top_stress_free=0, bottom_stress_free=0, theta_stress_free=0)}


def build(name):
    flags = dict(VARIANTS.get(name, EXTRA.get(name, {})))
    flags.pop("_dims", None)
    flags.pop("_decomp", None)
    mag = flags.pop("_magnetic", False)
    p, prof, v0, dt, _ = problem.build((64, 64, 128), decomp=(2, 2, 4), magnetic=mag, n_rho=5.0 if mag else 3.0)
    for k, val in flags.items():
        setattr(p, k, val)
    rng = np.random.default_rng(sum(map(ord, name)))
    v = v0.copy()
    v[1:4] = 1e-2 * rng.standard_normal(v[1:4].shape)
    return p, prof, v, dt


def rel(a, b):
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


@pytest.mark.parametrize("name", CASES)
def test_fused_stage_parity(name, gpu_available):
    from css_b200.context import Simulation
    p, prof, v, dt = build(name)
    sim = Simulation(p, prof)
    assert sim.fused, "64x64x128 at 2x2x4 should take the two-pass stage"
    g = sim.step_host(v, dt, 3)
    sim.set_fused(False)
    g4 = sim.step_host(v, dt, 3)
    sim.close()
    o = O.Oracle(p, prof).step(v, dt, 3)
    assert np.isfinite(g).all()
    check(p, prof, v, g, o, bar=1e-10)
    errs = [rel(g[i], g4[i]) for i in range(g.shape[0])]
    assert max(errs) < 1e-12, errs


def test_fused_refused_where_it_does_not_apply(gpu_available):
    from css_b200._lib import CssError
    from css_b200.context import Simulation
    p, prof, v0, dt, _ = problem.build((32, 32, 64), decomp=(2, 2, 4))  # 16-point blocks
    sim = Simulation(p, prof)
    assert not sim.fused
    with pytest.raises(CssError):
        sim.set_fused(True)
    sim.close()
