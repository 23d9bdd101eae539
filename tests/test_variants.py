"""GPU parity over the boundary and physics options the workloads leave at
their defaults (Read_Input, mhdsph_mpi.f90:1302-1462; the BC integers of
derivatives.f90:50-57; the SLD switches of diffusion.f90:8-11).

Each variant changes one group of flags from the default run: no-slip walls
(lbcr_v 1, 2, 3), a constant-flux top, theta walls without the stress-free
u_r condition (lbct_u 1), a uniform radial grid, SLD Prandtl scalings,
mass diffusion or viscous heating off, a reduced sound speed (xi_cs < 1),
block sizes other than 16 and 32 (the generic kernels; ragged blocks always
include an odd size, which css_create rejects), and for MHD perfectly
conducting walls in r and theta.  Every variant: the RHS of a stirred state (calls 1
and 2), the SLD tendency, and 5 RK4 steps against the oracle at the FP64
bar.  The entropy tendency is held to 1e-12 of its largest summand (the
conduction stencil at the constant-flux wall, see test_radheat)."""
import numpy as np
import pytest

from css_b200 import problem
from css_b200.params import PROF_NAMES
from oracle import oracle as O

pytestmark = pytest.mark.gpu

VARIANTS = {
    "no-slip-both": dict(top_stress_free=0, bottom_stress_free=0),
    "no-slip-top": dict(top_stress_free=0),
    "no-slip-bottom": dict(bottom_stress_free=0),
    "constant-flux-top": dict(top_constant_temp=0),
    "theta-u-fixed": dict(theta_stress_free=0),
    "uniform-r": dict(non_uniform=0),
    "sld-prandtl": dict(sld_pr=0.5),
    "no-mass-diffusion": dict(mass_diffusion=0),
    "no-viscous-heating": dict(do_viscous_heating=0),
    "reduced-sound-speed": dict(xi_cs=0.5),
    "generic-block-sizes": dict(_dims=(44, 40, 60), _decomp=(2, 2, 3)),  # blocks 22, 20, 20
    "mhd-perfect-conductor": dict(_magnetic=True, theta_normal_field=0, theta_perf_conductor=1,
                                  top_radial_field=0, bottom_radial_field=0, top_perfect_cond=1,
                                  bottom_perfect_cond=1, sld_prm=0.5),
}


def build(name):
    flags = dict(VARIANTS[name])
    dims = flags.pop("_dims", (32, 32, 64))
    decomp = flags.pop("_decomp", (2, 2, 4))
    mag = flags.pop("_magnetic", False)
    p, prof, v0, dt, _ = problem.build(dims, decomp=decomp, magnetic=mag)
    for k, val in flags.items():
        setattr(p, k, val)
    rng = np.random.default_rng(sum(map(ord, name)))
    v = v0.copy()
    v[1:4] = 1e-2 * rng.standard_normal(v[1:4].shape)
    return p, prof, v, dt


def temperature(p, v):
    g, cv = p.gamma, p.cp / p.gamma
    return (1.0 / (cv * (g - 1.0))) * v[0] ** (g - 1.0) * np.exp(v[4] / cv)


def conduction_scale(p, prof, v):
    pr = prof.reshape(len(PROF_NAMES), p.nr)
    x, dxdr, ks = (pr[PROF_NAMES.index(k)] for k in ("x_ind", "dxdr", "ks"))
    if not p.non_uniform:
        dxdr = np.ones_like(dxdr)
    w = ks[:, None, None] * (dxdr[:, None, None] / np.diff(x).min()) ** 2
    return float((w / (v[0] * temperature(p, v)) * np.abs(v[4])).max())


def check(p, prof, v, g, o, bar=1e-12):
    for i in range(g.shape[0]):
        scale = np.abs(o[i]).max()
        if i == 4:
            scale = max(scale, conduction_scale(p, prof, v))
        err = np.abs(g[i] - o[i]).max()
        assert err <= bar * max(scale, 1e-300), (i, err / max(scale, 1e-300))


@pytest.mark.parametrize("name", list(VARIANTS))
def test_variant_parity(name, gpu_available):
    from css_b200.context import Simulation
    p, prof, v, dt = build(name)
    sim, orc = Simulation(p, prof), O.Oracle(p, prof)
    for call in (1, 2):
        _, dg = sim.rhs(v, call)
        _, do = orc.rhs(v, call)
        check(p, prof, v, dg, do)
    if p.magnetic:  # B from the RHS call, A alongside (Compute_Diffusion's inputs)
        vb = orc.rhs(v, 1)[0]
        _, dg = sim.diffusion(vb, v[5:])
        _, do = orc.diffusion(vb, v[5:])
    else:
        _, dg = sim.diffusion(v)
        _, do = orc.diffusion(v)
    check(p, prof, v, dg, do)
    g = sim.step_host(v, dt, 5)
    o = orc.step(v, dt, 5)
    check(p, prof, v, g, o, bar=1e-10)
    assert np.isfinite(g).all()


BOUND_CASES = dict(VARIANTS, **{"default": {}, "mhd-default": dict(_magnetic=True),
                                "open-top": dict(top_inout=1), "open-bottom": dict(bot_inout=1)})


@pytest.mark.parametrize("name", ["default", "no-slip-both", "theta-u-fixed", "mhd-default", "mhd-perfect-conductor",
                                  "open-top", "open-bottom"])
def test_bound_entry_point(name, gpu_available):
    """css_bound applies Bound() (rhs_mpi.f90:2395-2491) to a whole state
    exactly as the oracle does: the same entries zeroed, the rest untouched."""
    from css_b200.context import Simulation
    flags = dict(BOUND_CASES[name])
    mag = flags.pop("_magnetic", False)
    p, prof, v0, dt, _ = problem.build((32, 32, 64), decomp=(2, 2, 4), magnetic=mag)
    for k, val in flags.items():
        setattr(p, k, val)
    rng = np.random.default_rng(sum(map(ord, name)))
    v = v0 + 1e-2 * rng.standard_normal(v0.shape)
    g = Simulation(p, prof).bound(v)
    o = O.Oracle(p, prof).bound(v)
    assert np.array_equal(g, o)
    assert (g == 0.0).sum() > 0 and np.array_equal(g[:, 1:-1, :, 1:-1], v[:, 1:-1, :, 1:-1])
