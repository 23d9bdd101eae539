"""GPU parity: every CUDA entry point against the CPU oracle on the same
seeded inputs (normwise relative error = max|gpu - oracle| / max|oracle|
per field).  Tolerances are the FP64 bar of the hot path: derivatives and
RHS 1e-12, state after 100 RK4 steps 1e-10.  The two sides differ only in
rounding (the GPU contracts a*b+c into FMA, the x86 oracle does not, and
pow/exp/sin differ by an ulp), so the observed errors sit at 1e-15..7e-13.
One case is looser on purpose: the RHS of a state at rest, whose momentum
tendencies are the residual of a hydrostatic balance between terms ~1e4
times larger, is held to 1e-11."""
import numpy as np
import pytest

from css_b200 import params, problem
from css_b200.context import Simulation, compact_fd6, compact_lines, dbyd1_dt0
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


def fieldwise(a, b):
    return [rel(a[i], b[i]) for i in range(a.shape[0])]


@pytest.fixture(scope="module")
def cfg1():
    p, prof, v0, dt, info = problem.build("hydro-64x64x128")
    return p, prof, v0, dt


@pytest.fixture(scope="module")
def sims(cfg1, gpu_available):
    p, prof, v0, dt = cfg1
    return Simulation(p, prof), O.Oracle(p, prof)


def test_compact_fd6_shim_matches_reference_goldens(gpu_available):
    from test_oracle import golden_cases
    worst = 0.0
    for c in golden_cases():
        darr = np.zeros(c["n"])
        darr[0], darr[-1] = c["lo"], c["hi"]
        d = compact_fd6(c["dri"], c["f"], 0.0, 0.0, c["ibc"], 0, darr=darr)
        worst = max(worst, rel(d, c["out"]))
    assert worst < 1e-11, worst


def test_dbyd1_dt0_matches_oracle(gpu_available):
    rng = np.random.default_rng(3)
    x = np.cumsum(rng.standard_normal((7, 96)), axis=1) * 0.01
    for ibc in range(5):
        b1, b2 = rng.standard_normal(7), rng.standard_normal(7)
        g = dbyd1_dt0(x, b1, b2, ibc)
        o = O.dbyd1_dt0(x, b1, b2, ibc)
        assert rel(g, o) < 1e-13, ibc


@pytest.mark.parametrize("lphys,rphys", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("order", [1, 2])
def test_compact_lines_all_closures(lphys, rphys, order, gpu_available):
    rng = np.random.default_rng(11)
    n, nl = 32, 9
    x = np.sin(np.linspace(0, 3, n))[None, :] + 0.1 * rng.standard_normal((nl, n))
    hl, hh = rng.standard_normal((nl, 4)), rng.standard_normal((nl, 4))
    for bdry in range(5):
        bl, bh = rng.standard_normal(nl), rng.standard_normal(nl)
        g = compact_lines(x, order, lphys, rphys, bdry, bl, bh, hl, hh, dnum=31.0, scale=31.0 ** order)
        o = O.compact_lines(x, order, lphys, rphys, bdry, bl, bh, hl, hh, dnum=31.0, scale=31.0 ** order)
        assert rel(g, o) < 1e-13, (bdry, rel(g, o))


@pytest.mark.parametrize("n,nl", [(248, 37), (249, 5), (300, 20)])
def test_compact_lines_both_kernels(n, nl, gpu_available):
    """Lines up to 248 points run the shared-memory tiled kernel (16 lines
    per CTA, a partial last CTA here), longer ones the one-thread-per-line
    kernel; both against the oracle."""
    rng = np.random.default_rng(n)
    x = np.cos(np.linspace(0, 4, n))[None, :] + 0.1 * rng.standard_normal((nl, n))
    hl, hh = rng.standard_normal((nl, 4)), rng.standard_normal((nl, 4))
    for order in (1, 2):
        for lphys, rphys in ((True, False), (False, True), (False, False)):
            bl, bh = rng.standard_normal(nl), rng.standard_normal(nl)
            g = compact_lines(x, order, lphys, rphys, 2, bl, bh, hl, hh, dnum=7.0, scale=7.0 ** order)
            o = O.compact_lines(x, order, lphys, rphys, 2, bl, bh, hl, hh, dnum=7.0, scale=7.0 ** order)
            assert rel(g, o) < 1e-13, (order, lphys, rphys, rel(g, o))


@pytest.mark.parametrize("decomp,dims", [((2, 2, 4), (64, 64, 128)), ((3, 2, 3), (60, 64, 96)),
                                         ((2, 4, 3), (48, 80, 60))])
def test_deriv_parity_all_directions(decomp, dims, gpu_available):
    p, prof, v0, dt, _ = problem.build(dims, decomp=decomp)
    sim, orc = Simulation(p, prof), O.Oracle(p, prof)
    rng = np.random.default_rng(5)
    f = v0[4] + 1e-3 * rng.standard_normal(v0[4].shape)
    for direction in (0, 1, 2):
        face = (p.nth * p.nphi) if direction == 0 else (p.nphi * p.nr)
        for order in (1, 2):
            for bdry in (range(5) if direction < 2 else [0]):
                lo, hi = rng.standard_normal(face), rng.standard_normal(face)
                g = sim.deriv(direction, order, f, lo, hi, bdry)
                o = orc.deriv(direction, order, f, lo, hi, bdry)
                assert rel(g, o) < 1e-12, (direction, order, bdry, rel(g, o))


def test_rhs_parity_hydro(cfg1, sims):
    p, prof, v0, dt = cfg1
    sim, orc = sims
    rng = np.random.default_rng(9)
    v = v0.copy()
    v[1:4] = 1e-2 * rng.standard_normal(v[1:4].shape)  # exercise every advection term
    for call in (1, 2):
        _, dg = sim.rhs(v, call)
        _, do = orc.rhs(v, call)
        errs = fieldwise(dg, do)
        assert max(errs) < 1e-12, errs
    _, dg = sim.rhs(v0, 1)  # at rest: cancellation-limited momentum residual
    _, do = orc.rhs(v0, 1)
    errs = fieldwise(dg, do)
    assert max(errs) < 1e-11, errs


def test_sld_parity_hydro(cfg1, sims):
    p, prof, v0, dt = cfg1
    sim, orc = sims
    rng = np.random.default_rng(10)
    v = v0.copy()
    v[1:4] = 1e-2 * rng.standard_normal(v[1:4].shape)
    vg, dg = sim.diffusion(v)
    vo, do = orc.diffusion(v)
    assert np.array_equal(vg, vo)  # mean state subtracted in place, as the reference does
    errs = fieldwise(dg, do)
    assert max(errs) < 1e-12, errs


def test_step_parity_hydro_100_steps(cfg1, sims):
    """Config-1 workload: 100 RK4 steps at fixed CFL-0.4 dt from identical
    seeded state; FP64 GPU state within 1e-10 of the oracle."""
    p, prof, v0, dt = cfg1
    sim, orc = sims
    g1 = sim.step_host(v0, dt, 1)
    o1 = orc.step(v0, dt, 1)
    assert max(fieldwise(g1, o1)) < 1e-11, fieldwise(g1, o1)
    g = sim.step_host(v0, dt, 100)
    o = orc.step(v0, dt, 100)
    errs = fieldwise(g, o)
    assert max(errs) < 1e-10, errs
    assert np.isfinite(g).all()


@pytest.fixture(scope="module")
def mhd(gpu_available):
    p, prof, v0, dt, _ = problem.build((40, 40, 60), magnetic=True, decomp=(2, 2, 3), n_rho=3.0)
    rng = np.random.default_rng(21)
    v0 = v0.copy()
    v0[1:4] = 1e-2 * rng.standard_normal(v0[1:4].shape)
    return p, prof, v0, dt, Simulation(p, prof), O.Oracle(p, prof)


def test_mhd_curl_rhs_sld_parity(mhd):
    p, prof, v0, dt, sim, orc = mhd
    vg, dg = sim.rhs(v0, 1)
    vo, do = orc.rhs(v0, 1)
    assert max(fieldwise(vg[5:], vo[5:])) < 1e-12  # B = curl A handed back in slots 5..7
    errs = fieldwise(dg, do)
    assert max(errs) < 1e-12, errs
    _, dg2 = sim.rhs(v0, 3)
    _, do2 = orc.rhs(v0, 3)
    assert max(fieldwise(dg2, do2)) < 1e-12
    vb = vo.copy()
    sg = sim.diffusion(vb, v0[5:])[1]
    so = orc.diffusion(vb, v0[5:])[1]
    errs = fieldwise(sg, so)
    assert max(errs) < 1e-12, errs


def test_mhd_step_parity(mhd):
    p, prof, v0, dt, sim, orc = mhd
    g = sim.step_host(v0, dt, 10)
    o = orc.step(v0, dt, 10)
    errs = fieldwise(g, o)
    assert max(errs) < 1e-10, errs


def test_nan_is_reported(cfg1, sims):
    from css_b200._lib import CssError
    p, prof, v0, dt = cfg1
    sim, _ = sims
    v = v0.copy()
    v[4, 5, 7, 9] = np.nan
    with pytest.raises(CssError) as e:
        sim.step_host(v, dt, 1)
    assert e.value.code == 4


@pytest.mark.parametrize("dims,decomp", [((24, 512, 48), (2, 2, 4)), ((24, 32, 768), (2, 2, 3))])
def test_maximum_block_length_parity(dims, decomp, gpu_available):
    """256-point blocks (the reference's LOOP COUNT MAX of the line loops,
    the largest block the library accepts) in theta and in phi: the generic
    (run-time length) kernels, against the oracle."""
    p, prof, v0, dt, _ = problem.build(dims, decomp=decomp)
    sim, orc = Simulation(p, prof), O.Oracle(p, prof)
    rng = np.random.default_rng(21)
    v = v0.copy()
    v[1:4] = 1e-2 * rng.standard_normal(v[1:4].shape)
    _, dg = sim.rhs(v, 1)
    _, do = orc.rhs(v, 1)
    assert max(fieldwise(dg, do)) < 1e-12, fieldwise(dg, do)
    _, dg = sim.diffusion(v)
    _, do = orc.diffusion(v)
    assert max(fieldwise(dg, do)) < 1e-12, fieldwise(dg, do)
    g = sim.step_host(v, dt, 2)
    o = orc.step(v, dt, 2)
    assert max(fieldwise(g, o)) < 1e-11, fieldwise(g, o)


def test_empty_line_batches(gpu_available):
    x = np.zeros((0, 40))
    assert compact_lines(x, 1, True, True, 1).shape == (0, 40)
    assert dbyd1_dt0(x, np.zeros(0), np.zeros(0), 1).shape == (0, 40)


def test_mhd_step_parity_100_steps_32cubed_blocks(gpu_available):
    """MHD on 32^3 virtual blocks, the block shape of the 256x512x1024 MHD
    workload (its compile-time 32-point kernels), at 64x64x128 with
    decomposition 2x2x4, 5 density scale heights and the default walls:
    100 FP64 RK4 steps from the workload's own kind of initial state
    (entropy perturbation, random tapered vector potential) within 1e-10 of
    the oracle in every field."""
    p, prof, v0, dt, _ = problem.build((64, 64, 128), magnetic=True, decomp=(2, 2, 4), n_rho=5.0)
    sim, orc = Simulation(p, prof), O.Oracle(p, prof)
    g1 = sim.step_host(v0, dt, 1)
    o1 = orc.step(v0, dt, 1)
    assert max(fieldwise(g1, o1)) < 1e-11, fieldwise(g1, o1)
    g = sim.step_host(v0, dt, 100)
    o = orc.step(v0, dt, 100)
    errs = fieldwise(g, o)
    sim.close()
    orc.close()
    assert np.isfinite(g).all()
    assert max(errs) < 1e-10, errs


def test_hydro_bench_workload_one_step_parity(gpu_available):
    """The hydro bench workload itself (128x256x512, 4x8x16 blocks): one
    FP64 RK4 step against the oracle within 1e-11 in every field."""
    p, prof, v0, dt, _ = problem.build("hydro-128x256x512")
    sim = Simulation(p, prof)
    g = sim.step_host(v0, dt, 1)
    sim.close()
    orc = O.Oracle(p, prof)
    o = orc.step(v0, dt, 1)
    orc.close()
    errs = fieldwise(g, o)
    assert max(errs) < 1e-11, errs


def test_mhd_bench_workload_two_stage_forms_agree(gpu_available):
    """The MHD bench workload itself (256x512x1024, 8x16x32 blocks of 32^3,
    1.3e8 cells; the oracle is too slow at this size): two FP64 RK4 steps of
    the two-pass stage (with the TMA curl) against the four-kernel stage
    (with the tile curl kernels), independent kernels for every part of the
    step, within 1e-12 in every field, compared plane by plane."""
    p, prof, v0, dt, _ = problem.build("mhd-256x512x1024")
    rng = np.random.default_rng(12)
    v0[1:4] = 1e-2 * rng.standard_normal(v0[1:4].shape)  # a flow, so no field is a near-zero residual
    fused, four = Simulation(p, prof), Simulation(p, prof)
    assert fused.fused
    four.set_fused(False)
    four.set_curl_pass(0)
    for sim in (fused, four):
        sim.upload(v0)
        sim.step_rk4(dt, 2)
    del v0
    worst = 0.0
    for iv in range(8):
        dmax = amax = 0.0
        for ir in range(p.nr):
            a, b = fused.plane(iv, ir), four.plane(iv, ir)
            dmax = max(dmax, float(np.abs(a - b).max()))
            amax = max(amax, float(np.abs(b).max()))
        worst = max(worst, dmax / amax)
        assert dmax <= 1e-12 * amax, (iv, dmax / amax)
    print("two-pass against four-kernel stage, 2 steps, worst field:", worst)
    fused.close()
    four.close()
