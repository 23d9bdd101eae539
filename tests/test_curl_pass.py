"""B = curl A of magnetic runs: the theta and phi parts from TMA-staged
planes (k_curl_pl, the default on the two-pass stage's state buffers) and
in one pass over the A tiles (k_curl_tp, equal theta and phi blocks of 16
or 32) give the same state, bit for bit, as the separate theta and phi
passes -- in FP64 and mixed precision, on 32- and 16-point
blocks, after RK4 steps that form B at every stage (and for the ohmic
heating of the SLD)."""
import numpy as np
import pytest

from css_b200 import problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims,decomp", [((64, 64, 128), (2, 2, 4)), ((32, 32, 64), (2, 2, 4))])
@pytest.mark.parametrize("precision", [0, 1])
def test_one_pass_curl_is_bit_identical(gpu_available, dims, decomp, precision):
    from css_b200.context import Simulation
    p, prof, v0, dt, _ = problem.build(dims, magnetic=True, decomp=decomp)
    p.precision = precision
    rng = np.random.default_rng(1)
    v = v0.copy()
    v[1:4] = 1e-3 * rng.standard_normal(v[1:4].shape)
    out = []
    for mode in (2, 1, 0):
        sim = Simulation(p, prof)
        sim.set_curl_pass(mode)
        sim.upload(v)
        sim.step_rk4(dt, 3)
        out.append(sim.download())
        sim.close()
    assert np.isfinite(out[0]).all()
    assert np.array_equal(out[0], out[2]) and np.array_equal(out[1], out[2])
