"""torch.ops.css.deriv, the PyTorch face of the compact derivatives.

CPU: the operator is registered with a CUDA kernel only, so a CPU tensor
raises rather than falling back.  GPU: every direction and order equals the
host-array entry point (css_deriv) bit for bit, on PyTorch's current stream
and on a side stream; leading dimensions are independent fields; FP32
tensors come back as the FP64 result rounded; the boundary data reach the
closures."""
import numpy as np
import pytest
import torch

from css_b200 import problem
from css_b200 import torch_ops as T


def test_operator_has_no_cpu_kernel():
    x = torch.zeros(4, 4, 4, dtype=torch.float64)
    with pytest.raises(NotImplementedError):
        torch.ops.css.deriv(x, 0, 0, 1, None, None, 1)


@pytest.fixture(scope="module")
def field(gpu_available):
    from css_b200.context import Simulation
    p, prof, v0, dt, _ = problem.build((48, 48, 64), decomp=(2, 2, 4))
    rng = np.random.default_rng(17)
    f = v0[4] + 1e-3 * rng.standard_normal(v0[4].shape)
    return p, Simulation(p, prof), f, rng


OPS = [(0, 1, T.dbydr), (0, 2, T.d2bydr2), (1, 1, T.dbydt), (1, 2, T.d2bydt2), (2, 1, T.dbydp), (2, 2, T.d2bydp2)]


@pytest.mark.gpu
@pytest.mark.parametrize("direction,order,op", OPS)
def test_operator_equals_host_entry(field, direction, order, op):
    p, sim, f, rng = field
    lo = hi = None
    if direction < 2:
        shape = (p.nphi, p.nth) if direction == 0 else (p.nr, p.nphi)
        lo, hi = rng.standard_normal(shape), rng.standard_normal(shape)
    bdry = 4
    want = sim.deriv(direction, order, f, None if lo is None else lo.reshape(-1), None if hi is None else hi.reshape(-1),
                     bdry)
    x = torch.from_numpy(f).cuda()
    tl = None if lo is None else torch.from_numpy(lo).cuda()
    th = None if hi is None else torch.from_numpy(hi).cuda()
    got = op(x, sim, tl, th, bdry)
    assert got.dtype == torch.float64 and got.shape == x.shape
    assert np.array_equal(got.cpu().numpy(), want)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        got2 = op(x, sim, tl, th, bdry)
    torch.cuda.current_stream().wait_stream(side)
    assert torch.equal(got2, got)


@pytest.mark.gpu
def test_leading_dims_fp32_and_wall_data(field):
    p, sim, f, rng = field
    x = torch.from_numpy(np.stack([f, 2.0 * f + 1.0])).cuda()
    both = T.dbydt(x, sim, bdry=1)
    for k in range(2):
        assert torch.equal(both[k], T.dbydt(x[k].contiguous(), sim, bdry=1))
    x32 = x.to(torch.float32)
    g32 = T.dbydr(x32, sim, bdry=1)
    assert g32.dtype == torch.float32
    assert torch.equal(g32, T.dbydr(x32.to(torch.float64), sim, bdry=1).to(torch.float32))
    # a Neumann datum at the theta walls changes the answer; bdry 1 ignores it
    lo = torch.full((p.nr, p.nphi), 3.0, dtype=torch.float64, device="cuda")
    assert torch.equal(T.dbydt(x[0], sim, lo, lo, 1), T.dbydt(x[0], sim, None, None, 1))
    assert not torch.equal(T.dbydt(x[0], sim, lo, lo, 4), T.dbydt(x[0], sim, None, None, 4))


@pytest.mark.gpu
def test_reference_named_entry_points_take_var(field):
    """css_dbydr ... css_d2bydp2: var >= 1 picks the field's boundary
    variant from ibcr / ibct (derivatives.f90:558-562), var <= 0 is bdry =
    -var; the result equals css_deriv with that bdry, bit for bit."""
    import ctypes
    from css_b200 import _lib
    from css_b200._lib import CssError, check
    p, sim, f, rng = field
    x = np.ascontiguousarray(f)
    face_r, face_t = (p.nphi, p.nth), (p.nr, p.nphi)
    lo_r, hi_r = rng.standard_normal(face_r), rng.standard_normal(face_r)
    lo_t, hi_t = rng.standard_normal(face_t), rng.standard_normal(face_t)
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    L = _lib.lib()
    # the run's BC integers for field 2 (w) and 5 (s) under the default flags:
    # stress-free r faces (lbcr_v 4), constant-temperature top (lbcr_s 2),
    # theta walls lbct_w 1, lbct_s 0
    cases = [("css_dbydr", 0, 1, 2, 4, lo_r, hi_r), ("css_d2bydr2", 0, 2, 5, 2, lo_r, hi_r),
             ("css_dbydt", 1, 1, 2, 1, lo_t, hi_t), ("css_d2bydt2", 1, 2, 5, 0, lo_t, hi_t),
             ("css_dbydr", 0, 1, -3, 3, lo_r, hi_r), ("css_dbydt", 1, 1, 0, 0, lo_t, hi_t)]
    for name, d, order, var, bdry, lo, hi in cases:
        out = np.zeros_like(x)
        check(getattr(L, name)(sim.h, dp(x), dp(out), dp(np.ascontiguousarray(lo)), dp(np.ascontiguousarray(hi)), var))
        want = sim.deriv(d, order, x, lo.reshape(-1), hi.reshape(-1), bdry)
        assert np.array_equal(out, want), (name, var)
    for name, d, order in (("css_dbydp", 2, 1), ("css_d2bydp2", 2, 2)):
        out = np.zeros_like(x)
        check(getattr(L, name)(sim.h, dp(x), dp(out), 7))
        assert np.array_equal(out, sim.deriv(d, order, x, None, None, 1)), name
    out = np.zeros_like(x)
    with pytest.raises(CssError):
        check(L.css_dbydr(sim.h, dp(x), dp(out), None, None, 13))


@pytest.mark.gpu
@pytest.mark.parametrize("direction", [0, 1, 2])
@pytest.mark.parametrize("order", [1, 2])
def test_deriv_adjoint_dot_product(direction, order, gpu_available):
    """<D x, y> = <x, D^T y> for the blocked operator of every direction,
    order and boundary condition (the backward of torch.ops.css.deriv)."""
    import torch
    from css_b200 import problem, torch_ops  # noqa: F401
    from css_b200.context import Simulation
    p, prof, v0, dt, _ = problem.build((40, 40, 60), decomp=(2, 2, 3))
    sim = Simulation(p, prof)
    g = torch.Generator().manual_seed(direction * 10 + order)
    x = torch.randn(2, p.nr, p.nphi, p.nth, generator=g, dtype=torch.float64).cuda()
    y = torch.randn(2, p.nr, p.nphi, p.nth, generator=g, dtype=torch.float64).cuda()
    for bdry in (range(5) if direction < 2 else [0]):
        dx = torch.ops.css.deriv(x, sim.h.value, direction, order, None, None, bdry)
        aty = torch.ops.css.deriv_adjoint(y, sim.h.value, direction, order, bdry)
        lhs, rhs = float((dx * y).sum()), float((x * aty).sum())
        scale = float((dx.abs() * y.abs()).sum())
        assert abs(lhs - rhs) <= 1e-13 * scale, (bdry, lhs, rhs)
    sim.close()


@pytest.mark.gpu
def test_deriv_gradcheck(gpu_available):
    """torch.autograd.gradcheck (fast mode: random projections against
    finite differences) through torch.ops.css.deriv."""
    import torch
    from css_b200 import problem, torch_ops  # noqa: F401
    from css_b200.context import Simulation
    p, prof, v0, dt, _ = problem.build((40, 40, 60), decomp=(2, 2, 3))
    sim = Simulation(p, prof)
    x = torch.randn(p.nr, p.nphi, p.nth, dtype=torch.float64, device="cuda", requires_grad=True)
    for direction in (0, 1, 2):
        f = lambda t: torch.ops.css.deriv(t, sim.h.value, direction, 1, None, None, 1)
        assert torch.autograd.gradcheck(f, (x,), fast_mode=True, eps=1e-6, atol=1e-5, rtol=1e-4)
    sim.close()
