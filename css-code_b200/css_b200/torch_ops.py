"""PyTorch operators for the compact derivatives.

``torch.ops.css.deriv`` is the whole-field compact derivative of
``css_deriv_dev`` (Dbydr / Dbydt / Dbydp and D2bydr2 / D2bydt2 / D2bydp2,
derivatives.f90:547-1684) on CUDA tensors of shape (..., nr, nphi, nth): every
virtual block solved with its own closures, enqueued on PyTorch's current
stream, the result in a new tensor of the input's dtype.  FP64 tensors are
used as they are; FP32 tensors are computed in FP64 and the result rounded
back.  Only a CUDA kernel is registered, so CPU tensors raise.  The
``dbydr`` ... ``d2bydp2`` functions below name the six reference routines.
The op is differentiable in x: its backward is ``torch.ops.css.deriv_adjoint``
(the transpose of the blocked operator, css_deriv_adjoint_dev); boundary
data are treated as constants.

Like the reference, the r derivatives of a non-uniform grid are returned in
x-space (the caller multiplies by dxdr).  ``bdry`` is the reference's ibc
0..4 (its ``var <= 0`` form, derivatives.f90:558-562); ``bc_lo`` / ``bc_hi``
are the 1-deep boundary data at the physical faces, one face array
(r: (nphi, nth); theta: (nr, nphi)) shared by every leading index or one per
leading index.
"""
import ctypes
from typing import Optional

import torch

from . import _lib
from ._lib import check

_FACE = {0: lambda s: (s[-2], s[-1]), 1: lambda s: (s[-3], s[-2])}


def _vp(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


@torch.library.custom_op("css::deriv", mutates_args=(), device_types="cuda")
def deriv(x: torch.Tensor, ctx: int, direction: int, order: int, bc_lo: Optional[torch.Tensor],
          bc_hi: Optional[torch.Tensor], bdry: int) -> torch.Tensor:
    if direction not in (0, 1, 2) or order not in (1, 2):
        raise ValueError("css::deriv: direction 0..2 and order 1..2")
    if x.dim() < 3:
        raise ValueError("css::deriv: x must have shape (..., nr, nphi, nth)")
    xd = x.to(torch.float64).contiguous()
    out = torch.empty_like(xd)
    lead = xd.shape[:-3]
    nb = 1
    for d in lead:
        nb *= d
    xs, os_ = xd.reshape(nb, *xd.shape[-3:]), out.view(nb, *xd.shape[-3:])
    faces = []
    for bc in (bc_lo, bc_hi):
        if bc is None or direction == 2:
            faces.append(None)
            continue
        f = bc.to(device=xd.device, dtype=torch.float64).contiguous()
        fs = _FACE[direction](xd.shape)
        if f.shape == fs:
            faces.append(f.expand(nb, *fs))
        else:
            faces.append(f.reshape(nb, *fs))
    stream = ctypes.c_void_p(torch.cuda.current_stream(xd.device).cuda_stream)
    h = ctypes.c_void_p(ctx)
    for k in range(nb):
        lo = None if faces[0] is None else faces[0][k]
        hi = None if faces[1] is None else faces[1][k]
        check(_lib.lib().css_deriv_dev(h, int(direction), int(order), _vp(xs[k]), _vp(os_[k]), _vp(lo), _vp(hi),
                                       int(bdry), stream))
    return out.to(x.dtype)


@deriv.register_fake
def _(x, ctx, direction, order, bc_lo, bc_hi, bdry):
    return torch.empty_like(x)


@torch.library.custom_op("css::deriv_adjoint", mutates_args=(), device_types="cuda")
def deriv_adjoint(g: torch.Tensor, ctx: int, direction: int, order: int, bdry: int) -> torch.Tensor:
    """D^T g for the blocked compact derivative D of css::deriv (zero
    boundary data): css_deriv_adjoint_dev on every leading index."""
    gd = g.to(torch.float64).contiguous()
    out = torch.empty_like(gd)
    nb = 1
    for d in gd.shape[:-3]:
        nb *= d
    gs, os_ = gd.reshape(nb, *gd.shape[-3:]), out.view(nb, *gd.shape[-3:])
    stream = ctypes.c_void_p(torch.cuda.current_stream(gd.device).cuda_stream)
    h = ctypes.c_void_p(ctx)
    for k in range(nb):
        check(_lib.lib().css_deriv_adjoint_dev(h, int(direction), int(order), _vp(gs[k]), _vp(os_[k]), int(bdry),
                                               stream))
    return out.to(g.dtype)


@deriv_adjoint.register_fake
def _(g, ctx, direction, order, bdry):
    return torch.empty_like(g)


def _deriv_setup(ctx, inputs, output):
    x, c, direction, order, bc_lo, bc_hi, bdry = inputs
    ctx.args = (c, direction, order, bdry)


def _deriv_backward(ctx, grad):
    # the derivative is affine in x (the boundary data add a constant), so
    # its gradient is the adjoint; the boundary data are held fixed
    c, direction, order, bdry = ctx.args
    return torch.ops.css.deriv_adjoint(grad, c, direction, order, bdry), None, None, None, None, None, None


deriv.register_autograd(_deriv_backward, setup_context=_deriv_setup)


def _op(direction, order):
    def f(x, sim, bc_lo=None, bc_hi=None, bdry=1):
        return torch.ops.css.deriv(x, sim.h.value, direction, order, bc_lo, bc_hi, int(bdry))
    return f


dbydr = _op(0, 1)    # Dbydr, derivatives.f90:547
d2bydr2 = _op(0, 2)  # D2bydr2, :799
dbydt = _op(1, 1)    # Dbydt, :1010
d2bydt2 = _op(1, 2)  # D2bydt2, :1265
dbydp = _op(2, 1)    # Dbydp, :1480
d2bydp2 = _op(2, 2)  # D2bydp2, :1594
for _f, _name in ((dbydr, "dbydr"), (d2bydr2, "d2bydr2"), (dbydt, "dbydt"), (d2bydt2, "d2bydt2"),
                  (dbydp, "dbydp"), (d2bydp2, "d2bydp2")):
    _f.__name__ = _name
    _f.__doc__ = ("%s of a (..., nr, nphi, nth) CUDA tensor on the grid and blocks of `sim` "
                  "(a Simulation): torch.ops.css.deriv" % _name)
