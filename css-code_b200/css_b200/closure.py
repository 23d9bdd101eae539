"""The learned subgrid closure.

The reference closes its equations with slope-limited diffusion whose speed
follows a prescribed radial profile (Initialize_Diffusion,
diffusion.f90:19-63).  Here that profile can be replaced per cell by the
prediction of a small network trained on a resolved (fine) run:

1. ``dataset``: the fine state is box-filtered by ``factor`` in every
   direction into coarse fields and the twelve subgrid targets (stresses,
   entropy fluxes, EMFs: filtered products minus products of filtered
   fields); the features are the 3x3x3 coarse neighbourhoods of u_theta,
   u_phi, u_r, |B| and ds'/dr (135 values, BF16), the targets are scaled by
   their RMS.
2. ``Closure.fit``: Adam on the mean squared error of an MLP
   135 -> 128 -> 128 -> 128 -> 12 (GELU; BF16 weights, FP32 accumulate).
3. ``Closure.attach``: on a coarse run, the predicted subgrid velocity
   variance tau_tt + tau_pp + tau_rr becomes each cell's SLD speed^2; where
   the prediction is not finite the prescribed profile stays (SLD is the
   fallback and stays the operator that carries the closure).

Device buffers come from torch tensors; every computation is the library's.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check

NQ, NTARGET, XPAD, YPAD = 5, 12, 144, 16


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def dataset(fine_sim, factor=4):
    """Coarse fields, targets, features and scaled targets of a fine run."""
    import torch
    p = fine_sim.p
    nct, ncp, ncr = p.nth // factor, p.nphi // factor, p.nr // factor
    nc = nct * ncp * ncr
    dev = torch.device("cuda")
    fields = torch.empty(7 * nc, dtype=torch.float64, device=dev)
    targets = torch.empty(NTARGET * nc, dtype=torch.float64, device=dev)
    check(_lib.lib().css_box_filter(fine_sim.h, int(factor), _ptr(fields), _ptr(targets)))
    sc = (ctypes.c_float * (NQ + NTARGET))()
    check(_lib.lib().css_closure_scales(nct, ncp, ncr, _ptr(fields), _ptr(targets), sc))
    scales = np.array(sc[:], dtype=np.float32)
    return build_inputs(fields, (nct, ncp, ncr), scales[:NQ], targets, scales[NQ:])


def build_inputs(fields, dims, qscale, targets=None, tscale=None):
    """Features (and scaled targets) from coarse fields on the device."""
    import torch
    nct, ncp, ncr = dims
    nc = nct * ncp * ncr
    dev = fields.device
    qs = torch.tensor(np.asarray(qscale, dtype=np.float32), device=dev)
    x = torch.empty(nc * XPAD, dtype=torch.bfloat16, device=dev)
    check(_lib.lib().css_closure_features(nct, ncp, ncr, _ptr(fields), _ptr(qs), _ptr(x)))
    out = {"dims": dims, "nc": nc, "fields": fields, "x": x, "qscale": np.asarray(qscale, dtype=np.float32)}
    if targets is not None:
        ts = torch.tensor(np.asarray(tscale, dtype=np.float32), device=dev)
        tn = torch.empty(nc * YPAD, dtype=torch.float32, device=dev)
        check(_lib.lib().css_closure_targets(nc, _ptr(targets), _ptr(ts), _ptr(tn)))
        out.update({"targets": targets, "t": tn, "tscale": np.asarray(tscale, dtype=np.float32)})
    return out


class Mlp:
    """css_mlp: the closure network on the device."""

    def __init__(self, n_in=135, width=128, n_out=12, max_rows=65536, seed=0):
        h = ctypes.c_void_p()
        check(_lib.lib().css_mlp_create(n_in, width, n_out, max_rows, seed, ctypes.byref(h)))
        self.h = h
        d = (ctypes.c_int * 5)()
        check(_lib.lib().css_mlp_dims(self.h, d))
        self.dims = tuple(d)
        self.max_rows = max_rows
        self.n_out = n_out

    def forward(self, x, n):
        import torch
        y = torch.empty(n * self.dims[4], dtype=torch.float32, device=x.device)
        check(_lib.lib().css_mlp_forward(self.h, _ptr(x), n, _ptr(y)))
        return y

    def train_step(self, x, t, n, lr):
        loss = ctypes.c_float()
        check(_lib.lib().css_mlp_train_step(self.h, _ptr(x), _ptr(t), n, float(lr), ctypes.byref(loss)))
        return loss.value

    def set_fused(self, on=True):
        """Fused one-kernel forward (default) or the per-layer GEMM path."""
        check(_lib.lib().css_mlp_set_fused(self.h, 1 if on else 0))

    def set_stream(self, stream_handle):
        check(_lib.lib().css_mlp_set_stream(self.h, stream_handle))

    def params(self, layer):
        k, m = self.dims[layer], self.dims[layer + 1]
        w = np.zeros((k, m), dtype=np.float32)
        b = np.zeros(m, dtype=np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        check(_lib.lib().css_mlp_params(self.h, layer, w.ctypes.data_as(fp), b.ctypes.data_as(fp), 0))
        return w, b

    def set_params(self, layer, w, b):
        fp = ctypes.POINTER(ctypes.c_float)
        w = np.ascontiguousarray(w, dtype=np.float32)
        b = np.ascontiguousarray(b, dtype=np.float32)
        check(_lib.lib().css_mlp_params(self.h, layer, w.ctypes.data_as(fp), b.ctypes.data_as(fp), 1))

    def grads(self, layer):
        k, m = self.dims[layer], self.dims[layer + 1]
        gw = np.zeros((k, m), dtype=np.float32)
        gb = np.zeros(m, dtype=np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        check(_lib.lib().css_mlp_grads(self.h, layer, gw.ctypes.data_as(fp), gb.ctypes.data_as(fp)))
        return gw, gb

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().css_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Closure:
    """The trained network plus the scales it was trained with."""

    def __init__(self, width=128, seed=0, max_rows=65536):
        self.net = Mlp(135, width, NTARGET, max_rows, seed)
        self.qscale = None
        self.tscale = None

    def fit(self, data, steps=200, batch=16384, lr=1e-3, seed=0):
        """Adam over random row batches of one dataset; returns the losses."""
        import torch
        self.qscale, self.tscale = data["qscale"], data["tscale"]
        nc = data["nc"]
        x = data["x"].view(nc, XPAD)
        t = data["t"].view(nc, YPAD)
        g = torch.Generator(device="cpu").manual_seed(seed)
        losses = []
        batch = min(batch, nc, self.net.max_rows)
        for _ in range(steps):
            idx = torch.randperm(nc, generator=g)[:batch].to(x.device)
            xb = x.index_select(0, idx).contiguous()
            tb = t.index_select(0, idx).contiguous()
            losses.append(self.net.train_step(xb, tb, batch, lr))
        return losses

    def predict(self, data):
        return self.net.forward(data["x"], data["nc"])

    def speed2(self, data):
        """Per-cell SLD speed^2 of the coarse cells of ``data`` (device FP64)."""
        import torch
        y = self.predict(data)
        ts = torch.tensor(self.tscale, device=y.device)
        s2 = torch.empty(data["nc"], dtype=torch.float64, device=y.device)
        check(_lib.lib().css_closure_speed2(data["nc"], _ptr(y), _ptr(ts), _ptr(s2)))
        return s2

    @staticmethod
    def attach(coarse_sim, speed2):
        """Use speed2 (device, one value per coarse cell; None to detach) as the
        coarse run's SLD speed^2.  Keep speed2 alive while the run steps."""
        check(_lib.lib().css_set_sld_speed2(coarse_sim.h, None if speed2 is None else _ptr(speed2)))
        coarse_sim._speed2 = speed2
