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

    FORWARD_MODES = {"gemm": 0, "mma": 1, "tcgen05": 2}

    def set_fused(self, on=True):
        """Fused one-kernel forward on the tcgen05 tensor cores (default) or
        the per-layer GEMM path."""
        check(_lib.lib().css_mlp_set_fused(self.h, 2 if on else 0))

    def set_forward(self, mode):
        """Forward path: "tcgen05" (fused, 5th-generation tensor cores with
        tensor-memory accumulators; the default), "mma" (fused, BF16
        mma.sync) or "gemm" (one product kernel per layer)."""
        check(_lib.lib().css_mlp_set_fused(self.h, self.FORWARD_MODES[mode]))

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


# ---------------------------------------------------------------------------
# Evaluation: the closure against the prescribed profile, both judged by the
# filtered fine run
# ---------------------------------------------------------------------------
def coarse_statistics(u_t, u_p, u_r, s_pert, rhor, tr):
    """Statistics a coarse run is judged by, from (nr, nphi, nth) fields:
    the kinetic-energy spectrum in azimuthal wavenumber m summed over r and
    theta, E(m) = sum rhor |u_hat(m)|^2 over the three components, and the
    enthalpy-flux profile F(r) = rhor T ⟨u_r s'⟩ over theta and phi (the
    entropy form of rho c_p ⟨u_r T'⟩ about an adiabatic background)."""
    E = 0.0
    for u in (u_t, u_p, u_r):
        uh = np.fft.rfft(u, axis=1) / u.shape[1]
        E = E + (rhor[:, None, None] * np.abs(uh) ** 2).sum(axis=(0, 2))
    F = rhor * tr * (u_r * s_pert).mean(axis=(1, 2))
    return E, F


def rel_err(a, b, lo=0):
    return float(np.linalg.norm(a[lo:] - b[lo:]) / max(np.linalg.norm(b[lo:]), 1e-300))


def study(fine, coarse, factor=4, t_spin=10.0, t_win=2.0, nsnap=20, train_steps=400, refresh=20, seed=4):
    """Trains a closure on a fine run and compares two coarse runs with it.

    ``fine`` and ``coarse`` are (params, profiles, vars0, dt) of the two grids
    (coarse = fine / factor in every direction).  The fine run is spun up for
    t_spin time units, then over t_win it is box-filtered ``nsnap`` times:
    the snapshots are the training set and their statistics (time-averaged
    E(m) and F(r), see coarse_statistics) the reference.  Two coarse runs from
    the coarse seeded state then cover the same physical time: one with the
    prescribed SLD profile, one whose SLD speed^2 is the closure's prediction
    from its own state, refreshed every ``refresh`` steps.  Returns the
    relative errors of both against the filtered fine statistics (E over
    m >= 1, F over r) and the wall times of the fine and coarse windows."""
    import time
    import torch
    from .context import Simulation
    from .params import PROF_NAMES
    fp, fprof, fv0, fdt = fine
    cp, cprof, cv0, cdt = coarse
    cpr = np.asarray(cprof).reshape(len(PROF_NAMES), cp.nr)
    rhor, sr = cpr[PROF_NAMES.index("rhor")], cpr[PROF_NAMES.index("sr")]
    g, cv = cp.gamma, cp.cp / cp.gamma
    tr = (1.0 / (cv * (g - 1.0))) * rhor ** (g - 1.0) * np.exp(sr / cv)
    dims = (cp.nth, cp.nphi, cp.nr)

    fsim = Simulation(fp, fprof)
    fsim.upload(fv0)
    fsim.step_rk4(fdt, int(round(t_spin / fdt)))
    every = max(1, int(round(t_win / fdt)) // nsnap)
    Ef, Ff, snaps = [], [], []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(nsnap):
        fsim.step_rk4(fdt, every)
        d = dataset(fsim, factor)
        f = d["fields"].cpu().numpy().reshape(7, cp.nr, cp.nphi, cp.nth)
        e, fl = coarse_statistics(f[0], f[1], f[2], f[3], rhor, tr)
        Ef.append(e)
        Ff.append(fl)
        snaps.append(d)
    torch.cuda.synchronize()
    fine_wall = time.perf_counter() - t0
    Ef, Ff = np.mean(Ef, axis=0), np.mean(Ff, axis=0)
    x = torch.cat([d["x"].view(d["nc"], XPAD) for d in snaps]).contiguous()
    t = torch.cat([d["t"].view(d["nc"], YPAD) for d in snaps]).contiguous()
    data = dict(snaps[-1])
    data.update({"x": x.view(-1), "t": t.view(-1), "nc": x.shape[0]})
    clo = Closure(seed=seed)
    losses = clo.fit(data, steps=train_steps, batch=16384, lr=2e-3, seed=seed)
    nc = cp.nr * cp.nth * cp.nphi

    def coarse_run(learned):
        sim = Simulation(cp, cprof)
        sim.upload(cv0)
        fields = torch.empty(7 * nc, dtype=torch.float64, device="cuda")
        targ = torch.empty(NTARGET * nc, dtype=torch.float64, device="cuda")

        def advance(n):
            while n > 0:
                if learned:  # the closure's speed^2 from this run's own state
                    check(_lib.lib().css_box_filter(sim.h, 1, _ptr(fields), _ptr(targ)))
                    Closure.attach(sim, clo.speed2(build_inputs(fields, dims, clo.qscale)))
                k = min(refresh, n)
                sim.step_rk4(cdt, k)
                n -= k

        advance(int(round(t_spin / cdt)))
        cev = max(1, int(round(t_win / cdt)) // nsnap)
        E, F = [], []
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for _ in range(nsnap):
            advance(cev)
            v = sim.download()
            e, fl = coarse_statistics(v[1], v[2], v[3], v[4] - sr[:, None, None], rhor, tr)
            E.append(e)
            F.append(fl)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t1
        sim.close()
        return np.mean(E, axis=0), np.mean(F, axis=0), wall

    E0, F0, w0 = coarse_run(False)
    E1, F1, w1 = coarse_run(True)
    fsim.close()
    return {"spectrum_err_prescribed": rel_err(E0, Ef, 1), "spectrum_err_closure": rel_err(E1, Ef, 1),
            "flux_err_prescribed": rel_err(F0, Ff), "flux_err_closure": rel_err(F1, Ff),
            "fine_window_s": fine_wall, "coarse_window_s": w1, "coarse_prescribed_window_s": w0,
            "wall_ratio": fine_wall / max(w1, 1e-12), "loss_first": float(np.mean(losses[:10])),
            "loss_last": float(np.mean(losses[-10:])), "t_spin": t_spin, "t_win": t_win, "nsnap": nsnap,
            "E_fine": Ef, "E_prescribed": E0, "E_closure": E1, "F_fine": Ff, "F_prescribed": F0, "F_closure": F1}
