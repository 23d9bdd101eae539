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

    COUPLINGS = ("variance", "shaped")

    def speed2(self, data, coupling="variance", sim=None):
        """Per-cell SLD speed^2 of the coarse cells of ``data`` (device FP64).

        ``variance``: the predicted subgrid variance tau_tt + tau_pp + tau_rr
        itself (css_closure_speed2).  ``shaped``: the prescribed speed^2 of
        each radius times the prediction over its shell mean
        (css_closure_speed2_shaped; needs the coarse run ``sim``): the
        prescribed level per shell, placed by the network."""
        import torch
        y = self.predict(data)
        ts = torch.tensor(self.tscale, device=y.device)
        s2 = torch.empty(data["nc"], dtype=torch.float64, device=y.device)
        if coupling == "variance":
            check(_lib.lib().css_closure_speed2(data["nc"], _ptr(y), _ptr(ts), _ptr(s2)))
        elif coupling == "shaped":
            if sim is None:
                raise ValueError("the shaped coupling needs the coarse run")
            check(_lib.lib().css_closure_speed2_shaped(sim.h, _ptr(y), _ptr(ts), _ptr(s2)))
        else:
            raise ValueError("coupling %r (one of %s)" % (coupling, ", ".join(self.COUPLINGS)))
        return s2

    @staticmethod
    def attach(coarse_sim, speed2):
        """Use speed2 (device, one value per coarse cell; None to detach) as the
        coarse run's SLD speed^2.  Keep speed2 alive while the run steps."""
        check(_lib.lib().css_set_sld_speed2(coarse_sim.h, None if speed2 is None else _ptr(speed2)))
        coarse_sim._speed2 = speed2


# ---------------------------------------------------------------------------
# Evaluation: the closure against the prescribed profile, both measured against the
# filtered fine run
# ---------------------------------------------------------------------------
def restrict(fine_sim, coarse_sim, factor, fine_base=None, coarse_base=None):
    """Coarse state := coarse_base + the factor^3 box average of (fine state -
    fine_base) (css_restrict_state; bases are device tensors of each grid's
    state layout, None for zero)."""
    import torch
    torch.cuda.synchronize()
    check(_lib.lib().css_restrict_state(fine_sim.h, None if fine_base is None else _ptr(fine_base), int(factor),
                                        coarse_sim.h, None if coarse_base is None else _ptr(coarse_base)))


def prolong_add(coarse_sim, coarse_base, factor, fine_sim):
    """Fine state += trilinear interpolation of (coarse state - coarse_base)
    (css_prolong_add; coarse_base a device tensor of the state's layout or None)."""
    import torch
    torch.cuda.synchronize()
    check(_lib.lib().css_prolong_add(coarse_sim.h, None if coarse_base is None else _ptr(coarse_base),
                                     int(factor), fine_sim.h))


def statistics(sim, rhor):
    """The statistics a run is compared on, from its resident state: the kinetic-energy
    spectrum in azimuthal wavenumber m, E_K(m) = sum over r, theta and the
    three components of rhor(r) |u_hat(m)|^2 / 2, the magnetic one
    E_M(m) = sum |B_hat(m)|^2 / (8 pi) (B = curl A), and the enthalpy- and
    kinetic-energy-flux profiles (Shell_Average codes 16 and 17,
    report_mpi.f90:949-960).  u and B come from the library (a factor-1
    css_box_filter); the transforms and sums are torch's."""
    import torch
    p = sim.p
    nc = p.nr * p.nth * p.nphi
    fields = torch.empty(7 * nc, dtype=torch.float64, device="cuda")
    targ = torch.empty(NTARGET * nc, dtype=torch.float64, device="cuda")
    check(_lib.lib().css_box_filter(sim.h, 1, _ptr(fields), _ptr(targ)))
    f = fields.view(7, p.nr, p.nphi, p.nth)
    w = torch.as_tensor(np.asarray(rhor, dtype=np.float64), device="cuda")[None, :, None, None]

    def spec(q, weight):
        h = torch.fft.rfft(q, dim=2) / p.nphi
        e = (weight * h.abs() ** 2).sum(dim=(0, 1, 3))
        e[1:] *= 2.0  # m and -m
        return e.cpu().numpy()

    out = {"E_K": spec(f[0:3], 0.5 * w)}
    if p.magnetic:
        out["E_M"] = spec(f[4:7], 1.0 / (8.0 * np.pi))
    fl = sim.shell_averages([16, 17])
    out["F_en"], out["F_ke"] = fl[0], fl[1]
    return out


def rel_err(a, b, lo=0):
    return float(np.linalg.norm(a[lo:] - b[lo:]) / max(np.linalg.norm(b[lo:]), 1e-300))


def _mean_stats(samples):
    return {k: np.mean([s[k] for s in samples], axis=0) for k in samples[0]}


def study(fine, coarse, factor=4, n_pre=0, n_adjust=0, n_train=200, nsnap=4, n_win=200, nstat=4,
          train_steps=400, batch=16384, refresh=20, couplings=("variance", "shaped"), seed=4, cfl=0.4):
    """A posteriori evaluation of the closure on a fine run.

    ``fine`` and ``coarse`` are (params, profiles, vars0, dt, background) of
    the two grids (coarse = fine / factor in every direction; background =
    problem.background of that grid).  States move between the grids as
    perturbations about each grid's background.  Steps, in this order:

    1. optional pre-spin: ``n_pre`` coarse steps from the coarse seeded
       state, the developed coarse perturbation then added to the fine
       seeded state (css_prolong_add) -- a fine run that starts developed;
    2. ``n_adjust`` fine steps;
    3. ``n_train`` fine steps, box-filtered ``nsnap`` times: the training set;
       the network is trained on it (``train_steps`` Adam steps);
    4. the window: every coarse run starts from the filtered fine state at
       its start (css_restrict_state) and covers the physical time of
       ``n_win`` fine steps, sampled ``nstat`` times at the same times as
       the fine run, whose filtered state gets the same diagnostics
       (statistics()) on a coarse probe run.

    The coarse runs are the prescribed profile and one per coupling of the
    closure (Closure.speed2), the closure's speed^2 recomputed from the
    run's own state every ``refresh`` coarse steps.  Returns the
    time-averaged statistics of each run, their relative errors against the
    filtered fine run (spectra over m >= 1), the state error of each run at
    the end of the window against the filtered fine state (per field,
    relative to how far the filtered fine state moved in the window), and
    the wall times of the fine and coarse windows (stepping only).  Time
    steps are the given ones, lowered where the state's Courant limit at
    ``cfl`` (css_step_size) is below them: in chunks of 500 during the
    pre-spin, for the fine run after the pre-spin and the adjustment, for
    the coarse runs at the start of the window."""
    import time
    import torch
    from .context import Simulation
    from .params import PROF_NAMES
    fp, fprof, fv0, fdt, fbg = fine
    cp, cprof, cv0, cdt, cbg = coarse
    dims = (cp.nth, cp.nphi, cp.nr)
    nc = cp.nr * cp.nth * cp.nphi
    rhor = np.asarray(cprof).reshape(len(PROF_NAMES), cp.nr)[PROF_NAMES.index("rhor")]

    def timed_steps(sim, dt, n):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim.step_rk4(dt, n)
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    cbase = torch.from_numpy(np.ascontiguousarray(cbg, dtype=np.float64)).cuda()
    fbase = torch.from_numpy(np.ascontiguousarray(fbg, dtype=np.float64)).cuda()
    fsim = Simulation(fp, fprof)
    fsim.upload(fv0)
    pre_s = 0.0
    if n_pre > 0:
        pre = Simulation(cp, cprof)
        pre.upload(cv0)
        n = n_pre
        while n > 0:  # the developing flow tightens the Courant limit: dt follows it
            k = min(500, n)
            pre_s += timed_steps(pre, min(cdt, pre.step_size(cfl)["dtmax"]), k)
            n -= k
        prolong_add(pre, cbase, factor, fsim)
        pre.close()
    fdt = min(fdt, fsim.step_size(cfl)["dtmax"])
    if n_adjust > 0:
        fsim.step_rk4(fdt, n_adjust)
        fdt = min(fdt, fsim.step_size(cfl)["dtmax"])
    every = max(1, n_train // max(1, nsnap))
    snaps = []
    for _ in range(nsnap):
        fsim.step_rk4(fdt, every)
        snaps.append(dataset(fsim, factor))
    x = torch.cat([d["x"].view(d["nc"], XPAD) for d in snaps]).contiguous()
    t = torch.cat([d["t"].view(d["nc"], YPAD) for d in snaps]).contiguous()
    data = dict(snaps[-1])
    data.update({"x": x.view(-1), "t": t.view(-1), "nc": x.shape[0]})
    clo = Closure(seed=seed, max_rows=batch)
    losses = clo.fit(data, steps=train_steps, batch=batch, lr=2e-3, seed=seed)
    del x, t, data, snaps

    # the window: coarse runs from the filtered fine state at its start
    runs = {"prescribed": None}
    runs.update({c: c for c in couplings})
    sims = {}
    for name in runs:
        sims[name] = Simulation(cp, cprof)
        restrict(fsim, sims[name], factor, fbase, cbase)
    probe = Simulation(cp, cprof)
    restrict(fsim, probe, factor, fbase, cbase)
    start = probe.download()
    cdt = min(cdt, probe.step_size(cfl)["dtmax"])
    fstats, fine_s = [], 0.0
    fev = max(1, n_win // max(1, nstat))
    for _ in range(nstat):
        fine_s += timed_steps(fsim, fdt, fev)
        restrict(fsim, probe, factor, fbase, cbase)
        fstats.append(statistics(probe, rhor))
    fine_end = probe.download()
    t_win = fev * nstat * fdt
    ncs = nstat * int(np.ceil(t_win / (nstat * cdt)))  # coarse steps, a multiple of nstat
    cdt_run = t_win / ncs
    fields = torch.empty(7 * nc, dtype=torch.float64, device="cuda")
    targ = torch.empty(NTARGET * nc, dtype=torch.float64, device="cuda")
    out = {"fine": _mean_stats(fstats)}
    walls, end_err = {}, {}
    scale = [max(np.abs(fine_end[i] - start[i]).max(), 1e-300) for i in range(fine_end.shape[0])]
    for name, coupling in runs.items():
        sim = sims[name]
        stats, wall = [], 0.0
        for _ in range(nstat):
            n = ncs // nstat
            while n > 0:
                if coupling is not None:  # the closure's speed^2 from this run's own state
                    check(_lib.lib().css_box_filter(sim.h, 1, _ptr(fields), _ptr(targ)))
                    Closure.attach(sim, clo.speed2(build_inputs(fields, dims, clo.qscale), coupling, sim))
                k = min(refresh, n)
                wall += timed_steps(sim, cdt_run, k)
                n -= k
            stats.append(statistics(sim, rhor))
        out[name] = _mean_stats(stats)
        walls[name] = wall
        v = sim.download()
        end_err[name] = [float(np.abs(v[i] - fine_end[i]).max() / scale[i]) for i in range(v.shape[0])]
        Closure.attach(sim, None)
        sim.close()
    probe.close()
    fsim.close()
    errs = {}
    for name in runs:
        e = {"E_K": rel_err(out[name]["E_K"], out["fine"]["E_K"], 1),
             "F_en": rel_err(out[name]["F_en"], out["fine"]["F_en"]),
             "F_ke": rel_err(out[name]["F_ke"], out["fine"]["F_ke"])}
        if "E_M" in out["fine"]:
            e["E_M"] = rel_err(out[name]["E_M"], out["fine"]["E_M"], 1)
        errs[name] = e
    return {"errors": errs, "end_state_error": end_err, "stats": out, "fine_window_s": fine_s,
            "coarse_window_s": walls, "pre_spin_s": pre_s,
            "wall_ratio": {k: fine_s / max(w, 1e-12) for k, w in walls.items()},
            "loss_first": float(np.mean(losses[:10])), "loss_last": float(np.mean(losses[-10:])),
            "fine_steps": fev * nstat, "coarse_steps": ncs, "coarse_dt": cdt_run, "fine_dt": fdt, "t_window": t_win,
            "n_pre": n_pre, "n_adjust": n_adjust, "n_train": every * nsnap, "nsnap": nsnap, "nstat": nstat}
