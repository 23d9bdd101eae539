"""The learned subgrid closure: box filter and subgrid targets, stencil
features, the BF16 MLP (forward, gradients, Adam) and its use as the SLD
speed of a coarse run.

References: numpy statements of the filter, the targets and the features
(FP64, exact to rounding; the BF16 features bit for bit), and a numpy
forward/backward of the network that applies the same BF16 roundings
(activations, weights and the gradients fed to the products).  The
network's tolerances are relative to the largest magnitude of each output:
forward 2e-2 and gradients 5e-2 (a BF16 rounding is 4e-3, and a rounding
that falls differently in the last bit moves one activation by that much)."""
import math

import numpy as np
import pytest

from css_b200 import problem
from css_b200.params import PROF_NAMES

pytestmark = pytest.mark.gpu


def to_bf16(a):
    """Round FP32 values to BF16 (nearest even), returned as FP32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) & 0xFFFF0000).astype(np.uint32).view(np.float32)


C_GELU = math.sqrt(2.0 / math.pi)


def gelu(x):
    """GELU in its tanh form (Hendrycks & Gimpel), as the network uses it."""
    return 0.5 * x * (1.0 + np.tanh(C_GELU * (x + 0.044715 * x ** 3)))


def dgelu(x):
    t = np.tanh(C_GELU * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * C_GELU * (1.0 + 3.0 * 0.044715 * x * x)


def stirred(dims, magnetic, decomp):
    p, prof, v0, dt, _ = problem.build(dims, magnetic=magnetic, decomp=decomp)
    rng = np.random.default_rng(3)
    v = v0.copy()
    v[1:4] = 1e-2 * rng.standard_normal(v[1:4].shape)
    return p, prof, v, dt


def numpy_filter(p, prof, v, b, f):
    nr, nphi, nth = p.nr, p.nphi, p.nth
    sr = np.asarray(prof).reshape(len(PROF_NAMES), nr)[PROF_NAMES.index("sr")]
    box = lambda a: a.reshape(nr // f, f, nphi // f, f, nth // f, f).mean(axis=(1, 3, 5))
    ut, up, ur = v[1], v[2], v[3]
    sp = v[4] - sr[:, None, None]
    bt, bp, br = b
    fl = [box(q) for q in (ut, up, ur, sp, bt, bp, br)]
    m = lambda a, c: box(a * c)
    t = [m(ut, ut) - fl[0] * fl[0], m(ut, up) - fl[0] * fl[1], m(ut, ur) - fl[0] * fl[2],
         m(up, up) - fl[1] * fl[1], m(up, ur) - fl[1] * fl[2], m(ur, ur) - fl[2] * fl[2],
         m(ut, sp) - fl[0] * fl[3], m(up, sp) - fl[1] * fl[3], m(ur, sp) - fl[2] * fl[3],
         box(up * br - ur * bp) - (fl[1] * fl[6] - fl[2] * fl[5]),
         box(ur * bt - ut * br) - (fl[2] * fl[4] - fl[0] * fl[6]),
         box(ut * bp - up * bt) - (fl[0] * fl[5] - fl[1] * fl[4])]
    return np.stack(fl), np.stack(t)


def numpy_features(F, qscale):
    """F: (7, ncr, ncp, nct) coarse fields -> (nc, 144) features as FP32 of BF16."""
    ncr, ncp, nct = F.shape[1:]
    q = np.empty((5, ncr, ncp, nct))
    q[0:3] = F[0:3]
    q[3] = np.sqrt(F[4] ** 2 + F[5] ** 2 + F[6] ** 2)
    lo = np.maximum(np.arange(ncr) - 1, 0)
    hi = np.minimum(np.arange(ncr) + 1, ncr - 1)
    q[4] = (F[3][hi] - F[3][lo]) / (hi - lo)[:, None, None]
    cols = []
    for dr in (-1, 0, 1):
        jr = np.clip(np.arange(ncr) + dr, 0, ncr - 1)
        for dt in (-1, 0, 1):
            jt = np.clip(np.arange(nct) + dt, 0, nct - 1)
            for dp in (-1, 0, 1):
                jp = (np.arange(ncp) + dp) % ncp
                for k in range(5):
                    a = q[k][jr][:, jp][:, :, jt] / np.float64(qscale[k])
                    cols.append(to_bf16(a.astype(np.float32)).reshape(-1))
    x = np.stack(cols, axis=1)
    return np.concatenate([x, np.zeros((x.shape[0], 9), np.float32)], axis=1)


def test_box_filter_targets_and_features_match_numpy(gpu_available):
    import torch
    from css_b200 import closure as C
    from css_b200.context import Simulation
    from oracle import oracle as O
    p, prof, v, dt = stirred((48, 64, 128), True, (2, 2, 4))
    sim = Simulation(p, prof)
    sim.upload(v)
    data = C.dataset(sim, 4)
    ncr, ncp, nct = p.nr // 4, p.nphi // 4, p.nth // 4
    b = O.Oracle(p, prof).curl_b(v[5:8])
    F, T = numpy_filter(p, prof, v, b, 4)
    gf = data["fields"].cpu().numpy().reshape(7, ncr, ncp, nct)
    gt = data["targets"].cpu().numpy().reshape(12, ncr, ncp, nct)
    for k in range(7):
        assert np.abs(gf[k] - F[k]).max() <= 1e-10 * max(np.abs(F[k]).max(), 1e-300), k
    for k in range(12):
        assert np.abs(gt[k] - T[k]).max() <= 1e-9 * max(np.abs(T[k]).max(), 1e-300), k
    x = data["x"].view(-1, 144).float().cpu().numpy()
    xr = numpy_features(gf, data["qscale"])
    assert np.array_equal(x, xr)
    assert np.all(np.isfinite(data["t"].cpu().numpy()))


def numpy_net(mlp, x, t, nreal):
    """Forward and gradients with the device's BF16 roundings; x, t FP32."""
    Ws, Bs = zip(*[mlp.params(l) for l in range(4)])
    Wb = [to_bf16(w).astype(np.float64) for w in Ws]
    h, Z, H = x.astype(np.float64), [], [x.astype(np.float64)]
    for l in range(4):
        z = (h @ Wb[l] + Bs[l]).astype(np.float32).astype(np.float64)
        Z.append(z)
        if l < 3:
            h = to_bf16(gelu(z).astype(np.float32)).astype(np.float64)
            H.append(h)
    y = Z[3]
    n = x.shape[0]
    d = np.zeros_like(y)
    d[:, :nreal] = y[:, :nreal] - t[:, :nreal]
    dz = 2.0 * d / (n * nreal)
    grads = [None] * 4
    for l in (3, 2, 1, 0):
        dzb = to_bf16(dz.astype(np.float32)).astype(np.float64)
        grads[l] = (H[l].T @ dzb, dz.sum(axis=0))
        if l > 0:
            dh = dzb @ Wb[l].T
            dz = dh * dgelu(Z[l - 1])
    loss = float((d ** 2).sum() / (n * nreal))
    return y, grads, loss


def test_mlp_forward_and_gradients_match_numpy(gpu_available):
    import torch
    from css_b200 import closure as C
    rng = np.random.default_rng(0)
    n = 4096
    net = C.Mlp(135, 128, 12, max_rows=8192, seed=5)
    x = np.zeros((n, 144), np.float32)
    x[:, :135] = to_bf16(rng.standard_normal((n, 135)).astype(np.float32))
    t = np.zeros((n, 16), np.float32)
    t[:, :12] = rng.standard_normal((n, 12))
    xd = torch.from_numpy(x).to(torch.bfloat16).cuda()
    td = torch.from_numpy(t).cuda()
    y = net.forward(xd, n).cpu().numpy().reshape(n, 16)  # fused kernel, tcgen05 (the default)
    net.set_forward("mma")
    ym = net.forward(xd, n).cpu().numpy().reshape(n, 16)  # fused kernel, mma.sync
    net.set_forward("gemm")
    yg = net.forward(xd, n).cpu().numpy().reshape(n, 16)  # per-layer GEMMs
    net.set_forward("tcgen05")
    yr, grads, loss = numpy_net(net, x, t, 12)
    for out in (y, ym, yg):
        assert np.abs(out - yr).max() <= 2e-2 * np.abs(yr).max()
        assert np.abs(out[:, 12:]).max() == 0.0
    # the two fused kernels differ only in FP32 summation order (and the BF16
    # roundings of hidden activations that order can flip)
    assert np.abs(y - ym).max() <= 2e-2 * np.abs(ym).max()
    assert np.median(np.abs(y - ym)) <= 1e-4 * np.abs(ym).max()
    # a ragged row count takes the partial last tile of the fused kernel
    y7 = net.forward(xd[:4093].contiguous(), 4093).cpu().numpy().reshape(4093, 16)
    assert np.abs(y7 - y[:4093]).max() <= 1e-6 * np.abs(y).max()
    gloss = net.train_step(xd, td, n, 0.0)  # lr 0: gradients only
    assert abs(gloss - loss) <= 2e-2 * loss
    for l in range(4):
        gw, gb = net.grads(l)
        rw, rb = grads[l]
        assert np.abs(gw - rw).max() <= 5e-2 * np.abs(rw).max(), l
        assert np.abs(gb - rb).max() <= 5e-2 * np.abs(rb).max(), l


def test_mlp_learns_a_smooth_map(gpu_available):
    import torch
    from css_b200 import closure as C
    rng = np.random.default_rng(1)
    n = 16384
    a = rng.standard_normal((135, 12)) / math.sqrt(135.0)
    x = np.zeros((n, 144), np.float32)
    x[:, :135] = to_bf16(rng.standard_normal((n, 135)).astype(np.float32))
    t = np.zeros((n, 16), np.float32)
    t[:, :12] = np.tanh(x[:, :135] @ a)
    net = C.Mlp(135, 128, 12, max_rows=n, seed=2)
    xd = torch.from_numpy(x).to(torch.bfloat16).cuda()
    td = torch.from_numpy(t).cuda()
    losses = [net.train_step(xd, td, n, 3e-3) for _ in range(300)]
    assert losses[-1] < 0.1 * losses[0], (losses[0], losses[-1])


def test_closure_drives_a_coarse_run(gpu_available):
    import torch
    from css_b200 import closure as C
    from css_b200.context import Simulation
    # resolved run 96x128x256 -> 4x box filter -> training data on 24x32x64
    p, prof, v, dt = stirred((96, 128, 256), False, (3, 4, 8))
    fine = Simulation(p, prof)
    fine.upload(v)
    fine.step_rk4(dt, 5)
    data = C.dataset(fine, 4)
    clo = C.Closure(seed=4)
    losses = clo.fit(data, steps=150, batch=4096, lr=2e-3)
    assert np.isfinite(losses).all() and np.mean(losses[-10:]) < np.mean(losses[:10])
    # the coarse run: its own state, features of its own fields (a factor-1
    # filter is the identity), the learned speed^2 in place of the profile
    pc, profc, vc, dtc = stirred((24, 32, 64), False, (2, 2, 4))
    coarse = Simulation(pc, profc)
    coarse.upload(vc)
    nc = pc.nr * pc.nth * pc.nphi
    fields = torch.empty(7 * nc, dtype=torch.float64, device="cuda")
    tt = torch.empty(12 * nc, dtype=torch.float64, device="cuda")
    from css_b200 import _lib
    _lib.check(_lib.lib().css_box_filter(coarse.h, 1, C._ptr(fields), C._ptr(tt)))
    cdata = C.build_inputs(fields, (pc.nth, pc.nphi, pc.nr), clo.qscale)
    s2 = clo.speed2(cdata)
    assert torch.isfinite(s2).all() and (s2 >= 0).all()
    C.Closure.attach(coarse, s2)
    coarse.step_rk4(dtc, 3)
    with_closure = coarse.download()
    assert np.isfinite(with_closure).all()
    # detached, the prescribed profile returns: the same as a run that never had it
    C.Closure.attach(coarse, None)
    coarse.upload(vc)
    coarse.step_rk4(dtc, 3)
    ref = Simulation(pc, profc)
    ref.upload(vc)
    ref.step_rk4(dtc, 3)
    assert np.array_equal(coarse.download(), ref.download())
    assert not np.array_equal(with_closure, ref.download())


def test_study_reports_what_the_closure_gains(gpu_available):
    """The evaluation of closure.study on a short window: a 96x128x256 fine
    run filtered 4x onto 24x32x64 trains the network; coarse runs with the
    prescribed profile and with the learned speed^2 are compared with the
    filtered fine statistics.  The test shows the two errors side by side
    (printed) and checks what holds at any length of run: the statistics are
    finite, the learned speed^2 changes the coarse run, training lowers the
    loss, and the coarse window costs a fraction of the fine one."""
    from css_b200 import closure as C
    fp, fprof, fv0, fdt, _ = problem.build((96, 128, 256), decomp=(3, 4, 8))
    cp, cprof, cv0, cdt, _ = problem.build((24, 32, 64), decomp=(2, 2, 4))
    r = C.study((fp, fprof, fv0, fdt), (cp, cprof, cv0, cdt), t_spin=0.5, t_win=0.2, nsnap=4, train_steps=100)
    print({k: r[k] for k in ("spectrum_err_prescribed", "spectrum_err_closure", "flux_err_prescribed",
                             "flux_err_closure", "wall_ratio")})
    for k in ("spectrum_err_prescribed", "spectrum_err_closure", "flux_err_prescribed", "flux_err_closure"):
        assert np.isfinite(r[k])
    assert not np.allclose(r["E_prescribed"], r["E_closure"], rtol=1e-9, atol=0)
    assert r["loss_last"] < r["loss_first"]
    assert r["fine_window_s"] > r["coarse_window_s"]
