"""Synthetic inputs for the CSS hot path: grid, stratified background and
seeded initial state, generated on the host and handed identically to the
GPU library and to the CPU oracle.

Background: the reference's ``Isentropic`` n = 1.5 polytrope
(Read_Stellar_Model, mhdsph_mpi.f90:317-397) with the number of density
scale heights fixed by ``mstar``.  The non-uniform radial grid is a tanh
stretching of the uniform computational coordinate x in [0, 1] that clusters
points toward the top, supplied (as the reference's generic machinery
expects, rhs_mpi.f90:1278-1284) through r(x), dx/dr and d2x/dr2.

Initial state: rotation-compensated density and a seeded Gaussian entropy
perturbation with the reference's tapers (Initialize_Flow SLaplacian branch,
mhdsph_mpi.f90:711-733).  The reference seeds from the system clock
(mhdsph_mpi.f90:657-658) so its initial states are not reproducible; here a
numpy PCG64 generator with an explicit seed stands in.  MHD: a seeded random
vector potential with the tapers of Initialize_Mag (mhdsph_mpi.f90:1084-1126)
scaled so that B = curl A has the requested rms.
"""
import math

import numpy as np

from .params import NPROF

GCONST = 6.67e-8  # the reference's Gconst (mhdsph_mpi.f90:318)
A_CONST, C_LIGHT = 7.56577e-15, 2.99792458e10  # constants.f90:7


def tanh_grid(nr, r1, r2, stretch=1.0):
    """r(x) = r1 + (r2-r1) tanh(a x)/tanh(a) on x_ind = uniform [0, 1].

    Returns x_ind, r_ind, dr_ind, dxdr, d2xdr2.  dr_ind(1) is the distance to
    the point one cell below, as the reference extrapolates it
    (mhdsph_mpi.f90:332-335)."""
    a = float(stretch)
    x = np.arange(nr, dtype=np.float64) / float(nr - 1)
    ta = math.tanh(a)

    def rof(xx):
        return r1 + (r2 - r1) * np.tanh(a * xx) / ta

    r = rof(x)
    sech2 = 1.0 / np.cosh(a * x) ** 2
    drdx = (r2 - r1) * a * sech2 / ta
    d2rdx2 = (r2 - r1) * a * a * (-2.0 * sech2 * np.tanh(a * x)) / ta
    dxdr = 1.0 / drdx
    d2xdr2 = -d2rdx2 / drdx ** 3
    dr = np.empty(nr)
    dr[0] = r[0] - rof(np.array([x[0] - 1.0 / (nr - 1)]))[0]
    dr[1:] = r[1:] - r[:-1]
    return x, r, dr, dxdr, d2xdr2


def polytrope(p, n_rho, stretch=1.0, kappa=None, ra=1e5, pr=1.0, g0_exp=0.0, delta=1e-3):
    """Isentropic background profiles packed as include/css_b200.h expects
    (profiles[slot*nr + ir]), plus a dict of the scalars used to build them.

    ``n_rho`` density scale heights set mstar through
    rho(r1)/rho0 = (1 + alp (r2/r1 - 1))^(1/(gamma-1)) = exp(n_rho) with
    alp = G mstar / (Cp T0 r2) (mhdsph_mpi.f90:323-325).  The nominal Rayleigh
    number sets kappa = sqrt(g_mid d^3 delta / (Ra Pr)) for a superadiabatic
    entropy contrast delta*Cp, and the bottom luminosity gives the entropy
    gradient -delta*Cp/d through the constant-flux condition."""
    nr = p.nr
    gamma, cp = p.gamma, p.cp
    gamm1 = gamma - 1.0
    cv = cp / gamma
    rho0, t0 = 1.0, p.t0
    r1, r2 = p.r1, p.r2
    x, r, dr, dxdr, d2xdr2 = tanh_grid(nr, r1, r2, stretch)
    alp = (math.exp(n_rho * gamm1) - 1.0) / (r2 / r1 - 1.0)
    mstar = alp * cp * t0 * r2 / GCONST
    r_inv = 1.0 / r
    base = 1.0 + alp * (r2 * r_inv - 1.0)
    rhor = rho0 * base ** (1.0 / gamm1)
    gravity = GCONST * mstar * r_inv ** 2
    tr = t0 * base
    pr2 = gamm1 * cv * rho0 * t0
    sr2 = cv * (math.log(pr2) - gamma * math.log(rho0))
    sr = np.full(nr, sr2)
    d = r2 - r1
    if kappa is None:
        g_mid = GCONST * mstar / (0.5 * (r1 + r2)) ** 2
        kappa = math.sqrt(g_mid * d ** 3 * delta / (ra * pr))
    ks = kappa * rhor * tr * (rhor / rhor[-1]) ** g0_exp
    dlnks = -(gamma + g0_exp) * alp * r2 * r_inv ** 2 / base / gamm1
    eps = np.zeros(nr)
    # viscosity of the explicit-viscosity path (mhdsph_mpi.f90:352-354)
    mur = p.sld_pr * kappa * rhor
    dlnmu = -alp * r2 * r_inv ** 2 / base / gamm1
    lum = delta * cp / d * 4.0 * math.pi * r1 ** 2 * ks[0]
    p.lumr1 = lum
    p.lumr2 = lum
    # radiative diffusion (mhdsph_mpi.f90:365-386): kr carries the luminosity
    # on the background gradient, kr = 1 / [-16 pi a c r^2 T^3 g / (3 rho L)]
    # with g = T (dsdr/Cp - (gamma-1) rho gravity / (gamma P)) = -G mstar /
    # (Cp r^2) for the isentropic polytrope.  The reference differentiates
    # ln of the bracket with Dbyd1_dt0; the polytrope's closed form is used
    # here: d/dr ln[...] = (3 - 1/(gamma-1)) d ln(base)/dr (L constant).
    g_bg = -GCONST * mstar / (cp * r ** 2)
    kr_inv = -16.0 * math.pi * A_CONST * C_LIGHT * r ** 2 * tr ** 3 * g_bg / (3.0 * rhor * lum)
    kr = 1.0 / kr_inv
    dlnkr = (3.0 - 1.0 / gamm1) * (-alp * r2 * r_inv ** 2) / base
    prof = np.stack([x, r, dr, dxdr, d2xdr2, rhor, sr, gravity, ks, dlnks, eps, mur, dlnmu, kr,
                     dlnkr]).astype(np.float64)
    assert prof.shape[0] == NPROF
    info = dict(alp=alp, mstar=mstar, kappa=kappa, rho0=rho0, tr=tr, lum=lum)
    return np.ascontiguousarray(prof.reshape(-1)), info


def angles(p):
    dth = (p.th2 - p.th1) / (p.nth - 1)
    dphi = (p.phi2 - p.phi1) / p.nphi
    theta = dth * np.arange(p.nth) + p.th1
    phi = dphi * np.arange(p.nphi) + p.phi1
    return theta, phi, dth, dphi


def initial_state(p, prof, info, seed=1234, samp=1e-4, vamp=0.0, b_rel=1e-3):
    """Seeded initial state vars(it, ip, ir, iv) as a C-contiguous array of
    shape (nv, nr, nphi, nth) (the Fortran order of the reference)."""
    nr, nth, nphi = p.nr, p.nth, p.nphi
    nv = 8 if p.magnetic else 5
    gamm1 = p.gamma - 1.0
    prof = prof.reshape(NPROF, nr)
    r, rhor, sr = prof[1], prof[5], prof[6]
    theta, phi, _, _ = angles(p)
    rng = np.random.default_rng(seed)
    rand = rng.standard_normal((nr, nphi, nth))
    xv = math.pi * (theta - p.th1) / (p.th2 - p.th1)
    yv = math.pi * (r - p.r1) / (p.r2 - p.r1)
    # radial taper of the perturbation (mhdsph_mpi.f90:679-714): zero at a
    # closed face, left free at an open one (top_inout / bot_inout)
    top_open, bot_open = bool(getattr(p, "top_inout", 0)), bool(getattr(p, "bot_inout", 0))
    if top_open and bot_open:
        rtap = np.ones_like(r)
    elif top_open:
        rtap = 1.0 - np.cos(0.5 * yv) ** 16
    elif bot_open:
        rtap = 1.0 - np.sin(0.5 * yv) ** 16
    else:
        rtap = 1.0 - np.cos(yv) ** 16
    taper = rtap[:, None, None] * (1.0 - np.cos(xv)[None, None, :] ** 16)
    rand = rand * taper
    v = np.zeros((nv, nr, nphi, nth))
    v[0] = _rho_rotating(p, prof, info)[:, None, :]
    v[3] = vamp * rand
    v[4] = (1.0 + samp * rand) * sr[:, None, None]
    if p.magnetic:
        urand = rng.random((3, nr, nphi, nth)) * 2.0 - 1.0
        tap2 = (1.0 - np.cos(yv)[:, None, None] ** 2) * (1.0 - np.cos(xv)[None, None, :] ** 2)
        a = urand * tap2
        rr = (4.0 * (r - p.r1) * (p.r2 - r) / (p.r2 - p.r1) ** 2) ** 6
        tt = (4.0 * (theta - p.th1) * (p.th2 - theta) / (p.th2 - p.th1) ** 2) ** 11
        a[2] = a[2] - rr[:, None, None] * tt[None, None, :] * (p.th2 - p.th1) / 11.0
        # scale: B_rms = b_rel * sqrt(4 pi rho c_s^2) (pressure equipartition)
        b = curl_estimate(p, prof, a)
        brms = math.sqrt(float(np.mean(b ** 2)))
        cs2 = gamm1 * p.cp * info["tr"]
        beq = math.sqrt(float(np.mean(4.0 * math.pi * rhor * cs2)))
        scale = b_rel * beq / brms if brms > 0 else 0.0
        v[5:8] = a * scale
    return np.ascontiguousarray(v)


def _rho_rotating(p, prof, info):
    """Density (nr, nth) of the polytrope in the rotating frame, the density
    of the seeded initial state."""
    prof = prof.reshape(NPROF, p.nr)
    r, rhor = prof[1], prof[5]
    theta = angles(p)[0]
    gamm1 = p.gamma - 1.0
    bv = 0.5 * (p.omega_0 * p.r2) ** 2 / (p.cp * p.t0)
    cvar = (rhor / info["rho0"]) ** gamm1
    rs = (r[:, None] * np.sin(theta)[None, :] / p.r2) ** 2 - 1.0
    return info["rho0"] * (cvar[:, None] + bv * rs) ** (1.0 / gamm1)


def background(p, prof, info):
    """The initial state without its seeds, shape (nv, nr, nphi, nth): the
    rotating polytrope's density, u = 0, s = sr(r), A = 0.  Each grid's
    perturbations are measured from its own background when a state moves
    between resolutions."""
    nv = 8 if p.magnetic else 5
    prof = np.asarray(prof).reshape(NPROF, p.nr)
    v = np.zeros((nv, p.nr, p.nphi, p.nth))
    v[0] = _rho_rotating(p, prof, info)[:, None, :]
    v[4] = prof[6][:, None, None]
    return v


def curl_estimate(p, prof, a):
    """Second-order central-difference curl (amplitude normalisation only)."""
    prof = prof.reshape(NPROF, p.nr)
    r = prof[1]
    theta, phi, dth, dphi = angles(p)
    sth = np.sin(theta)[None, None, :]
    rr = r[:, None, None]
    at, ap, ar = a
    d_th = lambda f: np.gradient(f, dth, axis=2)
    d_ph = lambda f: np.gradient(f, dphi, axis=1)
    d_r = lambda f: np.gradient(f, r, axis=0)
    br = d_th(sth * ap) / (rr * sth) - d_ph(at) / (rr * sth)
    bt = d_ph(ar) / (rr * sth) - d_r(rr * ap) / rr
    bp = d_r(rr * at) / rr - d_th(ar) / rr
    return np.stack([bt, bp, br])


def cfl_dt(p, prof, vars0, bfield=None, cfl=0.4):
    """Fixed time step from Compute_Step_Size (rhs_mpi.f90:92-231): dt =
    cfl * min over cells of dxmin / sqrt(|u|^2 + (gamma-1) Cp xi^2 T [+ vA^2])
    with dxmin = min(dr, r min(dth, sin(theta) dphi))."""
    nr = p.nr
    prof = prof.reshape(NPROF, nr)
    r, dr = prof[1], prof[2]
    theta, _, dth, dphi = angles(p)
    gamm1 = p.gamma - 1.0
    cv = p.cp / p.gamma
    invtconst = (1.0 / cv) / gamm1
    rho, w, v, u, s = vars0[0], vars0[1], vars0[2], vars0[3], vars0[4]
    t = invtconst * rho ** gamm1 * np.exp(s / cv)
    sth = np.sin(theta)
    dxmin = np.minimum(dr[:, None], r[:, None] * np.minimum(dth, sth[None, :] * dphi))[:, None, :]
    ut = u * u + v * v + w * w + gamm1 * p.cp * p.xi_cs * p.xi_cs * t
    dtc = float(np.min(dxmin / np.sqrt(ut)))
    dtb = 1e4
    if p.magnetic and bfield is not None:
        b2 = np.sum(bfield ** 2, axis=0)
        dtb = float(np.min(dxmin / np.sqrt(ut + b2 / (4.0 * math.pi) / rho)))
    return min(dtb, dtc, 1e10) * cfl


# ---------------------------------------------------------------------------
# the five workloads (grid, decomposition, stratification)
# ---------------------------------------------------------------------------
WORKLOADS = {
    # name: (nr, nth, nphi, decomposition (nnr, nnt, nnp), magnetic, n_rho)
    "hydro-64x64x128": (64, 64, 128, (2, 2, 4), False, 3.0),
    "hydro-128x256x512": (128, 256, 512, (4, 8, 16), False, 3.0),
    "mhd-256x512x1024": (256, 512, 1024, (8, 16, 32), True, 5.0),
    "hydro-64x128x256": (64, 128, 256, (2, 4, 8), False, 3.0),
    "hydro-128x128x256": (128, 128, 256, (4, 4, 8), False, 3.0),
    "mhd-128x128x256": (128, 128, 256, (4, 4, 8), True, 5.0),
}


def build(name_or_dims, seed=1234, magnetic=None, decomp=None, n_rho=None, top_inout=False, bot_inout=False):
    """(params, profiles, vars0, dt, info) for a named workload or a
    (nr, nth, nphi) tuple; top_inout / bot_inout open those radial faces
    (and leave the initial perturbation untapered there)."""
    from .params import default_params
    if isinstance(name_or_dims, str):
        nr, nth, nphi, dec, mag, nrho = WORKLOADS[name_or_dims]
    else:
        nr, nth, nphi = name_or_dims
        dec, mag, nrho = (2, 2, 4), False, 3.0
    if magnetic is not None:
        mag = magnetic
    if decomp is not None:
        dec = decomp
    if n_rho is not None:
        nrho = n_rho
    p = default_params(nr, nth, nphi, dec, magnetic=mag)
    p.top_inout, p.bot_inout = int(bool(top_inout)), int(bool(bot_inout))
    if mag:
        p.sld_prm = 0.5  # magnetic Prandtl number 2 through the SLD scaling
    prof, info = polytrope(p, nrho, ra=1e6 if mag else 1e5)
    vars0 = initial_state(p, prof, info, seed=seed)
    bfield = curl_estimate(p, prof, vars0[5:8]) if mag else None
    dt = cfl_dt(p, prof, vars0, bfield)
    return p, prof, vars0, dt, info


def open_from_checkpoint(vars0, bottom=False, top=False, vamp=1.0):
    """startbio / starttio (mhdsph_mpi.f90:956-976): open radial faces of a
    state read from a closed-boundary checkpoint.  On an opened bottom u_r
    becomes vamp times the plane above it, on an opened top vamp times the
    plane below, each less its plane mean; an opened top also takes the
    entropy of the plane below.  Returns a new array (nv, nr, nphi, nth)."""
    v = np.array(vars0, dtype=np.float64, copy=True)
    if bottom:
        v[3, 0] = vamp * v[3, 1]
        v[3, 0] = v[3, 0] - v[3, 0].sum() / v[3, 0].size
    if top:
        v[3, -1] = v[3, -2] * vamp
        v[3, -1] = v[3, -1] - v[3, -1].sum() / v[3, -1].size
        v[4, -1] = v[4, -2]
    return v
