"""Run parameters of the CSS hot path: a ctypes mirror of ``css_params`` in
include/css_b200.h, plus builders for the synthetic workloads.

The field names follow the reference's namelists (mhdsph_mpi.f90:1142-1177,
defaults constants.f90:31-82, diffusion.f90:8-11).
"""
import ctypes

_FIELDS = [
    ("nr", ctypes.c_int), ("nth", ctypes.c_int), ("nphi", ctypes.c_int),
    ("nnr", ctypes.c_int), ("nnt", ctypes.c_int), ("nnp", ctypes.c_int),
    ("magnetic", ctypes.c_int), ("non_uniform", ctypes.c_int),
    ("r1", ctypes.c_double), ("r2", ctypes.c_double),
    ("th1", ctypes.c_double), ("th2", ctypes.c_double),
    ("phi1", ctypes.c_double), ("phi2", ctypes.c_double),
    ("gamma", ctypes.c_double), ("cp", ctypes.c_double), ("omega_0", ctypes.c_double),
    ("t0", ctypes.c_double), ("xi_cs", ctypes.c_double), ("damping_time", ctypes.c_double),
    ("lumr1", ctypes.c_double), ("lumr2", ctypes.c_double),
    ("slaplacian", ctypes.c_int), ("sldiffusion", ctypes.c_int),
    ("top_stress_free", ctypes.c_int), ("bottom_stress_free", ctypes.c_int),
    ("top_constant_temp", ctypes.c_int), ("bottom_constant_temp", ctypes.c_int),
    ("theta_stress_free", ctypes.c_int),
    ("theta_normal_field", ctypes.c_int), ("theta_perf_conductor", ctypes.c_int),
    ("top_radial_field", ctypes.c_int), ("bottom_radial_field", ctypes.c_int),
    ("top_perfect_cond", ctypes.c_int), ("bottom_perfect_cond", ctypes.c_int),
    ("set_stop", ctypes.c_int),
    ("sld_coef", ctypes.c_double), ("sld_speedh", ctypes.c_double), ("sld_speedr", ctypes.c_double),
    ("sld_exp", ctypes.c_double), ("sld_pr", ctypes.c_double), ("sld_prm", ctypes.c_double),
    ("sld_tanh_coef", ctypes.c_double), ("flux_cutoff", ctypes.c_double),
    ("dstype", ctypes.c_int), ("mass_diffusion", ctypes.c_int), ("magnetic_diffusion", ctypes.c_int),
    ("do_viscous_heating", ctypes.c_int), ("do_ohmic_heating", ctypes.c_int),
    ("flux_limiter", ctypes.c_int), ("ent_flux_limiter", ctypes.c_int), ("mag_flux_limiter", ctypes.c_int),
    ("precision", ctypes.c_int),
    ("time_stepper", ctypes.c_int),
    ("laplacian", ctypes.c_int),
    ("do_radheat", ctypes.c_int),
    ("top_inout", ctypes.c_int), ("bot_inout", ctypes.c_int),
    ("bottom_specified", ctypes.c_int), ("do_entropy_rain", ctypes.c_int),
    ("ufreq", ctypes.c_int),
    ("delta_s", ctypes.c_double),
]


class CssParams(ctypes.Structure):
    """ctypes image of ``css_params`` (include/css_b200.h)."""
    _fields_ = _FIELDS

    def nv(self):
        return 8 if self.magnetic else 5

    def copy(self):
        out = CssParams()
        ctypes.memmove(ctypes.byref(out), ctypes.byref(self), ctypes.sizeof(CssParams))
        return out

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in _FIELDS}


NPROF = 15  # CSS_NPROF
PROF_NAMES = ["x_ind", "r_ind", "dr_ind", "dxdr", "d2xdr2", "rhor", "sr", "gravity", "ks", "dlnks", "eps",
              "mur", "dlnmu", "kr", "dlnkr"]


def default_params(nr, nth, nphi, decomp, magnetic=False):
    """Parameters of the synthetic spherical-segment convection runs.

    Boundary choices (Read_Input, mhdsph_mpi.f90:1302-1462): stress-free
    top and bottom, constant temperature on top with thermal damping toward
    T0 (rhs_mpi.f90:1807-1818), constant flux at the bottom, stress-free
    impenetrable theta walls, and for MHD the radial-field / normal-field
    walls.  SLDiffusion on (the only setting whose RK4 weights are right,
    step_rk4.f90:385-388); explicit viscosity (Laplacian) off, entropy
    diffusion (SLaplacian) on.  sld_tanh_coef = 0 makes the speed-profile
    cutoff factor exactly 1/2 everywhere, which sidesteps the reference's
    non-conforming array expression at diffusion.f90:60.
    """
    p = CssParams()
    p.nr, p.nth, p.nphi = nr, nth, nphi
    p.nnr, p.nnt, p.nnp = decomp
    p.magnetic = 1 if magnetic else 0
    p.non_uniform = 1
    p.r1, p.r2 = 0.70, 0.97
    deg = 3.1415926535897932384626433832795028841972 / 180.0
    p.th1, p.th2 = 45.0 * deg, 135.0 * deg
    p.phi1, p.phi2 = 0.0, 90.0 * deg
    p.gamma, p.cp, p.omega_0 = 5.0 / 3.0, 1.0, 1.0
    p.t0 = 1.0
    p.xi_cs = 1.0
    p.damping_time = 0.1
    p.slaplacian, p.sldiffusion = 1, 1
    p.top_stress_free, p.bottom_stress_free = 1, 1
    p.top_constant_temp, p.bottom_constant_temp = 1, 0
    p.theta_stress_free = 1
    p.theta_normal_field, p.theta_perf_conductor = 1, 0
    p.top_radial_field, p.bottom_radial_field = 1, 1
    p.top_perfect_cond, p.bottom_perfect_cond = 0, 0
    p.set_stop = 0
    p.sld_coef, p.sld_speedh, p.sld_speedr, p.sld_exp = 0.5, 0.05, 0.0, -0.5
    p.sld_pr, p.sld_prm = 1.0, 1.0
    p.sld_tanh_coef, p.flux_cutoff = 0.0, 0.0
    p.dstype = 1
    p.mass_diffusion, p.magnetic_diffusion = 1, 1
    p.do_viscous_heating = 1
    p.do_ohmic_heating = 1 if magnetic else 0
    p.flux_limiter = p.ent_flux_limiter = p.mag_flux_limiter = -1
    p.precision = 0
    p.time_stepper = 4
    p.ufreq = 100
    return p
