"""ctypes binding of the CPU oracle (liboracle.so).  TEST INFRASTRUCTURE
ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline arm, never by the product package.

The oracle is a C restatement of the reference Fortran hot path; see
css_oracle.h for what each entry point restates.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.orc_create.argtypes = [ctypes.c_void_p, _dp, ctypes.POINTER(ctypes.c_void_p)]
        L.orc_create.restype = ctypes.c_int
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_deriv.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_int]
        L.orc_rhs.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_int]
        L.orc_diffusion.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        L.orc_step_rk4.argtypes = [ctypes.c_void_p, _dp, ctypes.c_double, ctypes.c_int]
        L.orc_dbyd1_dt0.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_curl_b.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.orc_compact_lines.argtypes = [_dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_double,
                                        ctypes.c_double]
        L.orc_scalars.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.orc_step_size.argtypes = [ctypes.c_void_p, _dp, ctypes.c_double, _dp]
        L.orc_shell_averages.argtypes = [ctypes.c_void_p, _dp, ctypes.POINTER(ctypes.c_int), ctypes.c_int, _dp, _dp]
        L.orc_spectrum.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int, _dp]
        L.orc_bound.argtypes = [ctypes.c_void_p, _dp]
        L.orc_set_clock.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_double, ctypes.c_double]
        L.orc_get_clock.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong), _dp]
        L.orc_inout_init.argtypes = [ctypes.c_void_p, _dp]
        L.orc_inout_state.argtypes = [ctypes.c_void_p, _dp]
        L.orc_set_rain_fields.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.orc_rain_fields.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.orc_set_ash_slices.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_double]
        L.orc_build_squalls.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp]
        L.orc_add_squalls.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp]
        _ip = ctypes.POINTER(ctypes.c_int)
        L.orc_voronoi.argtypes = [ctypes.c_int, _dp, _dp, _ip, _ip, _ip, _ip, _dp]
        L.orc_build_lanes.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double]
        L.orc_cyclic_lines.argtypes = [_dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        _LIB = L
    return _LIB


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def _check(rc):
    if rc != 0:
        raise RuntimeError("oracle error %d: %s" % (rc, lib().orc_last_error().decode()))


def set_threads(n):
    lib().orc_set_threads(int(n))


def dbyd1_dt0(x, bdat1, bdat2, ibc):
    """Batched Dbyd1_dt0 (derivatives.f90:2296) over the last axis."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    n1 = x.shape[-1]
    lines = x.reshape(-1, n1)
    nl = lines.shape[0]
    out = np.zeros_like(lines)
    b1 = np.ascontiguousarray(np.broadcast_to(np.asarray(bdat1, dtype=np.float64), (nl,)))
    b2 = np.ascontiguousarray(np.broadcast_to(np.asarray(bdat2, dtype=np.float64), (nl,)))
    _check(lib().orc_dbyd1_dt0(_ptr(lines), _ptr(out), _ptr(b1), _ptr(b2), n1, int(ibc), nl))
    return out.reshape(x.shape)


class Oracle:
    """One emulated (nnr x nnt x nnp)-rank run of the reference on the CPU."""

    def __init__(self, params, profiles):
        self.p = params.copy()
        self.prof = np.ascontiguousarray(profiles, dtype=np.float64)
        h = ctypes.c_void_p()
        _check(lib().orc_create(ctypes.byref(self.p), _ptr(self.prof), ctypes.byref(h)))
        self.h = h
        self.nv = 8 if self.p.magnetic else 5
        self.shape = (self.nv, self.p.nr, self.p.nphi, self.p.nth)

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def deriv(self, direction, order, x, bc_lo=None, bc_hi=None, bdry=1):
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.zeros_like(x)
        lo = None if bc_lo is None else np.ascontiguousarray(bc_lo, dtype=np.float64)
        hi = None if bc_hi is None else np.ascontiguousarray(bc_hi, dtype=np.float64)
        _check(lib().orc_deriv(self.h, direction, order, _ptr(x), _ptr(out), _ptr(lo), _ptr(hi), int(bdry)))
        return out

    def rhs(self, vars1, call_num=1):
        v = np.array(vars1, dtype=np.float64, order="C", copy=True)
        dv = np.zeros_like(v)
        _check(lib().orc_rhs(self.h, _ptr(v), _ptr(dv), int(call_num)))
        return v, dv

    def diffusion(self, vars1, avec=None):
        v = np.array(vars1, dtype=np.float64, order="C", copy=True)
        dv = np.zeros_like(v)
        a = None if avec is None else np.ascontiguousarray(avec, dtype=np.float64)
        _check(lib().orc_diffusion(self.h, _ptr(v), _ptr(a), _ptr(dv)))
        return v, dv

    def curl_b(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        b = np.zeros_like(a)
        _check(lib().orc_curl_b(self.h, _ptr(a), _ptr(b)))
        return b

    SCALAR_NAMES = ("kinener", "cke", "mcke", "drke", "umach", "magener", "bmax")
    STEP_SIZE_NAMES = ("dtmax", "Etot", "Ltot", "mtot", "mrsint")

    def scalars(self, vars0):
        v = np.ascontiguousarray(vars0, dtype=np.float64)
        out = np.zeros(7)
        _check(lib().orc_scalars(self.h, _ptr(v), _ptr(out)))
        return dict(zip(self.SCALAR_NAMES, out.tolist()))

    def step_size(self, vars0, cfl_safety):
        v = np.ascontiguousarray(vars0, dtype=np.float64)
        out = np.zeros(5)
        _check(lib().orc_step_size(self.h, _ptr(v), float(cfl_safety), _ptr(out)))
        return dict(zip(self.STEP_SIZE_NAMES, out.tolist()))

    def shell_averages(self, vars0, quantities, k0=None):
        v = np.ascontiguousarray(vars0, dtype=np.float64)
        q = np.ascontiguousarray(quantities, dtype=np.int32)
        out = np.zeros((len(q), self.p.nr))
        k = None if k0 is None else np.ascontiguousarray(k0, dtype=np.float64)
        _check(lib().orc_shell_averages(self.h, _ptr(v), q.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(q),
                                        _ptr(k), _ptr(out)))
        return out

    def spectrum(self, vars0, kind=0):
        v = np.ascontiguousarray(vars0, dtype=np.float64)
        out = np.zeros((self.p.nr, self.p.nphi // 2))
        _check(lib().orc_spectrum(self.h, _ptr(v), int(kind), _ptr(out)))
        return out

    def bound(self, vars1):
        v = np.array(vars1, dtype=np.float64, order="C", copy=True)
        _check(lib().orc_bound(self.h, _ptr(v)))
        return v

    def step(self, vars0, dt, nsteps=1):
        v = np.array(vars0, dtype=np.float64, order="C", copy=True)
        _check(lib().orc_step_rk4(self.h, _ptr(v), float(dt), int(nsteps)))
        return v

    # open radial boundaries (same semantics as the css_* entry points)
    def set_clock(self, istep, sim_time, deltat):
        _check(lib().orc_set_clock(self.h, int(istep), float(sim_time), float(deltat)))

    def clock(self):
        i, t = ctypes.c_longlong(), ctypes.c_double()
        _check(lib().orc_get_clock(self.h, ctypes.byref(i), ctypes.byref(t)))
        return i.value, t.value

    def inout_init(self, vars0):
        _check(lib().orc_inout_init(self.h, _ptr(np.ascontiguousarray(vars0, dtype=np.float64))))

    def inout_state(self):
        out = np.zeros(4)
        _check(lib().orc_inout_state(self.h, _ptr(out)))
        return dict(zip(("m0", "vol", "mtot", "ash_fen_mod"), out.tolist()))

    def set_rain_fields(self, dvel, dent):
        _check(lib().orc_set_rain_fields(self.h, _ptr(np.ascontiguousarray(dvel, dtype=np.float64)),
                                         _ptr(np.ascontiguousarray(dent, dtype=np.float64))))

    def rain_fields(self):
        dvel = np.zeros((self.p.nphi, self.p.nth))
        dent = np.zeros_like(dvel)
        _check(lib().orc_rain_fields(self.h, _ptr(dvel), _ptr(dent)))
        return dvel, dent

    def set_ash_slices(self, slices, times, ash_fen_mod):
        _check(lib().orc_set_ash_slices(self.h, _ptr(np.ascontiguousarray(slices, dtype=np.float64)),
                                        _ptr(np.ascontiguousarray(times, dtype=np.float64)), float(ash_fen_mod)))

    def build_squalls(self, squalls, sstruct=1):
        sq = np.ascontiguousarray(squalls, dtype=np.float64).reshape(-1, 6)
        _check(lib().orc_build_squalls(self.h, int(sstruct), sq.shape[0], _ptr(sq)))

    def add_squalls(self, squalls, sstruct=1):
        sq = np.ascontiguousarray(squalls, dtype=np.float64).reshape(-1, 6)
        _check(lib().orc_add_squalls(self.h, int(sstruct), sq.shape[0], _ptr(sq)))

    def build_lanes(self, cells, meansize, meanvel, meands):
        cl = np.ascontiguousarray(cells, dtype=np.float64).reshape(-1, 3)
        _check(lib().orc_build_lanes(self.h, cl.shape[0], _ptr(cl), float(meansize), float(meanvel), float(meands)))


def compact_lines(x, order=1, lphys=True, rphys=True, bdry=1, bc_lo=None, bc_hi=None,
                  halo_lo=None, halo_hi=None, dnum=1.0, scale=1.0):
    """Independent compact-FD lines with explicit closures (orc_compact_lines)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.shape[-1]
    lines = x.reshape(-1, n)
    nl = lines.shape[0]
    out = np.zeros_like(lines)

    def vec(a, k):
        if a is None:
            return None
        return np.ascontiguousarray(np.broadcast_to(np.asarray(a, dtype=np.float64), (nl, k) if k > 1 else (nl,)))

    _check(lib().orc_compact_lines(_ptr(lines), _ptr(out), n, nl, int(order), int(bool(lphys)), int(bool(rphys)),
                                   int(bdry), _ptr(vec(bc_lo, 1)), _ptr(vec(bc_hi, 1)), _ptr(vec(halo_lo, 4)),
                                   _ptr(vec(halo_hi, 4)), float(dnum), float(scale)))
    return out.reshape(x.shape)


def cyclic_lines(x, order=1, dnum=1.0):
    """Cyclic compact derivative along the last axis (orc_cyclic_lines):
    every line periodic, Sherman-Morrison on the cyclic tridiagonal system."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.shape[-1]
    lines = x.reshape(-1, n)
    out = np.zeros_like(lines)
    _check(lib().orc_cyclic_lines(_ptr(lines), _ptr(out), n, lines.shape[0], int(order), float(dnum)))
    return out.reshape(x.shape)


def dbydp_cyclic(p, field, order=1):
    """The cyclic phi derivative of one field (nr, nphi, nth) of run p, the
    oracle of css_dbydp_cyclic: lines along phi, dnum = 1/dphi."""
    f = np.ascontiguousarray(np.moveaxis(np.asarray(field, dtype=np.float64), 1, 2))  # (nr, nth, nphi)
    dphi = (p.phi2 - p.phi1) / p.nphi
    d = cyclic_lines(f, order, 1.0 / dphi)
    return np.ascontiguousarray(np.moveaxis(d, 2, 1))


def voronoi(x, y):
    """Voronoi cells of sites (x, y) as orc_voronoi / Compute_Voronoi give
    them: (degree, start, face, vxy) with cell g's vertices
    vxy[face[start[g]:start[g] + degree[g]]]."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    n = x.size
    deg, st = np.zeros(n, np.int32), np.zeros(n, np.int32)
    face = np.zeros(6 * n + 32, np.int32)
    vxy = np.zeros((2 * n + 8, 2))
    nv = ctypes.c_int()
    ip = ctypes.POINTER(ctypes.c_int)
    _check(lib().orc_voronoi(n, _ptr(x), _ptr(y), deg.ctypes.data_as(ip), st.ctypes.data_as(ip),
                             face.ctypes.data_as(ip), ctypes.byref(nv), _ptr(vxy)))
    return deg, st, face[:int(deg.sum())], vxy[:nv.value]
