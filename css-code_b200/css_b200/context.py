"""Host-side mirror of the reference's step / RHS / derivative interfaces on
top of the C ABI.

``Simulation`` plays the role of the Fortran driver's module state
(vars0 of parallel_mpi.f90:41 plus the tables Setup builds): create it from
parameters and radial profiles, upload an initial state, advance it with
``step_rk4`` (Step_RK4, step_rk4.f90:339), or call ``rhs`` (RHS(call_num),
rhs_mpi.f90:279), ``diffusion`` (Compute_Diffusion, diffusion.f90:70) and
``deriv`` (Dbydr/Dbydt/Dbydp and the second derivatives) for one field.
Arrays are numpy float64 of shape (nv, nr, nphi, nth), i.e. the Fortran
vars(it, ip, ir, iv) in memory order.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check, dp


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(dp)


class Simulation:
    def __init__(self, params, profiles):
        self.p = params.copy()
        self.prof = np.ascontiguousarray(profiles, dtype=np.float64)
        self.nv = 8 if self.p.magnetic else 5
        self.shape = (self.nv, self.p.nr, self.p.nphi, self.p.nth)
        h = ctypes.c_void_p()
        check(_lib.lib().css_create(ctypes.byref(self.p), _p(self.prof), ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().css_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # state ----------------------------------------------------------------
    def upload(self, vars0):
        v = np.ascontiguousarray(vars0, dtype=np.float64)
        assert v.shape == self.shape, (v.shape, self.shape)
        check(_lib.lib().css_upload_state(self.h, _p(v)))

    def download(self):
        out = np.empty(self.shape)
        check(_lib.lib().css_download_state(self.h, _p(out)))
        return out

    def step_rk4(self, dt, nsteps=1):
        check(_lib.lib().css_step_rk4(self.h, float(dt), int(nsteps)))

    def step_host(self, vars0, dt, nsteps=1):
        v = np.array(vars0, dtype=np.float64, order="C", copy=True)
        check(_lib.lib().css_step_rk4_host(self.h, _p(v), float(dt), int(nsteps)))
        return v

    def checkpoint_write(self, directory, istep, deltat, sim_time):
        """Write the resident state as a reference-layout checkpoint."""
        check(_lib.lib().css_checkpoint_write(self.h, str(directory).encode(), int(istep), float(deltat),
                                              float(sim_time)))

    def checkpoint_read(self, directory):
        """Replace the state from a reference-layout checkpoint; returns
        (istep, deltat, sim_time)."""
        st, dt, t = ctypes.c_int(), ctypes.c_double(), ctypes.c_double()
        check(_lib.lib().css_checkpoint_read(self.h, str(directory).encode(), ctypes.byref(st), ctypes.byref(dt),
                                             ctypes.byref(t)))
        return st.value, dt.value, t.value

    def sync(self):
        check(_lib.lib().css_sync(self.h))

    def device_state(self):
        """(device pointer, element count) of the resident state."""
        ptr = ctypes.c_void_p()
        n = ctypes.c_longlong()
        check(_lib.lib().css_state_device_ptr(self.h, ctypes.byref(ptr), ctypes.byref(n)))
        return ptr.value, n.value

    def launches(self):
        return _lib.lib().css_kernel_launches(self.h)

    def set_stream(self, stream_handle):
        """Run on the caller's cudaStream_t (int handle, e.g.
        torch.cuda.current_stream().cuda_stream); None = own stream."""
        check(_lib.lib().css_set_stream(self.h, stream_handle))

    def profile(self, enable=True):
        check(_lib.lib().css_profile(self.h, 1 if enable else 0))

    def kernel_stats(self):
        """{kernel name: (total ms, launches)} since profile(True)."""
        out = {}
        for k in range(64):
            nm = ctypes.c_char_p()
            ms = ctypes.c_double()
            cnt = ctypes.c_longlong()
            if _lib.lib().css_kernel_stats(self.h, k, ctypes.byref(nm), ctypes.byref(ms), ctypes.byref(cnt)):
                break  # past the last kernel kind
            if cnt.value:
                out[nm.value.decode()] = (ms.value, cnt.value)
        return out

    def autotune(self, reps=3):
        """Time every tile height of each sweep direction on the resident state
        and keep the fastest (css_autotune); returns (r, theta, phi) lines
        per CTA.  Results are unchanged bit for bit."""
        ch = (ctypes.c_int * 3)()
        check(_lib.lib().css_autotune(self.h, int(reps), ch))
        return tuple(ch)

    def dbydp_cyclic(self, field, order=1):
        """Cyclic phi derivative of one field (nr, nphi, nth): every whole
        phi line periodic, Sherman-Morrison (css_dbydp_cyclic; an extension
        beside the reference's block-closed Dbydp)."""
        f = np.ascontiguousarray(field, dtype=np.float64)
        assert f.shape == self.shape[1:], (f.shape, self.shape)
        out = np.empty_like(f)
        check(_lib.lib().css_dbydp_cyclic(self.h, _p(f), _p(out), int(order)))
        return out

    def set_fused(self, on):
        """Two-pass RK4 stage on or off (css_set_fused); on is refused for a
        run that does not qualify."""
        check(_lib.lib().css_set_fused(self.h, 1 if on else 0))

    def set_curl_pass(self, mode):
        """B = curl A's theta and phi parts (css_set_curl_pass): 2 from
        TMA-staged planes (default), 1 one pass over tiles, 0 two passes
        (True / False as 1 / 0); bit-identical results."""
        check(_lib.lib().css_set_curl_pass(self.h, int(mode)))

    @property
    def fused(self):
        return bool(_lib.lib().css_get_fused(self.h))

    def set_tiles(self, tl_r, tl_theta, tl_phi, phi_persistent=False):
        """The autotuner's choices by hand (css_set_tiles)."""
        check(_lib.lib().css_set_tiles(self.h, int(tl_r), int(tl_theta), int(tl_phi), 1 if phi_persistent else 0))

    # diagnostics of the current state ----------------------------------------
    SCALAR_NAMES = ("kinener", "cke", "mcke", "drke", "umach", "magener", "bmax")
    STEP_SIZE_NAMES = ("dtmax", "Etot", "Ltot", "mtot", "mrsint")

    def scalars(self):
        """Scalar_Output (report_mpi.f90:173-262) of the resident state, as a dict."""
        out = np.zeros(7)
        check(_lib.lib().css_scalars(self.h, _p(out)))
        return dict(zip(self.SCALAR_NAMES, out.tolist()))

    def step_size(self, cfl_safety):
        """Compute_Step_Size (rhs_mpi.f90:92-275): dtmax and the conservation totals."""
        out = np.zeros(5)
        check(_lib.lib().css_step_size(self.h, float(cfl_safety), _p(out)))
        return dict(zip(self.STEP_SIZE_NAMES, out.tolist()))

    def shell_averages(self, quantities, k0=None):
        """Shell_Average_Output (report_mpi.f90:783-1094): array (nq, nr) of the
        horizontal averages of the reference's quantity codes 1..18."""
        q = np.ascontiguousarray(quantities, dtype=np.int32)
        out = np.zeros((len(q), self.p.nr))
        k = None if k0 is None else np.ascontiguousarray(k0, dtype=np.float64)
        check(_lib.lib().css_shell_averages(self.h, q.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(q), _p(k),
                                            _p(out)))
        return out

    def spectrum(self, kind=0):
        """(theta, phi) spectrum per radius, array (nr, nphi/2), folded as
        CSS-IDL/spectral_analysis_new.pro:16-25 folds it (kind 0 kinetic energy
        density, 1 magnetic energy density, 2+iv state variable iv)."""
        out = np.zeros((self.p.nr, self.p.nphi // 2))
        check(_lib.lib().css_spectrum(self.h, int(kind), _p(out)))
        return out

    # parity entry points ----------------------------------------------------
    def rhs(self, vars1, call_num=1):
        v = np.array(vars1, dtype=np.float64, order="C", copy=True)
        dv = np.zeros_like(v)
        check(_lib.lib().css_rhs(self.h, _p(v), _p(dv), int(call_num)))
        return v, dv

    def bound(self, vars1):
        """Bound() on a copy of vars1 (css_bound)."""
        v = np.array(vars1, dtype=np.float64, order="C", copy=True)
        check(_lib.lib().css_bound(self.h, _p(v)))
        return v

    def diffusion(self, vars1, avec=None):
        v = np.array(vars1, dtype=np.float64, order="C", copy=True)
        dv = np.zeros_like(v)
        a = None if avec is None else np.ascontiguousarray(avec, dtype=np.float64)
        check(_lib.lib().css_diffusion(self.h, _p(v), _p(a), _p(dv)))
        return v, dv

    def plane(self, iv, ir):
        """Field iv of the resident state at radius ir, shape (nphi, nth)."""
        out = np.zeros((self.p.nphi, self.p.nth))
        check(_lib.lib().css_download_plane(self.h, int(iv), int(ir), _p(out)))
        return out

    # open radial boundaries (top_inout / bot_inout) ---------------------------
    def set_clock(self, istep, sim_time, deltat):
        """istep: the step index the RHS sees; deltat: the step size of the
        mean-flow terms for ``rhs`` (the step calls set it to their dt)."""
        check(_lib.lib().css_set_clock(self.h, int(istep), float(sim_time), float(deltat)))

    def clock(self):
        i, t = ctypes.c_longlong(), ctypes.c_double()
        check(_lib.lib().css_get_clock(self.h, ctypes.byref(i), ctypes.byref(t)))
        return i.value, t.value

    def inout_init(self):
        """m0, vol and mtot of the resident state, as the start-up computes them."""
        check(_lib.lib().css_inout_init(self.h))

    def inout_state(self):
        out = np.zeros(4)
        check(_lib.lib().css_inout_state(self.h, _p(out)))
        return dict(zip(("m0", "vol", "mtot", "ash_fen_mod"), out.tolist()))

    def set_rain_fields(self, dvel, dent):
        check(_lib.lib().css_set_rain_fields(self.h, _p(np.ascontiguousarray(dvel, dtype=np.float64)),
                                             _p(np.ascontiguousarray(dent, dtype=np.float64))))

    def rain_fields(self):
        dvel = np.zeros((self.p.nphi, self.p.nth))
        dent = np.zeros_like(dvel)
        check(_lib.lib().css_get_rain_fields(self.h, _p(dvel), _p(dent)))
        return dvel, dent

    def build_squalls(self, squalls, sstruct=1):
        """squalls: (nsq, 6) theta_loc, phi_loc, size, scaling, vel, dels;
        sstruct 1 Gaussian, 0 polynomial squalls."""
        sq = np.ascontiguousarray(squalls, dtype=np.float64).reshape(-1, 6)
        check(_lib.lib().css_build_squalls(self.h, int(sstruct), sq.shape[0], _p(sq)))

    def add_squalls(self, squalls, sstruct=1):
        """The same squalls added to the current rain fields (after the lanes)."""
        sq = np.ascontiguousarray(squalls, dtype=np.float64).reshape(-1, 6)
        check(_lib.lib().css_add_squalls(self.h, int(sstruct), sq.shape[0], _p(sq)))

    def build_lanes(self, cells, meansize, meanvel, meands):
        """Downflow lanes (css_build_lanes): cells (n, 3) phi_loc, theta_loc,
        scaling of the convection-cell sites; replaces the rain fields."""
        cl = np.ascontiguousarray(cells, dtype=np.float64).reshape(-1, 3)
        check(_lib.lib().css_build_lanes(self.h, cl.shape[0], _p(cl), float(meansize), float(meanvel), float(meands)))

    def set_ash_slices(self, slices, times, ash_fen_mod):
        """slices: (4 times, 4 fields u_r, u_theta, u_phi, s, nphi, nth)."""
        check(_lib.lib().css_set_ash_slices(self.h, _p(np.ascontiguousarray(slices, dtype=np.float64)),
                                            _p(np.ascontiguousarray(times, dtype=np.float64)), float(ash_fen_mod)))

    def deriv(self, direction, order, x, bc_lo=None, bc_hi=None, bdry=1):
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.zeros_like(x)
        lo = None if bc_lo is None else np.ascontiguousarray(bc_lo, dtype=np.float64)
        hi = None if bc_hi is None else np.ascontiguousarray(bc_hi, dtype=np.float64)
        check(_lib.lib().css_deriv(self.h, int(direction), int(order), _p(x), _p(out), _p(lo), _p(hi), int(bdry)))
        return out

    def deriv_pencils(self, direction, order, x, index=None, bc_lo=None, bc_hi=None, var=0):
        """The reference's per-pencil derivative calls, batched
        (css_deriv_pencils): direction 0 pencils are (nr, nth) arrays (the
        plane of phi index[p]), 1 and 2 (nphi, nth) arrays (the plane of
        radius index[p]); x has shape (npencils, ...).  var as the named
        routines take it."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.empty_like(x)
        vec = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        lo, hi = vec(bc_lo), vec(bc_hi)
        idx = None if index is None else np.ascontiguousarray(index, dtype=np.int32)
        ip = None if idx is None else idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        check(_lib.lib().css_deriv_pencils(self.h, int(direction), int(order), int(x.shape[0]), ip, _p(x), _p(out),
                                           _p(lo), _p(hi), int(var)))
        return out

    def deriv_device(self, direction, order, x_ptr, out_ptr, bc_lo_ptr=None, bc_hi_ptr=None, bdry=1, stream=None):
        check(_lib.lib().css_deriv_dev(self.h, int(direction), int(order), x_ptr, out_ptr, bc_lo_ptr, bc_hi_ptr,
                                       int(bdry), stream))


def dbyd1_dt0(x, bdat1, bdat2, ibc):
    """Batched Dbyd1_dt0 (derivatives.f90:2296) over the last axis, on the GPU."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    n1 = x.shape[-1]
    lines = x.reshape(-1, n1)
    nl = lines.shape[0]
    out = np.zeros_like(lines)
    b1 = np.ascontiguousarray(np.broadcast_to(np.asarray(bdat1, dtype=np.float64), (nl,)))
    b2 = np.ascontiguousarray(np.broadcast_to(np.asarray(bdat2, dtype=np.float64), (nl,)))
    check(_lib.lib().css_dbyd1_dt0(_p(lines), _p(out), _p(b1), _p(b2), n1, int(ibc), nl))
    return out.reshape(x.shape)


def compact_lines(x, order=1, lphys=True, rphys=True, bdry=1, bc_lo=None, bc_hi=None, halo_lo=None, halo_hi=None,
                  dnum=1.0, scale=1.0):
    """Independent compact-FD lines with explicit closures (css_compact_lines)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.shape[-1]
    lines = x.reshape(-1, n)
    nl = lines.shape[0]
    out = np.zeros_like(lines)

    def vec(a, k):
        if a is None:
            return None
        return np.ascontiguousarray(np.broadcast_to(np.asarray(a, dtype=np.float64), (nl, k) if k > 1 else (nl,)))

    check(_lib.lib().css_compact_lines(_p(lines), _p(out), n, nl, int(order), int(bool(lphys)), int(bool(rphys)),
                                       int(bdry), _p(vec(bc_lo, 1)), _p(vec(bc_hi, 1)), _p(vec(halo_lo, 4)),
                                       _p(vec(halo_hi, 4)), float(dnum), float(scale)))
    return out.reshape(x.shape)


def compact_fd6(dri, arr, b1, b2, ibc, dtype=0, darr=None):
    """Drop-in for CSS-Python derivatives.py:32 compact_fd6 (dtype=0, the
    whole-line form; the reference's dtype 1-3 closures do not converge).
    For ibc 2/4 (3/4) the Neumann datum is darr[0] (darr[-1]) in the
    reference's convention, f'(x_end)/dri.  Runs on the GPU."""
    if dtype != 0:
        raise ValueError("compact_fd6: only dtype=0 (whole line) is supported")
    a = np.asarray(arr, dtype=np.float64)
    n = a.shape[-1]
    dli = float(n - 1)
    drin = float(dri) * dli
    lo = hi = 0.0
    if darr is not None:
        d = np.asarray(darr, dtype=np.float64)
        if ibc in (2, 4):
            lo = d[..., 0] / dli * drin
        if ibc in (3, 4):
            hi = d[..., -1] / dli * drin
    return compact_lines(a, 1, True, True, int(ibc), lo, hi, dnum=drin, scale=drin)
