"""Checkpoints in the reference's layout, on the host (numpy), for analysis
scripts that do not start the GPU library.

Layout (Checkpoint_Output / Checkpoint_Input, checkpoint.f90:146-423): a
directory holding a text ``header`` -- nr nth nphi nv istep as Fortran
(5i9), deltat sim_time r1 r2 th1 th2 phi1 phi2 as (8e14.7) -- and one file
``checkpoint.<name>`` per field (rho w v u s bt bp br) with the raw FP64
array (nth, nphi, nr) in Fortran order.  ``css_checkpoint_write`` /
``css_checkpoint_read`` of the library write and read the same bytes.
"""
import os

import numpy as np

NAMES = ("rho", "w", "v", "u", "s", "bt", "bp", "br")


def fortran_e14_7(x):
    """One value in the Fortran edit descriptor E14.7: [-]0.dddddddE+xx,
    right-justified in 14 columns (exponents beyond 99 drop the E)."""
    x = float(x)
    if x == 0.0:
        body = "-0.0000000E+00" if np.signbit(x) else "0.0000000E+00"
    elif not np.isfinite(x):
        body = "NaN" if np.isnan(x) else ("Infinity" if x > 0 else "-Infinity")
    else:
        m = "%.6E" % abs(x)
        digits = m[0] + m[2:8]
        e10 = int(m[9:]) + 1
        sign = "-" if x < 0 else ""
        body = ("%s0.%s%+04d" % (sign, digits, e10)) if abs(e10) > 99 else ("%s0.%sE%+03d" % (sign, digits, e10))
    return body.rjust(14)[:14] if len(body) <= 14 else body[-14:]


def header_text(nr, nth, nphi, nv, istep, deltat, sim_time, r1, r2, th1, th2, phi1, phi2):
    line1 = "".join("%9d" % k for k in (nr, nth, nphi, nv, istep))
    line2 = "".join(fortran_e14_7(x) for x in (deltat, sim_time, r1, r2, th1, th2, phi1, phi2))
    return line1 + "\n" + line2 + "\n"


def write(directory, vars0, params, istep, deltat, sim_time):
    """vars0: array (nv, nr, nphi, nth) (the library's layout)."""
    os.makedirs(directory, exist_ok=True)
    v = np.ascontiguousarray(vars0, dtype=np.float64)
    nv = v.shape[0]
    with open(os.path.join(directory, "header"), "w") as f:
        f.write(header_text(params.nr, params.nth, params.nphi, nv, istep, deltat, sim_time, params.r1, params.r2,
                            params.th1, params.th2, params.phi1, params.phi2))
    for iv in range(nv):
        v[iv].tofile(os.path.join(directory, "checkpoint." + NAMES[iv]))


def read(directory):
    """(vars0 (nv, nr, nphi, nth), header dict)."""
    with open(os.path.join(directory, "header")) as f:
        toks = f.read().split()
    nr, nth, nphi, nv, istep = (int(t) for t in toks[:5])
    vals = [float(t.replace("D", "E")) for t in toks[5:13]]
    keys = ("deltat", "sim_time", "r1", "r2", "th1", "th2", "phi1", "phi2")
    head = dict(zip(keys, vals), nr=nr, nth=nth, nphi=nphi, nv=nv, istep=istep)
    v = np.empty((nv, nr, nphi, nth))
    for iv in range(nv):
        v[iv] = np.fromfile(os.path.join(directory, "checkpoint." + NAMES[iv]), dtype=np.float64).reshape(nr, nphi, nth)
    return v, head
