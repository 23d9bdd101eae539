"""Checkpoints in the reference's layout, on the host (numpy), for analysis
scripts that do not start the GPU library.

Layout (Checkpoint_Output / Checkpoint_Input, checkpoint.f90:146-423): a
directory holding a text ``header`` -- nr nth nphi nv istep as Fortran
(5i9), deltat sim_time r1 r2 th1 th2 phi1 phi2 as (8e14.7) -- and one file
``checkpoint.<name>`` per field (rho w v u s bt bp br) with the raw FP64
array (nth, nphi, nr) in Fortran order.  ``css_checkpoint_write`` /
``css_checkpoint_read`` of the library write and read the same bytes.

Runs with entropy rain add nsqualls to the header's first line and write
``checkpoint.rain_squalls`` (one direct-access record of 12 REAL*8 per
squall); a prescribed (ASH) bottom adds iashtime (checkpoint.f90:172-181,
:290-309, :371-395, :77-144).  The header's first line is then (6i9) or
(7i9): nr nth nphi nv istep [nsqualls] [iashtime].
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


def header_text(nr, nth, nphi, nv, istep, deltat, sim_time, r1, r2, th1, th2, phi1, phi2, nsqualls=None,
                iashtime=None):
    ints = [nr, nth, nphi, nv, istep] + ([nsqualls] if nsqualls is not None else []) + \
        ([iashtime] if iashtime is not None else [])
    line1 = "".join("%9d" % k for k in ints)
    line2 = "".join(fortran_e14_7(x) for x in (deltat, sim_time, r1, r2, th1, th2, phi1, phi2))
    return line1 + "\n" + line2 + "\n"


def write(directory, vars0, params, istep, deltat, sim_time, rain=None, iashtime=None):
    """vars0: array (nv, nr, nphi, nth) (the library's layout); rain: the
    run's css_b200.rain.RainSqualls (entropy rain), iashtime: the ASH
    slice counter (prescribed bottom)."""
    os.makedirs(directory, exist_ok=True)
    v = np.ascontiguousarray(vars0, dtype=np.float64)
    nv = v.shape[0]
    nsq = None if rain is None else len(rain.start)
    with open(os.path.join(directory, "header"), "w") as f:
        f.write(header_text(params.nr, params.nth, params.nphi, nv, istep, deltat, sim_time, params.r1, params.r2,
                            params.th1, params.th2, params.phi1, params.phi2, nsqualls=nsq, iashtime=iashtime))
    for iv in range(nv):
        v[iv].tofile(os.path.join(directory, "checkpoint." + NAMES[iv]))
    if rain is not None and nsq > 0:
        write_rain_squalls(os.path.join(directory, "checkpoint.rain_squalls"), rain)


def read(directory, rain=False, bottom_specified=False):
    """(vars0 (nv, nr, nphi, nth), header dict).  rain / bottom_specified
    say which header variant to expect (the reference decides by its own
    do_entropy_rain and Bottom_Specified); the dict then also holds
    nsqualls / iashtime."""
    with open(os.path.join(directory, "header")) as f:
        toks = f.read().split()
    nr, nth, nphi, nv, istep = (int(t) for t in toks[:5])
    k = 5
    extra = {}
    if rain:
        extra["nsqualls"] = int(toks[k])
        k += 1
    if bottom_specified:
        extra["iashtime"] = int(toks[k])
        k += 1
    vals = [float(t.replace("D", "E")) for t in toks[k:k + 8]]
    keys = ("deltat", "sim_time", "r1", "r2", "th1", "th2", "phi1", "phi2")
    head = dict(zip(keys, vals), nr=nr, nth=nth, nphi=nphi, nv=nv, istep=istep, **extra)
    v = np.empty((nv, nr, nphi, nth))
    for iv in range(nv):
        v[iv] = np.fromfile(os.path.join(directory, "checkpoint." + NAMES[iv]), dtype=np.float64).reshape(nr, nphi, nth)
    return v, head


# record layout of checkpoint.rain_squalls (checkpoint.f90:381-392, :117-129)
SQUALL_RECORD = ("Duration", "SigmaT", "Start_Time", "Size", "Dels", "Theta_loc", "Phi_loc", "Scaling", "loct",
                 "locp", "Vel", "Delr")


def write_rain_squalls(path, rain):
    """One record of 12 REAL*8 per squall, in SQUALL_RECORD order."""
    from . import rain as R
    rec = np.stack([rain.par[:, R.DUR], rain.sigma_t, rain.start, rain.par[:, R.SIZE], rain.par[:, R.DELS],
                    rain.par[:, R.THETA], rain.par[:, R.PHI], rain.scaling, rain.loct.astype(np.float64),
                    rain.locp.astype(np.float64), rain.par[:, R.VEL], rain.par[:, R.DELR]], axis=1)
    np.ascontiguousarray(rec, dtype="<f8").tofile(path)


def read_rain_squalls(path, rain):
    """Read_Rain_Squalls into an existing RainSqualls (its nsqualls records);
    the reference then runs Update_Rain_Squalls, which the caller does with
    rain.update before building the fields."""
    from . import rain as R
    n = len(rain.start)
    rec = np.fromfile(path, dtype="<f8", count=12 * n).reshape(n, 12)
    rain.par[:, R.DUR], rain.sigma_t[:], rain.start[:] = rec[:, 0], rec[:, 1], rec[:, 2]
    rain.par[:, R.SIZE], rain.par[:, R.DELS], rain.par[:, R.THETA] = rec[:, 3], rec[:, 4], rec[:, 5]
    rain.par[:, R.PHI], rain.scaling[:] = rec[:, 6], rec[:, 7]
    rain.loct[:], rain.locp[:] = rec[:, 8].astype(np.int64), rec[:, 9].astype(np.int64)
    rain.par[:, R.VEL], rain.par[:, R.DELR] = rec[:, 10], rec[:, 11]
