"""ASH inflow: the prescribed bottom fields of a run with bottom_specified,
read from the reference's `ash_inflow_data` file and regridded on the host,
then handed to the device (css_set_ash_slices), which interpolates them in
time every step and relaxes the bottom plane toward them.

Restated from ash_inflow.f90: Initialize_ASH_Inflow (:18-120) and
Read_ASH_Inflow (:124-186), with the regridding Interp2d of interp.f90
(:103-176).  The file is Fortran unformatted direct access: record r holds
one field of one time slice as REAL*4 (ashnth, ashnphi + 1), column-major;
the first column carries metadata (cos(theta) in field 2's record, the time
in element 6 of field 1's record) and columns 2.. the data.  Slice k of the
file occupies records 5k + 1 .. 5k + 5 (fields u_r, u_theta, u_phi, the
entropy perturbation and a fifth, unused field).  The record length is
ashnth*(ashnphi + 1) in units of `recl_unit` bytes (4: Intel Fortran's
default word unit, which makes a record exactly one array).

Interp2d is restated as written, including its index choices: along phi it
takes the points k-1, k, k+2, k+3 around the cell k of x (its ix(3) and
ix(4) are (k+1) mod n + 1 and (k+2) mod n + 1), and along theta it starts
from floor((y - y1)/dy) without the +1 and clamps at the ends.  The spacing
of each old axis is read at its middle (interp.f90:125-126).
"""
import math

import numpy as np

NFIELD = 5  # records per slice


class AshInflow:
    """The ASH slice file of one run.

    p: the run's parameters; rhor1, pr1: background density and pressure at
    the bottom (rhor(1), pr(1) of the reference, for the wall taper); cv
    defaults to cp/gamma.  iashtime = 3 is the start of a new run
    (ash_inflow.f90:27-29); a restart passes the checkpointed value."""

    def __init__(self, path, ashnth, ashnphi, p, rhor1, pr1, iashtime=3, recl_unit=4, cv=None):
        self.path, self.ashnth, self.ashnphi = path, int(ashnth), int(ashnphi)
        self.p = p
        self.rhor1, self.pr1 = float(rhor1), float(pr1)
        self.cv = p.cp / p.gamma if cv is None else float(cv)
        self.recbytes = self.ashnth * (self.ashnphi + 1) * int(recl_unit)
        self.iashtime = int(iashtime)
        # new grid (derivatives.f90:81-89) and the old phi grid (:30-32)
        self.theta = (p.th2 - p.th1) / (p.nth - 1) * np.arange(p.nth) + p.th1
        self.phi = (p.phi2 - p.phi1) / p.nphi * np.arange(p.nphi) + p.phi1
        self.ashphi = (p.phi2 - p.phi1) / self.ashnphi * np.arange(self.ashnphi) + p.phi1
        self.startt = float(self.record(6)[5, 0])  # ashstartt = readdata(6,1,1,1) of record 6
        slices, times = [], []
        for k in range(4):
            s, t = self.read_slice((self.iashtime - 3) + k)
            slices.append(s)
            times.append(t)
        self.slices = np.stack(slices)  # (4 times, 4 fields, nphi, nth)
        self.times = np.array(times) - self.startt

    def record(self, r):
        """Record r (1-based) as float64 (ashnth, ashnphi + 1), Fortran order."""
        with open(self.path, "rb") as f:
            f.seek((r - 1) * self.recbytes)
            raw = np.frombuffer(f.read(self.ashnth * (self.ashnphi + 1) * 4), dtype="<f4")
        return raw.reshape(self.ashnphi + 1, self.ashnth).T.astype(np.float64)

    def read_slice(self, k):
        """Slice k of the file, regridded and tapered: ((4, nphi, nth), time)."""
        recs = [self.record(k * NFIELD + iq + 1) for iq in range(NFIELD)]
        costheta = recs[1][:, 0]
        time = recs[0][5, 0]
        ashtheta = np.arccos(costheta)
        full = np.stack([interp2d(r[:, 1:], self.ashphi, ashtheta, self.phi, self.theta) for r in recs])
        return self.taper(full)[:4], time

    def taper(self, full):
        """Wall taper over the 16 theta points next to each wall
        (ash_inflow.f90:100-107): u_theta goes to zero at the walls and its
        kinetic energy moves into the entropy field."""
        th, nth = self.theta, self.p.nth
        f = full.copy()
        for it in range(16):
            tmp = math.sin(0.5 * math.pi * (th[it] - self.p.th1) / (th[15] - self.p.th1)) ** 2
            c = self.cv * (1.0 - tmp) * self.rhor1 / self.pr1
            for j in (it, nth - 1 - it):
                f[3, :, j] = f[3, :, j] + c * f[1, :, j] ** 2
                f[1, :, j] = tmp * f[1, :, j]
        return f

    def shift_if_due(self, sim_time):
        """Read_ASH_Inflow's shift: once sim_time reaches the third slice's
        time the oldest slice is dropped and the next one read.  Returns True
        when the slices changed."""
        if sim_time < self.times[2]:
            return False
        self.iashtime += 1
        s, t = self.read_slice(self.iashtime)
        self.slices = np.concatenate([self.slices[1:], s[None]])
        self.times = np.concatenate([self.times[1:], [t - self.startt]])
        return True


def interp2d(arr, ox, oy, nx, ny):
    """interp.f90:103-176: arr(iy, ix) on the old grid (oy, ox) to the new
    grid (ny, nx); returns (len(nx), len(ny)) indexed [phi, theta].  New x
    must not lie below ox[0] (Fortran's MOD of a negative differs there;
    the reference never asks for it)."""
    onx, ony = len(ox), len(oy)
    odx = ox[onx // 2 - 1] - ox[onx // 2 - 2]
    ody = oy[ony // 2 - 1] - oy[ony // 2 - 2]
    out = np.empty((len(nx), len(ny)))
    for i1, xc in enumerate(nx):
        # 1-based indices as written
        ix2 = math.floor((xc - ox[0]) / odx) % onx + 1
        ix3 = (ix2 + 1) % onx + 1
        ix1 = ix2 - 1
        if ix1 < 1:
            ix1 = onx + ix1
        ix4 = (ix2 + 2) % onx + 1
        mux = (xc - ox[ix2 - 1]) / (ox[ix3 - 1] - ox[ix2 - 1])
        cols = arr[:, [ix1 - 1, ix2 - 1, ix3 - 1, ix4 - 1]]
        ry_all = catmull_rom(cols[:, 0], cols[:, 1], cols[:, 2], cols[:, 3], mux)  # per old theta row
        for i2, yc in enumerate(ny):
            iy2 = max(math.floor((yc - oy[0]) / ody), 1)
            iy3 = min(iy2 + 1, ony)
            iy1 = max(iy2 - 1, 1)
            iy4 = min(iy2 + 2, ony)
            muy = (yc - oy[iy2 - 1]) / (oy[iy3 - 1] - oy[iy2 - 1])
            out[i1, i2] = catmull_rom(ry_all[iy1 - 1], ry_all[iy2 - 1], ry_all[iy3 - 1], ry_all[iy4 - 1], muy)
    return out


def catmull_rom(km1, k, kp1, kp2, mu):
    a3 = k
    a0 = -0.5 * km1 + 1.5 * a3 - 1.5 * kp1 + 0.5 * kp2
    a1 = km1 - 2.5 * a3 + 2.0 * kp1 - 0.5 * kp2
    a2 = -0.5 * km1 + 0.5 * kp1
    mu2 = mu * mu
    return a0 * (mu * mu2) + a1 * mu2 + a2 * mu + a3


def write_ash_file(path, slices, costheta, times, recl_unit=4):
    """A file in the layout AshInflow reads (synthetic inputs for tests and
    demonstrations): slices (nslice, 5, ashnth, ashnphi) float, times
    (nslice,); record 6 (slice 1, field 1) carries the start time in
    element 6, as every slice's first record carries its own time."""
    nslice, nf, ashnth, ashnphi = slices.shape
    assert nf == NFIELD and recl_unit == 4
    with open(path, "wb") as f:
        for k in range(nslice):
            for iq in range(NFIELD):
                rec = np.zeros((ashnth, ashnphi + 1), dtype="<f4")
                rec[:, 1:] = slices[k, iq]
                if iq == 1:
                    rec[:, 0] = costheta
                if iq == 0:
                    rec[5, 0] = times[k]
                f.write(np.asfortranarray(rec).T.tobytes())


def advance(sim, ash, dt, nsteps):
    """nsteps steps of a bottom_specified Simulation, shifting in the next
    slice whenever a step would start at or past the third slice's time
    (Read_ASH_Inflow at the top of each step, step_rk4.f90:345)."""
    for _ in range(nsteps):
        _, t = sim.clock()
        if ash.shift_if_due(t):
            sim.set_ash_slices(ash.slices, ash.times, sim.inout_state()["ash_fen_mod"])
        sim.step_rk4(dt, 1)
