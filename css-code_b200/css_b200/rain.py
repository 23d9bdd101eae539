"""Entropy rain: the rain-squall model of entropy_rain.f90 on the host,
feeding the device's squall builder (css_build_squalls) and the
top inflow/outflow relaxation that reads its fields.

As in the reference the squall bookkeeping is host work between steps
(Update_Rain_Squalls runs after every ufreq/10-th step on the top ranks,
step_rk4.f90:484-486); only the fields are built on the device.  Restated:
Initialize_Rain_Squalls for squalls (entropy_rain.f90:113-153), both squall shapes (sstruct 1 Gaussian,
0 polynomial, built on the device), Update_Rain_Squalls (:316-419),
Temporal_Structure (:851-880), Find_Position (:817-824),
Generate_New_Squall_Parameters (:737-814), Place_Cell (:930-945) and
Random_Exponential (:947-962); for the downflow lanes (build_lanes) the
convection cells' life cycle (ConvectionCells: Initialize_Rain_Squalls
:67-111, Update_Rain_Squalls :181-314, Generate_New_Cell_Parameters
:715-735, Find_Cell_Position :827-834, Temporal_Structure_Cell :836-849),
their Voronoi cells and lane field being the library's (css_build_lanes).

The reference seeds Fortran's random_number from system_clock
(:60-61), so its draws differ from run to run; here a seeded numpy
Generator draws from the same distributions (an exponential truncated to
(0.3, 4) by rejection, and the uniform placement with Place_Cell's
rejection loop), so a run is reproducible for a given seed.
"""
import math

import numpy as np

from .params import PROF_NAMES

# parameter columns of a squall (Generate_New_Squall_Parameters' params(:, 1..7))
DELS, SIZE, DUR, THETA, PHI, VEL, DELR = range(7)


class RainSqualls:
    """The squall population of one run.

    nsqualls, meandur, meansize, rainstats, tstruct, sstruct, rhotopin,
    stopin, utopin are the reference's namelist values (mhdsph_mpi.f90:
    1157-1159);
    p and profiles are the run's parameters and radial profiles."""

    def __init__(self, p, profiles, nsqualls, meandur, meansize, rhotopin, stopin, utopin, rainstats=1,
                 tstruct=0, sstruct=1, seed=0, sim_time=0.0):
        pr = np.asarray(profiles, dtype=np.float64).reshape(len(PROF_NAMES), p.nr)
        self.p = p
        self.rng = np.random.default_rng(seed)
        self.r2 = p.r2
        self.dth = (p.th2 - p.th1) / (p.nth - 1)
        self.dphi = (p.phi2 - p.phi1) / p.nphi
        self.meandur, self.meansize = float(meandur), float(meansize)
        self.rainstats, self.tstruct, self.sstruct = int(rainstats), int(tstruct), int(sstruct)
        # Initialize_Rain_Squalls (:55-58)
        self.meandrho = rhotopin * pr[PROF_NAMES.index("rhor")][-1]
        self.meands = float(stopin)
        self.meanvel = float(utopin)
        self.sigt = 3.0 * pr[PROF_NAMES.index("dr_ind")][-1] / abs(utopin)
        n = int(nsqualls)
        self.par = self.generate(n)
        self.sigma_t = np.full(n, self.sigt)
        self.start = np.full(n, sim_time - 1.0)
        self.scaling = np.zeros(n)
        self.loct = np.zeros(n, dtype=np.int64)
        self.locp = np.zeros(n, dtype=np.int64)
        for k in range(n):
            self.find_position(k)

    # random draws -----------------------------------------------------------
    def random_exponential(self, n, g0=0.3, g1=4.0):
        out = np.empty(n)
        i = 0
        while i < n:
            x = -math.log(self.rng.random())
            if g0 < x < g1:
                out[i] = x
                i += 1
        return out

    def place_cell(self):
        p = self.p
        th0 = 2.0 * p.th2
        while th0 > p.th2 or th0 < p.th1:
            th0 = p.th1 + (p.th2 - p.th1) * (1.1 * self.rng.random() - 0.1)
        ph0 = 2.0 * p.phi2
        while ph0 > p.phi2 or ph0 < p.phi1:
            ph0 = p.phi1 + (p.phi2 - p.phi1) * (1.1 * self.rng.random() - 0.1)
        return th0, ph0

    def generate(self, n):
        """Generate_New_Squall_Parameters: rainstats 1 scales every property
        by one exponential draw per squall, otherwise only the duration."""
        par = np.empty((n, 7))
        rand = self.random_exponential(n)
        for k in range(n):
            r = rand[k]
            par[k, DUR] = self.meandur * r
            if self.rainstats == 1:
                par[k, SIZE], par[k, VEL] = self.meansize * r, self.meanvel * r
                par[k, DELS], par[k, DELR] = self.meands * r, self.meandrho * r
            else:
                par[k, SIZE], par[k, VEL] = self.meansize, self.meanvel
                par[k, DELS], par[k, DELR] = self.meands, self.meandrho
            par[k, THETA], par[k, PHI] = self.place_cell()
        return par

    # per-squall rules ---------------------------------------------------------
    def find_position(self, k):
        p = self.p
        self.loct[k] = max(min(math.floor((self.par[k, THETA] - p.th1) / self.dth) + 1, p.nth), 1)
        self.locp[k] = max(min(math.floor((self.par[k, PHI] - p.phi1) / self.dphi) + 1, p.nphi), 1)

    def temporal_structure(self, k, t):
        t0, dur, sig = self.start[k], self.par[k, DUR], self.sigma_t[k]
        t1 = t0 + dur
        if self.tstruct == 1:
            ft = 1.0 if (t > t0 and t < t1) else 0.0
        elif t - t0 <= sig:
            ft = math.sin(0.5 * math.pi * (t - t0) / sig) ** 2
        elif t - t0 >= dur - sig:
            ft = math.sin(0.5 * math.pi * (dur - t - t0) / sig) ** 2  # as written (:873)
        else:
            ft = 1.0
        self.scaling[k] = ft

    def squalls(self):
        """(n, 6) theta_loc, phi_loc, size, scaling, vel, dels for the builder."""
        return np.stack([self.par[:, THETA], self.par[:, PHI], self.par[:, SIZE], self.scaling, self.par[:, VEL],
                         self.par[:, DELS]], axis=1)

    def update(self, sim_time, deltat, w_top, v_top):
        """Update_Rain_Squalls for squalls: age, advect by the surface flow
        (w_top, v_top: the top plane of vars0, shape (nphi, nth)), then the
        squall list the fields are built from (returned; the caller hands it
        to build_squalls with self.sstruct), then replace the dead squalls."""
        p = self.p
        n = len(self.start)
        iup = np.zeros(n, dtype=bool)
        for k in range(n):
            if self.start[k] + self.par[k, DUR] <= sim_time:
                iup[k] = True
                continue
            lct, lcp = self.loct[k], self.locp[k]
            self.temporal_structure(k, sim_time)
            self.par[k, THETA] = self.par[k, THETA] + deltat * w_top[lcp - 1, lct - 1] / self.r2
            if self.par[k, THETA] <= p.th1 or self.par[k, THETA] >= p.th2:
                self.start[k] = 0.0  # killed on the next step
                iup[k] = True
            self.par[k, PHI] = self.par[k, PHI] + deltat * v_top[lcp - 1, lct - 1] / self.r2
            if self.par[k, PHI] <= p.phi1:
                self.par[k, PHI] = p.phi2 + (self.par[k, PHI] - p.phi1)
            if self.par[k, PHI] >= p.phi2:
                self.par[k, PHI] = p.phi1 + (self.par[k, PHI] - p.phi2)
            self.find_position(k)
        built = self.squalls()
        nup = int(iup.sum())
        if nup:
            new = self.generate(nup)
            for k, row in zip(np.flatnonzero(iup), new):
                self.par[k] = row
                self.sigma_t[k] = self.sigt
                self.start[k] = sim_time
                self.scaling[k] = 0.0
                self.find_position(k)
        return built


class ConvectionCells:
    """The convection cells whose Voronoi edges are the downflow lanes
    (build_lanes).  ncells sites placed uniformly (Place_Cell), lasting
    1e12 (Generate_New_Cell_Parameters), their scaling ramping as
    sin^2(pi (t - t0) / 2e4) over the first 1e4 time units
    (Temporal_Structure_Cell), advected by the mean surface flow of their
    theta row and replaced when they leave the theta range
    (Update_Rain_Squalls).  meansize, stopin (meands) and utopin (meanvel)
    are the rain namelist values shared with RainSqualls."""

    def __init__(self, p, ncells, meansize, stopin, utopin, seed=0, sim_time=0.0, rng=None):
        self.p = p
        self.rng = rng if rng is not None else np.random.default_rng(seed)
        self.r2 = p.r2
        self.dth = (p.th2 - p.th1) / (p.nth - 1)
        self.dphi = (p.phi2 - p.phi1) / p.nphi
        self.meansize, self.meands, self.meanvel = float(meansize), float(stopin), float(utopin)
        n = int(ncells)
        self.phi, self.theta, self.dur = self.generate(n)
        self.start = np.full(n, sim_time - 1.0)
        self.scaling = np.zeros(n)
        self.loct = np.zeros(n, dtype=np.int64)
        self.locp = np.zeros(n, dtype=np.int64)
        for k in range(n):
            self.find_position(k)

    def place_cell(self):
        p = self.p
        th0 = 2.0 * p.th2
        while th0 > p.th2 or th0 < p.th1:
            th0 = p.th1 + (p.th2 - p.th1) * (1.1 * self.rng.random() - 0.1)
        ph0 = 2.0 * p.phi2
        while ph0 > p.phi2 or ph0 < p.phi1:
            ph0 = p.phi1 + (p.phi2 - p.phi1) * (1.1 * self.rng.random() - 0.1)
        return th0, ph0

    def generate(self, n):
        """Generate_New_Cell_Parameters: positions, duration 1e12."""
        phi, theta = np.empty(n), np.empty(n)
        for k in range(n):
            theta[k], phi[k] = self.place_cell()
        return phi, theta, np.full(n, 1e12)

    def find_position(self, k):
        p = self.p
        self.loct[k] = max(min(math.floor((self.theta[k] - p.th1) / self.dth) + 1, p.nth), 1)
        self.locp[k] = max(min(math.floor((self.phi[k] - p.phi1) / self.dphi) + 1, p.nphi), 1)

    def temporal_structure(self, k, t):
        dt_ = t - self.start[k]
        self.scaling[k] = math.sin(math.pi * dt_ / 2e4) ** 2 if dt_ <= 1e4 else 1.0

    def cells(self):
        """(n, 3) phi_loc, theta_loc, scaling for build_lanes."""
        return np.stack([self.phi, self.theta, self.scaling], axis=1)

    def update(self, sim_time, deltat, vs_theta, vs_phi):
        """The cells' part of Update_Rain_Squalls: vs_theta / vs_phi are the
        theta profiles (length nth) of u_theta and u_phi averaged over phi
        and the top block's radii; the sites move by deltat * vs / r2, the
        ones that left the theta range (or outlived their duration) are
        replaced after the scalings are set.  Returns the cells to build
        the lanes from."""
        p = self.p
        n = self.phi.size
        iup = np.zeros(n, dtype=bool)
        for k in range(n):
            if self.start[k] + self.dur[k] <= sim_time:
                iup[k] = True
                continue
            lct = self.loct[k]
            self.temporal_structure(k, sim_time)
            self.theta[k] = self.theta[k] + deltat * vs_theta[lct - 1] / self.r2
            if self.theta[k] <= p.th1 or self.theta[k] >= p.th2:
                self.start[k] = 0.0
                iup[k] = True
            self.phi[k] = self.phi[k] + deltat * vs_phi[lct - 1] / self.r2
            if self.phi[k] <= p.phi1:
                self.phi[k] = p.phi2 + (self.phi[k] - p.phi1)
            if self.phi[k] >= p.phi2:
                self.phi[k] = p.phi1 + (self.phi[k] - p.phi2)
            self.find_position(k)
        nup = int(iup.sum())
        if nup:
            phi, theta, dur = self.generate(nup)
            for j, k in enumerate(np.flatnonzero(iup)):
                self.phi[k], self.theta[k], self.dur[k] = phi[j], theta[j], dur[j]
                self.start[k] = sim_time
                self.scaling[k] = 0.0
                self.find_position(k)
        return self.cells()


def top_block_mean_velocity(sim):
    """theta profiles of u_theta and u_phi averaged over phi and the radii of
    the top radial block (what each top rank sums before the all-reduce,
    entropy_rain.f90:185-196)."""
    p = sim.p
    nr, nn = p.nr, p.nnr
    base, rem = nr // nn, nr % nn
    size_top = base + 1 if (rem > 0 and nn <= rem) else base  # Partition (parallel_mpi.f90:236-343)
    vt = np.zeros(p.nth)
    vp = np.zeros(p.nth)
    for ir in range(nr - size_top, nr):
        vt += sim.plane(1, ir).sum(axis=0)
        vp += sim.plane(2, ir).sum(axis=0)
    return vt / (size_top * p.nphi), vp / (size_top * p.nphi)


def advance(sim, rain, dt, nsteps, ufreq, lanes=None):
    """nsteps steps of a top_inout + do_entropy_rain Simulation with the
    rain model updated after every (ufreq // 10)-th step, as Step_RK4 does
    (step_rk4.f90:484-486): the fields of the update take effect from the
    next step on."""
    every = ufreq // 10
    if every < 1:
        raise ValueError("advance: ufreq must be at least 10 (the rain updates every ufreq/10 steps)")
    nr = sim.p.nr
    for _ in range(nsteps):
        sim.step_rk4(dt, 1)
        istep, t_end = sim.clock()
        if istep % every == 0:
            if lanes is not None:  # the lanes first, the squalls on top of them
                vt, vp = top_block_mean_velocity(sim)
                sim.build_lanes(lanes.update(t_end - dt, dt, vt, vp), lanes.meansize, lanes.meanvel, lanes.meands)
            built = rain.update(t_end - dt, dt, sim.plane(1, nr - 1), sim.plane(2, nr - 1))
            if lanes is not None:
                sim.add_squalls(built, rain.sstruct)
            else:
                sim.build_squalls(built, rain.sstruct)
