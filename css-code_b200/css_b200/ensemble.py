"""Batched ensembles of independent shells on one GPU, and their split over
ranks.

The reference runs one spherical shell per job (Program CSS2,
mhdsph_mpi.f90).  A parameter study of many small shells, each with its own
grid, decomposition, Rayleigh and Rossby numbers and hydro or MHD physics,
is run here as one ``Ensemble``: every member keeps its own context
(``Simulation``), one RK4 step of all members is captured once into a CUDA
graph with each member on a stream of its own, and the graph is replayed per
step (``css_ensemble_step``).  Across ranks the members are bin-packed by
their cost (longest processing time first); no collective is needed inside
a step.
"""
import ctypes
import math

import numpy as np

from . import _lib
from ._lib import check, dp

# ranges of the shell study: nr, ntheta, nphi; log10 Ra; Rossby number;
# magnetic Prandtl number of the MHD members (through the SLD scaling
# sld_prm = 1/Pm, as the MHD workload's Pm 2 is sld_prm 0.5)
NR_RANGE = (48, 160)
NTH_RANGE = (64, 256)
NPHI_RANGE = (128, 512)
LOG_RA_RANGE = (4.0, 6.0)
RO_RANGE = (0.3, 3.0)
PM_RANGE = (1.0, 4.0)


def _blocks(n, min_blocks):
    """Virtual blocks along one direction.  Block sizes must be even and in
    [10, 256] (the paired Thomas sweeps of derivatives.f90:755-792 read an
    unset row for odd sizes), so the blocks divide n evenly; 32- or 16-point
    blocks are preferred (the compile-time kernels), else the size nearest
    32."""
    best = None
    for nb in range(min_blocks, n // 10 + 1):
        if n % nb:
            continue
        m = n // nb
        if m % 2 or not 10 <= m <= 256:
            continue
        key = (0 if m in (32, 16) else 1, abs(m - 32), nb)
        if best is None or key < best[0]:
            best = (key, nb)
    if best is None:
        raise ValueError("no decomposition of %d points into >= %d even blocks" % (n, min_blocks))
    return best[1]


def shell_specs(count=48, seed=7):
    """Seeded member descriptions: sizes uniform in the ranges (theta and phi
    rounded to multiples of 16, r to a multiple of 4), Ra log-uniform, Ro
    uniform, every second member magnetic with Pm uniform."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        # nr a multiple of 4, so that two even blocks always exist
        nr = int(min(NR_RANGE[1], max(NR_RANGE[0], 4 * round(rng.integers(NR_RANGE[0], NR_RANGE[1] + 1) / 4))))
        nth = int(min(NTH_RANGE[1], max(NTH_RANGE[0], 16 * round(rng.uniform(*NTH_RANGE) / 16))))
        nphi = int(min(NPHI_RANGE[1], max(NPHI_RANGE[0], 16 * round(rng.uniform(*NPHI_RANGE) / 16))))
        ra = 10.0 ** rng.uniform(*LOG_RA_RANGE)
        ro = rng.uniform(*RO_RANGE)
        mag = i % 2 == 1
        pm = rng.uniform(*PM_RANGE)
        specs.append({"nr": nr, "nth": nth, "nphi": nphi, "ra": ra, "ro": ro, "magnetic": mag,
                      "pm": pm if mag else None, "decomp": (_blocks(nr, 2), _blocks(nth, 2), _blocks(nphi, 3))})
    return specs


def member_cost(spec):
    """Work of one step of a member: cells x fields."""
    return spec["nr"] * spec["nth"] * spec["nphi"] * (8 if spec["magnetic"] else 5)


def lpt_partition(costs, nranks):
    """Longest processing time first: members in decreasing cost, each to the
    least loaded rank (ties to the lowest rank).  Returns one index list per
    rank, each in increasing order."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * nranks
    parts = [[] for _ in range(nranks)]
    for i in order:
        r = min(range(nranks), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def build_member(spec, seed=1234, n_rho=3.0, precision=0):
    """(params, profiles, vars0, dt) of one member; precision 1 stores its
    RK4 stage states in FP32 (the mixed form)."""
    from . import problem
    from .params import default_params
    p = default_params(spec["nr"], spec["nth"], spec["nphi"], spec["decomp"], magnetic=spec["magnetic"])
    p.omega_0 = 0.5 / spec["ro"]
    p.precision = int(precision)
    if spec["magnetic"]:
        p.sld_prm = 1.0 / (spec.get("pm") or 2.0)
    prof, info = problem.polytrope(p, n_rho, ra=spec["ra"])
    vars0 = problem.initial_state(p, prof, info, seed=seed)
    bfield = problem.curl_estimate(p, prof, vars0[5:8]) if spec["magnetic"] else None
    dt = problem.cfl_dt(p, prof, vars0, bfield)
    return p, prof, vars0, dt


class Ensemble:
    """Members stepped together through one CUDA graph (css_ensemble_*).
    ``sims`` are ``Simulation`` objects; they stay owned by the caller."""

    def __init__(self, sims):
        self.sims = list(sims)
        arr = (ctypes.c_void_p * len(self.sims))(*[s.h.value for s in self.sims])
        h = ctypes.c_void_p()
        check(_lib.lib().css_ensemble_create(len(self.sims), arr, ctypes.byref(h)))
        self.h = h

    def step(self, dts, nsteps=1):
        d = np.ascontiguousarray(dts, dtype=np.float64)
        assert d.shape == (len(self.sims),)
        check(_lib.lib().css_ensemble_step(self.h, d.ctypes.data_as(dp), int(nsteps)))

    def launches(self):
        return _lib.lib().css_ensemble_launches(self.h)

    def last_ms(self):
        """Device time of the replays of the last step() call (CUDA events)."""
        return _lib.lib().css_ensemble_last_ms(self.h)

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().css_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cells(spec):
    return spec["nr"] * spec["nth"] * spec["nphi"]


def summary(specs):
    """Totals of a member list (cells, MHD count, bytes of FP64 state)."""
    n = sum(cells(s) for s in specs)
    return {"members": len(specs), "cells": n, "mhd": sum(1 for s in specs if s["magnetic"]),
            "state_bytes": sum(cells(s) * (8 if s["magnetic"] else 5) * 8 for s in specs),
            "largest": max(specs, key=cells) if specs else None, "log10_cells": math.log10(max(n, 1))}
