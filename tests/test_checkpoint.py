"""Checkpoints in the reference's layout (checkpoint.f90:146-423).

The header's number formats follow the Fortran edit descriptors (5i9) and
(8e14.7); the expected strings below are those descriptors applied by hand
(E14.7: sign, "0.", seven significant digits, E and a signed two-digit
exponent, right-justified in 14 columns; beyond exponent 99 the E is
dropped).  The field files are the raw FP64 array in Fortran (nth, nphi, nr)
order, which the reference's CSS-Python reader loads with numpy.fromfile
(CSS-Python/unformatted_read.py:17-33)."""
import os

import numpy as np
import pytest

from css_b200 import checkpoint as CK
from css_b200 import problem


def test_fortran_e14_7_by_hand():
    cases = {1.5: " 0.1500000E+01", -1.23456789e-4: "-0.1234568E-03", 0.0: " 0.0000000E+00",
             0.99999996: " 0.1000000E+01", 2.5e-7: " 0.2500000E-06", 1e100: " 0.1000000+101",
             -3.14159265358979: "-0.3141593E+01", 123456789.0: " 0.1234568E+09"}
    for x, want in cases.items():
        assert CK.fortran_e14_7(x) == want, (x, CK.fortran_e14_7(x))
        assert len(CK.fortran_e14_7(x)) == 14


def test_header_lines_have_the_fortran_widths():
    h = CK.header_text(64, 64, 128, 5, 1200, 2.5e-4, 0.3, 0.7, 0.97, 0.785, 2.356, 0.0, 1.5708)
    l1, l2 = h.splitlines()
    assert l1 == "       64       64      128        5     1200"
    assert len(l2) == 8 * 14 and l2.startswith(" 0.2500000E-03 0.3000000E+00")


def test_host_round_trip(tmp_path):
    p, prof, v0, dt, _ = problem.build((24, 32, 64), decomp=(2, 2, 4))
    d = tmp_path / "0001200"
    CK.write(str(d), v0, p, 1200, dt, 0.25)
    v, h = CK.read(str(d))
    assert np.array_equal(v, v0)
    assert h["istep"] == 1200 and h["nv"] == 5 and (h["nr"], h["nth"], h["nphi"]) == (24, 32, 64)
    assert abs(h["deltat"] - dt) <= 5e-7 * dt  # 7 significant digits, as the reference keeps it
    # a field file is the Fortran (nth, nphi, nr) array: theta fastest
    raw = np.fromfile(str(d / "checkpoint.s"), dtype=np.float64)
    assert raw.size == 24 * 32 * 64 and raw[1] == v0[4, 0, 0, 1] and raw[32] == v0[4, 0, 1, 0]


@pytest.mark.gpu
@pytest.mark.parametrize("magnetic", [False, True])
def test_library_checkpoints_equal_the_host_layout(gpu_available, tmp_path, magnetic):
    from css_b200.context import Simulation
    p, prof, v0, dt, _ = problem.build((24, 32, 64), magnetic=magnetic, decomp=(2, 2, 4))
    sim = Simulation(p, prof)
    sim.upload(v0)
    sim.step_rk4(dt, 2)
    state = sim.download()
    a, b = tmp_path / "lib", tmp_path / "host"
    sim.checkpoint_write(str(a), 2, dt, 2 * dt)
    CK.write(str(b), state, p, 2, dt, 2 * dt)
    for name in ["header"] + ["checkpoint." + n for n in CK.NAMES[:state.shape[0]]]:
        assert (a / name).read_bytes() == (b / name).read_bytes(), name
    # reading replaces the state; stepping continues exactly
    other = Simulation(p, prof)
    other.upload(v0)
    istep, dt_in, t_in = other.checkpoint_read(str(a))
    assert istep == 2 and abs(t_in - 2 * dt) <= 5e-7 * 2 * dt
    assert np.array_equal(other.download(), state)
    sim.step_rk4(dt, 1)
    other.step_rk4(dt, 1)
    assert np.array_equal(sim.download(), other.download())


def test_rain_and_ash_header_variants_and_squall_records(tmp_path):
    """checkpoint.f90:172-181, :290-309: the header's first line carries
    nsqualls (entropy rain) and iashtime (prescribed bottom); the squalls
    go to checkpoint.rain_squalls as 12 REAL*8 per record and read back."""
    from css_b200 import checkpoint as C, problem, rain
    p, prof, v0, dt, _ = problem.build((24, 32, 64), decomp=(2, 2, 4))
    r = rain.RainSqualls(p, prof, nsqualls=5, meandur=1.0, meansize=0.05, rhotopin=0.1, stopin=-1e-3,
                         utopin=-0.02, seed=3)
    r.scaling[:] = np.linspace(0.1, 0.5, 5)
    d = str(tmp_path / "ck")
    C.write(d, v0, p, 17, 1e-3, 2.5, rain=r, iashtime=9)
    first = open(d + "/header").read().splitlines()[0]
    assert len(first) == 7 * 9 and first.split()[-2:] == ["5", "9"]
    assert os.path.getsize(d + "/checkpoint.rain_squalls") == 5 * 12 * 8
    v, head = C.read(d, rain=True, bottom_specified=True)
    assert np.array_equal(v, v0) and head["nsqualls"] == 5 and head["iashtime"] == 9 and head["istep"] == 17
    r2 = rain.RainSqualls(p, prof, nsqualls=5, meandur=1.0, meansize=0.05, rhotopin=0.1, stopin=-1e-3,
                          utopin=-0.02, seed=99)
    C.read_rain_squalls(d + "/checkpoint.rain_squalls", r2)
    for a in ("par", "sigma_t", "start", "scaling", "loct", "locp"):
        assert np.array_equal(getattr(r2, a), getattr(r, a)), a
    C.write(str(tmp_path / "plain"), v0, p, 1, dt, 0.0, iashtime=4)
    assert len(open(str(tmp_path / "plain") + "/header").read().splitlines()[0]) == 6 * 9
