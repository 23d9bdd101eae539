"""The oracle's Voronoi cells (orc_voronoi, the walk of Compute_Voronoi,
voronoi.f90:30-280) pinned against scipy's Qhull: the same Voronoi
vertices (circumcentres of the Delaunay triangles) and, for every site, the
same set of vertices around it; cells inside the hull walked clockwise,
cells on the hull counterclockwise from their most clockwise triangle (the
closed chain's signed area is negative / positive)."""
import numpy as np
import pytest

from oracle import oracle as O


def signed_area(pts):
    x, y = pts[:, 0], pts[:, 1]
    return 0.5 * float(np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y))


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_oracle_voronoi_matches_qhull(seed):
    from scipy.spatial import Voronoi
    rng = np.random.default_rng(seed)
    n = 10
    # sites and their periodic copies, as the downflow lanes place them
    phi, th = rng.uniform(0.0, 1.5, n), rng.uniform(0.8, 2.3, n)
    x = np.concatenate([phi, phi - 1.5, phi + 1.5])
    y = np.concatenate([th, th, th])
    deg, st, face, vxy = O.voronoi(x, y)
    vor = Voronoi(np.stack([x, y], axis=1))
    key = lambda p: (round(p[0], 9), round(p[1], 9))
    assert sorted(map(key, vxy)) == sorted(map(key, vor.vertices))
    for g in range(x.size):
        ours = {key(vxy[k]) for k in face[st[g]:st[g] + deg[g]]}
        region = vor.regions[vor.point_region[g]]
        theirs = {key(vor.vertices[k]) for k in region if k >= 0}
        assert ours == theirs, g
        if deg[g] >= 3:
            area = signed_area(vxy[face[st[g]:st[g] + deg[g]]])
            if -1 in region:
                assert area > 0.0, g  # on the hull: counterclockwise
            else:
                assert area < 0.0, g  # inside: clockwise


def test_convection_cells_update():
    """Update_Rain_Squalls for the convection cells: advection by the mean
    surface flow of the site's theta row, the phi wrap, replacement of a
    cell that leaves the theta range (scaling 0, starting now), and the
    sin^2 ramp of Temporal_Structure_Cell."""
    import math
    from css_b200 import problem, rain
    p, prof, v0, dt, _ = problem.build((48, 48, 64), decomp=(2, 2, 4))
    cc = rain.ConvectionCells(p, 4, meansize=0.05, stopin=-1e-3, utopin=-0.02, seed=3)
    assert np.all(cc.scaling == 0.0) and np.all(cc.dur == 1e12)
    cc.theta[0], cc.phi[0] = 1.5, 0.5
    cc.theta[1], cc.phi[1] = 1.5, p.phi2 - 1e-4
    cc.theta[2] = p.th2 - 1e-5
    for k in range(4):
        cc.find_position(k)
    vt = np.full(p.nth, 2e-3)
    vp = np.full(p.nth, 3e-3)
    old2 = (cc.theta[2], cc.phi[2])
    out = cc.update(10.0, 1.0, vt, vp)
    assert out.shape == (4, 3)
    assert cc.theta[0] == pytest.approx(1.5 + 2e-3 / p.r2) and cc.phi[0] == pytest.approx(0.5 + 3e-3 / p.r2)
    assert p.phi1 <= cc.phi[1] < p.phi1 + 1e-2  # wrapped
    assert (cc.theta[2], cc.phi[2]) != old2 and cc.start[2] == 10.0 and cc.scaling[2] == 0.0
    assert cc.scaling[0] == pytest.approx(math.sin(math.pi * 11.0 / 2e4) ** 2)


def library_voronoi(x, y):
    import ctypes
    from css_b200 import _lib
    n = x.size
    deg, st = np.zeros(n, np.int32), np.zeros(n, np.int32)
    face = np.zeros(6 * n + 32, np.int32)
    vxy = np.zeros((2 * n + 8, 2))
    nv = ctypes.c_int()
    ip = ctypes.POINTER(ctypes.c_int)
    dp = ctypes.POINTER(ctypes.c_double)
    _lib.check(_lib.lib().css_voronoi(n, x.ctypes.data_as(dp), y.ctypes.data_as(dp), deg.ctypes.data_as(ip),
                                      st.ctypes.data_as(ip), face.ctypes.data_as(ip), ctypes.byref(nv),
                                      vxy.ctypes.data_as(dp)))
    return deg, st, face[:int(deg.sum())], vxy[:nv.value]


@pytest.mark.parametrize("seed", [0, 5, 11])
def test_library_voronoi_matches_oracle(seed):
    """css_voronoi (host code of the library: an incremental Delaunay
    construction) against the oracle's brute-force one and its restated
    walk: the same cells, vertex for vertex within 1e-12; a cell on the hull
    the same sequence, a closed cell the same cycle (its starting triangle
    follows the triangle numbering, which differs)."""
    rng = np.random.default_rng(seed)
    n = 12
    phi, th = rng.uniform(0.0, 1.5, n), rng.uniform(0.8, 2.3, n)
    x = np.ascontiguousarray(np.concatenate([phi, phi - 1.5, phi + 1.5]))
    y = np.ascontiguousarray(np.concatenate([th, th, th]))
    from scipy.spatial import Voronoi
    hull = [-1 in Voronoi(np.stack([x, y], axis=1)).regions[r] for r in
            Voronoi(np.stack([x, y], axis=1)).point_region]
    d1, s1, f1, v1 = library_voronoi(x, y)
    d2, s2, f2, v2 = O.voronoi(x, y)
    assert np.array_equal(d1, d2)
    for g in range(x.size):
        a = v1[f1[s1[g]:s1[g] + d1[g]]]
        b = v2[f2[s2[g]:s2[g] + d2[g]]]
        if not hull[g]:
            k = int(np.argmin(np.abs(b - a[0]).sum(axis=1)))
            b = np.roll(b, -k, axis=0)
        assert np.abs(a - b).max() <= 1e-12 * max(1.0, np.abs(b).max()), g
    # coincident sites are refused
    from css_b200._lib import CssError
    x2, y2 = x.copy(), y.copy()
    x2[1], y2[1] = x2[0], y2[0]
    with pytest.raises(CssError):
        library_voronoi(x2, y2)
