// css_voronoi.h -- host-side Voronoi cells of the convection-cell sites of
// entropy rain's downflow lanes (Compute_Voronoi, voronoi.f90:30-280, which
// Build_Downflow_Lanes, entropy_rain.f90:657-713, walks edge by edge).
//
// The triangulation is an incremental Bowyer-Watson Delaunay construction
// (a point's cavity = the triangles whose circumcircle holds it, re-fanned
// from the point; the hull closed by ghost triangles through a vertex at
// infinity), checked against the Euler count 2n - 2 - h.  Delaunay
// triangulations of points in general position are unique, so the cells
// are the reference's; what the reference's triangle numbering decides is
// only where a closed cell's walk starts, which moves no lane sample.  The
// walk around each site follows the reference's rules:
//   - a site inside the hull: its triangles clockwise, from the first
//     triangle (in triangle order) that holds it, the cell closed;
//   - a site on the hull: from its most clockwise triangle counterclockwise
//     to the hull again (Build_Downflow_Lanes then closes the chain with a
//     chord from the last vertex to the first, as it does every cell).
// Every triangle is stored counterclockwise.  Host code only.
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <vector>

namespace css {

struct VorTri {
  int v[3];
  double cx, cy, rr;  // circumcentre and squared radius
};

// circumcentre of (a, b, c), computed relative to a
inline void vor_circumcentre(double ax, double ay, double bx, double by, double cx, double cy, double &ux,
                             double &uy) {
  const double bxr = bx - ax, byr = by - ay, cxr = cx - ax, cyr = cy - ay;
  const double d = 2.0 * (bxr * cyr - byr * cxr);
  const double b2 = bxr * bxr + byr * byr, c2 = cxr * cxr + cyr * cyr;
  ux = ax + (cyr * b2 - byr * c2) / d;
  uy = ay + (bxr * c2 - cxr * b2) / d;
}

inline double vor_orient(double ax, double ay, double bx, double by, double cx, double cy) {
  return (bx - ax) * (cy - ay) - (by - ay) * (cx - ax);
}

// number of points on the convex hull's boundary, those in the middle of a
// hull edge included (the Euler count of a triangulation needs every
// boundary vertex): the strict hull by monotone chain, then every point on
// one of its edges
inline int vor_hull_size(int n, const double *x, const double *y) {
  std::vector<int> id(n);
  for (int i = 0; i < n; i++) id[i] = i;
  std::sort(id.begin(), id.end(), [&](int a, int b) { return x[a] < x[b] || (x[a] == x[b] && y[a] < y[b]); });
  std::vector<int> h(2 * n + 1);
  int k = 0;
  auto turn = [&](int i) {
    return vor_orient(x[h[k - 2]], y[h[k - 2]], x[h[k - 1]], y[h[k - 1]], x[i], y[i]);
  };
  for (int q = 0; q < n; q++) {  // lower chain, left to right
    while (k >= 2 && turn(id[q]) <= 0.0) k--;
    h[k++] = id[q];
  }
  const int lower = k + 1;
  for (int q = n - 2; q >= 0; q--) {  // upper chain, right to left
    while (k >= lower && turn(id[q]) <= 0.0) k--;
    h[k++] = id[q];
  }
  k--;  // the first point closed the chain
  int count = 0;
  for (int i = 0; i < n; i++)
    for (int e = 0; e < k; e++) {
      const int a = h[e], b = h[(e + 1) % k];
      if (i == a) { count++; break; }
      if (vor_orient(x[a], y[a], x[b], y[b], x[i], y[i]) != 0.0) continue;
      const double d = (x[i] - x[a]) * (x[b] - x[a]) + (y[i] - y[a]) * (y[b] - y[a]);
      const double l = (x[b] - x[a]) * (x[b] - x[a]) + (y[b] - y[a]) * (y[b] - y[a]);
      if (d > 0.0 && d < l) { count++; break; }
    }
  return count;
}

// > 0 when d lies inside the circle through the counterclockwise a, b, c
inline double vor_incircle(double ax, double ay, double bx, double by, double cx, double cy, double dx, double dy) {
  const double adx = ax - dx, ady = ay - dy, bdx = bx - dx, bdy = by - dy, cdx = cx - dx, cdy = cy - dy;
  const double a2 = adx * adx + ady * ady, b2 = bdx * bdx + bdy * bdy, c2 = cdx * cdx + cdy * cdy;
  return adx * (bdy * c2 - b2 * cdy) - ady * (bdx * c2 - b2 * cdx) + a2 * (bdx * cdy - bdy * cdx);
}

// Delaunay triangles of n distinct points (counterclockwise); 0, or -1 for
// fewer than 3 points, coincident or all-collinear points or a degenerate
// configuration.  The hull is closed by ghost triangles (u, w, infinity):
// the outside of the hull edge u -> w, lying on its left; a point
// conflicts with one when it is strictly on that side (or on the open
// edge), with a real triangle when it is strictly inside its circumcircle.
inline int vor_delaunay(int n, const double *x, const double *y, std::vector<VorTri> &tri) {
  tri.clear();
  if (n < 3) return -1;
  for (int p = 1; p < n; p++)
    for (int q = 0; q < p; q++)
      if (x[q] == x[p] && y[q] == y[p]) return -1;
  int k0 = -1;  // the first point off the line through points 0 and 1
  for (int k = 2; k < n && k0 < 0; k++)
    if (vor_orient(x[0], y[0], x[1], y[1], x[k], y[k]) != 0.0) k0 = k;
  if (k0 < 0) return -1;
  const int INF = -1;
  std::vector<std::array<int, 3>> cur, keep;
  {
    int a = 0, b = 1, c = k0;
    if (vor_orient(x[a], y[a], x[b], y[b], x[c], y[c]) < 0.0) std::swap(b, c);
    cur = {{a, b, c}, {b, a, INF}, {c, b, INF}, {a, c, INF}};
  }
  auto conflict = [&](const std::array<int, 3> &t, int p) {
    if (t[2] == INF) {
      const int u = t[0], w = t[1];
      const double o = vor_orient(x[u], y[u], x[w], y[w], x[p], y[p]);
      if (o > 0.0) return true;
      if (o < 0.0) return false;
      const double d = (x[p] - x[u]) * (x[w] - x[u]) + (y[p] - y[u]) * (y[w] - y[u]);
      const double l = (x[w] - x[u]) * (x[w] - x[u]) + (y[w] - y[u]) * (y[w] - y[u]);
      return d > 0.0 && d < l;
    }
    return vor_incircle(x[t[0]], y[t[0]], x[t[1]], y[t[1]], x[t[2]], y[t[2]], x[p], y[p]) > 0.0;
  };
  std::vector<std::array<int, 2>> edges;
  for (int p = 2; p < n; p++) {
    if (p == k0) continue;
    keep.clear();
    edges.clear();
    for (const auto &t : cur) {
      if (conflict(t, p)) {
        for (int e = 0; e < 3; e++) edges.push_back({t[e], t[(e + 1) % 3]});
      } else {
        keep.push_back(t);
      }
    }
    if (edges.empty()) return -1;
    for (size_t e = 0; e < edges.size(); e++) {  // the cavity's boundary: edges without their reverse
      bool inner = false;
      for (size_t f = 0; f < edges.size() && !inner; f++)
        inner = edges[f][0] == edges[e][1] && edges[f][1] == edges[e][0];
      if (inner) continue;
      const int a = edges[e][0], b = edges[e][1];
      if (a == INF) keep.push_back({b, p, INF});       // (inf, b, p) rotated: ghost of p -> ... edge b -> p
      else if (b == INF) keep.push_back({p, a, INF});  // (a, inf, p) rotated: ghost of edge p -> a
      else {
        if (vor_orient(x[a], y[a], x[b], y[b], x[p], y[p]) <= 0.0) return -1;
        keep.push_back({a, b, p});
      }
    }
    cur.swap(keep);
  }
  for (const auto &t : cur) {
    if (t[2] == INF) continue;
    VorTri v;
    v.v[0] = t[0]; v.v[1] = t[1]; v.v[2] = t[2];
    vor_circumcentre(x[t[0]], y[t[0]], x[t[1]], y[t[1]], x[t[2]], y[t[2]], v.cx, v.cy);
    const double dx = x[t[0]] - v.cx, dy = y[t[0]] - v.cy;
    v.rr = dx * dx + dy * dy;
    tri.push_back(v);
  }
  const int h = vor_hull_size(n, x, y);
  if ((int)tri.size() != 2 * n - 2 - h) return -1;
  return 0;
}

// Voronoi cells in Compute_Voronoi's form: degree[g] vertices of site g's
// cell, face[start[g] .. start[g] + degree[g] - 1] their indices into
// vxy (2 per vertex: the circumcentres of the Delaunay triangles).
inline int vor_cells(int n, const double *x, const double *y, std::vector<int> &degree, std::vector<int> &start,
                     std::vector<int> &face, std::vector<double> &vxy) {
  std::vector<VorTri> tri;
  if (int rc = vor_delaunay(n, x, y, tri)) return rc;
  const int nt = (int)tri.size();
  vxy.resize(2 * (size_t)nt);
  for (int t = 0; t < nt; t++) { vxy[2 * t] = tri[t].cx; vxy[2 * t + 1] = tri[t].cy; }
  // per site: its triangles with the vertex after it (succ) and before it (pred)
  std::vector<std::vector<std::array<int, 3>>> inc(n);
  for (int t = 0; t < nt; t++)
    for (int s = 0; s < 3; s++) inc[tri[t].v[s]].push_back({t, tri[t].v[(s + 1) % 3], tri[t].v[(s + 2) % 3]});
  degree.assign(n, 0);
  start.assign(n, 0);
  face.clear();
  for (int g = 0; g < n; g++) {
    const auto &L = inc[g];
    degree[g] = (int)L.size();
    start[g] = (int)face.size();
    if (L.empty()) continue;
    auto cw = [&](int k) {  // across the edge (g, succ): the triangle whose pred is that succ
      for (int j = 0; j < (int)L.size(); j++)
        if (L[j][2] == L[k][1]) return j;
      return -1;
    };
    auto ccw = [&](int k) {
      for (int j = 0; j < (int)L.size(); j++)
        if (L[j][1] == L[k][2]) return j;
      return -1;
    };
    int k = 0, steps = 0;
    bool hull = false;
    for (;;) {  // clockwise from the first triangle: closed, or the hull
      const int j = cw(k);
      if (j < 0) { hull = true; break; }
      if (j == 0 || ++steps > (int)L.size()) break;
      k = j;
    }
    if (!hull) {
      k = 0;
      for (int c = 0; c < (int)L.size(); c++) { face.push_back(L[k][0]); k = cw(k); }
    } else {
      for (int c = 0; c < (int)L.size() && k >= 0; c++) { face.push_back(L[k][0]); k = ccw(k); }
    }
    if ((int)face.size() - start[g] != degree[g]) return -1;
  }
  return 0;
}

}  // namespace css
