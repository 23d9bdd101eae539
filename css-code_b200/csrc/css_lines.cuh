// css_lines.cuh -- the compact sixth-order line operators on one block
// segment, solved by one thread with the precomputed LU (Thomas) tables.
//
// x points at the first point of the segment in shared memory; point j
// (1-based) sits at x[(j-1)*sx]; the four halo points below the segment at
// j = -3..0 and the four above at j = m+1..m+4.  At a physical end the
// boundary datum comes in bclo/bchi instead (the 1-deep BC slot of the
// reference's binfo, parallel_mpi.f90:351-530).
//
// dtype follows Determine_Dtype (derivatives.f90:529-544): 1 = halo below /
// physical above, 2 = physical below / halo above, 3 = halo both; 0 = both
// ends physical (the whole-line case the reference only reaches through
// Dbyd1_dt0 / CSS-Python compact_fd6).  The row formulas are those of
// Dbydr/Dbydt (derivatives.f90:564-728, :1031-1194), D2bydr2/D2bydt2
// (:816-939, :1286-1409) and Dbydp/D2bydp2 (:1491-1532, :1605-1627); the
// sweeps are :730-795.
#pragma once

namespace css {

// constants of the halo-closed rows (derivatives.f90:684-720)
struct HaloD1 {
  static constexpr double c1 = -1.0 / 180.0;
  static constexpr double c2 = c1 * 9.0;
  static constexpr double c3 = c1 * 45.0;
  static constexpr double c5 = 1.0 / 36.0;
  static constexpr double cnst = -(c3 + c5);
  static constexpr double beta1 = 7.0 / 9.0 - c2;
  static constexpr double alpha1 = c1 + c5;
  // right end
  static constexpr double r_c1 = 7.0 / 9.0, r_c2 = 1.0 / 36.0, r_c3 = -1.0 / 180.0;
  static constexpr double r_cnst = r_c2 + r_c3 * 45.0;
  static constexpr double r_beta1 = r_c3 * 9.0 - r_c1;
  static constexpr double r_alpha1 = -(r_c2 + r_c3);
  static constexpr double r_c4 = -r_c3 * 9.0;
  static constexpr double r_c5 = -r_c3 * 45.0;
  // preconditioned 5th-order physical row (derivatives.f90:604-619)
  static constexpr double pc = 1.0 / (0.75 - 3.0 * 0.125);
  static constexpr double pa2 = 0.75 * pc;
  static constexpr double pb1 = -3.0 * pc;
};

// Line addressing.  A line is read as xb[xi(j)], j 1-based (the halo points
// at j = -3..0 and m+1..m+4), and written as ob[oi(j)], j 0-based.  The
// base pointers are __restrict__ parameters of the solvers, so the compiler
// may move the line's loads ahead of the stores of its results; xi and oi
// only map indices (a stride, or the fused kernels' halo-apart and swizzled
// tiles).
struct StridedIn {
  int s;
  __host__ __device__ __forceinline__ int operator()(int j) const { return (j - 1) * s; }
};
struct StridedOut {
  int s;
  __host__ __device__ __forceinline__ int operator()(int j) const { return j * s; }
};

#define CSS_X(j) xb[xi(j)]

// Right-hand side of the first-derivative system, rows written to d[] (a
// per-thread scratch that aliases the output buffer).  Returns nothing; the
// caller runs the sweeps.
template <class X>
__host__ __device__ __forceinline__ double d1_row_lo1(const double *__restrict__ xb, const X &xi, int dtype, int bdry, double bclo,
                                             double dnum, double row2) {
  if (dtype == 1 || dtype == 3) {
    return (-HaloD1::c1) * CSS_X(-3) + HaloD1::c2 * CSS_X(-2) + HaloD1::cnst * CSS_X(-1) +
           (-(7.0 / 9.0)) * CSS_X(0) + HaloD1::c3 * CSS_X(1) + HaloD1::beta1 * CSS_X(2) +
           HaloD1::alpha1 * CSS_X(3);
  }
  double r = 0.0;
  if (bdry % 2 == 0) r = bclo / dnum;
  if (bdry == 0) r = 0.0;
  if (bdry == 1 || bdry == 3) {
    r = (-10.0 / 3.0) * CSS_X(1) + (-3.0) * CSS_X(2) + 6.0 * CSS_X(3) + (1.0 / 3.0) * CSS_X(4);
    r = HaloD1::pa2 * r + HaloD1::pb1 * row2;
  }
  return r;
}

template <class X>
__host__ __device__ __forceinline__ double d1_row_lo2(const double *__restrict__ xb, const X &xi, int dtype) {
  if (dtype == 1 || dtype == 3)
    return (7.0 / 9.0) * (CSS_X(3) - CSS_X(1)) + (1.0 / 36.0) * (CSS_X(4) - CSS_X(0));
  return (-43.0 / 96.0) * CSS_X(1) + (-5.0 / 6.0) * CSS_X(2) + (9.0 / 8.0) * CSS_X(3) + (1.0 / 6.0) * CSS_X(4) +
         (-1.0 / 96.0) * CSS_X(5);
}

template <class X>
__host__ __device__ __forceinline__ double d1_row_hi1(const double *__restrict__ xb, const X &xi, int m, int dtype) {  // row m-1
  if (dtype == 2 || dtype == 3)
    return HaloD1::r_c1 * (CSS_X(m) - CSS_X(m - 2)) + HaloD1::r_c2 * (CSS_X(m + 1) - CSS_X(m - 3));
  return (43.0 / 96.0) * CSS_X(m) + (5.0 / 6.0) * CSS_X(m - 1) + (-9.0 / 8.0) * CSS_X(m - 2) +
         (-1.0 / 6.0) * CSS_X(m - 3) + (1.0 / 96.0) * CSS_X(m - 4);
}

template <class X>
__host__ __device__ __forceinline__ double d1_row_hi2(const double *__restrict__ xb, const X &xi, int m, int dtype, int bdry, double bchi,
                                             double dnum, double rowm1) {  // row m
  if (dtype == 2 || dtype == 3)
    return HaloD1::r_c1 * CSS_X(m + 1) + HaloD1::r_cnst * CSS_X(m + 2) + HaloD1::r_c4 * CSS_X(m + 3) +
           HaloD1::r_c3 * CSS_X(m + 4) + HaloD1::r_beta1 * CSS_X(m - 1) + HaloD1::r_alpha1 * CSS_X(m - 2) +
           HaloD1::r_c5 * CSS_X(m);
  double r;
  if (bdry == 3 || bdry == 4) r = bchi / dnum;
  else r = 0.0;
  if (bdry == 1 || bdry == 2) {
    r = (10.0 / 3.0) * CSS_X(m) + 3.0 * CSS_X(m - 1) + (-6.0) * CSS_X(m - 2) + (-1.0 / 3.0) * CSS_X(m - 3);
    r = HaloD1::pa2 * r + HaloD1::pb1 * rowm1;
  }
  return r;
}

template <class X>
__host__ __device__ __forceinline__ double d1_row_int(const double *__restrict__ xb, const X &xi, int j) {
  return (7.0 / 9.0) * (CSS_X(j + 1) - CSS_X(j - 1)) + (1.0 / 36.0) * (CSS_X(j + 2) - CSS_X(j - 2));
}

// ---- second derivative rows ----
struct HaloD2 {
  static constexpr double c1 = 12.0 / 11.0, c2 = 3.0 / 44.0, c3 = -1.0 / 990.0;
};

template <class X>
__host__ __device__ __forceinline__ double d2_row_lo1(const double *__restrict__ xb, const X &xi, int dtype, int bdry, double bclo, double dnum) {
  if (dtype == 1 || dtype == 3) {
    double r = HaloD2::c3 * (2.0 * (CSS_X(-3) + CSS_X(3)) + (-27.0) * (CSS_X(-2) + CSS_X(2)) +
                             270.0 * (CSS_X(-1) + CSS_X(1)) + (-490.0) * CSS_X(0));
    return r + HaloD2::c1 * (CSS_X(2) - 2.0 * CSS_X(1) + CSS_X(0)) + HaloD2::c2 * (CSS_X(-1) - 2.0 * CSS_X(1) + CSS_X(3));
  }
  if (bdry % 2 == 0) {
    double c1 = -575.0 / 193.0 / dnum;
    if (bdry == 0) c1 = 0.0;
    return c1 * bclo + (-5827.0 / 2316.0) * CSS_X(2) + (1987.0 / 1158.0) * CSS_X(3) + (465.0 / 386.0) * CSS_X(4) +
           (-547.0 / 1158.0) * CSS_X(5) + (157.0 / 2316.0) * CSS_X(6);
  }
  return (1955.0 / 156.0) * CSS_X(1) + (-4057.0 / 156.0) * CSS_X(2) + (1117.0 / 78.0) * CSS_X(3) +
         (-55.0 / 78.0) * CSS_X(4) + (-29.0 / 156.0) * CSS_X(5) + (7.0 / 156.0) * CSS_X(6);
}

template <class X>
__host__ __device__ __forceinline__ double d2_row_lo2(const double *__restrict__ xb, const X &xi, int dtype) {
  if (dtype == 1 || dtype == 3)
    return HaloD2::c1 * (CSS_X(3) - 2.0 * CSS_X(2) + CSS_X(1)) + HaloD2::c2 * (CSS_X(0) - 2.0 * CSS_X(2) + CSS_X(4));
  return 1.2375 * CSS_X(1) + (-3.0) * CSS_X(2) + 2.325 * CSS_X(3) + (-0.6) * CSS_X(4) + 0.0375 * CSS_X(5);
}

template <class X>
__host__ __device__ __forceinline__ double d2_row_hi1(const double *__restrict__ xb, const X &xi, int m, int dtype) {
  if (dtype == 2 || dtype == 3)
    return HaloD2::c1 * (CSS_X(m) - 2.0 * CSS_X(m - 1) + CSS_X(m - 2)) +
           HaloD2::c2 * (CSS_X(m - 3) - 2.0 * CSS_X(m - 1) + CSS_X(m + 1));
  return 1.2375 * CSS_X(m) + (-3.0) * CSS_X(m - 1) + 2.325 * CSS_X(m - 2) + (-0.6) * CSS_X(m - 3) + 0.0375 * CSS_X(m - 4);
}

template <class X>
__host__ __device__ __forceinline__ double d2_row_hi2(const double *__restrict__ xb, const X &xi, int m, int dtype, int bdry, double bchi,
                                             double dnum) {
  if (dtype == 2 || dtype == 3) {
    double r = HaloD2::c1 * (CSS_X(m + 1) - 2.0 * CSS_X(m) + CSS_X(m - 1)) +
               HaloD2::c2 * (CSS_X(m - 2) - 2.0 * CSS_X(m) + CSS_X(m + 2));
    return r + HaloD2::c3 * (2.0 * (CSS_X(m - 2) + CSS_X(m + 4)) + (-27.0) * (CSS_X(m - 1) + CSS_X(m + 3)) +
                             270.0 * (CSS_X(m) + CSS_X(m + 2)) + (-490.0) * CSS_X(m + 1));
  }
  if (bdry == 1 || bdry == 2)
    return (1955.0 / 156.0) * CSS_X(m) + (-4057.0 / 156.0) * CSS_X(m - 1) + (1117.0 / 78.0) * CSS_X(m - 2) +
           (-55.0 / 78.0) * CSS_X(m - 3) + (-29.0 / 156.0) * CSS_X(m - 4) + (7.0 / 156.0) * CSS_X(m - 5);
  double c1 = 575.0 / 193.0 / dnum;
  if (bdry == 0) c1 = 0.0;
  return c1 * bchi + (-5827.0 / 2316.0) * CSS_X(m - 1) + (1987.0 / 1158.0) * CSS_X(m - 2) +
         (465.0 / 386.0) * CSS_X(m - 3) + (-547.0 / 1158.0) * CSS_X(m - 4) + (157.0 / 2316.0) * CSS_X(m - 5);
}

template <class X>
__host__ __device__ __forceinline__ double d2_row_int(const double *__restrict__ xb, const X &xi, int j) {
  return HaloD2::c1 * (CSS_X(j + 1) - 2.0 * CSS_X(j) + CSS_X(j - 1)) +
         HaloD2::c2 * (CSS_X(j - 2) - 2.0 * CSS_X(j) + CSS_X(j + 2));
}

// One line: ORDER 1 or 2.  G points at the 1-based tables of this block and
// bdry: g1 = G, g2 = G + ts, g3 = G + 2 ts.  phi = 1 selects the Dbydp /
// D2bydp2 sweep form (every row after the first as g2*(d + a*t)).
// ob[oi(j-1)] receives scale * solution of row j; the forward values pass
// through out on the way.
template <int ORDER, class X, class O>
__host__ __device__ __forceinline__ void line_solve_a(const double *__restrict__ xb, const X &xi, int m, int dtype, int bdry, double bclo, double bchi,
                                             const double *__restrict__ G, int ts, double dnum, double scale,
                                             int phi, double *__restrict__ ob, const O &oi) {
  const double *g1 = G, *g2 = G + ts, *g3 = G + 2 * ts;
  const double a1 = (ORDER == 1) ? -1.0 / 3.0 : -2.0 / 11.0;
  double r1, r2, rm1, rm;
  if (ORDER == 1) {
    r2 = d1_row_lo2(xb, xi, dtype);
    r1 = d1_row_lo1(xb, xi, dtype, bdry, bclo, dnum, r2);
    rm1 = d1_row_hi1(xb, xi, m, dtype);
    rm = d1_row_hi2(xb, xi, m, dtype, bdry, bchi, dnum, rm1);
  } else {
    r1 = d2_row_lo1(xb, xi, dtype, bdry, bclo, dnum);
    r2 = d2_row_lo2(xb, xi, dtype);
    rm1 = d2_row_hi1(xb, xi, m, dtype);
    rm = d2_row_hi2(xb, xi, m, dtype, bdry, bchi, dnum);
  }
  double t = g2[1] * r1;
  ob[oi(0)] = t;
  if (phi) {
    t = g2[2] * (r2 + a1 * t);
    ob[oi(1)] = t;
    for (int j = 3; j <= m - 2; j++) {
      double d = (ORDER == 1) ? d1_row_int(xb, xi, j) : d2_row_int(xb, xi, j);
      t = g2[j] * (d + a1 * t);
      ob[oi(j - 1)] = t;
    }
    t = g2[m - 1] * (rm1 + a1 * t);
    ob[oi(m - 2)] = t;
    t = g2[m] * (rm + a1 * t);
  } else {
    t = g2[2] * r2 + g3[2] * t;
    ob[oi(1)] = t;
    for (int j = 3; j <= m - 2; j++) {
      double d = (ORDER == 1) ? d1_row_int(xb, xi, j) : d2_row_int(xb, xi, j);
      t = g2[j] * (d + a1 * t);
      ob[oi(j - 1)] = t;
    }
    t = g2[m - 1] * rm1 + g3[m - 1] * t;
    ob[oi(m - 2)] = t;
    t = g2[m] * rm + g3[m] * t;
  }
  double sol = t;
  ob[oi(m - 1)] = scale * sol;
  for (int j = m - 1; j >= 1; j--) {
    sol = ob[oi(j - 1)] + g1[j + 1] * sol;
    ob[oi(j - 1)] = scale * sol;
  }
}

// Same operator with the block length M known at compile time: the sweeps
// are fully unrolled (the forward values go through the output buffer, so
// register use stays low); identical arithmetic to line_solve_a.
template <int ORDER, int M, class X, class O>
__device__ __forceinline__ void line_solve_ua(const double *__restrict__ xb, const X &xi, int dtype, int bdry, double bclo, double bchi,
                                              const double *__restrict__ G, int ts, double dnum, double scale,
                                              int phi, double *__restrict__ ob, const O &oi) {
  const double *g1 = G, *g2 = G + ts, *g3 = G + 2 * ts;
  const double a1 = (ORDER == 1) ? -1.0 / 3.0 : -2.0 / 11.0;
  double r1, r2, rm1, rm;
  if (ORDER == 1) {
    r2 = d1_row_lo2(xb, xi, dtype);
    r1 = d1_row_lo1(xb, xi, dtype, bdry, bclo, dnum, r2);
    rm1 = d1_row_hi1(xb, xi, M, dtype);
    rm = d1_row_hi2(xb, xi, M, dtype, bdry, bchi, dnum, rm1);
  } else {
    r1 = d2_row_lo1(xb, xi, dtype, bdry, bclo, dnum);
    r2 = d2_row_lo2(xb, xi, dtype);
    rm1 = d2_row_hi1(xb, xi, M, dtype);
    rm = d2_row_hi2(xb, xi, M, dtype, bdry, bchi, dnum);
  }
  double t = g2[1] * r1;
  ob[oi(0)] = t;
  if (phi) t = g2[2] * (r2 + a1 * t);
  else t = g2[2] * r2 + g3[2] * t;
  ob[oi(1)] = t;
#pragma unroll
  for (int j = 3; j <= M - 2; j++) {
    double d = (ORDER == 1) ? d1_row_int(xb, xi, j) : d2_row_int(xb, xi, j);
    t = g2[j] * (d + a1 * t);
    ob[oi(j - 1)] = t;
  }
  if (phi) {
    t = g2[M - 1] * (rm1 + a1 * t);
    ob[oi(M - 2)] = t;
    t = g2[M] * (rm + a1 * t);
  } else {
    t = g2[M - 1] * rm1 + g3[M - 1] * t;
    ob[oi(M - 2)] = t;
    t = g2[M] * rm + g3[M] * t;
  }
  double sol = t;
  ob[oi(M - 1)] = scale * sol;
#pragma unroll
  for (int j = M - 1; j >= 1; j--) {
    sol = ob[oi(j - 1)] + g1[j + 1] * sol;
    ob[oi(j - 1)] = scale * sol;
  }
}

// Same arithmetic as line_solve_ua with the forward values held in
// registers instead of the output buffer: the forward sweep then only
// loads and the backward sweep only stores, so nothing orders a load
// behind a store.  The tables are read through the read-only path (G must
// be global memory).
template <int ORDER, int M, class X, class O>
__device__ __forceinline__ void line_solve_r(const double *__restrict__ xb, const X &xi, int dtype, int bdry,
                                             double bclo, double bchi, const double *__restrict__ G, int ts,
                                             double dnum, double scale, int phi, double *__restrict__ ob,
                                             const O &oi) {
  const double *g1 = G, *g2 = G + ts, *g3 = G + 2 * ts;
  const double a1 = (ORDER == 1) ? -1.0 / 3.0 : -2.0 / 11.0;
  double r1, r2, rm1, rm;
  if (ORDER == 1) {
    r2 = d1_row_lo2(xb, xi, dtype);
    r1 = d1_row_lo1(xb, xi, dtype, bdry, bclo, dnum, r2);
    rm1 = d1_row_hi1(xb, xi, M, dtype);
    rm = d1_row_hi2(xb, xi, M, dtype, bdry, bchi, dnum, rm1);
  } else {
    r1 = d2_row_lo1(xb, xi, dtype, bdry, bclo, dnum);
    r2 = d2_row_lo2(xb, xi, dtype);
    rm1 = d2_row_hi1(xb, xi, M, dtype);
    rm = d2_row_hi2(xb, xi, M, dtype, bdry, bchi, dnum);
  }
  double t[M];
  t[0] = __ldg(g2 + 1) * r1;
  if (phi) t[1] = __ldg(g2 + 2) * (r2 + a1 * t[0]);
  else t[1] = __ldg(g2 + 2) * r2 + __ldg(g3 + 2) * t[0];
#pragma unroll
  for (int j = 3; j <= M - 2; j++) {
    const double d = (ORDER == 1) ? d1_row_int(xb, xi, j) : d2_row_int(xb, xi, j);
    t[j - 1] = __ldg(g2 + j) * (d + a1 * t[j - 2]);
  }
  if (phi) {
    t[M - 2] = __ldg(g2 + M - 1) * (rm1 + a1 * t[M - 3]);
    t[M - 1] = __ldg(g2 + M) * (rm + a1 * t[M - 2]);
  } else {
    t[M - 2] = __ldg(g2 + M - 1) * rm1 + __ldg(g3 + M - 1) * t[M - 3];
    t[M - 1] = __ldg(g2 + M) * rm + __ldg(g3 + M) * t[M - 2];
  }
  double sol = t[M - 1];
  ob[oi(M - 1)] = scale * sol;
#pragma unroll
  for (int j = M - 1; j >= 1; j--) {
    sol = t[j - 1] + __ldg(g1 + j + 1) * sol;
    ob[oi(j - 1)] = scale * sol;
  }
}

// pointer-and-stride forms: x[(j-1)*sx], out[(j-1)*so]
template <int ORDER>
__device__ __forceinline__ void line_solve(const double *__restrict__ x, int sx, int m, int dtype, int bdry,
                                           double bclo, double bchi, const double *__restrict__ G, int ts,
                                           double dnum, double scale, int phi, double *__restrict__ out,
                                           int so) {
  line_solve_a<ORDER>(x, StridedIn{sx}, m, dtype, bdry, bclo, bchi, G, ts, dnum, scale, phi, out, StridedOut{so});
}

template <int ORDER, int M>
__device__ __forceinline__ void line_solve_u(const double *__restrict__ x, int sx, int dtype, int bdry, double bclo,
                                             double bchi, const double *__restrict__ G, int ts, double dnum,
                                             double scale, int phi, double *__restrict__ out, int so) {
  line_solve_ua<ORDER, M>(x, StridedIn{sx}, dtype, bdry, bclo, bchi, G, ts, dnum, scale, phi, out, StridedOut{so});
}

// dispatch: compile-time block length when the direction's blocks all have
// length MT (MT > 0), the runtime loop otherwise
template <int ORDER, int MT>
__device__ __forceinline__ void solve(const double *__restrict__ x, int sx, int m, int dtype, int bdry, double bclo,
                                      double bchi, const double *__restrict__ G, int ts, double dnum, double scale,
                                      int phi, double *__restrict__ out, int so) {
  if (MT > 0)
    line_solve_u<ORDER, (MT > 0 ? MT : 16)>(x, sx, dtype, bdry, bclo, bchi, G, ts, dnum, scale, phi, out, so);
  else
    line_solve<ORDER>(x, sx, m, dtype, bdry, bclo, bchi, G, ts, dnum, scale, phi, out, so);
}

#undef CSS_X

}  // namespace css
