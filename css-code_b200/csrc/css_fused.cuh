// css_fused.cuh -- the RK4 stage in two passes over HBM, for runs whose
// virtual blocks are 32 points long in r, theta and phi (FP64 state, RK4,
// closed radial faces, SLaplacian/SLD physics; css_create decides).
//
//   k_thph    one CTA per (theta block, phi block, radius): the 32x32 plane
//             of the two blocks with 4-point halos in theta and phi is
//             staged once in shared memory; Source_Theta_Terms (+ Lorentz,
//             + Induction_Terms), Phi_Terms (+ Lorentz) and, on blocks with
//             no theta wall, Density_Terms_Theta run from it, and the
//             tendency of every field and the stage temperature are
//             written once.
//   k_rstage  one CTA per (r block, theta block, phi): the 32(r)x32(theta)
//             slab with 4-point radial halos is staged once; Radial_Terms
//             (+ Lorentz) with Density_Terms_Radial, Density_Terms_Theta on
//             the theta-wall blocks (its wall datum is the completed
//             dw/dt, available only here), the RK4 stage combination of
//             Step_RK4 and Bound, writing the accumulator and the next
//             stage state.
//
// Against the four-kernel stage (theta, phi, radial, update) this removes
// the read-modify-write of the tendency by the phi and radial passes and
// one read of the state and the tendency per stage.  The arithmetic per
// point is that of k_theta_terms, phi_tile_compute, radial_tile and
// k_rhot_update; only the order in which the density-theta term joins the
// sums differs (it follows the theta terms here), a rounding-level change.
#pragma once
#include "css_kernels.cuh"

namespace css {

constexpr int FM = 32;    // block length of the fused path (every direction)
constexpr int FNT = 256;  // threads per CTA of both kernels

// ---- k_thph shared-memory layout -----------------------------------------
// A field: 32 main rows (phi index p of the block), each 42 doubles of
// theta t0-4 .. t0+37 (the last two unused; 42 keeps every row 16-byte
// aligned for the asynchronous copies), then 8 phi-halo rows of the 32 theta
// points of the block (p0-4..p0-1, p0+32..p0+35).
constexpr int FA_RW = 42;
constexpr int FA_MAIN = FM * FA_RW;
constexpr int FA_FIELD = FA_MAIN + 8 * FM;
// a derivative tile: 32x32, element (p, t) at p*32 + (t ^ (p & 15)), so
// theta lines (one thread per p), phi lines (one thread per t) and the
// pointwise phase (t across the warp) all touch 16 distinct 8-byte banks
constexpr int FA_OUT = FM * FM;

template <int MAG>
struct ThphCfg {
  static constexpr int NF = MAG ? 8 : 5;     // rho w v u s [bt bp br]
  static constexpr int NO = MAG ? 8 : 6;     // derivative tiles per pass
  static constexpr size_t SMEM = 8 * ((size_t)NF * FA_FIELD + (size_t)NO * FA_OUT);
};

// index maps of the lines (css_lines.cuh: the solver reads xb[xi(j)] and
// writes ob[oi(j)])
// theta line: base = the row start, j = -3..36 -> column j+3
struct ThIdx {
  __device__ __forceinline__ int operator()(int j) const { return j + 3; }
};
// phi line at theta column t: base = the field
struct PhIdx {
  int t;
  __device__ __forceinline__ int operator()(int j) const {
    if (j < 1) return FA_MAIN + (j + 3) * FM + t;
    if (j > FM) return FA_MAIN + (j - FM + 3) * FM + t;
    return (j - 1) * FA_RW + t + 4;
  }
};
struct SwzRow {  // theta line p of a derivative tile: element (p, j)
  int p;
  __device__ __forceinline__ int operator()(int j) const { return p * FM + (j ^ (p & 15)); }
};
struct SwzCol {  // phi line t of a derivative tile: element (j, t)
  int t;
  __device__ __forceinline__ int operator()(int j) const { return j * FM + (t ^ (j & 15)); }
};
__device__ __forceinline__ double swz(const double *O, int p, int t) { return O[p * FM + (t ^ (p & 15))]; }

// ---------------------------------------------------------------------------
// k_thph.  grid: x = theta block * nbp + phi block, y = r.  cur = stage
// input (FP64), bf = B (MHD), dv = tendency (written), tbuf = T (written).
// ---------------------------------------------------------------------------
template <int MAG>
__global__ void __launch_bounds__(FNT, MAG ? 1 : 2) k_thph(CssGeo g, const double *__restrict__ cur,
                                                           const double *__restrict__ bf, double *__restrict__ dv,
                                                           double *__restrict__ tbuf) {
  using C = ThphCfg<MAG>;
  extern __shared__ __align__(16) double sm[];
  double *F = sm;                           // NF fields
  double *O = sm + (size_t)C::NF * FA_FIELD;  // NO derivative tiles
  const CssDir &DT = g.d[1], &DP = g.d[2];
  const int nbp = DP.nb;
  const int bt = blockIdx.x / nbp, bp = blockIdx.x - bt * nbp;
  const int ir = blockIdx.y;
  const int t0 = DT.start[bt], p0 = DP.start[bp];
  const int tid = threadIdx.x;
  const size_t n = (size_t)g.ncell, pl = plane(g, ir);
  const int nth = g.nth, nphi = g.nphi;
  const bool wall = DT.lphys[bt] || DT.rphys[bt];

  // ---- stage the plane: 16-byte copies, zero fill outside [0, nth) ----
  {
    const double *src[8];
    src[0] = cur; src[1] = cur + n; src[2] = cur + 2 * n; src[3] = cur + 3 * n; src[4] = cur + 4 * n;
    if (MAG) { src[5] = bf; src[6] = bf + n; src[7] = bf + 2 * n; }
    constexpr int MAINP = FM * 20, HALOP = 8 * 16, PER = MAINP + HALOP;
    for (int k = tid; k < C::NF * PER; k += FNT) {
      const int f = k / PER, q = k - f * PER;
      int p, tt, dst;
      if (q < MAINP) {
        p = q / 20;
        const int c = (q - p * 20) * 2;
        tt = t0 - 4 + c;
        p += p0;
        dst = (q / 20) * FA_RW + c;
      } else {
        const int h = (q - MAINP) / 16, c = (q - MAINP - h * 16) * 2;
        p = h < 4 ? p0 - 4 + h : p0 + FM + (h - 4);
        if (p < 0) p += nphi;
        else if (p >= nphi) p -= nphi;
        tt = t0 + c;
        dst = FA_MAIN + h * FM + c;
      }
      const bool in = tt >= 0 && tt < nth;
      const double *gp = src[f] + pl + (size_t)p * nth + (in ? tt : 0);
      cp_async16(F + (size_t)f * FA_FIELD + dst, gp, in ? 16 : 0);
    }
    cp_async_commit();
    cp_async_wait<0>();
  }
  __syncthreads();

  const double ri = g.r_inv[ir];
  // ---- theta solves: derivative tile k, line (row) p ----
  {
    // tiles: 0 dw 1 dv 2 du 3 ds 4 d2s [5 dbp 6 dbr] then d(rho) (no wall)
    const int nth_t = (MAG ? 7 : 5) + (wall ? 0 : 1);
    const int dtype = dtype_of(DT, bt);
    const double dn = DT.dnum[bt];
    const int k = tid >> 5, p = tid & 31;
    if (k < nth_t) {
      // field and bdry of each tile (var numbers of ibct)
      int f, var, order = 1;
      if (k < 4) { f = 1 + k; var = 2 + k; }
      else if (k == 4) { f = 4; var = 5; order = 2; }
      else if (MAG && k < 7) { f = k + 1; var = k + 3; }  // bp (8), br (9)
      else { f = 0; var = 1; }
      const int bdry = g.ibct[var];
      const double *x = F + (size_t)f * FA_FIELD + p * FA_RW;
      double lo = 0.0, hi = 0.0;
      if (f == 2) {  // stress-free datum cot(theta)*v on the walls (rhs_mpi.f90:414, :444)
        if (DT.lphys[bt]) lo = (g.cosines[0] / g.sines[0]) * x[4];
        if (DT.rphys[bt]) hi = (g.cosines[nth - 1] / g.sines[nth - 1]) * x[4 + FM - 1];
      }
      if (MAG && f == 6 && g.theta_normal_field) {  // (rhs_mpi.f90:421, :451)
        if (DT.lphys[bt]) lo = -(g.cosines[0] / g.sines[0]) * x[4];
        if (DT.rphys[bt]) hi = -(g.cosines[nth - 1] / g.sines[nth - 1]) * x[4 + FM - 1];
      }
      const int slot = (k == nth_t - 1 && !wall) ? C::NO - 1 : k;
      if (order == 2) {
        if (g.slaplacian)
          line_solve_ua<2, FM>(x, ThIdx{}, dtype, bdry, lo, hi, tabp(g, 1, bt, 2, bdry), g.tstride,
                               dnum_d2_theta(g, ir), dn * dn, 0, O + slot * FA_OUT, SwzRow{p});
      } else {
        line_solve_ua<1, FM>(x, ThIdx{}, dtype, bdry, lo, hi, tabp(g, 1, bt, 1, bdry), g.tstride, dn, dn, 0,
                             O + slot * FA_OUT, SwzRow{p});
      }
    }
  }
  __syncthreads();

  // ---- theta pointwise (Source_Theta_Terms, Lorentz, induction, and
  // Density_Terms_Theta off the walls): 4 points per thread, t = lane ----
  const int lane = tid & 31, wrp = tid >> 5;
  const int it = t0 + lane;
  constexpr int NA = MAG ? 8 : 5;
  double acc[4][NA], tk[4];
  {
    const double rv = g.r_ind[ir], epsr = g.eps[ir];
    const double omsq = rv * g.omega0 * g.omega0, om2 = 2.0 * g.omega0;
    const double sn = g.sines[it], cs = g.cosines[it], ct = g.cot[it];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int p = q * 8 + wrp;
      const int ic = p * FA_RW + lane + 4;
      const double rho = F[ic], w = F[FA_FIELD + ic], v = F[2 * FA_FIELD + ic], u = F[3 * FA_FIELD + ic],
                   s = F[4 * FA_FIELD + ic];
      double dw = omsq * sn * cs;
      double du = -g.grav[ir] + omsq * sn * sn;
      double drho = -rho * w * ct * ri;
      double dvv = -om2 * cs * w;
      du = du + ri * w * w;
      double w1 = swz(O, p, lane) * ri;
      drho = drho - rho * w1;
      dw = dw - w * w1;
      dw = dw + v * (ri * ct * v + om2 * cs);
      dvv = dvv - ri * v * w * ct;
      du = du + v * (ri * v + om2 * sn);
      w1 = swz(O + FA_OUT, p, lane) * ri;
      dvv = dvv - w * w1;
      drho = drho - 2.0 * ri * rho * u;
      dvv = dvv - u * (ri * v + om2 * sn);
      dw = dw - ri * u * w;
      w1 = swz(O + 2 * FA_OUT, p, lane) * ri;
      du = du - w * w1;
      const double t = temp_of(g, rho, s);
      tk[q] = t;
      const double invrho = 1.0 / rho;
      const double oorho_t = invrho / t;
      double ds;
      if (fabs(epsr) > 0.0) ds = epsr * oorho_t;
      else ds = 0.0;
      w1 = swz(O + 3 * FA_OUT, p, lane) * ri;
      dw = dw - g.gamm1 * t * w1;
      ds = ds - w * w1;
      if (g.slaplacian) {
        const double ddiff = ri * g.ks[ir];
        w1 = ddiff * w1 * oorho_t;
        ds = ds + ct * w1;
        const double dd2 = ddiff * ri * ri;  // ks/r^3 as rhs_mpi.f90:972 has it
        ds = ds + dd2 * swz(O + 4 * FA_OUT, p, lane) * oorho_t;
      }
      if (MAG) {
        double oo = invrho;
        oo = oo * ONE_OVER_4PI * ri;
        const double bt_ = F[5 * FA_FIELD + ic], bp_ = F[6 * FA_FIELD + ic], br_ = F[7 * FA_FIELD + ic];
        du = du - bt_ * bt_ * oo;
        dw = dw - bp_ * bp_ * ct * oo;
        dvv = dvv + bp_ * bt_ * ct * oo;
        du = du - bp_ * bp_ * oo;
        w1 = swz(O + 5 * FA_OUT, p, lane) * oo;
        dvv = dvv + bt_ * w1;
        dw = dw - bp_ * w1;
        w1 = swz(O + 6 * FA_OUT, p, lane) * oo;
        dw = dw + br_ * (bt_ * oo - w1);
        dvv = dvv + br_ * bp_ * oo;
        du = du + bt_ * w1;
        acc[q][NA - 3] = v * br_ - u * bp_;  // Induction_Terms: dA/dt = v x B
        acc[q][NA - 2] = u * bt_ - w * br_;
        acc[q][NA - 1] = w * bp_ - v * bt_;
      }
      if (!wall) {  // Density_Terms_Theta (rhs_mpi.f90:1522-1605), halo-closed rows
        w1 = ri * swz(O + (C::NO - 1) * FA_OUT, p, lane);
        drho = drho - w * w1;
        w1 = w1 * (1.0 / rho);
        dw = dw - g.pconst * w1 * t;
      }
      acc[q][0] = drho; acc[q][1] = dw; acc[q][2] = dvv; acc[q][3] = du; acc[q][4] = ds;
    }
    // global stores after every point's shared-memory reads, so the
    // compiler need not order those reads behind them
#pragma unroll
    for (int q = 0; q < 4; q++) tbuf[pl + (size_t)(p0 + q * 8 + wrp) * nth + it] = tk[q];
  }
  __syncthreads();

  // ---- phi solves: tiles 0 drho 1 dv 2 dw 3 du 4 ds 5 d2s [6 dbt 7 dbr] ----
  {
    const int k = tid >> 5, t = tid & 31;
    const int nph = MAG ? 8 : 6;
    if (k < nph) {
      const int f = k == 0 ? 0 : k == 1 ? 2 : k == 2 ? 1 : k == 3 ? 3 : k <= 5 ? 4 : (k == 6 ? 5 : 7);
      const double dn = DP.dnum[bp];
      const double *x = F + (size_t)f * FA_FIELD;
      if (k == 5) {
        if (g.slaplacian)
          line_solve_ua<2, FM>(x, PhIdx{t}, 3, 0, 0.0, 0.0, tabp(g, 2, bp, 2, 0), g.tstride, dn, dn * dn, 1,
                               O + k * FA_OUT, SwzCol{t});
      } else {
        line_solve_ua<1, FM>(x, PhIdx{t}, 3, 0, 0.0, 0.0, tabp(g, 2, bp, 1, 0), g.tstride, dn, dn, 1,
                             O + k * FA_OUT, SwzCol{t});
      }
    }
  }
  __syncthreads();

  // ---- phi pointwise (Phi_Terms + Lorentz), store the tendency ----
  {
    const double oors0 = ri * g.csc[it];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int p = q * 8 + wrp;
      const int ic = p * FA_RW + lane + 4;
      const double rho = F[ic], v = F[2 * FA_FIELD + ic];
      const double t = tk[q], oorho = 1.0 / rho, oors = oors0;
      double drho = acc[q][0], dw = acc[q][1], dvv = acc[q][2], du = acc[q][3], ds = acc[q][4];
      double w1 = swz(O, p, lane) * oors;
      drho = drho - v * w1;
      dvv = dvv - g.pconst * w1 * t * oorho;
      w1 = swz(O + FA_OUT, p, lane) * oors;
      dvv = dvv - v * w1;
      drho = drho - rho * w1;
      w1 = swz(O + 2 * FA_OUT, p, lane) * oors;
      dw = dw - v * w1;
      w1 = swz(O + 3 * FA_OUT, p, lane) * oors;
      du = du - v * w1;
      w1 = swz(O + 4 * FA_OUT, p, lane) * oors;
      ds = ds - v * w1;
      dvv = dvv - g.gamm1 * t * w1;
      if (g.slaplacian) {
        w1 = swz(O + 5 * FA_OUT, p, lane) * (oors * oors);
        ds = ds + g.ks[ir] * w1 * (oorho / t);
      }
      if (MAG) {
        const double oo = ONE_OVER_4PI * oorho * oors;
        const double bt_ = F[5 * FA_FIELD + ic], bp_ = F[6 * FA_FIELD + ic], br_ = F[7 * FA_FIELD + ic];
        w1 = swz(O + 6 * FA_OUT, p, lane) * oo;
        dvv = dvv - bt_ * w1;
        dw = dw + bp_ * w1;
        w1 = swz(O + 7 * FA_OUT, p, lane) * oo;
        dvv = dvv - br_ * w1;
        du = du + bp_ * w1;
      }
      acc[q][0] = drho; acc[q][1] = dw; acc[q][2] = dvv; acc[q][3] = du; acc[q][4] = ds;
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const size_t id = pl + (size_t)(p0 + q * 8 + wrp) * nth + it;
#pragma unroll
      for (int f = 0; f < NA; f++) dv[f * n + id] = acc[q][f];
    }
  }
}

// ---- k_rstage ----------------------------------------------------------------
// The slab: field f at H + f*FB_FIELD, row rr = 0..39 (r = r0-4+rr), 32
// theta values per row.  Derivative tiles O + k*FB_OUT, row r - r0.
constexpr int FB_FIELD = (FM + 8) * FM;
constexpr int FB_OUT = FM * FM;
template <int MAG>
struct RstageCfg {
  static constexpr int NH = MAG ? 7 : 5;  // w v u s rho [bt bp]
  static constexpr int ND = MAG ? 8 : 6;  // dw dv du ds d2s drho0 [dbt dbp]
  static constexpr size_t SMEM = 8 * ((size_t)NH * FB_FIELD + (size_t)ND * FB_OUT + 2 * FM);
};
// the theta-wall pass reuses the derivative tiles: rho rows with their theta
// halo (stride 41) and the d(rho)/dtheta rows (stride 33)
constexpr int FB_XS = 41, FB_YS = 33;

// STG: the RK4 stage (1..4), compiled in:
//   1: vs = (sld ? vs + dv/6 : dv); nx = v0 + dtcur*dv
//   2,3: vs = vs + dv/3;            nx = v0 + dtcur*dv
//   4: vs + dv/6 accumulated;       nx = v0 + dtcur*(vs + dv/6)  (nx is v0)
template <int MAG, int STG>
__global__ void __launch_bounds__(FNT, MAG ? 1 : 2) k_rstage(CssGeo g, const double *__restrict__ cur,
                                                             const double *__restrict__ bf, const double *dv,
                                                             const double *v0, double *vs, double *nx,
                                                             const double *__restrict__ tbuf, double dtcur,
                                                             int *flag) {
  using C = RstageCfg<MAG>;
  extern __shared__ __align__(16) double sm[];
  double *H = sm;
  double *O = sm + (size_t)C::NH * FB_FIELD;
  double *datum = O + (size_t)C::ND * FB_OUT;  // [0, 32): radial face datum per line; [32, 64): theta wall datum per row
  const CssDir &D = g.d[0], &DT = g.d[1];
  const int nbt = DT.nb;
  const int br = blockIdx.x / nbt, bt = blockIdx.x - br * nbt;
  const int ip = blockIdx.y;
  const int r0 = D.start[br], t0 = DT.start[bt];
  const int tid = threadIdx.x, lane = tid & 31, wrp = tid >> 5;
  const size_t n = (size_t)g.ncell, ps = (size_t)g.nth * g.nphi;
  const size_t base = (size_t)ip * g.nth + t0;  // (theta t0, phi ip) of plane 0
  const int nr = g.nr;

  // Lines the later phases read, toward L2 now (two 128-byte halves per
  // row): the tendency, T [and B_r] for the pointwise phase; vars0 and the
  // accumulator for the stage combination
  {
    const int nv = MAG ? 8 : 5;
    const bool need_s = !(STG == 1 && !g.sldiffusion);
    const int per = 2 * nv + 1 + (MAG ? 1 : 0) + (need_s ? nv : 0);
    for (int k = tid; k < 2 * FM * per; k += FNT) {
      const int row = k / per, f = k - row * per;
      const size_t id = base + (size_t)(r0 + (row >> 1)) * ps + (row & 1) * 16;
      const double *src;
      if (f < nv) src = dv + f * n;
      else if (f < 2 * nv) src = v0 + (f - nv) * n;
      else if (f == 2 * nv) src = tbuf;
      else if (MAG && f == 2 * nv + 1) src = bf + 2 * n;
      else src = vs + (f - 2 * nv - 1 - (MAG ? 1 : 0)) * n;
      prefetch_l2(src + id);
    }
  }
  // ---- stage the slab: 16-byte copies, zero fill outside [0, nr) ----
  {
    const double *src[7] = {cur + n, cur + 2 * n, cur + 3 * n, cur + 4 * n, cur, MAG ? bf : cur, MAG ? bf + n : cur};
    constexpr int PER = (FM + 8) * 16;
    for (int k = tid; k < C::NH * PER; k += FNT) {
      const int f = k / PER, q = k - f * PER;
      const int rr = q >> 4, c = (q & 15) * 2;
      const int gr = r0 - 4 + rr;
      const bool in = gr >= 0 && gr < nr;
      const double *gp = src[f] + (in ? (size_t)gr * ps + base + c : 0);
      cp_async16(H + (size_t)f * FB_FIELD + rr * FM + c, gp, in ? 16 : 0);
    }
    cp_async_commit();
    cp_async_wait<0>();
  }
  __syncthreads();

  // ---- radial solves: tile k, line t ----
  const int dtype = dtype_of(D, br);
  {
    const int var[8] = {2, 3, 4, 5, 5, 1, 7, 8};
    const int k = tid >> 5, l = tid & 31;
    if (k < C::ND && !(k == 4 && !g.slaplacian)) {
      const int hk = (k <= 3) ? k : (k == 4 ? 3 : (k == 5 ? 4 : k - 1));
      const double *x = H + (size_t)hk * FB_FIELD + 4 * FM + l;
      const int bdry = g.ibcr[var[k]];
      double lo = 0.0, hi = 0.0;
      if (k == 0 || k == 1) {  // stress-free datum w/r/dxdr (rhs_mpi.f90:578-614)
        if (D.lphys[br] && g.bottom_stress_free) lo = x[0] / g.r1 / g.dxdr[0];
        if (D.rphys[br]) {
          if (g.top_stress_free) hi = x[(FM - 1) * FM] / g.r2 / g.dxdr[nr - 1];
          else hi = x[(FM - 1) * FM];
        }
      }
      if (k == 3 || k == 4) {  // constant-flux datum (rhs_mpi.f90:584-592, :616-624)
        lo = g.s_flux_lo;
        hi = g.s_flux_hi;
      }
      const double dn = D.dnum[br];
      if (k == 4)
        line_solve_ua<2, FM>(x, StridedIn{FM}, dtype, bdry, lo, hi, tabp(g, 0, br, 2, bdry), g.tstride, dn, dn * dn,
                             0, O + k * FB_OUT + l, StridedOut{FM});
      else
        line_solve_ua<1, FM>(x, StridedIn{FM}, dtype, bdry, lo, hi, tabp(g, 0, br, 1, bdry), g.tstride, dn, dn, 0,
                             O + k * FB_OUT + l, StridedOut{FM});
    }
  }
  __syncthreads();

  auto gather = [&](int j, int l, RadIn &q, double t, double brv) {
    const double *hl = H + (size_t)(j + 4) * FM + l;
    const double *ol = O + (size_t)j * FM + l;
    q.u = hl[2 * FB_FIELD];
    q.rho = hl[4 * FB_FIELD];
    q.t = t;
    q.dw_r = ol[0]; q.dv_r = ol[FB_OUT]; q.du_r = ol[2 * FB_OUT]; q.ds_r = ol[3 * FB_OUT]; q.d2s_r = ol[4 * FB_OUT];
    if (MAG) {
      q.bt = hl[5 * FB_FIELD]; q.bp = hl[6 * FB_FIELD]; q.br = brv;
      q.dbt_r = ol[6 * FB_OUT]; q.dbp_r = ol[7 * FB_OUT];
    }
  };
  // hydrostatic datum of d(rho)/dr on a physical radial face (rhs_mpi.f90:1750-1768)
  const int phys = D.lphys[br] ? 1 : (D.rphys[br] ? 2 : 0);
  if (phys) {
    if (tid < FM) {
      const int j = phys == 1 ? 0 : FM - 1, l = tid;
      const size_t id = base + (size_t)(r0 + j) * ps + l;
      RadIn q;
      gather(j, l, q, __ldg(tbuf + id), MAG ? __ldg(bf + 2 * n + id) : 0.0);
      double drho = dv[id], dw = dv[n + id], dvv = dv[2 * n + id], du = dv[3 * n + id], ds = dv[4 * n + id];
      radial_point<MAG>(g, r0 + j, q, drho, dw, dvv, du, ds);
      double d;
      if (g.lbcr_rho == 4 || g.lbcr_rho == (phys == 1 ? 2 : 3)) d = du * q.rho * g.invpconst / q.t;
      else d = q.rho;
      if (g.non_uniform) d = d / g.dxdr[phys == 1 ? 0 : nr - 1];
      datum[l] = d;
    }
    __syncthreads();
  }

  // ---- radial pointwise: 4 points per thread (row j = q*8 + warp, t = lane) ----
  const double *resp = g.resp_r + (size_t)(2 * br + (phys == 2 ? 1 : 0)) * g.tstride;
  double d[4][5], tk[4];
  {
    double in[4][7];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int j = q * 8 + wrp;
      const size_t id = base + (size_t)(r0 + j) * ps + lane;
      in[q][0] = __ldg(dv + id); in[q][1] = __ldg(dv + n + id); in[q][2] = __ldg(dv + 2 * n + id);
      in[q][3] = __ldg(dv + 3 * n + id); in[q][4] = __ldg(dv + 4 * n + id); in[q][5] = __ldg(tbuf + id);
      in[q][6] = MAG ? __ldg(bf + 2 * n + id) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int j = q * 8 + wrp, ir = r0 + j;
      RadIn qq;
      gather(j, lane, qq, in[q][5], in[q][6]);
      double drho = in[q][0], dw = in[q][1], dvv = in[q][2], du = in[q][3], ds = in[q][4];
      radial_point<MAG>(g, ir, qq, drho, dw, dvv, du, ds);
      double w1 = O[5 * FB_OUT + (size_t)j * FM + lane];  // Density_Terms_Radial
      if (phys) w1 = w1 + datum[lane] * resp[j + 1];
      if (g.non_uniform) w1 = w1 * g.dxdr[ir];
      drho = drho - qq.u * w1;
      w1 = w1 * (1.0 / qq.rho);
      du = du - g.pconst * qq.t * w1;
      if (phys == 2 && j == FM - 1 && !g.set_stop) {  // rhs_mpi.f90:1807-1818
        drho = drho + qq.rho * (g.t0 - qq.t) / (g.damping_time * (g.gamma - 2.0) * qq.t);
        ds = ds - g.cv * (g.t0 - qq.t) / (g.damping_time * (g.gamma - 2.0) * qq.t);
      }
      d[q][0] = drho; d[q][1] = dw; d[q][2] = dvv; d[q][3] = du; d[q][4] = ds;
      tk[q] = qq.t;
    }
  }

  // ---- Density_Terms_Theta on a theta-wall block (rhs_mpi.f90:1522-1605):
  // its wall datum makes dw/dt vanish on the wall, so it needs the completed
  // dw/dt there; the other blocks had it in k_thph ----
  const bool lw = DT.lphys[bt], hw = DT.rphys[bt];
  if (lw || hw) {
    const int tw = lw ? 0 : FM - 1;
    __syncthreads();  // the derivative tiles are free from here on
    double *X = O, *Y = O + FM * FB_XS;
    if (lane == tw) {
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int j = q * 8 + wrp;
        const double rho = H[4 * FB_FIELD + (size_t)(j + 4) * FM + tw];
        datum[FM + j] = g.r_ind[r0 + j] * g.invpconst * d[q][1] * rho / tk[q];
      }
    }
    // rho rows with the theta halo of the inner side: X[j][c], c = t+4
    for (int k = tid; k < FM * FM; k += FNT) {
      const int j = k >> 5, c = k & 31;
      X[j * FB_XS + c + 4] = H[4 * FB_FIELD + (size_t)(j + 4) * FM + c];
    }
    for (int k = tid; k < FM * 4; k += FNT) {
      const int j = k >> 2, h = k & 3;
      const int c = lw ? FM + 4 + h : h;      // X column
      const int gt = t0 - 4 + c;              // theta index of the neighbour block
      X[j * FB_XS + c] = cur[base - t0 + (size_t)(r0 + j) * ps + gt];
    }
    __syncthreads();
    if (tid < FM) {
      const int j = tid;
      const int bdry = g.ibct[1];
      const double dn = DT.dnum[bt];
      const double lo = lw ? datum[FM + j] : 0.0, hi = hw ? datum[FM + j] : 0.0;
      line_solve_ua<1, FM>(X + j * FB_XS + 4, StridedIn{1}, dtype_of(DT, bt), bdry, lo, hi,
                           tabp(g, 1, bt, 1, bdry), g.tstride, dn, dn, 0, Y + j * FB_YS, StridedOut{1});
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int j = q * 8 + wrp;
      const double w = H[(size_t)(j + 4) * FM + lane], rho = H[4 * FB_FIELD + (size_t)(j + 4) * FM + lane];
      double w1 = g.r_inv[r0 + j] * Y[j * FB_YS + lane];
      d[q][0] = d[q][0] - w * w1;
      w1 = w1 * (1.0 / rho);
      d[q][1] = d[q][1] - g.pconst * w1 * tk[q];
    }
  }

  // ---- stage combination (Step_RK4, step_rk4.f90:385-475) and Bound
  // (rhs_mpi.f90:2395-2491), field by field ----
  const int nv = MAG ? 8 : 5;
  const int it = t0 + lane;
  const bool twall = (it == 0 || it == g.nth - 1);
  int bad = 0;
#pragma unroll
  for (int q = 0; q < 4; q++)
    if (g.xi_cs < 1.0) d[q][0] = (g.xi_cs * g.xi_cs) * d[q][0];
  // Every value is read once, before the same thread writes that address
  // (nx is vars0 in stage 4), and no other thread touches it, so the reads
  // go through the non-coherent path; the compiler may then start the next
  // field's reads before this field's stores.
#pragma unroll
  for (int iv = 0; iv < nv; iv++) {
    double dd[4], aa[4], ss[4];
    const bool need_s = !(STG == 1 && !g.sldiffusion);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int j = q * 8 + wrp;
      const size_t qi = (size_t)iv * n + base + (size_t)(r0 + j) * ps + lane;
      dd[q] = (iv < 5) ? d[q][iv < 5 ? iv : 0] : __ldg(dv + qi);
      aa[q] = __ldg(v0 + qi);
      ss[q] = need_s ? __ldg(vs + qi) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int j = q * 8 + wrp, ir = r0 + j;
      const size_t qi = (size_t)iv * n + base + (size_t)ir * ps + lane;
      const double dd_ = dd[q], a = aa[q];
      double o;
      if (STG == 1) {
        const double sv = g.sldiffusion ? ss[q] + dd_ / 6.0 : dd_;
        vs[qi] = sv;
        o = a + dtcur * dd_;
      } else if (STG == 4) {
        const double sv = ss[q] + dd_ / 6.0;
        o = a + dtcur * sv;
      } else {
        const double sv = ss[q] + dd_ / 3.0;
        vs[qi] = sv;
        o = a + dtcur * dd_;
      }
      const bool rlo = (ir == 0), rhi = (ir == nr - 1);
      if (twall || rlo || rhi) {
        if (iv == 1 && twall) o = 0.0;
        if (iv == 3 && !g.theta_stress_free && twall) o = 0.0;
        if (rlo) {
          if ((iv == 1 || iv == 2) && !g.bottom_stress_free) o = 0.0;
          if (iv == 3) o = 0.0;
        }
        if (rhi) {
          if ((iv == 1 || iv == 2) && !g.top_stress_free) o = 0.0;
          if (iv == 3) o = 0.0;
        }
        if (iv >= 5) {
          if (g.theta_perf_conductor) {
            if ((iv == 6 || iv == 7) && twall) o = 0.0;
          } else if (iv == 5 && twall) {
            o = 0.0;
          }
          if (rlo) {
            if (g.bottom_radial_field) { if (iv == 7) o = 0.0; }
            else if (g.bottom_perfect_cond) { if (iv == 5 || iv == 6) o = 0.0; }
          }
          if (rhi) {
            if (g.top_radial_field) { if (iv == 7) o = 0.0; }
            else if (g.top_perfect_cond) { if (iv == 5 || iv == 6) o = 0.0; }
          }
        }
      }
      if (!isfinite(o)) bad = 1;
      nx[qi] = o;
    }
  }
  if (bad && flag) atomicOr(flag, 1);
}

}  // namespace css
