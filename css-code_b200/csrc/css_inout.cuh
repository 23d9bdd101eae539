// css_inout.cuh -- open radial boundaries: the face sums and scalars of
// Top_Inflow_Outflow (rhs_mpi.f90:1955-2067) and Bottom_Inflow_Outflow
// (:1857-1953), the mass totals they relax toward (mhdsph_mpi.f90:863-999,
// rhs_mpi.f90:326-353), the rain-squall fields (Build_Gaussian_Squalls,
// entropy_rain.f90:423-523), the time interpolation of the prescribed
// bottom fields (Cubic_Time_Interp, ash_inflow.f90:188-219) and the ASH
// enthalpy-flux factor (ASH_Enthalpy_Flux, step_rk4.f90:495-518).  The
// per-cell terms themselves are applied in k_radial_terms; Bound's open-
// face exceptions live in k_rhot_update.
//
// Sums run per virtual block in a fixed tree order and the blocks are then
// added in block order, as the reference's ranks each sum their own part
// before the face communicator's reduction: the results are deterministic.
#pragma once
#include <math_constants.h>

#include "css_geo.cuh"

namespace css {

constexpr int IO_NT = 256;  // threads of the reduction kernels

// deterministic CTA sum of one value per thread (IO_NT threads)
__device__ __forceinline__ double io_block_sum(double x, double *sh) {
  sh[threadIdx.x] = x;
  __syncthreads();
  for (int s = IO_NT / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] = sh[threadIdx.x] + sh[threadIdx.x + s];
    __syncthreads();
  }
  double r = sh[0];
  __syncthreads();
  return r;
}
__device__ __forceinline__ double io_block_min(double x, double *sh) {
  sh[threadIdx.x] = x;
  __syncthreads();
  for (int s = IO_NT / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] = fmin(sh[threadIdx.x], sh[threadIdx.x + s]);
    __syncthreads();
  }
  double r = sh[0];
  __syncthreads();
  return r;
}

// One CTA per (theta block, phi block) of the open faces.  part[8*b + k]:
// top 0 sum u rho sin, 1 sum rho sin, 2 sum s, 3 sum rho sin (dvel_rain +
// u(nr-1)); bottom 4 sum rho(mynr) sin u(1), 5 sum rho(mynr) sin, 6 sum s(1),
// 7 |min u(2)| (1-based radii, as rhs_mpi.f90:1865-1878 and :1971-1998 read
// them; mynr is the bottom block's own top radius).
__global__ void __launch_bounds__(IO_NT) k_inout_sums(CssGeo g, const double *__restrict__ v,
                                                      double *__restrict__ part) {
  __shared__ double sh[IO_NT];
  const int jb = blockIdx.x / g.d[2].nb, kb = blockIdx.x - jb * g.d[2].nb;
  const int t0 = g.d[1].start[jb], nt = g.d[1].size[jb], p0 = g.d[2].start[kb], np_ = g.d[2].size[kb];
  const size_t n = (size_t)g.ncell;
  const int nr = g.nr, cells = nt * np_;
  double a[8];
  for (int k = 0; k < 8; k++) a[k] = 0.0;
  double umin = CUDART_INF;
  const bool top = g.top_inout, bot = g.bot_inout && !g.bottom_specified;
  const int mt = g.d[0].size[0] - 1;
  for (int q = threadIdx.x; q < cells; q += IO_NT) {
    const int ip = p0 + q / nt, it = t0 + q % nt;
    const double sn = g.sines[it];
    if (top) {
      const size_t id = css_idx(g, it, ip, nr - 1);
      const double tau = v[id] * sn;
      a[0] += v[3 * n + id] * tau;
      a[1] += tau;
      a[2] += v[4 * n + id];
      if (g.rain) a[3] += tau * (g.dvel_rain[it + (size_t)g.nth * ip] + v[3 * n + css_idx(g, it, ip, nr - 2)]);
    }
    if (bot) {
      const size_t i0 = css_idx(g, it, ip, 0);
      const double tau = v[css_idx(g, it, ip, mt)] * sn;
      a[4] += tau * v[3 * n + i0];
      a[5] += tau;
      a[6] += v[4 * n + i0];
      umin = fmin(umin, v[3 * n + css_idx(g, it, ip, 1)]);
    }
  }
  for (int k = 0; k < 7; k++) a[k] = io_block_sum(a[k], sh);
  umin = io_block_min(umin, sh);
  if (threadIdx.x == 0) {
    for (int k = 0; k < 7; k++) part[8 * blockIdx.x + k] = a[k];
    part[8 * blockIdx.x + 7] = fabs(umin);
  }
}

// The face scalars of this RHS from the block parts (one thread; at most
// CSS_MAXBLK^2 parts).  Every formula follows the reference line cited.
__global__ void k_inout_scalars(CssGeo g, const double *__restrict__ part, double *io, double deltat,
                                double sim_time) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int nb = g.d[1].nb * g.d[2].nb, nr = g.nr;
  double s[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int b = 0; b < nb; b++) {
    for (int k = 0; k < 7; k++) s[k] = s[k] + part[8 * b + k];
    s[7] = fmax(s[7], part[8 * b + 7]);  // 'csm': the last entry is a max (mhdsph_mpi.f90:1511-1521)
  }
  const double ntot = (double)g.nth * (double)g.nphi;
  const double c_top = sqrt(g.gamm1 * g.cp * g.t0);  // sqrt(gamm1 Cp Tr(nr)), Tr(nr) = T0 (mhdsph_mpi.f90:343)
  if (g.top_inout) {  // rhs_mpi.f90:2003-2017, :1982
    const double tau = c_top / g.dr_ind[nr - 1] / 20.0;
    io[IO_TOP_TAU] = tau;
    io[IO_TOP_MEANU] = -s[0] / s[1] / deltat;
    io[IO_TOP_MEANS] = tau * (g.sr[0] + g.delta_s - s[2] / ntot);
    io[IO_TOP_MDVEL] = -s[3] / s[1];
    io[IO_TOP_NRAT] = g.rhor[nr - 2] / g.rhor[nr - 1];
    const int r0 = g.d[0].start[g.d[0].nb - 1];
    double q = (g.r_ind[nr - 1] - g.r_ind[r0]) / (g.r2 - g.r_ind[r0]);
    q = (q * q) * (q * q);
    io[IO_TOP_TAUR] = c_top * q / g.dr_ind[nr - 1] / 2.0;
  }
  if (g.bot_inout) {
    const double m0 = io[IO_M0], vol = io[IO_VOL], mtot = io[IO_MTOT];
    if (g.bottom_specified) {  // rhs_mpi.f90:1913-1916
      const double tau = c_top / (20.0 * g.dr_ind[0]);
      const double tconst = fmin(fabs(sim_time) / 1e5, 1.0);
      io[IO_BOT_TAU] = tau;
      io[IO_BOT_TCONST] = tconst;
      io[IO_BOT_MEANU] = tau * (m0 - mtot) / vol;
      io[IO_BOT_FEN] = tconst * io[IO_ASH_FEN_MOD];
    } else {  // :1880-1888, :1940
      const double tau = s[7] / g.dr_ind[0];
      io[IO_BOT_TAU] = tau;
      io[IO_BOT_MEANU] = -s[4] / s[5] / deltat;
      io[IO_BOT_MEANS] = g.sr[0] - s[6] / ntot;
      io[IO_BOT_NRAT] = g.rhor[1] / g.rhor[0];
      io[IO_BOT_TCONST] = tau * (m0 - mtot) / vol;
    }
  }
}

// part[ir] = dr r^2 * (sum over the plane of sin rho), one CTA per radius
// (the mass total of rhs_mpi.f90:326-353; the lines are summed in a tree)
__global__ void __launch_bounds__(IO_NT) k_plane_mass(CssGeo g, const double *__restrict__ v,
                                                      double *__restrict__ part) {
  __shared__ double sh[IO_NT];
  const int ir = blockIdx.x;
  const size_t np = (size_t)g.nth * g.nphi, pl = (size_t)ir * np;
  double a = 0.0, vl = 0.0;
  for (size_t q = threadIdx.x; q < np; q += IO_NT) {
    const double sn = g.sines[q % g.nth];
    a += sn * v[pl + q];
    vl += sn;
  }
  a = io_block_sum(a, sh);
  vl = io_block_sum(vl, sh);
  if (threadIdx.x == 0) {
    const double rt = g.dr_ind[ir] * (g.r_ind[ir] * g.r_ind[ir]);
    part[ir] = a * rt;
    part[g.nr + ir] = vl * rt / (double)g.nphi;  // the volume, summed over theta only (mhdsph_mpi.f90:877)
  }
}

// io[slot] = dth dphi * sum over radii of part (in radius order); with
// slot_vol >= 0 also the volume
__global__ void k_mass_finish(CssGeo g, const double *__restrict__ part, double *io, int slot, int slot_vol) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double m = 0.0, vl = 0.0;
  for (int ir = 0; ir < g.nr; ir++) {
    m = m + part[ir];
    vl = vl + part[g.nr + ir];
  }
  io[slot] = m * g.dth * g.dphi;
  if (slot_vol >= 0) io[slot_vol] = vl * g.dth * g.dphi;
}

// ashv[iq] = Catmull-Rom interpolation of the four slices at mu
// (Cubic_Time_Interp, ash_inflow.f90:199-216)
__global__ void k_ash_interp(const double *__restrict__ slices, size_t np, double mu, double *__restrict__ ashv) {
  const double mu2 = mu * mu, mu3 = mu * mu2;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < 4 * np; i += (size_t)gridDim.x * blockDim.x) {
    const size_t iq = i / np, q = i - iq * np;
    const double t1 = slices[(0 * 4 + iq) * np + q], a3 = slices[(1 * 4 + iq) * np + q];
    const double t3 = slices[(2 * 4 + iq) * np + q], t4 = slices[(3 * 4 + iq) * np + q];
    const double a0 = -0.5 * t1 + 1.5 * a3 - 1.5 * t3 + 0.5 * t4;
    const double a1 = t1 - 2.5 * a3 + 2.0 * t3 - 0.5 * t4;
    const double a2 = -0.5 * t1 + 0.5 * t3;
    ashv[i] = a0 * mu3 + a1 * mu2 + a2 * mu + a3;
  }
}

// ASH_Enthalpy_Flux (step_rk4.f90:495-518) on the bottom plane of the new
// state with the last stage's temperature; one CTA, two passes
__global__ void __launch_bounds__(IO_NT) k_ash_flux(CssGeo g, const double *__restrict__ v,
                                                    const double *__restrict__ tb, double *io, double sim_time,
                                                    double four_pi) {
  __shared__ double sh[IO_NT];
  const size_t n = (size_t)g.ncell, np = (size_t)g.nth * g.nphi;
  const double ntot = (double)g.nphi * (double)g.nth;
  double su = 0.0, st = 0.0;
  for (size_t q = threadIdx.x; q < np; q += IO_NT) {
    su += v[3 * n + q];
    st += tb[q];
  }
  su = io_block_sum(su, sh);
  st = io_block_sum(st, sh);
  const double uravg = su / ntot, t2avg = st / ntot;
  double len = 0.0;
  for (size_t q = threadIdx.x; q < np; q += IO_NT) len += v[q] * (v[3 * n + q] - uravg) * (tb[q] - t2avg);
  len = io_block_sum(len, sh);
  if (threadIdx.x == 0) {
    len = g.cp * len / ntot;
    len = four_pi * (g.r1 * g.r1) * len / g.lumr1;
    len = 1.3 * fmin(1.0 / fmin(2.0, fmax(0.0, fabs(len))), 2.0);
    double f = 0.5 * (len + io[IO_ASH_FEN_MOD]);
    if (fmin(fabs(sim_time) / 1e5, 1.0) < 1.0) f = 1.0;
    io[IO_ASH_FEN_MOD] = f;
  }
}

// Build_Gaussian_Squalls (entropy_rain.f90:423-523) or, with poly,
// Build_Polynomial_Squalls (:525-655, the density summing |term|), one
// thread per top-plane cell.  sq: 8 per squall (theta_loc, phi_loc, size, scaling, vel, dels,
// loct, locp; loct/locp 1-based as Find_Position makes them).  A cell's
// block sees a squall whose centre lies within one block width of it, with
// the periodic images on the first and last phi blocks; terms below 1e-5
// are dropped (polynomials: beyond the squall's size).
__global__ void k_squalls(CssGeo g, const double *__restrict__ sq, int nsq, int poly, double phi1, double phi2,
                          int add, double *__restrict__ dvel, double *__restrict__ dent) {
  const size_t np = (size_t)g.nth * g.nphi;
  for (size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x; id < np; id += (size_t)gridDim.x * blockDim.x) {
    const int it = (int)(id % g.nth), ip = (int)(id / g.nth);
    int jb = 0, kb = 0;
    while (jb + 1 < g.d[1].nb && g.d[1].start[jb + 1] <= it) jb++;
    while (kb + 1 < g.d[2].nb && g.d[2].start[kb + 1] <= ip) kb++;
    const int myth1 = g.d[1].start[jb] + 1, mynth = g.d[1].size[jb], myth2 = myth1 + mynth - 1;
    const int myphi1 = g.d[2].start[kb] + 1, mynphi = g.d[2].size[kb], myphi2 = myphi1 + mynphi - 1;
    const double th = g.theta[it], ph = g.dphi * (double)ip + phi1;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int pass = 0; pass < 2; pass++) {
      const double dens = pass ? 1.0 / (acc[0] + 1.0) : 0.0;
      for (int is = 0; is < nsq; is++) {
        const double *q = sq + 8 * is;
        const int lct = (int)q[6], lcp = (int)q[7];
        if (!(lct + mynth >= myth1 && lct - mynth <= myth2)) continue;
        const double w2 = (g.r2 / q[2]) * (g.r2 / q[2]);
        const double dt_ = th - q[0], thtmp = dt_ * dt_;
        for (int a = 0; a < 3; a++) {
          double dp = ph - q[1];
          if (a == 0) {
            if (!(lcp + mynphi >= myphi1 && lcp - mynphi <= myphi2)) continue;
          } else if (a == 1) {
            if (!(lcp + mynphi > g.nphi && myphi1 == 1)) continue;
            dp = dp + phi2 - phi1;
          } else {
            if (!(lcp - mynphi < 1 && myphi2 == g.nphi)) continue;
            dp = dp - phi2 + phi1;
          }
          double val;
          if (poly) {  // Build_Polynomial_Squalls (entropy_rain.f90:525-655)
            const double e = (thtmp + dp * dp) * w2;
            if (!(e <= 1.0)) continue;
            const double tt = sqrt(e), x1 = tt * tt, x2 = x1 * tt, x3 = x2 * tt;
            const double f = 1.0 - 18.0 * x1 + 32.0 * x2 - 15.0 * x3;
            val = pass == 0 ? fabs(q[3] * f) : q[3] * dens * f;
          } else {
            const double e = -(thtmp + dp * dp) * w2;
            if (!(e > -11.5)) continue;
            val = q[3] * exp(e);
            if (pass) val = val * dens;
          }
          if (pass == 0) {
            acc[0] += val;
          } else {
            acc[1] += q[4] * val;
            acc[2] += q[5] * val;
          }
        }
      }
    }
    if (add) {  // on top of the downflow lanes, as Update_Rain_Squalls builds them after the lanes
      dvel[id] += acc[1];
      dent[id] += acc[2];
    } else {
      dvel[id] = acc[1];
      dent[id] = acc[2];
    }
  }
}

// Build_Downflow_Lanes (entropy_rain.f90:657-713), one thread per top-plane
// cell.  smp: 3 per lane sample (phi, theta, scaling of its cell), in the
// reference's order (cell, edge, point along the edge).  A sample counts
// for a cell when it lies in the window of the cell's block: the block's
// theta and phi range widened by xsz in phi and ysz in theta, as each top
// rank's window is.  The cell's sum of scaling * exp(-rtmp * distance^2)
// runs in sample order; a term whose exponent is below -746 is zero in
// double precision and is skipped.  *maxbits collects the largest sum
// (sums are non-negative, so their bit patterns order as the values do).
__global__ void k_lanes(CssGeo g, const double *__restrict__ smp, int ns, double phi1, double xsz, double ysz,
                        double rtmp, double *__restrict__ dvel, unsigned long long *__restrict__ maxbits) {
  const size_t np = (size_t)g.nth * g.nphi;
  for (size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x; id < np; id += (size_t)gridDim.x * blockDim.x) {
    const int it = (int)(id % g.nth), ip = (int)(id / g.nth);
    int jb = 0, kb = 0;
    while (jb + 1 < g.d[1].nb && g.d[1].start[jb + 1] <= it) jb++;
    while (kb + 1 < g.d[2].nb && g.d[2].start[kb + 1] <= ip) kb++;
    const int t0 = g.d[1].start[jb], t1 = t0 + g.d[1].size[jb] - 1;
    const int p0 = g.d[2].start[kb], p1 = p0 + g.d[2].size[kb] - 1;
    const double xlo = g.dphi * (double)p0 + phi1 - xsz, xhi = g.dphi * (double)p1 + phi1 + xsz;
    const double ylo = g.theta[t0] - ysz, yhi = g.theta[t1] + ysz;
    const double th = g.theta[it], ph = g.dphi * (double)ip + phi1;
    double acc = 0.0;
    for (int s = 0; s < ns; s++) {
      const double xv = smp[3 * s], yv = smp[3 * s + 1];
      if (!(xv >= xlo && xv <= xhi && yv >= ylo && yv <= yhi)) continue;
      const double a = th - yv, b = ph - xv;
      const double e = rtmp * (a * a + b * b);
      if (e <= 746.0) acc += smp[3 * s + 2] * exp(-e);
    }
    dvel[id] = acc;
    atomicMax(maxbits, (unsigned long long)__double_as_longlong(acc));
  }
}

// the lanes' normalisation: dvel / max(largest, 1), then dent = meands
// times it and dvel = meanvel times it (entropy_rain.f90:708-712)
__global__ void k_lanes_scale(size_t np, const unsigned long long *__restrict__ maxbits, double meanvel,
                              double meands, double *__restrict__ dvel, double *__restrict__ dent) {
  const double m = fmax(__longlong_as_double((long long)*maxbits), 1.0);
  for (size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x; id < np; id += (size_t)gridDim.x * blockDim.x) {
    const double d = dvel[id] / m;
    dent[id] = meands * d;
    dvel[id] = meanvel * d;
  }
}

}  // namespace css
