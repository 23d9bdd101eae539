// css_lap.cuh -- explicit viscosity (the reference's Laplacian switch) and
// radiative diffusion (do_radheat), the two diffusion options that run as a
// pass of line derivatives plus pointwise kernels around the fused sweeps.
//
// The viscous terms of Source_Theta_Terms (rhs_mpi.f90:844-927), Phi_Terms
// (:1123-1199) and Radial_Terms (:1317-1435), and the cross terms of
// Laplacian_Cross_Terms_Radial / _Theta (:2070-2296), as one pass that runs
// after the phi sweep and before the radial kernel (which reads du at the
// walls for the density datum) and the density-theta / update kernel (dw at
// the walls).  The pass is: per direction, the first and second derivatives
// of w, v, u by the generic line kernels (k_deriv_*, the same compact
// solves), then one pointwise kernel that adds that direction's terms into
// the tendency and keeps the derivative fields the cross terms need; then
// the radial and theta derivatives of those fields and a last pointwise
// kernel.  Every kernel here is HBM-bound (a few FP64 loads and stores per
// cell); the derivative kernels move 16 B per cell each.
//
// Buffers: S[0..5] six derivative fields of the current direction; L[0..5]
// the fields the sweeps leave for the cross terms (the reference's vars2):
//   L0 = ri dw/dth, L1 = ri dv/dth, L2 = ri du/dth,
//   L3 = dv/dph/(r sin), L4 = dw/dph/(r sin), L5 = du/dph/(r sin).
// Tendency layout dv[iv*n + id]: 1 w, 2 v, 3 u, 4 s.
#pragma once
#include "css_geo.cuh"

namespace css {

#define LAP_13 (1.0 / 3.0)
#define LAP_23 (2.0 / 3.0)
#define LAP_43 (4.0 / 3.0)
#define LAP_73 (7.0 / 3.0)

__device__ __forceinline__ void lap_cell(const CssGeo &g, size_t id, int &it, int &ip, int &ir) {
  const size_t pl = (size_t)g.nth * g.nphi;
  ir = (int)(id / pl);
  const size_t rem = id - (size_t)ir * pl;
  ip = (int)(rem / g.nth);
  it = (int)(rem - (size_t)ip * g.nth);
}

// theta-wall datum of v, cot(theta) v (rhs_mpi.f90:414, :444): [ip + nphi*ir]
__global__ void k_lap_bc_theta(CssGeo g, const double *__restrict__ cur, double *__restrict__ lo,
                               double *__restrict__ hi) {
  const size_t n = (size_t)g.ncell, nf = (size_t)g.nphi * g.nr;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nf; k += (size_t)gridDim.x * blockDim.x) {
    const int ip = (int)(k % g.nphi), ir = (int)(k / g.nphi);
    lo[k] = g.cot[0] * cur[2 * n + css_idx(g, 0, ip, ir)];
    hi[k] = g.cot[g.nth - 1] * cur[2 * n + css_idx(g, g.nth - 1, ip, ir)];
  }
}

// radial-wall data of w and v (rhs_mpi.f90:578-611): stress-free x/r/dxdr,
// else 0 at the bottom and the face value at the top: [it + nth*ip]
__global__ void k_lap_bc_r(CssGeo g, const double *__restrict__ cur, double *__restrict__ wlo,
                           double *__restrict__ whi, double *__restrict__ vlo, double *__restrict__ vhi) {
  const size_t n = (size_t)g.ncell, nf = (size_t)g.nth * g.nphi;
  const int nr = g.nr;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nf; k += (size_t)gridDim.x * blockDim.x) {
    const size_t lo = k, hi = (size_t)(nr - 1) * nf + k;
    const double w0 = cur[n + lo], v0 = cur[2 * n + lo], w1 = cur[n + hi], v1 = cur[2 * n + hi];
    wlo[k] = g.bottom_stress_free ? w0 / g.r1 / g.dxdr[0] : 0.0;
    vlo[k] = g.bottom_stress_free ? v0 / g.r1 / g.dxdr[0] : 0.0;
    whi[k] = g.top_stress_free ? w1 / g.r2 / g.dxdr[nr - 1] : w1;
    vhi[k] = g.top_stress_free ? v1 / g.r2 / g.dxdr[nr - 1] : v1;
  }
}

// theta sweep terms (rhs_mpi.f90:844-862, :883-891, :914-926).
// S: d/dth of w, v, u; d2/dth2 of w, v, u.
__global__ void k_lap_theta(CssGeo g, const double *__restrict__ cur, const double *__restrict__ S,
                            double *__restrict__ L, double *__restrict__ dv) {
  const size_t n = (size_t)g.ncell;
  for (size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x; id < n; id += (size_t)gridDim.x * blockDim.x) {
    int it, ip, ir;
    lap_cell(g, id, it, ip, ir);
    const double ri = g.r_inv[ir], dlm = g.dlnmu[ir];
    const double rho = cur[id], w = cur[n + id], v = cur[2 * n + id];
    const double M = g.mur[ir] * (1.0 / rho);
    const double cot = g.cot[it], sn = g.sines[it], csc2 = 1.0 / (sn * sn);
    const double W1 = S[id] * ri, V1 = S[n + id] * ri, U1 = S[2 * n + id] * ri;
    double dw = dv[n + id], dvv = dv[2 * n + id], du = dv[3 * n + id];
    dw = dw + (-LAP_43 * ri * ri * csc2 - ri * dlm) * M * w;
    double t1 = W1 * M;
    du = du + (-LAP_13 * (7.0 * ri + 2.0 * dlm)) * (ri * M * cot * w + t1);
    dw = dw + LAP_43 * ri * cot * t1;
    dw = dw + LAP_43 * ri * ri * M * S[3 * n + id];
    dvv = dvv + ri * M * (cot * V1 - (ri * csc2 + dlm) * v);
    dvv = dvv + ri * ri * M * S[4 * n + id];
    t1 = U1 * M;
    dw = dw + (2.0 * LAP_43 * ri + dlm) * t1;
    du = du + ri * cot * t1;
    du = du + ri * ri * M * S[5 * n + id];
    dv[n + id] = dw;
    dv[2 * n + id] = dvv;
    dv[3 * n + id] = du;
    L[id] = W1;
    L[n + id] = V1;
    L[2 * n + id] = U1;
  }
}

// phi sweep terms with the theta-theta/phi-phi and theta-phi viscous
// heating (rhs_mpi.f90:1123-1199).  S: d/dph of v, w, u; d2/dph2 of v, w, u.
__global__ void k_lap_phi(CssGeo g, const double *__restrict__ cur, const double *__restrict__ tbuf,
                          const double *__restrict__ S, double *__restrict__ L, double *__restrict__ dv) {
  const size_t n = (size_t)g.ncell;
  for (size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x; id < n; id += (size_t)gridDim.x * blockDim.x) {
    int it, ip, ir;
    lap_cell(g, id, it, ip, ir);
    const double ri = g.r_inv[ir], dlm = g.dlnmu[ir];
    const double rho = cur[id], w = cur[n + id], v = cur[2 * n + id], u = cur[3 * n + id], t = tbuf[id];
    const double csc = g.csc[it], oors = ri * csc, oors2 = oors * oors, cot = g.cosines[it] * csc;
    const double M = (1.0 / rho) * g.mur[ir];
    const double Pv = S[id] * oors, Pw = S[n + id] * oors, Pu = S[2 * n + id] * oors;
    const double W1 = L[id], V1 = L[n + id];
    double dw = dv[n + id], dvv = dv[2 * n + id], du = dv[3 * n + id], ds = dv[4 * n + id];
    ds = ds + LAP_43 * M * (W1 + u * ri) * (W1 + 2.0 * u * ri - Pv - ri * cot * w) / t;
    double t1 = Pv * M;
    const double dd = -LAP_73 * ri, dd2 = dd - LAP_23 * dlm;
    dw = dw + dd * cot * t1;
    du = du + dd2 * t1;
    dvv = dvv + LAP_43 * (S[3 * n + id] * oors2) * M;
    const double q = V1 + Pw - ri * cot * v;
    ds = ds + M * (q * q) / t;
    dvv = dvv + LAP_73 * ri * cot * (Pw * M);
    dw = dw + (S[4 * n + id] * oors2) * M;
    dvv = dvv + (2.0 * LAP_43 * ri + dlm) * Pu * M;
    du = du + (S[5 * n + id] * oors2) * M;
    dv[n + id] = dw;
    dv[2 * n + id] = dvv;
    dv[3 * n + id] = du;
    dv[4 * n + id] = ds;
    L[3 * n + id] = Pv;
    L[4 * n + id] = Pw;
    L[5 * n + id] = Pu;
  }
}

// radial sweep terms with the r-theta, r-phi and r-r viscous heating
// (rhs_mpi.f90:1317-1435), as written: the cot(theta) dw/dr / (3 r) term of
// du has no mur/rho factor, and the r-theta heating is added a second time
// with du/dr in place of dw/dr.  S: d/dx of w, v, u; d2/dx2 of w, v, u (x the
// computational coordinate; dx/dr applied here).  Afterwards S holds the
// cross-term inputs r L0, r L5, r L2, r L3, sin L3, sin L4.
__global__ void k_lap_r(CssGeo g, const double *__restrict__ cur, const double *__restrict__ tbuf,
                        double *__restrict__ S, const double *__restrict__ L, double *__restrict__ dv) {
  const size_t n = (size_t)g.ncell;
  const int nu = g.non_uniform;
  for (size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x; id < n; id += (size_t)gridDim.x * blockDim.x) {
    int it, ip, ir;
    lap_cell(g, id, it, ip, ir);
    const double ri = g.r_inv[ir], dx = g.dxdr[ir];
    const double w9 = g.d2xdr2[ir] / dx, w5 = 2.0 * ri + g.dlnmu[ir];
    const double rho = cur[id], w = cur[n + id], v = cur[2 * n + id], u = cur[3 * n + id], t = tbuf[id];
    const double M = g.mur[ir] * (1.0 / rho), cot = g.cot[it];
    double Rw = S[id], Rv = S[n + id], Ru = S[2 * n + id];
    double D2w = S[3 * n + id], D2v = S[4 * n + id], D2u = S[5 * n + id];
    if (nu) {
      Rw = Rw * dx; Rv = Rv * dx; Ru = Ru * dx;
      D2w = D2w * (dx * dx); D2v = D2v * (dx * dx); D2u = D2u * (dx * dx);
    }
    const double W1 = L[id], U1 = L[2 * n + id], Pv = L[3 * n + id], Pw = L[4 * n + id], Pu = L[5 * n + id];
    double dw = dv[n + id], dvv = dv[2 * n + id], du = dv[3 * n + id], ds = dv[4 * n + id];
    du = du + LAP_13 * cot * ri * Rw;
    dw = dw + M * w5 * Rw;
    double q = Rw + U1 - w * ri;
    ds = ds + M * (q * q) / t;
    if (nu) dw = dw + w9 * Rw * M;
    dw = dw + D2w * M;
    q = Rv + Pu - v * ri;
    ds = ds + M * (q * q) / t;
    dvv = dvv + Rv * w5 * M;
    if (nu) dvv = dvv + w9 * Rv * M;
    dvv = dvv + D2v * M;
    du = du + LAP_43 * M * w5 * (Ru - u * ri);
    if (nu) du = du + LAP_43 * w9 * Ru * M;
    ds = ds + LAP_43 * M * Ru * (Ru - W1 - u * ri) / t;
    q = Ru + Pu - v * ri;
    ds = ds + M * (q * q) / t;
    const double a = Pv + (cot * w + u) * ri;
    ds = ds + LAP_43 * M * a * (a - Ru) / t;
    du = du + LAP_43 * D2u * M;
    dv[n + id] = dw;
    dv[2 * n + id] = dvv;
    dv[3 * n + id] = du;
    dv[4 * n + id] = ds;
    const double r = g.r_ind[ir], sn = g.sines[it];
    S[id] = r * W1;
    S[n + id] = r * Pu;
    S[2 * n + id] = r * U1;
    S[3 * n + id] = r * Pv;
    S[4 * n + id] = sn * Pv;
    S[5 * n + id] = sn * Pw;
  }
}

// face data of the cross terms (rhs_mpi.f90:2112-2124, :2241-2250): radial
// faces [it + nth*ip] of r L0 (bottom) and r L3 (top), both under
// Bottom_Stress_Free as the reference writes them; theta faces
// [ip + nphi*ir] of sin L3 = sin (L3 cos / sin).  Slots the reference never
// writes are 0.
__global__ void k_lap_bc_cross(CssGeo g, const double *__restrict__ L, double *__restrict__ rlo,
                               double *__restrict__ rhi, double *__restrict__ tlo, double *__restrict__ thi) {
  const size_t n = (size_t)g.ncell, nfr = (size_t)g.nth * g.nphi, nft = (size_t)g.nphi * g.nr;
  const size_t nf = nfr > nft ? nfr : nft;
  const int nr = g.nr, nth = g.nth;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nf; k += (size_t)gridDim.x * blockDim.x) {
    if (k < nfr) {
      rlo[k] = g.bottom_stress_free ? g.r1 * (L[k] / g.r1 / g.dxdr[0]) : 0.0;
      rhi[k] = g.bottom_stress_free ? g.r2 * (L[3 * n + (size_t)(nr - 1) * nfr + k] / g.r2 / g.dxdr[nr - 1]) : 0.0;
    }
    if (k < nft) {
      const int ip = (int)(k % g.nphi), ir = (int)(k / g.nphi);
      const double a = L[3 * n + css_idx(g, 0, ip, ir)], b = L[3 * n + css_idx(g, nth - 1, ip, ir)];
      tlo[k] = g.sines[0] * (a * g.cosines[0] / g.sines[0]);
      thi[k] = g.sines[nth - 1] * (b * g.cosines[nth - 1] / g.sines[nth - 1]);
    }
  }
}

// cross terms (rhs_mpi.f90:2125-2204, :2252-2295).  L now holds the radial
// derivatives (d/dx) of r L0, r L5, r L2, r L3 and the theta derivatives of
// sin L3, sin L4.  The radial factor uses the cell's own 1/rho (the
// reference's invrho(it+ir-1, ip, :) reads an undefined index).
__global__ void k_lap_cross(CssGeo g, const double *__restrict__ cur, const double *__restrict__ L,
                            double *__restrict__ dv) {
  const size_t n = (size_t)g.ncell;
  const int nu = g.non_uniform;
  for (size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x; id < n; id += (size_t)gridDim.x * blockDim.x) {
    int it, ip, ir;
    lap_cell(g, id, it, ip, ir);
    const double invrho = 1.0 / cur[id], f = nu ? g.dxdr[ir] : 1.0;
    double a0 = L[id], a1 = L[n + id], a2 = L[2 * n + id], a3 = L[3 * n + id];
    if (nu) { a0 = a0 * f; a1 = a1 * f; a2 = a2 * f; a3 = a3 * f; }
    const double w6 = LAP_13 * g.mur[ir] * g.r_inv[ir] * invrho;
    double du = dv[3 * n + id] + w6 * a0;
    double dvv = dv[2 * n + id] + w6 * a1;
    double dw = dv[n + id] + w6 * a2;
    du = du + w6 * a3;
    const double w4 = LAP_13 * (g.r_inv[ir] * g.mur[ir]) * invrho / g.sines[it];
    dw = dw + w4 * L[4 * n + id];
    dvv = dvv + w4 * L[5 * n + id];
    dv[n + id] = dw;
    dv[2 * n + id] = dvv;
    dv[3 * n + id] = du;
  }
}

// ---------------------------------------------------------------------------
// Resistive induction under the Laplacian switch (Induction_Terms,
// rhs_mpi.f90:2303-2364): J = curl B (VectorCurl, derivatives.f90:1894-2104),
// dA/dt += -eta J (the v x B part is already in the tendency) and ds += (4 pi
// / c^2) eta |J|^2 / (rho T), eta = ks.  B (bf) is B_theta, B_phi, B_r.
// ---------------------------------------------------------------------------
__global__ void k_mhd_curl_in(CssGeo g, const double *__restrict__ bf, double *__restrict__ S) {
  const size_t n = (size_t)g.ncell;
  for (size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x; id < n; id += (size_t)gridDim.x * blockDim.x) {
    int it, ip, ir;
    lap_cell(g, id, it, ip, ir);
    const double bt = bf[id], bp = bf[n + id], r = g.r_ind[ir];
    S[id] = g.sines[it] * bp;
    S[n + id] = r * bt;
    S[2 * n + id] = r * bp;
  }
}

// D: d(sin B_phi)/dth, dB_r/dth, dB_r/dph, dB_theta/dph, d(r B_theta)/dx, d(r B_phi)/dx
__global__ void k_mhd_resist(CssGeo g, const double *__restrict__ cur, const double *__restrict__ tb,
                             const double *__restrict__ D0, const double *__restrict__ D1, double *__restrict__ dv) {
  const size_t n = (size_t)g.ncell;
  const double jconst = 4.0 * 3.1415926535897932384626433832795028841972 / (2.99792458e10 * 2.99792458e10);
  for (size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x; id < n; id += (size_t)gridDim.x * blockDim.x) {
    int it, ip, ir;
    lap_cell(g, id, it, ip, ir);
    const double invr = g.r_inv[ir], csc = g.csc[it];
    double jr = D0[id] * csc * invr;
    double jp = -D0[n + id] * invr;
    double jt = invr * D0[2 * n + id] * csc;
    jr = jr - invr * D1[id] * csc;
    double a = D1[n + id], b = D1[2 * n + id];
    if (g.non_uniform) { a = a * g.dxdr[ir]; b = b * g.dxdr[ir]; }
    jp = jp + a * invr;
    jt = jt - b * invr;
    const double etar = g.ks[ir];
    dv[4 * n + id] = dv[4 * n + id] + (jconst * etar) * (jt * jt + jp * jp + jr * jr) * (1.0 / cur[id]) / tb[id];
    dv[5 * n + id] = dv[5 * n + id] + (-etar * jt);
    dv[6 * n + id] = dv[6 * n + id] + (-etar * jp);
    dv[7 * n + id] = dv[7 * n + id] + (-etar * jr);
  }
}

// ---------------------------------------------------------------------------
// Radiative diffusion (do_radheat): ds += coef [T''/T + T'/T (geometry +
// 3 T'/T - rho'/rho)] per direction, coef = (4 a c kr / 3) T^3 / rho^2
// (rhs_mpi.f90:388-392), as Phi_Terms (:1092-1106), Density_Terms_Theta
// (:1590-1602) and Density_Terms_Radial (:1820-1853) write it.  The pass
// runs after the radial kernel: the theta density datum reads the final dw
// (the same value the density-theta update kernel reads next), and the
// radial kernel has kept d ln(rho)/dr (its density datum built from du
// before the density term changed it) and ds/dr.
// ---------------------------------------------------------------------------
#define RAD_AC (7.56577e-15 * 2.99792458e10)  // a_const * c_light, constants.f90:7

// face data: theta [ip + nphi*ir]: the hydrostatic datum of d(rho)/dth,
// r/(pconst) dw rho / T (rhs_mpi.f90:1553-1564), and T on the walls;
// r [it + nth*ip]: the datum of dT/dr, T ((gamma-1) dlnrho/dr + ds/dr / Cv)
// / dxdr on the walls (:1822-1831)
__global__ void k_rad_bc(CssGeo g, const double *__restrict__ cur, const double *__restrict__ dv,
                         const double *__restrict__ tb, double *__restrict__ rlo_t, double *__restrict__ rhi_t,
                         double *__restrict__ tlo_t, double *__restrict__ thi_t, double *__restrict__ tlo_r,
                         double *__restrict__ thi_r) {
  const size_t n = (size_t)g.ncell, nfr = (size_t)g.nth * g.nphi, nft = (size_t)g.nphi * g.nr;
  const size_t nf = nfr > nft ? nfr : nft;
  const int nr = g.nr, nth = g.nth;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nf; k += (size_t)gridDim.x * blockDim.x) {
    if (k < nft) {
      const int ip = (int)(k % g.nphi), ir = (int)(k / g.nphi);
      const double rv = g.r_ind[ir] * g.invpconst;
      const size_t a = css_idx(g, 0, ip, ir), b = css_idx(g, nth - 1, ip, ir);
      rlo_t[k] = rv * dv[n + a] * cur[a] / tb[a];
      rhi_t[k] = rv * dv[n + b] * cur[b] / tb[b];
      tlo_t[k] = tb[a];
      thi_t[k] = tb[b];
    }
    if (k < nfr) {
      const size_t a = k, b = (size_t)(nr - 1) * nfr + k;
      tlo_r[k] = tb[a] * (g.gamm1 * g.rad_lnrho_r[a] + g.invcv * g.rad_dsdr[a]) / g.dxdr[0];
      thi_r[k] = tb[b] * (g.gamm1 * g.rad_lnrho_r[b] + g.invcv * g.rad_dsdr[b]) / g.dxdr[nr - 1];
    }
  }
}

// S: d rho/dth, dT/dth, d2T/dth2, d rho/dph, dT/dph, d2T/dph2, dT/dx, d2T/dx2
__global__ void k_rad_point(CssGeo g, const double *__restrict__ cur, const double *__restrict__ tb,
                            const double *__restrict__ S, double *__restrict__ dv) {
  const size_t n = (size_t)g.ncell;
  const int nu = g.non_uniform;
  for (size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x; id < n; id += (size_t)gridDim.x * blockDim.x) {
    int it, ip, ir;
    lap_cell(g, id, it, ip, ir);
    const double t = tb[id], invrho = 1.0 / cur[id], ri = g.r_inv[ir];
    const double coef = (4.0 * RAD_AC * g.kr[ir] / 3.0) * (t * t * t) * (invrho * invrho);
    double ds = dv[4 * n + id];
    // phi
    const double oors = ri * g.csc[it];
    const double w = (S[3 * n + id] * oors) * invrho;
    double a = S[4 * n + id] * oors / t;
    ds = ds + coef * (3.0 * a - w) * a;
    ds = ds + coef * (S[5 * n + id] * (oors * oors)) / t;
    // theta
    const double rho_t = (ri * S[id]) * invrho;
    a = ri * S[n + id] / t;
    ds = ds + coef * a * (3.0 * a + ri * g.cot[it] - rho_t);
    ds = ds + (ri * ri) * coef * S[2 * n + id] / t;
    // r
    const double dx = g.dxdr[ir];
    a = S[6 * n + id];
    if (nu) a = a * dx;
    a = a / t;
    ds = ds + coef * a * ((2.0 * ri - g.dlnkr[ir]) + 3.0 * a - g.rad_lnrho_r[id]);
    if (nu) ds = ds + coef * a * (g.d2xdr2[ir] / dx);
    double d2 = S[7 * n + id];
    if (nu) d2 = d2 * (dx * dx);
    ds = ds + coef * d2 / t;
    dv[4 * n + id] = ds;
  }
}

}  // namespace css
