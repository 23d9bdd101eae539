// css_stats.cuh -- on-device diagnostics of the current state: the sums,
// extrema and fluxes of Scalar_Output (report_mpi.f90:173-262),
// Shell_Average_Output (report_mpi.f90:783-1094) and Compute_Step_Size
// (rhs_mpi.f90:92-275), and the (theta, phi) spectrum of
// CSS-IDL/spectral_analysis_new.pro:16-25.
//
// Reductions are two-level and deterministic: a (chunk, radius) grid of CTAs
// writes one partial per accumulator, then one CTA per radius combines the
// partials in chunk order.  Every accumulator is a per-radius quantity; the
// whole-domain scalars are formed from the per-radius results on the host,
// in radius order.
#pragma once
#include "css_geo.cuh"

namespace css {

// per-radius accumulators.  Pass 1 reads the state (and B, ds/dr); pass 2
// needs the per-radius means of pass 1 (the reference's avgvr, avgT, avgP).
enum StatAcc {
  SA_RHO = 0, SA_T, SA_S, SA_RHOT, SA_VR, SA_VT, SA_VP, SA_KE, SA_DSDR,  // Shell_Average 1-9 (sums)
  SA_BR, SA_BT, SA_BP, SA_ME, SA_BPOL,                                      // 10-14 (sums)
  SA_RU2, SA_RW2, SA_RV2, SA_RUSQ, SA_BSQ,                                  // Scalar_Output sums
  SA_UMACH, SA_BMAX2,                                                       // maxima
  SA_DTC, SA_DTB,                                                           // minima (Courant limits)
  SA_E, SA_L, SA_M, SA_MRS,                                                 // conservation sums
  SA_NPASS1,
  SA_FEN = SA_NPASS1, SA_FKE, SA_FAC,                                       // pass 2 fluxes
  SA_N
};
#define SA_NPASS2 3

__device__ __forceinline__ int sa_kind(int a) {  // 0 sum, 1 max, 2 min
  return (a == SA_UMACH || a == SA_BMAX2) ? 1 : (a == SA_DTC || a == SA_DTB) ? 2 : 0;
}
__device__ __forceinline__ double sa_init(int a) {
  int k = sa_kind(a);
  return k == 0 ? 0.0 : (k == 1 ? -INFINITY : INFINITY);
}
__device__ __forceinline__ double sa_comb(int kind, double x, double y) {
  return kind == 0 ? x + y : (kind == 1 ? fmax(x, y) : fmin(x, y));
}

// block reduction of NA per-thread accumulators (first accumulator index A0)
// into out[0..NA); blockDim.x a multiple of 32, at most 1024
template <int NA, int A0>
__device__ __forceinline__ void block_reduce_store(double (&acc)[NA], double *red, double *out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int a = 0; a < NA; a++) {
    const int k = sa_kind(A0 + a);
    double x = acc[a];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = sa_comb(k, x, __shfl_down_sync(0xffffffffu, x, o));
    if (lane == 0) red[warp * NA + a] = x;
  }
  __syncthreads();
  if (threadIdx.x < NA) {
    const int a = threadIdx.x, k = sa_kind(A0 + a);
    double x = red[a];
    for (int w = 1; w < nw; w++) x = sa_comb(k, x, red[w * NA + a]);
    out[a] = x;
  }
}

// Pass 1.  grid (nchunk, nr); part[(ir*nchunk + chunk)*SA_NPASS1 + a].
// bf = B (theta, phi, r) for MHD, dsdr = d s / d r in grid units (NULL: 0).
__global__ void __launch_bounds__(256) k_stats_pass1(CssGeo g, const double *__restrict__ v,
                                                     const double *__restrict__ bf,
                                                     const double *__restrict__ dsdr, double *__restrict__ part) {
  __shared__ double red[32 * SA_NPASS1];
  const int ir = blockIdx.y, nchunk = gridDim.x;
  const size_t n = (size_t)g.ncell, np = (size_t)g.nth * g.nphi;
  const size_t c0 = np * blockIdx.x / nchunk, c1 = np * (blockIdx.x + 1) / nchunk;
  double acc[SA_NPASS1];
#pragma unroll
  for (int a = 0; a < SA_NPASS1; a++) acc[a] = sa_init(a);
  const double radius = g.r_ind[ir], drad = g.dr_ind[ir];
  const double dxr = g.non_uniform ? g.dxdr[ir] : 1.0;
  const double cs2 = g.gamm1 * g.cp * g.xi_cs * g.xi_cs;
  const double tprime = g.gamm1 * g.cp;
  const double wvol = drad * g.dth * g.dphi;
  const int mag = g.magnetic;
  const size_t base = (size_t)ir * np;
  for (size_t k = c0 + threadIdx.x; k < c1; k += blockDim.x) {
    const size_t id = base + k;
    const int it = (int)(k % (size_t)g.nth);
    const double rho = v[id], w = v[n + id], vp = v[2 * n + id], u = v[3 * n + id], s = v[4 * n + id];
    const double T = temp_of(g, rho, s);
    const double u2 = u * u, w2 = w * w, v2 = vp * vp;
    const double usq = w2 + v2 + u2;
    const double ke = 0.5 * rho * usq;
    acc[SA_RHO] += rho;
    acc[SA_T] += T;
    acc[SA_S] += s;
    acc[SA_RHOT] += rho * T;
    acc[SA_VR] += u;
    acc[SA_VT] += w;
    acc[SA_VP] += vp;
    acc[SA_KE] += ke;
    if (dsdr) acc[SA_DSDR] += dsdr[id] * dxr;
    acc[SA_RU2] += rho * u2;
    acc[SA_RW2] += rho * w2;
    acc[SA_RV2] += rho * v2;
    acc[SA_RUSQ] += rho * usq;
    double bsq = 0.0;
    if (mag) {
      const double bt = bf[id], bp = bf[n + id], br = bf[2 * n + id];
      bsq = br * br + bt * bt + bp * bp;
      acc[SA_BR] += br;
      acc[SA_BT] += bt;
      acc[SA_BP] += bp;
      acc[SA_ME] += (0.125 * bsq) / 3.14159265358979323846;
      acc[SA_BPOL] += sqrt(br * br + bt * bt);
      acc[SA_BSQ] += bsq;
      acc[SA_BMAX2] = fmax(acc[SA_BMAX2], bsq);
    }
    const double Tp = T * tprime;  // Scalar_Output's temperature carries gamm1*Cp
    const double um = mag ? usq / (2.0 * bsq / rho + usq + Tp) : usq / (usq + Tp);
    acc[SA_UMACH] = fmax(acc[SA_UMACH], um);
    // Courant limits (rhs_mpi.f90:182-214)
    const double sinth = g.sines[it];
    const double dxmin = fmin(drad, radius * fmin(g.dth, sinth * g.dphi));
    const double ut = u2 + v2 + w2 + cs2 * T;
    acc[SA_DTC] = fmin(acc[SA_DTC], dxmin / sqrt(ut));
    if (mag) acc[SA_DTB] = fmin(acc[SA_DTB], dxmin / sqrt(ut + bsq * ONE_OVER_4PI / rho));
    // conservation (rhs_mpi.f90:186-205)
    const double r2s = radius * radius * sinth * wvol;
    double e = rho * (g.cv * T + 0.5 * (u2 + w2 + v2));
    if (mag) e += 0.5 * bsq * ONE_OVER_4PI;
    acc[SA_E] += r2s * e;
    const double vr = vp + radius * sinth * g.omega0;
    acc[SA_L] += radius * r2s * rho * sqrt(w2 + sinth * sinth * vr * vr);
    acc[SA_M] += r2s * rho;
    acc[SA_MRS] += radius * r2s * sinth * sinth * rho;
  }
  block_reduce_store<SA_NPASS1, 0>(acc, red, part + ((size_t)ir * nchunk + blockIdx.x) * SA_NPASS1);
}

// Pass 2 (fluxes about the per-radius means).  res[ir*SA_N + a] holds the
// pass-1 sums; part2[(ir*nchunk + chunk)*SA_NPASS2 + a].
__global__ void __launch_bounds__(256) k_stats_pass2(CssGeo g, const double *__restrict__ v,
                                                     const double *__restrict__ res, double *__restrict__ part) {
  __shared__ double red[32 * SA_NPASS2];
  const int ir = blockIdx.y, nchunk = gridDim.x;
  const size_t n = (size_t)g.ncell, np = (size_t)g.nth * g.nphi;
  const size_t c0 = np * blockIdx.x / nchunk, c1 = np * (blockIdx.x + 1) / nchunk;
  const double inv = 1.0 / (double)np;
  const double ubar = res[(size_t)ir * SA_N + SA_VR] * inv;
  const double tbar = res[(size_t)ir * SA_N + SA_T] * inv;
  const double pbar = g.gamm1 * g.cv * res[(size_t)ir * SA_N + SA_RHOT] * inv;
  double acc[SA_NPASS2] = {0.0, 0.0, 0.0};
  const size_t base = (size_t)ir * np;
  for (size_t k = c0 + threadIdx.x; k < c1; k += blockDim.x) {
    const size_t id = base + k;
    const double rho = v[id], w = v[n + id], vp = v[2 * n + id], u = v[3 * n + id], s = v[4 * n + id];
    const double T = temp_of(g, rho, s);
    const double du = u - ubar;
    acc[0] += du * rho * (T - tbar);
    acc[1] += 0.5 * rho * (u * u + vp * vp + w * w) * du;
    acc[2] += (g.gamm1 * g.cv * rho * T - pbar) * du;
  }
  block_reduce_store<SA_NPASS2, SA_NPASS1>(acc, red, part + ((size_t)ir * nchunk + blockIdx.x) * SA_NPASS2);
}

// combine the chunk partials of each radius in chunk order: grid nr,
// res[ir*SA_N + a0 + a] for a < na
__global__ void k_stats_combine(const double *__restrict__ part, int nchunk, int na, int a0,
                                double *__restrict__ res) {
  const int ir = blockIdx.x;
  for (int a = threadIdx.x; a < na; a += blockDim.x) {
    const int k = sa_kind(a0 + a);
    double x = part[((size_t)ir * nchunk) * na + a];
    for (int c = 1; c < nchunk; c++) x = sa_comb(k, x, part[((size_t)ir * nchunk + c) * na + a]);
    res[(size_t)ir * SA_N + a0 + a] = x;
  }
}

// ---------------------------------------------------------------------------
// Spectrum.  For a real field the folded FFT of spectral_analysis_new.pro
// (fftcube[kt,kp] = F[kt,kp] + F[nth-kt,nphi-kp], kept as a real number) is
// 2 Re F[kt,kp], so the phi spectrum
//   S[kp] = (1/(nth/2)) sum_{kt=1}^{nth/2-1} 2 Re F[kt,kp]     (kp >= 1)
//   S[0]  = F[0,0] / (nth/2),   F = forward 2D DFT / (nth nphi)
// factors into a theta reduction with W(t) = sum_kt exp(-2 pi i kt t/nth)
// (times the apodisation) followed by one phi DFT per radius.
// ---------------------------------------------------------------------------
// pointwise field of a spectrum: 0 kinetic energy density, 1 magnetic
// energy density, 2 + iv state variable iv
__device__ __forceinline__ double spec_field(const CssGeo &g, const double *__restrict__ v,
                                             const double *__restrict__ bf, int kind, size_t id) {
  const size_t n = (size_t)g.ncell;
  if (kind == 0) {
    const double rho = v[id], w = v[n + id], vp = v[2 * n + id], u = v[3 * n + id];
    return 0.5 * rho * (u * u + vp * vp + w * w);
  }
  if (kind == 1) {
    const double bt = bf[id], bp = bf[n + id], br = bf[2 * n + id];
    return (0.125 * (br * br + bt * bt + bp * bp)) / 3.14159265358979323846;
  }
  return v[(size_t)(kind - 2) * n + id];
}

// grid (ceil(nphi/8), nr), 256 threads: one warp per phi line.
// wt = [apod | apod*Re W | apod*Im W] (3 nth); b[(ir*nphi + ip)*3 + {0,1,2}]
__global__ void __launch_bounds__(256) k_spec_theta(CssGeo g, const double *__restrict__ v,
                                                    const double *__restrict__ bf, int kind,
                                                    const double *__restrict__ wt, double *__restrict__ b) {
  const int lane = threadIdx.x & 31;
  const int ip = blockIdx.x * 8 + (threadIdx.x >> 5), ir = blockIdx.y;
  if (ip >= g.nphi) return;
  double a0 = 0.0, ar = 0.0, ai = 0.0;
  const size_t line = ((size_t)ir * g.nphi + ip) * g.nth;
  for (int it = lane; it < g.nth; it += 32) {
    const double a = spec_field(g, v, bf, kind, line + it);
    a0 += a * wt[it];
    ar += a * wt[g.nth + it];
    ai += a * wt[2 * g.nth + it];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a0 += __shfl_down_sync(0xffffffffu, a0, o);
    ar += __shfl_down_sync(0xffffffffu, ar, o);
    ai += __shfl_down_sync(0xffffffffu, ai, o);
  }
  if (lane == 0) {
    double *o = b + ((size_t)ir * g.nphi + ip) * 3;
    o[0] = a0;
    o[1] = ar;
    o[2] = ai;
  }
}

// grid nr, 256 threads, dynamic smem 3*nphi doubles; tw = [cos | sin] of
// 2 pi j / nphi (2 nphi); out[ir*(nphi/2) + kp]
__global__ void __launch_bounds__(256) k_spec_phi(const double *__restrict__ b, const double *__restrict__ tw,
                                                  int nth, int nphi, double *__restrict__ out) {
  extern __shared__ double sb[];
  const int ir = blockIdx.x;
  for (int k = threadIdx.x; k < 3 * nphi; k += blockDim.x) sb[k] = b[(size_t)ir * nphi * 3 + k];
  __syncthreads();
  const double nn = (double)nth * (double)nphi;
  for (int kp = threadIdx.x; kp < nphi / 2; kp += blockDim.x) {
    double acc = 0.0;
    if (kp == 0) {
      for (int p = 0; p < nphi; p++) acc += sb[3 * p];
      out[(size_t)ir * (nphi / 2)] = (acc / nn) / (0.5 * nth);
    } else {
      int j = 0;
      for (int p = 0; p < nphi; p++) {
        acc += sb[3 * p + 1] * tw[j] + sb[3 * p + 2] * tw[nphi + j];
        j += kp;
        if (j >= nphi) j -= nphi;
      }
      out[(size_t)ir * (nphi / 2) + kp] = 2.0 * (acc / nn) / (0.5 * nth);
    }
  }
}

}  // namespace css
