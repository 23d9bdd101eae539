// css_kernels.cuh -- the CSS right-hand side, slope-limited diffusion and RK4
// stage kernels for sm_100a, FP64.
//
// Each RHS term group of the reference is one kernel over shared-memory
// tiles: a tile is one virtual block segment along the sweep direction
// (+4 halo points each side, exactly the reference's halo depth) times TL
// lines.  The line solves run one thread per (field, line); the pointwise
// physics then runs one thread per point with coalesced (theta-contiguous)
// global reads/writes of the state and the tendency.
//
//   theta_terms   Source_Theta_Terms (+ its Lorentz part) + Induction_Terms
//   phi_terms     Phi_Terms (+ Lorentz)
//   radial_terms  Radial_Terms (+ Lorentz) fused with Density_Terms_Radial
//   rhot_update   Density_Terms_Theta fused with the RK4 stage combination
//                 of Step_RK4 and Bound
//   curl_*        VectorCurlA (+ Compute_B's boundary zeroing)
//   sld_*         Compute_Diffusion / Diffusion_R / _Th / _Phi
#pragma once
#include "css_geo.cuh"
#include "css_lines.cuh"

namespace css {

#define ONE_OVER_4PI (1.0 / 3.14159265358979323846264338327950288 / 4.0)

__device__ __forceinline__ const double *tabp(const CssGeo &g, int dir, int blk, int order, int bdry) {
  int off = (order == 1 ? g.d[dir].tab1[blk] : g.d[dir].tab2[blk]);
  return g.tab + off + (size_t)bdry * 3 * g.tstride;
}

__device__ __forceinline__ int dtype_of(const CssDir &d, int b) {
  int lp = d.lphys[b], rp = d.rphys[b];
  return lp ? (rp ? 0 : 2) : (rp ? 1 : 3);
}

// temperature (rhs_mpi.f90:376-385)
// invtconst * rho^(gamma-1) * exp(s/Cv) as one exponential: the reference's
// pow * exp product to within a few roundings of its exponent
__device__ __forceinline__ double temp_of(const CssGeo &g, double rho, double s) {
  return g.invtconst * exp(fma(g.gamm1, log(rho), s * g.invcv));
}

__device__ __forceinline__ double dnum_d2_theta(const CssGeo &g, int ir) {
  // D2bydt2 divides the theta Neumann datum by the rank's dri
  // (derivatives.f90:1322, :1338)
  return g.d[0].dnum[__ldg(g.rblk + ir)];
}

// A stage state is stored either as FP64 values (the FP64 path, and vars0)
// or as FP32 perturbations of rho and s about a background that depends on
// r and theta (CssGeo::bg2: the phi means of the state last uploaded; the
// mixed path, the other fields plain FP32).  st_val returns the FP64 value:
// the stored number, plus the background at (r, theta) -- bidx = r*nth +
// theta -- when it is FP32 and a background is given.
template <typename TS>
__device__ __forceinline__ double st_val(const TS *p, size_t off, const double *mean, size_t bidx) {
  double x = (double)__ldg(p + off);
  if constexpr (sizeof(TS) == 4) {
    if (mean) x += mean[bidx];
  }
  return x;
}
// backgrounds of rho and s for the FP32 stage states (2-D, nr x nth)
__device__ __forceinline__ const double *bg_rho(const CssGeo &g) { return g.bg2; }
__device__ __forceinline__ const double *bg_s(const CssGeo &g) {
  return g.bg2 ? g.bg2 + (size_t)g.nr * g.nth : nullptr;
}
__device__ __forceinline__ size_t bgi(const CssGeo &g, int r, int t) { return (size_t)r * g.nth + t; }

// the stored form of a new stage value (inverse of st_val)
template <typename TO>
__device__ __forceinline__ TO st_store(double x, double mean) {
  if constexpr (sizeof(TO) == 4) return (TO)(x - mean);
  else return x;
}

// asynchronous global -> shared copies (completion tracked per commit group)
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, int src_bytes) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// bring a 128-byte line into L2 ahead of its use (no register, no wait)
__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p)); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// ---------------------------------------------------------------------------
// tile loaders
// ---------------------------------------------------------------------------
// theta tile: S[l*SR + j+4], j in [-4, m+4), lines = phi indices pb..pb+TL-1
template <typename TS>
__device__ __forceinline__ void load_theta_tile(const CssGeo &g, const TS *__restrict__ f, double *S, int SR,
                                                int t0, int m, int pb, int TL, int ir, bool halo) {
  int w = m + 8;
  for (int idx = threadIdx.x; idx < TL * w; idx += blockDim.x) {
    int l = idx / w, jj = idx - l * w;
    int gt = t0 + jj - 4, gp = pb + l;
    if ((!halo && (jj < 4 || jj >= m + 4)) || gt < 0 || gt >= g.nth || gp >= g.nphi) continue;
    S[l * SR + jj] = (double)__ldg(f + css_idx(g, gt, gp, ir));
  }
}

// phi tile: S[(j+4)*SR + l], lines = theta indices tb..tb+TL-1, periodic in phi
template <typename TS>
__device__ __forceinline__ void load_phi_tile(const CssGeo &g, const TS *__restrict__ f, double *S, int SR,
                                              int p0, int m, int tb, int TL, int ir, bool halo) {
  int w = m + 8;
  for (int idx = threadIdx.x; idx < TL * w; idx += blockDim.x) {
    int jj = idx / TL, l = idx - jj * TL;
    if (!halo && (jj < 4 || jj >= m + 4)) continue;
    int gp = p0 + jj - 4;
    gp = (gp + g.nphi) % g.nphi;
    int gt = tb + l;
    if (gt >= g.nth) continue;
    S[jj * SR + l] = (double)__ldg(f + css_idx(g, gt, gp, ir));
  }
}

// r tile: S[(j+4)*SR + l], lines = theta indices tb..tb+TL-1 at fixed phi
template <typename TS>
__device__ __forceinline__ void load_r_tile(const CssGeo &g, const TS *__restrict__ f, double *S, int SR, int r0,
                                            int m, int tb, int TL, int ip, bool halo) {
  int w = m + 8;
  for (int idx = threadIdx.x; idx < TL * w; idx += blockDim.x) {
    int jj = idx / TL, l = idx - jj * TL;
    int gr = r0 + jj - 4, gt = tb + l;
    if ((!halo && (jj < 4 || jj >= m + 4)) || gr < 0 || gr >= g.nr || gt >= g.nth) continue;
    S[jj * SR + l] = (double)__ldg(f + css_idx(g, gt, ip, gr));
  }
}

// copies the LU tables (g1|g2|g3, 1-based, m+2 each) of one block into dst
__device__ __forceinline__ void stage_table(const CssGeo &g, int dir, int blk, int order, int bdry, int m,
                                            double *dst) {
  const double *src = tabp(g, dir, blk, order, bdry);
  const int ts = m + 2;
  for (int k = threadIdx.x; k < 3 * ts; k += blockDim.x) {
    int a = k / ts, j = k - a * ts;
    dst[k] = src[(size_t)a * g.tstride + j];
  }
}

// plane offset of radius ir, line offset of (ip) inside a plane
__device__ __forceinline__ size_t plane(const CssGeo &g, int ir) { return (size_t)ir * g.nth * g.nphi; }

// theta tile: S[l*SR + j+4], lines = phi indices pb..pb+TL-1 of radius ir
template <int MT, int TLC, typename TS>
__device__ __forceinline__ void tile_theta(const CssGeo &g, const TS *__restrict__ f, double *S, int SR, int t0,
                                           int m_, int pb, int TL_, int ir, const double *mean = nullptr) {
  const int m = MT ? MT : m_, TL = TLC ? TLC : TL_, w = m + 8;
  const TS *fp = f + plane(g, ir);
  for (int idx = threadIdx.x; idx < TL * w; idx += blockDim.x) {
    int l = idx / w, jj = idx - l * w;
    int gt = t0 + jj - 4, gp = pb + l;
    if (gt < 0 || gt >= g.nth || gp >= g.nphi) continue;
    S[l * SR + jj] = st_val(fp, (size_t)gp * g.nth + gt, mean, bgi(g, ir, gt));
  }
}

// phi tile: S[(j+4)*SR + l], lines = theta indices tb..tb+TL-1, periodic phi
template <int MT, int TLC, typename TS>
__device__ __forceinline__ void tile_phi(const CssGeo &g, const TS *__restrict__ f, double *S, int SR, int p0,
                                         int m_, int tb, int TL_, int ir, const double *mean = nullptr) {
  const int m = MT ? MT : m_, TL = TLC ? TLC : TL_, w = m + 8;
  const TS *fp = f + plane(g, ir);
  for (int idx = threadIdx.x; idx < TL * w; idx += blockDim.x) {
    int jj = idx / TL, l = idx - jj * TL;
    int gp = p0 + jj - 4, gt = tb + l;
    if (gp < 0) gp += g.nphi;
    else if (gp >= g.nphi) gp -= g.nphi;
    if (gt >= g.nth) continue;
    S[jj * SR + l] = st_val(fp, (size_t)gp * g.nth + gt, mean, bgi(g, ir, gt));
  }
}

// r tile: S[(j+4)*SR + l], lines = theta indices tb..tb+TL-1 at phi ip
template <int MT, int TLC, typename TS>
__device__ __forceinline__ void tile_r(const CssGeo &g, const TS *__restrict__ f, double *S, int SR, int r0,
                                       int m_, int tb, int TL_, int ip, const double *mean = nullptr) {
  const int m = MT ? MT : m_, TL = TLC ? TLC : TL_, w = m + 8;
  const size_t ps = (size_t)g.nth * g.nphi;
  const TS *fp = f + (size_t)ip * g.nth + tb;
  for (int idx = threadIdx.x; idx < TL * w; idx += blockDim.x) {
    int jj = idx / TL, l = idx - jj * TL;
    int gr = r0 + jj - 4;
    if (gr < 0 || gr >= g.nr || tb + l >= g.nth) continue;
    S[jj * SR + l] = st_val(fp, (size_t)gr * ps + l, mean, bgi(g, gr, tb + l));
  }
}

// threads per CTA of the line-solve kernels (every launch uses this count)
constexpr int NT = 128;

// Compile-time tiles of NF fields at once (MT, TLC > 0): every thread issues
// all of its global loads (NF fields x ceil(TLC*(MT+8)/NT) points) before it
// stores any of them to shared memory, so a CTA has NF times more loads in
// flight than a field-by-field loop.  DIR 1: theta tile S[l*SR + jj] of
// radius `fixed`, lines = phi indices lb..; DIR 2: phi tile S[jj*SR + l],
// periodic in phi, lines = theta indices lb..; DIR 0: r tile S[jj*SR + l]
// at phi index `fixed`, lines = theta indices lb...  a0 = first point of
// the block along the sweep; jj = 0..MT+7 covers the 4-point halos.
template <int NF, int MT, int TLC, int DIR, typename TS, int NTT = NT>
__device__ __forceinline__ void tiles_ct(const CssGeo &g, const TS *const *f, double *S, size_t FS, int SR,
                                         int a0, int lb, int fixed, const double *const *mp = nullptr) {
  constexpr int W = MT + 8, N = TLC * W, IT = (N + NTT - 1) / NTT;
  double val[NF][IT];
  int so[IT];
  size_t go[IT], bb[IT];
#pragma unroll
  for (int k = 0; k < IT; k++) {
    const int idx = threadIdx.x + k * NTT;
    int l, jj;
    if (DIR == 1) { l = idx / W; jj = idx - l * W; }
    else { jj = idx / TLC; l = idx - jj * TLC; }
    bool ok = idx < N;
    size_t off;
    if (DIR == 1) {
      const int gt = a0 + jj - 4, gp = lb + l;
      ok = ok && gt >= 0 && gt < g.nth && gp < g.nphi;
      off = plane(g, fixed) + (size_t)gp * g.nth + gt;
      so[k] = l * SR + jj;
    } else if (DIR == 2) {
      int gp = a0 + jj - 4;
      if (gp < 0) gp += g.nphi;
      else if (gp >= g.nphi) gp -= g.nphi;
      const int gt = lb + l;
      ok = ok && gt < g.nth;
      off = plane(g, fixed) + (size_t)gp * g.nth + gt;
      so[k] = jj * SR + l;
    } else {
      const int gr = a0 + jj - 4, gt = lb + l;
      ok = ok && gr >= 0 && gr < g.nr && gt < g.nth;
      off = plane(g, gr < 0 ? 0 : gr) + (size_t)fixed * g.nth + gt;
      so[k] = jj * SR + l;
    }
    {
      const int r_ = DIR == 0 ? (ok ? a0 + jj - 4 : 0) : fixed;
      const int t_ = DIR == 1 ? a0 + jj - 4 : lb + l;
      bb[k] = ok ? bgi(g, r_, t_) : 0;
    }
    if (!ok) so[k] = -1;
    go[k] = ok ? off : 0;
  }
#pragma unroll
  for (int q = 0; q < NF; q++)
#pragma unroll
    for (int k = 0; k < IT; k++) val[q][k] = (so[k] >= 0) ? st_val(f[q], go[k], mp ? mp[q] : nullptr, bb[k]) : 0.0;
#pragma unroll
  for (int q = 0; q < NF; q++)
#pragma unroll
    for (int k = 0; k < IT; k++)
      if (so[k] >= 0) S[(size_t)q * FS + so[k]] = val[q][k];
}

// Line-solve phase, field of a slot.  With 16-line tiles and 128 threads,
// slot = task / 16 and a warp holds two slots.  When the fields leave room
// (nd <= 7) the second-derivative field k2 gets slot 6 with slot 7 idle, and
// the others fill slots 0.. in order, so no warp runs both line operators
// one after the other.  -1: an idle slot.
template <int TLC>
__device__ __forceinline__ int solve_field(int slot, int nd, int k2) {
  if (TLC != 16 || nd > 7) return slot < nd ? slot : -1;
  if (slot == 6) return k2;
  if (slot >= 7 || slot >= nd - 1) return -1;
  return slot < k2 ? slot : slot + 1;
}
template <int TLC>
__device__ __forceinline__ int solve_tasks(int nd, int TL) {
  return (TLC == 16 && nd <= 7) ? 8 * TL : nd * TL;
}

// ---------------------------------------------------------------------------
// Source_Theta_Terms (rhs_mpi.f90:786-1029) + Induction_Terms (:2340-2346)
// grid: x = theta block * nchunk + phi chunk, y = r.  cur = stage input
// (vars1), B = curl A (MHD) in bf, dv = dvars1 (written, not read), tbuf =
// the stage temperature (written here, read by the later kernels).
// ---------------------------------------------------------------------------
template <int MT, int TLC, typename TV, int MAG>
__global__ void __launch_bounds__(128) k_theta_terms(CssGeo g, const TV *__restrict__ cur,
                                                     const double *__restrict__ bf, double *__restrict__ dv,
                                                     double *__restrict__ tbuf, int TLrt) {
  extern __shared__ double sm[];
  const int TL = TLC ? TLC : TLrt;
  const int nchunk = (g.nphi + TL - 1) / TL;
  const int bt = blockIdx.x / nchunk, pb = (blockIdx.x - bt * nchunk) * TL;
  const int ir = blockIdx.y;
  const CssDir &D = g.d[1];
  const int t0 = D.start[bt], m = MT ? MT : D.size[bt];
  const int dtype = dtype_of(D, bt);
  constexpr int mag = MAG;  // compile-time: a hydro run carries no MHD code
  const int SR = m + 9, SO = m + 1, TS = 3 * (m + 2);
  const size_t n = (size_t)g.ncell;
  const int nh = mag ? 6 : 4;   // w v u s [bp br]
  const int nd = mag ? 7 : 5;   // dw dv du ds d2s [dbp dbr]
  double *H = sm;
  double *O = H + (size_t)nh * TL * SR;
  double *Tb = O + (size_t)nd * TL * SO;
  const TV *fs[4] = {cur + n, cur + 2 * n, cur + 3 * n, cur + 4 * n};
  const double *ms[4] = {nullptr, nullptr, nullptr, bg_s(g)};
  const double *fb[2] = {bf + n, bf + 2 * n};
  if constexpr (MT > 0 && TLC > 0) {
    tiles_ct<4, MT, TLC, 1>(g, fs, H, (size_t)TL * SR, SR, t0, pb, ir, ms);
    if (mag) tiles_ct<2, MT, TLC, 1>(g, fb, H + (size_t)4 * TL * SR, (size_t)TL * SR, SR, t0, pb, ir);
  } else {
    for (int k = 0; k < 4; k++) tile_theta<MT, TLC>(g, fs[k], H + (size_t)k * TL * SR, SR, t0, m, pb, TL, ir, ms[k]);
    for (int k = 4; k < nh; k++) tile_theta<MT, TLC>(g, fb[k - 4], H + (size_t)k * TL * SR, SR, t0, m, pb, TL, ir);
  }
  const int var[7] = {2, 3, 4, 5, 5, 8, 9};
  for (int k = 0; k < nd; k++) stage_table(g, 1, bt, k == 4 ? 2 : 1, g.ibct[var[k]], m, Tb + k * TS);
  __syncthreads();
  const double ri = g.r_inv[ir];
  for (int task = threadIdx.x; task < solve_tasks<TLC>(nd, TL); task += blockDim.x) {
    const int slot = task / TL, l = task - slot * TL;
    const int k = solve_field<TLC>(slot, nd, 4);
    if (k < 0 || pb + l >= g.nphi) continue;
    if (k == 4 && !g.slaplacian) continue;
    int hk = (k <= 3) ? k : (k == 4 ? 3 : k - 1);
    const double *x = H + ((size_t)hk * TL + l) * SR + 4;
    double *o = O + ((size_t)k * TL + l) * SO;
    int bdry = g.ibct[var[k]];
    double lo = 0.0, hi = 0.0;
    if (k == 1) {  // stress-free datum cot(theta)*v on the walls (rhs_mpi.f90:414, :444)
      if (D.lphys[bt]) lo = (g.cosines[0] / g.sines[0]) * x[0];
      if (D.rphys[bt]) hi = (g.cosines[g.nth - 1] / g.sines[g.nth - 1]) * x[m - 1];
    }
    if (k == 5 && g.theta_normal_field) {  // (rhs_mpi.f90:421, :451)
      if (D.lphys[bt]) lo = -(g.cosines[0] / g.sines[0]) * x[0];
      if (D.rphys[bt]) hi = -(g.cosines[g.nth - 1] / g.sines[g.nth - 1]) * x[m - 1];
    }
    if (k == 4)
      solve<2, MT>(x, 1, m, dtype, bdry, lo, hi, Tb + k * TS, m + 2, dnum_d2_theta(g, ir), D.dnum[bt] * D.dnum[bt],
                   0, o, 1);
    else
      solve<1, MT>(x, 1, m, dtype, bdry, lo, hi, Tb + k * TS, m + 2, D.dnum[bt], D.dnum[bt], 0, o, 1);
  }
  __syncthreads();
  const double rv = g.r_ind[ir], epsr = g.eps[ir];
  const double omsq = rv * g.omega0 * g.omega0, om2 = 2.0 * g.omega0;
  const size_t pl = plane(g, ir);
  // points per thread: their global loads (rho, B_theta) go out before any store
  constexpr int PPT = (MT > 0 && TLC > 0) ? (MT * TLC + NT - 1) / NT : 1;
  constexpr int STRIDE = (MT > 0 && TLC > 0) ? NT : 0;
  const int stride = STRIDE ? STRIDE : blockDim.x;
  for (int pt0 = threadIdx.x; pt0 < TL * m; pt0 += PPT * stride) {
  double rho_[PPT], bt_in[PPT];
#pragma unroll
  for (int k = 0; k < PPT; k++) {
    const int pt = pt0 + k * stride;
    const int l = pt / m, j = pt - l * m;
    const bool ok = pt < TL * m && pb + l < g.nphi;
    const size_t id = pl + (size_t)(pb + l) * g.nth + t0 + j;
    rho_[k] = ok ? st_val(cur, id, bg_rho(g), bgi(g, ir, t0 + j)) : 1.0;
    bt_in[k] = (ok && mag) ? __ldg(bf + id) : 0.0;
  }
#pragma unroll
  for (int k = 0; k < PPT; k++) {
    const int pt = pt0 + k * stride;
    if (pt >= TL * m) continue;
    int l = pt / m, j = pt - l * m;
    int it = t0 + j, ip = pb + l;
    if (ip >= g.nphi) continue;
    size_t id = pl + (size_t)ip * g.nth + it;
    double sn = g.sines[it], cs = g.cosines[it], ct = g.cot[it];
    double rho = rho_[k];
    const double *hl = H + (size_t)l * SR + 4 + j;
    double w = hl[0], v = hl[(size_t)TL * SR], u = hl[(size_t)2 * TL * SR], s = hl[(size_t)3 * TL * SR];
    const double *ol = O + (size_t)l * SO + j;
    double dw = omsq * sn * cs;
    double du = -g.grav[ir] + omsq * sn * sn;
    double drho = -rho * w * ct * ri;
    double dvv = -om2 * cs * w;
    du = du + ri * w * w;
    double w1 = ol[0] * ri;
    drho = drho - rho * w1;
    dw = dw - w * w1;
    dw = dw + v * (ri * ct * v + om2 * cs);
    dvv = dvv - ri * v * w * ct;
    du = du + v * (ri * v + om2 * sn);
    w1 = ol[(size_t)1 * TL * SO] * ri;
    dvv = dvv - w * w1;
    dv[id] = drho - 2.0 * ri * rho * u;
    dvv = dvv - u * (ri * v + om2 * sn);
    dw = dw - ri * u * w;
    w1 = ol[(size_t)2 * TL * SO] * ri;
    du = du - w * w1;
    double t = temp_of(g, rho, s);
    tbuf[id] = t;
    double invrho = 1.0 / rho;
    const double oorho_t = invrho / t;
    double ds;
    if (fabs(epsr) > 0.0) ds = epsr * oorho_t;
    else ds = 0.0;
    w1 = ol[(size_t)3 * TL * SO] * ri;
    double dwfin = dw - g.gamm1 * t * w1;
    ds = ds - w * w1;
    if (g.slaplacian) {
      double ddiff = ri * g.ks[ir];
      double oorho = oorho_t;
      w1 = ddiff * w1 * oorho;
      ds = ds + ct * w1;
      double dd2 = ddiff * ri * ri;  // ks/r^3 as rhs_mpi.f90:972 has it
      ds = ds + dd2 * ol[(size_t)4 * TL * SO] * oorho;
    }
    dv[4 * n + id] = ds;
    if (!mag) {
      dv[n + id] = dwfin;
      dv[2 * n + id] = dvv;
      dv[3 * n + id] = du;
    } else {
      dw = dwfin;
      double oo = invrho;
      oo = oo * ONE_OVER_4PI * ri;
      double bt_ = bt_in[k], bp_ = hl[(size_t)4 * TL * SR], br_ = hl[(size_t)5 * TL * SR];
      du = du - bt_ * bt_ * oo;
      dw = dw - bp_ * bp_ * ct * oo;
      dvv = dvv + bp_ * bt_ * ct * oo;
      du = du - bp_ * bp_ * oo;
      w1 = ol[(size_t)5 * TL * SO] * oo;
      dvv = dvv + bt_ * w1;
      dw = dw - bp_ * w1;
      w1 = ol[(size_t)6 * TL * SO] * oo;
      dv[n + id] = dw + br_ * (bt_ * oo - w1);
      dv[2 * n + id] = dvv + br_ * bp_ * oo;
      dv[3 * n + id] = du + bt_ * w1;
      // Induction_Terms: dA/dt = v x B
      dv[5 * n + id] = v * br_ - u * bp_;
      dv[6 * n + id] = u * bt_ - w * br_;
      dv[7 * n + id] = w * bp_ - v * bt_;
    }
  }
  }
}

// ---------------------------------------------------------------------------
// Phi_Terms (rhs_mpi.f90:1032-1261).  grid: x = phi block * nchunk + theta
// chunk, y = r.
// ---------------------------------------------------------------------------
// tables, line solves and pointwise physics of one phi tile whose fields are
// in H (shared by the one-tile-per-CTA kernel and the persistent one)
template <int MT, int TLC, int MAG>
__device__ __forceinline__ void phi_tile_compute(const CssGeo &g, const double *__restrict__ bf,
                                                 double *__restrict__ dv, const double *__restrict__ tbuf, int TL,
                                                 int bp, int tb, int ir, double *H, double *O, double *Tb) {
  const CssDir &D = g.d[2];
  const int p0 = D.start[bp], m = MT ? MT : D.size[bp];
  constexpr int mag = MAG;
  const int SR = TL + 1, TS = 3 * (m + 2);
  const size_t n = (size_t)g.ncell;
  const int nd = mag ? 8 : 6;
  const size_t HS = (size_t)(m + 8) * SR, OS = (size_t)m * SR;
  stage_table(g, 2, bp, 1, 0, m, Tb);
  stage_table(g, 2, bp, 2, 0, m, Tb + TS);
  __syncthreads();
  for (int task = threadIdx.x; task < solve_tasks<TLC>(nd, TL); task += blockDim.x) {
    const int slot = task / TL, l = task - slot * TL;
    const int k = solve_field<TLC>(slot, nd, 5);
    if (k < 0 || tb + l >= g.nth) continue;
    if (k == 5 && !g.slaplacian) continue;
    int hk = (k <= 4) ? k : (k == 5 ? 4 : k - 1);
    const double *x = H + hk * HS + 4 * SR + l;
    double *o = O + k * OS + l;
    if (k == 5)
      solve<2, MT>(x, SR, m, 3, 0, 0.0, 0.0, Tb + TS, m + 2, D.dnum[bp], D.dnum[bp] * D.dnum[bp], 1, o, SR);
    else
      solve<1, MT>(x, SR, m, 3, 0, 0.0, 0.0, Tb, m + 2, D.dnum[bp], D.dnum[bp], 1, o, SR);
  }
  __syncthreads();
  const double ri = g.r_inv[ir];
  const size_t pl = plane(g, ir);
  // points per thread; the loads of all of a thread's points are issued
  // before any store (dv is read and written, so the compiler cannot move
  // loads across the stores by itself)
  constexpr int PPT = (MT > 0 && TLC > 0) ? (MT * TLC + 127) / 128 : 1;
  for (int pt0 = threadIdx.x; pt0 < TL * m; pt0 += PPT * blockDim.x) {
    double in_[PPT][6];
    size_t ids[PPT];
    bool ok[PPT];
#pragma unroll
    for (int k = 0; k < PPT; k++) {
      int pt = pt0 + k * blockDim.x;
      int j = pt / TL, l = pt - j * TL;
      ok[k] = pt < TL * m && tb + l < g.nth;
      ids[k] = pl + (size_t)(p0 + j) * g.nth + tb + l;
      if (ok[k]) {
        size_t id = ids[k];
        in_[k][0] = dv[id]; in_[k][1] = dv[n + id]; in_[k][2] = dv[2 * n + id];
        in_[k][3] = dv[3 * n + id]; in_[k][4] = dv[4 * n + id]; in_[k][5] = __ldg(tbuf + id);
      }
    }
#pragma unroll
    for (int k = 0; k < PPT; k++) {
      if (!ok[k]) continue;
      int pt = pt0 + k * blockDim.x;
      int j = pt / TL, l = pt - j * TL;
      int it = tb + l;
      size_t id = ids[k];
      const double *hl = H + (size_t)(j + 4) * SR + l;
      double rho = hl[0], v = hl[HS];
      const double *ol = O + (size_t)j * SR + l;
      double cscth = g.csc[it];
      double oors = ri * cscth;
      double t = in_[k][5], oorho = 1.0 / rho;
      double w1 = ol[0] * oors;
      double drho = in_[k][0];
      double dvv = in_[k][2];
      drho = drho - v * w1;
      dvv = dvv - g.pconst * w1 * t * oorho;
      double ds = in_[k][4];
      w1 = ol[OS] * oors;
      dvv = dvv - v * w1;
      double drho_out = drho - rho * w1;
      double dw = in_[k][1];
      w1 = ol[2 * OS] * oors;
      dw = dw - v * w1;
      double du = in_[k][3];
      w1 = ol[3 * OS] * oors;
      du = du - v * w1;
      w1 = ol[4 * OS] * oors;
      ds = ds - v * w1;
      dvv = dvv - g.gamm1 * t * w1;
      if (g.slaplacian) {
        w1 = ol[5 * OS] * (oors * oors);
        ds = ds + g.ks[ir] * w1 * (oorho / t);
      }
      dv[id] = drho_out;
      dv[4 * n + id] = ds;
      if (!mag) {
        dv[n + id] = dw;
        dv[3 * n + id] = du;
        dv[2 * n + id] = dvv;
      } else {
        double oo = ONE_OVER_4PI * oorho * oors;
        double bt_ = hl[5 * HS], br_ = hl[6 * HS], bp_ = __ldg(bf + n + id);
        w1 = ol[6 * OS] * oo;
        dvv = dvv - bt_ * w1;
        dv[n + id] = dw + bp_ * w1;
        w1 = ol[7 * OS] * oo;
        dv[2 * n + id] = dvv - br_ * w1;
        dv[3 * n + id] = du + bp_ * w1;
      }
    }
  }
}

template <int MT, int TLC, typename TV, int MAG>
__global__ void __launch_bounds__(128) k_phi_terms(CssGeo g, const TV *__restrict__ cur,
                                                   const double *__restrict__ bf, double *__restrict__ dv,
                                                   const double *__restrict__ tbuf, int TLrt) {
  extern __shared__ double sm[];
  const int TL = TLC ? TLC : TLrt;
  const int nchunk = (g.nth + TL - 1) / TL;
  const int bp = blockIdx.x / nchunk, tb = (blockIdx.x - bp * nchunk) * TL;
  const int ir = blockIdx.y;
  const CssDir &D = g.d[2];
  const int p0 = D.start[bp], m = MT ? MT : D.size[bp];
  constexpr int mag = MAG;
  const int SR = TL + 1;
  const size_t n = (size_t)g.ncell;
  const int nh = mag ? 7 : 5;  // rho v w u s [bt br]
  const int nd = mag ? 8 : 6;  // drho dv dw du ds d2s [dbt dbr]
  const size_t HS = (size_t)(m + 8) * SR, OS = (size_t)m * SR;
  double *H = sm;
  double *O = H + nh * HS;
  double *Tb = O + nd * OS;
  // the pointwise phase reads dv (5 fields), T [and B_phi] at every point of
  // the tile: start those lines toward L2 now, they are needed after the solves
  for (int k = threadIdx.x; k < m; k += blockDim.x) {
    const size_t id = plane(g, ir) + (size_t)(p0 + k) * g.nth + tb;
    if (tb < g.nth) {
      for (int f = 0; f < 5; f++) prefetch_l2(dv + f * n + id);
      prefetch_l2(tbuf + id);
      if (mag) prefetch_l2(bf + n + id);
    }
  }
  const TV *fs[5] = {cur, cur + 2 * n, cur + n, cur + 3 * n, cur + 4 * n};
  const double *ms[5] = {bg_rho(g), nullptr, nullptr, nullptr, bg_s(g)};
  const double *fb[2] = {bf, bf + 2 * n};
  if constexpr (MT > 0 && TLC > 0) {
    tiles_ct<5, MT, TLC, 2>(g, fs, H, HS, SR, p0, tb, ir, ms);
    if (mag) tiles_ct<2, MT, TLC, 2>(g, fb, H + 5 * HS, HS, SR, p0, tb, ir);
  } else {
    for (int k = 0; k < 5; k++) tile_phi<MT, TLC>(g, fs[k], H + k * HS, SR, p0, m, tb, TL, ir, ms[k]);
    for (int k = 5; k < nh; k++) tile_phi<MT, TLC>(g, fb[k - 5], H + k * HS, SR, p0, m, tb, TL, ir);
  }
  phi_tile_compute<MT, TLC, MAG>(g, bf, dv, tbuf, TL, bp, tb, ir, H, O, Tb);
}

// Phi_Terms as a persistent kernel (FP64 stage input, compile-time block
// length and tile height): each CTA walks tiles t = blockIdx.x,
// blockIdx.x + gridDim.x, ... in the (r, phi block, theta chunk) order of
// k_phi_terms; the next tile's fields stream into the second of two
// shared-memory buffers with asynchronous 8-byte copies (zero fill past
// nth, periodic phi) while the current tile is solved and its physics done.
template <int NF, int MT, int TLC>
__device__ __forceinline__ void phi_tile_issue(const CssGeo &g, const double *const *f, double *S, size_t FS,
                                               int SR, int p0, int tb, int ir) {
  constexpr int W = MT + 8, N = TLC * W;
  const size_t pl = plane(g, ir);
  for (int idx = threadIdx.x; idx < N; idx += NT) {
    const int jj = idx / TLC, l = idx - jj * TLC;
    int gp = p0 + jj - 4;
    if (gp < 0) gp += g.nphi;
    else if (gp >= g.nphi) gp -= g.nphi;
    const int gt = tb + l;
    const bool in = gt < g.nth;
    const size_t off = pl + (size_t)gp * g.nth + (in ? gt : 0);
#pragma unroll
    for (int q = 0; q < NF; q++) cp_async8(S + q * FS + (size_t)jj * SR + l, f[q] + off, in ? 8 : 0);
  }
}

template <int MT, int TLC>
__global__ void __launch_bounds__(128) k_phi_terms_p(CssGeo g, const double *__restrict__ cur,
                                                     const double *__restrict__ bf, double *__restrict__ dv,
                                                     const double *__restrict__ tbuf) {
  static_assert(MT > 0 && TLC > 0, "persistent phi kernel needs compile-time sizes");
  extern __shared__ double sm[];
  constexpr int TL = TLC, m = MT, SR = TLC + 1;
  const int nchunk = (g.nth + TL - 1) / TL, nbp = g.d[2].nb;
  const long long per_r = (long long)nbp * nchunk, ntile = per_r * g.nr;
  const int mag = g.magnetic;
  const int nh = mag ? 7 : 5, nd = mag ? 8 : 6;
  const size_t n = (size_t)g.ncell;
  const size_t HS = (size_t)(m + 8) * SR, OS = (size_t)m * SR;
  double *Hb[2] = {sm, sm + (size_t)nh * HS};
  double *O = sm + (size_t)2 * nh * HS;
  double *Tb = O + (size_t)nd * OS;
  const double *fs[5] = {cur, cur + 2 * n, cur + n, cur + 3 * n, cur + 4 * n};
  const double *fb[2] = {bf, bf + 2 * n};
  auto issue = [&](long long t, double *H) {
    const int ir = (int)(t / per_r), x = (int)(t - (long long)ir * per_r);
    const int bp = x / nchunk, tb = (x - bp * nchunk) * TL;
    const int p0 = g.d[2].start[bp];
    phi_tile_issue<5, MT, TLC>(g, fs, H, HS, SR, p0, tb, ir);
    if (mag) phi_tile_issue<2, MT, TLC>(g, fb, H + 5 * HS, HS, SR, p0, tb, ir);
    cp_async_commit();
  };
  long long t = blockIdx.x;
  if (t < ntile) issue(t, Hb[0]);
  for (int it = 0; t < ntile; it++, t += gridDim.x) {
    double *H = Hb[it & 1];
    cp_async_wait<0>();
    __syncthreads();  // tile t is in H; the previous tile's readers are done
    if (t + gridDim.x < ntile) issue(t + gridDim.x, Hb[(it + 1) & 1]);
    const int ir = (int)(t / per_r), x = (int)(t - (long long)ir * per_r);
    const int bp = x / nchunk, tb = (x - bp * nchunk) * TL;
    if (mag) phi_tile_compute<MT, TLC, 1>(g, bf, dv, tbuf, TL, bp, tb, ir, H, O, Tb);
    else phi_tile_compute<MT, TLC, 0>(g, bf, dv, tbuf, TL, bp, tb, ir, H, O, Tb);
  }
  cp_async_wait<0>();
}

// pointwise Radial_Terms (rhs_mpi.f90:1302-1517) for one point: updates
// drho, dw, dv, du, ds (in: the values accumulated so far)
struct RadIn {
  double u, rho, t, dw_r, dv_r, du_r, ds_r, d2s_r, bt, bp, br, dbt_r, dbp_r;
};
template <int MAG>
__device__ __forceinline__ void radial_point(const CssGeo &g, int ir, const RadIn &q, double &drho, double &dw,
                                             double &dvv, double &du, double &ds) {
  const int nu = g.non_uniform;
  const double w3 = g.dxdr[ir];
  const double invrho = 1.0 / q.rho;
  double w1 = q.dw_r;
  if (nu) w1 = w1 * w3;
  dw = dw - q.u * w1;
  w1 = q.dv_r;
  if (nu) w1 = w1 * w3;
  dvv = dvv - q.u * w1;
  w1 = q.du_r;
  if (nu) w1 = w1 * w3;
  du = du - q.u * w1;
  drho = drho - q.rho * w1;
  w1 = q.ds_r;
  if (nu) w1 = w1 * w3;
  du = du - g.gamm1 * q.t * w1;
  ds = ds - q.u * w1;
  if (g.slaplacian) {
    double oorho = invrho / q.t;
    double work6 = (2.0 * g.r_inv[ir] + g.dlnks[ir]) * g.ks[ir];
    w1 = w1 * oorho;
    ds = ds + w1 * work6;
    if (nu) ds = ds + (g.d2xdr2[ir] / w3) * w1 * g.ks[ir];
    double d2 = q.d2s_r;
    if (nu) d2 = d2 * (w3 * w3);
    ds = ds + g.ks[ir] * d2 * oorho;
  }
  if (MAG) {
    double oo = invrho * ONE_OVER_4PI;
    w1 = q.dbt_r;
    if (nu) w1 = w1 * w3;
    w1 = w1 * oo;
    du = du - q.bt * w1;
    dw = dw + q.br * w1;
    w1 = q.dbp_r;
    if (nu) w1 = w1 * w3;
    w1 = w1 * oo;
    dvv = dvv + q.br * w1;
    du = du - q.bp * w1;
  }
}

// The face-plane relaxation of an open radial boundary at one point of the
// radial tile: hl is the point's row of the tile (w, v, u, s at 0..3 HS),
// q its plane index.  Top: rhs_mpi.f90:2042-2066; bottom: :1913-1952.
__device__ __forceinline__ void inout_face(const CssGeo &g, int j, int m, bool top, const double *hl, int SR,
                                           size_t HS, size_t q, double &drho, double &dw, double &dvv, double &du,
                                           double &ds) {
  const double *io = g.inout;
  if (top) {
    if (j != m - 1) return;
    const double ut = hl[2 * HS], st = hl[3 * HS], ub = hl[2 * HS - SR], sb = hl[3 * HS - SR];
    if (g.rain) {
      const double taur = io[IO_TOP_TAUR];
      du = du + (io[IO_TOP_MDVEL] + g.dvel_rain[q] + ub - 2.0 * ut) * taur + io[IO_TOP_MEANU];
      ds = ds + (g.sr[0] + g.delta_s + g.dent_rain[q] + sb - 2.0 * st) * taur;
    } else {
      const double tau = io[IO_TOP_TAU];
      du = du + tau * (io[IO_TOP_NRAT] * ub - ut) + io[IO_TOP_MEANU];
      ds = ds + tau * (sb - st) + io[IO_TOP_MEANS];
    }
    return;
  }
  if (j != 0) return;
  const double u0 = hl[2 * HS], s0 = hl[3 * HS], tau = io[IO_BOT_TAU];
  if (g.bottom_specified) {
    const size_t np = (size_t)g.nth * g.nphi;
    const double tc = io[IO_BOT_TCONST];
    drho = drho + io[IO_BOT_MEANU];
    // the u_theta term is added in k_rhot_update, after Density_Terms_Theta
    // has read the accumulated dw for its wall datum (rhs_mpi.f90:705, :724)
    dvv = dvv + tau * (tc * g.ashv[2 * np + q] - hl[HS]);
    du = du + tau * (tc * g.ashv[q] - u0);
    ds = ds + tau * ((g.sr[0] + io[IO_BOT_FEN] * g.ashv[3 * np + q]) - s0);
  } else {
    const double ua = hl[2 * HS + SR], sa = hl[3 * HS + SR];
    drho = drho + io[IO_BOT_TCONST];
    du = du + tau * (io[IO_BOT_NRAT] * ua - u0) + io[IO_BOT_MEANU];
    ds = ds + tau * (sa - s0 + io[IO_BOT_MEANS]);
  }
}

// ---------------------------------------------------------------------------
// Radial_Terms (rhs_mpi.f90:1264-1519) + Density_Terms_Radial (:1710-1855)
// grid: x = r block * nchunk + theta chunk, y = phi.
// d(rho)/dr on a block with a physical face is linear in the face datum
// (the hydrostatic condition built from the completed du/dt on that face):
// it is solved with a zero datum together with the other derivatives and
// the datum times the block's unit response (resp) is added afterwards.
// ---------------------------------------------------------------------------
// One tile of Radial_Terms + Density_Terms_Radial: r block br, theta lines
// tb .. tb+TL-1, phi ip; sm is the CTA's shared buffer.  KIND: 0 a closed
// hydro run, 1 a hydro run with open radial faces, 2 MHD; KIND 1 compiles
// the open radial boundaries in (a run with top_inout or bot_inout); the
// closed instance carries none of their code.
template <int MT, int TLC, typename TV, int KIND>
__device__ __forceinline__ void radial_tile(const CssGeo &g, const TV *__restrict__ cur, const double *__restrict__ bf,
                                            double *__restrict__ dv, const double *__restrict__ tbuf, int TL, int br,
                                            int tb, int ip, double *sm) {
  const CssDir &D = g.d[0];
  const int r0 = D.start[br], m = MT ? MT : D.size[br];
  const int dtype = dtype_of(D, br);
  constexpr int mag = KIND == 2;  // known at compile time: a hydro run carries no MHD code
  const int SR = TL, TS = 3 * (m + 2);  // lines contiguous, unpadded (4 CTAs per SM)
  const size_t n = (size_t)g.ncell;
  const int nh = mag ? 7 : 5;  // w v u s rho [bt bp]
  const int nd = mag ? 8 : 6;  // dw dv du ds d2s drho0 [dbt dbp]
  const size_t HS = (size_t)(m + 8) * SR, OS = (size_t)m * SR;
  double *H = sm;
  double *O = H + nh * HS;
  double *Tb = O + nd * OS;
  double *datum = Tb + nd * TS;
  // lines of dv (5 fields), T [and B_r] the pointwise phase will read
  for (int k = threadIdx.x; k < m; k += blockDim.x) {
    const size_t id = (size_t)ip * g.nth + tb + (size_t)(r0 + k) * g.nth * g.nphi;
    if (tb < g.nth) {
      for (int f = 0; f < 5; f++) prefetch_l2(dv + f * n + id);
      prefetch_l2(tbuf + id);
      if (mag) prefetch_l2(bf + 2 * n + id);
    }
  }
  const TV *fs[5] = {cur + n, cur + 2 * n, cur + 3 * n, cur + 4 * n, cur};
  const double *ms[5] = {nullptr, nullptr, nullptr, bg_s(g), bg_rho(g)};
  const double *fb[2] = {bf, bf + n};
  if constexpr (MT > 0 && TLC > 0) {
    tiles_ct<5, MT, TLC, 0>(g, fs, H, HS, SR, r0, tb, ip, ms);
    if (mag) tiles_ct<2, MT, TLC, 0>(g, fb, H + 5 * HS, HS, SR, r0, tb, ip);
  } else {
    for (int k = 0; k < 5; k++) tile_r<MT, TLC>(g, fs[k], H + k * HS, SR, r0, m, tb, TL, ip, ms[k]);
    for (int k = 5; k < nh; k++) tile_r<MT, TLC>(g, fb[k - 5], H + k * HS, SR, r0, m, tb, TL, ip);
  }
  const int var[8] = {2, 3, 4, 5, 5, 1, 7, 8};
  // open faces (a radial block has at most one physical face): the top one
  // takes d(rho)/dr with bdry 2 and no datum, the bottom one with the datum
  // left in x-space (rhs_mpi.f90:2020-2023, :1895-1898)
  const bool top_open = KIND == 1 && D.rphys[br] && g.top_inout, bot_open = KIND == 1 && D.lphys[br] && g.bot_inout;
  auto bdry_of = [&](int k) { return (k == 5 && top_open) ? 2 : g.ibcr[var[k]]; };
  for (int k = 0; k < nd; k++) stage_table(g, 0, br, k == 4 ? 2 : 1, bdry_of(k), m, Tb + k * TS);
  __syncthreads();
  const int nr = g.nr;
  for (int task = threadIdx.x; task < solve_tasks<TLC>(nd, TL); task += blockDim.x) {
    const int slot = task / TL, l = task - slot * TL;
    const int k = solve_field<TLC>(slot, nd, 4);
    if (k < 0 || tb + l >= g.nth) continue;
    if (k == 4 && !g.slaplacian) continue;
    int hk = (k <= 3) ? k : (k == 4 ? 3 : (k == 5 ? 4 : k - 1));
    const double *x = H + hk * HS + 4 * SR + l;
    double *o = O + k * OS + l;
    int bdry = bdry_of(k);
    double lo = 0.0, hi = 0.0;
    if (k == 0 || k == 1) {  // stress-free datum w/r/dxdr (rhs_mpi.f90:578-614)
      if (D.lphys[br] && g.bottom_stress_free) lo = x[0] / g.r1 / g.dxdr[0];
      if (D.rphys[br]) {
        if (g.top_stress_free) hi = x[(m - 1) * SR] / g.r2 / g.dxdr[nr - 1];
        else hi = x[(m - 1) * SR];
      }
    }
    if (k == 3 || k == 4) {  // constant-flux datum (rhs_mpi.f90:584-592, :616-624)
      lo = g.s_flux_lo;
      hi = g.s_flux_hi;
    }
    if (bot_open) lo = 0.0;  // open faces: data of w, v, u, s zero (rhs_mpi.f90:594-596, :626-628)
    if (top_open) hi = 0.0;
    if (k == 4)
      solve<2, MT>(x, SR, m, dtype, bdry, lo, hi, Tb + k * TS, m + 2, D.dnum[br], D.dnum[br] * D.dnum[br], 0, o, SR);
    else
      solve<1, MT>(x, SR, m, dtype, bdry, lo, hi, Tb + k * TS, m + 2, D.dnum[br], D.dnum[br], 0, o, SR);
  }
  __syncthreads();
  const size_t ps = (size_t)g.nth * g.nphi;
  const size_t base = (size_t)ip * g.nth + tb;
  auto gather = [&](int j, int l, RadIn &q) {
    const double *hl = H + (size_t)(j + 4) * SR + l;
    const double *ol = O + (size_t)j * SR + l;
    size_t id = base + (size_t)(r0 + j) * ps + l;
    q.u = hl[2 * HS];
    q.rho = hl[4 * HS];
    q.t = __ldg(tbuf + id);
    q.dw_r = ol[0]; q.dv_r = ol[OS]; q.du_r = ol[2 * OS]; q.ds_r = ol[3 * OS]; q.d2s_r = ol[4 * OS];
    if (mag) {
      q.bt = hl[5 * HS]; q.bp = hl[6 * HS]; q.br = __ldg(bf + 2 * n + id);
      q.dbt_r = ol[6 * OS]; q.dbp_r = ol[7 * OS];
    }
    return id;
  };
  // hydrostatic datum of d(rho)/dr on a physical face (rhs_mpi.f90:1750-1768)
  const int phys = D.lphys[br] ? 1 : (D.rphys[br] && !top_open ? 2 : 0);
  if (phys) {
    for (int l = threadIdx.x; l < TL; l += blockDim.x) {
      if (tb + l >= g.nth) continue;
      int j = phys == 1 ? 0 : m - 1;
      RadIn q;
      size_t id = gather(j, l, q);
      double drho = dv[id], dw = dv[n + id], dvv = dv[2 * n + id], du = dv[3 * n + id], ds = dv[4 * n + id];
      radial_point<mag>(g, r0 + j, q, drho, dw, dvv, du, ds);
      double d;
      if (bot_open) {
        d = g.invpconst * q.rho * du / q.t;  // rhs_mpi.f90:1894
      } else {
        if (g.lbcr_rho == 4 || g.lbcr_rho == (phys == 1 ? 2 : 3)) d = du * q.rho * g.invpconst / q.t;
        else d = q.rho;
        if (g.non_uniform) d = d / g.dxdr[phys == 1 ? 0 : nr - 1];
      }
      datum[l] = d;
    }
    __syncthreads();
  }
  const double *resp = g.resp_r + (size_t)(2 * br + (phys == 2 ? 1 : 0)) * g.tstride;
  constexpr int PPT = (MT > 0 && TLC > 0) ? (MT * TLC + 127) / 128 : 1;
  for (int pt0 = threadIdx.x; pt0 < TL * m; pt0 += PPT * blockDim.x) {
    double in_[PPT][7];
    bool ok[PPT];
#pragma unroll
    for (int k = 0; k < PPT; k++) {
      int pt = pt0 + k * blockDim.x;
      int j = pt / TL, l = pt - j * TL;
      ok[k] = pt < TL * m && tb + l < g.nth;
      if (ok[k]) {
        size_t id = base + (size_t)(r0 + j) * ps + l;
        in_[k][0] = dv[id]; in_[k][1] = dv[n + id]; in_[k][2] = dv[2 * n + id];
        in_[k][3] = dv[3 * n + id]; in_[k][4] = dv[4 * n + id]; in_[k][5] = __ldg(tbuf + id);
        in_[k][6] = mag ? __ldg(bf + 2 * n + id) : 0.0;
      }
    }
#pragma unroll
    for (int k = 0; k < PPT; k++) {
      if (!ok[k]) continue;
      int pt = pt0 + k * blockDim.x;
      int j = pt / TL, l = pt - j * TL;
      int ir = r0 + j;
      size_t id = base + (size_t)(r0 + j) * ps + l;
      const double *hl = H + (size_t)(j + 4) * SR + l;
      const double *ol = O + (size_t)j * SR + l;
      RadIn q;
      q.u = hl[2 * HS];
      q.rho = hl[4 * HS];
      q.t = in_[k][5];
      q.dw_r = ol[0]; q.dv_r = ol[OS]; q.du_r = ol[2 * OS]; q.ds_r = ol[3 * OS]; q.d2s_r = ol[4 * OS];
      if (mag) {
        q.bt = hl[5 * HS]; q.bp = hl[6 * HS]; q.br = in_[k][6];
        q.dbt_r = ol[6 * OS]; q.dbp_r = ol[7 * OS];
      }
      double drho = in_[k][0], dw = in_[k][1], dvv = in_[k][2], du = in_[k][3], ds = in_[k][4];
      radial_point<mag>(g, ir, q, drho, dw, dvv, du, ds);
      // Density_Terms_Radial
      double w1 = O[5 * OS + (size_t)j * SR + l];
      if (phys) w1 = w1 + datum[l] * resp[j + 1];
      if (top_open || bot_open) {
        // Top_/Bottom_Inflow_Outflow: no dxdr, their own product orders
        // (rhs_mpi.f90:2032-2033, :1906-1907), then the face plane's
        // relaxation (:2042-2066, :1913-1952)
        drho = drho - q.u * w1;
        if (top_open) du = du - g.pconst * q.t * (1.0 / q.rho) * w1;
        else du = du - g.pconst * q.t * w1 * (1.0 / q.rho);
        inout_face(g, j, m, top_open, hl, SR, HS, base + l, drho, dw, dvv, du, ds);
      } else {
        if (g.non_uniform) w1 = w1 * g.dxdr[ir];
        drho = drho - q.u * w1;
        w1 = w1 * (1.0 / q.rho);
        du = du - g.pconst * q.t * w1;
      }
      if (g.rad_lnrho_r) {  // kept for the radiative pass (rhs_mpi.f90:1454, :1821)
        g.rad_lnrho_r[id] = w1;
        g.rad_dsdr[id] = g.non_uniform ? q.ds_r * g.dxdr[ir] : q.ds_r;
      }
      if (phys == 2 && j == m - 1 && !g.set_stop && !g.radheat) {  // rhs_mpi.f90:1807-1818
        drho = drho + q.rho * (g.t0 - q.t) / (g.damping_time * (g.gamma - 2.0) * q.t);
        ds = ds - g.cv * (g.t0 - q.t) / (g.damping_time * (g.gamma - 2.0) * q.t);
      }
      dv[id] = drho;
      dv[n + id] = dw;
      dv[2 * n + id] = dvv;
      dv[3 * n + id] = du;
      dv[4 * n + id] = ds;
    }
  }
}

// grid: x = r block * nchunk + theta chunk, y = phi; one tile per CTA
template <int MT, int TLC, typename TV, int KIND>
__global__ void __launch_bounds__(128, 4) k_radial_terms(CssGeo g, const TV *__restrict__ cur,
                                                      const double *__restrict__ bf, double *__restrict__ dv,
                                                      const double *__restrict__ tbuf, int TLrt) {
  extern __shared__ double sm[];
  const int TL = TLC ? TLC : TLrt;
  const int nchunk = (g.nth + TL - 1) / TL;
  const int br = blockIdx.x / nchunk;
  radial_tile<MT, TLC, TV, KIND>(g, cur, bf, dv, tbuf, TL, br, (blockIdx.x - br * nchunk) * TL, blockIdx.y, sm);
}

// ---------------------------------------------------------------------------
// Density_Terms_Theta (rhs_mpi.f90:1522-1605) fused with the RK4 stage
// combination of Step_RK4 (step_rk4.f90:385-475) and Bound (rhs_mpi.f90:
// 2395-2491).  stage 0 = no update (the RHS alone).  grid: x = theta block
// * nchunk + phi chunk, y = r.
//   stage 1: vs = (sld ? vs + dv/6 : dv); nx = v0 + dtcur*dv
//   stage 2,3: vs = vs + dv/3;            nx = v0 + dtcur*dv
//   stage 4: vs = vs + dv/6;              nx = v0 + dtcur*vs  (nx may be v0)
// and the TVD schemes (Step_RK2_TVD / Step_RK3_TVD, step_rk4.f90:31-335),
// where vs holds the step's SLD tendency:
//   stage 5: nx = ca*v0 + cb*cur + dtcur*dv
//   stage 6: nx = (ca*v0 + cb*cur + dtcur*dv) + dsld*vs  (nx may be v0)
// ---------------------------------------------------------------------------
template <int MT, int TLC, typename TS, typename TO, int STG = -1>
__global__ void __launch_bounds__(128) k_rhot_update(CssGeo g, const TS *__restrict__ cur,
                                                     double *__restrict__ dv, const double *v0, double *vs, TO *nx,
                                                     const double *__restrict__ tbuf, int stage_rt, double dtcur,
                                                     double ca, double cb, double dsld, int TLrt, int *flag) {
  // STG >= 0: the stage is known at compile time (the RK4 stages of an FP64
  // run), so the combination carries no per-point stage branches
  const int stage = STG >= 0 ? STG : stage_rt;
  extern __shared__ double sm[];
  const int TL = TLC ? TLC : TLrt;
  const int nchunk = (g.nphi + TL - 1) / TL;
  const int bt = blockIdx.x / nchunk, pb = (blockIdx.x - bt * nchunk) * TL;
  const int ir = blockIdx.y;
  const CssDir &D = g.d[1];
  const int t0 = D.start[bt], m = MT ? MT : D.size[bt];
  const int dtype = dtype_of(D, bt);
  const int SR = m + 9, SO = m + 1;
  const size_t n = (size_t)g.ncell;
  double *H = sm;
  double *O = H + (size_t)TL * SR;
  double *Tb = O + (size_t)TL * SO;
  // lines the stage combination reads at every point of the tile: dv, vars0
  // and the accumulator of every field, T and u_theta (128-byte steps along
  // the tile's theta segment of each line)
  {
    const int seg = (m * 8 + 127) / 128, nl = TL * seg;
    const size_t pl0 = plane(g, ir);
    for (int k = threadIdx.x; k < nl; k += blockDim.x) {
      const int l = k / seg, q = k - l * seg;
      if (pb + l >= g.nphi) continue;
      const size_t id = pl0 + (size_t)(pb + l) * g.nth + t0 + q * 16;
      prefetch_l2(tbuf + id);
      prefetch_l2(cur + n + id);
      for (int f = 0; f < g.nv; f++) {
        prefetch_l2(dv + f * n + id);
        if (stage > 0) prefetch_l2(v0 + f * n + id);
        if ((stage > 1 && stage <= 4) || (stage == 1 && g.sldiffusion) || (stage == 6 && dsld != 0.0))
          prefetch_l2(vs + f * n + id);
        if (stage >= 5 && cb != 0.0) prefetch_l2(cur + f * n + id);
      }
    }
  }
  if constexpr (MT > 0 && TLC > 0) {
    const TS *f1[1] = {cur};
    const double *m1[1] = {bg_rho(g)};
    tiles_ct<1, MT, TLC, 1>(g, f1, H, 0, SR, t0, pb, ir, m1);
  } else {
    tile_theta<MT, TLC>(g, cur, H, SR, t0, m, pb, TL, ir, bg_rho(g));
  }
  const int bdry = g.ibct[1];
  stage_table(g, 1, bt, 1, bdry, m, Tb);
  __syncthreads();
  const double rvv = g.r_ind[ir] * g.invpconst, ri = g.r_inv[ir];
  const size_t pl = plane(g, ir);
  for (int l = threadIdx.x; l < TL; l += blockDim.x) {
    if (pb + l >= g.nphi) continue;
    const double *x = H + (size_t)l * SR + 4;
    double lo = 0.0, hi = 0.0;
    if (D.lphys[bt]) {  // rhs_mpi.f90:1553-1555: make dw = 0 on the wall
      size_t id = pl + (size_t)(pb + l) * g.nth + t0;
      lo = rvv * dv[n + id] * x[0] / __ldg(tbuf + id);
    } else if (D.rphys[bt]) {
      size_t id = pl + (size_t)(pb + l) * g.nth + t0 + m - 1;
      hi = rvv * dv[n + id] * x[m - 1] / __ldg(tbuf + id);
    }
    solve<1, MT>(x, 1, m, dtype, bdry, lo, hi, Tb, m + 2, D.dnum[bt], D.dnum[bt], 0, O + (size_t)l * SO, 1);
  }
  __syncthreads();
  const int nv = g.nv;
  int bad = 0;
  // each thread's points: the density term with all points' loads issued
  // first, then the stage combination field by field, again loading every
  // point of a field before storing any (nx may be v0, so the compiler
  // could not reorder these itself)
  constexpr int PPT = (MT > 0 && TLC > 0) ? (MT * TLC + NT - 1) / NT : 1;
  const int stride = (MT > 0 && TLC > 0) ? NT : (int)blockDim.x;
  for (int pt0 = threadIdx.x; pt0 < TL * m; pt0 += PPT * stride) {
    size_t idk[PPT];
    bool okk[PPT];
    int itk[PPT];
    double d0k[PPT], d1k[PPT], wk[PPT], tk[PPT];
#pragma unroll
    for (int k = 0; k < PPT; k++) {
      const int pt = pt0 + k * stride;
      const int l = pt / m, j = pt - l * m;
      okk[k] = pt < TL * m && pb + l < g.nphi;
      itk[k] = t0 + j;
      idk[k] = pl + (size_t)(pb + l) * g.nth + t0 + j;
      if (okk[k]) {
        wk[k] = st_val(cur + n, idk[k], nullptr, 0);
        tk[k] = __ldg(tbuf + idk[k]);
        d0k[k] = dv[idk[k]];
        d1k[k] = dv[n + idk[k]];
      }
    }
#pragma unroll
    for (int k = 0; k < PPT; k++) {
      if (!okk[k]) continue;
      const int pt = pt0 + k * stride;
      const int l = pt / m, j = pt - l * m;
      const double rho = H[(size_t)l * SR + 4 + j];
      double w1 = ri * O[(size_t)l * SO + j];
      double d0 = d0k[k] - wk[k] * w1;
      w1 = w1 * (1.0 / rho);
      double d1 = d1k[k] - g.pconst * w1 * tk[k];
      if (ir == 0 && g.bottom_specified)  // prescribed bottom, u_theta (rhs_mpi.f90:1932)
        d1 = d1 + g.inout[IO_BOT_TAU] * (g.inout[IO_BOT_TCONST] * g.ashv[(size_t)g.nth * g.nphi + idk[k]] - wk[k]);
      if (g.xi_cs < 1.0) d0 = (g.xi_cs * g.xi_cs) * d0;
      d0k[k] = d0;
      d1k[k] = d1;
    }
    if (stage == 0) {
#pragma unroll
      for (int k = 0; k < PPT; k++)
        if (okk[k]) {
          dv[idk[k]] = d0k[k];
          dv[n + idk[k]] = d1k[k];
        }
      continue;
    }
    const bool rlo = (ir == 0), rhi = (ir == g.nr - 1);
    for (int iv = 0; iv < nv; iv++) {
      double dd[PPT], aa[PPT], ss[PPT], cc[PPT];
      const bool need_s = stage <= 4 ? !(stage == 1 && !g.sldiffusion) : (stage == 6 && dsld != 0.0);
      const bool need_c = stage >= 5 && cb != 0.0;
      const double *bg = iv == 0 ? bg_rho(g) : (iv == 4 ? bg_s(g) : nullptr);  // background of an FP32 stage state
#pragma unroll
      for (int k = 0; k < PPT; k++) {
        if (!okk[k]) continue;
        const size_t q = (size_t)iv * n + idk[k];
        dd[k] = (iv == 0) ? d0k[k] : (iv == 1) ? d1k[k] : dv[q];
        aa[k] = v0[q];
        ss[k] = need_s ? vs[q] : 0.0;
        cc[k] = need_c ? st_val(cur + (size_t)iv * n, idk[k], bg, bgi(g, ir, itk[k])) : 0.0;
      }
#pragma unroll
      for (int k = 0; k < PPT; k++) {
        if (!okk[k]) continue;
        const size_t q = (size_t)iv * n + idk[k];
        const double d = dd[k], a = aa[k];
        double o;
        if (stage == 1) {
          double sv = g.sldiffusion ? ss[k] + d / 6.0 : d;
          vs[q] = sv;
          o = a + dtcur * d;
        } else if (stage == 4) {
          double sv = ss[k] + d / 6.0;
          o = a + dtcur * sv;
        } else if (stage <= 3) {
          double sv = ss[k] + d / 3.0;
          vs[q] = sv;
          o = a + dtcur * d;
        } else {
          o = ca * a + cb * cc[k] + dtcur * d;
          if (stage == 6 && dsld != 0.0) o = o + dsld * ss[k];
        }
        const bool twall = (itk[k] == 0 || itk[k] == g.nth - 1);
        // Bound (rhs_mpi.f90:2395-2491)
        if (twall || rlo || rhi) {
          if (iv == 1 && twall) o = 0.0;
          if (iv == 3 && !g.theta_stress_free && twall) o = 0.0;
          if (rlo) {
            if ((iv == 1 || iv == 2) && !g.bottom_stress_free) o = 0.0;
            if (iv == 3 && !g.bot_inout) o = 0.0;
          }
          if (rhi && !g.top_inout) {  // an open top keeps every field (rhs_mpi.f90:2420-2432)
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
        double bgv = 0.0;
        if constexpr (sizeof(TO) == 4) {
          if (iv == 0) bgv = bg_rho(g)[bgi(g, ir, itk[k])];
          else if (iv == 4) bgv = bg_s(g)[bgi(g, ir, itk[k])];
        }
        nx[q] = st_store<TO>(o, bgv);
      }
    }
  }
  if (bad && flag) atomicOr(flag, 1);
}

// ---------------------------------------------------------------------------
// Bound (rhs_mpi.f90:2395-2491) on a whole state, for callers that change
// the state themselves (the step kernels apply the same rules inside the
// stage update).  One thread per (theta, phi) column of the two radial faces
// and per (phi, r) line of the two theta walls; every rule only sets zeros.
// ---------------------------------------------------------------------------
__global__ void k_bound(CssGeo g, double *v) {
  const size_t n = (size_t)g.ncell, np = (size_t)g.nth * g.nphi;
  const size_t nwall = (size_t)g.nphi * g.nr;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < np + nwall; k += (size_t)gridDim.x * blockDim.x) {
    if (k < np) {  // radial faces at this (theta, phi)
      const size_t lo = k, hi = (size_t)(g.nr - 1) * np + k;
      if (!g.bottom_stress_free) { v[n + lo] = 0.0; v[2 * n + lo] = 0.0; }
      if (!g.bot_inout) v[3 * n + lo] = 0.0;
      if (!g.top_inout) {
        if (!g.top_stress_free) { v[n + hi] = 0.0; v[2 * n + hi] = 0.0; }
        v[3 * n + hi] = 0.0;
      }
      if (g.magnetic) {
        if (!g.bot_inout) {
          if (g.bottom_radial_field) v[7 * n + lo] = 0.0;
          else if (g.bottom_perfect_cond) { v[5 * n + lo] = 0.0; v[6 * n + lo] = 0.0; }
        }
        if (!g.top_inout) {
          if (g.top_radial_field) v[7 * n + hi] = 0.0;
          else if (g.top_perfect_cond) { v[5 * n + hi] = 0.0; v[6 * n + hi] = 0.0; }
        }
      }
    } else {  // theta walls of this (phi, r) line
      const size_t q = k - np, ip = q % g.nphi, ir = q / g.nphi;
      const size_t a = css_idx(g, 0, (int)ip, (int)ir), b = css_idx(g, g.nth - 1, (int)ip, (int)ir);
      v[n + a] = 0.0;
      v[n + b] = 0.0;
      if (!g.theta_stress_free) { v[3 * n + a] = 0.0; v[3 * n + b] = 0.0; }
      if (g.magnetic) {
        if (g.theta_perf_conductor) {
          v[6 * n + a] = 0.0; v[7 * n + a] = 0.0; v[6 * n + b] = 0.0; v[7 * n + b] = 0.0;
        } else {
          v[5 * n + a] = 0.0; v[5 * n + b] = 0.0;
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// VectorCurlA (derivatives.f90:2106-2294): out = curl(a), fields ordered
// (theta, phi, r).  Three kernels, one per sweep direction; the r sweep
// optionally applies Compute_B's boundary zeroing (:1842-1883).
// ---------------------------------------------------------------------------
template <int MT, int TLC, typename TS>
__global__ void __launch_bounds__(128) k_curl_theta(CssGeo g, const TS *__restrict__ a, double *__restrict__ out,
                                                    int TL) {
  extern __shared__ double sm[];
  const int nchunk = (g.nphi + TL - 1) / TL;
  const int bt = blockIdx.x / nchunk, pb = (blockIdx.x - bt * nchunk) * TL;
  const int ir = blockIdx.y;
  const CssDir &D = g.d[1];
  const int t0 = D.start[bt], m = MT ? MT : D.size[bt];
  const int dtype = dtype_of(D, bt);
  const int SR = m + 9, SO = m + 1;
  const size_t n = (size_t)g.ncell;
  double *H = sm;                      // 0: sin*A_phi, 1: A_r
  double *O = H + (size_t)2 * TL * SR;
  if constexpr (MT > 0 && TLC > 0) {
    const TS *fs[2] = {a + n, a + 2 * n};
    tiles_ct<2, MT, TLC, 1>(g, fs, H, (size_t)TL * SR, SR, t0, pb, ir);
  } else {
    load_theta_tile(g, a + n, H, SR, t0, m, pb, TL, ir, true);
    load_theta_tile(g, a + 2 * n, H + (size_t)TL * SR, SR, t0, m, pb, TL, ir, true);
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < TL * (m + 8); idx += blockDim.x) {
    int l = idx / (m + 8), jj = idx - l * (m + 8);
    int gt = t0 + jj - 4;
    if (gt < 0 || gt >= g.nth) continue;
    H[(size_t)l * SR + jj] *= g.sines[gt];
  }
  __syncthreads();
  for (int task = threadIdx.x; task < 2 * TL; task += blockDim.x) {
    int k = task / TL, l = task - k * TL;
    if (pb + l >= g.nphi) continue;
    int bdry = g.ibct[k == 0 ? 11 : 12];
    solve<1, MT>(H + ((size_t)k * TL + l) * SR + 4, 1, m, dtype, bdry, 0.0, 0.0, tabp(g, 1, bt, 1, bdry), g.tstride,
                  D.dnum[bt], D.dnum[bt], 0, O + ((size_t)k * TL + l) * SO, 1);
  }
  __syncthreads();
  const double invr = g.r_inv[ir];
  for (int pt = threadIdx.x; pt < TL * m; pt += blockDim.x) {
    int l = pt / m, j = pt - l * m;
    int it = t0 + j, ip = pb + l;
    if (ip >= g.nphi) continue;
    size_t id = css_idx(g, it, ip, ir);
    out[2 * n + id] = O[(size_t)l * SO + j] * g.csc[it] * invr;
    out[n + id] = -O[(size_t)(TL + l) * SO + j] * invr;
  }
}

template <int MT, int TLC, typename TS>
__global__ void __launch_bounds__(128) k_curl_phi(CssGeo g, const TS *__restrict__ a, double *__restrict__ out,
                                                  int TL) {
  extern __shared__ double sm[];
  const int nchunk = (g.nth + TL - 1) / TL;
  const int bp = blockIdx.x / nchunk, tb = (blockIdx.x - bp * nchunk) * TL;
  const int ir = blockIdx.y;
  const CssDir &D = g.d[2];
  const int p0 = D.start[bp], m = MT ? MT : D.size[bp];
  const int SR = TL + 1;
  const size_t n = (size_t)g.ncell;
  const size_t HS = (size_t)(m + 8) * SR, OS = (size_t)m * SR;
  double *H = sm;  // 0: A_r, 1: A_theta
  double *O = H + 2 * HS;
  if constexpr (MT > 0 && TLC > 0) {
    const TS *fs[2] = {a + 2 * n, a};
    tiles_ct<2, MT, TLC, 2>(g, fs, H, HS, SR, p0, tb, ir);
  } else {
    load_phi_tile(g, a + 2 * n, H, SR, p0, m, tb, TL, ir, true);
    load_phi_tile(g, a, H + HS, SR, p0, m, tb, TL, ir, true);
  }
  __syncthreads();
  for (int task = threadIdx.x; task < 2 * TL; task += blockDim.x) {
    int k = task / TL, l = task - k * TL;
    if (tb + l >= g.nth) continue;
    solve<1, MT>(H + k * HS + 4 * SR + l, SR, m, 3, 0, 0.0, 0.0, tabp(g, 2, bp, 1, 0), g.tstride, D.dnum[bp],
                  D.dnum[bp], 1, O + k * OS + l, SR);
  }
  __syncthreads();
  const double invr = g.r_inv[ir];
  // all of a thread's read-modify-write loads before its stores
  constexpr int PPT = (MT > 0 && TLC > 0) ? (MT * TLC + NT - 1) / NT : 1;
  const int stride = (MT > 0 && TLC > 0) ? NT : (int)blockDim.x;
  for (int pt0 = threadIdx.x; pt0 < TL * m; pt0 += PPT * stride) {
    double prev[PPT];
#pragma unroll
    for (int k = 0; k < PPT; k++) {
      const int pt = pt0 + k * stride, j = pt / TL, l = pt - j * TL;
      if (pt < TL * m && tb + l < g.nth) prev[k] = out[2 * n + css_idx(g, tb + l, p0 + j, ir)];
    }
#pragma unroll
    for (int k = 0; k < PPT; k++) {
      const int pt = pt0 + k * stride, j = pt / TL, l = pt - j * TL;
      const int it = tb + l, ip = p0 + j;
      if (pt >= TL * m || it >= g.nth) continue;
      const size_t id = css_idx(g, it, ip, ir);
      const double csc = g.csc[it];
      out[id] = invr * O[(size_t)j * SR + l] * csc;
      out[2 * n + id] = prev[k] - invr * O[OS + (size_t)j * SR + l] * csc;
    }
  }
}

// The theta and phi parts of B = curl A in one pass over a theta block x phi
// block tile of one radius (both directions MT points per block): the
// theta lines of sin(theta) A_phi and A_r, the phi lines of A_r and A_theta
// (VectorCurlA, derivatives.f90:1769-1828, as k_curl_theta and k_curl_phi
// split it), with B_r complete and the theta / phi parts of B_theta / B_phi
// written once -- the same expressions in the same order as the two kernels
// (bit for bit), without the phi kernel's read-modify-write of B_r.
// grid: x = theta block + phi block * (theta blocks), y = r; 256 threads
// (the loads of a tile spread over 8 warps; 2 CTAs per SM, no register
// cap below what the unrolled 32-point solves hold: 2.53 ms on MHD
// 256x512x1024 against 2.64 with 3 CTAs of 80 registers, which spill, and
// 3.09 with 128 threads).
template <int MT, typename TS>
__global__ void __launch_bounds__(256, 2) k_curl_tp(CssGeo g, const TS *__restrict__ a, double *__restrict__ out) {
  extern __shared__ double sm[];
  constexpr int W = MT + 8, SRT = MT + 9, SOT = MT + 1, SRP = MT + 1;
  constexpr size_t FT = (size_t)MT * SRT, HSP = (size_t)W * SRP, OT = (size_t)MT * SOT, OP = (size_t)MT * SRP;
  const int bt = blockIdx.x % g.d[1].nb, bp = blockIdx.x / g.d[1].nb, ir = blockIdx.y;
  const CssDir &DT = g.d[1], &DP = g.d[2];
  const int t0 = DT.start[bt], p0 = DP.start[bp];
  const size_t n = (size_t)g.ncell;
  double *Ht = sm;               // theta lines: 0 sin*A_phi, 1 A_r   [phi line][theta + halo]
  double *Hp = Ht + 2 * FT;      // phi lines: 0 A_r, 1 A_theta      [phi + halo][theta line]
  double *Ot = Hp + 2 * HSP;     // d/dtheta of the theta lines      [phi line][theta]
  double *Op = Ot + 2 * OT;      // d/dphi of the phi lines          [phi][theta line]
  {
    const TS *ft[2] = {a + n, a + 2 * n};
    tiles_ct<2, MT, MT, 1, TS, 256>(g, ft, Ht, FT, SRT, t0, p0, ir);
    const TS *fp[2] = {a + 2 * n, a};
    tiles_ct<2, MT, MT, 2, TS, 256>(g, fp, Hp, HSP, SRP, p0, t0, ir);
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < MT * W; idx += blockDim.x) {
    const int l = idx / W, jj = idx - l * W, gt = t0 + jj - 4;
    if (gt < 0 || gt >= g.nth) continue;
    Ht[(size_t)l * SRT + jj] *= g.sines[gt];
  }
  __syncthreads();
  const int dtype = dtype_of(DT, bt);
  for (int task = threadIdx.x; task < 4 * MT; task += blockDim.x) {
    const int k = task / MT, l = task - k * MT;
    if (k < 2) {
      const int bdry = g.ibct[k == 0 ? 11 : 12];
      solve<1, MT>(Ht + ((size_t)k * MT + l) * SRT + 4, 1, MT, dtype, bdry, 0.0, 0.0, tabp(g, 1, bt, 1, bdry),
                   g.tstride, DT.dnum[bt], DT.dnum[bt], 0, Ot + ((size_t)k * MT + l) * SOT, 1);
    } else {
      const int q = k - 2;
      solve<1, MT>(Hp + q * HSP + 4 * SRP + l, SRP, MT, 3, 0, 0.0, 0.0, tabp(g, 2, bp, 1, 0), g.tstride,
                   DP.dnum[bp], DP.dnum[bp], 1, Op + q * OP + l, SRP);
    }
  }
  __syncthreads();
  const double invr = g.r_inv[ir];
  for (int pt = threadIdx.x; pt < MT * MT; pt += blockDim.x) {
    const int jp = pt / MT, jt = pt - jp * MT;  // theta fastest: coalesced stores
    const int it = t0 + jt;
    const size_t id = css_idx(g, it, p0 + jp, ir);
    const double csc = g.csc[it];
    out[id] = invr * Op[(size_t)jp * SRP + jt] * csc;
    out[n + id] = -Ot[(size_t)(MT + jp) * SOT + jt] * invr;
    // the theta part rounded on its own, as the two-pass form stores it before the phi pass subtracts
    const double prev = __dmul_rn(__dmul_rn(Ot[(size_t)jp * SOT + jt], csc), invr);
    out[2 * n + id] = prev - invr * Op[OP + (size_t)jp * SRP + jt] * csc;
  }
}

template <int MT, int TLC, typename TS>
__global__ void __launch_bounds__(128) k_curl_r(CssGeo g, const TS *__restrict__ a, double *__restrict__ out,
                                                int TL, int apply_bc) {
  extern __shared__ double sm[];
  const int nchunk = (g.nth + TL - 1) / TL;
  const int br = blockIdx.x / nchunk, tb = (blockIdx.x - br * nchunk) * TL;
  const int ip = blockIdx.y;
  const CssDir &D = g.d[0];
  const int r0 = D.start[br], m = MT ? MT : D.size[br];
  const int dtype = dtype_of(D, br);
  const int SR = TL + 1;
  const size_t n = (size_t)g.ncell;
  const size_t HS = (size_t)(m + 8) * SR, OS = (size_t)m * SR;
  double *H = sm;  // 0: r*A_theta, 1: r*A_phi
  double *O = H + 2 * HS;
  if constexpr (MT > 0 && TLC > 0) {
    const TS *fs[2] = {a, a + n};
    tiles_ct<2, MT, TLC, 0>(g, fs, H, HS, SR, r0, tb, ip);
  } else {
    load_r_tile(g, a, H, SR, r0, m, tb, TL, ip, true);
    load_r_tile(g, a + n, H + HS, SR, r0, m, tb, TL, ip, true);
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < TL * (m + 8); idx += blockDim.x) {
    int jj = idx / TL, l = idx - jj * TL;
    int gr = r0 + jj - 4;
    if (gr < 0 || gr >= g.nr) continue;
    H[(size_t)jj * SR + l] *= g.r_ind[gr];
    H[HS + (size_t)jj * SR + l] *= g.r_ind[gr];
  }
  __syncthreads();
  for (int task = threadIdx.x; task < 2 * TL; task += blockDim.x) {
    int k = task / TL, l = task - k * TL;
    if (tb + l >= g.nth) continue;
    int bdry = g.ibcr[k == 0 ? 10 : 11];
    solve<1, MT>(H + k * HS + 4 * SR + l, SR, m, dtype, bdry, 0.0, 0.0, tabp(g, 0, br, 1, bdry), g.tstride,
                  D.dnum[br], D.dnum[br], 0, O + k * OS + l, SR);
  }
  __syncthreads();
  constexpr int PPT = (MT > 0 && TLC > 0) ? (MT * TLC + NT - 1) / NT : 1;
  const int stride = (MT > 0 && TLC > 0) ? NT : (int)blockDim.x;
  for (int pt0 = threadIdx.x; pt0 < TL * m; pt0 += PPT * stride) {
  double in_t[PPT], in_p[PPT], in_r[PPT];
#pragma unroll
  for (int k = 0; k < PPT; k++) {
    const int pt = pt0 + k * stride, j = pt / TL, l = pt - j * TL;
    if (pt < TL * m && tb + l < g.nth) {
      const size_t id = css_idx(g, tb + l, ip, r0 + j);
      in_t[k] = out[id];
      in_p[k] = out[n + id];
      in_r[k] = out[2 * n + id];
    }
  }
#pragma unroll
  for (int k = 0; k < PPT; k++) {
    const int pt = pt0 + k * stride;
    int j = pt / TL, l = pt - j * TL;
    int it = tb + l, ir = r0 + j;
    if (pt >= TL * m || it >= g.nth) continue;
    size_t id = css_idx(g, it, ip, ir);
    double d = O[(size_t)j * SR + l];
    if (g.non_uniform) d = d * g.dxdr[ir];
    double bp_ = in_p[k] + d * g.r_inv[ir];
    d = O[OS + (size_t)j * SR + l];
    if (g.non_uniform) d = d * g.dxdr[ir];
    double bt_ = in_t[k] - d * g.r_inv[ir];
    double br_ = in_r[k];
    if (apply_bc) {
      if (it == 0 || it == g.nth - 1) {
        if (g.theta_perf_conductor) bt_ = 0.0;
        else { bp_ = 0.0; br_ = 0.0; }
      }
      if (ir == 0) {
        if (g.bottom_radial_field) { bt_ = 0.0; bp_ = 0.0; }
        else if (g.bottom_perfect_cond) br_ = 0.0;
      }
      if (ir == g.nr - 1) {
        if (g.top_radial_field) { bt_ = 0.0; bp_ = 0.0; }
        else if (g.top_perfect_cond) br_ = 0.0;
      }
      out[2 * n + id] = br_;
    }
    out[id] = bt_;
    out[n + id] = bp_;
  }
  }
}

// ---------------------------------------------------------------------------
// Slope-limited diffusion (diffusion.f90:70-474).  The block faces between
// ranks only carry neighbour data here (halos and the ghost ring of vcc are
// the neighbour's own values), so only the physical faces need the per-
// variable ghost rules of Diffusion_R / Diffusion_Th.
// ---------------------------------------------------------------------------
// vcc = speed^2(r) + |u|^2 [+ vA^2] (diffusion.f90:177-286), dstype = 1
__global__ void k_sld_vcc(CssGeo g, const double *__restrict__ v, const double *__restrict__ bf,
                          double *__restrict__ vcc) {
  size_t n = (size_t)g.ncell;
  for (size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x; id < n; id += (size_t)gridDim.x * blockDim.x) {
    int ir = (int)(id / ((size_t)g.nth * g.nphi));
    double c = g.dspeed[ir];
    if (g.speed2) {
      const double s2 = g.speed2[id];
      if (s2 >= 0.0) c = s2;
    }
    if (g.dstype == 1) {
      for (int iv = 1; iv <= 3; iv++) {
        double q = __ldg(v + iv * n + id);
        c = c + q * q;
      }
      if (g.magnetic) {
        double ir_ = 1.0 / __ldg(v + id);
        for (int k = 0; k < 3; k++) {
          double q = __ldg(bf + k * n + id);
          c = c + ONE_OVER_4PI * ir_ * (q * q);
        }
      }
    }
    vcc[id] = c;
  }
}

// q * max(0, min(1, q*qph / max(|q|,tiny)^2)).  For |q| >= tiny the ratio is
// qph/q, so the limited value is 0 (opposite signs), q (|qph| >= |q|) or qph:
// a minmod, evaluated without the division (equal to the reference's
// product to within its roundings); below tiny the formula as written.
__device__ __forceinline__ double sld_limiter(double q, double qph, double tiny, double inv_tiny) {
  const double a = fabs(q);
  if (a >= tiny) {
    if (!(q * qph > 0.0)) return q * 0.0;
    return fabs(qph) >= a ? q : qph;
  }
  double rtmp = inv_tiny;  // 1/tiny, the same correctly rounded quotient
  rtmp = q * (rtmp * rtmp);
  rtmp = rtmp * qph;
  rtmp = fmin(1.0, rtmp);
  return q * fmax(0.0, rtmp);
}

// limited face difference delta at the face whose neighbours are
// x(-2..+1) around it: qmh = x_{-1}-x_{-2}, qph = x_0-x_{-1}, qp3h = x_1-x_0
__device__ __forceinline__ double sld_face(double xm2, double xm1, double x0, double x1, double tiny,
                                         double inv_tiny) {
  double qmh = xm1 - xm2, qph = x0 - xm1, qp3h = x1 - x0;
  double pl = sld_limiter(qmh, qph, tiny, inv_tiny), pr = sld_limiter(qp3h, qph, tiny, inv_tiny);
  return qph - 0.5 * (pr + pl);
}

// value of field iv (0-based) the SLD sees: rho - rhor, s - sr, A for iv>=5
__device__ __forceinline__ double sld_val(const CssGeo &g, const double *__restrict__ v, const double *__restrict__ av,
                                          int iv, int it, int ip, int ir) {
  size_t id = css_idx(g, it, ip, ir);
  size_t n = (size_t)g.ncell;
  if (iv >= 5) return __ldg(av + (iv - 5) * n + id);
  double q = __ldg(v + iv * n + id);
  if (iv == 0) q = q - g.rhor[ir];
  if (iv == 4) q = q - g.sr[ir];
  return q;
}

// ghost value just outside a physical radial face (diffusion.f90:582-728):
// lo = 1 for the bottom (x(-1) from x(0..3)), 0 for the top (x(nr) from
// x(nr-1..nr-4)); iv1 is the reference's 1-based variable index
__device__ double sld_ghost_r(const CssGeo &g, const double *__restrict__ v, const double *__restrict__ av, int iv,
                              int it, int ip, int lo) {
  const double *r = g.r_ind, *dr = g.dr_ind;
  int iv1 = iv + 1, nr = g.nr;
  if (lo) {
    double t1 = sld_val(g, v, av, iv, it, ip, 0);
    switch (iv1) {
      case 1: return 0.0;
      case 2: case 3:
        return -10.0 * (1.0 / 3.0) * t1 / r[0] + 6.0 * sld_val(g, v, av, iv, it, ip, 1) / r[1] -
               2.0 * sld_val(g, v, av, iv, it, ip, 2) / r[2] + (1.0 / 3.0) * sld_val(g, v, av, iv, it, ip, 3) / r[3];
      case 5:
        if (!g.bottom_constant_temp && g.slaplacian)
          return t1 + dr[0] * (g.lumr1 * ONE_OVER_4PI / (g.r1 * g.r1 * g.ks[0] * g.dxdr[0]));
        return 0.0;
      case 6: case 7: return g.bottom_perfect_cond ? 0.0 : t1;
      default: return t1;
    }
  }
  int m = nr - 1;
  double tm = sld_val(g, v, av, iv, it, ip, m);
  switch (iv1) {
    case 1: return 0.0;
    case 2: case 3:
      return -10.0 * (1.0 / 3.0) * tm / r[m] + 6.0 * sld_val(g, v, av, iv, it, ip, m - 1) / r[m - 1] -
             2.0 * sld_val(g, v, av, iv, it, ip, m - 2) / r[m - 2] +
             (1.0 / 3.0) * sld_val(g, v, av, iv, it, ip, m - 3) / r[m - 3];
    case 5:
      if (!g.top_constant_temp && g.slaplacian)
        return tm - dr[0] * (g.lumr2 * ONE_OVER_4PI / (g.r2 * g.r2 * g.ks[nr - 1] * g.dxdr[nr - 1]));
      return 0.0;
    case 6: case 7: return g.top_perfect_cond ? 0.0 : tm;
    default: return tm;
  }
}

// ghost just outside a physical theta face (diffusion.f90:1008-1118), from
// the four tile values nearest the wall (q0 at the wall)
__device__ __forceinline__ double sld_ghost_t(const CssGeo &g, int iv, double q0, double q1, double q2, double q3,
                                              int lo) {
  const double *sn = g.sines;
  int iv1 = iv + 1, m = g.nth - 1;
  switch (iv1) {
    case 2: return 0.0;
    case 3:
      if (lo)
        return -10.0 * (1.0 / 3.0) * q0 / sn[0] + 6.0 * q1 / sn[1] - 2.0 * q2 / sn[2] + (1.0 / 3.0) * q3 / sn[3];
      return -10.0 * (1.0 / 3.0) * q0 / sn[m] + 6.0 * q1 / sn[m - 1] - 2.0 * q2 / sn[m - 2] + (1.0 / 3.0) * q3 / sn[m - 3];
    case 6: return g.theta_normal_field ? 0.0 : q0;
    case 7: case 8: return g.theta_perf_conductor ? 0.0 : q0;
    default: return q0;
  }
}

// Slope-limited diffusion, all three directions and all nsld fields in one
// pass.  CTA = a 32 (theta) x 8 (phi) plane tile marching over an r chunk of
// SLD_RC radii.  Per radius: the plane values of every field (2-point halo)
// and the speed plane (1-point halo) go to shared memory, every theta and
// phi face flux is computed once, the r faces come from a 4-point window
// per field carried in registers (one new global load per field and
// radius), then viscous heating and the mass-diffusion corrections
// (diffusion.f90:375-428) per cell.  NF = number of diffused fields.
//
// The theta and phi faces difference the values of one radius, where the
// subtracted mean state (diffusion.f90:125-175) is a constant: (x_a - m) -
// (x_b - m) equals x_a - x_b bit for bit whenever x lies within a factor 2
// of m (the two inner subtractions are then exact), so the plane values are
// differenced raw.  The r faces difference across radii and subtract the
// mean of each radius (sld_val).
#define SLD_TT 32
#define SLD_TP 8
#define SLD_RC 32
#define SLD_XW (SLD_TT + 4)  // plane row: 36 doubles = 288 B, so 16-byte copies stay aligned
#define SLD_VW (SLD_TT + 3)
template <int NF>
struct SldSmem {
  double X[2][NF][SLD_TP + 4][SLD_XW];    // field planes (halo 2) of radii ir and ir+1
  double V[2][SLD_TP + 2][SLD_VW];        // vcc planes (halo 1)
  double FT[NF][SLD_TP][SLD_TT + 1];      // theta face fluxes
  double FP[NF][SLD_TP + 1][SLD_TT];      // phi face fluxes
};

// This thread's share of one radius's plane copies, fixed for the CTA: one
// 16-byte theta pair of every field (the tile's first theta is even, and
// so is nth on this path; zero fill outside 0 <= theta < nth, periodic phi)
// and up to two speed values (theta clamped).  Offsets are within a plane.
struct SldCopy {
  int xs, xg, xn;       // smem offset in a field plane, global offset, bytes (16 or 0); xs < 0: none
  int vs0, vg0, vs1, vg1;  // speed plane: smem / global offsets; vs < 0: none
};

__device__ __forceinline__ SldCopy sld_copy_plan(const CssGeo &g, int t0, int p0) {
  constexpr int PAIRS = SLD_XW / 2, NXP = (SLD_TP + 4) * PAIRS, NVV = (SLD_TP + 2) * (SLD_TT + 2);
  const int nth = g.nth, nphi = g.nphi, k = threadIdx.x;
  SldCopy c;
  c.xs = -1; c.xg = 0; c.xn = 0;
  if (k < NXP) {
    const int bb = k / PAIRS, a2 = k - bb * PAIRS;
    const int gt = t0 - 2 + 2 * a2;
    int gp = p0 + bb - 2;
    gp = gp < 0 ? gp + nphi : (gp >= nphi ? gp - nphi : gp);
    const bool in = gt >= 0 && gt < nth;
    c.xs = bb * SLD_XW + 2 * a2;
    c.xg = in ? gp * nth + gt : 0;
    c.xn = in ? 16 : 0;
  }
  auto vslot = [&](int kk, int &vs, int &vg) {
    vs = -1; vg = 0;
    if (kk < NVV) {
      const int a = kk % (SLD_TT + 2), bb = kk / (SLD_TT + 2);
      const int gt = min(max(t0 + a - 1, 0), nth - 1);
      int gp = p0 + bb - 1;
      gp = gp < 0 ? gp + nphi : (gp >= nphi ? gp - nphi : gp);
      vs = bb * SLD_VW + a;
      vg = gp * nth + gt;
    }
  };
  vslot(k, c.vs0, c.vg0);
  vslot(k + SLD_TT * SLD_TP, c.vs1, c.vg1);
  return c;
}

// starts the copies of radius ir's planes into buffer `buf`
template <int NF>
__device__ __forceinline__ void sld_issue_plane(const CssGeo &g, const double *__restrict__ v,
                                                const double *__restrict__ av, const double *__restrict__ vcc,
                                                SldSmem<NF> &S, const SldCopy &c, int buf, int ir, int off) {
  const size_t n = (size_t)g.ncell, pl = plane(g, ir);
  if (c.xs >= 0) {
#pragma unroll
    for (int f = 0; f < NF; f++) {
      const int iv = f + off;
      const double *fp = (iv >= 5 ? av + (size_t)(iv - 5) * n : v + (size_t)iv * n) + pl;
      cp_async16(&S.X[buf][f][0][0] + c.xs, fp + c.xg, c.xn);
    }
  }
  const double *vp = vcc + pl;
  if (c.vs0 >= 0) cp_async8(&S.V[buf][0][0] + c.vs0, vp + c.vg0, 8);
  if (c.vs1 >= 0) cp_async8(&S.V[buf][0][0] + c.vs1, vp + c.vg1, 8);
  cp_async_commit();
}

template <int NF, int OFF>
__global__ void __launch_bounds__(SLD_TT * SLD_TP, 2) k_sld(CssGeo g, const double *__restrict__ v,
                                                            const double *__restrict__ av,
                                                            const double *__restrict__ vcc,
                                                            double *__restrict__ dout, unsigned wmask,
                                                            const double *__restrict__ tb) {
  constexpr int off = OFF;  // first diffused field: every field index below is a constant
  extern __shared__ double sm_raw[];
  SldSmem<NF> &S = *reinterpret_cast<SldSmem<NF> *>(sm_raw);
  auto &FT = S.FT;
  auto &FP = S.FP;
  const size_t n = (size_t)g.ncell;
  const int nth = g.nth, nphi = g.nphi, nr = g.nr;
  const int tx = threadIdx.x % SLD_TT, ty = threadIdx.x / SLD_TT;
  const int t0 = blockIdx.x * SLD_TT, p0 = blockIdx.y * SLD_TP;
  const int r0 = blockIdx.z * SLD_RC, r1 = min(r0 + SLD_RC, nr);
  const int it = t0 + tx, ip = p0 + ty;
  const bool live = it < nth && ip < nphi;
  const int itc = min(it, nth - 1), ipc = min(ip, nphi - 1);
  // this launch diffuses fields off .. off+NF-1 and writes the fields of
  // wmask (a field it writes but does not diffuse gets zero)
  const bool hydro_part = (wmask & 0x1Fu) != 0;  // the fields the corrections act on
  const bool edge_lo = t0 == 0, edge_hi = t0 + SLD_TT >= nth;
  // theta faces of this thread: the upper face of its cell, and for warp 1
  // the lower face of row tx (lane < SLD_TP); their sin(face) factors
  const int gt_hi = t0 + tx + 1;
  const bool th_hi_in = gt_hi > 0 && gt_hi < nth;
  const bool lo_t = ty == 1 && tx < SLD_TP, lo_p = ty == 0;
  const bool th_lo_in = t0 > 0 && t0 < nth;
  const SldCopy cp = sld_copy_plan(g, t0, p0);
  // per-field r window: x(ir-1), x(ir), x(ir+1), x(ir+2), and the de of the
  // lower r face of the current radius
  double win[NF][4], carry[NF];
#pragma unroll
  for (int f = 0; f < NF; f++) {
    const int iv = f + off;
    auto xr = [&](int q) -> double {  // x at radius q of this column (ghosts outside)
      if (q >= 0 && q < nr) return sld_val(g, v, av, iv, itc, ipc, q);
      if (q == -1) return sld_ghost_r(g, v, av, iv, itc, ipc, 1);
      if (q == nr) return sld_ghost_r(g, v, av, iv, itc, ipc, 0);
      return 0.0;
    };
    win[f][0] = xr(r0 - 1);
    win[f][1] = xr(r0);
    win[f][2] = xr(r0 + 1);
    win[f][3] = xr(r0 + 2);
    carry[f] = 0.0;
    if (r0 > 0) {
      const double vc = __ldg(vcc + css_idx(g, itc, ipc, r0)), vcm = __ldg(vcc + css_idx(g, itc, ipc, r0 - 1));
      carry[f] = (g.sld_coef * sqrt(0.5 * (vc + vcm))) *
                 (sld_face(xr(r0 - 2), win[f][0], win[f][1], win[f][2], g.tinyvar[iv], g.inv_tinyvar[iv]) * g.sld_r[2 * nr + r0]);
    }
  }
  sld_issue_plane<NF>(g, v, av, vcc, S, cp, 0, r0, off);
  // the speed of this column at radii ir and ir+1, one radius ahead
  double vc_a = __ldg(vcc + css_idx(g, itc, ipc, r0));
  double vc_b = r0 < nr - 1 ? __ldg(vcc + css_idx(g, itc, ipc, r0 + 1)) : vc_a;
  for (int ir = r0; ir < r1; ir++) {
    const int cb = (ir - r0) & 1;
    auto &X = S.X[cb];
    auto &V = S.V[cb];
    const double t3 = g.sld_r[ir], rfac = g.sld_r[nr + ir], rhi2 = g.sld_r[3 * nr + ir];
    const double cphl = g.sld_th[nth + itc], cphh = g.sld_th[3 * nth + itc];
    const double geom = g.sld_th[4 * nth + itc] * (rfac / g.dphi);
    const double vr_hi = g.sld_coef * sqrt(0.5 * (vc_b + vc_a));
    const double vc_n = ir + 1 < nr - 1 ? __ldg(vcc + css_idx(g, itc, ipc, ir + 2)) : vc_b;
    // this cell's rho and T for the corrections, issued early
    const size_t idc = css_idx(g, itc, ipc, ir);
    double rho_c = 1.0, t_c = 1.0;
    if (hydro_part) {
      rho_c = __ldg(v + idc);
      t_c = tb ? __ldg(tb + idc) : __ldg(v + 4 * n + idc);
    }
    // next window value x(ir+3), issued early
    double nxt[NF];
#pragma unroll
    for (int f = 0; f < NF; f++) {
      const int q = ir + 3;
      nxt[f] = (q < nr) ? sld_val(g, v, av, f + off, itc, ipc, q) : 0.0;
    }
    // radius ir+1 streams into the other buffer while this radius is computed
    // (that buffer's last readers finished before the previous radius's
    // last barrier)
    if (ir + 1 < r1) {
      sld_issue_plane<NF>(g, v, av, vcc, S, cp, cb ^ 1, ir + 1, off);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    // theta ghosts next to the walls (diffusion.f90:1008-1118)
    if (edge_lo || edge_hi) {
      if (edge_lo)
        for (int k = threadIdx.x; k < NF * (SLD_TP + 4); k += blockDim.x) {
          int f = k / (SLD_TP + 4), b = k - f * (SLD_TP + 4);
          X[f][b][1] = sld_ghost_t(g, f + off, X[f][b][2], X[f][b][3], X[f][b][4], X[f][b][5], 1);
        }
      if (edge_hi)
        for (int k = threadIdx.x; k < NF * (SLD_TP + 4); k += blockDim.x) {
          int f = k / (SLD_TP + 4), b = k - f * (SLD_TP + 4), a = nth - t0 + 2;
          X[f][b][a] = sld_ghost_t(g, f + off, X[f][b][a - 1], X[f][b][a - 2], X[f][b][a - 3], X[f][b][a - 4], 0);
        }
      __syncthreads();
    }
    // face speeds (shared by every field): theta faces carry sin(face)
    const double st_hi =
        th_hi_in ? (g.sld_coef * sqrt(0.5 * (V[ty + 1][tx + 2] + V[ty + 1][tx + 1]))) * __ldg(g.sld_th + gt_hi) : 0.0;
    const double sp_hi = g.sld_coef * sqrt(0.5 * (V[ty + 1][tx + 1] + V[ty + 2][tx + 1]));
    double s_lo = 0.0;
    if (lo_p) s_lo = g.sld_coef * sqrt(0.5 * (V[0][tx + 1] + V[1][tx + 1]));
    else if (lo_t && th_lo_in) s_lo = (g.sld_coef * sqrt(0.5 * (V[tx + 1][1] + V[tx + 1][0]))) * __ldg(g.sld_th + t0);
    // face fluxes of every field: each thread takes the upper theta face and
    // the upper phi face of its cell; warp 0 also the phi faces of row 0,
    // warp 1 the theta faces of column 0.  Unrolled over the fields: their
    // limiter chains are independent, and with every field index static the
    // longer code no longer costs instruction-cache stalls (2.21 -> 2.03 ms
    // on 128x256x512)
#pragma unroll
    for (int f = 0; f < NF; f++) {
      const double tiny = g.tinyvar[f + off], itiny = g.inv_tinyvar[f + off];
      const double *xr = &X[f][ty + 2][tx + 1];
      FT[f][ty][tx + 1] = th_hi_in ? st_hi * sld_face(xr[0], xr[1], xr[2], xr[3], tiny, itiny) : 0.0;
      FP[f][ty + 1][tx] = sp_hi * sld_face(X[f][ty + 1][tx + 2], X[f][ty + 2][tx + 2], X[f][ty + 3][tx + 2],
                                           X[f][ty + 4][tx + 2], tiny, itiny);
      if (lo_p) {
        FP[f][0][tx] = s_lo * sld_face(X[f][0][tx + 2], X[f][1][tx + 2], X[f][2][tx + 2], X[f][3][tx + 2], tiny, itiny);
      } else if (lo_t) {
        const double *xl = &X[f][tx + 2][0];
        FT[f][tx][0] = th_lo_in ? s_lo * sld_face(xl[0], xl[1], xl[2], xl[3], tiny, itiny) : 0.0;
      }
    }
    // the velocities of this cell, taken from the tile when they are diffused
    // fields (before the barrier: the next radius's copies reuse the buffer)
    double uu[4] = {0.0, 0.0, 0.0, 0.0};
    if (hydro_part)
#pragma unroll
      for (int k = 1; k <= 3; k++) {
        const int f = k - off;
        uu[k] = (f >= 0 && f < NF) ? X[f >= 0 && f < NF ? f : 0][ty + 2][tx + 2]
                                   : __ldg(v + k * n + css_idx(g, itc, ipc, ir));
      }
    __syncthreads();
    double Dv[NF];
#pragma unroll
    for (int f = 0; f < NF; f++) {
      const int iv = f + off, iv1 = iv + 1;
      double prR = 1.0, prTP = 1.0;
      if (g.sld_pr != 1.0 || g.sld_prm != 1.0) {
        if (iv1 <= 3) prR = g.sld_pr; else if (iv1 >= 5) prR = g.sld_prm;
        if (iv1 < 5) prTP = g.sld_pr; else if (iv1 > 5) prTP = g.sld_prm;
      }
      double dup = (ir == nr - 1) ? 0.0
                                  : vr_hi * (sld_face(win[f][0], win[f][1], win[f][2], win[f][3], g.tinyvar[iv],
                                                      g.inv_tinyvar[iv]) * rhi2);
      double flux = t3 * (dup - carry[f]);
      if (prR != 1.0) flux = prR * flux;
      double acc = flux;
      carry[f] = dup;
      flux = (rfac / (cphl - cphh)) * (FT[f][ty][tx + 1] - FT[f][ty][tx]);
      if (prTP != 1.0) flux = prTP * flux;
      acc = acc + flux;
      flux = FP[f][ty + 1][tx] - FP[f][ty][tx];
      if (prTP != 1.0) flux = prTP * flux;
      acc = acc + geom * flux;
      Dv[f] = acc;
      // slide the window: x(ir+3) is a ghost exactly when ir+3 == nr
      win[f][0] = win[f][1];
      win[f][1] = win[f][2];
      win[f][2] = win[f][3];
      win[f][3] = (ir + 3 == nr) ? sld_ghost_r(g, v, av, iv, itc, ipc, 0) : nxt[f];
    }
    vc_a = vc_b;
    vc_b = vc_n;
    if (!live) continue;
    const size_t id = css_idx(g, it, ip, ir);
    double D[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      int f = k - off;
      D[k] = (f >= 0 && f < NF) ? Dv[f >= 0 && f < NF ? f : 0] : 0.0;
    }
    if (hydro_part) {
      const double rho = rho_c;
      double invrho = 1.0 / rho;
      // 1/T: from the temperature of this state when the caller has it (tb),
      // else rho^(1-gamma) exp(-s/Cv) / invtconst as one exponential (t_c = s)
      double itemp = tb ? 1.0 / t_c : exp(-fma(g.gamm1, log(rho), t_c * g.invcv)) / g.invtconst;
      if (g.do_viscous_heating)
#pragma unroll
        for (int k = 1; k <= 3; k++) D[4] = D[4] - uu[k] * D[k] * itemp;
      if (g.mass_diffusion) {
#pragma unroll
        for (int k = 1; k <= 3; k++) D[k] = D[k] - invrho * uu[k] * D[0];
        D[4] = D[4] - (g.gamm1 * g.cv) * invrho * D[0];
      }
    }
#pragma unroll
    for (int k = 0; k < 8; k++)
      if (k < g.nv && ((wmask >> k) & 1u)) dout[k * n + id] = D[k];
  }
}

// ohmic heating (diffusion.f90:430-455): Ds -= B . curl(D_A) / (8 pi rho T)
__global__ void k_sld_ohmic(CssGeo g, const double *__restrict__ v, const double *__restrict__ bf,
                            const double *__restrict__ cda, double *__restrict__ dout) {
  size_t n = (size_t)g.ncell;
  for (size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x; id < n; id += (size_t)gridDim.x * blockDim.x) {
    double rho = __ldg(v + id);
    double itemp = (pow(rho, -g.gamm1)) * exp(-__ldg(v + 4 * n + id) * g.invcv) / g.invtconst;
    double f = (0.5 * ONE_OVER_4PI) * (1.0 / rho) * itemp;
    double ds = dout[4 * n + id];
    for (int k = 0; k < 3; k++) ds = ds - __ldg(bf + k * n + id) * __ldg(cda + k * n + id) * f;
    dout[4 * n + id] = ds;
  }
}

// ---------------------------------------------------------------------------
// generic single-field derivative (css_deriv): one kernel per direction
// ---------------------------------------------------------------------------
template <int ORDER, int MT>
__global__ void __launch_bounds__(128) k_deriv_theta(CssGeo g, const double *__restrict__ f, double *__restrict__ out,
                                                     const double *__restrict__ bclo, const double *__restrict__ bchi,
                                                     int bdry, int TL) {
  extern __shared__ double sm[];
  const int nchunk = (g.nphi + TL - 1) / TL;
  const int bt = blockIdx.x / nchunk, pb = (blockIdx.x - bt * nchunk) * TL;
  const int ir = blockIdx.y;
  const CssDir &D = g.d[1];
  const int t0 = D.start[bt], m = D.size[bt];
  const int SR = m + 9, SO = m + 1;
  double *H = sm, *O = H + (size_t)TL * SR;
  load_theta_tile(g, f, H, SR, t0, m, pb, TL, ir, true);
  __syncthreads();
  for (int l = threadIdx.x; l < TL; l += blockDim.x) {
    int ip = pb + l;
    if (ip >= g.nphi) continue;
    double lo = (D.lphys[bt] && bclo) ? bclo[ip + (size_t)g.nphi * ir] : 0.0;
    double hi = (D.rphys[bt] && bchi) ? bchi[ip + (size_t)g.nphi * ir] : 0.0;
    double dn = (ORDER == 1) ? D.dnum[bt] : dnum_d2_theta(g, ir);
    double sc = (ORDER == 1) ? D.dnum[bt] : D.dnum[bt] * D.dnum[bt];
    solve<ORDER, MT>(H + (size_t)l * SR + 4, 1, m, dtype_of(D, bt), bdry, lo, hi, tabp(g, 1, bt, ORDER, bdry),
                      g.tstride, dn, sc, 0, O + (size_t)l * SO, 1);
  }
  __syncthreads();
  for (int pt = threadIdx.x; pt < TL * m; pt += blockDim.x) {
    int l = pt / m, j = pt - l * m;
    if (pb + l >= g.nphi) continue;
    out[css_idx(g, t0 + j, pb + l, ir)] = O[(size_t)l * SO + j];
  }
}

template <int ORDER, int MT>
__global__ void __launch_bounds__(128) k_deriv_phi(CssGeo g, const double *__restrict__ f, double *__restrict__ out,
                                                   int TL) {
  extern __shared__ double sm[];
  const int nchunk = (g.nth + TL - 1) / TL;
  const int bp = blockIdx.x / nchunk, tb = (blockIdx.x - bp * nchunk) * TL;
  const int ir = blockIdx.y;
  const CssDir &D = g.d[2];
  const int p0 = D.start[bp], m = D.size[bp];
  const int SR = TL + 1;
  double *H = sm, *O = H + (size_t)(m + 8) * SR;
  load_phi_tile(g, f, H, SR, p0, m, tb, TL, ir, true);
  __syncthreads();
  for (int l = threadIdx.x; l < TL; l += blockDim.x) {
    if (tb + l >= g.nth) continue;
    double sc = (ORDER == 1) ? D.dnum[bp] : D.dnum[bp] * D.dnum[bp];
    solve<ORDER, MT>(H + 4 * SR + l, SR, m, 3, 0, 0.0, 0.0, tabp(g, 2, bp, ORDER, 0), g.tstride, D.dnum[bp], sc, 1,
                      O + l, SR);
  }
  __syncthreads();
  for (int pt = threadIdx.x; pt < TL * m; pt += blockDim.x) {
    int j = pt / TL, l = pt - j * TL;
    if (tb + l >= g.nth) continue;
    out[css_idx(g, tb + l, p0 + j, ir)] = O[(size_t)j * SR + l];
  }
}

template <int ORDER, int MT>
__global__ void __launch_bounds__(128) k_deriv_r(CssGeo g, const double *__restrict__ f, double *__restrict__ out,
                                                 const double *__restrict__ bclo, const double *__restrict__ bchi,
                                                 int bdry, int TL) {
  extern __shared__ double sm[];
  const int nchunk = (g.nth + TL - 1) / TL;
  const int br = blockIdx.x / nchunk, tb = (blockIdx.x - br * nchunk) * TL;
  const int ip = blockIdx.y;
  const CssDir &D = g.d[0];
  const int r0 = D.start[br], m = D.size[br];
  const int SR = TL + 1;
  double *H = sm, *O = H + (size_t)(m + 8) * SR;
  load_r_tile(g, f, H, SR, r0, m, tb, TL, ip, true);
  __syncthreads();
  for (int l = threadIdx.x; l < TL; l += blockDim.x) {
    int it = tb + l;
    if (it >= g.nth) continue;
    double lo = (D.lphys[br] && bclo) ? bclo[it + (size_t)g.nth * ip] : 0.0;
    double hi = (D.rphys[br] && bchi) ? bchi[it + (size_t)g.nth * ip] : 0.0;
    double sc = (ORDER == 1) ? D.dnum[br] : D.dnum[br] * D.dnum[br];
    solve<ORDER, MT>(H + 4 * SR + l, SR, m, dtype_of(D, br), bdry, lo, hi, tabp(g, 0, br, ORDER, bdry), g.tstride,
                      D.dnum[br], sc, 0, O + l, SR);
  }
  __syncthreads();
  for (int pt = threadIdx.x; pt < TL * m; pt += blockDim.x) {
    int j = pt / TL, l = pt - j * TL;
    if (tb + l >= g.nth) continue;
    out[css_idx(g, tb + l, ip, r0 + j)] = O[(size_t)j * SR + l];
  }
}

// Cyclic phi derivative of one field (css_dbydp_cyclic; an extension with
// no counterpart in the reference, whose Dbydp closes each block with halo
// rows, derivatives.f90:1480-1591): every whole phi line is periodic and
// takes Dbydp's interior rows at every point; the cyclic tridiagonal
// system is solved by Sherman-Morrison, A = B + u v^T with gamma = -1, as
// x = y - (v.y)/(1 + v.z) z.  T holds, for this order and nphi, B's
// elimination factors w[j], pivots piv[j], the vector z = B^-1 u and v.z.
// One thread per (theta, r) line; consecutive threads take consecutive
// theta, so every load and store is coalesced.
__global__ void k_dbydp_cyclic(CssGeo g, const double *__restrict__ x, double *__restrict__ out,
                               const double *__restrict__ T, int order, double scale) {
  const int nth = g.nth, n = g.nphi;
  const size_t line = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (line >= (size_t)nth * g.nr) return;
  const int t = (int)(line % nth), r = (int)(line / nth);
  const size_t base = (size_t)r * nth * n + t;
  const double *w = T, *piv = T + n, *z = T + 2 * n;
  const double vz = T[3 * n];
  const double alpha = order == 1 ? 1.0 / 3.0 : 2.0 / 11.0, ag = -alpha;  // alpha / gamma, gamma = -1
  auto X = [&](int j) { return __ldg(x + base + (size_t)j * nth); };
  double fm2 = X(n - 2), fm1 = X(n - 1), f0 = X(0), fp1 = X(1), fp2 = X(2);
  double prev = 0.0;
  for (int j = 0; j < n; j++) {
    const double rhs = order == 1 ? (7.0 / 9.0) * (fp1 - fm1) + (1.0 / 36.0) * (fp2 - fm2)
                                  : (12.0 / 11.0) * (fp1 - 2.0 * f0 + fm1) + (3.0 / 44.0) * (fp2 - 2.0 * f0 + fm2);
    const double y = j == 0 ? rhs / __ldg(piv) : (rhs - alpha * prev) / __ldg(piv + j);
    out[base + (size_t)j * nth] = y;
    prev = y;
    fm2 = fm1; fm1 = f0; f0 = fp1; fp1 = fp2;
    int k = j + 3;
    if (k >= n) k -= n;
    fp2 = X(k);
  }
  const double yl = prev;
  double next = prev;
  for (int j = n - 2; j >= 0; j--) {
    const double y = out[base + (size_t)j * nth] - __ldg(w + j + 1) * next;
    out[base + (size_t)j * nth] = y;
    next = y;
  }
  const double fact = (next + ag * yl) / (1.0 + vz);
  for (int j = 0; j < n; j++) {
    const size_t q = base + (size_t)j * nth;
    out[q] = scale * (out[q] - fact * __ldg(z + j));
  }
}

// Adjoint of the whole-field compact derivative along direction dir (the
// backward of torch.ops.css.deriv): gx = D^T g with zero boundary data.
// M holds every block's dense operator, rows = the block's m outputs,
// columns = its m + 8 inputs (4 halo points below, the block, 4 above),
// at M + off[b].  A point is an input of its own block and, within four
// points of a block face, a halo input of the neighbouring block (phi
// periodic), so gx at that point gathers one column of each: a fixed-order
// sum, deterministic.  One thread per point.
__global__ void k_deriv_adjoint(CssGeo g, int dir, const double *__restrict__ M, const int *__restrict__ off,
                                const double *__restrict__ gin, double *__restrict__ gout) {
  const size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (id >= (size_t)g.ncell) return;
  const int it = (int)(id % g.nth), ip = (int)((id / g.nth) % g.nphi), ir = (int)(id / ((size_t)g.nth * g.nphi));
  const CssDir &D = g.d[dir];
  const int a = dir == 0 ? ir : (dir == 1 ? it : ip);
  int b = 0;
  while (b + 1 < D.nb && D.start[b + 1] <= a) b++;
  const int i = a - D.start[b], m = D.size[b];
  auto gat = [&](int aa) -> double {
    return __ldg(gin + (dir == 0 ? css_idx(g, it, ip, aa) : (dir == 1 ? css_idx(g, aa, ip, ir) : css_idx(g, it, aa, ir))));
  };
  auto col = [&](int bb, int c) -> double {
    const int mb = D.size[bb], s0 = D.start[bb];
    const double *Mb = M + off[bb];
    double acc = 0.0;
    for (int q = 0; q < mb; q++) acc += __ldg(Mb + (size_t)q * (mb + 8) + c) * gat(s0 + q);
    return acc;
  };
  double acc = col(b, i + 4);
  const bool periodic = dir == 2;
  if (i < 4) {
    int bb = b - 1;
    if (bb < 0 && periodic) bb = D.nb - 1;
    if (bb >= 0) acc += col(bb, D.size[bb] + 4 + i);
  }
  if (i >= m - 4) {
    int bb = b + 1;
    if (bb >= D.nb && periodic) bb = 0;
    if (bb < D.nb) acc += col(bb, i - (m - 4));
  }
  gout[id] = acc;
}

// independent lines with explicit closures, staged through shared memory:
// a CTA of 128 threads takes KL_LINES consecutive lines (contiguous in
// memory, so the whole CTA reads and writes them with consecutive
// addresses), one thread solves each line from its shared row (rows of
// n + 9 doubles, an odd stride: the solving threads touch distinct banks),
// and the results go back the same way.  The arithmetic per line is
// k_lines's.  n <= KL_MAXN.
#define KL_LINES 16
#define KL_MAXN 248
__global__ void __launch_bounds__(128) k_lines_tiled(const double *__restrict__ x, double *__restrict__ out, int n,
                                                     int nlines, int order, int dtype, int bdry,
                                                     const double *__restrict__ bclo, const double *__restrict__ bchi,
                                                     const double *__restrict__ hlo, const double *__restrict__ hhi,
                                                     const double *__restrict__ tab, int ts, double dnum,
                                                     double scale) {
  extern __shared__ double sm[];
  const int sr = n + 9;  // n + 8 used, odd
  double *X = sm, *Y = sm + (size_t)KL_LINES * sr;
  const int l0 = blockIdx.x * KL_LINES, nl = min(KL_LINES, nlines - l0);
  const size_t base = (size_t)l0 * n;
  for (int k = threadIdx.x; k < nl * n; k += blockDim.x) {
    const int l = k / n, j = k - l * n;
    X[l * sr + 4 + j] = x[base + k];
  }
  for (int k = threadIdx.x; k < nl * 8; k += blockDim.x) {
    const int l = k >> 3, q = k & 7;
    const double *h = q < 4 ? hlo : hhi;
    X[l * sr + (q < 4 ? q : n + q)] = h ? h[(size_t)4 * (l0 + l) + (q & 3)] : 0.0;
  }
  __syncthreads();
  if (threadIdx.x < nl) {
    const int l = threadIdx.x;
    const double lo = bclo ? bclo[l0 + l] : 0.0, hi = bchi ? bchi[l0 + l] : 0.0;
    const double *G = tab + (size_t)bdry * 3 * ts;
    if (order == 1)
      line_solve<1>(X + l * sr + 4, 1, n, dtype, bdry, lo, hi, G, ts, dnum, scale, 0, Y + l * sr, 1);
    else
      line_solve<2>(X + l * sr + 4, 1, n, dtype, bdry, lo, hi, G, ts, dnum, scale, 0, Y + l * sr, 1);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < nl * n; k += blockDim.x) {
    const int l = k / n, j = k - l * n;
    out[base + k] = Y[l * sr + j];
  }
}

// independent lines with explicit closures (css_compact_lines /
// Dbyd1_dt0): one thread per line on global memory, lines contiguous.
__global__ void k_lines(const double *__restrict__ x, double *__restrict__ out, int n, int nlines, int order,
                        int dtype, int bdry, const double *__restrict__ bclo, const double *__restrict__ bchi,
                        const double *__restrict__ hlo, const double *__restrict__ hhi, const double *__restrict__ tab,
                        int ts, double dnum, double scale, double *__restrict__ work) {
  int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nlines) return;
  double *xs = work + (size_t)l * (n + 8);
  for (int k = 0; k < 4; k++) {
    xs[k] = hlo ? hlo[(size_t)4 * l + k] : 0.0;
    xs[n + 4 + k] = hhi ? hhi[(size_t)4 * l + k] : 0.0;
  }
  for (int j = 0; j < n; j++) xs[j + 4] = x[(size_t)l * n + j];
  double lo = bclo ? bclo[l] : 0.0, hi = bchi ? bchi[l] : 0.0;
  const double *G = tab + (size_t)bdry * 3 * ts;
  if (order == 1)
    line_solve<1>(xs + 4, 1, n, dtype, bdry, lo, hi, G, ts, dnum, scale, 0, out + (size_t)l * n, 1);
  else
    line_solve<2>(xs + 4, 1, n, dtype, bdry, lo, hi, G, ts, dnum, scale, 0, out + (size_t)l * n, 1);
}

}  // namespace css
