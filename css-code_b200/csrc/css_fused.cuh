// css_fused.cuh -- the RK4 stage in two passes over HBM, for runs whose
// virtual blocks are 32 points long in r, theta and phi (FP64 state, RK4,
// closed radial faces, SLaplacian/SLD physics; css_create decides).
//
//   k_thph    tiles of one (theta block, phi block, radius) plane: the
//             32x32 plane of the two blocks with 4-point halos in theta and
//             phi is staged once in shared memory, and the theta and phi
//             line solves of every field run at once; Source_Theta_Terms
//             (+ Lorentz, + Induction_Terms), Phi_Terms (+ Lorentz) and, on
//             blocks with no theta wall, Density_Terms_Theta run from it, and
//             the tendency of every field and the stage temperature are
//             written once.
//   k_rstage  tiles of one (r block, theta block, phi) slab: the
//             32(r)x32(theta) slab with 4-point radial halos, and the
//             tendency and temperature of its points, are staged once;
//             Radial_Terms (+ Lorentz) with Density_Terms_Radial,
//             Density_Terms_Theta on the theta-wall blocks (its wall datum is
//             the completed dw/dt, available only here), the RK4 stage
//             combination of Step_RK4 and Bound, writing the accumulator and
//             the next stage state.
//
// The plane pass is persistent (one 512-thread CTA per SM walks the tiles;
// hydro double-buffers its planes, MHD refills its one plane buffer by TMA
// under the pointwise phases: an L2 prefetch of the next tile's lines made
// it slower); the slab
// pass brings each tile's per-point lines toward L2 while its slab arrives,
// one tile per CTA for hydro, persistent for MHD.  Inside a tile the line solves of different
// fields and directions run side by side on different warps (forward values in registers, css_lines.cuh
// line_solve_r), with the spare warps computing the pointwise quantities
// (temperature, 1/rho) the physics phase needs.
//
// Against the four-kernel stage (theta, phi, radial, update) this removes
// the read-modify-write of the tendency by the phi and radial passes and
// one read of the state and the tendency per stage.  The arithmetic per
// point is that of k_theta_terms, phi_tile_compute, radial_tile and
// k_rhot_update; only the order in which the density-theta term joins the
// sums differs (it follows the theta terms here), a rounding-level change.
#pragma once
#include <cuda.h>  // CUtensorMap
#include <cstdint>
#include "css_kernels.cuh"

namespace css {

constexpr int FM = 32;    // block length of the fused path (every direction)
constexpr int FNT = 512;  // threads per CTA of both kernels (one CTA per SM)

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

// offset of field f in a plane buffer: MHD's B_phi (field 6) has no phi
// derivative, so it is staged without its phi-halo rows and B_r follows its
// main rows (10944 doubles in: still 128-byte aligned)
__host__ __device__ constexpr int thph_foff(int mag, int f) {
  return f * FA_FIELD - ((mag && f == 7) ? 8 * FM : 0);
}

template <int MAG>
struct ThphCfg {
  static constexpr int NF = MAG ? 8 : 5;     // rho w v u s [bt bp br]
  // derivative tiles: both directions' at once (theta 0-5, phi 6-11 hydro;
  // theta 0-7, phi 8-15 MHD)
  static constexpr int NO = MAG ? 16 : 12;
  static constexpr int PHI0 = MAG ? 8 : 6;   // first phi tile
  static constexpr int PLANE = MAG ? 7 * FA_FIELD + FA_MAIN : NF * FA_FIELD;  // doubles of one plane buffer
  // hydro stages the next tile's plane into a second buffer while it
  // computes the current one; MHD (eight fields) has room for one plane,
  // refilled with the next tile's once the solves are done with it
  static constexpr int NBUF = MAG ? 1 : 2;
  // + one mbarrier per plane buffer
  static constexpr size_t SMEM = 8 * ((size_t)NBUF * PLANE + (size_t)NO * FA_OUT + NBUF);
  // bytes one plane's copies deliver
  static constexpr unsigned TX = 8u * PLANE;
};
static_assert(ThphCfg<1>::SMEM <= 232448, "MHD plane pass: one plane and sixteen tiles fit 227 KB");

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

// ---- TMA tile copies completing on an mbarrier (each into this CTA's own
// shared memory only) -------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// orders the barrier initialisation (generic proxy) before the async proxy's
// use of it
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// orders this thread's earlier shared-memory accesses (and those the barrier
// before it made visible) before later async-proxy copies into that memory
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// waits for the phase of the given parity, for at most about `cycles` SM
// clocks; false when the limit ran out
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, long long cycles) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > cycles) return false;
  return true;
}
// one 4-D box of a tiled tensor map into shared memory; x (the innermost,
// theta) start is a multiple of 2 doubles, so 16-byte aligned
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *tm, int x, int y, int z, int w,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
      : "memory");
}
// about two seconds at the B200's clocks: a bound no healthy copy reaches
constexpr long long kWaitCycles = 4000000000ll;
// bit of the step flag a timed-out wait sets (bit 0 is a non-finite state)
constexpr int kFlagTimeout = 2;

// The tensor maps of one state buffer: 4-D (theta, phi, r, field) FP64,
// boxes of the plane's main rows (42 theta x 32 phi) and of its phi halo
// (32 theta x 4 phi).
struct PlaneMaps {
  CUtensorMap main, halo;
};
// The tensor maps of the stage kernel's slab: the state buffer (or B) with
// a 32 theta x 1 phi x 40 r box, and the wall d(rho)/dtheta rows (theta 32,
// side 2, phi, r) with a 32 x 1 x 1 x 32 box.
struct SlabMaps {
  CUtensorMap slab;
};

// ---------------------------------------------------------------------------
// k_thph.  Persistent: CTA b takes tiles b, b + gridDim.x, ...; a tile is
// (theta block bt, phi block bp, radius ir), phi block fastest.  cur =
// stage input (FP64), bf = B (MHD), dv = tendency (written), tbuf = T
// (written).
// ---------------------------------------------------------------------------
struct ThphTile {
  int bt, bp, ir, t0, p0;
};
__device__ __forceinline__ ThphTile thph_tile(const CssGeo &g, int q) {
  const int nbp = g.d[2].nb, nbt = g.d[1].nb;
  ThphTile T;
  T.bp = q % nbp;
  const int r = q / nbp;
  T.bt = r % nbt;
  T.ir = r / nbt;
  T.t0 = g.d[1].start[T.bt];
  T.p0 = g.d[2].start[T.bp];
  return T;
}

// stage the plane with TMA boxes (called by one thread): per field the main
// rows over theta t0-4 .. t0+37 (zero outside [0, nth)) and the two 4-row
// phi halos (periodic; blocks are 32 long, so a halo box never wraps)
template <int NF>
__device__ __forceinline__ void thph_stage_tma(const CssGeo &g, const PlaneMaps &mc, const PlaneMaps &mb,
                                               const ThphTile &T, double *F, uint64_t *bar) {
  const int plo = T.p0 >= 4 ? T.p0 - 4 : g.nphi - 4;
  const int phi = T.p0 + FM < g.nphi ? T.p0 + FM : 0;
  constexpr int MAGF = NF == 8;
  mbar_expect_tx(bar, 8u * ThphCfg<MAGF>::PLANE);
#pragma unroll
  for (int f = 0; f < NF; f++) {
    const PlaneMaps &m = f < 5 ? mc : mb;
    const int w = f < 5 ? f : f - 5;
    double *Fd = F + thph_foff(MAGF, f);
    tma_load_4d(Fd, &m.main, T.t0 - 4, T.p0, T.ir, w, bar);
    if (MAGF && f == 6) continue;  // B_phi: main rows only
    tma_load_4d(Fd + FA_MAIN, &m.halo, T.t0, plo, T.ir, w, bar);
    tma_load_4d(Fd + FA_MAIN + 4 * FM, &m.halo, T.t0, phi, T.ir, w, bar);
  }
}

// theta line solve of derivative tile k (0 dw 1 dv 2 du 3 ds 4 d2s [5 dbp
// 6 dbr] then d(rho) off the walls), line (phi row) p
template <int MAG>
__device__ __forceinline__ void thph_theta_solve(const CssGeo &g, const double *F, double *O, const ThphTile &T,
                                                 int k, int p) {
  const CssDir &DT = g.d[1];
  const int bt = T.bt;
  int f, var, order = 1;
  if (k < 4) { f = 1 + k; var = 2 + k; }
  else if (k == 4) { f = 4; var = 5; order = 2; }
  else if (MAG && k < 7) { f = k + 1; var = k + 3; }  // bp (8), br (9)
  else { f = 0; var = 1; }
  const int bdry = g.ibct[var];
  const double *x = F + thph_foff(MAG, f) + p * FA_RW;
  double lo = 0.0, hi = 0.0;
  const int nth = g.nth;
  if (f == 2) {  // stress-free datum cot(theta)*v on the walls (rhs_mpi.f90:414, :444)
    if (DT.lphys[bt]) lo = (g.cosines[0] / g.sines[0]) * x[4];
    if (DT.rphys[bt]) hi = (g.cosines[nth - 1] / g.sines[nth - 1]) * x[4 + FM - 1];
  }
  if (MAG && f == 6 && g.theta_normal_field) {  // (rhs_mpi.f90:421, :451)
    if (DT.lphys[bt]) lo = -(g.cosines[0] / g.sines[0]) * x[4];
    if (DT.rphys[bt]) hi = -(g.cosines[nth - 1] / g.sines[nth - 1]) * x[4 + FM - 1];
  }
  const int dtype = dtype_of(DT, bt);
  const double dn = DT.dnum[bt];
  if (order == 2) {
    if (g.slaplacian)
      line_solve_r<2, FM>(x, ThIdx{}, dtype, bdry, lo, hi, tabp(g, 1, bt, 2, bdry), g.tstride, dnum_d2_theta(g, T.ir),
                          dn * dn, 0, O + k * FA_OUT, SwzRow{p});
  } else {
    line_solve_r<1, FM>(x, ThIdx{}, dtype, bdry, lo, hi, tabp(g, 1, bt, 1, bdry), g.tstride, dn, dn, 0,
                        O + k * FA_OUT, SwzRow{p});
  }
}

// phi line solve of derivative tile k (0 drho 1 dv 2 dw 3 du 4 ds 5 d2s
// [6 dbt 7 dbr]) into O + k0 + k, line (theta column) t
template <int MAG>
__device__ __forceinline__ void thph_phi_solve(const CssGeo &g, const double *F, double *O, const ThphTile &T, int k,
                                               int k0, int t) {
  const int f = k == 0 ? 0 : k == 1 ? 2 : k == 2 ? 1 : k == 3 ? 3 : k <= 5 ? 4 : (k == 6 ? 5 : 7);
  const double dn = g.d[2].dnum[T.bp];
  const double *x = F + thph_foff(MAG, f);
  if (k == 5) {
    if (g.slaplacian)
      line_solve_r<2, FM>(x, PhIdx{t}, 3, 0, 0.0, 0.0, tabp(g, 2, T.bp, 2, 0), g.tstride, dn, dn * dn, 1,
                          O + (k0 + k) * FA_OUT, SwzCol{t});
  } else {
    line_solve_r<1, FM>(x, PhIdx{t}, 3, 0, 0.0, 0.0, tabp(g, 2, T.bp, 1, 0), g.tstride, dn, dn, 1,
                        O + (k0 + k) * FA_OUT, SwzCol{t});
  }
}

// d(rho)/dtheta with a zero wall datum on a theta-wall block (bdry ibct(1)),
// line p, into rtw (k_rstage adds the datum times the unit response)
__device__ __forceinline__ void thph_wall_rho(const CssGeo &g, const double *F, const ThphTile &T, int p,
                                              double *__restrict__ rtw) {
  const CssDir &DT = g.d[1];
  const int bdry = g.ibct[1], side = DT.lphys[T.bt] ? 0 : 1;
  const double dn = DT.dnum[T.bt];
  double *o = rtw + (((size_t)T.ir * g.nphi + T.p0 + p) * 2 + side) * FM;
  line_solve_r<1, FM>(F + p * FA_RW, ThIdx{}, dtype_of(DT, T.bt), bdry, 0.0, 0.0, tabp(g, 1, T.bt, 1, bdry),
                      g.tstride, dn, dn, 0, o, StridedOut{1});
}

template <int MAG>
__global__ void __launch_bounds__(FNT, 1) k_thph(CssGeo g, const double *__restrict__ cur,
                                                 const double *__restrict__ bf, double *__restrict__ dv,
                                                 double *__restrict__ tbuf, double *__restrict__ rtw,
                                                 const __grid_constant__ PlaneMaps mc,
                                                 const __grid_constant__ PlaneMaps mb, int *flag) {
  using C = ThphCfg<MAG>;
  constexpr int NA = MAG ? 8 : 5;
  // plane buffers (128-byte aligned boxes: a field is 12800 bytes), the
  // derivative tiles, the buffers' mbarriers
  extern __shared__ __align__(128) double sm[];
  double *O = sm + (size_t)C::NBUF * C::PLANE;  // NO derivative tiles
  uint64_t *bar = reinterpret_cast<uint64_t *>(O + (size_t)C::NO * FA_OUT);
  const int tid = threadIdx.x, lane = tid & 31, wrp = tid >> 5;
  const size_t n = (size_t)g.ncell;
  const int ntile = g.nr * g.d[1].nb * g.d[2].nb;
  if (tid == 0) {
    for (int b = 0; b < C::NBUF; b++) mbar_init(bar + b, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (C::NBUF == 2 && tid == 0 && (int)blockIdx.x < ntile)
    thph_stage_tma<C::NF>(g, mc, mb, thph_tile(g, blockIdx.x), sm, bar);
  for (int q = blockIdx.x, i = 0; q < ntile; q += gridDim.x, i++) {
    const ThphTile T = thph_tile(g, q);
    const int b = C::NBUF == 2 ? (i & 1) : 0;
    double *F = sm + (size_t)b * C::PLANE;
    const bool more = q + (int)gridDim.x < ntile;
    if (C::NBUF == 2) {
      // the next plane into the other buffer: its last readers passed the
      // barrier that ended the previous tile
      if (more && tid == 0) {
        fence_proxy_async();
        thph_stage_tma<C::NF>(g, mc, mb, thph_tile(g, q + gridDim.x), sm + (size_t)(b ^ 1) * C::PLANE,
                              bar + (b ^ 1));
      }
    } else if (tid == 0 && i == 0) {
      // MHD: the first tile's planes; each later tile's copies start under
      // the previous tile's pointwise phases, once its plane values are in
      // registers (bringing the next tile's lines toward L2 instead, as an
      // earlier form did, cost 11.6 against 9.8 ms a launch)
      fence_proxy_async();
      thph_stage_tma<C::NF>(g, mc, mb, T, F, bar);
    }
    // this plane's copies: buffer b's (i >> 1)-th use (every use for MHD)
    const unsigned parity = C::NBUF == 2 ? ((unsigned)(i >> 1) & 1u) : ((unsigned)i & 1u);
    const bool late = !mbar_wait_bounded(bar + b, parity, kWaitCycles);
    if (__syncthreads_or(late)) {
      // a copy that never completes: report it and stop, after giving the
      // copies still in flight the same bound to land
      if (tid == 0) {
        atomicOr(flag, kFlagTimeout);
        mbar_wait_bounded(bar + b, parity, kWaitCycles);
        if (C::NBUF == 2 && more) mbar_wait_bounded(bar + (b ^ 1), (unsigned)((i + 1) >> 1) & 1u, kWaitCycles);
      }
      return;
    }
    const CssDir &DT = g.d[1];
    const bool wall = DT.lphys[T.bt] || DT.rphys[T.bt];
    const int ir = T.ir, it = T.t0 + lane;
    // ---- T, 1/rho and 1/(rho T) of this thread's two points (rows wrp,
    // wrp + 16, theta t0 + lane), T also to tbuf ----
    double tq[2], rq[2], rtq[2];
    {
      const size_t pl = plane(g, ir);
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int ic = (wrp + 16 * h) * FA_RW + lane + 4;
        const double rho = F[ic], s = F[4 * FA_FIELD + ic];
        tq[h] = temp_of(g, rho, s);
        rq[h] = 1.0 / rho;
        rtq[h] = rq[h] / tq[h];
      }
#pragma unroll
      for (int h = 0; h < 2; h++) tbuf[pl + (size_t)(T.p0 + wrp + 16 * h) * g.nth + it] = tq[h];
    }
    // ---- solves: theta (warps 0-5 hydro, 0-7 MHD), phi (warps 6-11 hydro,
    // 8-15 MHD), all at once ----
    {
      const int nth_t = (MAG ? 7 : 5) + (wall ? 0 : 1);
      const int nthw = MAG ? 8 : 6;  // theta warps; the last one solves d(rho)/dtheta
      if (wrp < nthw) {
        if (wrp < nth_t) thph_theta_solve<MAG>(g, F, O, T, wrp, lane);
        else thph_wall_rho(g, F, T, lane, rtw);
      } else if (wrp < (MAG ? 16 : 12)) {
        thph_phi_solve<MAG>(g, F, O, T, wrp - nthw, C::PHI0, lane);
      }
    }
    __syncthreads();
    // this thread's plane values of the pointwise phases; for MHD the plane
    // buffer is then free and the next tile's copies start under them (8.27
    // against 6.92 ms a launch at 256x512x1024)
    double pv[2][7];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int ic = (wrp + 16 * h) * FA_RW + lane + 4;
      pv[h][0] = F[ic]; pv[h][1] = F[FA_FIELD + ic]; pv[h][2] = F[2 * FA_FIELD + ic]; pv[h][3] = F[3 * FA_FIELD + ic];
      if (MAG) { pv[h][4] = F[5 * FA_FIELD + ic]; pv[h][5] = F[6 * FA_FIELD + ic]; pv[h][6] = F[thph_foff(MAG, 7) + ic]; }
    }
    if (C::NBUF == 1) {
      __syncthreads();
      if (more && tid == 0) {
        fence_proxy_async();
        thph_stage_tma<C::NF>(g, mc, mb, thph_tile(g, q + gridDim.x), F, bar);
      }
    }
    // ---- theta pointwise (Source_Theta_Terms, Lorentz, induction, and
    // Density_Terms_Theta off the walls): two points per thread ----
    const double ri = g.r_inv[ir];
    double acc[2][NA];
    {
      const double rv = g.r_ind[ir], epsr = g.eps[ir];
      const double omsq = rv * g.omega0 * g.omega0, om2 = 2.0 * g.omega0;
      const double sn = g.sines[it], cs = g.cosines[it], ct = g.cot[it];
      const int dtt = MAG ? 7 : 5;  // tile of d(rho)/dtheta
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int p = wrp + 16 * h;
        const double rho = pv[h][0], w = pv[h][1], v = pv[h][2], u = pv[h][3];
        const double t = tq[h], invrho = rq[h], oorho_t = rtq[h];
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
          const double bt_ = pv[h][4], bp_ = pv[h][5], br_ = pv[h][6];
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
          acc[h][NA - 3] = v * br_ - u * bp_;  // Induction_Terms: dA/dt = v x B
          acc[h][NA - 2] = u * bt_ - w * br_;
          acc[h][NA - 1] = w * bp_ - v * bt_;
        }
        if (!wall) {  // Density_Terms_Theta (rhs_mpi.f90:1522-1605), halo-closed rows
          w1 = ri * swz(O + dtt * FA_OUT, p, lane);
          drho = drho - w * w1;
          w1 = w1 * invrho;
          dw = dw - g.pconst * w1 * t;
        }
        acc[h][0] = drho; acc[h][1] = dw; acc[h][2] = dvv; acc[h][3] = du; acc[h][4] = ds;
      }
    }
    // ---- phi pointwise (Phi_Terms + Lorentz), then the stores ----
    {
      const double oors = ri * g.csc[it];
      const double *OP = O + C::PHI0 * FA_OUT;
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int p = wrp + 16 * h;
        const double rho = pv[h][0], v = pv[h][2];
        const double t = tq[h], oorho = rq[h], oorho_t = rtq[h];
        double drho = acc[h][0], dw = acc[h][1], dvv = acc[h][2], du = acc[h][3], ds = acc[h][4];
        double w1 = swz(OP, p, lane) * oors;
        drho = drho - v * w1;
        dvv = dvv - g.pconst * w1 * t * oorho;
        w1 = swz(OP + FA_OUT, p, lane) * oors;
        dvv = dvv - v * w1;
        drho = drho - rho * w1;
        w1 = swz(OP + 2 * FA_OUT, p, lane) * oors;
        dw = dw - v * w1;
        w1 = swz(OP + 3 * FA_OUT, p, lane) * oors;
        du = du - v * w1;
        w1 = swz(OP + 4 * FA_OUT, p, lane) * oors;
        ds = ds - v * w1;
        dvv = dvv - g.gamm1 * t * w1;
        if (g.slaplacian) {
          w1 = swz(OP + 5 * FA_OUT, p, lane) * (oors * oors);
          ds = ds + g.ks[ir] * w1 * oorho_t;
        }
        if (MAG) {
          const double oo = ONE_OVER_4PI * oorho * oors;
          const double bt_ = pv[h][4], bp_ = pv[h][5], br_ = pv[h][6];
          w1 = swz(OP + 6 * FA_OUT, p, lane) * oo;
          dvv = dvv - bt_ * w1;
          dw = dw + bp_ * w1;
          w1 = swz(OP + 7 * FA_OUT, p, lane) * oo;
          dvv = dvv - br_ * w1;
          du = du + bp_ * w1;
        }
        acc[h][0] = drho; acc[h][1] = dw; acc[h][2] = dvv; acc[h][3] = du; acc[h][4] = ds;
      }
      const size_t pl = plane(g, ir);
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const size_t id = pl + (size_t)(T.p0 + wrp + 16 * h) * g.nth + it;
#pragma unroll
        for (int f = 0; f < NA; f++) dv[f * n + id] = acc[h][f];
      }
    }
    __syncthreads();  // the next tile overwrites the plane and the tiles
  }
}

// ---- k_curl_pl: B = curl A's theta and phi parts from TMA-staged planes ----
// The plane tiles of k_thph (same tile order, same maps) carrying only A:
// fields 5, 6, 7 (A_theta, A_phi, A_r) of a state buffer; persistent CTAs.
// Per tile: sin(theta)
// A_phi in place, the theta lines of sin A_phi and A_r and the phi lines of
// A_r and A_theta (one warp each, one line per lane), then B_r complete and
// the theta / phi parts of B_theta / B_phi, with the expressions of
// k_curl_tp (VectorCurlA, derivatives.f90:1769-1828); k_curl_r adds the
// radial parts.
template <int NBUF, int NTH>
struct CurlCfg {
  static constexpr int NF = 3;
  static constexpr int NO = 4;
  static constexpr int NT = NTH;
  static constexpr size_t SMEM = 8 * ((size_t)NBUF * NF * FA_FIELD + (size_t)NO * FA_OUT + NBUF);
};

__device__ __forceinline__ void curl_stage_tma(const CssGeo &g, const PlaneMaps &m, const ThphTile &T, double *F,
                                               uint64_t *bar) {
  const int plo = T.p0 >= 4 ? T.p0 - 4 : g.nphi - 4;
  const int phi = T.p0 + FM < g.nphi ? T.p0 + FM : 0;
  mbar_expect_tx(bar, 8u * 3 * FA_FIELD);
#pragma unroll
  for (int f = 0; f < 3; f++) {
    double *Fd = F + (size_t)f * FA_FIELD;
    tma_load_4d(Fd, &m.main, T.t0 - 4, T.p0, T.ir, 5 + f, bar);
    tma_load_4d(Fd + FA_MAIN, &m.halo, T.t0, plo, T.ir, 5 + f, bar);
    tma_load_4d(Fd + FA_MAIN + 4 * FM, &m.halo, T.t0, phi, T.ir, 5 + f, bar);
  }
}

// NBUF 2: two plane buffers, the next tile's copies under the current
// tile; NBUF 1: one buffer and more CTAs per SM, so that one CTA's copies
// overlap another's solves, and each CTA's next copies start under its own
// stores (1.51 -> 1.44 ms a launch on MHD 256x512x1024; bringing the next
// tile's lines toward L2 at the start of a tile instead, as an earlier form
// did, cost 1.61 against 1.51 ms).
template <int NBUF, int NTH>
__global__ void __launch_bounds__(NTH, NBUF == 2 ? 2 : 3) k_curl_pl(CssGeo g, double *__restrict__ out,
                                                                    const __grid_constant__ PlaneMaps m, int *flag) {
  using C = CurlCfg<NBUF, NTH>;
  extern __shared__ __align__(128) double sm[];
  double *O = sm + (size_t)NBUF * C::NF * FA_FIELD;
  uint64_t *bar = reinterpret_cast<uint64_t *>(O + (size_t)C::NO * FA_OUT);
  const int tid = threadIdx.x, lane = tid & 31, wrp = tid >> 5;
  const size_t n = (size_t)g.ncell;
  const int ntile = g.nr * g.d[1].nb * g.d[2].nb;
  if (tid == 0) {
    for (int k = 0; k < NBUF; k++) mbar_init(bar + k, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (NBUF == 2 && tid == 0 && (int)blockIdx.x < ntile) curl_stage_tma(g, m, thph_tile(g, blockIdx.x), sm, bar);
  for (int q = blockIdx.x, i = 0; q < ntile; q += gridDim.x, i++) {
    const ThphTile T = thph_tile(g, q);
    const int b = NBUF == 2 ? (i & 1) : 0;
    double *F = sm + (size_t)b * C::NF * FA_FIELD;
    const bool more = q + (int)gridDim.x < ntile;
    if (NBUF == 2) {
      // the next planes into the other buffer: its last readers passed the
      // barrier that ended the previous tile
      if (more && tid == 0) {
        fence_proxy_async();
        curl_stage_tma(g, m, thph_tile(g, q + gridDim.x), sm + (size_t)(b ^ 1) * C::NF * FA_FIELD, bar + (b ^ 1));
      }
    } else if (tid == 0 && i == 0) {
      // the first tile's planes; each later tile's copies start once the
      // previous tile's solves are done with the buffer
      fence_proxy_async();
      curl_stage_tma(g, m, T, F, bar);
    }
    const unsigned parity = NBUF == 2 ? ((unsigned)(i >> 1) & 1u) : ((unsigned)i & 1u);
    const bool late = !mbar_wait_bounded(bar + b, parity, kWaitCycles);
    if (__syncthreads_or(late)) {
      if (tid == 0) {
        atomicOr(flag, kFlagTimeout);
        mbar_wait_bounded(bar + b, parity, kWaitCycles);
        if (NBUF == 2 && more) mbar_wait_bounded(bar + (b ^ 1), (unsigned)((i + 1) >> 1) & 1u, kWaitCycles);
      }
      return;
    }
    // sin(theta) A_phi on the main rows (the theta lines' input)
    double *Fp = F + FA_FIELD;
    for (int k = tid; k < FM * (FM + 8); k += C::NT) {
      const int p = k / (FM + 8), c = k - p * (FM + 8), gt = T.t0 - 4 + c;
      if (gt >= 0 && gt < g.nth) Fp[p * FA_RW + c] *= g.sines[gt];
    }
    __syncthreads();
    if (wrp < 4) {
      const CssDir &DT = g.d[1];
      if (wrp < 2) {  // theta lines (line = phi row p = lane): sin A_phi (ibct 11), A_r (ibct 12)
        const int bdry = g.ibct[wrp == 0 ? 11 : 12];
        const double dn = DT.dnum[T.bt];
        line_solve_r<1, FM>(F + (size_t)(1 + wrp) * FA_FIELD + lane * FA_RW, ThIdx{}, dtype_of(DT, T.bt), bdry, 0.0,
                            0.0, tabp(g, 1, T.bt, 1, bdry), g.tstride, dn, dn, 0, O + wrp * FA_OUT, SwzRow{lane});
      } else {  // phi lines (line = theta column t = lane): A_r, A_theta
        const double dn = g.d[2].dnum[T.bp];
        line_solve_r<1, FM>(F + (size_t)(wrp == 2 ? 2 : 0) * FA_FIELD, PhIdx{lane}, 3, 0, 0.0, 0.0,
                            tabp(g, 2, T.bp, 1, 0), g.tstride, dn, dn, 1, O + wrp * FA_OUT, SwzCol{lane});
      }
    }
    __syncthreads();
    // the stores read only the derivative tiles: with one buffer, the next
    // tile's planes arrive under them
    if (NBUF == 1 && more && tid == 0) {
      fence_proxy_async();
      curl_stage_tma(g, m, thph_tile(g, q + gridDim.x), F, bar);
    }
    const double invr = g.r_inv[T.ir];
    const size_t pl = plane(g, T.ir);
#pragma unroll
    for (int k = 0; k < FM * FM / C::NT; k++) {
      const int pt = tid + k * C::NT, jp = pt >> 5, jt = pt & 31;
      const int it = T.t0 + jt;
      const size_t id = pl + (size_t)(T.p0 + jp) * g.nth + it;
      const double csc = g.csc[it];
      out[id] = invr * swz(O + 2 * FA_OUT, jp, jt) * csc;
      out[n + id] = -swz(O + FA_OUT, jp, jt) * invr;
      const double prev = __dmul_rn(__dmul_rn(swz(O, jp, jt), csc), invr);
      out[2 * n + id] = prev - invr * swz(O + 3 * FA_OUT, jp, jt) * csc;
    }
    __syncthreads();  // the tiles and this buffer are free for the next tiles
  }
}

// ---- k_rstage ----------------------------------------------------------------
// The slab: field f at H + f*FB_FIELD, row rr = 0..39 (r = r0-4+rr), 32
// theta values per row.  Derivative tiles O + k*FB_OUT, row r - r0.  On a
// theta-wall block W holds the zero-datum d(rho)/dtheta rows k_thph left in
// rtw.  Hydro: one tile per CTA, 256 threads, two CTAs per SM (the block
// scheduler keeps the SM's two tiles in different phases, so one's loads
// overlap the other's solves).  MHD, with room for one CTA per SM: 512
// threads, persistent; after the solves each thread holds its points' slab
// values in registers and the next tile's slab arrives under the pointwise
// phases and the stage combination (11.66 -> 10.65 ms a launch on
// 256x512x1024, against one tile per CTA).
constexpr int FB_FIELD = (FM + 8) * FM;
constexpr int FB_OUT = FM * FM;
template <int MAG>
struct RstageCfg {
  static constexpr int NH = MAG ? 7 : 5;  // w v u s rho [bt bp]
  static constexpr int ND = MAG ? 8 : 6;  // dw dv du ds d2s drho0 [dbt dbp]
  static constexpr int NT = MAG ? 512 : 256;  // threads per CTA
  static constexpr int NW = NT / 32;           // warps
  static constexpr int PPT = FM * FM / NT;     // points per thread
  // + the slab's mbarrier
  static constexpr size_t SMEM = 8 * ((size_t)NH * FB_FIELD + (size_t)ND * FB_OUT + FB_OUT + 2 * FM + 1);
};

struct RstageTile {
  int br, bt, ip, r0, t0;
};
__device__ __forceinline__ RstageTile rstage_tile(const CssGeo &g, int q) {
  const int nbt = g.d[1].nb, nbr = g.d[0].nb;
  RstageTile T;
  T.bt = q % nbt;
  const int r = q / nbt;
  T.br = r % nbr;
  T.ip = r / nbr;
  T.r0 = g.d[0].start[T.br];
  T.t0 = g.d[1].start[T.bt];
  return T;
}

// ---- k_curl_rs: the radial parts of B = curl A from a TMA-staged slab ------
// One (r block, theta block, phi) slab per CTA (the tiles of k_rstage):
// A_theta and A_phi over the block's 32 radii with 4-point halos arrive by
// TMA (the slab box of the state buffer's maps) while the threads load the
// theta / phi parts of B that k_curl_pl wrote; r A_theta and r A_phi are
// solved along r (one warp each, one theta column per lane) and
// B_phi += d(r A_theta)/dr / r, B_theta -= d(r A_phi)/dr / r (times dxdr on a
// non-uniform grid), then Compute_B's face zeroing (derivatives.f90:
// 1830-1892) -- the arithmetic of k_curl_r, in the same order.
constexpr int CR_NT = 128;
constexpr int CR_PPT = FM * FM / CR_NT;
constexpr size_t CR_SMEM = 8 * (2 * (size_t)FB_FIELD + 2 * (size_t)FB_OUT + 1);

// Four CTAs per SM (128 registers, 80 bytes spilled): 2.13-2.17 ms per curl
// on MHD 256x512x1024, against 2.30 with three (164 registers), 2.33 with
// six (80 registers, 272 bytes spilled) and 3.07 with six CTAs of 64
// threads that load their B parts after the solves; the two-pass form's
// k_curl_r takes 2.46.
__global__ void __launch_bounds__(CR_NT, 4) k_curl_rs(CssGeo g, double *__restrict__ out,
                                                   const __grid_constant__ SlabMaps ms, int apply_bc, int *flag) {
  extern __shared__ __align__(128) double sm[];
  double *H = sm;                   // 0: A_theta, 1: A_phi, then times r
  double *O = H + 2 * FB_FIELD;     // d/dr of the two lines
  uint64_t *bar = reinterpret_cast<uint64_t *>(O + 2 * FB_OUT);
  const int tid = threadIdx.x, lane = tid & 31, wrp = tid >> 5;
  const size_t n = (size_t)g.ncell;
  const RstageTile T = rstage_tile(g, blockIdx.x);
  const CssDir &D = g.d[0];
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
  }
  __syncthreads();  // the barrier is initialised before anyone waits on it
  if (tid == 0) {
    mbar_expect_tx(bar, 8u * 2 * FB_FIELD);
    tma_load_4d(H, &ms.slab, T.t0, T.ip, T.r0 - 4, 5, bar);
    tma_load_4d(H + FB_FIELD, &ms.slab, T.t0, T.ip, T.r0 - 4, 6, bar);
  }
  // this thread's points (row j = r - r0, theta column lane): the theta
  // and phi parts of B, loaded while the slab arrives
  double in_t[CR_PPT], in_p[CR_PPT], in_r[CR_PPT];
#pragma unroll
  for (int k = 0; k < CR_PPT; k++) {
    const int j = wrp + 4 * k;
    const size_t id = css_idx(g, T.t0 + lane, T.ip, T.r0 + j);
    in_t[k] = out[id];
    in_p[k] = out[n + id];
    in_r[k] = out[2 * n + id];
  }
  if (__syncthreads_or(!mbar_wait_bounded(bar, 0u, kWaitCycles))) {
    if (tid == 0) {
      atomicOr(flag, kFlagTimeout);
      mbar_wait_bounded(bar, 0u, kWaitCycles);
    }
    return;
  }
  for (int idx = tid; idx < 2 * FB_FIELD; idx += CR_NT) {
    const int rr = (idx % FB_FIELD) / FM, gr = T.r0 + rr - 4;
    if (gr >= 0 && gr < g.nr) H[idx] *= g.r_ind[gr];
  }
  __syncthreads();
  if (wrp < 2) {
    const int bdry = g.ibcr[wrp == 0 ? 10 : 11];
    const double dn = D.dnum[T.br];
    line_solve_r<1, FM>(H + (size_t)wrp * FB_FIELD + 4 * FM + lane, StridedIn{FM}, dtype_of(D, T.br), bdry, 0.0, 0.0,
                        tabp(g, 0, T.br, 1, bdry), g.tstride, dn, dn, 0, O + wrp * FB_OUT + lane, StridedOut{FM});
  }
  __syncthreads();
  const int it = T.t0 + lane;
#pragma unroll
  for (int k = 0; k < CR_PPT; k++) {
    const int j = wrp + 4 * k, ir = T.r0 + j;
    const size_t id = css_idx(g, it, T.ip, ir);
    double d = O[j * FM + lane];
    if (g.non_uniform) d = d * g.dxdr[ir];
    double bp_ = in_p[k] + d * g.r_inv[ir];
    d = O[FB_OUT + j * FM + lane];
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

// the slab of tile T [and the wall rows of d(rho)/dtheta] by TMA boxes: per
// field the 40 radial rows r0-4 .. r0+35 of the 32 theta values (zero
// outside [0, nr)), on one mbarrier armed with the byte count
template <int MAG>
__device__ __forceinline__ void rstage_stage_tma(const CssGeo &g, const RstageTile &T, double *H, double *W,
                                                 const SlabMaps &sc, const SlabMaps &sb, const SlabMaps &sw,
                                                 uint64_t *bar) {
  using C = RstageCfg<MAG>;
  const bool lw = g.d[1].lphys[T.bt], hw = g.d[1].rphys[T.bt];
  mbar_expect_tx(bar, 8u * (C::NH * FB_FIELD + ((lw || hw) ? FB_OUT : 0)));
#pragma unroll
  for (int f = 0; f < C::NH; f++) {
    // H order w v u s rho [bt bp]: fields 1 2 3 4 0 of the state, 0 1 of B
    const CUtensorMap *m = f < 5 ? &sc.slab : &sb.slab;
    const int w = f < 4 ? f + 1 : (f == 4 ? 0 : f - 5);
    tma_load_4d(H + (size_t)f * FB_FIELD, m, T.t0, T.ip, T.r0 - 4, w, bar);
  }
  if (lw || hw) tma_load_4d(W, &sw.slab, 0, lw ? 0 : 1, T.ip, T.r0, bar);
}

// STG: the RK4 stage (1..4), compiled in:
//   1: vs = (sld ? vs + dv/6 : dv); nx = v0 + dtcur*dv
//   2,3: vs = vs + dv/3;            nx = v0 + dtcur*dv
//   4: vs + dv/6 accumulated;       nx = v0 + dtcur*(vs + dv/6)  (nx is v0)
template <int MAG, int STG>
__global__ void __launch_bounds__(RstageCfg<MAG>::NT, MAG ? 1 : 2) k_rstage(CssGeo g, const double *__restrict__ cur,
                                                              const double *__restrict__ bf, const double *dv,
                                                              const double *v0, double *vs, double *nx,
                                                              const double *__restrict__ tbuf,
                                                              const double *__restrict__ rtw, double dtcur,
                                                              int *flag, const __grid_constant__ SlabMaps sc,
                                                              const __grid_constant__ SlabMaps sb,
                                                              const __grid_constant__ SlabMaps sw) {
  using C = RstageCfg<MAG>;
  constexpr int nv = MAG ? 8 : 5;
  extern __shared__ __align__(128) double sm[];
  double *H = sm;  // fields of 10240 bytes: every TMA box lands 128-byte aligned
  double *O = H + (size_t)C::NH * FB_FIELD;
  double *W = O + (size_t)C::ND * FB_OUT;
  double *datum = W + FB_OUT;  // [0, 32): radial face datum per line; [32, 64): theta wall datum per row
  uint64_t *bar = reinterpret_cast<uint64_t *>(datum + 2 * FM);
  const CssDir &D = g.d[0], &DT = g.d[1];
  const int tid = threadIdx.x, lane = tid & 31, wrp = tid >> 5;
  const size_t n = (size_t)g.ncell, ps = (size_t)g.nth * g.nphi;
  const int nr = g.nr;
  const bool need_s = !(STG == 1 && !g.sldiffusion);
  int bad = 0;
  // hydro: one tile per CTA (the grid covers the tiles); MHD: persistent,
  // one CTA per SM, the next tile's slab arriving under this tile's
  // pointwise phases
  const int ntile = g.d[0].nb * g.d[1].nb * g.nphi;
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
  }
  __syncthreads();  // the barrier is initialised before anyone waits on it
  for (int q = blockIdx.x, i = 0; q < ntile; q += gridDim.x, i++) {
    const RstageTile T = rstage_tile(g, q);
    const bool more = q + (int)gridDim.x < ntile;
    const size_t base = (size_t)T.ip * g.nth + T.t0;  // (theta t0, phi ip) of plane 0
    // the per-point lines the later phases read, toward L2 now (two
    // 128-byte halves per row): the tendency, T [and B_r], vars0 [and the
    // accumulator]
    {
      const int ns = 6 + (MAG ? 1 : 0) + nv + (need_s ? nv : 0);
      for (int k = tid; k < ns * FM * 2; k += C::NT) {
        const int f = k / (FM * 2), rr = (k >> 1) % FM;
        const double *b;
        if (f < 5) b = dv + (size_t)f * n;
        else if (f == 5) b = tbuf;
        else if (MAG && f == 6) b = bf + 2 * n;
        else {
          const int g2 = f - 6 - (MAG ? 1 : 0);
          b = g2 < nv ? v0 + (size_t)g2 * n : vs + (size_t)(g2 - nv) * n;
        }
        prefetch_l2(b + (size_t)(T.r0 + rr) * ps + base + (k & 1) * 16);
      }
    }
    // ---- the slab: the first tile's copies now, each later tile's issued
    // under the previous tile's pointwise phases (MHD) ----
    const bool lw = DT.lphys[T.bt], hw = DT.rphys[T.bt];
    if (i == 0 && tid == 0) rstage_stage_tma<MAG>(g, T, H, W, sc, sb, sw, bar);
    const unsigned parity = (unsigned)i & 1u;
    if (__syncthreads_or(!mbar_wait_bounded(bar, parity, kWaitCycles))) {
      // copies that never complete: report them and stop, after giving the
      // ones still in flight the same bound to land
      if (tid == 0) {
        atomicOr(flag, kFlagTimeout);
        mbar_wait_bounded(bar, parity, kWaitCycles);
      }
      return;
    }

    // ---- radial solves: tile k = warp, line = lane ----
    const int dtype = dtype_of(D, T.br);
    if (wrp < C::ND) {
      const int var[8] = {2, 3, 4, 5, 5, 1, 7, 8};
      const int k = wrp, l = lane;
      if (!(k == 4 && !g.slaplacian)) {
        const int hk = (k <= 3) ? k : (k == 4 ? 3 : (k == 5 ? 4 : k - 1));
        const double *x = H + (size_t)hk * FB_FIELD + 4 * FM + l;
        const int bdry = g.ibcr[var[k]];
        double lo = 0.0, hi = 0.0;
        if (k == 0 || k == 1) {  // stress-free datum w/r/dxdr (rhs_mpi.f90:578-614)
          if (D.lphys[T.br] && g.bottom_stress_free) lo = x[0] / g.r1 / g.dxdr[0];
          if (D.rphys[T.br]) {
            if (g.top_stress_free) hi = x[(FM - 1) * FM] / g.r2 / g.dxdr[nr - 1];
            else hi = x[(FM - 1) * FM];
          }
        }
        if (k == 3 || k == 4) {  // constant-flux datum (rhs_mpi.f90:584-592, :616-624)
          lo = g.s_flux_lo;
          hi = g.s_flux_hi;
        }
        const double dn = D.dnum[T.br];
        if (k == 4)
          line_solve_r<2, FM>(x, StridedIn{FM}, dtype, bdry, lo, hi, tabp(g, 0, T.br, 2, bdry), g.tstride, dn,
                              dn * dn, 0, O + k * FB_OUT + l, StridedOut{FM});
        else
          line_solve_r<1, FM>(x, StridedIn{FM}, dtype, bdry, lo, hi, tabp(g, 0, T.br, 1, bdry), g.tstride, dn, dn,
                              0, O + k * FB_OUT + l, StridedOut{FM});
      }
    }
    __syncthreads();

    auto gather = [&](int j, int l, RadIn &qq, double t, double brv) {
      const double *hl = H + (size_t)(j + 4) * FM + l;
      const double *ol = O + (size_t)j * FM + l;
      qq.u = hl[2 * FB_FIELD];
      qq.rho = hl[4 * FB_FIELD];
      qq.t = t;
      qq.dw_r = ol[0]; qq.dv_r = ol[FB_OUT]; qq.du_r = ol[2 * FB_OUT]; qq.ds_r = ol[3 * FB_OUT];
      qq.d2s_r = ol[4 * FB_OUT];
      if (MAG) {
        qq.bt = hl[5 * FB_FIELD]; qq.bp = hl[6 * FB_FIELD]; qq.br = brv;
        qq.dbt_r = ol[6 * FB_OUT]; qq.dbp_r = ol[7 * FB_OUT];
      }
    };
    // hydrostatic datum of d(rho)/dr on a physical radial face (rhs_mpi.f90:1750-1768)
    const int phys = D.lphys[T.br] ? 1 : (D.rphys[T.br] ? 2 : 0);
    if (phys) {
      if (tid < FM) {
        const int j = phys == 1 ? 0 : FM - 1, l = tid;
        const size_t id = base + (size_t)(T.r0 + j) * ps + l;
        RadIn qq;
        gather(j, l, qq, __ldg(tbuf + id), MAG ? __ldg(bf + 2 * n + id) : 0.0);
        double drho = __ldg(dv + id), dw = __ldg(dv + n + id), dvv = __ldg(dv + 2 * n + id),
               du = __ldg(dv + 3 * n + id), ds = __ldg(dv + 4 * n + id);
        radial_point<MAG>(g, T.r0 + j, qq, drho, dw, dvv, du, ds);
        double d;
        if (g.lbcr_rho == 4 || g.lbcr_rho == (phys == 1 ? 2 : 3)) d = du * qq.rho * g.invpconst / qq.t;
        else d = qq.rho;
        if (g.non_uniform) d = d / g.dxdr[phys == 1 ? 0 : nr - 1];
        datum[l] = d;
      }
      __syncthreads();
    }

    // MHD: this thread's slab values of the later phases (u rho bt bp w and
    // the wall row), then the slab buffer is free for the next tile's copies
    double hv[C::PPT][6];
    if (MAG) {
#pragma unroll
      for (int h = 0; h < C::PPT; h++) {
        const double *hl = H + (size_t)(wrp + C::NW * h + 4) * FM + lane;
        hv[h][0] = hl[2 * FB_FIELD]; hv[h][1] = hl[4 * FB_FIELD];
        hv[h][2] = hl[5 * FB_FIELD]; hv[h][3] = hl[6 * FB_FIELD];
        hv[h][4] = hl[0];
        hv[h][5] = (lw || hw) ? W[(wrp + C::NW * h) * FM + lane] : 0.0;
      }
      __syncthreads();
      if (more && tid == 0) {
        fence_proxy_async();
        rstage_stage_tma<MAG>(g, rstage_tile(g, q + gridDim.x), H, W, sc, sb, sw, bar);
      }
    }
    // ---- radial pointwise: PPT points per thread (row j = warp + NW h, t = lane) ----
    const double *resp = g.resp_r + (size_t)(2 * T.br + (phys == 2 ? 1 : 0)) * g.tstride;
    double d[C::PPT][5], tk[C::PPT];
    {
      double in[C::PPT][7];
#pragma unroll
      for (int h = 0; h < C::PPT; h++) {
        const size_t id = base + (size_t)(T.r0 + wrp + C::NW * h) * ps + lane;
        in[h][0] = __ldg(dv + id); in[h][1] = __ldg(dv + n + id); in[h][2] = __ldg(dv + 2 * n + id);
        in[h][3] = __ldg(dv + 3 * n + id); in[h][4] = __ldg(dv + 4 * n + id); in[h][5] = __ldg(tbuf + id);
        in[h][6] = MAG ? __ldg(bf + 2 * n + id) : 0.0;
      }
#pragma unroll
      for (int h = 0; h < C::PPT; h++) {
        const int j = wrp + C::NW * h, ir = T.r0 + j;
        RadIn qq;
        if (MAG) {
          const double *ol = O + (size_t)j * FM + lane;
          qq.u = hv[h][0]; qq.rho = hv[h][1]; qq.t = in[h][5];
          qq.dw_r = ol[0]; qq.dv_r = ol[FB_OUT]; qq.du_r = ol[2 * FB_OUT]; qq.ds_r = ol[3 * FB_OUT];
          qq.d2s_r = ol[4 * FB_OUT];
          qq.bt = hv[h][2]; qq.bp = hv[h][3]; qq.br = in[h][6];
          qq.dbt_r = ol[6 * FB_OUT]; qq.dbp_r = ol[7 * FB_OUT];
        } else {
          gather(j, lane, qq, in[h][5], in[h][6]);
        }
        double drho = in[h][0], dw = in[h][1], dvv = in[h][2], du = in[h][3], ds = in[h][4];
        radial_point<MAG>(g, ir, qq, drho, dw, dvv, du, ds);
        double w1 = O[5 * FB_OUT + j * FM + lane];  // Density_Terms_Radial
        if (phys) w1 = w1 + datum[lane] * resp[j + 1];
        if (g.non_uniform) w1 = w1 * g.dxdr[ir];
        drho = drho - qq.u * w1;
        w1 = w1 * (1.0 / qq.rho);
        du = du - g.pconst * qq.t * w1;
        if (phys == 2 && j == FM - 1 && !g.set_stop) {  // rhs_mpi.f90:1807-1818
          drho = drho + qq.rho * (g.t0 - qq.t) / (g.damping_time * (g.gamma - 2.0) * qq.t);
          ds = ds - g.cv * (g.t0 - qq.t) / (g.damping_time * (g.gamma - 2.0) * qq.t);
        }
        d[h][0] = drho; d[h][1] = dw; d[h][2] = dvv; d[h][3] = du; d[h][4] = ds;
        tk[h] = qq.t;
      }
    }

    // ---- Density_Terms_Theta on a theta-wall block (rhs_mpi.f90:1522-1605):
    // the wall datum (rvv dw rho / T on the wall, making dw/dt vanish there)
    // needs the completed dw/dt; d(rho)/dtheta is linear in it: the
    // zero-datum solve from k_thph plus datum times the block's unit
    // response ----
    if (lw || hw) {
      const int tw = lw ? 0 : FM - 1;
      if (lane == tw) {
#pragma unroll
        for (int h = 0; h < C::PPT; h++) {
          const int j = wrp + C::NW * h;
          const double rho = MAG ? hv[h][1] : H[4 * FB_FIELD + (size_t)(j + 4) * FM + tw];
          datum[FM + j] = g.r_ind[T.r0 + j] * g.invpconst * d[h][1] * rho / tk[h];
        }
      }
      __syncthreads();
      const double *rt = g.resp_t + (size_t)(2 * T.bt + (lw ? 0 : 1)) * g.tstride;
      const double rl = rt[lane + 1];
#pragma unroll
      for (int h = 0; h < C::PPT; h++) {
        const int j = wrp + C::NW * h;
        const double w = MAG ? hv[h][4] : H[(size_t)(j + 4) * FM + lane],
                     rho = MAG ? hv[h][1] : H[4 * FB_FIELD + (size_t)(j + 4) * FM + lane];
        double w1 = g.r_inv[T.r0 + j] * ((MAG ? hv[h][5] : W[j * FM + lane]) + datum[FM + j] * rl);
        d[h][0] = d[h][0] - w * w1;
        w1 = w1 * (1.0 / rho);
        d[h][1] = d[h][1] - g.pconst * w1 * tk[h];
      }
    }

    // ---- stage combination (Step_RK4, step_rk4.f90:385-475) and Bound
    // (rhs_mpi.f90:2395-2491).  Every value is read once, before the same
    // thread writes that address (nx is vars0 in stage 4), and no other
    // thread touches it, so the reads go through the non-coherent path and
    // the compiler may start later fields' reads before earlier stores. ----
    const int it = T.t0 + lane;
    const bool twall = (it == 0 || it == g.nth - 1);
#pragma unroll
    for (int h = 0; h < C::PPT; h++)
      if (g.xi_cs < 1.0) d[h][0] = (g.xi_cs * g.xi_cs) * d[h][0];
#pragma unroll
    for (int iv = 0; iv < nv; iv++) {
      double dd[C::PPT], aa[C::PPT], ss[C::PPT];
#pragma unroll
      for (int h = 0; h < C::PPT; h++) {
        const size_t qi = (size_t)iv * n + base + (size_t)(T.r0 + wrp + C::NW * h) * ps + lane;
        dd[h] = (iv < 5) ? d[h][iv < 5 ? iv : 0] : __ldg(dv + qi);
        aa[h] = __ldg(v0 + qi);
        ss[h] = need_s ? __ldg(vs + qi) : 0.0;
      }
#pragma unroll
      for (int h = 0; h < C::PPT; h++) {
        const int ir = T.r0 + wrp + C::NW * h;
        const size_t qi = (size_t)iv * n + base + (size_t)ir * ps + lane;
        const double dd_ = dd[h], a = aa[h];
        double o;
        if (STG == 1) {
          const double sv = g.sldiffusion ? ss[h] + dd_ / 6.0 : dd_;
          vs[qi] = sv;
          o = a + dtcur * dd_;
        } else if (STG == 4) {
          const double sv = ss[h] + dd_ / 6.0;
          o = a + dtcur * sv;
        } else {
          const double sv = ss[h] + dd_ / 3.0;
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
  }
  if (bad && flag) atomicOr(flag, 1);
}

}  // namespace css
