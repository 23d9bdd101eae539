// css_geo.cuh -- device-side description of one CSS run: grid, virtual block
// decomposition, LU tables, radial profiles and physics constants.  Passed
// to every kernel by value (it lands in the kernel parameter bank, so all
// threads read it as uniform constants).
#pragma once
#include <cstddef>

#define CSS_MAXBLK 64   // virtual blocks per direction
#define CSS_MAXM 256    // points per block (the reference's LOOP COUNT MAX is 252)

// One direction's blocks (Partition, parallel_mpi.f90:236-343).
struct CssDir {
  int nb;
  int start[CSS_MAXBLK];
  int size[CSS_MAXBLK];
  unsigned char lphys[CSS_MAXBLK], rphys[CSS_MAXBLK];
  double dnum[CSS_MAXBLK];   // dri / dti / dpi of the block (derivatives.f90:91-97)
  int tab1[CSS_MAXBLK];      // offset of the first-derivative tables
  int tab2[CSS_MAXBLK];      // offset of the second-derivative tables
  int maxm;
};

struct CssGeo {
  int nr, nth, nphi, nv, magnetic, non_uniform;
  long long ncell;
  CssDir d[3];              // 0 = r, 1 = theta, 2 = phi
  int tstride;              // length of one 1-based table array (maxm + 2)
  const double *tab;        // [.. bdry][g1|g2|g3][tstride]
  const int *rblk;          // radial block index of each global ir
  const double *resp_r;     // [r block][lo|hi][tstride]: unit response of d/dr to the face datum of rho
  const double *resp_t;     // [theta block][lo|hi][tstride]: the same for d/dtheta of rho (ibct(1))
  // mixed precision: backgrounds of rho and s about which FP32 stage states
  // are stored, [2][nr][nth] (phi means of the state last uploaded); NULL
  // for FP64 runs
  const double *bg2;
  // radial profiles (length nr)
  const double *r_ind, *r_inv, *dr_ind, *dxdr, *d2xdr2, *rhor, *sr, *grav, *ks, *dlnks, *eps, *dspeed;
  const double *mur, *dlnmu;  // viscosity and its log-derivative (explicit-viscosity path)
  const double *kr, *dlnkr;   // inverse opacity and the reference's dlnkr (radiative diffusion)
  // radiative diffusion: when set, the radial kernel keeps d ln(rho)/dr (after
  // the density datum) and ds/dr of every cell for the radiative pass
  double *rad_lnrho_r, *rad_dsdr;
  int radheat;
  // per-cell SLD speed^2 replacing dspeed (a learned closure's output);
  // NULL, or a negative entry, means the prescribed radial profile
  const double *speed2;
  // theta profiles (length nth)
  const double *sines, *cosines, *theta, *cot, *csc;  // cot = cos/sin, csc = 1/sin
  // SLD cell geometry (diffusion.f90:806-849, :1196-1247, :1316-1351):
  // per theta: sin/cos of the lower and upper faces and the phi geometry
  // factor; per r: 3/(r+^3 - r-^3), the volume-averaged 1/r factor, r-^2, r+^2
  const double *sld_th;  // [5][nth]: sphl, cphl, sphh, cphh, geom
  const double *sld_r;   // [4][nr]:  t3, rfac, rlo^2, rhi^2
  // constants (Initialize_Physics, rhs_mpi.f90:63-75)
  double gamma, gamm1, cp, cv, invcv, invtconst, pconst, invpconst;
  double omega0, t0, damping_time, lumr1, lumr2, r1, r2, dth, dphi, xi_cs;
  int slaplacian, sldiffusion, set_stop;
  int top_stress_free, bottom_stress_free, top_constant_temp, bottom_constant_temp;
  int theta_stress_free, theta_normal_field, theta_perf_conductor;
  int top_radial_field, bottom_radial_field, top_perfect_cond, bottom_perfect_cond;
  int ibcr[13], ibct[13];   // 1-based, as derivatives.f90:50-57
  int lbcr_rho;
  double s_flux_lo, s_flux_hi;  // entropy-gradient datum at constant-flux faces
  // slope-limited diffusion
  double sld_coef, sld_pr, sld_prm;
  double tinyvar[8], inv_tinyvar[8];  // floors of the SLD limiter and their reciprocals
  int nsld, varlist[8];
  int dstype, mass_diffusion, do_viscous_heating, do_ohmic_heating;
  // open radial boundaries (Top_/Bottom_Inflow_Outflow, rhs_mpi.f90:1857-2067)
  int top_inout, bot_inout, bottom_specified, rain;
  double delta_s;
  const double *inout;                  // face scalars of the current RHS (k_inout_scalars)
  const double *dvel_rain, *dent_rain;  // rain fields (nth*nphi)
  const double *ashv;                   // prescribed bottom fields u_r, u_theta, u_phi, s (4 x nth*nphi)
};

// slots of CssGeo::inout
enum {
  IO_TOP_TAU, IO_TOP_MEANU, IO_TOP_MEANS, IO_TOP_MDVEL, IO_TOP_TAUR, IO_TOP_NRAT,
  IO_BOT_TAU, IO_BOT_MEANU, IO_BOT_MEANS, IO_BOT_NRAT, IO_BOT_TCONST, IO_BOT_FEN,
  IO_M0, IO_VOL, IO_MTOT, IO_ASH_FEN_MOD, IO_COUNT
};

__host__ __device__ inline size_t css_idx(const CssGeo &g, int it, int ip, int ir) {
  return (size_t)it + (size_t)g.nth * ((size_t)ip + (size_t)g.nphi * (size_t)ir);
}
