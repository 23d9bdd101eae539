/*
 * css_oracle.c -- TEST INFRASTRUCTURE ONLY: CPU FP64 restatement of the CSS
 * reference hot path, the parity oracle for the B200 library.  See
 * css_oracle.h for what it restates and how it is pinned.  Nothing in the
 * product library links this file; the product fails loudly without its
 * CUDA extension instead of falling back here.
 *
 * Conventions: arrays are the reference's Fortran order vars(it,ip,ir,iv)
 * flattened with 0-based indices, it + nth*(ip + nphi*(ir + nr*iv)).
 * Line work arrays inside the derivative routines are 1-based (element 0
 * unused) so that every statement reads like the Fortran it restates.
 * Every virtual block is one MPI rank of the reference; halos are read from
 * the neighbouring block's part of the global array, which is what the
 * Isend/Irecv exchanges of parallel_mpi.f90:633-696 deliver, because vars1
 * does not change while an RHS runs.
 */
#include "css_oracle.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI 3.1415926535897932384626433832795028841972
#define ONE_OVER_4PI (1.0 / PI / 4.0)
#define ONETHIRD (1.0 / 3.0)
#define A_CONST 7.56577e-15    /* constants.f90:7 */
#define C_LIGHT 2.99792458e10

static __thread char g_err[512];
static void set_err(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}
const char *orc_last_error(void) { return g_err; }

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* ------------------------------------------------------------------------ */
/* context                                                                  */
/* ------------------------------------------------------------------------ */
typedef struct {
  int r0, nr, t0, nt, p0, np;   /* 0-based start and size of the block     */
  int rlo, rhi, tlo, thi;       /* 1 if the face is a physical boundary    */
  int dtype1, dtype2;           /* Determine_Dtype, derivatives.f90:529    */
  double dri, dti, dpi, dri2, dti2, dpi2;
  /* 1-based LU tables per bdry (derivatives.f90:106-287), length n+2     */
  double *g1r[5], *g2r[5], *g3r[5], *h1r[5], *h2r[5], *h3r[5];
  double *g1t[5], *g2t[5], *g3t[5], *h1t[5], *h2t[5], *h3t[5];
  double *g1p, *g2p, *g3p, *h1p, *h2p, *h3p;
} blk_t;

struct orc_ctx {
  css_params p;
  int nr, nth, nphi, nv, ncell;
  double *x_ind, *r_ind, *r_inv, *dr_ind, *dxdr, *d2xdr2, *rhor, *sr, *grav, *ks,
      *dlnks, *eps, *mur, *dlnmu, *kr, *dlnkr;
  double *theta, *phi, *sines, *cosines;
  double dth, dphi;
  int ibcr[13], ibct[13]; /* 1-based as the reference's ibcr/ibct */
  int lbcr_rho;
  int nblk;
  blk_t *blk;
  int *rblk_of; /* radial block index of each global ir */
  double *dspeed; /* diffusion_speed squared per global radius index */
  /* derived constants (Initialize_Physics, rhs_mpi.f90:63-75) */
  double gamm1, cv, invcp, invcv, pconst, invpconst, invtconst;
  /* work arrays */
  double *temperature, *invrho, *maga, *vars2, *vars_save, *dvars1, *vars1, *tmpf, *tmpg, *da;
  /* explicit viscosity: the velocity derivatives the sweeps leave for the
   * cross terms (the reference's vars2 under Laplacian), 6 fields:
   * LAP_W1 ri dw/dth, LAP_V1 ri dv/dth, LAP_U1 ri du/dth,
   * LAP_PV dv/dph/(r sin), LAP_PW dw/dph/(r sin), LAP_PU du/dph/(r sin) */
  double *lap;
  int cond; /* entropy conduction on: Laplacian .or. SLaplacian */
  /* radiative diffusion: rad1 = (4 a c kr / 3) T^3 / rho^2 and rad2 = ds/dr,
   * the reference's dvars2(:,:,:,1:2) under do_radheat */
  double *rad1, *rad2;
  /* open radial boundaries (rhs_mpi.f90:1857-2067): the run's clock (the
   * step index the RHS sees, sim_time, deltat), the mass totals m0, vol,
   * mtot (rhs_mpi.f90:10), the rain fields dvel_rain / dent_rain
   * (entropy_rain.f90:40), the ASH slices and times with the prescribed
   * bottom fields interpolated from them (ashvars, ash_inflow.f90:12-13)
   * and the enthalpy-flux factor ash_fen_mod */
  long long istep;
  double sim_time, deltat, m0, vol, mtot, ash_fen_mod;
  double *dvel_rain, *dent_rain, *ash_slices, *ashv;
  double ash_times[4];
};
enum { LAP_W1 = 0, LAP_V1, LAP_U1, LAP_PV, LAP_PW, LAP_PU, LAP_N };

#define IDX(c, it, ip, ir) ((it) + (c)->nth * ((ip) + (c)->nphi * (size_t)(ir)))
#define FLD(c, a, iv) ((a) + (size_t)(iv) * (c)->ncell)

static double *dalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

/* ------------------------------------------------------------------------ */
/* Initialize_Derivatives tables (derivatives.f90:106-287 for r and theta,  */
/* :172-219 for phi).  lphys/rphys play the roles of (myr1 .eq. 1) and      */
/* (myr2 .eq. nr).                                                          */
/* ------------------------------------------------------------------------ */
static void tables_d1(int m, int lphys, int rphys, double **G1, double **G2, double **G3) {
  for (int iv = 0; iv <= 4; iv++) {
    double *g1 = G1[iv], *g2 = G2[iv], *g3 = G3[iv];
    double alpha = 1.0 / 3.0, a2 = 0.75, g2c = 0.125, a1 = 6.0, b1 = 3.0;
    double cn = 1.0 / (a2 - b1 * g2c);
    double up1 = (a1 * a2 - b1) * cn, up2;
    if ((iv != 1) && (iv != 2)) up2 = 0.0; else up2 = up1;
    if (iv % 2 == 0) up1 = 0.0;
    double c1 = 1.0, c2 = 1.0, c3;
    g1[1] = c2; g2[1] = c2; g3[1] = c2;
    if (lphys) {
      c3 = up1 * c2; g1[2] = c3; c2 = c1 / (c1 - g2c * c3); g2[2] = c2;
      c3 = a2 * c2; g1[3] = c3; c2 = c1 / (c1 - alpha * c3); g2[3] = c2;
      g3[2] = -g2c * g2[2];
    } else {
      c3 = alpha * c2; g1[2] = c3; c2 = c1 / (c1 - alpha * c3); g2[2] = c2;
      g3[2] = -alpha * g2[2];
      c3 = alpha * c2; g1[3] = c3; c2 = c1 / (c1 - alpha * c3); g2[3] = c2;
    }
    for (int ir = 4; ir <= m - 2; ir++) {
      c3 = alpha * c2; g1[ir] = c3; c2 = c1 / (c1 - alpha * c3); g2[ir] = c2;
    }
    for (int ir = 3; ir <= m - 2; ir++) g3[ir] = -alpha * g2[ir];
    if (rphys) {
      c3 = alpha * c2; g1[m - 1] = c3; c2 = c1 / (c1 - a2 * c3); g2[m - 1] = c2;
      c3 = g2c * c2; g1[m] = c3; c2 = c1 / (c1 - up2 * c3); g2[m] = c2;
      g3[m - 1] = -a2 * g2[m - 1];
      g3[m] = -up2 * g2[m];
    } else {
      c3 = alpha * c2; g1[m - 1] = c3; c2 = c1 / (c1 - alpha * c3); g2[m - 1] = c2;
      c3 = alpha * c2; g1[m] = c3; c2 = c1 / (c1 - alpha * c3); g2[m] = c2;
      g3[m - 1] = -alpha * g2[m - 1];
      g3[m] = -alpha * g2[m];
    }
    for (int j = 1; j <= m; j++) g1[j] = -g1[j];
  }
}

static void tables_d2(int m, int lphys, int rphys, double **H1, double **H2, double **H3) {
  for (int iv = 0; iv <= 4; iv++) {
    double *g1 = H1[iv], *g2 = H2[iv], *g3 = H3[iv];
    double alpha = 2.0 / 11.0, up1 = 0, up2 = 0;
    switch (iv) {
      case 0: up1 = 707.0 / 193.0; up2 = 707.0 / 193.0; break;
      case 1: up1 = 137.0 / 13.0; up2 = 137.0 / 13.0; break;
      case 2: up1 = 707.0 / 193.0; up2 = 137.0 / 13.0; break;
      case 3: up1 = 137.0 / 13.0; up2 = 707.0 / 193.0; break;
      case 4: up1 = 707.0 / 193.0; up2 = 707.0 / 193.0; break;
    }
    double a2 = -0.35, g2c = 0.1;
    double c1 = 1.0, c2 = 1.0, c3;
    g1[1] = c2; g2[1] = c2; g3[1] = c2;
    if (lphys) {
      c3 = up1; g1[2] = c3; c2 = c1 / (c1 - g2c * c3); g2[2] = c2;
      c3 = a2 * c2; g1[3] = c3; c2 = c1 / (c1 - alpha * c3); g2[3] = c2;
      g3[2] = -g2c * g2[2];
    } else {
      c3 = alpha * c2; g1[2] = c3; c2 = c1 / (c1 - alpha * c3); g2[2] = c2;
      g3[2] = -alpha * g2[2];
      c3 = alpha * c2; g1[3] = c3; c2 = c1 / (c1 - alpha * c3); g2[3] = c2;
    }
    for (int ir = 4; ir <= m - 2; ir++) {
      c3 = alpha * c2; g1[ir] = c3; c2 = c1 / (c1 - alpha * c3); g2[ir] = c2;
    }
    for (int ir = 3; ir <= m - 2; ir++) g3[ir] = -alpha * g2[ir];
    g2c = a2;
    a2 = 0.1;
    if (rphys) {
      c3 = alpha * c2; g1[m - 1] = c3; c2 = c1 / (c1 - g2c * c3); g2[m - 1] = c2;
      c3 = a2 * c2; g1[m] = c3; c2 = c1 / (c1 - up2 * c3); g2[m] = c2;
      g3[m - 1] = -g2c * g2[m - 1];
      g3[m] = -up2 * g2[m];
    } else {
      c3 = alpha * c2; g1[m - 1] = c3; c2 = c1 / (c1 - alpha * c3); g2[m - 1] = c2;
      c3 = alpha * c2; g1[m] = c3; c2 = c1 / (c1 - alpha * c3); g2[m] = c2;
      g3[m - 1] = -alpha * g2[m - 1];
      g3[m] = -alpha * g2[m];
    }
    for (int j = 1; j <= m; j++) g1[j] = -g1[j];
  }
}

static void tables_p(int m, double alpha, double *g1, double *g2, double *g3) {
  double c1 = 1.0, c2 = 1.0, c3;
  g1[1] = c1; g2[1] = c1; g3[1] = c1;
  c3 = alpha * c2; g1[2] = c3; c2 = c1 / (c1 - alpha * c3); g2[2] = c2;
  g3[2] = -alpha * g2[2];
  for (int ir = 3; ir <= m; ir++) {
    c3 = alpha * c2; g1[ir] = c3; c2 = c1 / (c1 - alpha * c3); g2[ir] = c2;
  }
  for (int ir = 3; ir <= m; ir++) g3[ir] = -alpha * g2[ir];
  for (int j = 1; j <= m; j++) g1[j] = -g1[j];
}

/* ------------------------------------------------------------------------ */
/* Line operators.  x[1..m], b1[1..4] (b1[4] nearest the line), b2[1..4]    */
/* (b2[1] nearest); at a physical end b1[1]/b2[1] carry the boundary datum. */
/* dtype: 1 = halo left/physical right, 2 = physical left/halo right,       */
/* 3 = halo both (Select Case (dtype1), derivatives.f90:564-721).           */
/* dnum is the dri/dti that divides the Neumann datum.                      */
/* ------------------------------------------------------------------------ */
static void thomas(int m, const double *d, const double *g1, const double *g2,
                   const double *g3, double alpha1, double scale, double *out) {
  /* forward/backward sweeps, derivatives.f90:730-795 */
  double t[m + 2];
  double c1 = g3[2], c2 = g3[m - 1], c3 = g3[m];
  t[1] = g2[1] * d[1];
  t[2] = g2[2] * d[2] + c1 * t[1];
  for (int j = 3; j <= m - 2; j++) t[j] = g2[j] * (d[j] + alpha1 * t[j - 1]);
  t[m - 1] = g2[m - 1] * d[m - 1] + c2 * t[m - 2];
  t[m] = g2[m] * d[m] + c3 * t[m - 1];
  out[m] = t[m];
  for (int j = m - 1; j >= 1; j--) out[j] = t[j] + g1[j + 1] * out[j + 1];
  for (int j = 1; j <= m; j++) out[j] = scale * out[j];
}

static void d1_rhs_left_halo(const double *x, const double *b1, double *d) {
  double c1 = -1.0 / 180.0, c2 = 9.0, c3 = 45.0, c4 = 7.0 / 9.0, c5 = 1.0 / 36.0;
  c2 = c1 * c2; c3 = c1 * c3;
  double cnst = -(c3 + c5), beta1 = c4 - c2, alpha1 = c1 + c5;
  c1 = -c1; c4 = -c4;
  d[1] = c1 * b1[1] + c2 * b1[2] + cnst * b1[3] + c4 * b1[4] + c3 * x[1] + beta1 * x[2] + alpha1 * x[3];
  c4 = 7.0 / 9.0; c5 = 1.0 / 36.0;
  d[2] = c4 * (x[3] - x[1]) + c5 * (x[4] - b1[4]);
}

static void d1_rhs_right_halo(const double *x, int m, const double *b2, double *d) {
  double c1 = 7.0 / 9.0, c2 = 1.0 / 36.0, c3 = -1.0 / 180.0, c4 = 9.0, c5 = 45.0;
  d[m - 1] = c1 * (x[m] - x[m - 2]) + c2 * (b2[1] - x[m - 3]);
  double cnst = c2 + c3 * c5, beta1 = c3 * c4 - c1, alpha1 = -(c2 + c3);
  c4 = -c3 * c4; c5 = -c3 * c5;
  d[m] = c1 * b2[1] + cnst * b2[2] + c4 * b2[3] + c3 * b2[4] + beta1 * x[m - 1] + alpha1 * x[m - 2] + c5 * x[m];
}

/* Dbydr / Dbydt body (derivatives.f90:564-795, :1031-1261) */
static void d1_line(const double *x, int m, const double *b1, const double *b2, int dtype, int bdry,
                    double *const *G1, double *const *G2, double *const *G3, double dnum, double scale,
                    double *out) {
  double d[m + 2];
  double c1, c2, c3, c4, c5, alpha2, beta1, cnst;
  switch (dtype) {
    case 1:
      d1_rhs_left_halo(x, b1, d);
      c1 = 43.0 / 96.0; c2 = 5.0 / 6.0; c3 = -9.0 / 8.0; c4 = -1.0 / 6.0; c5 = 1.0 / 96.0;
      d[m - 1] = c1 * x[m] + c2 * x[m - 1] + c3 * x[m - 2] + c4 * x[m - 3] + c5 * x[m - 4];
      if ((bdry == 3) || (bdry == 4)) d[m] = b2[1] / dnum; else d[m] = 0.0;
      if ((bdry == 1) || (bdry == 2)) {
        alpha2 = 0.75; double gamma2 = 0.125; beta1 = 3.0;
        cnst = 1.0 / (alpha2 - beta1 * gamma2);
        alpha2 = alpha2 * cnst; beta1 = -beta1 * cnst;
        c1 = 10.0 / 3.0; c2 = 3.0; c3 = -6.0; c4 = -1.0 / 3.0;
        d[m] = c1 * x[m] + c2 * x[m - 1] + c3 * x[m - 2] + c4 * x[m - 3];
        d[m] = alpha2 * d[m] + beta1 * d[m - 1];
      }
      break;
    case 2:
      if (bdry % 2 == 0) d[1] = b1[1] / dnum;
      if (bdry == 0) d[1] = 0.0;
      c1 = -43.0 / 96.0; c2 = -5.0 / 6.0; c3 = 9.0 / 8.0; c4 = 1.0 / 6.0; c5 = -1.0 / 96.0;
      d[2] = c1 * x[1] + c2 * x[2] + c3 * x[3] + c4 * x[4] + c5 * x[5];
      if ((bdry == 1) || (bdry == 3)) {
        alpha2 = 0.75; double gamma2 = 0.125; beta1 = 3.0;
        cnst = 1.0 / (alpha2 - beta1 * gamma2);
        alpha2 = alpha2 * cnst; beta1 = -beta1 * cnst;
        c1 = -10.0 / 3.0; c2 = -3.0; c3 = 6.0; c4 = 1.0 / 3.0;
        d[1] = c1 * x[1] + c2 * x[2] + c3 * x[3] + c4 * x[4];
        d[1] = alpha2 * d[1] + beta1 * d[2];
      }
      d1_rhs_right_halo(x, m, b2, d);
      break;
    case 0: /* both ends physical: the whole-line extension (no reference
             * block runs it; compact_fd6(dtype=0) and Dbyd1_dt0 do) */
      if (bdry % 2 == 0) d[1] = b1[1] / dnum;
      if (bdry == 0) d[1] = 0.0;
      c1 = -43.0 / 96.0; c2 = -5.0 / 6.0; c3 = 9.0 / 8.0; c4 = 1.0 / 6.0; c5 = -1.0 / 96.0;
      d[2] = c1 * x[1] + c2 * x[2] + c3 * x[3] + c4 * x[4] + c5 * x[5];
      alpha2 = 0.75; beta1 = 3.0;
      cnst = 1.0 / (alpha2 - beta1 * 0.125);
      alpha2 = alpha2 * cnst; beta1 = -beta1 * cnst;
      if ((bdry == 1) || (bdry == 3)) {
        c1 = -10.0 / 3.0; c2 = -3.0; c3 = 6.0; c4 = 1.0 / 3.0;
        d[1] = c1 * x[1] + c2 * x[2] + c3 * x[3] + c4 * x[4];
        d[1] = alpha2 * d[1] + beta1 * d[2];
      }
      c1 = 43.0 / 96.0; c2 = 5.0 / 6.0; c3 = -9.0 / 8.0; c4 = -1.0 / 6.0; c5 = 1.0 / 96.0;
      d[m - 1] = c1 * x[m] + c2 * x[m - 1] + c3 * x[m - 2] + c4 * x[m - 3] + c5 * x[m - 4];
      if ((bdry == 3) || (bdry == 4)) d[m] = b2[1] / dnum; else d[m] = 0.0;
      if ((bdry == 1) || (bdry == 2)) {
        c1 = 10.0 / 3.0; c2 = 3.0; c3 = -6.0; c4 = -1.0 / 3.0;
        d[m] = c1 * x[m] + c2 * x[m - 1] + c3 * x[m - 2] + c4 * x[m - 3];
        d[m] = alpha2 * d[m] + beta1 * d[m - 1];
      }
      break;
    default:
      d1_rhs_left_halo(x, b1, d);
      d1_rhs_right_halo(x, m, b2, d);
      break;
  }
  c4 = 7.0 / 9.0; c5 = 1.0 / 36.0;
  for (int j = 3; j <= m - 2; j++) d[j] = c4 * (x[j + 1] - x[j - 1]) + c5 * (x[j + 2] - x[j - 2]);
  int b = bdry;
  thomas(m, d, G1[b], G2[b], G3[b], -1.0 / 3.0, scale, out);
}

static void d2_rhs_left_halo(const double *x, const double *b1, double *d) {
  double c1 = 12.0 / 11.0, c2 = 3.0 / 44.0, c3 = -1.0 / 990.0, c4 = 2.0, c5 = -27.0, c6 = 270.0, c7 = -490.0;
  d[1] = c3 * (c4 * (b1[1] + x[3]) + c5 * (b1[2] + x[2]) + c6 * (b1[3] + x[1]) + c7 * b1[4]);
  d[1] = d[1] + c1 * (x[2] - 2.0 * x[1] + b1[4]) + c2 * (b1[3] - 2.0 * x[1] + x[3]);
  d[2] = c1 * (x[3] - 2.0 * x[2] + x[1]) + c2 * (b1[4] - 2.0 * x[2] + x[4]);
}

static void d2_rhs_right_halo(const double *x, int m, const double *b2, double *d) {
  double c1 = 12.0 / 11.0, c2 = 3.0 / 44.0, c3 = -1.0 / 990.0, c4 = 2.0, c5 = -27.0, c6 = 270.0, c7 = -490.0;
  d[m - 1] = c1 * (x[m] - 2.0 * x[m - 1] + x[m - 2]) + c2 * (x[m - 3] - 2.0 * x[m - 1] + b2[1]);
  d[m] = c1 * (b2[1] - 2.0 * x[m] + x[m - 1]) + c2 * (x[m - 2] - 2.0 * x[m] + b2[2]);
  d[m] = d[m] + c3 * (c4 * (x[m - 2] + b2[4]) + c5 * (x[m - 1] + b2[3]) + c6 * (x[m] + b2[2]) + c7 * b2[1]);
}

/* D2bydr2 / D2bydt2 body (derivatives.f90:816-1006, :1286-1476).  dnum is
 * the reference's dri in both (D2bydt2 uses dri, not dti, :1322, :1338). */
static void d2_line(const double *x, int m, const double *b1, const double *b2, int dtype, int bdry,
                    double *const *H1, double *const *H2, double *const *H3, double dnum, double scale2, double *out) {
  double d[m + 2];
  double c1, c2, c3, c4, c5, c6;
  switch (dtype) {
    case 1:
      d2_rhs_left_halo(x, b1, d);
      c1 = 1.2375; c2 = -3.0; c3 = 2.325; c4 = -0.6; c5 = 0.0375;
      d[m - 1] = c1 * x[m] + c2 * x[m - 1] + c3 * x[m - 2] + c4 * x[m - 3] + c5 * x[m - 4];
      if ((bdry == 1) || (bdry == 2)) {
        c1 = 1955.0 / 156.0; c2 = -4057.0 / 156.0; c3 = 1117.0 / 78.0; c4 = -55.0 / 78.0;
        c5 = -29.0 / 156.0; c6 = 7.0 / 156.0;
        d[m] = c1 * x[m] + c2 * x[m - 1] + c3 * x[m - 2] + c4 * x[m - 3] + c5 * x[m - 4] + c6 * x[m - 5];
      } else {
        c1 = 575.0 / 193.0 / dnum; c2 = -5827.0 / 2316.0; c3 = 1987.0 / 1158.0; c4 = 465.0 / 386.0;
        c5 = -547.0 / 1158.0; c6 = 157.0 / 2316.0;
        if (bdry == 0) c1 = 0.0;
        d[m] = c1 * b2[1] + c2 * x[m - 1] + c3 * x[m - 2] + c4 * x[m - 3] + c5 * x[m - 4] + c6 * x[m - 5];
      }
      break;
    case 2:
      if (bdry % 2 == 0) {
        c1 = -575.0 / 193.0 / dnum; c2 = -5827.0 / 2316.0; c3 = 1987.0 / 1158.0; c4 = 465.0 / 386.0;
        c5 = -547.0 / 1158.0; c6 = 157.0 / 2316.0;
        if (bdry == 0) c1 = 0.0;
        d[1] = c1 * b1[1] + c2 * x[2] + c3 * x[3] + c4 * x[4] + c5 * x[5] + c6 * x[6];
      } else {
        c1 = 1955.0 / 156.0; c2 = -4057.0 / 156.0; c3 = 1117.0 / 78.0; c4 = -55.0 / 78.0;
        c5 = -29.0 / 156.0; c6 = 7.0 / 156.0;
        d[1] = c1 * x[1] + c2 * x[2] + c3 * x[3] + c4 * x[4] + c5 * x[5] + c6 * x[6];
      }
      c1 = 1.2375; c2 = -3.0; c3 = 2.325; c4 = -0.6; c5 = 0.0375;
      d[2] = c1 * x[1] + c2 * x[2] + c3 * x[3] + c4 * x[4] + c5 * x[5];
      d2_rhs_right_halo(x, m, b2, d);
      break;
    case 0: /* both ends physical (whole-line extension) */
      if (bdry % 2 == 0) {
        c1 = -575.0 / 193.0 / dnum; c2 = -5827.0 / 2316.0; c3 = 1987.0 / 1158.0; c4 = 465.0 / 386.0;
        c5 = -547.0 / 1158.0; c6 = 157.0 / 2316.0;
        if (bdry == 0) c1 = 0.0;
        d[1] = c1 * b1[1] + c2 * x[2] + c3 * x[3] + c4 * x[4] + c5 * x[5] + c6 * x[6];
      } else {
        c1 = 1955.0 / 156.0; c2 = -4057.0 / 156.0; c3 = 1117.0 / 78.0; c4 = -55.0 / 78.0;
        c5 = -29.0 / 156.0; c6 = 7.0 / 156.0;
        d[1] = c1 * x[1] + c2 * x[2] + c3 * x[3] + c4 * x[4] + c5 * x[5] + c6 * x[6];
      }
      c1 = 1.2375; c2 = -3.0; c3 = 2.325; c4 = -0.6; c5 = 0.0375;
      d[2] = c1 * x[1] + c2 * x[2] + c3 * x[3] + c4 * x[4] + c5 * x[5];
      d[m - 1] = c1 * x[m] + c2 * x[m - 1] + c3 * x[m - 2] + c4 * x[m - 3] + c5 * x[m - 4];
      if ((bdry == 1) || (bdry == 2)) {
        c1 = 1955.0 / 156.0; c2 = -4057.0 / 156.0; c3 = 1117.0 / 78.0; c4 = -55.0 / 78.0;
        c5 = -29.0 / 156.0; c6 = 7.0 / 156.0;
        d[m] = c1 * x[m] + c2 * x[m - 1] + c3 * x[m - 2] + c4 * x[m - 3] + c5 * x[m - 4] + c6 * x[m - 5];
      } else {
        c1 = 575.0 / 193.0 / dnum; c2 = -5827.0 / 2316.0; c3 = 1987.0 / 1158.0; c4 = 465.0 / 386.0;
        c5 = -547.0 / 1158.0; c6 = 157.0 / 2316.0;
        if (bdry == 0) c1 = 0.0;
        d[m] = c1 * b2[1] + c2 * x[m - 1] + c3 * x[m - 2] + c4 * x[m - 3] + c5 * x[m - 4] + c6 * x[m - 5];
      }
      break;
    default:
      d2_rhs_left_halo(x, b1, d);
      d2_rhs_right_halo(x, m, b2, d);
      break;
  }
  c1 = 12.0 / 11.0; c2 = 3.0 / 44.0;
  for (int j = 3; j <= m - 2; j++)
    d[j] = c1 * (x[j + 1] - 2.0 * x[j] + x[j - 1]) + c2 * (x[j - 2] - 2.0 * x[j] + x[j + 2]);
  int b = bdry;
  thomas(m, d, H1[b], H2[b], H3[b], -2.0 / 11.0, scale2, out);
}

/* Dbydp (derivatives.f90:1480-1591) and D2bydp2 (:1594-1684) */
static void dp_line(const double *x, int m, const double *b1, const double *b2, int order,
                    const double *g1, const double *g2, double scale, double *out) {
  double d[m + 2], t[m + 2];
  double c1;
  if (order == 1) {
    d1_rhs_left_halo(x, b1, d);
    double c4 = 7.0 / 9.0, c5 = 1.0 / 36.0;
    for (int j = 3; j <= m - 2; j++) d[j] = c4 * (x[j + 1] - x[j - 1]) + c5 * (x[j + 2] - x[j - 2]);
    d1_rhs_right_halo(x, m, b2, d);
    c1 = -1.0 / 3.0;
  } else {
    d2_rhs_left_halo(x, b1, d);
    double c1a = 12.0 / 11.0, c2a = 3.0 / 44.0;
    for (int j = 3; j <= m - 2; j++)
      d[j] = c1a * (x[j + 1] - 2.0 * x[j] + x[j - 1]) + c2a * (x[j - 2] - 2.0 * x[j] + x[j + 2]);
    d2_rhs_right_halo(x, m, b2, d);
    c1 = -2.0 / 11.0;
  }
  t[1] = g2[1] * d[1];
  for (int j = 2; j <= m; j++) t[j] = g2[j] * (d[j] + c1 * t[j - 1]);
  out[m] = t[m];
  for (int j = m - 1; j >= 1; j--) out[j] = t[j] + g1[j + 1] * out[j + 1];
  for (int j = 1; j <= m; j++) out[j] = scale * out[j];
}

/* Dbyd1_dt0 (derivatives.f90:2296-2476): 1D whole-line first derivative   */
static void dbyd1_dt0_line(const double *x0, double *dxdy0, double bdat1, double bdat2, int n1, int ibc) {
  const double *x = x0 - 1;
  double dx[n1 + 2], dtmp[n1 + 2], gam[n1 + 2];
  for (int j = 0; j <= n1 + 1; j++) dx[j] = 0.0;
  double c1 = 7.0 / 9.0, c2 = 1.0 / 36.0, c3, c4, c5;
  if (ibc == 2) dx[1] = bdat1;
  else if (ibc == 3) dx[n1] = bdat2;
  else if (ibc == 4) { dx[1] = bdat1; dx[n1] = bdat2; }
  for (int j = 3; j <= n1 - 2; j++) dx[j] = c1 * (x[j + 1] - x[j - 1]) + c2 * (x[j + 2] - x[j - 2]);
  double alpha = 1.0 / 3.0, alpha2 = 3.0 / 4.0, gamma2 = 1.0 / 8.0, alpha1 = 6.0, beta1 = 3.0;
  double cnst = 1.0 / (alpha2 - beta1 * gamma2);
  double up1 = (alpha1 * alpha2 - beta1) * cnst, up2 = 0.0;
  c1 = -43.0 / 96.0; c2 = -5.0 / 6.0; c3 = 9.0 / 8.0; c4 = 1.0 / 6.0; c5 = -1.0 / 96.0;
  dx[2] = c1 * x[1] + c2 * x[2] + c3 * x[3] + c4 * x[4] + c5 * x[5];
  c1 = -10.0 / 3.0; c2 = -3.0; c3 = 6.0; c4 = 1.0 / 3.0;
  if (ibc == 0) dx[1] = 0.0;
  else if ((ibc == 1) || (ibc == 3)) dx[1] = c1 * x[1] + c2 * x[2] + c3 * x[3] + c4 * x[4];
  if (ibc % 2 != 0) dx[1] = (alpha2 * dx[1] - beta1 * dx[2]) * cnst;
  if (ibc % 2 == 0) up1 = 0.0;
  c1 = -43.0 / 96.0; c2 = -5.0 / 6.0; c3 = 9.0 / 8.0; c4 = 1.0 / 6.0; c5 = -1.0 / 96.0;
  dx[n1 - 1] = -(c1 * x[n1] + c2 * x[n1 - 1] + c3 * x[n1 - 2] + c4 * x[n1 - 3] + c5 * x[n1 - 4]);
  c1 = -10.0 / 3.0; c2 = -3.0; c3 = 6.0; c4 = 1.0 / 3.0;
  if (ibc == 0) dx[n1] = 0.0;
  else if ((ibc == 1) || (ibc == 2)) dx[n1] = -(c1 * x[n1] + c2 * x[n1 - 1] + c3 * x[n1 - 2] + c4 * x[n1 - 3]);
  if ((ibc == 1) || (ibc == 2)) dx[n1] = (alpha2 * dx[n1] - beta1 * dx[n1 - 1]) * cnst;
  if (ibc >= 0) {
    if ((ibc != 1) && (ibc != 2)) up2 = 0.0; else up2 = up1;
  }
  double cc1 = 1.0, cc2 = 1.0, cc3;
  dtmp[1] = dx[1];
  cc3 = up1 * cc2; gam[2] = cc3; cc2 = cc1 / (cc1 - gamma2 * cc3);
  dtmp[2] = (dx[2] - gamma2 * dtmp[1]) * cc2;
  cc3 = alpha2 * cc2; gam[3] = cc3; cc2 = cc1 / (cc1 - alpha * cc3);
  dtmp[3] = (dx[3] - alpha * dtmp[2]) * cc2;
  for (int j = 4; j <= n1 - 2; j++) {
    cc3 = alpha * cc2; gam[j] = cc3; cc2 = cc1 / (cc1 - alpha * cc3);
    dtmp[j] = (dx[j] - alpha * dtmp[j - 1]) * cc2;
  }
  cc3 = alpha * cc2; gam[n1 - 1] = cc3; cc2 = cc1 / (cc1 - alpha2 * cc3);
  dtmp[n1 - 1] = (dx[n1 - 1] - alpha2 * dtmp[n1 - 2]) * cc2;
  cc3 = gamma2 * cc2; gam[n1] = cc3; cc2 = cc1 / (cc1 - up2 * cc3);
  dtmp[n1] = (dx[n1] - up2 * dtmp[n1 - 1]) * cc2;
  dx[n1] = dtmp[n1];
  for (int j = n1 - 1; j >= 1; j--) dx[j] = dtmp[j] - gam[j + 1] * dx[j + 1];
  for (int j = 1; j <= n1; j++) dxdy0[j - 1] = dx[j];
}

int orc_dbyd1_dt0(const double *x, double *dxdy, const double *bdat1, const double *bdat2, int n1,
                  int ibc, int nlines) {
  if (n1 < 14 || ibc < 0 || ibc > 4 || nlines < 0) {
    set_err("orc_dbyd1_dt0: need n1 >= 14 and ibc in 0..4");
    return CSS_ERR_ARG;
  }
#pragma omp parallel for schedule(static)
  for (int l = 0; l < nlines; l++)
    dbyd1_dt0_line(x + (size_t)l * n1, dxdy + (size_t)l * n1, bdat1 ? bdat1[l] : 0.0,
                   bdat2 ? bdat2[l] : 0.0, n1, ibc);
  return CSS_OK;
}

/* Independent lines of n points with explicit closures: lphys/rphys select a
 * physical end (boundary datum bc_lo[l]/bc_hi[l]) or a halo-closed end
 * (halo_lo[4*l..4*l+3] = the 4 points below, farthest first; halo_hi = the 4
 * points above, nearest first).  dx holds d/dx in units of the grid step
 * times scale (scale = dri for a first derivative, dri^2 for a second);
 * dnum divides the Neumann datum as dri does in Dbydr/D2bydr2.  With both
 * ends physical this is compact_fd6(dtype=0) of CSS-Python
 * derivatives.py:32 (up to its dri factor). */
int orc_compact_lines(const double *x, double *dx, int n, int nlines, int order, int lphys, int rphys,
                      int bdry, const double *bc_lo, const double *bc_hi, const double *halo_lo,
                      const double *halo_hi, double dnum, double scale) {
  if (n < 10 || order < 1 || order > 2 || bdry < 0 || bdry > 4) {
    set_err("orc_compact_lines: need n >= 10, order 1|2, bdry 0..4");
    return CSS_ERR_ARG;
  }
  double *G[3][5], *H[3][5];
  for (int i = 0; i < 5; i++)
    for (int k = 0; k < 3; k++) { G[k][i] = dalloc(n + 2); H[k][i] = dalloc(n + 2); }
  tables_d1(n, lphys, rphys, G[0], G[1], G[2]);
  tables_d2(n, lphys, rphys, H[0], H[1], H[2]);
  int dtype = lphys ? (rphys ? 0 : 2) : (rphys ? 1 : 3);
#pragma omp parallel for schedule(static)
  for (int l = 0; l < nlines; l++) {
    double xx[n + 2], b1[5] = {0, 0, 0, 0, 0}, b2[5] = {0, 0, 0, 0, 0}, o[n + 2];
    for (int j = 1; j <= n; j++) xx[j] = x[(size_t)l * n + j - 1];
    if (lphys) b1[1] = bc_lo ? bc_lo[l] : 0.0;
    else for (int k = 1; k <= 4; k++) b1[k] = halo_lo[4 * (size_t)l + k - 1];
    if (rphys) b2[1] = bc_hi ? bc_hi[l] : 0.0;
    else for (int k = 1; k <= 4; k++) b2[k] = halo_hi[4 * (size_t)l + k - 1];
    if (order == 1) d1_line(xx, n, b1, b2, dtype, bdry, G[0], G[1], G[2], dnum, scale, o);
    else d2_line(xx, n, b1, b2, dtype, bdry, H[0], H[1], H[2], dnum, scale, o);
    for (int j = 1; j <= n; j++) dx[(size_t)l * n + j - 1] = o[j];
  }
  for (int i = 0; i < 5; i++)
    for (int k = 0; k < 3; k++) { free(G[k][i]); free(H[k][i]); }
  return CSS_OK;
}

/* ------------------------------------------------------------------------ */
/* Partition (parallel_mpi.f90:236-343)                                     */
/* ------------------------------------------------------------------------ */
static int partition(int n, int nn, int *start, int *size) {
  int base = n / nn;
  if (base < 9) return -1;
  int irem = n % nn;
  if (irem > 0) {
    int d2prev = 0;
    for (int ii = 1; ii <= nn; ii++) {
      int nd = (ii == 1) ? base + 1 : ((ii <= irem) ? base + 1 : base);
      int d1 = (ii == 1) ? 1 : d2prev + 1;
      int d2 = d1 + nd - 1;
      start[ii - 1] = d1 - 1;
      size[ii - 1] = nd;
      d2prev = d2;
    }
  } else {
    for (int ii = 0; ii < nn; ii++) { start[ii] = ii * base; size[ii] = base; }
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* create                                                                   */
/* ------------------------------------------------------------------------ */
static void free_blk(blk_t *b) {
  for (int i = 0; i < 5; i++) {
    free(b->g1r[i]); free(b->g2r[i]); free(b->g3r[i]); free(b->h1r[i]); free(b->h2r[i]); free(b->h3r[i]);
    free(b->g1t[i]); free(b->g2t[i]); free(b->g3t[i]); free(b->h1t[i]); free(b->h2t[i]); free(b->h3t[i]);
  }
  free(b->g1p); free(b->g2p); free(b->g3p); free(b->h1p); free(b->h2p); free(b->h3p);
}

void orc_destroy(orc_ctx *c) {
  if (!c) return;
  for (int i = 0; i < c->nblk; i++) free_blk(&c->blk[i]);
  free(c->blk); free(c->rblk_of);
  free(c->x_ind); free(c->r_ind); free(c->r_inv); free(c->dr_ind); free(c->dxdr); free(c->d2xdr2);
  free(c->rhor); free(c->sr); free(c->grav); free(c->ks); free(c->dlnks); free(c->eps);
  free(c->mur); free(c->dlnmu); free(c->lap); free(c->kr); free(c->dlnkr); free(c->rad1); free(c->rad2);
  free(c->theta); free(c->phi); free(c->sines); free(c->cosines); free(c->dspeed);
  free(c->temperature); free(c->invrho); free(c->maga); free(c->vars2); free(c->vars_save);
  free(c->dvars1); free(c->vars1); free(c->tmpf); free(c->tmpg); free(c->da);
  free(c->dvel_rain); free(c->dent_rain); free(c->ash_slices); free(c->ashv);
  free(c);
}

int orc_create(const css_params *p, const double *prof, orc_ctx **out) {
  *out = NULL;
  if (!p || !prof) { set_err("orc_create: NULL argument"); return CSS_ERR_ARG; }
  if (p->nnr < 2 || p->nnt < 2 || p->nnp < 3) {
    set_err("orc_create: the reference needs nnr>=2, nnt>=2 (no dtype 0 case) and nnp>=3 (phi halos)");
    return CSS_ERR_DECOMP;
  }
  if (p->top_inout || p->bot_inout || p->bottom_specified || p->do_entropy_rain) {
    if (p->magnetic || p->laplacian || p->do_radheat || p->precision) {
      set_err("orc_create: open radial boundaries are restated for hydro FP64 runs without explicit viscosity "
              "or radiative diffusion");
      return CSS_ERR_ARG;
    }
    if ((p->bottom_specified && !p->bot_inout) || (p->do_entropy_rain && !p->top_inout)) {
      set_err("orc_create: bottom_specified needs bot_inout and do_entropy_rain needs top_inout");
      return CSS_ERR_ARG;
    }
  }
  if (p->flux_limiter > 0 || p->ent_flux_limiter > 0 || p->mag_flux_limiter > 0) {
    set_err("orc_create: SLD power flux limiters are not restated (all configs keep them off)");
    return CSS_ERR_ARG;
  }
  orc_ctx *c = (orc_ctx *)calloc(1, sizeof(orc_ctx));
  c->p = *p;
  c->nr = p->nr; c->nth = p->nth; c->nphi = p->nphi;
  c->nv = p->magnetic ? 8 : 5;
  c->ncell = p->nr * p->nth * p->nphi;
  int nr = c->nr, nth = c->nth, nphi = c->nphi;
  double **dst[] = {&c->x_ind, &c->r_ind, &c->dr_ind, &c->dxdr, &c->d2xdr2, &c->rhor,
                    &c->sr,    &c->grav,  &c->ks,     &c->dlnks, &c->eps, &c->mur, &c->dlnmu,
                    &c->kr,    &c->dlnkr};
  for (int k = 0; k < CSS_NPROF; k++) {
    *dst[k] = dalloc(nr);
    memcpy(*dst[k], prof + (size_t)k * nr, sizeof(double) * nr);
  }
  c->r_inv = dalloc(nr);
  for (int i = 0; i < nr; i++) c->r_inv[i] = 1.0 / c->r_ind[i];
  if (!p->non_uniform)
    for (int i = 0; i < nr; i++) { c->dxdr[i] = 1.0; c->d2xdr2[i] = 1.0; }
  /* angles (derivatives.f90:81-89) */
  c->dth = (p->th2 - p->th1) / (double)(nth - 1);
  c->dphi = (p->phi2 - p->phi1) / (double)nphi;
  c->theta = dalloc(nth); c->phi = dalloc(nphi); c->sines = dalloc(nth); c->cosines = dalloc(nth);
  for (int it = 0; it < nth; it++) {
    c->theta[it] = c->dth * (double)it + p->th1;
    c->sines[it] = sin(c->theta[it]);
    c->cosines[it] = cos(c->theta[it]);
  }
  for (int ip = 0; ip < nphi; ip++) c->phi[ip] = c->dphi * (double)ip + p->phi1;

  /* constants (Initialize_Physics, rhs_mpi.f90:63-75; Read_Input :1286-1287) */
  c->gamm1 = p->gamma - 1.0;
  c->cv = p->cp / p->gamma;
  c->invcp = 1.0 / p->cp;
  c->invcv = 1.0 / c->cv;
  c->pconst = c->gamm1 * p->cp;
  c->invpconst = c->invcp / c->gamm1;
  c->invtconst = c->invcv / c->gamm1;

  /* BC integers (Read_Input, mhdsph_mpi.f90:1317-1461) */
  int lbcr_v, lbcr_s, lbcr_u = p->top_inout ? 3 : 1, lbcr_rho = 4, lbcr_t = 4; /* mhdsph_mpi.f90:1355-1359 */
  int tn = !p->top_stress_free, bn = !p->bottom_stress_free;
  if (tn && bn) lbcr_v = 1;
  else if (tn && !bn) lbcr_v = 2;
  else if (!tn && bn) lbcr_v = 3;
  else lbcr_v = 4;
  int tt = p->top_constant_temp, bt = p->bottom_constant_temp;
  if (tt && bt) lbcr_s = 1;
  else if (tt && !bt) lbcr_s = 2;
  else if (!tt && bt) lbcr_s = 3;
  else lbcr_s = 4;
  int lbct_rho = 4, lbct_t = 0, lbct_w = 1, lbct_u = p->theta_stress_free ? 0 : 1, lbct_v = 4, lbct_s = 0;
  int lbcr_br = 0, lbcr_bt = 0, lbcr_bp = 0, lbcr_ar = 0, lbcr_at = 0, lbcr_ap = 0;
  int lbct_br = 0, lbct_bt = 0, lbct_bp = 0, lbct_ar = 0, lbct_at = 0, lbct_ap = 0;
  if (p->magnetic) {
    if (p->top_radial_field && p->bottom_radial_field) {
      lbcr_br = 4; lbcr_bt = 1; lbcr_bp = 1; lbcr_ar = 1; lbcr_at = 0; lbcr_ap = 0;
    }
    if (p->top_perfect_cond && p->bottom_perfect_cond) {
      lbcr_br = 1; lbcr_bt = 1; lbcr_bp = 1; lbcr_ar = 1; lbcr_at = 1; lbcr_ap = 1;
    }
    if (p->theta_normal_field) {
      lbct_br = 1; lbct_bt = 4; lbct_bp = 1; lbct_ar = 0; lbct_at = 1; lbct_ap = 0;
    }
    if (p->theta_perf_conductor) {
      lbct_br = 1; lbct_bt = 1; lbct_bp = 1; lbct_ar = 1; lbct_at = 1; lbct_ap = 1;
    }
  }
  /* ibcr/ibct (derivatives.f90:50-57) */
  int ir_[13] = {0, lbcr_rho, lbcr_v, lbcr_v, lbcr_u, lbcr_s, lbcr_t,
                 lbcr_bt, lbcr_bp, lbcr_br, lbcr_at, lbcr_ap, lbcr_ar};
  int it_[13] = {0, lbct_rho, lbct_w, lbct_v, lbct_u, lbct_s, lbct_t,
                 lbct_bt, lbct_bp, lbct_br, lbct_at, lbct_ap, lbct_ar};
  memcpy(c->ibcr, ir_, sizeof ir_);
  memcpy(c->ibct, it_, sizeof it_);
  c->lbcr_rho = lbcr_rho;

  /* virtual blocks */
  int rs[64], rn[64], ts[64], tn_[64], ps[64], pn[64];
  if (p->nnr > 64 || p->nnt > 64 || p->nnp > 64 || partition(nr, p->nnr, rs, rn) ||
      partition(nth, p->nnt, ts, tn_) || partition(nphi, p->nnp, ps, pn)) {
    set_err("orc_create: fewer than 9 points per block (parallel_mpi.f90:250-315)");
    orc_destroy(c);
    return CSS_ERR_DECOMP;
  }
  for (int i = 0; i < p->nnr; i++) if (rn[i] % 2 || rn[i] < 10) goto odd;
  for (int i = 0; i < p->nnt; i++) if (tn_[i] % 2 || tn_[i] < 10) goto odd;
  for (int i = 0; i < p->nnp; i++) if (pn[i] % 2 || pn[i] < 10) goto odd;
  goto even;
odd:
  set_err("orc_create: block sizes must be even and >= 10 (the reference's paired sweeps "
          "read an unset row for odd sizes, derivatives.f90:755-792)");
  orc_destroy(c);
  return CSS_ERR_DECOMP;
even:
  c->nblk = p->nnr * p->nnt * p->nnp;
  c->blk = (blk_t *)calloc(c->nblk, sizeof(blk_t));
  c->rblk_of = (int *)calloc(nr, sizeof(int));
  for (int ib = 0; ib < p->nnr; ib++)
    for (int j = rs[ib]; j < rs[ib] + rn[ib]; j++) c->rblk_of[j] = ib;
  int k = 0;
  for (int ib = 0; ib < p->nnr; ib++)
    for (int jb = 0; jb < p->nnt; jb++)
      for (int kb = 0; kb < p->nnp; kb++, k++) {
        blk_t *b = &c->blk[k];
        b->r0 = rs[ib]; b->nr = rn[ib]; b->t0 = ts[jb]; b->nt = tn_[jb]; b->p0 = ps[kb]; b->np = pn[kb];
        b->rlo = (ib == 0); b->rhi = (ib == p->nnr - 1);
        b->tlo = (jb == 0); b->thi = (jb == p->nnt - 1);
        b->dtype1 = b->rlo ? 2 : (b->rhi ? 1 : 3);
        b->dtype2 = b->tlo ? 2 : (b->thi ? 1 : 3);
        int myr1 = b->r0, myr2 = b->r0 + b->nr - 1;
        int myt1 = b->t0, myt2 = b->t0 + b->nt - 1;
        int myp1 = b->p0, myp2 = b->p0 + b->np - 1;
        b->dri = 1.0 / (c->x_ind[myr2] - c->x_ind[myr1]);
        b->dti = 1.0 / (c->theta[myt2] - c->theta[myt1]);
        b->dpi = 1.0 / (c->phi[myp2] - c->phi[myp1]);
        b->dri = (double)(b->nr - 1) * b->dri;
        b->dti = (double)(b->nt - 1) * b->dti;
        b->dpi = (double)(b->np - 1) * b->dpi;
        b->dri2 = b->dri * b->dri; b->dti2 = b->dti * b->dti; b->dpi2 = b->dpi * b->dpi;
        for (int i = 0; i < 5; i++) {
          b->g1r[i] = dalloc(b->nr + 2); b->g2r[i] = dalloc(b->nr + 2); b->g3r[i] = dalloc(b->nr + 2);
          b->h1r[i] = dalloc(b->nr + 2); b->h2r[i] = dalloc(b->nr + 2); b->h3r[i] = dalloc(b->nr + 2);
          b->g1t[i] = dalloc(b->nt + 2); b->g2t[i] = dalloc(b->nt + 2); b->g3t[i] = dalloc(b->nt + 2);
          b->h1t[i] = dalloc(b->nt + 2); b->h2t[i] = dalloc(b->nt + 2); b->h3t[i] = dalloc(b->nt + 2);
        }
        tables_d1(b->nr, b->rlo, b->rhi, b->g1r, b->g2r, b->g3r);
        tables_d2(b->nr, b->rlo, b->rhi, b->h1r, b->h2r, b->h3r);
        tables_d1(b->nt, b->tlo, b->thi, b->g1t, b->g2t, b->g3t);
        tables_d2(b->nt, b->tlo, b->thi, b->h1t, b->h2t, b->h3t);
        b->g1p = dalloc(b->np + 2); b->g2p = dalloc(b->np + 2); b->g3p = dalloc(b->np + 2);
        b->h1p = dalloc(b->np + 2); b->h2p = dalloc(b->np + 2); b->h3p = dalloc(b->np + 2);
        tables_p(b->np, 1.0 / 3.0, b->g1p, b->g2p, b->g3p);
        tables_p(b->np, 2.0 / 11.0, b->h1p, b->h2p, b->h3p);
      }

  /* SLD speed profile (Initialize_Diffusion, diffusion.f90:51-61): one value
   * per global radius, speed(r) = [0.5*(speedh*(rho/rho_top)^exp + speedr)
   * *(1 + tanh(c*(r - r_cut)/(r2 - r1)))]^2.  Block ghost entries are never
   * used (the ghosts of vcc are rebuilt from neighbours or copied).         */
  c->dspeed = dalloc(nr);
  for (int i = 0; i < nr; i++) {
    double ds = p->sld_speedh * pow(c->rhor[i] / c->rhor[nr - 1], p->sld_exp) + p->sld_speedr;
    ds = 0.5 * ds * (1.0 + tanh(p->sld_tanh_coef * (c->r_ind[i] - p->flux_cutoff) / (p->r2 - p->r1)));
    c->dspeed[i] = ds * ds;
  }

  size_t n = (size_t)c->ncell;
  c->temperature = dalloc(n); c->invrho = dalloc(n); c->maga = dalloc(3 * n);
  c->vars2 = dalloc(n * c->nv); c->vars_save = dalloc(n * c->nv);
  c->dvars1 = dalloc(n * c->nv); c->vars1 = dalloc(n * c->nv);
  c->tmpf = dalloc(n); c->tmpg = dalloc(n);
  if (p->magnetic) c->da = dalloc(3 * n);
  if (p->laplacian) c->lap = dalloc(n * LAP_N);
  if (p->do_radheat) { c->rad1 = dalloc(n); c->rad2 = dalloc(n); }
  c->cond = p->slaplacian || p->laplacian;
  if (p->top_inout || p->bot_inout) {
    size_t np = (size_t)nth * nphi;
    c->dvel_rain = dalloc(np); c->dent_rain = dalloc(np);
    c->ash_slices = dalloc(16 * np); c->ashv = dalloc(4 * np);
  }
  *out = c;
  return CSS_OK;
}

/* ------------------------------------------------------------------------ */
/* Halo gather.  dir 0 (r): line at fixed (it=a, ip=q); dir 1 (theta):     */
/* fixed (ip=a, ir=q); dir 2 (phi): fixed (it=a, ir=q).  Returns x[1..m],   */
/* b1[1..4], b2[1..4]; at a physical face b1[1]/b2[1] = bclo/bchi.          */
/* ------------------------------------------------------------------------ */
static void gather(const orc_ctx *c, const blk_t *b, int dir, const double *f, int a, int q,
                   double bclo, double bchi, double *x, double *b1, double *b2) {
  int m;
  for (int k = 1; k <= 4; k++) { b1[k] = 0.0; b2[k] = 0.0; }
  if (dir == 0) {
    m = b->nr;
    for (int j = 1; j <= m; j++) x[j] = f[IDX(c, a, q, b->r0 + j - 1)];
    if (b->rlo) b1[1] = bclo;
    else for (int k = 1; k <= 4; k++) b1[k] = f[IDX(c, a, q, b->r0 - 5 + k)];
    if (b->rhi) b2[1] = bchi;
    else for (int k = 1; k <= 4; k++) b2[k] = f[IDX(c, a, q, b->r0 + m + k - 1)];
  } else if (dir == 1) {
    m = b->nt;
    for (int j = 1; j <= m; j++) x[j] = f[IDX(c, b->t0 + j - 1, a, q)];
    if (b->tlo) b1[1] = bclo;
    else for (int k = 1; k <= 4; k++) b1[k] = f[IDX(c, b->t0 - 5 + k, a, q)];
    if (b->thi) b2[1] = bchi;
    else for (int k = 1; k <= 4; k++) b2[k] = f[IDX(c, b->t0 + m + k - 1, a, q)];
  } else {
    int np = c->nphi;
    m = b->np;
    for (int j = 1; j <= m; j++) x[j] = f[IDX(c, a, b->p0 + j - 1, q)];
    for (int k = 1; k <= 4; k++) {
      b1[k] = f[IDX(c, a, (b->p0 - 5 + k + np) % np, q)];
      b2[k] = f[IDX(c, a, (b->p0 + m + k - 1) % np, q)];
    }
  }
}

/* derivative of field f along dir on block b for the line (a, q); out[1..m].
 * For dir 1 the D2 Neumann datum is divided by the dri of the radial block
 * holding radius q (the D2bydt2 quirk).                                      */
static void line_deriv(const orc_ctx *c, const blk_t *b, int dir, int order, const double *f, int a,
                       int q, int bdry, double bclo, double bchi, double *out) {
  int m = dir == 0 ? b->nr : (dir == 1 ? b->nt : b->np);
  double x[m + 2], b1[5], b2[5];
  gather(c, b, dir, f, a, q, bclo, bchi, x, b1, b2);
  if (dir == 0) {
    if (order == 1) d1_line(x, m, b1, b2, b->dtype1, bdry, b->g1r, b->g2r, b->g3r, b->dri, b->dri, out);
    else d2_line(x, m, b1, b2, b->dtype1, bdry, b->h1r, b->h2r, b->h3r, b->dri, b->dri2, out);
  } else if (dir == 1) {
    if (order == 1) d1_line(x, m, b1, b2, b->dtype2, bdry, b->g1t, b->g2t, b->g3t, b->dti, b->dti, out);
    else {
      /* dri of the rank that owns this r-plane */
      const blk_t *rb = NULL;
      for (int i = 0; i < c->nblk; i++)
        if (c->blk[i].r0 <= q && q < c->blk[i].r0 + c->blk[i].nr) { rb = &c->blk[i]; break; }
      d2_line(x, m, b1, b2, b->dtype2, bdry, b->h1t, b->h2t, b->h3t, rb->dri, b->dti2, out);
    }
  } else {
    if (order == 1) dp_line(x, m, b1, b2, 1, b->g1p, b->g2p, b->dpi, out);
    else dp_line(x, m, b1, b2, 2, b->h1p, b->h2p, b->dpi2, out);
  }
}

int orc_deriv(orc_ctx *c, int dir, int order, const double *x, double *dx, const double *bc_lo,
              const double *bc_hi, int bdry) {
  if (dir < 0 || dir > 2 || order < 1 || order > 2 || bdry < 0 || bdry > 4) {
    set_err("orc_deriv: bad dir/order/bdry");
    return CSS_ERR_ARG;
  }
  int nth = c->nth, nphi = c->nphi;
  for (int k = 0; k < c->nblk; k++) {
    const blk_t *b = &c->blk[k];
    if (dir == 0) {
#pragma omp parallel for collapse(2) schedule(static)
      for (int ip = b->p0; ip < b->p0 + b->np; ip++)
        for (int it = b->t0; it < b->t0 + b->nt; it++) {
          double o[b->nr + 2];
          double lo = bc_lo ? bc_lo[it + nth * ip] : 0.0, hi = bc_hi ? bc_hi[it + nth * ip] : 0.0;
          line_deriv(c, b, 0, order, x, it, ip, bdry, lo, hi, o);
          for (int j = 1; j <= b->nr; j++) dx[IDX(c, it, ip, b->r0 + j - 1)] = o[j];
        }
    } else if (dir == 1) {
#pragma omp parallel for collapse(2) schedule(static)
      for (int ir = b->r0; ir < b->r0 + b->nr; ir++)
        for (int ip = b->p0; ip < b->p0 + b->np; ip++) {
          double o[b->nt + 2];
          double lo = bc_lo ? bc_lo[ip + nphi * ir] : 0.0, hi = bc_hi ? bc_hi[ip + nphi * ir] : 0.0;
          line_deriv(c, b, 1, order, x, ip, ir, bdry, lo, hi, o);
          for (int j = 1; j <= b->nt; j++) dx[IDX(c, b->t0 + j - 1, ip, ir)] = o[j];
        }
    } else {
#pragma omp parallel for collapse(2) schedule(static)
      for (int ir = b->r0; ir < b->r0 + b->nr; ir++)
        for (int it = b->t0; it < b->t0 + b->nt; it++) {
          double o[b->np + 2];
          line_deriv(c, b, 2, order, x, it, ir, 0, 0.0, 0.0, o);
          for (int j = 1; j <= b->np; j++) dx[IDX(c, it, b->p0 + j - 1, ir)] = o[j];
        }
    }
  }
  return CSS_OK;
}

/* ------------------------------------------------------------------------ */
/* VectorCurlA (derivatives.f90:2106-2294) + Compute_B zeroing (:1842-1883) */
/* a: A_theta, A_phi, A_r (3 fields); b: B_theta, B_phi, B_r.               */
/* ------------------------------------------------------------------------ */
static void vector_curl_a(orc_ctx *c, const double *a, double *b) {
  int nth = c->nth, nphi = c->nphi, nr = c->nr;
  size_t n = c->ncell;
  const double *at = a, *ap = a + n, *ar = a + 2 * n;
  double *bt = b, *bp = b + n, *br = b + 2 * n;
  double *f = c->tmpf;
  /* theta sweep: B_r = d(sin A_phi)/dtheta/(r sin); B_phi = -dA_r/dtheta/r */
  for (size_t i = 0; i < n; i++) f[i] = c->sines[i % nth] * ap[i];
  for (int k = 0; k < c->nblk; k++) {
    const blk_t *B = &c->blk[k];
#pragma omp parallel for collapse(2) schedule(static)
    for (int ir = B->r0; ir < B->r0 + B->nr; ir++)
      for (int ip = B->p0; ip < B->p0 + B->np; ip++) {
        double o[B->nt + 2];
        double invr = c->r_inv[ir];
        line_deriv(c, B, 1, 1, f, ip, ir, c->ibct[11], 0.0, 0.0, o);
        for (int j = 1; j <= B->nt; j++) {
          int it = B->t0 + j - 1;
          br[IDX(c, it, ip, ir)] = o[j] * (1.0 / c->sines[it]) * invr;
        }
        line_deriv(c, B, 1, 1, ar, ip, ir, c->ibct[12], 0.0, 0.0, o);
        for (int j = 1; j <= B->nt; j++) bp[IDX(c, B->t0 + j - 1, ip, ir)] = -o[j] * invr;
      }
  }
  /* phi sweep */
  for (int k = 0; k < c->nblk; k++) {
    const blk_t *B = &c->blk[k];
#pragma omp parallel for collapse(2) schedule(static)
    for (int ir = B->r0; ir < B->r0 + B->nr; ir++)
      for (int it = B->t0; it < B->t0 + B->nt; it++) {
        double o[B->np + 2];
        double invr = c->r_inv[ir], csc = 1.0 / c->sines[it];
        line_deriv(c, B, 2, 1, ar, it, ir, 0, 0.0, 0.0, o);
        for (int j = 1; j <= B->np; j++) bt[IDX(c, it, B->p0 + j - 1, ir)] = invr * o[j] * csc;
        line_deriv(c, B, 2, 1, at, it, ir, 0, 0.0, 0.0, o);
        for (int j = 1; j <= B->np; j++) {
          size_t id = IDX(c, it, B->p0 + j - 1, ir);
          br[id] = br[id] - invr * o[j] * csc;
        }
      }
  }
  /* r sweep: B_phi += d(r A_theta)/dr / r, B_theta -= d(r A_phi)/dr / r */
  double *g = c->tmpg;
  for (int ir = 0; ir < nr; ir++)
    for (int ip = 0; ip < nphi; ip++)
      for (int it = 0; it < nth; it++) {
        size_t id = IDX(c, it, ip, ir);
        f[id] = c->r_ind[ir] * at[id];
        g[id] = c->r_ind[ir] * ap[id];
      }
  for (int k = 0; k < c->nblk; k++) {
    const blk_t *B = &c->blk[k];
#pragma omp parallel for collapse(2) schedule(static)
    for (int ip = B->p0; ip < B->p0 + B->np; ip++)
      for (int it = B->t0; it < B->t0 + B->nt; it++) {
        double o[B->nr + 2];
        line_deriv(c, B, 0, 1, f, it, ip, c->ibcr[10], 0.0, 0.0, o);
        for (int j = 1; j <= B->nr; j++) {
          int ir = B->r0 + j - 1;
          double d = o[j];
          if (c->p.non_uniform) d = d * c->dxdr[ir];
          size_t id = IDX(c, it, ip, ir);
          bp[id] = bp[id] + d * c->r_inv[ir];
        }
        line_deriv(c, B, 0, 1, g, it, ip, c->ibcr[11], 0.0, 0.0, o);
        for (int j = 1; j <= B->nr; j++) {
          int ir = B->r0 + j - 1;
          double d = o[j];
          if (c->p.non_uniform) d = d * c->dxdr[ir];
          size_t id = IDX(c, it, ip, ir);
          bt[id] = bt[id] - d * c->r_inv[ir];
        }
      }
  }
}

static void compute_b_bc(orc_ctx *c, double *b) {
  int nth = c->nth, nphi = c->nphi, nr = c->nr;
  size_t n = c->ncell;
  double *bt = b, *bp = b + n, *br = b + 2 * n;
  for (int ir = 0; ir < nr; ir++)
    for (int ip = 0; ip < nphi; ip++) {
      if (c->p.theta_perf_conductor) {
        bt[IDX(c, 0, ip, ir)] = 0.0;
        bt[IDX(c, nth - 1, ip, ir)] = 0.0;
      } else {
        bp[IDX(c, 0, ip, ir)] = 0.0; br[IDX(c, 0, ip, ir)] = 0.0;
        bp[IDX(c, nth - 1, ip, ir)] = 0.0; br[IDX(c, nth - 1, ip, ir)] = 0.0;
      }
    }
  for (int ip = 0; ip < nphi; ip++)
    for (int it = 0; it < nth; it++) {
      size_t lo = IDX(c, it, ip, 0), hi = IDX(c, it, ip, nr - 1);
      if (c->p.bottom_radial_field) { bt[lo] = 0.0; bp[lo] = 0.0; }
      else if (c->p.bottom_perfect_cond) br[lo] = 0.0;
      if (c->p.top_radial_field) { bt[hi] = 0.0; bp[hi] = 0.0; }
      else if (c->p.top_perfect_cond) br[hi] = 0.0;
    }
}

int orc_curl_b(orc_ctx *c, const double *a, double *b) {
  if (!c->p.magnetic) { set_err("orc_curl_b: hydro context"); return CSS_ERR_ARG; }
  vector_curl_a(c, a, b);
  compute_b_bc(c, b);
  return CSS_OK;
}

/* ------------------------------------------------------------------------ */
/* RHS (rhs_mpi.f90:279-783)                                                */
/* ------------------------------------------------------------------------ */
#define TWOTHIRDS (2.0 / 3.0)
#define FOURTHIRDS (4.0 / 3.0)
#define SEVENTHIRDS (7.0 / 3.0)

static void source_theta_terms(orc_ctx *c, const blk_t *B, const double *v1, double *dv1) {
  const css_params *p = &c->p;
  int mag = p->magnetic, lapl = p->laplacian;
  size_t n = c->ncell;
  const double *rhoF = v1, *wF = v1 + n, *vF = v1 + 2 * n, *uF = v1 + 3 * n, *sF = v1 + 4 * n;
  double om2 = 2.0 * p->omega_0;
#pragma omp parallel for collapse(2) schedule(static)
  for (int ir = B->r0; ir < B->r0 + B->nr; ir++)
    for (int ip = B->p0; ip < B->p0 + B->np; ip++) {
      int m = B->nt, t0 = B->t0, nth = c->nth;
      double ri = c->r_inv[ir], rv = c->r_ind[ir], epsr = c->eps[ir];
      double omsq = rv * p->omega_0 * p->omega_0;
      double dw[m + 2], du[m + 2], dvv[m + 2], drho[m + 2], ds[m + 2], w1[m + 2];
      double lo, hi;
#define PT(F, j) F[IDX(c, t0 + (j)-1, ip, ir)]
#define SN(j) c->sines[t0 + (j)-1]
#define CS(j) c->cosines[t0 + (j)-1]
#define CT(j) (c->cosines[t0 + (j)-1] / c->sines[t0 + (j)-1])
#define CSC2(j) (1.0 / (c->sines[t0 + (j)-1] * c->sines[t0 + (j)-1]))
      for (int j = 1; j <= m; j++) {
        double rho = PT(rhoF, j), w = PT(wF, j);
        dw[j] = omsq * SN(j) * CS(j);
        du[j] = -c->grav[ir] + omsq * SN(j) * SN(j);
        drho[j] = -rho * w * CT(j) * ri;
        dvv[j] = -om2 * CS(j) * w;
        du[j] = du[j] + ri * w * w;
      }
      /* dw/dtheta: BC data slot of w is never set (lbct_w = 1, unused) */
      line_deriv(c, B, 1, 1, wF, ip, ir, c->ibct[2], 0.0, 0.0, w1);
      for (int j = 1; j <= m; j++) {
        double rho = PT(rhoF, j), w = PT(wF, j);
        w1[j] = w1[j] * ri;
        drho[j] = drho[j] - rho * w1[j];
        dw[j] = dw[j] - w * w1[j];
      }
      /* explicit viscosity, w terms (rhs_mpi.f90:844-862); mu6 = mur/rho */
      double mu6[m + 2], o2[m + 2];
      if (lapl) {
        double dlm = c->dlnmu[ir];
        for (int j = 1; j <= m; j++) {
          size_t id = IDX(c, t0 + j - 1, ip, ir);
          double w = PT(wF, j);
          mu6[j] = c->mur[ir] * c->invrho[id];
          double ddiff = -FOURTHIRDS * ri * ri;
          dw[j] = dw[j] + (ddiff * CSC2(j) - ri * dlm) * mu6[j] * w;
          c->lap[LAP_W1 * n + id] = w1[j];
          double t1 = w1[j] * mu6[j];
          ddiff = -ONETHIRD * (7.0 * ri + 2.0 * dlm);
          du[j] = du[j] + ddiff * (ri * mu6[j] * CT(j) * w + t1);
          ddiff = FOURTHIRDS * ri;
          dw[j] = dw[j] + ddiff * CT(j) * t1;
        }
        line_deriv(c, B, 1, 2, wF, ip, ir, c->ibct[2], 0.0, 0.0, o2);
        for (int j = 1; j <= m; j++) dw[j] = dw[j] + FOURTHIRDS * ri * ri * mu6[j] * o2[j];
      }
      for (int j = 1; j <= m; j++) {
        double w = PT(wF, j), v = PT(vF, j);
        dw[j] = dw[j] + v * (ri * CT(j) * v + om2 * CS(j));
        dvv[j] = dvv[j] - ri * v * w * CT(j);
        du[j] = du[j] + v * (ri * v + om2 * SN(j));
      }
      /* dv/dtheta with the stress-free datum cot(theta)*v (rhs_mpi.f90:414, :444) */
      lo = (c->cosines[0] / c->sines[0]) * vF[IDX(c, 0, ip, ir)];
      hi = (c->cosines[nth - 1] / c->sines[nth - 1]) * vF[IDX(c, nth - 1, ip, ir)];
      line_deriv(c, B, 1, 1, vF, ip, ir, c->ibct[3], lo, hi, w1);
      for (int j = 1; j <= m; j++) {
        w1[j] = w1[j] * ri;
        dvv[j] = dvv[j] - PT(wF, j) * w1[j];
      }
      /* explicit viscosity, v terms (rhs_mpi.f90:883-891) */
      if (lapl) {
        double dlm = c->dlnmu[ir];
        for (int j = 1; j <= m; j++) {
          size_t id = IDX(c, t0 + j - 1, ip, ir);
          double v = PT(vF, j);
          dvv[j] = dvv[j] + ri * mu6[j] * (CT(j) * w1[j] - (ri * CSC2(j) + dlm) * v);
          c->lap[LAP_V1 * n + id] = w1[j];
        }
        line_deriv(c, B, 1, 2, vF, ip, ir, c->ibct[3], lo, hi, o2);
        for (int j = 1; j <= m; j++) dvv[j] = dvv[j] + ri * ri * mu6[j] * o2[j];
      }
      for (int j = 1; j <= m; j++) {
        double rho = PT(rhoF, j), w = PT(wF, j), v = PT(vF, j), u = PT(uF, j);
        PT(dv1, j) = drho[j] - 2.0 * ri * rho * u; /* dvars1(:,:,ir,1) */
        dvv[j] = dvv[j] - u * (ri * v + om2 * SN(j));
        dw[j] = dw[j] - ri * u * w;
        if (!mag) dv1[2 * n + IDX(c, t0 + j - 1, ip, ir)] = dvv[j];
      }
      line_deriv(c, B, 1, 1, uF, ip, ir, c->ibct[4], 0.0, 0.0, w1);
      for (int j = 1; j <= m; j++) {
        w1[j] = w1[j] * ri;
        du[j] = du[j] - PT(wF, j) * w1[j];
      }
      /* explicit viscosity, u terms (rhs_mpi.f90:914-926) */
      if (lapl) {
        double ddiff = 2.0 * FOURTHIRDS * ri + c->dlnmu[ir];
        for (int j = 1; j <= m; j++) {
          size_t id = IDX(c, t0 + j - 1, ip, ir);
          c->lap[LAP_U1 * n + id] = w1[j];
          double t1 = w1[j] * mu6[j];
          dw[j] = dw[j] + ddiff * t1;
          du[j] = du[j] + ri * CT(j) * t1;
        }
        line_deriv(c, B, 1, 2, uF, ip, ir, c->ibct[4], 0.0, 0.0, o2);
        for (int j = 1; j <= m; j++) du[j] = du[j] + ri * ri * mu6[j] * o2[j];
      }
      for (int j = 1; j <= m; j++) {
        if (!mag) dv1[3 * n + IDX(c, t0 + j - 1, ip, ir)] = du[j];
        double t = c->temperature[IDX(c, t0 + j - 1, ip, ir)];
        if (fabs(epsr) > 0.0) ds[j] = epsr * c->invrho[IDX(c, t0 + j - 1, ip, ir)] / t;
        else ds[j] = 0.0;
      }
      line_deriv(c, B, 1, 1, sF, ip, ir, c->ibct[5], 0.0, 0.0, w1);
      for (int j = 1; j <= m; j++) {
        size_t id = IDX(c, t0 + j - 1, ip, ir);
        double w = PT(wF, j), t = c->temperature[id];
        w1[j] = w1[j] * ri;
        if (mag) dw[j] = dw[j] - c->gamm1 * t * w1[j];
        else dv1[1 * n + id] = dw[j] - c->gamm1 * t * w1[j];
        ds[j] = ds[j] - w * w1[j];
      }
      if (c->cond) {
        double ddiff = ri * c->ks[ir];
        for (int j = 1; j <= m; j++) {
          size_t id = IDX(c, t0 + j - 1, ip, ir);
          double oorho = c->invrho[id] / c->temperature[id];
          w1[j] = ddiff * w1[j] * oorho;
          ds[j] = ds[j] + CT(j) * w1[j];
        }
        line_deriv(c, B, 1, 2, sF, ip, ir, c->ibct[5], 0.0, 0.0, o2);
        double dd2 = ddiff * ri * ri; /* ks/r^3 as rhs_mpi.f90:972 has it */
        for (int j = 1; j <= m; j++) {
          size_t id = IDX(c, t0 + j - 1, ip, ir);
          double oorho = c->invrho[id] / c->temperature[id];
          ds[j] = ds[j] + dd2 * o2[j] * oorho;
        }
      }
      for (int j = 1; j <= m; j++) dv1[4 * n + IDX(c, t0 + j - 1, ip, ir)] = ds[j];
      if (mag) {
        const double *btF = v1 + 5 * n, *bpF = v1 + 6 * n, *brF = v1 + 7 * n;
        double oo[m + 2];
        for (int j = 1; j <= m; j++) {
          size_t id = IDX(c, t0 + j - 1, ip, ir);
          oo[j] = c->invrho[id];
          oo[j] = oo[j] * ONE_OVER_4PI * ri;
          double bt = btF[id], bp = bpF[id];
          du[j] = du[j] - bt * bt * oo[j];
          dw[j] = dw[j] - bp * bp * CT(j) * oo[j];
          dvv[j] = dvv[j] + bp * bt * CT(j) * oo[j];
          du[j] = du[j] - bp * bp * oo[j];
        }
        lo = -(c->cosines[0] / c->sines[0]) * bpF[IDX(c, 0, ip, ir)];
        hi = -(c->cosines[nth - 1] / c->sines[nth - 1]) * bpF[IDX(c, nth - 1, ip, ir)];
        if (!p->theta_normal_field) { lo = 0.0; hi = 0.0; }
        line_deriv(c, B, 1, 1, bpF, ip, ir, c->ibct[8], lo, hi, w1);
        for (int j = 1; j <= m; j++) {
          size_t id = IDX(c, t0 + j - 1, ip, ir);
          w1[j] = w1[j] * oo[j];
          dvv[j] = dvv[j] + btF[id] * w1[j];
          dw[j] = dw[j] - bpF[id] * w1[j];
        }
        line_deriv(c, B, 1, 1, brF, ip, ir, c->ibct[9], 0.0, 0.0, w1);
        for (int j = 1; j <= m; j++) {
          size_t id = IDX(c, t0 + j - 1, ip, ir);
          double bt = btF[id], bp = bpF[id], br = brF[id];
          w1[j] = w1[j] * oo[j];
          dv1[1 * n + id] = dw[j] + br * (bt * oo[j] - w1[j]);
          dv1[2 * n + id] = dvv[j] + br * bp * oo[j];
          dv1[3 * n + id] = du[j] + bt * w1[j];
        }
      }
#undef PT
#undef SN
#undef CS
#undef CT
#undef CSC2
    }
}

static void phi_terms(orc_ctx *c, const blk_t *B, const double *v1, double *dv1) {
  const css_params *p = &c->p;
  int mag = p->magnetic, lapl = p->laplacian;
  size_t n = c->ncell;
  const double *rhoF = v1, *wF = v1 + n, *vF = v1 + 2 * n, *uF = v1 + 3 * n, *sF = v1 + 4 * n;
#pragma omp parallel for collapse(2) schedule(static)
  for (int ir = B->r0; ir < B->r0 + B->nr; ir++)
    for (int it = B->t0; it < B->t0 + B->nt; it++) {
      int m = B->np, p0 = B->p0;
      double ri = c->r_inv[ir];
      double cscth = 1.0 / c->sines[it];
      double oors = ri * cscth;
      double w1[m + 2], dw[m + 2], dvv[m + 2], du[m + 2], ds[m + 2], drho[m + 2];
#define PI_(j) IDX(c, it, p0 + (j)-1, ir)
      line_deriv(c, B, 2, 1, rhoF, it, ir, 0, 0.0, 0.0, w1);
      for (int j = 1; j <= m; j++) {
        size_t id = PI_(j);
        drho[j] = dv1[id];
        w1[j] = w1[j] * oors;
        dvv[j] = dv1[2 * n + id];
        drho[j] = drho[j] - vF[id] * w1[j];
        double oorho = c->invrho[id], t = c->temperature[id];
        dvv[j] = dvv[j] - c->pconst * w1[j] * t * oorho;
        ds[j] = dv1[4 * n + id];
      }
      if (p->do_radheat) { /* radiative diffusion, phi (rhs_mpi.f90:1092-1106) */
        double wr[m + 2], o[m + 2];
        for (int j = 1; j <= m; j++) wr[j] = w1[j] * c->invrho[PI_(j)];
        line_deriv(c, B, 2, 1, c->temperature, it, ir, 0, 0.0, 0.0, o);
        for (int j = 1; j <= m; j++) {
          size_t id = PI_(j);
          o[j] = o[j] * oors / c->temperature[id];
          ds[j] = ds[j] + c->rad1[id] * (3.0 * o[j] - wr[j]) * o[j];
        }
        line_deriv(c, B, 2, 2, c->temperature, it, ir, 0, 0.0, 0.0, o);
        for (int j = 1; j <= m; j++) {
          size_t id = PI_(j);
          o[j] = o[j] * (oors * oors);
          ds[j] = ds[j] + c->rad1[id] * o[j] / c->temperature[id];
        }
      }
      line_deriv(c, B, 2, 1, vF, it, ir, 0, 0.0, 0.0, w1);
      for (int j = 1; j <= m; j++) {
        size_t id = PI_(j);
        w1[j] = w1[j] * oors;
        dvv[j] = dvv[j] - vF[id] * w1[j];
        dv1[id] = drho[j] - rhoF[id] * w1[j];
        dw[j] = dv1[n + id];
        du[j] = dv1[3 * n + id];
      }
      /* explicit viscosity (rhs_mpi.f90:1123-1199): mu2 = mur/rho; viscous
       * heating theta-theta/phi-phi, theta-phi; cot = cos * (1/sin) here */
      double mu2[m + 2], o2[m + 2];
      double cot = c->cosines[it] * cscth;
      if (lapl) {
        for (int j = 1; j <= m; j++) {
          size_t id = PI_(j);
          double u = uF[id], w = wF[id], t = c->temperature[id], w1t = c->lap[LAP_W1 * n + id];
          mu2[j] = c->invrho[id] * c->mur[ir];
          c->lap[LAP_PV * n + id] = w1[j];
          ds[j] = ds[j] + FOURTHIRDS * mu2[j] * (w1t + u * ri) * (w1t + 2.0 * u * ri - w1[j] - ri * cot * w) / t;
          double t1 = w1[j] * mu2[j];
          double ddiff = -SEVENTHIRDS * ri, ddiff2 = ddiff - TWOTHIRDS * c->dlnmu[ir];
          dw[j] = dw[j] + ddiff * cot * t1;
          du[j] = du[j] + ddiff2 * t1;
        }
        line_deriv(c, B, 2, 2, vF, it, ir, 0, 0.0, 0.0, o2);
        for (int j = 1; j <= m; j++) {
          o2[j] = o2[j] * (oors * oors);
          dvv[j] = dvv[j] + FOURTHIRDS * o2[j] * mu2[j];
        }
      }
      line_deriv(c, B, 2, 1, wF, it, ir, 0, 0.0, 0.0, w1);
      for (int j = 1; j <= m; j++) {
        size_t id = PI_(j);
        w1[j] = w1[j] * oors;
        dw[j] = dw[j] - vF[id] * w1[j];
      }
      if (lapl) {
        for (int j = 1; j <= m; j++) {
          size_t id = PI_(j);
          double v = vF[id], t = c->temperature[id], v1t = c->lap[LAP_V1 * n + id];
          double q = v1t + w1[j] - ri * cot * v;
          ds[j] = ds[j] + mu2[j] * (q * q) / t;
          c->lap[LAP_PW * n + id] = w1[j];
          dvv[j] = dvv[j] + SEVENTHIRDS * ri * cot * (w1[j] * mu2[j]);
        }
        line_deriv(c, B, 2, 2, wF, it, ir, 0, 0.0, 0.0, o2);
        for (int j = 1; j <= m; j++) {
          o2[j] = o2[j] * (oors * oors);
          dw[j] = dw[j] + o2[j] * mu2[j];
        }
      }
      for (int j = 1; j <= m; j++)
        if (!mag) dv1[n + PI_(j)] = dw[j];
      line_deriv(c, B, 2, 1, uF, it, ir, 0, 0.0, 0.0, w1);
      for (int j = 1; j <= m; j++) {
        size_t id = PI_(j);
        w1[j] = w1[j] * oors;
        du[j] = du[j] - vF[id] * w1[j];
      }
      if (lapl) {
        double ddiff = 2.0 * FOURTHIRDS * ri + c->dlnmu[ir];
        for (int j = 1; j <= m; j++) {
          c->lap[LAP_PU * n + PI_(j)] = w1[j];
          dvv[j] = dvv[j] + ddiff * w1[j] * mu2[j];
        }
        line_deriv(c, B, 2, 2, uF, it, ir, 0, 0.0, 0.0, o2);
        for (int j = 1; j <= m; j++) {
          o2[j] = o2[j] * (oors * oors);
          du[j] = du[j] + o2[j] * mu2[j];
        }
      }
      for (int j = 1; j <= m; j++)
        if (!mag) dv1[3 * n + PI_(j)] = du[j];
      line_deriv(c, B, 2, 1, sF, it, ir, 0, 0.0, 0.0, w1);
      for (int j = 1; j <= m; j++) {
        size_t id = PI_(j);
        double t = c->temperature[id];
        w1[j] = w1[j] * oors;
        ds[j] = ds[j] - vF[id] * w1[j];
        dvv[j] = dvv[j] - c->gamm1 * t * w1[j];
        if (!mag) dv1[2 * n + id] = dvv[j];
      }
      if (c->cond) {
        line_deriv(c, B, 2, 2, sF, it, ir, 0, 0.0, 0.0, w1);
        double ddiff = c->ks[ir];
        for (int j = 1; j <= m; j++) {
          size_t id = PI_(j);
          double oorho = c->invrho[id], t = c->temperature[id];
          w1[j] = w1[j] * (oors * oors);
          ds[j] = ds[j] + ddiff * w1[j] * (oorho / t);
        }
      }
      for (int j = 1; j <= m; j++) dv1[4 * n + PI_(j)] = ds[j];
      if (mag) {
        const double *btF = v1 + 5 * n, *bpF = v1 + 6 * n, *brF = v1 + 7 * n;
        double oo[m + 2];
        for (int j = 1; j <= m; j++) oo[j] = ONE_OVER_4PI * c->invrho[PI_(j)] * oors;
        line_deriv(c, B, 2, 1, btF, it, ir, 0, 0.0, 0.0, w1);
        for (int j = 1; j <= m; j++) {
          size_t id = PI_(j);
          w1[j] = w1[j] * oo[j];
          dvv[j] = dvv[j] - btF[id] * w1[j];
          dv1[n + id] = dw[j] + bpF[id] * w1[j];
        }
        line_deriv(c, B, 2, 1, brF, it, ir, 0, 0.0, 0.0, w1);
        for (int j = 1; j <= m; j++) {
          size_t id = PI_(j);
          w1[j] = w1[j] * oo[j];
          dv1[2 * n + id] = dvv[j] - brF[id] * w1[j];
          dv1[3 * n + id] = du[j] + bpF[id] * w1[j];
        }
      }
#undef PI_
    }
}

static void radial_terms(orc_ctx *c, const blk_t *B, const double *v1, double *dv1) {
  const css_params *p = &c->p;
  int mag = p->magnetic, nu = p->non_uniform, lapl = p->laplacian;
  size_t n = c->ncell;
  const double *rhoF = v1, *wF = v1 + n, *vF = v1 + 2 * n, *uF = v1 + 3 * n, *sF = v1 + 4 * n;
#pragma omp parallel for collapse(2) schedule(static)
  for (int ip = B->p0; ip < B->p0 + B->np; ip++)
    for (int it = B->t0; it < B->t0 + B->nt; it++) {
      int m = B->nr, r0 = B->r0, nr = c->nr, nth = c->nth;
      double w1[m + 2], dw[m + 2], dvv[m + 2], du[m + 2], ds[m + 2];
      double lo, hi;
#define RI_(j) IDX(c, it, ip, r0 + (j)-1)
#define W3(j) c->dxdr[r0 + (j)-1]
#define W9(j) (c->d2xdr2[r0 + (j)-1] / c->dxdr[r0 + (j)-1])
      /* dw/dr, stress-free datum w/r/dxdr (rhs_mpi.f90:580, :609) */
      lo = 0.0; hi = 0.0;
      if (p->bottom_stress_free) lo = wF[IDX(c, it, ip, 0)] / p->r1 / c->dxdr[0];
      if (p->top_stress_free) hi = wF[IDX(c, it, ip, nr - 1)] / p->r2 / c->dxdr[nr - 1];
      else hi = wF[IDX(c, it, ip, nr - 1)];
      if (p->bot_inout) lo = 0.0; /* open faces: data 2:5 zero (rhs_mpi.f90:594-596, :626-628) */
      if (p->top_inout) hi = 0.0;
      line_deriv(c, B, 0, 1, wF, it, ip, c->ibcr[2], lo, hi, w1);
      for (int j = 1; j <= m; j++) {
        size_t id = RI_(j);
        if (nu) w1[j] = w1[j] * W3(j);
        dw[j] = dv1[n + id];
        dw[j] = dw[j] - uF[id] * w1[j];
        du[j] = dv1[3 * n + id];
        ds[j] = dv1[4 * n + id];
      }
      /* explicit viscosity (rhs_mpi.f90:1317-1435): mu2 = mur/rho, w5 =
       * 2/r + dlnmu, cot = cos/sin.  The cot(theta) u_theta' / (3 r) term of
       * du carries no mur/rho, and the r-theta heating is added once with
       * dv/dr and once with du/dr, both as the reference writes them. */
      double mu2[m + 2], o2[m + 2];
      double cot = c->cosines[it] / c->sines[it];
#define W5(j) (2.0 * c->r_inv[r0 + (j)-1] + c->dlnmu[r0 + (j)-1])
#define RV(j) c->r_inv[r0 + (j)-1]
      if (lapl) {
        for (int j = 1; j <= m; j++) {
          size_t id = RI_(j);
          int ir = r0 + j - 1;
          mu2[j] = c->mur[ir] * c->invrho[id];
          du[j] = du[j] + ONETHIRD * cot * RV(j) * w1[j];
          dw[j] = dw[j] + mu2[j] * W5(j) * w1[j];
          double q = w1[j] + c->lap[LAP_U1 * n + id] - wF[id] * RV(j);
          ds[j] = ds[j] + mu2[j] * (q * q) / c->temperature[id];
        }
        if (nu)
          for (int j = 1; j <= m; j++) dw[j] = dw[j] + W9(j) * w1[j] * mu2[j];
        line_deriv(c, B, 0, 2, wF, it, ip, c->ibcr[2], lo, hi, o2);
        for (int j = 1; j <= m; j++) {
          if (nu) o2[j] = o2[j] * (W3(j) * W3(j));
          dw[j] = dw[j] + o2[j] * mu2[j];
        }
      }
      for (int j = 1; j <= m; j++)
        if (!mag) dv1[n + RI_(j)] = dw[j];
      lo = 0.0;
      if (p->bottom_stress_free) lo = vF[IDX(c, it, ip, 0)] / p->r1 / c->dxdr[0];
      if (p->top_stress_free) hi = vF[IDX(c, it, ip, nr - 1)] / p->r2 / c->dxdr[nr - 1];
      else hi = vF[IDX(c, it, ip, nr - 1)];
      if (p->bot_inout) lo = 0.0;
      if (p->top_inout) hi = 0.0;
      line_deriv(c, B, 0, 1, vF, it, ip, c->ibcr[3], lo, hi, w1);
      for (int j = 1; j <= m; j++) {
        size_t id = RI_(j);
        if (nu) w1[j] = w1[j] * W3(j);
        dvv[j] = dv1[2 * n + id];
        dvv[j] = dvv[j] - uF[id] * w1[j];
      }
      if (lapl) {
        for (int j = 1; j <= m; j++) {
          size_t id = RI_(j);
          double q = w1[j] + c->lap[LAP_PU * n + id] - vF[id] * RV(j);
          ds[j] = ds[j] + mu2[j] * (q * q) / c->temperature[id];
          dvv[j] = dvv[j] + w1[j] * W5(j) * mu2[j];
          if (nu) dvv[j] = dvv[j] + W9(j) * w1[j] * mu2[j];
        }
        line_deriv(c, B, 0, 2, vF, it, ip, c->ibcr[3], lo, hi, o2);
        for (int j = 1; j <= m; j++) {
          if (nu) o2[j] = o2[j] * (W3(j) * W3(j));
          dvv[j] = dvv[j] + o2[j] * mu2[j];
        }
      }
      for (int j = 1; j <= m; j++)
        if (!mag) dv1[2 * n + RI_(j)] = dvv[j];
      line_deriv(c, B, 0, 1, uF, it, ip, c->ibcr[4], 0.0, 0.0, w1);
      for (int j = 1; j <= m; j++) {
        size_t id = RI_(j);
        if (nu) w1[j] = w1[j] * W3(j);
        du[j] = du[j] - uF[id] * w1[j];
        dv1[id] = dv1[id] - rhoF[id] * w1[j];
      }
      if (lapl) {
        for (int j = 1; j <= m; j++) {
          size_t id = RI_(j);
          double u = uF[id], v = vF[id], w = wF[id], t = c->temperature[id];
          du[j] = du[j] + FOURTHIRDS * mu2[j] * W5(j) * (w1[j] - u * RV(j));
          if (nu) du[j] = du[j] + FOURTHIRDS * W9(j) * w1[j] * mu2[j];
          ds[j] = ds[j] + FOURTHIRDS * mu2[j] * w1[j] * (w1[j] - c->lap[LAP_W1 * n + id] - u * RV(j)) / t;
          double q = w1[j] + c->lap[LAP_PU * n + id] - v * RV(j);
          ds[j] = ds[j] + mu2[j] * (q * q) / t;
          double a = c->lap[LAP_PV * n + id] + (cot * w + u) * RV(j);
          ds[j] = ds[j] + FOURTHIRDS * mu2[j] * a * (a - w1[j]) / t;
        }
        line_deriv(c, B, 0, 2, uF, it, ip, c->ibcr[4], 0.0, 0.0, o2);
        for (int j = 1; j <= m; j++) {
          if (nu) o2[j] = o2[j] * (W3(j) * W3(j));
          du[j] = du[j] + FOURTHIRDS * o2[j] * mu2[j];
        }
      }
#undef W5
#undef RV
      /* ds/dr with the constant-flux datum (rhs_mpi.f90:584-592, :616-624) */
      lo = 0.0; hi = 0.0;
      if (!p->bottom_constant_temp) {
        if (c->cond) lo = -p->lumr1 * ONE_OVER_4PI / (p->r1 * p->r1 * c->ks[0] * c->dxdr[0]);
        else lo = 0.0 / c->dxdr[0]; /* dsdr1 = dsdrm(1) = 0 for the Isentropic model */
      }
      if (!p->top_constant_temp) {
        if (c->cond) hi = -p->lumr2 * ONE_OVER_4PI / (p->r2 * p->r2 * c->ks[nr - 1] * c->dxdr[nr - 1]);
        else hi = 0.0 / c->dxdr[nr - 1];
      }
      if (p->bot_inout) lo = 0.0;
      if (p->top_inout) hi = 0.0;
      line_deriv(c, B, 0, 1, sF, it, ip, c->ibcr[5], lo, hi, w1);
      for (int j = 1; j <= m; j++) {
        size_t id = RI_(j);
        double t = c->temperature[id];
        if (nu) w1[j] = w1[j] * W3(j);
        du[j] = du[j] - c->gamm1 * t * w1[j];
        ds[j] = ds[j] - uF[id] * w1[j];
        if (p->do_radheat) c->rad2[id] = w1[j]; /* dvars2(:,ip,:,2), rhs_mpi.f90:1454 */
      }
      if (c->cond) {
        for (int j = 1; j <= m; j++) {
          size_t id = RI_(j);
          int ir = r0 + j - 1;
          double oorho = c->invrho[id] / c->temperature[id];
          double work6 = (2.0 * c->r_inv[ir] + c->dlnks[ir]) * c->ks[ir];
          w1[j] = w1[j] * oorho;
          ds[j] = ds[j] + w1[j] * work6;
          if (nu) ds[j] = ds[j] + W9(j) * w1[j] * c->ks[ir];
        }
        line_deriv(c, B, 0, 2, sF, it, ip, c->ibcr[5], lo, hi, o2);
        for (int j = 1; j <= m; j++) {
          size_t id = RI_(j);
          int ir = r0 + j - 1;
          double oorho = c->invrho[id] / c->temperature[id];
          if (nu) o2[j] = o2[j] * (W3(j) * W3(j));
          ds[j] = ds[j] + c->ks[ir] * o2[j] * oorho;
        }
      }
      for (int j = 1; j <= m; j++) {
        size_t id = RI_(j);
        if (!mag) dv1[3 * n + id] = du[j];
        dv1[4 * n + id] = ds[j];
      }
      if (mag) {
        const double *btF = v1 + 5 * n, *bpF = v1 + 6 * n, *brF = v1 + 7 * n;
        double bclo = 0.0, bchi = 0.0;
        line_deriv(c, B, 0, 1, btF, it, ip, c->ibcr[7], bclo, bchi, w1);
        for (int j = 1; j <= m; j++) {
          size_t id = RI_(j);
          double oo = c->invrho[id] * ONE_OVER_4PI;
          if (nu) w1[j] = w1[j] * W3(j);
          w1[j] = w1[j] * oo;
          du[j] = du[j] - btF[id] * w1[j];
          dv1[n + id] = dw[j] + brF[id] * w1[j];
        }
        line_deriv(c, B, 0, 1, bpF, it, ip, c->ibcr[8], bclo, bchi, w1);
        for (int j = 1; j <= m; j++) {
          size_t id = RI_(j);
          double oo = c->invrho[id] * ONE_OVER_4PI;
          if (nu) w1[j] = w1[j] * W3(j);
          w1[j] = w1[j] * oo;
          dv1[2 * n + id] = dvv[j] + brF[id] * w1[j];
          dv1[3 * n + id] = du[j] - bpF[id] * w1[j];
        }
      }
      (void)nth;
#undef RI_
#undef W3
#undef W9
    }
}

static void density_terms_theta(orc_ctx *c, const blk_t *B, const double *v1, double *dv1) {
  size_t n = c->ncell;
  const double *rhoF = v1, *wF = v1 + n;
#pragma omp parallel for collapse(2) schedule(static)
  for (int ir = B->r0; ir < B->r0 + B->nr; ir++)
    for (int ip = B->p0; ip < B->p0 + B->np; ip++) {
      int m = B->nt, t0 = B->t0;
      double rv = c->r_ind[ir] * c->invpconst, ri = c->r_inv[ir];
      double w1[m + 2];
      double lo = 0.0, hi = 0.0;
      /* BC datum so that dw = 0 on the theta walls (rhs_mpi.f90:1553-1564) */
      if (B->tlo) {
        size_t id = IDX(c, t0, ip, ir);
        lo = rv * dv1[n + id] * rhoF[id] / c->temperature[id];
      } else if (B->thi) {
        size_t id = IDX(c, t0 + m - 1, ip, ir);
        hi = rv * dv1[n + id] * rhoF[id] / c->temperature[id];
      }
      line_deriv(c, B, 1, 1, rhoF, ip, ir, c->ibct[1], lo, hi, w1);
      for (int j = 1; j <= m; j++) {
        size_t id = IDX(c, t0 + j - 1, ip, ir);
        double dw = dv1[n + id], t = c->temperature[id];
        w1[j] = ri * w1[j];
        dv1[id] = dv1[id] - wF[id] * w1[j];
        w1[j] = w1[j] * c->invrho[id];
        dv1[n + id] = dw - c->pconst * w1[j] * t;
      }
      if (c->p.do_radheat) { /* radiative diffusion, theta (rhs_mpi.f90:1590-1602) */
        double o[m + 2];
        double tlo = c->temperature[IDX(c, 0, ip, ir)], thi = c->temperature[IDX(c, c->nth - 1, ip, ir)];
        line_deriv(c, B, 1, 1, c->temperature, ip, ir, c->ibct[6], tlo, thi, o);
        for (int j = 1; j <= m; j++) {
          int it = t0 + j - 1;
          size_t id = IDX(c, it, ip, ir);
          double t = c->temperature[id], cot = c->cosines[it] / c->sines[it];
          o[j] = ri * o[j] / t;
          dv1[4 * n + id] = dv1[4 * n + id] + c->rad1[id] * o[j] * (3.0 * o[j] + ri * cot - w1[j]);
        }
        line_deriv(c, B, 1, 2, c->temperature, ip, ir, c->ibct[6], tlo, thi, o);
        for (int j = 1; j <= m; j++) {
          size_t id = IDX(c, t0 + j - 1, ip, ir);
          dv1[4 * n + id] = dv1[4 * n + id] + (ri * ri) * c->rad1[id] * o[j] / c->temperature[id];
        }
      }
    }
}

static void density_terms_radial(orc_ctx *c, const blk_t *B, const double *v1, double *dv1) {
  const css_params *p = &c->p;
  size_t n = c->ncell;
  const double *rhoF = v1, *uF = v1 + 3 * n;
  int nu = p->non_uniform;
#pragma omp parallel for collapse(2) schedule(static)
  for (int ip = B->p0; ip < B->p0 + B->np; ip++)
    for (int it = B->t0; it < B->t0 + B->nt; it++) {
      int m = B->nr, r0 = B->r0;
      double w1[m + 2];
      double lo = 0.0, hi = 0.0;
      if (B->rlo) {
        size_t id = IDX(c, it, ip, r0);
        if ((c->lbcr_rho == 2) || (c->lbcr_rho == 4)) lo = dv1[3 * n + id] * rhoF[id] * c->invpconst / c->temperature[id];
        else lo = rhoF[id];
        if (nu) lo = lo / c->dxdr[r0];
      } else if (B->rhi) {
        size_t id = IDX(c, it, ip, r0 + m - 1);
        if ((c->lbcr_rho == 3) || (c->lbcr_rho == 4)) hi = dv1[3 * n + id] * rhoF[id] * c->invpconst / c->temperature[id];
        else hi = rhoF[id];
        if (nu) hi = hi / c->dxdr[r0 + m - 1];
      }
      line_deriv(c, B, 0, 1, rhoF, it, ip, c->ibcr[1], lo, hi, w1);
      for (int j = 1; j <= m; j++) {
        size_t id = IDX(c, it, ip, r0 + j - 1);
        double du = dv1[3 * n + id], t = c->temperature[id];
        if (nu) w1[j] = w1[j] * c->dxdr[r0 + j - 1];
        dv1[id] = dv1[id] - uF[id] * w1[j];
        w1[j] = w1[j] * c->invrho[id];
        dv1[3 * n + id] = du - c->pconst * t * w1[j];
      }
      /* thermal damping toward T0 on the top shell (rhs_mpi.f90:1807-1818) */
      if (B->rhi && !p->set_stop && !p->do_radheat) {
        size_t id = IDX(c, it, ip, r0 + m - 1);
        double t = c->temperature[id], rho = rhoF[id];
        dv1[id] = dv1[id] + rho * (p->t0 - t) / (p->damping_time * (p->gamma - 2.0) * t);
        dv1[4 * n + id] = dv1[4 * n + id] - c->cv * (p->t0 - t) / (p->damping_time * (p->gamma - 2.0) * t);
      }
      if (p->do_radheat) { /* radiative diffusion, r (rhs_mpi.f90:1820-1853); w1 = d ln(rho)/dr */
        double o[m + 2];
        double tlo = 0.0, thi = 0.0;
        if (B->rlo) {
          size_t id = IDX(c, it, ip, r0);
          tlo = c->temperature[id] * (c->gamm1 * w1[1] + c->invcv * c->rad2[id]) / c->dxdr[0];
        }
        if (B->rhi) {
          size_t id = IDX(c, it, ip, r0 + m - 1);
          thi = c->temperature[id] * (c->gamm1 * w1[m] + c->invcv * c->rad2[id]) / c->dxdr[c->nr - 1];
        }
        line_deriv(c, B, 0, 1, c->temperature, it, ip, c->ibcr[6], tlo, thi, o);
        for (int j = 1; j <= m; j++) {
          int ir = r0 + j - 1;
          size_t id = IDX(c, it, ip, ir);
          double t = c->temperature[id], w4 = 2.0 * c->r_inv[ir] - c->dlnkr[ir];
          if (nu) o[j] = o[j] * c->dxdr[ir];
          o[j] = o[j] / t;
          dv1[4 * n + id] = dv1[4 * n + id] + c->rad1[id] * o[j] * (w4 + 3.0 * o[j] - w1[j]);
          if (nu) dv1[4 * n + id] = dv1[4 * n + id] + c->rad1[id] * o[j] * (c->d2xdr2[ir] / c->dxdr[ir]);
        }
        line_deriv(c, B, 0, 2, c->temperature, it, ip, c->ibcr[6], tlo, thi, o);
        for (int j = 1; j <= m; j++) {
          int ir = r0 + j - 1;
          size_t id = IDX(c, it, ip, ir);
          if (nu) o[j] = o[j] * (c->dxdr[ir] * c->dxdr[ir]);
          dv1[4 * n + id] = dv1[4 * n + id] + c->rad1[id] * o[j] / c->temperature[id];
        }
      }
    }
}

/* ------------------------------------------------------------------------ */
/* Open radial boundaries.  On the blocks of an open face Top_Inflow_Outflow */
/* (rhs_mpi.f90:1955-2067) or Bottom_Inflow_Outflow (:1857-1953) replaces    */
/* Density_Terms_Radial (:723-729): d(rho)/dr with the open closure, then   */
/* the face plane relaxed toward its inner neighbour with mean-flow and     */
/* mean-entropy corrections from sums over the whole face (the top_comm /   */
/* bot_comm reductions).  Neither routine applies the non-uniform dxdr to   */
/* d(rho)/dr or its datum, unlike Density_Terms_Radial; restated as written. */
/* ------------------------------------------------------------------------ */
typedef struct {
  double top[4]; /* sum u rho sin, sum rho sin, sum s, sum rho sin (dvel_rain + u(nr-1)) */
  double bot[4]; /* sum rho(mynr) sin u(1), sum rho(mynr) sin, sum s(1), max of |min u(2)| */
} inout_sums_t;

/* Tr(nr) of the Isentropic background: T0 (mhdsph_mpi.f90:343 at r = r2) */
static double tr_top(const orc_ctx *c) { return c->p.t0; }

static void inout_sums(orc_ctx *c, const double *v1, inout_sums_t *S) {
  const css_params *p = &c->p;
  size_t n = c->ncell;
  int nr = c->nr;
  memset(S, 0, sizeof *S);
  for (int k = 0; k < c->nblk; k++) {
    const blk_t *B = &c->blk[k];
    if (p->top_inout && B->rhi) { /* rhs_mpi.f90:1987-1998 / :1971-1985 */
      double a[4] = {0.0, 0.0, 0.0, 0.0};
      for (int ip = B->p0; ip < B->p0 + B->np; ip++)
        for (int it = B->t0; it < B->t0 + B->nt; it++) {
          size_t id = IDX(c, it, ip, nr - 1);
          double tau = v1[id] * c->sines[it];
          a[0] = a[0] + v1[3 * n + id] * tau;
          a[1] = a[1] + tau;
          a[2] = a[2] + v1[4 * n + id];
          if (p->do_entropy_rain)
            a[3] = a[3] + tau * (c->dvel_rain[it + (size_t)c->nth * ip] + v1[3 * n + IDX(c, it, ip, nr - 2)]);
        }
      for (int q = 0; q < 4; q++) S->top[q] += a[q];
    }
    if (p->bot_inout && B->rlo && !p->bottom_specified) { /* rhs_mpi.f90:1865-1884 */
      double a[3] = {0.0, 0.0, 0.0}, umin = 0.0;
      int first = 1, mt = B->nr - 1; /* the block's own top radius (mynr) */
      for (int ip = B->p0; ip < B->p0 + B->np; ip++)
        for (int it = B->t0; it < B->t0 + B->nt; it++) {
          double tau = v1[IDX(c, it, ip, mt)] * c->sines[it];
          a[0] = a[0] + tau * v1[3 * n + IDX(c, it, ip, 0)];
          a[1] = a[1] + tau;
          a[2] = a[2] + v1[4 * n + IDX(c, it, ip, 0)];
          double u2 = v1[3 * n + IDX(c, it, ip, 1)];
          if (first || u2 < umin) umin = u2;
          first = 0;
        }
      for (int q = 0; q < 3; q++) S->bot[q] += a[q];
      S->bot[3] = fmax(S->bot[3], fabs(umin)); /* 'csm': sums, then the max (mhdsph_mpi.f90:1511-1521) */
    }
  }
}

static void top_inflow_outflow(orc_ctx *c, const blk_t *B, const double *v1, double *dv1, const inout_sums_t *S) {
  const css_params *p = &c->p;
  size_t n = c->ncell;
  int nr = c->nr;
  const double *rhoF = v1, *uF = v1 + 3 * n, *sF = v1 + 4 * n;
  double ntot = (double)c->nth * (double)c->nphi;
  double meanu = -S->top[0] / S->top[1] / c->deltat;
  double means = c->sr[0] + p->delta_s - S->top[2] / ntot;
  double mdvel = -S->top[3] / S->top[1];
  double tau = sqrt(c->gamm1 * p->cp * tr_top(c)) / c->dr_ind[nr - 1] / 20.0;
  means = tau * means;
  double nrat = c->rhor[nr - 2] / c->rhor[nr - 1];
  double q4 = (c->r_ind[nr - 1] - c->r_ind[B->r0]) / (p->r2 - c->r_ind[B->r0]);
  q4 = (q4 * q4) * (q4 * q4);
  double taur = sqrt(c->gamm1 * p->cp * tr_top(c)) * q4 / c->dr_ind[nr - 1] / 2.0;
#pragma omp parallel for collapse(2) schedule(static)
  for (int ip = B->p0; ip < B->p0 + B->np; ip++)
    for (int it = B->t0; it < B->t0 + B->nt; it++) {
      int m = B->nr, r0 = B->r0;
      double w1[m + 2];
      line_deriv(c, B, 0, 1, rhoF, it, ip, 2, 0.0, 0.0, w1); /* dbydr(rho, ..., bc1, 0, -2) */
      for (int j = 1; j <= m; j++) {
        size_t id = IDX(c, it, ip, r0 + j - 1);
        dv1[id] = dv1[id] - uF[id] * w1[j];
        dv1[3 * n + id] = dv1[3 * n + id] - c->pconst * c->temperature[id] * c->invrho[id] * w1[j];
      }
      size_t top = IDX(c, it, ip, nr - 1), below = IDX(c, it, ip, nr - 2);
      if (p->do_entropy_rain) { /* rhs_mpi.f90:2042-2054 */
        size_t q = it + (size_t)c->nth * ip;
        dv1[3 * n + top] = dv1[3 * n + top] +
                           (mdvel + c->dvel_rain[q] + uF[below] - 2.0 * uF[top]) * taur + meanu;
        dv1[4 * n + top] = dv1[4 * n + top] +
                           (c->sr[0] + p->delta_s + c->dent_rain[q] + sF[below] - 2.0 * sF[top]) * taur;
      } else { /* :2055-2066 */
        dv1[3 * n + top] = dv1[3 * n + top] + tau * (nrat * uF[below] - uF[top]) + meanu;
        dv1[4 * n + top] = dv1[4 * n + top] + tau * (sF[below] - sF[top]) + means;
      }
    }
}

static void bottom_inflow_outflow(orc_ctx *c, const blk_t *B, const double *v1, double *dv1,
                                  const inout_sums_t *S) {
  const css_params *p = &c->p;
  size_t n = c->ncell;
  const double *rhoF = v1, *wF = v1 + n, *vF = v1 + 2 * n, *uF = v1 + 3 * n, *sF = v1 + 4 * n;
  double meanu = 0.0, means = 0.0, tau = 0.0, nrat = 0.0, tconst;
  if (!p->bottom_specified) {
    double ntot = (double)c->nth * (double)c->nphi;
    meanu = -S->bot[0] / S->bot[1] / c->deltat;
    means = c->sr[0] - S->bot[2] / ntot;
    tau = S->bot[3] / c->dr_ind[0];
    nrat = c->rhor[1] / c->rhor[0];
  }
#pragma omp parallel for collapse(2) schedule(static)
  for (int ip = B->p0; ip < B->p0 + B->np; ip++)
    for (int it = B->t0; it < B->t0 + B->nt; it++) {
      int m = B->nr, r0 = B->r0;
      double w1[m + 2];
      size_t i0 = IDX(c, it, ip, r0);
      double lo = c->invpconst * rhoF[i0] * dv1[3 * n + i0] / c->temperature[i0];
      line_deriv(c, B, 0, 1, rhoF, it, ip, 4, lo, 0.0, w1); /* dbydr(rho, ..., bc1, bc2, -4) */
      for (int j = 1; j <= m; j++) {
        size_t id = IDX(c, it, ip, r0 + j - 1);
        dv1[id] = dv1[id] - uF[id] * w1[j];
        dv1[3 * n + id] = dv1[3 * n + id] - c->pconst * c->temperature[id] * w1[j] * c->invrho[id];
      }
    }
  if (p->bottom_specified) { /* rhs_mpi.f90:1913-1938 */
    tau = sqrt(c->gamm1 * p->cp * tr_top(c)) / (20.0 * c->dr_ind[0]);
    tconst = fmin(fabs(c->sim_time) / 1e5, 1.0);
    meanu = tau * (c->m0 - c->mtot) / c->vol;
    size_t np = (size_t)c->nth * c->nphi;
    for (int ip = B->p0; ip < B->p0 + B->np; ip++)
      for (int it = B->t0; it < B->t0 + B->nt; it++) {
        size_t id = IDX(c, it, ip, 0), q = it + (size_t)c->nth * ip;
        const double *a = c->ashv;
        dv1[id] = dv1[id] + meanu;
        dv1[n + id] = dv1[n + id] + tau * (tconst * a[np + q] - wF[id]);
        dv1[2 * n + id] = dv1[2 * n + id] + tau * (tconst * a[2 * np + q] - vF[id]);
        dv1[3 * n + id] = dv1[3 * n + id] + tau * (tconst * a[q] - uF[id]);
        dv1[4 * n + id] = dv1[4 * n + id] + tau * ((c->sr[0] + tconst * c->ash_fen_mod * a[3 * np + q]) - sF[id]);
      }
  } else { /* :1939-1952 */
    tconst = tau * (c->m0 - c->mtot) / c->vol;
    for (int ip = B->p0; ip < B->p0 + B->np; ip++)
      for (int it = B->t0; it < B->t0 + B->nt; it++) {
        size_t id = IDX(c, it, ip, 0), up = IDX(c, it, ip, 1);
        dv1[id] = dv1[id] + tconst;
        dv1[3 * n + id] = dv1[3 * n + id] + tau * (nrat * uF[up] - uF[id]) + meanu;
        dv1[4 * n + id] = dv1[4 * n + id] + tau * (sF[up] - sF[id] + means);
      }
  }
}

/* mass total as the RHS refreshes it every ufreq steps (rhs_mpi.f90:326-353)
 * and the start-up computes it for bot_inout (mhdsph_mpi.f90:979-999):
 * sum over r of dr r^2 sum over the plane of sin rho, times dth dphi */
static double mass_total(const orc_ctx *c, const double *v1) {
  double mt = 0.0;
  for (int ir = 0; ir < c->nr; ir++) {
    double rt = c->dr_ind[ir] * (c->r_ind[ir] * c->r_ind[ir]);
    for (int ip = 0; ip < c->nphi; ip++) {
      double ln = 0.0;
      for (int it = 0; it < c->nth; it++) ln = ln + c->sines[it] * v1[IDX(c, it, ip, ir)];
      mt = mt + ln * rt;
    }
  }
  return mt * c->dth * c->dphi;
}

/* Laplacian_Cross_Terms_Radial (rhs_mpi.f90:2070-2205): radial derivatives
 * of r*X for the sweeps' X = ri dw/dth, du/dph/(r sin), ri du/dth and
 * dv/dph/(r sin), added with mur/(3 r rho) to du, dv, dw, du.  Interior block
 * faces read the neighbours' r*X (Boundary_Exchange_Lapl(1)).  At physical
 * faces the data are r1 (or r2) times the exchange buffer, which the
 * reference fills only for stress-free walls: X1/r1/dxdr(1) on the bottom and
 * X4/r2/dxdr(nr) on the top, both under Bottom_Stress_Free as written
 * (:2112-2124); the other slots are never written for a hydro run and are
 * taken as 0 here.  The reference scales by invrho(it+ir-1, ip, :) with it
 * undefined (:2133); the cell's own 1/rho is used. */
static void lap_cross_radial(orc_ctx *c, double *dv1) {
  const css_params *p = &c->p;
  size_t n = c->ncell, np = (size_t)c->nth * c->nphi;
  int nr = c->nr, nu = p->non_uniform;
  static const int src[4] = {LAP_W1, LAP_PU, LAP_U1, LAP_PV};
  double *F = dalloc(4 * n);
  for (int k = 0; k < 4; k++)
    for (size_t i = 0; i < n; i++) F[k * n + i] = c->r_ind[i / np] * c->lap[src[k] * n + i];
  const int bc[4] = {c->ibcr[2], c->ibcr[4], c->ibcr[4], c->ibcr[3]};
  for (int kb = 0; kb < c->nblk; kb++) {
    const blk_t *B = &c->blk[kb];
#pragma omp parallel for collapse(2) schedule(static)
    for (int ip = B->p0; ip < B->p0 + B->np; ip++)
      for (int it = B->t0; it < B->t0 + B->nt; it++) {
        int m = B->nr, r0 = B->r0;
        double o[4][m + 2];
        for (int k = 0; k < 4; k++) {
          double lo = 0.0, hi = 0.0;
          if (k == 0 && p->bottom_stress_free)
            lo = p->r1 * (c->lap[LAP_W1 * n + IDX(c, it, ip, 0)] / p->r1 / c->dxdr[0]);
          if (k == 3 && p->bottom_stress_free)
            hi = p->r2 * (c->lap[LAP_PV * n + IDX(c, it, ip, nr - 1)] / p->r2 / c->dxdr[nr - 1]);
          line_deriv(c, B, 0, 1, F + k * n, it, ip, bc[k], lo, hi, o[k]);
          if (nu)
            for (int j = 1; j <= m; j++) o[k][j] = o[k][j] * c->dxdr[r0 + j - 1];
        }
        for (int j = 1; j <= m; j++) {
          int ir = r0 + j - 1;
          size_t id = IDX(c, it, ip, ir);
          double w6 = ONETHIRD * c->mur[ir] * c->r_inv[ir] * c->invrho[id];
          double du = dv1[3 * n + id] + w6 * o[0][j];
          dv1[2 * n + id] = dv1[2 * n + id] + w6 * o[1][j];
          dv1[n + id] = dv1[n + id] + w6 * o[2][j];
          dv1[3 * n + id] = du + w6 * o[3][j];
        }
      }
  }
  free(F);
}

/* Laplacian_Cross_Terms_Theta (rhs_mpi.f90:2207-2296): theta derivatives of
 * sin(theta) dv/dph/(r sin) and sin(theta) dw/dph/(r sin), added with
 * mur/(3 r rho sin) to dw and dv.  Wall data of the first: sin * (X cos/sin)
 * at the wall (:2241-2250); of the second: never written, 0. */
static void lap_cross_theta(orc_ctx *c, double *dv1) {
  size_t n = c->ncell;
  int nth = c->nth;
  double *F = dalloc(2 * n);
  for (size_t i = 0; i < n; i++) {
    double sn = c->sines[i % nth];
    F[i] = sn * c->lap[LAP_PV * n + i];
    F[n + i] = sn * c->lap[LAP_PW * n + i];
  }
  for (int kb = 0; kb < c->nblk; kb++) {
    const blk_t *B = &c->blk[kb];
#pragma omp parallel for collapse(2) schedule(static)
    for (int ir = B->r0; ir < B->r0 + B->nr; ir++)
      for (int ip = B->p0; ip < B->p0 + B->np; ip++) {
        int m = B->nt, t0 = B->t0;
        double o[2][m + 2];
        double pv0 = c->lap[LAP_PV * n + IDX(c, 0, ip, ir)], pv1 = c->lap[LAP_PV * n + IDX(c, nth - 1, ip, ir)];
        double lo = c->sines[0] * (pv0 * c->cosines[0] / c->sines[0]);
        double hi = c->sines[nth - 1] * (pv1 * c->cosines[nth - 1] / c->sines[nth - 1]);
        line_deriv(c, B, 1, 1, F, ip, ir, c->ibct[3], lo, hi, o[0]);
        line_deriv(c, B, 1, 1, F + n, ip, ir, c->ibct[2], 0.0, 0.0, o[1]);
        double ri = c->r_inv[ir] * c->mur[ir];
        for (int j = 1; j <= m; j++) {
          int it = t0 + j - 1;
          size_t id = IDX(c, it, ip, ir);
          double w4 = ONETHIRD * ri * c->invrho[id] / c->sines[it];
          dv1[n + id] = dv1[n + id] + w4 * o[0][j];
          dv1[2 * n + id] = dv1[2 * n + id] + w4 * o[1][j];
        }
      }
  }
  free(F);
}

/* VectorCurl (derivatives.f90:1894-2104): J = curl B of b (B_theta, B_phi,
 * B_r) into j (J_theta, J_phi, J_r).  The theta derivatives take bdry 1 under
 * Theta_Normal_Field and 0 otherwise (var -1 / 0), the phi derivatives none,
 * the radial ones the B BCs (var 7, 8); none of these read a wall datum. */
static void vector_curl_b(orc_ctx *c, const double *b, double *j) {
  size_t n = c->ncell, np = (size_t)c->nth * c->nphi;
  int nth = c->nth, nu = c->p.non_uniform;
  const double *bt = b, *bp = b + n, *br = b + 2 * n;
  double *jt = j, *jp = j + n, *jr = j + 2 * n;
  const int bdry_t = c->p.theta_normal_field ? 1 : 0;
  double *F = dalloc(3 * n);
  for (size_t i = 0; i < n; i++) {
    double r = c->r_ind[i / np];
    F[i] = c->sines[i % nth] * bp[i];
    F[n + i] = r * bt[i];
    F[2 * n + i] = r * bp[i];
  }
  for (int kb = 0; kb < c->nblk; kb++) {
    const blk_t *B = &c->blk[kb];
#pragma omp parallel for collapse(2) schedule(static)
    for (int ir = B->r0; ir < B->r0 + B->nr; ir++)
      for (int ip = B->p0; ip < B->p0 + B->np; ip++) {
        double o[B->nt + 2], invr = c->r_inv[ir];
        line_deriv(c, B, 1, 1, F, ip, ir, bdry_t, 0.0, 0.0, o);
        for (int q = 1; q <= B->nt; q++) {
          int it = B->t0 + q - 1;
          jr[IDX(c, it, ip, ir)] = o[q] * (1.0 / c->sines[it]) * invr;
        }
        line_deriv(c, B, 1, 1, br, ip, ir, bdry_t, 0.0, 0.0, o);
        for (int q = 1; q <= B->nt; q++) jp[IDX(c, B->t0 + q - 1, ip, ir)] = -o[q] * invr;
      }
  }
  for (int kb = 0; kb < c->nblk; kb++) {
    const blk_t *B = &c->blk[kb];
#pragma omp parallel for collapse(2) schedule(static)
    for (int ir = B->r0; ir < B->r0 + B->nr; ir++)
      for (int it = B->t0; it < B->t0 + B->nt; it++) {
        double o[B->np + 2], invr = c->r_inv[ir], csc = 1.0 / c->sines[it];
        line_deriv(c, B, 2, 1, br, it, ir, 0, 0.0, 0.0, o);
        for (int q = 1; q <= B->np; q++) jt[IDX(c, it, B->p0 + q - 1, ir)] = invr * o[q] * csc;
        line_deriv(c, B, 2, 1, bt, it, ir, 0, 0.0, 0.0, o);
        for (int q = 1; q <= B->np; q++) {
          size_t id = IDX(c, it, B->p0 + q - 1, ir);
          jr[id] = jr[id] - invr * o[q] * csc;
        }
      }
  }
  for (int kb = 0; kb < c->nblk; kb++) {
    const blk_t *B = &c->blk[kb];
#pragma omp parallel for collapse(2) schedule(static)
    for (int ip = B->p0; ip < B->p0 + B->np; ip++)
      for (int it = B->t0; it < B->t0 + B->nt; it++) {
        double o[B->nr + 2];
        line_deriv(c, B, 0, 1, F + n, it, ip, c->ibcr[7], 0.0, 0.0, o);
        for (int q = 1; q <= B->nr; q++) {
          int ir = B->r0 + q - 1;
          if (nu) o[q] = o[q] * c->dxdr[ir];
          size_t id = IDX(c, it, ip, ir);
          jp[id] = jp[id] + o[q] * c->r_inv[ir];
        }
        line_deriv(c, B, 0, 1, F + 2 * n, it, ip, c->ibcr[8], 0.0, 0.0, o);
        for (int q = 1; q <= B->nr; q++) {
          int ir = B->r0 + q - 1;
          if (nu) o[q] = o[q] * c->dxdr[ir];
          size_t id = IDX(c, it, ip, ir);
          jt[id] = jt[id] - o[q] * c->r_inv[ir];
        }
      }
  }
  free(F);
}

static void thermo(orc_ctx *c, const double *v1) {
  size_t n = c->ncell;
  /* rhs_mpi.f90:376-387 */
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; i++) {
    double ir = pow(v1[i], c->gamm1);
    double t = c->invtconst * ir;
    ir = v1[4 * n + i] * c->invcv;
    ir = exp(ir);
    t = t * ir;
    c->temperature[i] = t;
    c->invrho[i] = 1.0 / v1[i];
  }
  if (c->p.do_radheat) { /* rhs_mpi.f90:388-392 */
    size_t np = (size_t)c->nth * c->nphi;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) {
      double t = c->temperature[i], ir = c->invrho[i];
      c->rad1[i] = (4.0 * A_CONST * C_LIGHT * c->kr[i / np] / 3.0) * (t * t * t) * (ir * ir);
    }
  }
}

int orc_rhs(orc_ctx *c, double *vars1, double *dvars1, int call_num) {
  size_t n = c->ncell;
  int nv = c->nv;
  memset(dvars1, 0, sizeof(double) * n * nv);
  if (c->p.magnetic) {
    /* Compute_B(1): maga = A; vars1(6:8) = B (derivatives.f90:1830-1892) */
    memcpy(c->maga, vars1 + 5 * n, sizeof(double) * 3 * n);
    vector_curl_a(c, c->maga, dvars1 + 5 * n);
    compute_b_bc(c, dvars1 + 5 * n);
    memcpy(vars1 + 5 * n, dvars1 + 5 * n, sizeof(double) * 3 * n);
    memset(dvars1 + 5 * n, 0, sizeof(double) * 3 * n);
  }
  thermo(c, vars1);
  if ((c->p.top_inout || c->p.bot_inout) && call_num == 1 && c->p.ufreq > 0 && c->istep % c->p.ufreq == 0)
    c->mtot = mass_total(c, vars1);
  for (int k = 0; k < c->nblk; k++) source_theta_terms(c, &c->blk[k], vars1, dvars1);
  for (int k = 0; k < c->nblk; k++) phi_terms(c, &c->blk[k], vars1, dvars1);
  for (int k = 0; k < c->nblk; k++) radial_terms(c, &c->blk[k], vars1, dvars1);
  if (c->p.laplacian) {
    lap_cross_radial(c, dvars1);
    lap_cross_theta(c, dvars1);
  }
  for (int k = 0; k < c->nblk; k++) density_terms_theta(c, &c->blk[k], vars1, dvars1);
  if (c->p.top_inout || c->p.bot_inout) {
    inout_sums_t S;
    inout_sums(c, vars1, &S);
    for (int k = 0; k < c->nblk; k++) {
      const blk_t *B = &c->blk[k];
      if (c->p.bot_inout && B->rlo) bottom_inflow_outflow(c, B, vars1, dvars1, &S);
      else if (c->p.top_inout && B->rhi) top_inflow_outflow(c, B, vars1, dvars1, &S);
      else density_terms_radial(c, B, vars1, dvars1);
    }
  } else {
    for (int k = 0; k < c->nblk; k++) density_terms_radial(c, &c->blk[k], vars1, dvars1);
  }
  if (c->p.magnetic) {
    /* Induction_Terms: under Laplacian the resistive part first (rhs_mpi.f90:
     * 2303-2327): J = curl B, eta J / rho / T ohmic heating with jconst =
     * 4 pi / c^2 and etar = ks (mhdsph_mpi.f90:316, :349), -eta J kept for
     * dA/dt; then dA/dt = v x B (:2340-2346) plus -eta J (:2347-2364) */
    double *ej = NULL;
    if (c->p.laplacian) {
      size_t np = (size_t)c->nth * c->nphi;
      double *J = dalloc(3 * n);
      ej = dalloc(3 * n);
      vector_curl_b(c, vars1 + 5 * n, J);
      const double jconst = 4.0 * PI / (C_LIGHT * C_LIGHT);
      for (size_t i = 0; i < n; i++) {
        double etar = c->ks[i / np];
        for (int k = 0; k < 3; k++) ej[k * n + i] = -etar * J[k * n + i];
        dvars1[4 * n + i] = dvars1[4 * n + i] + (jconst * etar) *
                                                    (J[i] * J[i] + J[n + i] * J[n + i] + J[2 * n + i] * J[2 * n + i]) *
                                                    c->invrho[i] / c->temperature[i];
      }
      free(J);
    }
    const double *w = vars1 + n, *v = vars1 + 2 * n, *u = vars1 + 3 * n;
    const double *bt = vars1 + 5 * n, *bp = vars1 + 6 * n, *br = vars1 + 7 * n;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) {
      dvars1[5 * n + i] = v[i] * br[i] - u[i] * bp[i];
      dvars1[6 * n + i] = u[i] * bt[i] - w[i] * br[i];
      dvars1[7 * n + i] = w[i] * bp[i] - v[i] * bt[i];
    }
    if (ej) {
      for (size_t i = 0; i < 3 * n; i++) dvars1[5 * n + i] = dvars1[5 * n + i] + ej[i];
      free(ej);
    }
    if (call_num > 1) memcpy(vars1 + 5 * n, c->maga, sizeof(double) * 3 * n);
  }
  if (c->p.xi_cs < 1.0)
    for (size_t i = 0; i < n; i++) dvars1[i] = (c->p.xi_cs * c->p.xi_cs) * dvars1[i];
  return CSS_OK;
}

/* ------------------------------------------------------------------------ */
/* Compute_Diffusion (diffusion.f90:70-474)                                 */
/* ------------------------------------------------------------------------ */
static inline double limiter(double q, double qph, double tiny) {
  /* Van Albada-type slope limiter, diffusion.f90:749-754 */
  double rtmp = fabs(q);
  rtmp = 1.0 / fmax(rtmp, tiny);
  rtmp = q * (rtmp * rtmp);
  rtmp = rtmp * qph;
  rtmp = fmin(1.0, rtmp);
  return q * fmax(0.0, rtmp);
}

/* vcc of block B at local (jt, jp, jr), each in 0..n+1 (ghost rings) */
typedef struct { int nt, np, nr; double *v; } vcc_t;
#define VCC(V, jt, jp, jr) (V).v[(jt) + ((V).nt + 2) * ((jp) + ((V).np + 2) * (size_t)(jr))]

static void build_vcc(orc_ctx *c, const blk_t *B, const double *v1, vcc_t *V) {
  const css_params *p = &c->p;
  size_t n = c->ncell;
  int nth = c->nth, nphi = c->nphi;
  V->nt = B->nt; V->np = B->np; V->nr = B->nr;
  V->v = dalloc((size_t)(B->nt + 2) * (B->np + 2) * (B->nr + 2));
  /* vcc(:,:,ir) = diffusion_speed(ir) at the radius of local index ir */
  for (int jr = 0; jr <= B->nr + 1; jr++) {
    int gr = B->r0 + jr - 1;
    if (gr < 0) gr = 0;
    if (gr > c->nr - 1) gr = c->nr - 1;
    for (int jp = 0; jp <= B->np + 1; jp++)
      for (int jt = 0; jt <= B->nt + 1; jt++) VCC(*V, jt, jp, jr) = c->dspeed[gr];
  }
  if (p->dstype == 1) {
    for (int iv = 1; iv <= 3; iv++) {
      const double *f = v1 + (size_t)iv * n;
      if (!B->rlo)
        for (int jp = 1; jp <= B->np; jp++)
          for (int jt = 1; jt <= B->nt; jt++) {
            double q = f[IDX(c, B->t0 + jt - 1, B->p0 + jp - 1, B->r0 - 1)];
            VCC(*V, jt, jp, 0) += q * q;
          }
      for (int jr = 1; jr <= B->nr; jr++) {
        int gr = B->r0 + jr - 1;
        for (int jt = 1; jt <= B->nt; jt++) {
          double q = f[IDX(c, B->t0 + jt - 1, (B->p0 - 1 + nphi) % nphi, gr)];
          VCC(*V, jt, 0, jr) += q * q;
        }
        for (int jp = 1; jp <= B->np; jp++) {
          int gp = B->p0 + jp - 1;
          if (!B->tlo) {
            double q = f[IDX(c, B->t0 - 1, gp, gr)];
            VCC(*V, 0, jp, jr) += q * q;
          }
          for (int jt = 1; jt <= B->nt; jt++) {
            double q = f[IDX(c, B->t0 + jt - 1, gp, gr)];
            VCC(*V, jt, jp, jr) += q * q;
          }
          if (!B->thi) {
            double q = f[IDX(c, B->t0 + B->nt, gp, gr)];
            VCC(*V, B->nt + 1, jp, jr) += q * q;
          }
        }
        for (int jt = 1; jt <= B->nt; jt++) {
          double q = f[IDX(c, B->t0 + jt - 1, (B->p0 + B->np) % nphi, gr)];
          VCC(*V, jt, B->np + 1, jr) += q * q;
        }
      }
      if (!B->rhi)
        for (int jp = 1; jp <= B->np; jp++)
          for (int jt = 1; jt <= B->nt; jt++) {
            double q = f[IDX(c, B->t0 + jt - 1, B->p0 + jp - 1, B->r0 + B->nr)];
            VCC(*V, jt, jp, B->nr + 1) += q * q;
          }
    }
    if (p->magnetic) {
      const double *rho = v1;
      for (int iv = 5; iv <= 7; iv++) {
        const double *f = v1 + (size_t)iv * n;
#define GH(id) (ONE_OVER_4PI * (f[id] * f[id]) / rho[id])
        if (!B->rlo)
          for (int jp = 1; jp <= B->np; jp++)
            for (int jt = 1; jt <= B->nt; jt++)
              VCC(*V, jt, jp, 0) += GH(IDX(c, B->t0 + jt - 1, B->p0 + jp - 1, B->r0 - 1));
        for (int jr = 1; jr <= B->nr; jr++) {
          int gr = B->r0 + jr - 1;
          for (int jt = 1; jt <= B->nt; jt++)
            VCC(*V, jt, 0, jr) += GH(IDX(c, B->t0 + jt - 1, (B->p0 - 1 + nphi) % nphi, gr));
          for (int jp = 1; jp <= B->np; jp++) {
            int gp = B->p0 + jp - 1;
            if (!B->tlo) VCC(*V, 0, jp, jr) += GH(IDX(c, B->t0 - 1, gp, gr));
            for (int jt = 1; jt <= B->nt; jt++) {
              size_t id = IDX(c, B->t0 + jt - 1, gp, gr);
              VCC(*V, jt, jp, jr) += ONE_OVER_4PI * c->invrho[id] * (f[id] * f[id]);
            }
            if (!B->thi) VCC(*V, B->nt + 1, jp, jr) += GH(IDX(c, B->t0 + B->nt, gp, gr));
          }
          for (int jt = 1; jt <= B->nt; jt++)
            VCC(*V, jt, B->np + 1, jr) += GH(IDX(c, B->t0 + jt - 1, (B->p0 + B->np) % nphi, gr));
        }
        if (!B->rhi)
          for (int jp = 1; jp <= B->np; jp++)
            for (int jt = 1; jt <= B->nt; jt++)
              VCC(*V, jt, jp, B->nr + 1) += GH(IDX(c, B->t0 + jt - 1, B->p0 + jp - 1, B->r0 + B->nr));
#undef GH
      }
    }
  }
  /* copy into the ghost ring at physical faces (diffusion.f90:288-302) */
  if (B->rlo)
    for (int jp = 0; jp <= B->np + 1; jp++)
      for (int jt = 0; jt <= B->nt + 1; jt++) VCC(*V, jt, jp, 0) = VCC(*V, jt, jp, 1);
  if (B->rhi)
    for (int jp = 0; jp <= B->np + 1; jp++)
      for (int jt = 0; jt <= B->nt + 1; jt++) VCC(*V, jt, jp, B->nr + 1) = VCC(*V, jt, jp, B->nr);
  if (B->tlo)
    for (int jr = 0; jr <= B->nr + 1; jr++)
      for (int jp = 0; jp <= B->np + 1; jp++) VCC(*V, 0, jp, jr) = VCC(*V, 1, jp, jr);
  if (B->thi)
    for (int jr = 0; jr <= B->nr + 1; jr++)
      for (int jp = 0; jp <= B->np + 1; jp++) VCC(*V, B->nt + 1, jp, jr) = VCC(*V, B->nt, jp, jr);
  (void)nth;
}

/* field values used by the SLD sweeps: rho and s mean-subtracted in v1
 * already, A from avec for iv >= 5 (maga in the reference) */
static inline const double *sld_field(orc_ctx *c, const double *v1, const double *avec, int iv) {
  size_t n = c->ncell;
  if (iv >= 5) return avec + (size_t)(iv - 5) * n;
  return v1 + (size_t)iv * n;
}

static double prandtl_r(const css_params *p, int iv1) {
  /* diffusion.f90:854-862: iv <= 3 -> sld_pr, iv >= 5 -> sld_prm (1-based iv) */
  if ((p->sld_pr != 1.0) || (p->sld_prm != 1.0)) {
    if (iv1 <= 3) return p->sld_pr;
    if (iv1 >= 5) return p->sld_prm;
  }
  return 1.0;
}
static double prandtl_tp(const css_params *p, int iv1) {
  /* diffusion.f90:1255-1263, :1473-1481: iv < 5 -> sld_pr, iv > 5 -> sld_prm */
  if ((p->sld_pr != 1.0) || (p->sld_prm != 1.0)) {
    if (iv1 < 5) return p->sld_pr;
    if (iv1 > 5) return p->sld_prm;
  }
  return 1.0;
}

static void diffusion_r(orc_ctx *c, const blk_t *B, const vcc_t *V, const double *v1, const double *avec,
                        double *dv1, int iv, double tiny) {
  const css_params *p = &c->p;
  size_t n = c->ncell;
  int iv1 = iv + 1;
  const double *f = sld_field(c, v1, avec, iv);
  double pr = prandtl_r(p, iv1);
  int myr1 = B->r0, myr2 = B->r0 + B->nr - 1, nr = c->nr;
#pragma omp parallel for collapse(2) schedule(static)
  for (int ip = B->p0; ip < B->p0 + B->np; ip++)
    for (int it = B->t0; it < B->t0 + B->nt; it++) {
      int m = B->nr;
      double tmp[m + 2], b1[5], b2[5], qmh[m + 3], qph[m + 3], qp3h[m + 3], de[m + 3], rph[m + 3];
      for (int j = 1; j <= m; j++) tmp[j] = f[IDX(c, it, ip, myr1 + j - 1)];
      for (int k = 1; k <= 4; k++) { b1[k] = 0.0; b2[k] = 0.0; }
      if (!B->rlo) for (int k = 1; k <= 4; k++) b1[k] = f[IDX(c, it, ip, myr1 - 5 + k)];
      if (!B->rhi) for (int k = 1; k <= 4; k++) b2[k] = f[IDX(c, it, ip, myr2 + k)];
      const double *ri = c->r_ind, *dri = c->dr_ind;
      if (B->rlo) {
        switch (iv1) {
          case 1: for (int k = 1; k <= 4; k++) b1[k] = 0.0; break;
          case 2: case 3:
            b1[1] = tmp[1]; b1[2] = tmp[1];
            b1[4] = -10.0 * ONETHIRD * tmp[1] / ri[0] + 6.0 * tmp[2] / ri[1] - 2.0 * tmp[3] / ri[2] + ONETHIRD * tmp[4] / ri[3];
            b1[3] = 8.0 * b1[4] / (ri[0] - dri[0]) - 8.0 * tmp[2] / ri[1] + tmp[3] / ri[2];
            break;
          case 4: for (int k = 1; k <= 4; k++) b1[k] = tmp[1]; break;
          case 5:
            if (!p->bottom_constant_temp && c->cond) {
              double q = p->lumr1 * ONE_OVER_4PI / (p->r1 * p->r1 * c->ks[0] * c->dxdr[0]);
              b1[1] = tmp[1] + 4.0 * dri[0] * q; b1[2] = tmp[1] + 3.0 * dri[0] * q;
              b1[3] = tmp[1] + 2.0 * dri[0] * q; b1[4] = tmp[1] + dri[0] * q;
            } else for (int k = 1; k <= 4; k++) b1[k] = 0.0;
            break;
          case 6: case 7:
            if (p->bottom_perfect_cond) for (int k = 1; k <= 4; k++) b1[k] = 0.0;
            else for (int k = 1; k <= 4; k++) b1[k] = tmp[1];
            break;
          default: for (int k = 1; k <= 4; k++) b1[k] = tmp[1]; break;
        }
      }
      if (B->rhi) {
        switch (iv1) {
          case 1: for (int k = 1; k <= 4; k++) b2[k] = 0.0; break;
          case 2: case 3:
            b2[1] = -10.0 * ONETHIRD * tmp[m] / ri[nr - 1] + 6.0 * tmp[m - 1] / ri[nr - 2] - 2.0 * tmp[m - 2] / ri[nr - 3] + ONETHIRD * tmp[m - 3] / ri[nr - 4];
            b2[2] = tmp[m - 2] / ri[nr - 3] - 8.0 * tmp[m - 1] / ri[nr - 2] + 8.0 * b2[1] / (ri[nr - 1] + dri[nr - 1]);
            b2[3] = tmp[m]; b2[4] = tmp[m];
            break;
          case 4: for (int k = 1; k <= 4; k++) b2[k] = tmp[m]; break;
          case 5:
            if (!p->top_constant_temp && c->cond) {
              double q = p->lumr2 * ONE_OVER_4PI / (p->r2 * p->r2 * c->ks[nr - 1] * c->dxdr[nr - 1]);
              b2[1] = tmp[m] - dri[0] * q; b2[2] = tmp[m] - 2.0 * dri[0] * q;
              b2[3] = tmp[m] - 3.0 * dri[0] * q; b2[4] = tmp[m] - 4.0 * dri[0] * q;
            } else for (int k = 1; k <= 4; k++) b2[k] = 0.0;
            break;
          case 6: case 7:
            if (p->top_perfect_cond) for (int k = 1; k <= 4; k++) b2[k] = 0.0;
            else for (int k = 1; k <= 4; k++) b2[k] = tmp[m];
            break;
          default: for (int k = 1; k <= 4; k++) b2[k] = tmp[m]; break;
        }
      }
      qmh[1] = b1[4] - b1[3];
      qmh[2] = tmp[1] - b1[4];
      for (int j = 3; j <= m + 1; j++) qmh[j] = tmp[j - 1] - tmp[j - 2];
      for (int j = 1; j <= m; j++) qph[j] = qmh[j + 1];
      qph[m + 1] = b2[1] - tmp[m];
      for (int j = 1; j <= m; j++) qp3h[j] = qph[j + 1];
      qp3h[m + 1] = b2[2] - b2[1];
      for (int j = 1; j <= m + 1; j++) {
        double pl = limiter(qmh[j], qph[j], tiny);
        double pr_ = limiter(qp3h[j], qph[j], tiny);
        de[j] = qph[j] - 0.5 * (pr_ + pl);
      }
      if (B->rlo) { rph[1] = ri[0] - 0.5 * dri[0]; de[1] = 0.0; }
      else { rph[1] = 0.5 * (ri[myr1 - 1] + ri[myr1]); de[1] = de[1] * (rph[1] * rph[1]); }
      for (int j = 2; j <= m; j++) rph[j] = 0.5 * (ri[myr1 + j - 1] + ri[myr1 + j - 2]);
      for (int j = 2; j <= m; j++) de[j] = de[j] * (rph[j] * rph[j]);
      if (B->rhi) { rph[m + 1] = ri[myr2] + 0.5 * dri[myr2]; de[m + 1] = 0.0; }
      else { rph[m + 1] = 0.5 * (ri[myr2 + 1] + ri[myr2]); de[m + 1] = de[m + 1] * (rph[m + 1] * rph[m + 1]); }
      int jt = it - B->t0 + 1, jp = ip - B->p0 + 1;
      for (int j = 1; j <= m + 1; j++) {
        double vt = p->sld_coef * sqrt(0.5 * (VCC(*V, jt, jp, j) + VCC(*V, jt, jp, j - 1)));
        de[j] = vt * de[j];
      }
      for (int j = 1; j <= m; j++) {
        double t3 = rph[j + 1] * rph[j + 1] * rph[j + 1] - rph[j] * rph[j] * rph[j];
        t3 = 3.0 / t3;
        double flux = t3 * (de[j + 1] - de[j]);
        if (pr != 1.0) flux = pr * flux;
        size_t id = IDX(c, it, ip, myr1 + j - 1);
        dv1[(size_t)iv * n + id] = dv1[(size_t)iv * n + id] + flux;
      }
    }
}

static void diffusion_th(orc_ctx *c, const blk_t *B, const vcc_t *V, const double *v1, const double *avec,
                         double *dv1, int iv, double tiny) {
  const css_params *p = &c->p;
  size_t n = c->ncell;
  int iv1 = iv + 1;
  const double *f = sld_field(c, v1, avec, iv);
  double pr = prandtl_tp(p, iv1);
  int myt1 = B->t0, myt2 = B->t0 + B->nt - 1, nth = c->nth;
  const double *th = c->theta, *sn = c->sines;
  double dth = c->dth;
#pragma omp parallel for collapse(2) schedule(static)
  for (int ir = B->r0; ir < B->r0 + B->nr; ir++)
    for (int ip = B->p0; ip < B->p0 + B->np; ip++) {
      int m = B->nt;
      double tmp[m + 2], b1[5], b2[5], qmh[m + 3], qph[m + 3], qp3h[m + 3], de[m + 3], sph[m + 3], cph[m + 3];
      for (int j = 1; j <= m; j++) tmp[j] = f[IDX(c, myt1 + j - 1, ip, ir)];
      for (int k = 1; k <= 4; k++) { b1[k] = 0.0; b2[k] = 0.0; }
      if (!B->tlo) for (int k = 1; k <= 4; k++) b1[k] = f[IDX(c, myt1 - 5 + k, ip, ir)];
      if (!B->thi) for (int k = 1; k <= 4; k++) b2[k] = f[IDX(c, myt2 + k, ip, ir)];
      if (B->tlo) {
        switch (iv1) {
          case 2: for (int k = 1; k <= 4; k++) b1[k] = 0.0; break;
          case 3:
            b1[1] = tmp[1]; b1[2] = tmp[1];
            b1[4] = -10.0 * ONETHIRD * tmp[1] / sn[0] + 6.0 * tmp[2] / sn[1] - 2.0 * tmp[3] / sn[2] + ONETHIRD * tmp[4] / sn[3];
            b1[3] = 8.0 * b1[4] / sin(th[0] - dth) - 8.0 * tmp[2] / sn[1] + tmp[3] / sn[2];
            break;
          case 6:
            if (p->theta_normal_field) for (int k = 1; k <= 4; k++) b1[k] = 0.0;
            else for (int k = 1; k <= 4; k++) b1[k] = tmp[1];
            break;
          case 7: case 8:
            if (p->theta_perf_conductor) for (int k = 1; k <= 4; k++) b1[k] = 0.0;
            else for (int k = 1; k <= 4; k++) b1[k] = tmp[1];
            break;
          default: for (int k = 1; k <= 4; k++) b1[k] = tmp[1]; break;
        }
      }
      if (B->thi) {
        switch (iv1) {
          case 2: for (int k = 1; k <= 4; k++) b2[k] = 0.0; break;
          case 3:
            b2[1] = -10.0 * ONETHIRD * tmp[m] / sn[nth - 1] + 6.0 * tmp[m - 1] / sn[nth - 2] - 2.0 * tmp[m - 2] / sn[nth - 3] + ONETHIRD * tmp[m - 3] / sn[nth - 4];
            b2[2] = tmp[m - 2] / sn[nth - 3] - 8.0 * tmp[m - 1] / sn[nth - 2] + 8.0 * b2[1] / sin(th[nth - 1] + dth);
            b2[3] = tmp[m]; b2[4] = tmp[m];
            break;
          case 6:
            if (p->theta_normal_field) for (int k = 1; k <= 4; k++) b2[k] = 0.0;
            else for (int k = 1; k <= 4; k++) b2[k] = tmp[m];
            break;
          case 7: case 8:
            if (p->theta_perf_conductor) for (int k = 1; k <= 4; k++) b2[k] = 0.0;
            else for (int k = 1; k <= 4; k++) b2[k] = tmp[m];
            break;
          default: for (int k = 1; k <= 4; k++) b2[k] = tmp[m]; break;
        }
      }
      qmh[1] = b1[4] - b1[3];
      qmh[2] = tmp[1] - b1[4];
      for (int j = 3; j <= m + 1; j++) qmh[j] = tmp[j - 1] - tmp[j - 2];
      for (int j = 1; j <= m; j++) qph[j] = qmh[j + 1];
      qph[m + 1] = b2[1] - tmp[m];
      for (int j = 1; j <= m; j++) qp3h[j] = qph[j + 1];
      qp3h[m + 1] = b2[2] - b2[1];
      for (int j = 1; j <= m + 1; j++) {
        double pl = limiter(qmh[j], qph[j], tiny);
        double pr_ = limiter(qp3h[j], qph[j], tiny);
        de[j] = qph[j] - 0.5 * (pr_ + pl);
      }
      if (B->tlo) {
        de[1] = 0.0;
        sph[1] = fabs(sin(th[0] - 0.5 * dth));
        cph[1] = cos(th[0] - 0.5 * dth);
      } else {
        sph[1] = sin(0.5 * (th[myt1 - 1] + th[myt1]));
        cph[1] = cos(0.5 * (th[myt1 - 1] + th[myt1]));
      }
      for (int j = 2; j <= m; j++) {
        sph[j] = sin(0.5 * (th[myt1 + j - 1] + th[myt1 + j - 2]));
        cph[j] = cos(0.5 * (th[myt1 + j - 1] + th[myt1 + j - 2]));
      }
      if (B->thi) {
        de[m + 1] = 0.0;
        sph[m + 1] = sin(th[myt2] + 0.5 * dth);
        cph[m + 1] = cos(th[myt2] + 0.5 * dth);
      } else {
        sph[m + 1] = sin(0.5 * (th[myt2] + th[myt2 + 1]));
        cph[m + 1] = cos(0.5 * (th[myt2] + th[myt2 + 1]));
      }
      int jp = ip - B->p0 + 1, jr = ir - B->r0 + 1;
      for (int j = 1; j <= m + 1; j++) {
        double vt = p->sld_coef * sqrt(0.5 * (VCC(*V, j, jp, jr) + VCC(*V, j - 1, jp, jr)));
        de[j] = vt * sph[j] * de[j];
      }
      double stmp, rtmp;
      if (B->rlo && ir == B->r0) stmp = c->r_ind[0] - 0.5 * c->dr_ind[0];
      else stmp = 0.5 * (c->r_ind[ir] + c->r_ind[ir - 1]);
      if (B->rhi && ir == B->r0 + B->nr - 1) rtmp = c->r_ind[c->nr - 1] + 0.5 * c->dr_ind[c->nr - 1];
      else rtmp = 0.5 * (c->r_ind[ir + 1] + c->r_ind[ir]);
      rtmp = 1.5 * (rtmp * rtmp - stmp * stmp) / (rtmp * rtmp * rtmp - stmp * stmp * stmp);
      for (int j = 1; j <= m; j++) {
        double t = rtmp / (cph[j] - cph[j + 1]);
        double flux = t * (de[j + 1] - de[j]);
        if (pr != 1.0) flux = pr * flux;
        size_t id = IDX(c, myt1 + j - 1, ip, ir);
        dv1[(size_t)iv * n + id] = dv1[(size_t)iv * n + id] + flux;
      }
    }
}

static void diffusion_phi(orc_ctx *c, const blk_t *B, const vcc_t *V, const double *v1, const double *avec,
                          double *dv1, int iv, double tiny) {
  const css_params *p = &c->p;
  size_t n = c->ncell;
  int iv1 = iv + 1;
  const double *f = sld_field(c, v1, avec, iv);
  double pr = prandtl_tp(p, iv1);
  int nth = c->nth, nphi = c->nphi;
  const double *th = c->theta;
  double dth = c->dth;
#pragma omp parallel for collapse(2) schedule(static)
  for (int ir = B->r0; ir < B->r0 + B->nr; ir++)
    for (int it = B->t0; it < B->t0 + B->nt; it++) {
      int m = B->np, p0 = B->p0;
      double rtmp, stmp, ctmp;
      /* geom (diffusion.f90:1316-1351) for global theta index it */
      if (it == 0) { rtmp = th[0] - 0.5 * dth; stmp = cos(rtmp); }
      else { rtmp = 0.5 * (th[it] + th[it - 1]); stmp = cos(rtmp); }
      if (it == nth - 1) { ctmp = th[it] + 0.5 * dth; rtmp = ctmp - rtmp; ctmp = cos(ctmp); }
      else { ctmp = 0.5 * (th[it + 1] + th[it]); rtmp = ctmp - rtmp; ctmp = cos(ctmp); }
      double geom = rtmp / (stmp - ctmp);
      double sr_, rr_;
      if (B->rlo && ir == B->r0) sr_ = c->r_ind[0] - 0.5 * c->dr_ind[0];
      else sr_ = 0.5 * (c->r_ind[ir] + c->r_ind[ir - 1]);
      if (B->rhi && ir == B->r0 + B->nr - 1) rr_ = c->r_ind[c->nr - 1] + 0.5 * c->dr_ind[c->nr - 1];
      else rr_ = 0.5 * (c->r_ind[ir + 1] + c->r_ind[ir]);
      rr_ = 1.5 * (rr_ * rr_ - sr_ * sr_) / (rr_ * rr_ * rr_ - sr_ * sr_ * sr_) / c->dphi;
      geom = geom * rr_;
      double tmp[m + 2], b1[5], b2[5], qmh[m + 3], qph[m + 3], qp3h[m + 3], de[m + 3];
      for (int j = 1; j <= m; j++) tmp[j] = f[IDX(c, it, p0 + j - 1, ir)];
      for (int k = 1; k <= 4; k++) {
        b1[k] = f[IDX(c, it, (p0 - 5 + k + nphi) % nphi, ir)];
        b2[k] = f[IDX(c, it, (p0 + m + k - 1) % nphi, ir)];
      }
      qmh[1] = b1[4] - b1[3];
      qmh[2] = tmp[1] - b1[4];
      for (int j = 3; j <= m + 1; j++) qmh[j] = tmp[j - 1] - tmp[j - 2];
      for (int j = 1; j <= m; j++) qph[j] = qmh[j + 1];
      qph[m + 1] = b2[1] - tmp[m];
      for (int j = 1; j <= m; j++) qp3h[j] = qph[j + 1];
      qp3h[m + 1] = b2[2] - b2[1];
      for (int j = 1; j <= m + 1; j++) {
        double pl = limiter(qmh[j], qph[j], tiny);
        double pr_ = limiter(qp3h[j], qph[j], tiny);
        de[j] = qph[j] - 0.5 * (pr_ + pl);
      }
      int jt = it - B->t0 + 1, jr = ir - B->r0 + 1;
      for (int j = 1; j <= m + 1; j++) {
        double vt = p->sld_coef * sqrt(0.5 * (VCC(*V, jt, j - 1, jr) + VCC(*V, jt, j, jr)));
        de[j] = vt * de[j];
      }
      for (int j = 1; j <= m; j++) {
        double flux = de[j + 1] - de[j];
        if (pr != 1.0) flux = pr * flux;
        size_t id = IDX(c, it, p0 + j - 1, ir);
        dv1[(size_t)iv * n + id] = dv1[(size_t)iv * n + id] + geom * flux;
      }
    }
}

int orc_diffusion(orc_ctx *c, double *vars1, const double *avec, double *dvars1) {
  const css_params *p = &c->p;
  size_t n = c->ncell;
  int nv = c->nv;
  if (p->magnetic && !avec) { set_err("orc_diffusion: MHD needs the vector potential"); return CSS_ERR_ARG; }
  if (p->magnetic && p->do_ohmic_heating && !p->magnetic_diffusion) {
    set_err("orc_diffusion: ohmic heating needs magnetic diffusion");
    return CSS_ERR_ARG;
  }
  memset(dvars1, 0, sizeof(double) * n * nv);
  double tinyvar[8] = {1e-8 * c->rhor[c->nr - 1], 1e-8, 1e-8, 1e-8, 1e-8 * 1e5, 1e-8 * 1e8, 1e-8 * 1e8, 1e-8 * 1e8};
  int varlist[8], nsld = 0;
  if (p->magnetic && p->magnetic_diffusion) {
    if (p->mass_diffusion) varlist[nsld++] = 0;
    for (int i = 1; i <= 7; i++) varlist[nsld++] = i;
  } else {
    if (p->mass_diffusion) varlist[nsld++] = 0;
    for (int i = 1; i <= 4; i++) varlist[nsld++] = i;
  }
  /* invrho and inverse temperature before the mean subtraction (:117-123) */
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; i++) {
    c->invrho[i] = 1.0 / vars1[i];
    c->temperature[i] = (pow(vars1[i], -c->gamm1)) * exp(-vars1[4 * n + i] * c->invcv) / c->invtconst;
  }
  /* vcc from the unmodified velocities / fields (equivalent to building it
   * after the subtraction, which only touches rho and s) */
  vcc_t *V = (vcc_t *)calloc(c->nblk, sizeof(vcc_t));
  for (int k = 0; k < c->nblk; k++) build_vcc(c, &c->blk[k], vars1, &V[k]);
  /* meanV = (rhor, sr) (update_background off), subtracted in place */
  for (int ir = 0; ir < c->nr; ir++)
    for (int q = 0; q < c->nth * c->nphi; q++) {
      size_t id = (size_t)ir * c->nth * c->nphi + q;
      vars1[id] = vars1[id] - c->rhor[ir];
      vars1[4 * n + id] = vars1[4 * n + id] - c->sr[ir];
    }
  for (int isl = 0; isl < nsld; isl++)
    for (int k = 0; k < c->nblk; k++)
      diffusion_r(c, &c->blk[k], &V[k], vars1, avec, dvars1, varlist[isl], tinyvar[varlist[isl]]);
  for (int isl = 0; isl < nsld; isl++)
    for (int k = 0; k < c->nblk; k++)
      diffusion_th(c, &c->blk[k], &V[k], vars1, avec, dvars1, varlist[isl], tinyvar[varlist[isl]]);
  for (int isl = 0; isl < nsld; isl++)
    for (int k = 0; k < c->nblk; k++)
      diffusion_phi(c, &c->blk[k], &V[k], vars1, avec, dvars1, varlist[isl], tinyvar[varlist[isl]]);
  for (int k = 0; k < c->nblk; k++) free(V[k].v);
  free(V);
  if (p->do_viscous_heating)
    for (int iv = 1; iv <= 3; iv++)
#pragma omp parallel for schedule(static)
      for (size_t i = 0; i < n; i++)
        dvars1[4 * n + i] = dvars1[4 * n + i] - vars1[(size_t)iv * n + i] * dvars1[(size_t)iv * n + i] * c->temperature[i];
  if (p->mass_diffusion) {
    for (int iv = 1; iv <= 3; iv++)
#pragma omp parallel for schedule(static)
      for (size_t i = 0; i < n; i++)
        dvars1[(size_t)iv * n + i] = dvars1[(size_t)iv * n + i] - c->invrho[i] * vars1[(size_t)iv * n + i] * dvars1[i];
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++)
      dvars1[4 * n + i] = dvars1[4 * n + i] - (c->gamm1 * c->cv) * c->invrho[i] * dvars1[i];
  }
  if (p->magnetic && p->do_ohmic_heating) {
    /* curl of the A-tendency; heating -B.curl(D_A)/(8 pi rho T) (:430-461) */
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) c->temperature[i] = (0.5 * ONE_OVER_4PI) * c->invrho[i] * c->temperature[i];
    double *da = c->da; /* copy of dvars1(6:8), restored below */
    memcpy(da, dvars1 + 5 * n, sizeof(double) * 3 * n);
    vector_curl_a(c, da, dvars1 + 5 * n);
    for (int iv = 5; iv <= 7; iv++)
#pragma omp parallel for schedule(static)
      for (size_t i = 0; i < n; i++)
        dvars1[4 * n + i] = dvars1[4 * n + i] - vars1[(size_t)iv * n + i] * dvars1[(size_t)iv * n + i] * c->temperature[i];
    memcpy(dvars1 + 5 * n, da, sizeof(double) * 3 * n);
  }
  return CSS_OK;
}

/* ------------------------------------------------------------------------ */
/* Bound (rhs_mpi.f90:2395-2491) and Step_RK4 (step_rk4.f90:339-493)        */
/* ------------------------------------------------------------------------ */
static void bound(orc_ctx *c, double *v1) {
  const css_params *p = &c->p;
  size_t n = c->ncell;
  int nth = c->nth, nphi = c->nphi, nr = c->nr;
  for (int ir = 0; ir < nr; ir++)
    for (int ip = 0; ip < nphi; ip++) {
      v1[n + IDX(c, 0, ip, ir)] = 0.0;
      if (!p->theta_stress_free) v1[3 * n + IDX(c, 0, ip, ir)] = 0.0;
      v1[n + IDX(c, nth - 1, ip, ir)] = 0.0;
      if (!p->theta_stress_free) v1[3 * n + IDX(c, nth - 1, ip, ir)] = 0.0;
    }
  for (int ip = 0; ip < nphi; ip++)
    for (int it = 0; it < nth; it++) {
      size_t lo = IDX(c, it, ip, 0), hi = IDX(c, it, ip, nr - 1);
      if (!p->bottom_stress_free) { v1[n + lo] = 0.0; v1[2 * n + lo] = 0.0; }
      if (!p->bot_inout) v1[3 * n + lo] = 0.0;
      if (p->bottom_constant_temp) {
        /* sr1 = vars1(:,1,1,5) of the initial state; not restated: the
         * parity configs use a constant-flux bottom */
      }
      if (!p->top_inout) { /* an open top keeps every field (rhs_mpi.f90:2420-2432) */
        if (!p->top_stress_free) { v1[n + hi] = 0.0; v1[2 * n + hi] = 0.0; }
        v1[3 * n + hi] = 0.0;
      }
    }
  if (p->magnetic) {
    for (int ir = 0; ir < nr; ir++)
      for (int ip = 0; ip < nphi; ip++) {
        if (p->theta_perf_conductor) {
          v1[6 * n + IDX(c, 0, ip, ir)] = 0.0; v1[7 * n + IDX(c, 0, ip, ir)] = 0.0;
          v1[6 * n + IDX(c, nth - 1, ip, ir)] = 0.0; v1[7 * n + IDX(c, nth - 1, ip, ir)] = 0.0;
        } else {
          v1[5 * n + IDX(c, 0, ip, ir)] = 0.0;
          v1[5 * n + IDX(c, nth - 1, ip, ir)] = 0.0;
        }
      }
    for (int ip = 0; ip < nphi; ip++)
      for (int it = 0; it < nth; it++) {
        size_t lo = IDX(c, it, ip, 0), hi = IDX(c, it, ip, nr - 1);
        if (p->bottom_radial_field) v1[7 * n + lo] = 0.0;
        else if (p->bottom_perfect_cond) { v1[5 * n + lo] = 0.0; v1[6 * n + lo] = 0.0; }
        if (p->top_radial_field) v1[7 * n + hi] = 0.0;
        else if (p->top_perfect_cond) { v1[5 * n + hi] = 0.0; v1[6 * n + hi] = 0.0; }
      }
  }
}

/* The clock around one step (Program CSS2, mhdsph_mpi.f90:28-43): the step
 * index advances before the step and the time after it; with a prescribed
 * bottom the ASH fields are interpolated at the step's start time
 * (Read_ASH_Inflow -> Cubic_Time_Interp, ash_inflow.f90:124-219) and every
 * ufreq steps the enthalpy-flux factor is updated at its end
 * (ASH_Enthalpy_Flux, step_rk4.f90:477-482, :495-518). */
static void ash_interp(orc_ctx *c) {
  size_t np = (size_t)c->nth * c->nphi;
  double mu = (c->sim_time - c->ash_times[1]) / (c->ash_times[2] - c->ash_times[1]);
  double mu2 = mu * mu, mu3 = mu * mu2;
  for (int iq = 0; iq < 4; iq++)
    for (size_t q = 0; q < np; q++) {
      double t1 = c->ash_slices[(0 * 4 + iq) * np + q], a3 = c->ash_slices[(1 * 4 + iq) * np + q];
      double t3 = c->ash_slices[(2 * 4 + iq) * np + q], t4 = c->ash_slices[(3 * 4 + iq) * np + q];
      double a0 = -0.5 * t1 + 1.5 * a3 - 1.5 * t3 + 0.5 * t4;
      double a1 = t1 - 2.5 * a3 + 2.0 * t3 - 0.5 * t4;
      double a2 = -0.5 * t1 + 0.5 * t3;
      c->ashv[iq * np + q] = a0 * mu3 + a1 * mu2 + a2 * mu + a3;
    }
}

static void ash_refresh(orc_ctx *c) {
  if (c->p.bottom_specified && c->ash_times[2] > c->ash_times[1]) ash_interp(c);
}

static int step_begin(orc_ctx *c, double dt) {
  c->istep++;
  c->deltat = dt;
  if (c->p.bottom_specified) {
    if (!(c->sim_time < c->ash_times[2])) {
      set_err("step: sim_time %.17g is past the third ASH slice time %.17g; shift in the next slice first",
              c->sim_time, c->ash_times[2]);
      return CSS_ERR_ARG;
    }
    ash_refresh(c);
  }
  return CSS_OK;
}

static void step_end(orc_ctx *c, const double *vars0, double dt) {
  const css_params *p = &c->p;
  if (p->bottom_specified && p->ufreq > 0 && c->istep % p->ufreq == 0) {
    size_t n = c->ncell;
    double ntot = (double)c->nphi * (double)c->nth, su = 0.0, st = 0.0, len = 0.0;
    for (int ip = 0; ip < c->nphi; ip++)
      for (int it = 0; it < c->nth; it++) {
        size_t id = IDX(c, it, ip, 0);
        su = su + vars0[3 * n + id];
        st = st + c->temperature[id]; /* the last RHS's temperature, as the module array holds it */
      }
    double uravg = su / ntot, t2avg = st / ntot;
    for (int ip = 0; ip < c->nphi; ip++)
      for (int it = 0; it < c->nth; it++) {
        size_t id = IDX(c, it, ip, 0);
        len = len + vars0[id] * (vars0[3 * n + id] - uravg) * (c->temperature[id] - t2avg);
      }
    len = p->cp * len / ntot;
    len = 4.0 * PI * (p->r1 * p->r1) * len / p->lumr1;
    len = 1.3 * fmin(1.0 / fmin(2.0, fmax(0.0, fabs(len))), 2.0);
    c->ash_fen_mod = 0.5 * (len + c->ash_fen_mod);
    if (fmin(fabs(c->sim_time) / 1e5, 1.0) < 1.0) c->ash_fen_mod = 1.0;
  }
  c->sim_time = c->sim_time + dt;
}

int orc_set_clock(orc_ctx *c, long long istep, double sim_time, double deltat) {
  c->istep = istep; c->sim_time = sim_time; c->deltat = deltat;
  if (c->ash_slices) ash_refresh(c);
  return CSS_OK;
}

int orc_get_clock(orc_ctx *c, long long *istep, double *sim_time) {
  if (istep) *istep = c->istep;
  if (sim_time) *sim_time = c->sim_time;
  return CSS_OK;
}

/* start-up mass bookkeeping (mhdsph_mpi.f90:863-947, :979-999) */
int orc_inout_init(orc_ctx *c, const double *vars0) {
  double m0 = 0.0, vol = 0.0;
  for (int ir = 0; ir < c->nr; ir++) {
    double radius = c->r_ind[ir], drad = c->dr_ind[ir];
    for (int it = 0; it < c->nth; it++) {
      double sinth = c->sines[it], srho = 0.0;
      for (int ip = 0; ip < c->nphi; ip++) srho = srho + vars0[IDX(c, it, ip, ir)];
      m0 = m0 + radius * radius * sinth * srho * drad * c->dth * c->dphi;
      vol = vol + sinth * radius * radius * drad * c->dth * c->dphi;
    }
  }
  c->m0 = m0;
  c->vol = vol;
  c->mtot = c->p.bot_inout ? mass_total(c, vars0) : m0;
  return CSS_OK;
}

int orc_inout_state(orc_ctx *c, double *out) {
  out[0] = c->m0; out[1] = c->vol; out[2] = c->mtot; out[3] = c->ash_fen_mod;
  return CSS_OK;
}

int orc_set_rain_fields(orc_ctx *c, const double *dvel, const double *dent) {
  if (!c->dvel_rain) { set_err("orc_set_rain_fields: the run has no open boundary"); return CSS_ERR_ARG; }
  size_t np = (size_t)c->nth * c->nphi;
  memcpy(c->dvel_rain, dvel, sizeof(double) * np);
  memcpy(c->dent_rain, dent, sizeof(double) * np);
  return CSS_OK;
}

int orc_rain_fields(orc_ctx *c, double *dvel, double *dent) {
  if (!c->dvel_rain) { set_err("orc_rain_fields: the run has no open boundary"); return CSS_ERR_ARG; }
  size_t np = (size_t)c->nth * c->nphi;
  memcpy(dvel, c->dvel_rain, sizeof(double) * np);
  memcpy(dent, c->dent_rain, sizeof(double) * np);
  return CSS_OK;
}

int orc_set_ash_slices(orc_ctx *c, const double *slices, const double *times, double ash_fen_mod) {
  if (!c->ash_slices) { set_err("orc_set_ash_slices: the run has no open boundary"); return CSS_ERR_ARG; }
  memcpy(c->ash_slices, slices, sizeof(double) * 16 * (size_t)c->nth * c->nphi);
  memcpy(c->ash_times, times, sizeof(double) * 4);
  c->ash_fen_mod = ash_fen_mod;
  ash_refresh(c);
  return CSS_OK;
}

/* Build_Gaussian_Squalls (entropy_rain.f90:423-523; sstruct 1) or
 * Build_Polynomial_Squalls (:525-655; sstruct 0) on the top plane: each
 * top block evaluates the squalls whose centre (loct, locp of Find_Position,
 * :817-824) lies within one block width of it, with the periodic images
 * across phi1/phi2 on the first and last phi blocks; Gaussians below 1e-5
 * (exponent -11.5) are dropped, polynomials beyond the squall's size.  The
 * squall density 1/(1 + sum) (of |term| for the polynomial) then
 * weights each squall's velocity and entropy.  sq: 6 per squall, theta_loc,
 * phi_loc, size, scaling, vel, dels. */
static int squalls_into(orc_ctx *c, int sstruct, int nsq, const double *sq, int add);
int orc_build_squalls(orc_ctx *c, int sstruct, int nsq, const double *sq) { return squalls_into(c, sstruct, nsq, sq, 0); }
/* the squalls on top of the current fields (after the lanes, as
   Update_Rain_Squalls adds them, entropy_rain.f90:171-421) */
int orc_add_squalls(orc_ctx *c, int sstruct, int nsq, const double *sq) { return squalls_into(c, sstruct, nsq, sq, 1); }

static int squalls_into(orc_ctx *c, int sstruct, int nsq, const double *sq, int add) {
  const css_params *p = &c->p;
  if (!c->dvel_rain) { set_err("orc_build_squalls: the run has no open boundary"); return CSS_ERR_ARG; }
  const int poly = sstruct == 0;
  int nth = c->nth, nphi = c->nphi;
  size_t np = (size_t)nth * nphi;
  double *dens = dalloc(np);
  if (!add) {
    memset(c->dvel_rain, 0, sizeof(double) * np);
    memset(c->dent_rain, 0, sizeof(double) * np);
  }
  for (int pass = 0; pass < 2; pass++) {
    for (int k = 0; k < c->nblk; k++) {
      const blk_t *B = &c->blk[k];
      if (!B->rhi) continue;
      int myth1 = B->t0 + 1, myth2 = B->t0 + B->nt, mynth = B->nt;
      int myphi1 = B->p0 + 1, myphi2 = B->p0 + B->np, mynphi = B->np;
      for (int is = 0; is < nsq; is++) {
        const double *q = sq + 6 * is;
        int lct = (int)floor((q[0] - p->th1) / c->dth) + 1, lcp = (int)floor((q[1] - p->phi1) / c->dphi) + 1;
        lct = lct > nth ? nth : (lct < 1 ? 1 : lct);
        lcp = lcp > nphi ? nphi : (lcp < 1 ? 1 : lcp);
        if (!(lct + mynth >= myth1 && lct - mynth <= myth2)) continue;
        double w2 = (p->r2 / q[2]) * (p->r2 / q[2]);
        double shift[3];
        int ns = 0;
        if (lcp + mynphi >= myphi1 && lcp - mynphi <= myphi2) shift[ns++] = 0.0;
        if (lcp + mynphi > nphi && myphi1 == 1) shift[ns++] = 1.0;
        if (lcp - mynphi < 1 && myphi2 == nphi) shift[ns++] = -1.0;
        for (int a = 0; a < ns; a++)
          for (int ip = B->p0; ip < B->p0 + B->np; ip++)
            for (int it = B->t0; it < B->t0 + B->nt; it++) {
              double dt_ = c->theta[it] - q[0], thtmp = dt_ * dt_;
              double dp = c->phi[ip] - q[1];
              if (shift[a] > 0.0) dp = dp + p->phi2 - p->phi1;
              else if (shift[a] < 0.0) dp = dp - p->phi2 + p->phi1;
              size_t id = it + (size_t)nth * ip;
              double val;
              if (poly) { /* Build_Polynomial_Squalls (:525-655) */
                double e = (thtmp + dp * dp) * w2;
                if (!(e <= 1.0)) continue;
                double tt = sqrt(e), x1 = tt * tt, x2 = x1 * tt, x3 = x2 * tt;
                double f = 1.0 - 18.0 * x1 + 32.0 * x2 - 15.0 * x3;
                val = pass == 0 ? fabs(q[3] * f) : q[3] * dens[id] * f;
              } else {
                double e = -(thtmp + dp * dp) * w2;
                if (!(e > -11.5)) continue;
                val = q[3] * exp(e);
                if (pass) val = val * dens[id];
              }
              if (pass == 0) {
                dens[id] = dens[id] + val;
              } else {
                c->dvel_rain[id] = c->dvel_rain[id] + q[4] * val;
                c->dent_rain[id] = c->dent_rain[id] + q[5] * val;
              }
            }
      }
    }
    if (pass == 0)
      for (size_t i = 0; i < np; i++) dens[i] = 1.0 / (dens[i] + 1.0);
  }
  free(dens);
  return CSS_OK;
}

int orc_bound(orc_ctx *c, double *vars1) {
  bound(c, vars1);
  return CSS_OK;
}

/* Step_RK2_TVD / Step_RK3_TVD (step_rk4.f90:31-335): the SLD tendency of
   the step's start (forward Euler) is added once, after the last stage's
   combination and before its Bound */
static void step_tvd(orc_ctx *c, double *vars0, double dt, int order, double *av) {
  const css_params *p = &c->p;
  size_t N = (size_t)c->ncell * c->nv;
  double *v1 = c->vars1, *dv = c->dvars1, *v2 = c->vars2, *vs = c->vars_save;
  const double onethird = 1.0 / 3.0, twothirds = 2.0 / 3.0;
  double dtcur = dt;
  memcpy(v1, vars0, sizeof(double) * N);
  orc_rhs(c, v1, dv, 1);
  if (p->sldiffusion) {
    memcpy(v2, dv, sizeof(double) * N);
    if (p->magnetic) memcpy(av, c->maga, sizeof(double) * 3 * c->ncell);
    orc_diffusion(c, v1, av, dv);
    memcpy(vs, dv, sizeof(double) * N);
    memcpy(dv, v2, sizeof(double) * N);
  }
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < N; i++) v1[i] = vars0[i] + dtcur * dv[i];
  bound(c, v1);
  if (order == 2) {
    dtcur = 0.5 * dt;
    orc_rhs(c, v1, dv, 2);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < N; i++) v1[i] = 0.5 * vars0[i] + 0.5 * v1[i] + dtcur * dv[i];
  } else {
    dtcur = dt / 4.0;
    orc_rhs(c, v1, dv, 2);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < N; i++) v1[i] = 0.75 * vars0[i] + 0.25 * v1[i] + dtcur * dv[i];
    bound(c, v1);
    dtcur = 2.0 * dt / 3.0;
    orc_rhs(c, v1, dv, 3);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < N; i++) v1[i] = onethird * vars0[i] + twothirds * v1[i] + dtcur * dv[i];
  }
  if (p->sldiffusion) {
    dtcur = dt;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < N; i++) v1[i] = v1[i] + dtcur * vs[i];
  }
  bound(c, v1);
  memcpy(vars0, v1, sizeof(double) * N);
}

int orc_step_rk4(orc_ctx *c, double *vars0, double dt, int nsteps) {
  const css_params *p = &c->p;
  size_t N = (size_t)c->ncell * c->nv;
  double *v1 = c->vars1, *dv = c->dvars1, *v2 = c->vars2, *vs = c->vars_save;
  double *av = NULL;
  if (p->magnetic) av = (double *)malloc(sizeof(double) * 3 * c->ncell);
  if (p->time_stepper == 2 || p->time_stepper == 3) {
    for (int step = 0; step < nsteps; step++) {
      int rc = step_begin(c, dt);
      if (rc) { free(av); return rc; }
      step_tvd(c, vars0, dt, p->time_stepper, av);
      step_end(c, vars0, dt);
    }
    free(av);
    return CSS_OK;
  }
  for (int step = 0; step < nsteps; step++) {
    int rc = step_begin(c, dt);
    if (rc) { free(av); return rc; }
    double dtcur = dt / 2.0;
    memcpy(v1, vars0, sizeof(double) * N);
    orc_rhs(c, v1, dv, 1);
    if (p->sldiffusion) {
      memcpy(v2, dv, sizeof(double) * N);
      if (p->magnetic) memcpy(av, c->maga, sizeof(double) * 3 * c->ncell);
      orc_diffusion(c, v1, av, dv);
#pragma omp parallel for schedule(static)
      for (size_t i = 0; i < N; i++) vs[i] = dv[i] + v2[i] / 6.0;
      memcpy(dv, v2, sizeof(double) * N);
    } else {
      memcpy(vs, dv, sizeof(double) * N);
    }
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < N; i++) v1[i] = vars0[i] + dtcur * dv[i];
    bound(c, v1);
    /* k2 */
    dtcur = dt / 2.0;
    orc_rhs(c, v1, dv, 2);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < N; i++) { vs[i] = vs[i] + dv[i] / 3.0; v1[i] = vars0[i] + dtcur * dv[i]; }
    bound(c, v1);
    /* k3 */
    dtcur = dt;
    orc_rhs(c, v1, dv, 3);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < N; i++) { vs[i] = vs[i] + dv[i] / 3.0; v1[i] = vars0[i] + dtcur * dv[i]; }
    bound(c, v1);
    /* k4 */
    dtcur = dt;
    orc_rhs(c, v1, dv, 4);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < N; i++) { vs[i] = vs[i] + dv[i] / 6.0; v1[i] = vars0[i] + dtcur * vs[i]; }
    bound(c, v1);
    memcpy(vars0, v1, sizeof(double) * N);
    step_end(c, vars0, dt);
  }
  free(av);
  return CSS_OK;
}

/* ------------------------------------------------------------------------ */
/* Diagnostics of vars0: Scalar_Output (report_mpi.f90:173-262),            */
/* Compute_Step_Size (rhs_mpi.f90:92-275), Shell_Average_Output             */
/* (report_mpi.f90:783-1094, with Compute_Derivatives :264-439 for ds/dr)   */
/* and the spectrum of CSS-IDL/spectral_analysis_new.pro:16-25.  Sums run   */
/* in the Fortran array order of one plane (theta fastest).                 */
/* ------------------------------------------------------------------------ */
/* B = curl A of vars0 (Compute_B(0)), or NULL for hydro; caller frees */
static double *diag_b(orc_ctx *c, const double *vars0) {
  if (!c->p.magnetic) return NULL;
  double *b = dalloc(3 * (size_t)c->ncell);
  vector_curl_a(c, vars0 + 5 * (size_t)c->ncell, b);
  compute_b_bc(c, b);
  return b;
}

int orc_scalars(orc_ctx *c, const double *vars0, double *out) {
  size_t n = c->ncell;
  const double *prho = vars0, *pw = vars0 + n, *pv = vars0 + 2 * n, *pu = vars0 + 3 * n, *ps = vars0 + 4 * n;
  double *b = diag_b(c, vars0);
  double nsize = (double)n;
  double magener = 0.0, bmax = 0.0, cke = 0.0, mcke = 0.0, drke = 0.0, kinener = 0.0, umach = -1.0;
  double sumb = 0.0, maxb = 0.0, s;
  if (b) {
    for (size_t i = 0; i < n; i++) {
      double bsq = b[2 * n + i] * b[2 * n + i] + b[i] * b[i] + b[n + i] * b[n + i];
      sumb += bsq;
      if (i == 0 || sqrt(bsq) > maxb) maxb = sqrt(bsq);
    }
    magener = sumb / (8 * PI * nsize);
  }
  s = 0.0;
  for (size_t i = 0; i < n; i++) s += prho[i] * (pu[i] * pu[i]);
  cke = s / (double)(2 * n);
  s = 0.0;
  for (size_t i = 0; i < n; i++) s += prho[i] * (pw[i] * pw[i]);
  mcke = cke + s / (double)(2 * n);
  s = 0.0;
  for (size_t i = 0; i < n; i++) s += prho[i] * (pv[i] * pv[i]);
  drke = s / (double)(2 * n);
  s = 0.0;
  for (size_t i = 0; i < n; i++) {
    double t = pow(prho[i], c->gamm1) * exp(ps[i] * c->invcv) * c->invtconst * c->gamm1 * c->p.cp;
    double usqr = pw[i] * pw[i] + pv[i] * pv[i] + pu[i] * pu[i];
    double q;
    if (b) {
      double bsq = b[2 * n + i] * b[2 * n + i] + b[i] * b[i] + b[n + i] * b[n + i];
      q = usqr / (2.0 * bsq / prho[i] + usqr + t);
    } else {
      q = usqr / (usqr + t);
    }
    if (q > umach) umach = q;
    s += prho[i] * usqr;
  }
  kinener = s / (double)(2 * n);
  umach = sqrt(umach);
  if (b) bmax = maxb * 2.0 * sqrt(2.0 * PI);
  out[0] = kinener; out[1] = cke; out[2] = mcke; out[3] = drke; out[4] = umach; out[5] = magener; out[6] = bmax;
  free(b);
  return CSS_OK;
}

int orc_step_size(orc_ctx *c, const double *vars0, double cfl_safety, double *out) {
  size_t n = c->ncell;
  int nth = c->nth, nphi = c->nphi, nr = c->nr;
  double *b = diag_b(c, vars0);
  double dtmaxb = 1e4, dtmaxc = 1e4, etot = 0.0, ltot = 0.0, mtot = 0.0, mrsint = 0.0;
  const double dth = c->dth, dphi = c->dphi, om = c->p.omega_0;
  for (int ir = 0; ir < nr; ir++) {
    double radius = c->r_ind[ir], drad = c->dr_ind[ir];
    for (int it = 0; it < nth; it++) {
      double sinth = c->sines[it];
      double dxmin = fmin(drad, radius * fmin(dth, sinth * dphi));
      double srho = 0.0, sl = 0.0, se = 0.0, vmax = INFINITY, sb = 0.0, vamax = INFINITY;
      for (int ip = 0; ip < nphi; ip++) {
        size_t i = IDX(c, it, ip, ir);
        double rho = vars0[i], wt = vars0[n + i] * vars0[n + i], vt = vars0[2 * n + i], ut = vars0[3 * n + i] * vars0[3 * n + i];
        double tt = c->invtconst * pow(rho, c->gamm1) * exp(vars0[4 * n + i] * c->invcv);
        double q = vt + radius * sinth * om;
        srho += rho;
        sl += rho * sqrt(wt + sinth * sinth * (q * q));
        vt = vt * vt;
        se += rho * (c->cv * tt + 0.5 * (ut + wt + vt));
        tt = c->gamm1 * c->p.cp * c->p.xi_cs * c->p.xi_cs * tt;
        ut = ut + vt + wt + tt;
        vmax = fmin(vmax, dxmin / sqrt(ut));
        if (b) {
          double btt = b[i] * b[i], bpt = b[n + i] * b[n + i], brt = b[2 * n + i] * b[2 * n + i];
          sb += brt + btt + bpt;
          vamax = fmin(vamax, dxmin / sqrt(ut + (brt + btt + bpt) * ONE_OVER_4PI / rho));
        }
      }
      mtot += radius * radius * sinth * srho * drad * dth * dphi;
      mrsint += radius * radius * radius * sinth * sinth * sinth * srho * drad * dth * dphi;
      ltot += radius * radius * radius * sinth * sl * drad * dth * dphi;
      etot += radius * radius * sinth * se * drad * dth * dphi;
      dtmaxc = fmin(dtmaxc, vmax);
      if (b) {
        etot += 0.5 * radius * radius * sinth * sb * drad * dth * dphi * ONE_OVER_4PI;
        dtmaxb = fmin(dtmaxb, vamax);
      }
    }
  }
  double dtmaxd = 1e10;
  if (c->p.laplacian) { /* rhs_mpi.f90:194-198 (etar = ks, mhdsph_mpi.f90:349) */
    double drmin = c->dr_ind[0], ksmax = c->ks[0], mumax = c->mur[0] / c->rhor[0];
    for (int ir = 1; ir < c->nr; ir++) {
      drmin = fmin(drmin, c->dr_ind[ir]);
      ksmax = fmax(ksmax, c->ks[ir]);
      mumax = fmax(mumax, c->mur[ir] / c->rhor[ir]);
    }
    double h = fmin(drmin, c->p.r1 * fmin(fmin(c->sines[0], c->sines[c->nth - 1]) * c->dphi, c->dth));
    dtmaxd = h * h / fmax(fmax(ksmax, mumax), ksmax);
  }
  out[0] = fmin(fmin(dtmaxb, dtmaxc), dtmaxd) * cfl_safety;
  out[1] = etot; out[2] = ltot; out[3] = mtot; out[4] = mrsint;
  free(b);
  return CSS_OK;
}

int orc_shell_averages(orc_ctx *c, const double *vars0, const int *q, int nq, const double *k0, double *out) {
  size_t n = c->ncell;
  int nth = c->nth, nphi = c->nphi, nr = c->nr;
  size_t np = (size_t)nth * nphi;
  const css_params *p = &c->p;
  for (int iq = 0; iq < nq; iq++)
    if (q[iq] < 1 || q[iq] > 18 || (q[iq] >= 10 && q[iq] <= 14 && !p->magnetic) || (q[iq] == 15 && p->do_radheat)) {
      set_err("orc_shell_averages: quantity %d not available", q[iq]);
      return CSS_ERR_ARG;
    }
  const double *prho = vars0, *pw = vars0 + n, *pv = vars0 + 2 * n, *pu = vars0 + 3 * n, *ps = vars0 + 4 * n;
  double *b = diag_b(c, vars0);
  double *temp = dalloc(n), *dsdr = dalloc(n), *flo = dalloc(np), *fhi = dalloc(np);
  /* Compute_Derivatives: ds/dr with dsdr1/dxdr(1), dsdr2/dxdr(nr) (or the face value) at the faces */
  double dsdr1 = 0.0, dsdr2 = 0.0; /* dsdrm of the isentropic background */
  if (p->slaplacian) {
    if (!p->bottom_constant_temp) dsdr1 = -p->lumr1 * ONE_OVER_4PI / (c->ks[0] * p->r1 * p->r1);
    if (!p->top_constant_temp) dsdr2 = -p->lumr2 * ONE_OVER_4PI / (c->ks[nr - 1] * p->r2 * p->r2);
  }
  int lbs = c->ibcr[5];
  for (size_t k = 0; k < np; k++) {
    flo[k] = (lbs == 2 || lbs == 4) ? dsdr1 / c->dxdr[0] : ps[k];
    fhi[k] = (lbs == 3 || lbs == 4) ? dsdr2 / c->dxdr[nr - 1] : ps[(size_t)(nr - 1) * np + k];
  }
  orc_deriv(c, 0, 1, ps, dsdr, flo, fhi, lbs);
  if (p->non_uniform)
    for (size_t i = 0; i < n; i++) dsdr[i] = dsdr[i] * c->dxdr[i / np];
  for (size_t i = 0; i < n; i++) temp[i] = pow(prho[i], c->gamm1) * exp(ps[i] * c->invcv) * c->invtconst;
  double nsize = (double)np;
  for (int ir = 0; ir < nr; ir++) {
    size_t o = (size_t)ir * np;
    double avgT = 0, avgrho = 0, avgP = 0, avgvr = 0, sumrt = 0;
    for (size_t k = 0; k < np; k++) { avgT += temp[o + k]; avgrho += prho[o + k]; sumrt += prho[o + k] * temp[o + k]; avgvr += pu[o + k]; }
    avgP = c->gamm1 * c->cv * sumrt;
    avgT /= nsize; avgrho /= nsize; avgP /= nsize; avgvr /= nsize;
    for (int iq = 0; iq < nq; iq++) {
      double s = 0.0, v;
      for (size_t k = 0; k < np; k++) {
        size_t i = o + k;
        double usqr = 0.5 * prho[i] * (pu[i] * pu[i] + pv[i] * pv[i] + pw[i] * pw[i]);
        double bt = b ? b[i] : 0, bp = b ? b[n + i] : 0, br = b ? b[2 * n + i] : 0;
        switch (q[iq]) {
          case 1: s += prho[i]; break;
          case 2: s += temp[i]; break;
          case 3: s += ps[i]; break;
          case 4: s += prho[i] * temp[i]; break;
          case 5: s += pu[i]; break;
          case 6: s += pw[i]; break;
          case 7: s += pv[i]; break;
          case 8: s += usqr; break;
          case 9: case 15: s += dsdr[i]; break;
          case 10: s += br; break;
          case 11: s += bt; break;
          case 12: s += bp; break;
          case 13: s += 0.125 * (br * br + bt * bt + bp * bp) / PI; break;
          case 14: s += sqrt(br * br + bt * bt); break;
          case 16: s += (pu[i] - avgvr) * prho[i] * (temp[i] - avgT); break;
          case 17: s += usqr * (pu[i] - avgvr); break;
          case 18: s += (c->gamm1 * c->cv * prho[i] * temp[i] - avgP) * (pu[i] - avgvr); break;
        }
      }
      switch (q[iq]) {
        case 4: v = c->gamm1 * c->cv * s / nsize; break;
        case 5: v = avgvr; break;
        case 15: v = (c->cond ? -c->ks[ir] * s / nsize : 0.0) + (k0 ? k0[ir] : 0.0); break;
        case 16: v = p->cp * s / nsize; break;
        default: v = s / nsize;
      }
      out[(size_t)iq * nr + ir] = v;
    }
  }
  free(b); free(temp); free(dsdr); free(flo); free(fhi);
  return CSS_OK;
}

int orc_spectrum(orc_ctx *c, const double *vars0, int kind, double *out) {
  size_t n = c->ncell;
  int nth = c->nth, nphi = c->nphi, nr = c->nr;
  if (nth % 2 || nphi % 2 || kind < 0 || kind > 1 + c->nv || (kind == 1 && !c->p.magnetic)) {
    set_err("orc_spectrum: bad kind or odd grid");
    return CSS_ERR_ARG;
  }
  double *b = kind == 1 ? diag_b(c, vars0) : NULL;
  double *apod = dalloc(nth), *a = dalloc((size_t)nth * nphi);
  double *xr = dalloc((size_t)nth * nphi), *xi = dalloc((size_t)nth * nphi);
  double *tr = dalloc((size_t)nth * nphi), *ti = dalloc((size_t)nth * nphi);
  double th0 = c->theta[0], thn = c->theta[nth - 1];
  for (int t = 0; t < nth; t++) apod[t] = 1.0 - pow(cos(PI * (c->theta[t] - th0) / (thn - th0)), 64);
  double nn = (double)nth * (double)nphi;
  double *cp_ = dalloc(nphi), *sp_ = dalloc(nphi), *ct_ = dalloc(nth), *st_ = dalloc(nth);
  for (int j = 0; j < nphi; j++) { cp_[j] = cos(2.0 * PI * (double)j / (double)nphi); sp_[j] = sin(2.0 * PI * (double)j / (double)nphi); }
  for (int j = 0; j < nth; j++) { ct_[j] = cos(2.0 * PI * (double)j / (double)nth); st_[j] = sin(2.0 * PI * (double)j / (double)nth); }
  for (int ir = 0; ir < nr; ir++) {
    for (int ip = 0; ip < nphi; ip++)
      for (int t = 0; t < nth; t++) {
        size_t i = IDX(c, t, ip, ir);
        double f;
        if (kind == 0) f = 0.5 * vars0[i] * (vars0[3 * n + i] * vars0[3 * n + i] + vars0[2 * n + i] * vars0[2 * n + i] + vars0[n + i] * vars0[n + i]);
        else if (kind == 1) f = 0.125 * (b[2 * n + i] * b[2 * n + i] + b[i] * b[i] + b[n + i] * b[n + i]) / PI;
        else f = vars0[(size_t)(kind - 2) * n + i];
        a[t + (size_t)nth * ip] = f * apod[t];
      }
    /* forward 2D DFT (IDL fft(.,-1) divides by the number of points): phi then theta */
    for (int t = 0; t < nth; t++)
      for (int kp = 0; kp < nphi; kp++) {
        double sr = 0, si = 0;
        for (int ip = 0; ip < nphi; ip++) {
          int j = (int)(((long long)kp * ip) % nphi);
          sr += a[t + (size_t)nth * ip] * cp_[j];
          si -= a[t + (size_t)nth * ip] * sp_[j];
        }
        xr[t + (size_t)nth * kp] = sr; xi[t + (size_t)nth * kp] = si;
      }
    for (int kp = 0; kp < nphi; kp++)
      for (int kt = 0; kt < nth; kt++) {
        double sr = 0, si = 0;
        for (int t = 0; t < nth; t++) {
          int j = (int)(((long long)kt * t) % nth);
          double cr = ct_[j], ci = -st_[j];
          double yr = xr[t + (size_t)nth * kp], yi = xi[t + (size_t)nth * kp];
          sr += yr * cr - yi * ci;
          si += yr * ci + yi * cr;
        }
        tr[kt + (size_t)nth * kp] = sr / nn; ti[kt + (size_t)nth * kp] = si / nn;
      }
    /* fold: cube[0,0] = F[0,0]; cube[kt,kp] = F[kt,kp] + F[nth-kt,nphi-kp] for 1 <= kt < nth/2,
       1 <= kp < nphi/2, stored into a real array (real part); total over kt / (nth/2) */
    for (int kp = 0; kp < nphi / 2; kp++) {
      double s = 0.0;
      if (kp == 0) s = tr[0];
      else
        for (int kt = 1; kt < nth / 2; kt++) s += tr[kt + (size_t)nth * kp] + tr[(nth - kt) + (size_t)nth * (nphi - kp)];
      out[(size_t)ir * (nphi / 2) + kp] = s / (nth / 2.0);
    }
  }
  free(b); free(apod); free(a); free(xr); free(xi); free(tr); free(ti);
  free(cp_); free(sp_); free(ct_); free(st_);
  return CSS_OK;
}

/* ------------------------------------------------------------------------
 * Cyclic phi derivative (an extension with no counterpart in the
 * reference, whose Dbydp / D2bydp2, derivatives.f90:1480-1684, close every
 * block with halo rows).  The whole periodic line of n points takes the
 * interior rows of Dbydp / D2bydp2 at every point:
 *   alpha f'_{j-1} + f'_j + alpha f'_{j+1} = rhs_j (periodic indices),
 * alpha = 1/3, rhs = 7/9 (f_{j+1}-f_{j-1}) + 1/36 (f_{j+2}-f_{j-2}) for the
 * first derivative; alpha = 2/11, rhs = 12/11 (f_{j+1}-2f_j+f_{j-1}) + 3/44
 * (f_{j+2}-2f_j+f_{j-2}) for the second; times dnum (dnum^2).  The cyclic
 * tridiagonal system is split as A = B + u v^T (Sherman-Morrison, with
 * gamma = -1: B's first diagonal 1 - gamma, its last 1 - alpha^2/gamma,
 * u = (gamma, 0.., alpha), v = (1, 0.., alpha/gamma)) and solved as
 * x = y - (v.y)/(1 + v.z) z with B y = rhs, B z = u by Gaussian
 * elimination without pivoting (B is diagonally dominant).
 * ------------------------------------------------------------------------ */
static void orc_tridiag(int n, double alpha, double b0, double bn, const double *d, double *x, double *w) {
  /* solves B x = d, B = tridiag(alpha, b, alpha), b = 1 but b[0] = b0, b[n-1] = bn;
   * w is scratch of n */
  double piv = b0;
  x[0] = d[0] / piv;
  for (int j = 1; j < n; j++) {
    w[j] = alpha / piv;
    const double bj = (j == n - 1) ? bn : 1.0;
    piv = bj - alpha * w[j];
    x[j] = (d[j] - alpha * x[j - 1]) / piv;
  }
  for (int j = n - 2; j >= 0; j--) x[j] -= w[j + 1] * x[j + 1];
}

int orc_cyclic_lines(const double *x, double *dx, int n, int nlines, int order, double dnum) {
  if (!x || !dx || n < 5 || nlines < 0 || order < 1 || order > 2) {
    set_err("orc_cyclic_lines: bad argument");
    return CSS_ERR_ARG;
  }
  const double alpha = order == 1 ? 1.0 / 3.0 : 2.0 / 11.0, gamma = -1.0;
  const double b0 = 1.0 - gamma, bn = 1.0 - alpha * alpha / gamma;
  const double scale = order == 1 ? dnum : dnum * dnum;
  double *u = malloc(sizeof(double) * n), *z = malloc(sizeof(double) * n), *w = malloc(sizeof(double) * n);
  for (int j = 0; j < n; j++) u[j] = 0.0;
  u[0] = gamma;
  u[n - 1] = alpha;
  orc_tridiag(n, alpha, b0, bn, u, z, w);
  const double vz = z[0] + (alpha / gamma) * z[n - 1];
  free(u);
  free(w);
#pragma omp parallel for schedule(static)
  for (int l = 0; l < nlines; l++) {
    const double *f = x + (size_t)l * n;
    double *o = dx + (size_t)l * n;
    double *r = malloc(sizeof(double) * n), *y = malloc(sizeof(double) * n), *ws = malloc(sizeof(double) * n);
    for (int j = 0; j < n; j++) {
      const double fm2 = f[(j - 2 + n) % n], fm1 = f[(j - 1 + n) % n], f0 = f[j], fp1 = f[(j + 1) % n],
                   fp2 = f[(j + 2) % n];
      if (order == 1) r[j] = (7.0 / 9.0) * (fp1 - fm1) + (1.0 / 36.0) * (fp2 - fm2);
      else r[j] = (12.0 / 11.0) * (fp1 - 2.0 * f0 + fm1) + (3.0 / 44.0) * (fp2 - 2.0 * f0 + fm2);
    }
    orc_tridiag(n, alpha, b0, bn, r, y, ws);
    const double fact = (y[0] + (alpha / gamma) * y[n - 1]) / (1.0 + vz);
    for (int j = 0; j < n; j++) o[j] = scale * (y[j] - fact * z[j]);
    free(r);
    free(y);
    free(ws);
  }
  free(z);
  return CSS_OK;
}

/* ------------------------------------------------------------------------
 * Voronoi cells (Compute_Voronoi, voronoi.f90:30-280) and the downflow
 * lanes of entropy rain (Build_Downflow_Lanes, entropy_rain.f90:657-713).
 *
 * The Delaunay triangulation here is the definition itself, by brute
 * force: every triple of sites whose circumcircle holds no other site,
 * stored counterclockwise, in lexicographic order of the triple (the
 * reference builds it incrementally, dtris2 of voronoi.f90:376-681; for
 * sites in general position the triangles are the same, only their
 * numbering differs).  The walk around each site restates Compute_Voronoi's
 * loops (:129-276): from the first triangle holding the site, step to the
 * triangle across the edge to the next node until the start returns or
 * the hull is met; then walk again from there, recording the triangles.
 * ------------------------------------------------------------------------ */
static double orc_orient(double ax, double ay, double bx, double by, double cx, double cy) {
  return (bx - ax) * (cy - ay) - (by - ay) * (cx - ax);
}

int orc_voronoi(int n, const double *x, const double *y, int *degree, int *start, int *face, int *nvert,
                double *vxy) {
  if (n < 3) { set_err("orc_voronoi: fewer than 3 sites"); return CSS_ERR_ARG; }
  int cap = 2 * n + 8, nt = 0;
  int *tri = (int *)malloc(sizeof(int) * 3 * cap);
  for (int i = 0; i < n; i++)
    for (int j = i + 1; j < n; j++)
      for (int k = j + 1; k < n; k++) {
        double o = orc_orient(x[i], y[i], x[j], y[j], x[k], y[k]);
        if (o == 0.0) continue;
        /* circumcircle of (i, j, k), relative to site i */
        double bx = x[j] - x[i], by = y[j] - y[i], cx = x[k] - x[i], cy = y[k] - y[i];
        double d = 2.0 * (bx * cy - by * cx), b2 = bx * bx + by * by, c2 = cx * cx + cy * cy;
        double ux = x[i] + (cy * b2 - by * c2) / d, uy = y[i] + (bx * c2 - cx * b2) / d;
        double rr = (x[i] - ux) * (x[i] - ux) + (y[i] - uy) * (y[i] - uy);
        int empty = 1;
        for (int m = 0; m < n && empty; m++) {
          if (m == i || m == j || m == k) continue;
          double dx = x[m] - ux, dy = y[m] - uy;
          if (dx * dx + dy * dy < rr) empty = 0;
        }
        if (!empty) continue;
        if (nt == cap) { free(tri); set_err("orc_voronoi: degenerate sites"); return CSS_ERR_ARG; }
        tri[3 * nt] = i;
        tri[3 * nt + 1] = o > 0.0 ? j : k;
        tri[3 * nt + 2] = o > 0.0 ? k : j;
        vxy[2 * nt] = ux;
        vxy[2 * nt + 1] = uy;
        nt++;
      }
  *nvert = nt;
  for (int g = 0; g < n; g++) degree[g] = 0;
  for (int v = 0; v < nt; v++)
    for (int s = 0; s < 3; s++) degree[tri[3 * v + s]]++;
  int count = 0;
  for (int g = 0; g < n; g++) {
    int vn = -1, sn = -1;
    for (int v = 0; v < nt && vn < 0; v++)
      for (int s = 0; s < 3; s++)
        if (tri[3 * v + s] == g) { vn = v; sn = s; break; }
    start[g] = count;
    if (vn < 0) continue;
    /* one step: across the edge from g to the node after the current one */
#define ORC_VOR_STEP()                                                      \
  do {                                                                      \
    sn = (sn + 1) % 3;                                                      \
    gn = tri[3 * vn + sn];                                                  \
    if (gn == g) { sn = (sn + 1) % 3; gn = tri[3 * vn + sn]; }              \
    vold = vn;                                                              \
    vn = -1;                                                                \
    for (int v = 0; v < nt && vn < 0; v++) {                                \
      if (v == vold) continue;                                              \
      for (int s = 0; s < 3; s++)                                           \
        if (tri[3 * v + s] == g) {                                          \
          int s1 = (s + 1) % 3;                                             \
          if (tri[3 * v + s1] == gn) { vn = v; sn = s1; break; }            \
          s1 = (s + 2) % 3;                                                 \
          if (tri[3 * v + s1] == gn) { vn = v; sn = s1; break; }            \
        }                                                                   \
    }                                                                       \
  } while (0)
    int gn, vold, vsave = vn;
    for (;;) {
      ORC_VOR_STEP();
      if (vn == vsave) break;
      if (vn < 0) { vn = vold; break; }
    }
    vsave = vn;
    face[count++] = vn;
    for (;;) {
      ORC_VOR_STEP();
      if (vn == vsave || vn < 0) break;
      face[count++] = vn;
    }
#undef ORC_VOR_STEP
  }
  free(tri);
  return CSS_OK;
}

/* Build_Downflow_Lanes (entropy_rain.f90:657-713) with the periodic copies
   of the sites (:80-89); cells[3k..] = phi_loc, theta_loc, scaling.  Each
   top block (rank) walks every cell edge and adds the Gaussian of every
   edge point inside its window to all of its cells. */
int orc_build_lanes(orc_ctx *c, int ncells, const double *cells, double meansize, double meanvel, double meands) {
  const css_params *p = &c->p;
  if (!c->dvel_rain) { set_err("orc_build_lanes: the run has no open boundary"); return CSS_ERR_ARG; }
  int nth = c->nth, nphi = c->nphi, n3 = 3 * ncells;
  size_t np = (size_t)nth * nphi;
  double *x = dalloc(n3), *y = dalloc(n3), *sc = dalloc(n3), *vxy = dalloc(4 * (size_t)n3 + 16);
  int *deg = (int *)calloc(n3, sizeof(int)), *st = (int *)calloc(n3, sizeof(int));
  int *fc = (int *)calloc(6 * (size_t)n3 + 32, sizeof(int)), nv = 0;
  for (int k = 0; k < ncells; k++) {
    x[k] = cells[3 * k];
    x[k + ncells] = cells[3 * k] - (p->phi2 - p->phi1);
    x[k + 2 * ncells] = (p->phi2 - p->phi1) + cells[3 * k];
    y[k] = y[k + ncells] = y[k + 2 * ncells] = cells[3 * k + 1];
    sc[k] = sc[k + ncells] = sc[k + 2 * ncells] = cells[3 * k + 2];
  }
  int rc = orc_voronoi(n3, x, y, deg, st, fc, &nv, vxy);
  if (rc == CSS_OK) {
    double smin = 1.0;
    for (int it = 0; it < nth; it++) smin = fmin(smin, sin(c->theta[it]));
    int isz = (int)ceil(meansize * sqrt(-log(1e-5)) / (p->r2 * fmin(c->dth, c->dphi * smin)));
    int nmax = (int)sqrt((double)nth * nth + (double)nphi * nphi);
    double xsz = isz * c->dphi, ysz = isz * c->dth, rtmp = (p->r2 / meansize) * (p->r2 / meansize);
    memset(c->dvel_rain, 0, sizeof(double) * np);
    for (int b = 0; b < c->nblk; b++) {
      const blk_t *B = &c->blk[b];
      if (!B->rhi) continue;
      double xlo = c->phi[B->p0] - xsz, xhi = c->phi[B->p0 + B->np - 1] + xsz;
      double ylo = c->theta[B->t0] - ysz, yhi = c->theta[B->t0 + B->nt - 1] + ysz;
      for (int ic = 0; ic < n3; ic++)
        for (int ie = 0; ie < deg[ic]; ie++) {
          int va = fc[st[ic] + ie], vb = fc[st[ic] + (ie + 1 < deg[ic] ? ie + 1 : 0)];
          double x1 = vxy[2 * va], y1 = vxy[2 * va + 1];
          double dvx = vxy[2 * vb] - x1, dvy = vxy[2 * vb + 1] - y1;
          double gx = dvx / c->dphi, gy = dvy / c->dth, len = sqrt(gx * gx + gy * gy);
          int my = len >= (double)nmax ? nmax : (int)len;
          for (int k = 0; k < my; k++) {
            double t = (double)k / (double)my, xv = x1 + dvx * t, yv = y1 + dvy * t;
            if (!(xv >= xlo && xv <= xhi && yv >= ylo && yv <= yhi)) continue;
            for (int ip = B->p0; ip < B->p0 + B->np; ip++)
              for (int it = B->t0; it < B->t0 + B->nt; it++) {
                double a = c->theta[it] - yv, bb = c->phi[ip] - xv;
                size_t id = it + (size_t)nth * ip;
                c->dvel_rain[id] = c->dvel_rain[id] + sc[ic] * exp(-rtmp * (a * a + bb * bb));
              }
          }
        }
    }
    double m = 0.0;
    for (size_t i = 0; i < np; i++) m = fmax(m, c->dvel_rain[i]);
    m = fmax(m, 1.0);
    for (size_t i = 0; i < np; i++) {
      double d = c->dvel_rain[i] / m;
      c->dent_rain[i] = meands * d;
      c->dvel_rain[i] = meanvel * d;
    }
  }
  free(x); free(y); free(sc); free(vxy); free(deg); free(st); free(fc);
  return rc;
}
