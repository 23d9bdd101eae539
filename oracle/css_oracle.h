/*
 * css_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of the CSS reference hot path (orvedahl/CSS-Code,
 * Fortran 90 + MPI) used as the parity oracle for the B200 library.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
 * arm may load it.  It is never linked into the product library.
 *
 * The Fortran cannot be compiled in this environment (no Fortran compiler,
 * no MPI, no LAPACK, Intel-only IFPORT in checkpoint.f90:3), so this file
 * restates, routine by routine, the algorithm of
 *   derivatives.f90 (Initialize_Derivatives, Dbydr..D2bydp2, VectorCurlA,
 *                    Compute_B, Dbyd1_dt0),
 *   parallel_mpi.f90 (Partition, the halo semantics of the exchanges),
 *   rhs_mpi.f90     (RHS, Source_Theta_Terms, Phi_Terms, Radial_Terms,
 *                    Density_Terms_Theta/_Radial, Induction_Terms, Bound),
 *   diffusion.f90   (Initialize_Diffusion, Compute_Diffusion, Diffusion_R,
 *                    Diffusion_Th, Diffusion_Phi),
 *   step_rk4.f90    (Step_RK4, Step_RK2_TVD, Step_RK3_TVD),
 *   report_mpi.f90  (Scalar_Output, Shell_Average_Output and the ds/dr of
 *                    Compute_Derivatives), rhs_mpi.f90 Compute_Step_Size,
 *   CSS-IDL/spectral_analysis_new.pro (the folded FFT spectrum),
 * emulating the MPI ranks serially (one virtual rank per block).
 *
 * Pinning: Dbyd1_dt0 / the whole-line closures are checked against golden
 * vectors produced by the reference's own CSS-Python derivatives.py
 * compact_fd6 (tests/golden/); block operators against the analytic
 * known-answer fields of validation.f90:17-28 and 6th-order convergence.
 */
#ifndef CSS_ORACLE_H
#define CSS_ORACLE_H
#include "../include/css_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

int orc_create(const css_params *p, const double *profiles, orc_ctx **out);
void orc_destroy(orc_ctx *c);
const char *orc_last_error(void);
void orc_set_threads(int n);

/* same semantics as the css_* entry points of include/css_b200.h */
int orc_deriv(orc_ctx *c, int dir, int order, const double *x, double *dx,
              const double *bc_lo, const double *bc_hi, int bdry);
int orc_rhs(orc_ctx *c, double *vars1, double *dvars1, int call_num);
int orc_diffusion(orc_ctx *c, double *vars1, const double *avec, double *dvars1);
int orc_step_rk4(orc_ctx *c, double *vars0, double dt, int nsteps);
int orc_bound(orc_ctx *c, double *vars1);
int orc_dbyd1_dt0(const double *x, double *dxdy, const double *bdat1,
                  const double *bdat2, int n1, int ibc, int nlines);
int orc_compact_lines(const double *x, double *dx, int n, int nlines, int order, int lphys, int rphys,
                      int bdry, const double *bc_lo, const double *bc_hi, const double *halo_lo,
                      const double *halo_hi, double dnum, double scale);
/* cyclic (Sherman-Morrison) compact derivative of whole periodic lines: the
 * phi extension css_dbydp_cyclic; x, dx: nlines x n, line-contiguous */
int orc_cyclic_lines(const double *x, double *dx, int n, int nlines, int order, double dnum);
/* curl of A (VectorCurlA + Compute_B boundary zeroing): b = curl(a), 3 fields */
int orc_curl_b(orc_ctx *c, const double *a, double *b);
/* diagnostics of vars0, same outputs as css_scalars / css_step_size /
 * css_shell_averages / css_spectrum */
int orc_scalars(orc_ctx *c, const double *vars0, double *out);
int orc_step_size(orc_ctx *c, const double *vars0, double cfl_safety, double *out);
int orc_shell_averages(orc_ctx *c, const double *vars0, const int *q, int nq, const double *k0, double *out);
int orc_spectrum(orc_ctx *c, const double *vars0, int kind, double *out);
/* open radial boundaries: clock, mass bookkeeping, rain and ASH inputs */
int orc_set_clock(orc_ctx *c, long long istep, double sim_time, double deltat);
int orc_get_clock(orc_ctx *c, long long *istep, double *sim_time);
int orc_inout_init(orc_ctx *c, const double *vars0);
int orc_inout_state(orc_ctx *c, double *out);
int orc_set_rain_fields(orc_ctx *c, const double *dvel, const double *dent);
int orc_rain_fields(orc_ctx *c, double *dvel, double *dent);
int orc_set_ash_slices(orc_ctx *c, const double *slices, const double *times, double ash_fen_mod);
int orc_build_squalls(orc_ctx *c, int sstruct, int nsq, const double *sq);
int orc_add_squalls(orc_ctx *c, int sstruct, int nsq, const double *sq);
/* Voronoi cells (Compute_Voronoi, voronoi.f90:30-280; brute-force
 * Delaunay) and the downflow lanes (Build_Downflow_Lanes,
 * entropy_rain.f90:657-713), outputs as css_voronoi / css_build_lanes */
int orc_voronoi(int n, const double *x, const double *y, int *degree, int *start, int *face, int *nvert,
                double *vxy);
int orc_build_lanes(orc_ctx *c, int ncells, const double *cells, double meansize, double meanvel, double meands);

#ifdef __cplusplus
}
#endif
#endif
