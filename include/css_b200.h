/*
 * css_b200.h -- C ABI of the B200 (sm_100a) implementation of the CSS
 * (Compressible Spherical Segment) time-step hot path: compact 6th-order
 * derivatives, hydro/MHD right-hand side, slope-limited diffusion (SLD) and
 * the RK4 update.
 *
 * Every entry point takes plain pointers and sizes and returns an int status
 * (CSS_OK == 0).  The reference has no return codes (errors print and call
 * Graceful_Exit, parallel_mpi.f90:886-889); here the caller decides.
 *
 * Array layout (host and device): the reference's Fortran order
 *   vars(it, ip, ir, iv)  ->  vars[it + nth*(ip + nphi*(ir + nr*iv))]
 * (theta fastest, then phi, then r, then the field index), as allocated in
 * Initialize_Physics (rhs_mpi.f90:24).  Field order: 0 rho, 1 w (u_theta),
 * 2 v (u_phi), 3 u (u_r), 4 s, and for MHD 5..7 = the vector potential
 * A_theta, A_phi, A_r in the state (B_theta, B_phi, B_r while an RHS runs),
 * as rhs_mpi.f90:819-1027 and checkpoint.f90:289-296 name them.
 *
 * The reference runs one MPI rank per block of an (nnr, nnt, nnp) Cartesian
 * decomposition and its derivative closures depend on the block faces
 * (derivatives.f90:564-721).  Here the whole domain lives on one GPU and the
 * decomposition is virtual: every block of the line is solved independently
 * with the same halo-closed rows, so results equal the reference run on
 * nnr*nnt*nnp ranks.
 *
 * Threading: one host thread per context; every call is stream-ordered on
 * the context's own CUDA stream and synchronous unless documented otherwise.
 */
#ifndef CSS_B200_H
#define CSS_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define CSS_OK           0
#define CSS_ERR_ARG      1   /* bad argument / unsupported flag combination  */
#define CSS_ERR_DECOMP   2   /* decomposition the reference cannot run       */
#define CSS_ERR_CUDA     3   /* CUDA runtime error (message: css_last_error) */
#define CSS_ERR_NAN      4   /* non-finite value in the state after a step   */
#define CSS_ERR_NOMEM    5   /* device allocation failed                     */
#define CSS_ERR_NODEV    6   /* no CUDA device                               */

/* ---- radial profile slots: profiles[slot*nr + ir] ----------------------- */
/* The reference keeps these as module globals (constants.f90:19-25,
 * derivatives.f90:32); Read_Stellar_Model fills them (mhdsph_mpi.f90:317-397). */
enum {
  CSS_PROF_X = 0,     /* x_ind: uniform computational coordinate            */
  CSS_PROF_R,         /* r_ind: radius at each grid point                    */
  CSS_PROF_DR,        /* dr_ind: r(ir) - r(ir-1), dr_ind(1) extrapolated     */
  CSS_PROF_DXDR,      /* dx/dr                                               */
  CSS_PROF_D2XDR2,    /* d2x/dr2                                             */
  CSS_PROF_RHO,       /* background density rhor                             */
  CSS_PROF_S,         /* background entropy sr                               */
  CSS_PROF_G,         /* gravity                                             */
  CSS_PROF_KS,        /* entropy conductivity ks                             */
  CSS_PROF_DLNKS,     /* d ln ks / dr                                        */
  CSS_PROF_EPS,       /* internal heating eps                                */
  CSS_PROF_MUR,       /* dynamic viscosity mur (explicit-viscosity path)     */
  CSS_PROF_DLNMU,     /* d ln mur / dr                                       */
  CSS_PROF_KR,        /* inverse Rosseland opacity kr (radiative diffusion)  */
  CSS_PROF_DLNKR,     /* dlnkr as the reference keeps it: d ln(1/kr) / dr    */
  CSS_NPROF
};

/* ---- run parameters (mirror of the four reference namelists,
 *      mhdsph_mpi.f90:1142-1177; defaults constants.f90:31-82) ----------- */
typedef struct css_params {
  int nr, nth, nphi;          /* global grid                                   */
  int nnr, nnt, nnp;          /* virtual block decomposition (MPI dims)        */
  int magnetic;               /* 1: nv = 8 (MHD), 0: nv = 5                    */
  int non_uniform;            /* 1: r from r_ind/dxdr/d2xdr2 profiles          */
  double r1, r2;              /* radial extent                                 */
  double th1, th2;            /* colatitude extent, radians                    */
  double phi1, phi2;          /* azimuthal extent (periodic), radians          */
  double gamma, cp, omega_0;  /* ratio of heats, Cp, frame rotation rate      */
  double t0;                  /* top temperature (thermal damping target)      */
  double xi_cs;               /* sound-speed reduction factor (1 = none)       */
  double damping_time;        /* top thermal damping time                      */
  double lumr1, lumr2;        /* luminosity for constant-flux boundaries       */
  int slaplacian;             /* entropy diffusion ks*laplacian(s)             */
  int sldiffusion;            /* slope-limited diffusion once per step         */
  int top_stress_free, bottom_stress_free;       /* else no-slip               */
  int top_constant_temp, bottom_constant_temp;   /* else constant flux         */
  int theta_stress_free;
  int theta_normal_field, theta_perf_conductor;
  int top_radial_field, bottom_radial_field;
  int top_perfect_cond, bottom_perfect_cond;
  int set_stop;
  /* slope-limited diffusion (diffusion.f90:8-11) */
  double sld_coef, sld_speedh, sld_speedr, sld_exp, sld_pr, sld_prm;
  double sld_tanh_coef, flux_cutoff;
  int dstype;                 /* 1: add |u|^2 (+vA^2) to the diffusion speed^2 */
  int mass_diffusion, magnetic_diffusion;
  int do_viscous_heating, do_ohmic_heating;
  int flux_limiter, ent_flux_limiter, mag_flux_limiter;  /* <= 0: off         */
  int precision;              /* 0: FP64 (drop-in), 1: FP32 perturbation form  */
  int time_stepper;           /* 4: Step_RK4 (default), 2: Step_RK2_TVD, 3:
                                 Step_RK3_TVD (step_rk4.f90:31-335; the
                                 RK2TVD / RK3TVD namelist switches)         */
  int laplacian;              /* 1: explicit viscosity (the Laplacian switch,
                                 rhs_mpi.f90:844-927, :1123-1199, :1317-1435,
                                 :2070-2296); also turns the entropy
                                 conduction on, as SLaplacian does           */
  int do_radheat;             /* 1: radiative diffusion of heat (rhs_mpi.f90:
                                 388-393, :1092-1106, :1590-1602, :1820-1853);
                                 also turns the top thermal damping off      */
  /* open radial boundaries (constants.f90:55, :69-72; hydro FP64 only) */
  int top_inout;              /* 1: inflow/outflow top, Top_Inflow_Outflow
                                 (rhs_mpi.f90:1955-2067): u_r free at r2,
                                 top plane relaxed toward its neighbour     */
  int bot_inout;              /* 1: inflow/outflow bottom, Bottom_Inflow_
                                 Outflow (rhs_mpi.f90:1857-1953)             */
  int bottom_specified;       /* with bot_inout: bottom plane relaxed toward
                                 prescribed fields (the ASH inflow slices,
                                 css_set_ash_slices)                        */
  int do_entropy_rain;        /* with top_inout: top relaxation toward the
                                 rain-squall fields (css_set_rain_fields)   */
  int ufreq;                  /* step cadence of the mass-total refresh and
                                 the ASH enthalpy-flux factor (<= 0: never) */
  double delta_s;             /* entropy offset of the top relaxation       */
} css_params;

typedef struct css_ctx css_ctx;

/* Human-readable message for the last failing call on this thread. */
const char *css_last_error(void);

/* Builds a device-resident context: derivative LU tables for every virtual
 * block (Initialize_Derivatives, derivatives.f90:39-520), the SLD speed
 * profile (Initialize_Diffusion, diffusion.f90:19-63), the BC integers
 * (Read_Input, mhdsph_mpi.f90:1302-1462) and the state buffers.
 * Replaces Setup's Initialize_* chain (mhdsph_mpi.f90:92-123).            */
int css_create(const css_params *p, const double *profiles, css_ctx **out);
void css_destroy(css_ctx *ctx);

/* Host <-> device state copies; vars holds nth*nphi*nr*nv doubles in the
 * layout above (vars0 of parallel_mpi.f90:41).                            */
int css_upload_state(css_ctx *ctx, const double *vars);
int css_download_state(css_ctx *ctx, double *vars);

/* One plane of the resident state: field iv at radius ir, nth*nphi values
 * [it + nth*ip] into the host buffer `plane` (a face of vars0, as the rain
 * model reads the surface velocities, entropy_rain.f90:338-343).           */
int css_download_plane(css_ctx *ctx, int iv, int ir, double *plane);

/* nsteps RK4 steps of size dt on the device-resident state.  Replaces the
 * loop body of Program CSS2 (mhdsph_mpi.f90:28-48) calling Step_RK4
 * (step_rk4.f90:339-493).  Returns CSS_ERR_NAN if the state became
 * non-finite (the reference's Debug NaN abort, rhs_mpi.f90:288-322).      */
int css_step_rk4(css_ctx *ctx, double dt, int nsteps);

/* Host-buffer convenience: upload vars0, nsteps steps, download into vars0. */
int css_step_rk4_host(css_ctx *ctx, double *vars0, double dt, int nsteps);

/* RHS(call_num) (rhs_mpi.f90:279-783) on host buffers.  vars1 is in/out as
 * in the reference: for MHD, slots 5..7 come back holding B = curl A when
 * call_num == 1 and A otherwise (rhs_mpi.f90:325, :750-752).  A run with an
 * open radial boundary needs the clock's deltat set (css_set_clock) first. */
int css_rhs(css_ctx *ctx, double *vars1, double *dvars1, int call_num);

/* Bound() (rhs_mpi.f90:2395-2491) on a host state, in place: the wall and
 * face zeroing of velocities (and of the vector potential for MHD) that the
 * step entry points already apply after every stage, for a driver that
 * changes the state itself.                                               */
int css_bound(css_ctx *ctx, double *vars1);

/* Compute_Diffusion(1) (diffusion.f90:70-474) on host buffers: dvars1 gets
 * the SLD tendency.  As in the reference, vars1 comes back with the mean
 * state subtracted from rho and s (diffusion.f90:168-175).  For MHD, vars1
 * slots 5..7 must hold B and avec the vector potential A (the reference's
 * maga); avec may be NULL for hydro.                                      */
int css_diffusion(css_ctx *ctx, double *vars1, const double *avec, double *dvars1);

/* Whole-field compact derivative along one direction, every virtual block
 * solved with its own closures.  dir: 0 = r (Dbydr/D2bydr2,
 * derivatives.f90:547, :799), 1 = theta (Dbydt/D2bydt2, :1010, :1265),
 * 2 = phi (Dbydp/D2bydp2, :1480, :1594).  order 1 or 2.  bdry = the
 * reference's ibc 0..4 (its `var <= 0` form, derivatives.f90:558-562).
 * bc_lo / bc_hi: the 1-deep boundary datum at the physical low/high face
 * (r: nth*nphi values [it + nth*ip]; theta: nphi*nr values [ip + nphi*ir];
 * phi: unused, may be NULL).  Non-uniform r is returned in x-space, as the
 * reference returns it before the caller's dxdr multiply.
 * Host pointers.                                                          */
int css_deriv(css_ctx *ctx, int dir, int order, const double *x, double *dx,
              const double *bc_lo, const double *bc_hi, int bdry);

/* The six routines by the reference's names and with its `var` argument:
 * Dbydr, D2bydr2 (derivatives.f90:547, :799), Dbydt, D2bydt2 (:1010,
 * :1265), Dbydp, D2bydp2 (:1480, :1594).  var >= 1 takes the boundary
 * condition of field var (1-based, 1..12) from the run's ibcr / ibct
 * tables, var <= 0 means bdry = -var (derivatives.f90:558-562); the phi
 * routines have no boundary variants and ignore var.  Whole fields: the
 * reference's loop of per-pencil calls (one x(mynth, mynr) per phi for r)
 * becomes one call; b1 / b2 are the physical-face data as in css_deriv.
 * Host pointers.                                                          */
int css_dbydr(css_ctx *ctx, const double *x, double *dx, const double *b1, const double *b2, int var);
int css_d2bydr2(css_ctx *ctx, const double *x, double *dx, const double *b1, const double *b2, int var);
int css_dbydt(css_ctx *ctx, const double *x, double *dx, const double *b1, const double *b2, int var);
int css_d2bydt2(css_ctx *ctx, const double *x, double *dx, const double *b1, const double *b2, int var);
int css_dbydp(css_ctx *ctx, const double *x, double *dx, int var);
int css_d2bydp2(css_ctx *ctx, const double *x, double *dx, int var);

/* The reference's pencil calls, batched: npencils pencils in one call.
 * dir 0 (Dbydr / D2bydr2, derivatives.f90:547, :799): a pencil is the
 * (theta, r) plane of one phi, x(nth, nr) in Fortran order ([ir][it]);
 * bc_lo / bc_hi hold nth values per pencil (the r faces' datum).  dir 1
 * (Dbydt / D2bydt2, :1010, :1265) and dir 2 (Dbydp / D2bydp2, :1480,
 * :1594): a pencil is the (theta, phi) plane of one radius, x(nth, nphi)
 * ([ip][it]); for dir 1 bc_lo / bc_hi hold nphi values per pencil (the
 * theta faces' datum), dir 2 has none.  index[p] is pencil p's phi index
 * (dir 0) or radius (dir 1, 2): D2bydt2 divides its Neumann datum by the
 * radial block's dri (derivatives.f90:1322, :1338), so a theta pencil's
 * result depends on its radius; NULL means index p (mod nphi or nr).
 * var as in the named routines.  The pencils of a call are consecutive in
 * x and dx (pencil p at p * nth * nr, or p * nth * nphi); each comes back
 * as the same plane of the whole-field derivative.  Host pointers.  Like
 * css_deriv it works in the stage buffers, so it must not overlap a step
 * of the same context on another stream.                                  */
int css_deriv_pencils(css_ctx *ctx, int dir, int order, int npencils, const int *index,
                      const double *x, double *dx, const double *bc_lo, const double *bc_hi,
                      int var);

/* Same on device pointers, enqueued on `stream` (a cudaStream_t, NULL =
 * the context stream); returns after enqueueing.                           */
int css_deriv_dev(css_ctx *ctx, int dir, int order, const double *x, double *dx,
                  const double *bc_lo, const double *bc_hi, int bdry, void *stream);

/* Adjoint of css_deriv_dev with zero boundary data: gx = D^T g, where
 * dx = D x is the blocked compact derivative of direction dir, order and
 * bdry (the transpose of Dbydr ... D2bydp2, derivatives.f90:547-1684, as
 * one linear map of the field).  It has no counterpart in the reference;
 * it is the backward of torch.ops.css.deriv, so networks trained through
 * the derivatives (the closure) can differentiate them.  Device pointers
 * (g and gx must differ), enqueued on `stream`; the first call for a
 * (dir, order, bdry) builds that operator's dense per-block matrices.     */
int css_deriv_adjoint_dev(css_ctx *ctx, int dir, int order, const double *g, double *gx, int bdry,
                          void *stream);

/* Cyclic phi derivative (an extension, off the reference path: the
 * reference's Dbydp / D2bydp2, derivatives.f90:1480-1684, close every phi
 * block with halo rows, and css_dbydp / css_deriv reproduce that).  Here
 * every whole phi line is one periodic system: Dbydp's interior rows at
 * every point (alpha 1/3 or 2/11), the cyclic tridiagonal system solved by
 * Sherman-Morrison; order 1 or 2, times 1/dphi or 1/dphi^2.  It differs from
 * the reference's blocked operator at truncation level only.  x, dx: one
 * field (nth, nphi, nr) in Fortran order, host arrays; the _dev form takes
 * device pointers (not overlapping) and enqueues on `stream` (NULL = the
 * context stream).                                                         */
int css_dbydp_cyclic(css_ctx *ctx, const double *x, double *dx, int order);
int css_dbydp_cyclic_dev(css_ctx *ctx, const double *x, double *dx, int order, void *stream);

/* Batched 1D whole-line first derivative Dbyd1_dt0 (derivatives.f90:2296)
 * on nlines contiguous lines of n1 points, host pointers; bdat1/bdat2 per
 * line (may be NULL).  Returns d/dx in grid units, as the Fortran does.
 * Equals CSS-Python compact_fd6(dtype=0)/dri except for ibc = 2, where the
 * Fortran routine drops the last row's lower coefficient (its up2 is copied
 * from an already zeroed up1, derivatives.f90:2355-2386) and this entry
 * point reproduces that.                                                  */
int css_dbyd1_dt0(const double *x, double *dxdy, const double *bdat1,
                  const double *bdat2, int n1, int ibc, int nlines);

/* Independent compact-FD lines of n points (nlines, contiguous), order 1
 * or 2, with explicit closures: lphys/rphys = 1 closes that end with the
 * physical-boundary rows of bdry (datum bc_lo[l] / bc_hi[l]), 0 closes it
 * with halo rows fed by halo_lo[4l..4l+3] (the four points below, farthest
 * first) / halo_hi[4l..4l+3] (the four above, nearest first).  dx = scale *
 * solution; dnum divides the Neumann datum (dri in Dbydr).  With both ends
 * physical this is CSS-Python derivatives.py:32 compact_fd6(dtype=0).
 * Host pointers.                                                          */
int css_compact_lines(const double *x, double *dx, int n, int nlines, int order,
                      int lphys, int rphys, int bdry, const double *bc_lo,
                      const double *bc_hi, const double *halo_lo,
                      const double *halo_hi, double dnum, double scale);

/* Allocation-free variant of css_compact_lines, for callers that cannot
 * allocate device memory when they need a derivative: codes that gave all
 * device memory to their own pool or a framework's caching allocator at
 * start-up, and codes that must not stall on cudaMalloc/cudaFree, which
 * synchronize the whole device.  It has no counterpart in the reference.
 * x, dx, bc_lo, bc_hi, halo_lo, halo_hi are DEVICE pointers (same layout as
 * css_compact_lines; the boundary and halo arrays may be NULL as there);
 * work is enqueued on `stream` (NULL = the default stream) and the call
 * returns without waiting.  Scratch (the LU tables and halo-padded copies
 * of the lines) lives in one fixed 2 MiB device array per GPU, held from
 * the library's first use until the process exits: a call needs
 * 15*(n+2) + nlines*(n+8) doubles of it, at most 262144, and larger
 * requests fail with CSS_ERR_ARG.  Nothing in the array needs to start at
 * zero: each call writes every table entry and every padded line before
 * reading it.  The array is shared by every call on a device, so calls that
 * overlap on the GPU (other streams, other host threads) race: serialize
 * them on one stream.  The first call on each device (nlines may be 0:
 * such a call only does this set-up) looks up the array's device address;
 * under CUDA's lazy module loading that lookup is also when the library's
 * device code, and with it the array, is placed on that device.  So make
 * that first call at start-up, before handing device memory to a pool and
 * before any stream capture.  Later calls allocate nothing, on the device
 * or the host; concurrent first calls from several host threads are safe. */
int css_compact_lines_noalloc(const double *x, double *dx, int n, int nlines,
                              int order, int lphys, int rphys, int bdry,
                              const double *bc_lo, const double *bc_hi,
                              const double *halo_lo, const double *halo_hi,
                              double dnum, double scale, void *stream);

/* Checkpoints in the reference's layout (Checkpoint_Output / Checkpoint_Input,
 * checkpoint.f90:146-423): directory `dir` (created if missing) holds a
 * text `header` -- nr nth nphi nv istep as (5i9), then deltat sim_time r1
 * r2 th1 th2 phi1 phi2 as (8e14.7), so deltat is kept to 7 significant
 * digits as the reference keeps it -- and `checkpoint.rho`, `.w`, `.v`,
 * `.u`, `.s` (+ `.bt`, `.bp`, `.br`: the vector potential of an MHD run)
 * with the raw FP64 field in Fortran (nth, nphi, nr) order.  Reading needs
 * the same grid (the reference's horizontal interpolation is not
 * provided: CSS_ERR_ARG) and reads min(nv, nv of the file) fields, as the
 * reference does; the state of the context is replaced.                   */
int css_checkpoint_write(css_ctx *ctx, const char *dir, int istep,
                         double deltat, double sim_time);
int css_checkpoint_read(css_ctx *ctx, const char *dir, int *istep,
                        double *deltat, double *sim_time);

/* Block until all work on the context stream is done. */
int css_sync(css_ctx *ctx);

/* Device pointer of the current state (vars0) and its element count, for
 * zero-copy use from PyTorch or a CUDA-aware caller.                       */
int css_state_device_ptr(css_ctx *ctx, double **dptr, long long *nelem);

/* Number of kernels this library launched on ctx since creation. */
long long css_kernel_launches(css_ctx *ctx);

/* Run all further work of ctx on the caller's stream (a cudaStream_t; NULL
 * returns to the context's own stream).  Lets a CUDA-aware caller (PyTorch,
 * a Fortran driver with its own stream) order and time the library's
 * kernels on its stream.                                                   */
int css_set_stream(css_ctx *ctx, void *stream);

/* Per-kernel timing with CUDA events recorded around every launch on the
 * context stream (the reference's Do_Timings phase timers, rhs_mpi.f90:
 * 324-766).  css_profile(ctx, 1) clears and enables, 0 disables;
 * css_kernel_stats returns, for kernel kind 0..10 (theta_terms, phi_terms,
 * radial_terms, rhot_update, curl_theta, curl_phi, curl_r, sld_vcc, sld,
 * sld_ohmic, deriv), its name, summed milliseconds and launch count.      */
int css_profile(css_ctx *ctx, int enable);
int css_kernel_stats(css_ctx *ctx, int kind, const char **name, double *total_ms,
                     long long *launches);

/* ---- tile autotuning and batched ensembles ---------------------------------
 * css_autotune times, on the resident state and with reps RHS evaluations
 * per candidate, every tile height (lines per CTA) that each sweep
 * direction's kernels offer and keeps the fastest; chosen[3] (may be NULL)
 * receives the r, theta and phi choices.  The state is not modified and no
 * result changes: every line's arithmetic is the same for any tile height.
 * This has no counterpart in the reference (its per-rank loops have fixed
 * extents).                                                                */
int css_autotune(css_ctx *ctx, int reps, int *chosen);
/* The same choices made by hand: lines per CTA of the r, theta and phi
 * kernels (8 or 16 for 16/32-point blocks; 4, 8 or 16 otherwise) and 1 to
 * run Phi_Terms as a persistent kernel that streams the next tile into
 * shared memory while the current one is computed.                         */
int css_set_tiles(css_ctx *ctx, int tl_r, int tl_theta, int tl_phi, int phi_persistent);

/* The RK4 stage of Step_RK4 (step_rk4.f90:339-493) in two passes over the
 * device memory instead of four: one kernel per (theta block, phi block,
 * radius) plane for Source_Theta_Terms, Phi_Terms and Density_Terms_Theta
 * (rhs_mpi.f90:786-1261, :1522-1605), one per (r block, theta block, phi)
 * slab for Radial_Terms with Density_Terms_Radial (:1264-1519, :1710-1855),
 * the theta-wall part of Density_Terms_Theta, the stage combination and
 * Bound (:2395-2491).  css_create turns it on for runs that qualify: 32-point
 * virtual blocks in r, theta and phi, FP64 RK4, closed radial faces, no
 * explicit viscosity, radiative diffusion or prescribed bottom.
 * css_set_fused(ctx, 0) selects the four-kernel stage (same results to
 * rounding); css_set_fused(ctx, 1) on a run that does not qualify fails
 * with CSS_ERR_ARG.  css_get_fused returns the current choice.            */
int css_set_fused(css_ctx *ctx, int on);
int css_get_fused(css_ctx *ctx);
/* B = curl A (VectorCurlA, derivatives.f90:1769-1828) of magnetic runs,
 * its theta and phi parts: mode 2 (the default) from planes staged by TMA
 * in a persistent kernel, for the stage's own state buffers of runs that
 * take the two-pass stage; mode 1 in one pass over tiles (equal theta and
 * phi block sizes of 16 or 32); mode 0 a theta pass and a phi pass.  A mode
 * that does not apply falls back to the next lower one.  The results are
 * the same bit for bit. */
int css_set_curl_pass(css_ctx *ctx, int mode);

/* A batched ensemble of independent runs (many small shells, each with its
 * own grid, decomposition and parameters: hydro and MHD members may mix).
 * css_ensemble_step advances every member by nsteps RK4 steps of its own
 * dt[i]: one step of all members is captured once into a CUDA graph, each
 * member's kernels on a stream of its own so small members share the GPU,
 * and the graph is replayed per step (it is captured again when a dt
 * changes).  The first call, and every call with a new dt, must not be made
 * during another stream capture.  Member contexts stay owned by the caller
 * and must outlive the ensemble; a member must not be stepped through
 * css_step_rk4 while an ensemble step is running.  Returns CSS_ERR_NAN
 * (naming the member) when a member's state went non-finite.  The ensemble
 * has no counterpart in the reference, which runs one shell per job.       */
typedef struct css_ensemble css_ensemble;
int css_ensemble_create(int nmem, css_ctx *const *members, css_ensemble **out);
int css_ensemble_step(css_ensemble *ens, const double *dt, int nsteps);
/* kernels launched by all replays so far */
long long css_ensemble_launches(css_ensemble *ens);
/* device time (CUDA events on the ensemble stream) of the replays of the
 * last css_ensemble_step call, in milliseconds                             */
double css_ensemble_last_ms(css_ensemble *ens);
void css_ensemble_destroy(css_ensemble *ens);

/* ---- learned subgrid closure ------------------------------------------------
 * New: the reference prescribes the SLD speed profile (Initialize_Diffusion,
 * diffusion.f90:19-63); these entry points learn it per cell from a fine
 * run instead.  All array arguments are DEVICE pointers; the functions
 * without a context run on the default stream and return when done.
 *
 * css_set_sld_speed2: use speed2[ncell] (or NULL to return to the prescribed
 * profile) as the per-cell SLD speed^2 of ctx; a negative entry falls back
 * to the prescribed value of that radius.  The array must stay valid while
 * ctx steps.
 * css_box_filter: average the resident state over f x f x f cells (f
 * divides nr, nth, nphi) into fields[7*nc] (u_theta, u_phi, u_r, s - sr,
 * B_theta, B_phi, B_r; B = 0 for hydro) and targets[12*nc] (tau_tt tp tr pp
 * pr rr, q_t q_p q_r, emf_t emf_p emf_r: filtered products minus products
 * of filtered fields), coarse index it + nct*(ip + ncp*ir).
 * css_closure_scales: RMS of the five stencil quantities (u_theta, u_phi,
 * u_r, |B|, ds'/dr in coarse index units) and of the twelve targets
 * (targets may be NULL) -> scales[17] on the host.
 * css_closure_features: x[nc*144] BF16, the 3x3x3 neighbourhood (r, theta
 * clamped, phi periodic) of the five quantities divided by scale[5]: 135
 * features and 9 zeros per row.
 * css_closure_targets: tn[nc*16] FP32 = targets / tscale[12], zero padded.
 * css_closure_speed2: speed2[nc] = max(0, tau_tt + tau_pp + tau_rr) from
 * network outputs y[nc*16] times tscale, or -1 where not finite.          */
int css_set_sld_speed2(css_ctx *ctx, const double *speed2);
int css_box_filter(css_ctx *ctx, int f, double *fields, double *targets);
int css_closure_scales(int nct, int ncp, int ncr, const double *fields,
                       const double *targets, float *scales);
int css_closure_features(int nct, int ncp, int ncr, const double *fields,
                         const float *scale, void *x_bf16);
int css_closure_targets(long long nc, const double *targets,
                        const float *tscale, float *tn);
int css_closure_speed2(long long nc, const float *y, const float *tscale,
                       double *speed2);
/* css_closure_speed2_shaped: speed2[ncell of ctx] = the prescribed speed^2
 * of the cell's radius (diffusion_speed, Initialize_Diffusion,
 * diffusion.f90:19-63) times k / <k>_shell, k = max(0, tau_tt + tau_pp +
 * tau_rr) of the cell and <k>_shell its mean over the cell's radius: each
 * shell keeps the prescribed mean and the network places it; -1 where the
 * output is not finite or the shell mean is not positive.  y holds one row
 * per cell of ctx, in the state's cell order. */
int css_closure_speed2_shaped(css_ctx *ctx, const float *y, const float *tscale,
                              double *speed2);
/* Grids of one run at two resolutions (same device, same variables, fine =
 * f x coarse in r, theta and phi).  Bases are device arrays of the state's
 * layout on their grid (each grid's background state), NULL meaning zero.
 * css_restrict_state sets the coarse state to coarse_base + the f^3 box
 * average of (fine state - fine_base): a coarse run started from the
 * filtered fine perturbation, in its own grid's balance.  css_prolong_add
 * adds to the fine state the trilinear (index-space; theta and r clamped,
 * phi periodic) interpolation of (coarse state - coarse_base): a flow
 * developed on the coarse grid carried to the fine grid as a perturbation
 * of the fine grid's own state. */
int css_restrict_state(css_ctx *fine, const double *fine_base, int f,
                       css_ctx *coarse, const double *coarse_base);
int css_prolong_add(css_ctx *coarse, const double *coarse_base, int f, css_ctx *fine);

/* The closure network: n_in -> width -> width -> width -> n_out, GELU
 * (tanh form, hardware tanh) after the hidden layers, BF16 weights and activations, FP32
 * accumulation (the products are tensor-core GEMMs), FP32 master weights
 * and Adam moments.  Rows are padded to multiples of 16 (dims[5] returns
 * the padded widths: the input rows of css_mlp_forward /
 * css_mlp_train_step have dims[0] BF16 values, their outputs and targets
 * dims[4] FP32 values, row-major).  css_mlp_train_step does one Adam step
 * on the mean squared error over the n_out real outputs of n <= max_rows
 * rows and returns the loss before the step.  css_mlp_params gets (set=0)
 * or sets (set=1) layer l's FP32 weights (row-major dims[l] x dims[l+1])
 * and biases on the host; css_mlp_grads returns the last step's gradients. */
typedef struct css_mlp css_mlp;
int css_mlp_create(int n_in, int width, int n_out, int max_rows,
                   unsigned long long seed, css_mlp **out);
void css_mlp_destroy(css_mlp *mlp);
int css_mlp_dims(css_mlp *mlp, int *dims);
int css_mlp_forward(css_mlp *mlp, const void *x_bf16, long long n, float *y);
int css_mlp_train_step(css_mlp *mlp, const void *x_bf16, const float *t,
                       long long n, float lr, float *loss);
int css_mlp_params(css_mlp *mlp, int layer, float *w, float *b, int set);
int css_mlp_grads(css_mlp *mlp, int layer, float *gw, float *gb);
/* run the network's work on the caller's cudaStream_t (NULL: its own) */
int css_mlp_set_stream(css_mlp *mlp, void *stream);
/* forward passes of a 144/128/128/128/16 network run as one fused kernel:
 * on = 2 (the default) on the tcgen05 tensor cores (weights in shared
 * memory, 128-row tiles, FP32 accumulators in tensor memory), on = 1 on
 * BF16 mma.sync with the layers chained in registers, on = 0 the per-layer
 * GEMM path                                                               */
int css_mlp_set_fused(css_mlp *mlp, int on);

/* ---- diagnostics of the current state (vars0), computed on the device ----
 * Each call reads the state left by css_upload_state / css_step_rk4, uses
 * the stage buffers as scratch (so it must not overlap a step on another
 * stream), and returns on the host when its results are there.  For a
 * magnetic run B = curl A with Compute_B's boundary zeroing
 * (derivatives.f90:1830-1892) is formed first, as the reference's output
 * routines do.                                                             */

/* Scalar_Output (report_mpi.f90:173-262): out[7] = kinener, cke, mcke,
 * drke, umach, magener, bmax (the two magnetic entries are 0 for hydro).  */
#define CSS_NSCALARS 7
int css_scalars(css_ctx *ctx, double *out);

/* Compute_Step_Size (rhs_mpi.f90:92-275): out[5] = dtmax (the Courant limit
 * min(dtmaxb, dtmaxc, dtmaxd) times cfl_safety), Etot, Ltot, mtot, mrsint.
 * dtmaxd is the reference's 1e10 (no explicit Laplacian viscosity).       */
#define CSS_NSTEPSIZE 5
int css_step_size(css_ctx *ctx, double cfl_safety, double *out);

/* Shell_Average_Output (report_mpi.f90:783-1094): horizontal averages per
 * radius of quantities[0..nq) with the reference's codes 1..18 (1 rho,
 * 2 T, 3 s, 4 P, 5 v_r, 6 v_theta, 7 v_phi, 8 KE, 9 ds/dr, 10 B_r,
 * 11 B_theta, 12 B_phi, 13 ME, 14 |B_pol|, 15 F_ks, 16 F_en, 17 F_ke,
 * 18 F_ac); out is (nr, nq) in Fortran order, out[iq*nr + ir].  k0 (nr,
 * may be NULL = 0) is the prescribed radiative flux profile of F_ks.
 * Code 19 (the SLD entropy flux) and magnetic codes on a hydro run return
 * CSS_ERR_ARG.                                                             */
int css_shell_averages(css_ctx *ctx, const int *quantities, int nq,
                       const double *k0, double *out);

/* Horizontal spectrum per radius with the folding of
 * CSS-IDL/spectral_analysis_new.pro:16-25 (apodisation in theta, forward
 * 2D FFT normalised by 1/(nth nphi), F[kt,kp] + F[nth-kt,nphi-kp] kept as
 * a real number, summed over 1 <= kt < nth/2 and divided by nth/2) of one
 * snapshot: out[ir*(nphi/2) + kp], kp = 0..nphi/2-1.  kind 0 = kinetic
 * energy density rho|u|^2/2, 1 = magnetic energy density |B|^2/(8 pi),
 * 2+iv = state variable iv.  nth and nphi must be even.                    */
int css_spectrum(css_ctx *ctx, int kind, double *out);

/* ---- open radial boundaries (top_inout / bot_inout) ---------------------
 * The reference's Top_Inflow_Outflow and Bottom_Inflow_Outflow
 * (rhs_mpi.f90:1857-2067) read run state beyond the fields: the step index
 * and time of Program CSS2's loop (mhdsph_mpi.f90:28-43), the step size, the
 * mass totals m0, vol and mtot, the rain fields of the squall model and the
 * prescribed (ASH) bottom fields.  These calls set and read that state; the
 * step entry points advance it.  Every call returns CSS_ERR_ARG on a run
 * without an open boundary (except the clock, which every run keeps).     */

/* The clock: istep = the step index the RHS sees (the last step started),
 * sim_time, and deltat, the step size of the mean-flow terms
 * (rhs_mpi.f90:1882, :2012) for the RHS entry point.  Each step advances
 * istep by one before it and sim_time by dt after it, and sets deltat = dt.
 * Defaults 0, 0, 0.                                                        */
int css_set_clock(css_ctx *ctx, long long istep, double sim_time, double deltat);
int css_get_clock(css_ctx *ctx, long long *istep, double *sim_time);

/* Mass bookkeeping of the start-up (mhdsph_mpi.f90:863-947, :979-999): m0,
 * vol and mtot of the resident state.  The RHS refreshes mtot at the first
 * call of every step whose index is a multiple of ufreq (rhs_mpi.f90:
 * 326-353).  css_inout_state: out[0..3] = m0, vol, mtot, ash_fen_mod.     */
int css_inout_init(css_ctx *ctx);
int css_inout_state(css_ctx *ctx, double *out);

/* Entropy rain (do_entropy_rain): the squall fields dvel_rain, dent_rain
 * (entropy_rain.f90:40; nth*nphi each, [it + nth*ip]) the top relaxation
 * reads, set directly or built from squalls: sstruct 1 Gaussian squalls
 * (Build_Gaussian_Squalls, entropy_rain.f90:423-523), 0 polynomial ones
 * (Build_Polynomial_Squalls, :525-655); squalls[6*k ..] = theta_loc,
 * phi_loc, size, scaling, vel, dels.  The squall life cycle
 * (Update_Rain_Squalls, :171-421) is the caller's, between steps, as in the
 * reference.  Host pointers.                                              */
int css_set_rain_fields(css_ctx *ctx, const double *dvel_rain, const double *dent_rain);
int css_get_rain_fields(css_ctx *ctx, double *dvel_rain, double *dent_rain);
int css_build_squalls(css_ctx *ctx, int sstruct, int nsq, const double *squalls);
/* css_add_squalls: the same squalls added to the current fields instead of
 * replacing them -- Update_Rain_Squalls builds its squalls on top of the
 * downflow lanes (entropy_rain.f90:171-421). */
int css_add_squalls(css_ctx *ctx, int sstruct, int nsq, const double *squalls);
/* Downflow lanes of entropy rain (build_lanes): Build_Downflow_Lanes
 * (entropy_rain.f90:657-713) on the Voronoi cells of the convection-cell
 * sites.  cells[3*k ..] = phi_loc, theta_loc, scaling (>= 0) of the ncells
 * sites; the periodic copies one phi-domain width to each side are added
 * here (:80-89).  Replaces dvel_rain / dent_rain by meanvel and meands
 * times the lane field over max(its maximum, 1); meansize sets the lanes'
 * width (r2/meansize)^2 and, through isz_max (:58), the window a top block
 * sees.  The Voronoi cells are computed on the host (css_voronoi); the
 * field on the device.  The cells' life cycle is the caller's. */
int css_build_lanes(css_ctx *ctx, int ncells, const double *cells, double meansize,
                    double meanvel, double meands);
/* css_voronoi: Voronoi cells of n >= 3 distinct sites (x, y) in the form of
 * Compute_Voronoi (voronoi.f90:30-280): degree[g] vertices of site g's
 * cell at face[start[g] ..], indices into vxy (2 per vertex, nvert of
 * them: the circumcentres of the Delaunay triangles); a cell inside the
 * hull is walked clockwise, one on the hull from its most clockwise
 * triangle counterclockwise.  face needs room for 6n entries, vxy for 4n.
 * Host only (no device work). */
int css_voronoi(int n, const double *x, const double *y, int *degree, int *start,
                int *face, int *nvert, double *vxy);

/* Prescribed bottom (bottom_specified): the four time slices of the ASH
 * fields after the reader's spatial interpolation and wall taper
 * (ash_inflow.f90:18-120), slices[((is*4 + iq)*nphi + ip)*nth + it] with
 * iq = 0 u_r, 1 u_theta, 2 u_phi, 3 entropy (ashvars(:,:,1..4)); their
 * times (ashtimes, from the data's start); and the enthalpy-flux factor
 * ash_fen_mod.  Each step interpolates the slices at its start time
 * (Cubic_Time_Interp, :188-219); a step that would start at sim_time >=
 * times[2] returns CSS_ERR_ARG, as the reference would read the next slice
 * there (Read_ASH_Inflow, :124-186): the caller shifts it in first.  Every
 * ufreq steps ash_fen_mod is updated from the bottom enthalpy flux
 * (ASH_Enthalpy_Flux, step_rk4.f90:495-518).  Host pointers.              */
int css_set_ash_slices(css_ctx *ctx, const double *slices, const double *times, double ash_fen_mod);

#ifdef __cplusplus
}
#endif
#endif /* CSS_B200_H */
