// css_api.cu -- C ABI of the CSS B200 library (include/css_b200.h): context
// set-up (virtual decomposition, LU tables, profiles), device buffers, the
// RK4 step loop and the parity entry points.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>
#include <sys/stat.h>

#include "../../include/css_b200.h"
#include "css_kernels.cuh"
#include "css_stats.cuh"
#include "css_closure.cuh"
#include "css_lap.cuh"
#include "css_inout.cuh"
#include "css_fused.cuh"
#include "css_voronoi.h"

using namespace css;

static thread_local char g_err[512];
static void set_err(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}
extern "C" const char *css_last_error(void) { return g_err; }

#define CUDA_TRY(x)                                                                  \
  do {                                                                               \
    cudaError_t e_ = (x);                                                            \
    if (e_ != cudaSuccess) {                                                         \
      set_err("%s:%d %s: %s", __FILE__, __LINE__, #x, cudaGetErrorString(e_));       \
      return e_ == cudaErrorMemoryAllocation ? CSS_ERR_NOMEM : CSS_ERR_CUDA;         \
    }                                                                                \
  } while (0)

// kernel kinds, for the per-kernel CUDA-event timing of css_profile
enum KernelId { KI_THETA = 0, KI_PHI, KI_RADIAL, KI_RHOT_UPDATE, KI_CURL_THETA, KI_CURL_PHI, KI_CURL_R,
                KI_SLD_VCC, KI_SLD, KI_SLD_OHMIC, KI_DERIV, KI_THPH, KI_RSTAGE, KI_COUNT };
static const char *kKernelNames[KI_COUNT] = {"theta_terms", "phi_terms", "radial_terms", "rhot_update",
                                             "curl_theta", "curl_phi", "curl_r", "sld_vcc", "sld", "sld_ohmic",
                                             "deriv", "thph", "rstage"};

struct css_ctx {
  css_params p;
  CssGeo g;
  int nv;
  size_t ncell;
  cudaStream_t stream;
  // device buffers
  double *tab, *prof, *theta_prof, *sld_geo, *resp;
  int *rblk;
  double *v0, *vA, *vB, *dv, *vs;  // state, stage ping-pong, tendency, RK accumulator
  double *bf;                       // B = curl A (MHD)
  double *vcc;                      // SLD speed^2
  double *cda;                      // curl of the A-tendency (MHD ohmic heating)
  double *tbuf;                     // temperature of the current stage input
  double *rtw = nullptr;            // two-pass stage: zero-datum d(rho)/dtheta on the theta-wall blocks
  double *cyc = nullptr;            // cyclic phi derivative tables, per order: w, piv, z (nphi each), v.z
  double *bg2 = nullptr;            // mixed precision: rho and s backgrounds, [2][nr][nth]
  // adjoints of css_deriv (torch backward): dense block operators per
  // (direction, order, bdry), built on first use, and their block offsets
  double *adjM[3][2][5] = {};
  int *adjOff[3][2][5] = {};
  PlaneMaps pmaps[5];               // two-pass stage: TMA maps of v0, vA, vB, bf (plane kernel) and vs (curl)
  int vs_map = 0;                   // pmaps[4] and vs_slab hold vs's maps
  SlabMaps vs_slab;
  SlabMaps smaps[5];                // the same for the stage kernel's slabs, then rtw
  double *lapbuf = nullptr;         // explicit viscosity: 6 derivative + 6 kept fields
  double *lapface = nullptr;        // explicit viscosity: face data, 6 x max face size
  double *radbuf = nullptr;         // radiative diffusion: d ln(rho)/dr, ds/dr, 8 derivative fields
  double *radface = nullptr;        // radiative diffusion: face data, 6 x max face size
  // open radial boundaries: face scalars and mass totals (IO_COUNT), block
  // parts of the face sums, rain fields (2 x nth*nphi), ASH slices (16 x
  // nth*nphi), the interpolated bottom fields (4 x nth*nphi), squalls
  double *io = nullptr, *io_part = nullptr, *rain = nullptr, *ash_slices = nullptr, *ashv = nullptr;
  double *squalls = nullptr;
  int squall_cap = 0;
  double *lanes = nullptr;  // lane samples (3 per sample) + the running maximum's 8 bytes
  size_t lane_cap = 0;
  // the run's clock: the step index the RHS sees (Program CSS2's istep),
  // sim_time, deltat; the ASH slice times; the RHS call number in progress
  long long istep = 0;
  double sim_time = 0.0, deltat = 0.0, ash_times[4] = {0.0, 0.0, 0.0, 0.0};
  int rhs_call = 0;
  double dtd = 1e10;                // viscous time-step limit of Compute_Step_Size
  double rep_flux_lo = 0.0, rep_flux_hi = 0.0;  // dsdr1/dxdr(1), dsdr2/dxdr(nr) of the reports
  int mt[3];                        // compile-time block length per direction (0 = generic)
  int *flag;
  long long launches;
  int tl_theta, tl_phi, tl_r;
  int phi_pers = 0;                 // 1: persistent double-buffered phi kernel (autotuned)
  int fused_ok = 0;                 // the run qualifies for the two-pass RK4 stage (css_fused.cuh)
  int fused = 0;                    // 1: FP64 RK4 stages run k_thph + k_rstage
  int curl_tp = 2;                  // B = curl A's theta and phi parts: 0 two passes, 1 one pass (k_curl_tp),
                                    // 2 one pass from TMA-staged planes (k_curl_pl) where the maps exist
  int nsm = 148;                    // SMs of the device
  cudaStream_t own_stream;
  // per-kernel event timing (css_profile)
  int profiling;
  std::vector<cudaEvent_t> ev;     // pairs (start, stop)
  std::vector<int> ev_kind;
  size_t ev_used;
  double k_ms[KI_COUNT];
  long long k_count[KI_COUNT];
};

static void prof_begin(css_ctx *c, int kind) {
  if (!c->profiling) return;
  if (c->ev_used + 2 > c->ev.size()) {
    for (int i = 0; i < 64; i++) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      c->ev.push_back(e);
    }
    c->ev_kind.resize(c->ev.size() / 2);
  }
  c->ev_kind[c->ev_used / 2] = kind;
  cudaEventRecord(c->ev[c->ev_used], c->stream);
}
static void prof_end(css_ctx *c) {
  if (!c->profiling) return;
  cudaEventRecord(c->ev[c->ev_used + 1], c->stream);
  c->ev_used += 2;
}
static void prof_collect(css_ctx *c) {
  if (c->ev_used == 0) return;
  cudaStreamSynchronize(c->stream);
  for (size_t i = 0; i + 1 < c->ev_used; i += 2) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[i], c->ev[i + 1]);
    int k = c->ev_kind[i / 2];
    c->k_ms[k] += ms;
    c->k_count[k] += 1;
  }
  c->ev_used = 0;
}

// ---------------------------------------------------------------------------
// LU tables (Initialize_Derivatives, derivatives.f90:106-287 for r/theta,
// :172-219 for phi), 1-based arrays g1|g2|g3 per bdry.
// ---------------------------------------------------------------------------
static void tab_d1(int m, int lphys, int rphys, int iv, double *g1, double *g2, double *g3) {
  double alpha = 1.0 / 3.0, a2 = 0.75, g2c = 0.125, a1 = 6.0, b1 = 3.0;
  double cn = 1.0 / (a2 - b1 * g2c);
  double up1 = (a1 * a2 - b1) * cn, up2;
  up2 = ((iv != 1) && (iv != 2)) ? 0.0 : up1;
  if (iv % 2 == 0) up1 = 0.0;
  double c1 = 1.0, c2 = 1.0, c3;
  g1[1] = g2[1] = g3[1] = c2;
  if (lphys) {
    c3 = up1 * c2; g1[2] = c3; c2 = c1 / (c1 - g2c * c3); g2[2] = c2;
    c3 = a2 * c2; g1[3] = c3; c2 = c1 / (c1 - alpha * c3); g2[3] = c2;
    g3[2] = -g2c * g2[2];
  } else {
    c3 = alpha * c2; g1[2] = c3; c2 = c1 / (c1 - alpha * c3); g2[2] = c2;
    g3[2] = -alpha * g2[2];
    c3 = alpha * c2; g1[3] = c3; c2 = c1 / (c1 - alpha * c3); g2[3] = c2;
  }
  for (int i = 4; i <= m - 2; i++) { c3 = alpha * c2; g1[i] = c3; c2 = c1 / (c1 - alpha * c3); g2[i] = c2; }
  for (int i = 3; i <= m - 2; i++) g3[i] = -alpha * g2[i];
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

static void tab_d2(int m, int lphys, int rphys, int iv, double *g1, double *g2, double *g3) {
  static const double U1[5] = {707.0 / 193.0, 137.0 / 13.0, 707.0 / 193.0, 137.0 / 13.0, 707.0 / 193.0};
  static const double U2[5] = {707.0 / 193.0, 137.0 / 13.0, 137.0 / 13.0, 707.0 / 193.0, 707.0 / 193.0};
  double alpha = 2.0 / 11.0, up1 = U1[iv], up2 = U2[iv];
  double a2 = -0.35, g2c = 0.1;
  double c1 = 1.0, c2 = 1.0, c3;
  g1[1] = g2[1] = g3[1] = c2;
  if (lphys) {
    c3 = up1; g1[2] = c3; c2 = c1 / (c1 - g2c * c3); g2[2] = c2;
    c3 = a2 * c2; g1[3] = c3; c2 = c1 / (c1 - alpha * c3); g2[3] = c2;
    g3[2] = -g2c * g2[2];
  } else {
    c3 = alpha * c2; g1[2] = c3; c2 = c1 / (c1 - alpha * c3); g2[2] = c2;
    g3[2] = -alpha * g2[2];
    c3 = alpha * c2; g1[3] = c3; c2 = c1 / (c1 - alpha * c3); g2[3] = c2;
  }
  for (int i = 4; i <= m - 2; i++) { c3 = alpha * c2; g1[i] = c3; c2 = c1 / (c1 - alpha * c3); g2[i] = c2; }
  for (int i = 3; i <= m - 2; i++) g3[i] = -alpha * g2[i];
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

static void tab_p(int m, double alpha, double *g1, double *g2, double *g3) {
  double c1 = 1.0, c2 = 1.0, c3;
  g1[1] = g2[1] = g3[1] = c1;
  c3 = alpha * c2; g1[2] = c3; c2 = c1 / (c1 - alpha * c3); g2[2] = c2;
  g3[2] = -alpha * g2[2];
  for (int i = 3; i <= m; i++) { c3 = alpha * c2; g1[i] = c3; c2 = c1 / (c1 - alpha * c3); g2[i] = c2; }
  for (int i = 3; i <= m; i++) g3[i] = -alpha * g2[i];
  for (int j = 1; j <= m; j++) g1[j] = -g1[j];
}

// Partition (parallel_mpi.f90:236-343): the remainder goes to the first blocks
static int partition(int n, int nn, int *start, int *size) {
  int base = n / nn;
  if (base < 9) return -1;
  int irem = n % nn;
  int pos = 0;
  for (int i = 0; i < nn; i++) {
    int sz = (irem > 0 && (i == 0 || i + 1 <= irem)) ? base + 1 : base;
    start[i] = pos;
    size[i] = sz;
    pos += sz;
  }
  return 0;
}

static size_t smem_theta(int nh, int nd, int m, int TL) { return 8 * ((size_t)nh * TL * (m + 9) + (size_t)nd * TL * (m + 1)); }
// shared memory of the RHS kernels: tiles + derivative buffers + staged LU tables
static size_t smem_theta_terms(int mag, int m, int TL) {
  int nh = mag ? 6 : 4, nd = mag ? 7 : 5;
  return 8 * ((size_t)nh * TL * (m + 9) + (size_t)nd * TL * (m + 1) + (size_t)nd * 3 * (m + 2));
}
static size_t smem_phi_terms(int mag, int m, int TL) {
  int nh = mag ? 7 : 5, nd = mag ? 8 : 6;
  return 8 * ((size_t)nh * (m + 8) * (TL + 1) + (size_t)nd * m * (TL + 1) + (size_t)2 * 3 * (m + 2));
}
static size_t smem_radial_terms(int mag, int m, int TL) {
  int nh = mag ? 7 : 5, nd = mag ? 8 : 6;
  return 8 * ((size_t)nh * (m + 8) * TL + (size_t)nd * m * TL + (size_t)nd * 3 * (m + 2) + TL);
}
static size_t smem_rhot(int m, int TL) { return 8 * ((size_t)TL * (m + 9) + (size_t)TL * (m + 1) + 3 * (m + 2)); }
static size_t smem_line(int nh, int nd, int na, int m, int TL) {
  return 8 * ((size_t)nh * (m + 8) * (TL + 1) + (size_t)(nd + na) * m * (TL + 1));
}
static const size_t kSmemCap = 100 * 1024;

extern "C" void css_destroy(css_ctx *c) {
  if (!c) return;
  cudaFree(c->tab); cudaFree(c->prof); cudaFree(c->theta_prof); cudaFree(c->rblk); cudaFree(c->sld_geo); cudaFree(c->resp);
  cudaFree(c->v0); cudaFree(c->vA); cudaFree(c->vB); cudaFree(c->dv); cudaFree(c->vs);
  for (int d = 0; d < 3; d++)
    for (int o = 0; o < 2; o++)
      for (int b = 0; b < 5; b++) { cudaFree(c->adjM[d][o][b]); cudaFree(c->adjOff[d][o][b]); }
  cudaFree(c->bf); cudaFree(c->vcc); cudaFree(c->cda); cudaFree(c->flag); cudaFree(c->tbuf); cudaFree(c->rtw); cudaFree(c->cyc); cudaFree(c->bg2);
  cudaFree(c->lapbuf); cudaFree(c->lapface); cudaFree(c->radbuf); cudaFree(c->radface);
  cudaFree(c->io); cudaFree(c->io_part); cudaFree(c->rain); cudaFree(c->ash_slices); cudaFree(c->ashv);
  cudaFree(c->squalls);
  cudaFree(c->lanes);
  for (auto e : c->ev) cudaEventDestroy(e);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
}

template <int MT, int TLC>
static int setup_mt() {
  int mx = 200 * 1024;
#define CSS_SMEM_ATTR(...) CUDA_TRY(cudaFuncSetAttribute(__VA_ARGS__, cudaFuncAttributeMaxDynamicSharedMemorySize, mx))
  CSS_SMEM_ATTR(k_theta_terms<MT, TLC, double, 0>);
  CSS_SMEM_ATTR(k_theta_terms<MT, TLC, float, 0>);
  CSS_SMEM_ATTR(k_phi_terms<MT, TLC, double, 0>);
  CSS_SMEM_ATTR(k_phi_terms<MT, TLC, float, 0>);
  CSS_SMEM_ATTR(k_theta_terms<MT, TLC, double, 1>);
  CSS_SMEM_ATTR(k_theta_terms<MT, TLC, float, 1>);
  CSS_SMEM_ATTR(k_phi_terms<MT, TLC, double, 1>);
  CSS_SMEM_ATTR(k_phi_terms<MT, TLC, float, 1>);
  CSS_SMEM_ATTR(k_radial_terms<MT, TLC, double, 0>);
  CSS_SMEM_ATTR(k_radial_terms<MT, TLC, float, 0>);
  CSS_SMEM_ATTR(k_radial_terms<MT, TLC, double, 1>);
  CSS_SMEM_ATTR(k_radial_terms<MT, TLC, float, 1>);
  CSS_SMEM_ATTR(k_radial_terms<MT, TLC, double, 2>);
  CSS_SMEM_ATTR(k_radial_terms<MT, TLC, float, 2>);
  CSS_SMEM_ATTR(k_rhot_update<MT, TLC, double, double>);
  CSS_SMEM_ATTR(k_rhot_update<MT, TLC, double, double, 1>);
  CSS_SMEM_ATTR(k_rhot_update<MT, TLC, double, double, 2>);
  CSS_SMEM_ATTR(k_rhot_update<MT, TLC, double, double, 3>);
  CSS_SMEM_ATTR(k_rhot_update<MT, TLC, double, double, 4>);
  CSS_SMEM_ATTR(k_rhot_update<MT, TLC, double, float, 1>);
  CSS_SMEM_ATTR(k_rhot_update<MT, TLC, float, float, 2>);
  CSS_SMEM_ATTR(k_rhot_update<MT, TLC, float, float, 3>);
  CSS_SMEM_ATTR(k_rhot_update<MT, TLC, float, double, 4>);
  CSS_SMEM_ATTR(k_rhot_update<MT, TLC, double, float>);
  CSS_SMEM_ATTR(k_rhot_update<MT, TLC, float, float>);
  CSS_SMEM_ATTR(k_rhot_update<MT, TLC, float, double>);
  CSS_SMEM_ATTR(k_curl_theta<MT, TLC, double>);
  CSS_SMEM_ATTR(k_curl_theta<MT, TLC, float>);
  CSS_SMEM_ATTR(k_curl_phi<MT, TLC, double>);
  CSS_SMEM_ATTR(k_curl_phi<MT, TLC, float>);
  CSS_SMEM_ATTR(k_curl_r<MT, TLC, double>);
  CSS_SMEM_ATTR(k_curl_r<MT, TLC, float>);
  if constexpr (MT > 0 && TLC > 0) CSS_SMEM_ATTR(k_phi_terms_p<MT, TLC>);
#undef CSS_SMEM_ATTR
  return CSS_OK;
}

static int setup_kernels() {
  static bool done = false;
  if (done) return CSS_OK;
  if (int rc = setup_mt<0, 0>()) return rc;
  CUDA_TRY(cudaFuncSetAttribute(k_sld<4, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SldSmem<4>)));
  CUDA_TRY(cudaFuncSetAttribute(k_sld<5, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SldSmem<5>)));
  CUDA_TRY(cudaFuncSetAttribute(k_sld<3, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SldSmem<3>)));
  CUDA_TRY(cudaFuncSetAttribute(k_curl_tp<32, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
  CUDA_TRY(cudaFuncSetAttribute(k_curl_pl<1, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)CurlCfg<1, 128>::SMEM));
  CUDA_TRY(cudaFuncSetAttribute(k_curl_tp<32, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
  if (int rc = setup_mt<16, 16>()) return rc;
  if (int rc = setup_mt<32, 16>()) return rc;
  if (int rc = setup_mt<16, 8>()) return rc;
  if (int rc = setup_mt<32, 8>()) return rc;
  int mx = 200 * 1024;
#define CSS_FUSED_ATTR(K, CFG) \
  CUDA_TRY(cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CFG::SMEM))
  CSS_FUSED_ATTR(k_thph<0>, ThphCfg<0>);
  CSS_FUSED_ATTR(k_thph<1>, ThphCfg<1>);
  CSS_FUSED_ATTR((k_rstage<0, 1>), RstageCfg<0>);
  CSS_FUSED_ATTR((k_rstage<0, 2>), RstageCfg<0>);
  CSS_FUSED_ATTR((k_rstage<0, 3>), RstageCfg<0>);
  CSS_FUSED_ATTR((k_rstage<0, 4>), RstageCfg<0>);
  CSS_FUSED_ATTR((k_rstage<1, 1>), RstageCfg<1>);
  CSS_FUSED_ATTR((k_rstage<1, 2>), RstageCfg<1>);
  CSS_FUSED_ATTR((k_rstage<1, 3>), RstageCfg<1>);
  CSS_FUSED_ATTR((k_rstage<1, 4>), RstageCfg<1>);
#undef CSS_FUSED_ATTR
  CUDA_TRY(cudaFuncSetAttribute(k_deriv_theta<1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  CUDA_TRY(cudaFuncSetAttribute(k_deriv_theta<2, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  CUDA_TRY(cudaFuncSetAttribute(k_deriv_phi<1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  CUDA_TRY(cudaFuncSetAttribute(k_deriv_phi<2, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  CUDA_TRY(cudaFuncSetAttribute(k_deriv_r<1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  CUDA_TRY(cudaFuncSetAttribute(k_deriv_r<2, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  done = true;
  return CSS_OK;
}

// launch KERNEL<MT> with MT = c->mt[DIR] chosen at run time
// and the compile-time tile of TLV lines (8 or 16) when MT > 0; XT is the
// parenthesised list of the kernel's storage-type template arguments
#define CSS_STRIP(...) __VA_ARGS__
#define LAUNCH_MT(DIR, TLV, KERNEL, XT, GRID, SMEM, ...)                                 \
  do {                                                                                    \
    switch (c->mt[DIR] * 100 + (TLV)) {                                                   \
      case 1616: KERNEL<16, 16, CSS_STRIP XT><<<GRID, 128, SMEM, c->stream>>>(__VA_ARGS__); break; \
      case 3216: KERNEL<32, 16, CSS_STRIP XT><<<GRID, 128, SMEM, c->stream>>>(__VA_ARGS__); break; \
      case 1608: KERNEL<16, 8, CSS_STRIP XT><<<GRID, 128, SMEM, c->stream>>>(__VA_ARGS__); break;  \
      case 3208: KERNEL<32, 8, CSS_STRIP XT><<<GRID, 128, SMEM, c->stream>>>(__VA_ARGS__); break;  \
      default: KERNEL<0, 0, CSS_STRIP XT><<<GRID, 128, SMEM, c->stream>>>(__VA_ARGS__); break;     \
    }                                                                                     \
  } while (0)

// Tables of the cyclic phi derivative (k_dbydp_cyclic) for n points:
// B = tridiag(alpha, 1, alpha) with first diagonal 1 - gamma and last
// 1 - alpha^2/gamma (gamma = -1); elimination factors w[j] = alpha /
// piv[j-1], pivots piv[j] = b_j - alpha w[j], z = B^-1 u with u = (gamma,
// 0.., alpha), and v.z = z[0] + (alpha/gamma) z[n-1].  out: w | piv | z | v.z
static void cyclic_tables(int n, int order, double *out) {
  const double alpha = order == 1 ? 1.0 / 3.0 : 2.0 / 11.0, gamma = -1.0;
  double *w = out, *piv = out + n, *z = out + 2 * n;
  w[0] = 0.0;
  piv[0] = 1.0 - gamma;
  for (int j = 1; j < n; j++) {
    w[j] = alpha / piv[j - 1];
    const double bj = j == n - 1 ? 1.0 - alpha * alpha / gamma : 1.0;
    piv[j] = bj - alpha * w[j];
  }
  // z: forward then back substitution on u
  z[0] = gamma / piv[0];
  for (int j = 1; j < n; j++) z[j] = ((j == n - 1 ? alpha : 0.0) - alpha * z[j - 1]) / piv[j];
  for (int j = n - 2; j >= 0; j--) z[j] -= w[j + 1] * z[j + 1];
  out[3 * n] = z[0] + (alpha / gamma) * z[n - 1];
}

// TMA maps of the two-pass stage's plane staging (css_fused.cuh
// thph_stage_tma): for each state buffer (vars0, the two stage buffers) and
// B, a 4-D FP64 map (theta, phi, r, field) with a 42x32 main-row box and a
// 32x4 phi-halo box.  Returns false when the driver offers no encoder (the
// run then keeps the four-kernel stage).
static bool plane_maps(css_ctx *c) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q;
    void *fn = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return false;
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  const CssGeo &g = c->g;
  double *bufs[4] = {c->v0, c->vA, c->vB, c->bf};
  for (int k = 0; k < 4; k++) {
    if (!bufs[k]) {
      memset(&c->pmaps[k], 0, sizeof(PlaneMaps));
      memset(&c->smaps[k], 0, sizeof(SlabMaps));
      continue;
    }
    const cuuint64_t dims[4] = {(cuuint64_t)g.nth, (cuuint64_t)g.nphi, (cuuint64_t)g.nr, (cuuint64_t)(k < 3 ? c->nv : 3)};
    const cuuint64_t strides[3] = {(cuuint64_t)g.nth * 8, (cuuint64_t)g.nth * g.nphi * 8, (cuuint64_t)c->ncell * 8};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const cuuint32_t bmain[4] = {FA_RW, FM, 1, 1}, bhalo[4] = {FM, 4, 1, 1};
    if (encode(&c->pmaps[k].main, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, bufs[k], dims, strides, bmain, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
    if (encode(&c->pmaps[k].halo, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, bufs[k], dims, strides, bhalo, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
    // the stage kernel's slab box: 32 theta x 1 phi x 40 r
    const cuuint32_t bslab[4] = {FM, 1, FM + 8, 1};
    if (encode(&c->smaps[k].slab, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, bufs[k], dims, strides, bslab, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
  }
  memset(&c->pmaps[4], 0, sizeof(PlaneMaps));
  c->vs_map = 0;
  if (c->vs && c->g.magnetic) {  // the SLD tendency: the ohmic heating's curl of its A part
    const cuuint64_t dims[4] = {(cuuint64_t)g.nth, (cuuint64_t)g.nphi, (cuuint64_t)g.nr, (cuuint64_t)c->nv};
    const cuuint64_t strides[3] = {(cuuint64_t)g.nth * 8, (cuuint64_t)g.nth * g.nphi * 8, (cuuint64_t)c->ncell * 8};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const cuuint32_t bmain[4] = {FA_RW, FM, 1, 1}, bhalo[4] = {FM, 4, 1, 1};
    if (encode(&c->pmaps[4].main, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, c->vs, dims, strides, bmain, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS ||
        encode(&c->pmaps[4].halo, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, c->vs, dims, strides, bhalo, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      memset(&c->pmaps[4], 0, sizeof(PlaneMaps));  // the ohmic curl keeps its tile kernels
    else {
      const cuuint32_t bslab[4] = {FM, 1, FM + 8, 1};
      if (encode(&c->vs_slab.slab, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, c->vs, dims, strides, bslab, estr,
                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS)
        c->vs_map = 1;
    }
  }
  {  // rtw: (theta 32, side 2, phi, r), box 32 x 1 x 1 x 32
    const cuuint64_t dims[4] = {32, 2, (cuuint64_t)g.nphi, (cuuint64_t)g.nr};
    const cuuint64_t strides[3] = {32 * 8, 64 * 8, (cuuint64_t)g.nphi * 64 * 8};
    const cuuint32_t estr[4] = {1, 1, 1, 1}, box[4] = {FM, 1, 1, FM};
    if (encode(&c->smaps[4].slab, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, c->rtw, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
  }
  return true;
}

extern "C" int css_create(const css_params *pp, const double *prof, css_ctx **out) {
  if (!out) { set_err("css_create: NULL out"); return CSS_ERR_ARG; }
  *out = nullptr;
  if (!pp || !prof) { set_err("css_create: NULL argument"); return CSS_ERR_ARG; }
  const css_params &p = *pp;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_err("css_create: no CUDA device");
    return CSS_ERR_NODEV;
  }
  if (p.nnr < 2 || p.nnt < 2 || p.nnp < 3) {
    set_err("css_create: the reference needs nnr>=2, nnt>=2 (no dtype 0 case, derivatives.f90:564) and nnp>=3 "
            "(phi halos from distinct neighbours, parallel_mpi.f90:646-665)");
    return CSS_ERR_DECOMP;
  }
  if (p.nnr > CSS_MAXBLK || p.nnt > CSS_MAXBLK || p.nnp > CSS_MAXBLK) {
    set_err("css_create: at most %d blocks per direction", CSS_MAXBLK);
    return CSS_ERR_DECOMP;
  }
  if (p.flux_limiter > 0 || p.ent_flux_limiter > 0 || p.mag_flux_limiter > 0 || p.bottom_constant_temp ||
      (p.top_constant_temp && p.set_stop) || p.dstype != 1 || p.xi_cs > 1.0) {
    set_err("css_create: unsupported option (SLD power flux limiter, bottom constant temperature, Set_Stop, "
            "dstype != 1 or xi_cs > 1)");
    return CSS_ERR_ARG;
  }
  if (p.magnetic && p.do_ohmic_heating && !p.magnetic_diffusion) {
    set_err("css_create: ohmic heating needs magnetic diffusion");
    return CSS_ERR_ARG;
  }
  if (p.time_stepper != 0 && p.time_stepper != 2 && p.time_stepper != 3 && p.time_stepper != 4) {
    set_err("css_create: time_stepper %d unknown (4 RK4, 2 RK2-TVD, 3 RK3-TVD)", p.time_stepper);
    return CSS_ERR_ARG;
  }
  if (p.sldiffusion && (p.nth % 2)) {
    // the SLD kernel streams theta pairs with 16-byte copies
    set_err("css_create: slope-limited diffusion needs an even nth (got %d)", p.nth);
    return CSS_ERR_ARG;
  }
  if (p.precision != 0 && p.precision != 1) {
    set_err("css_create: precision %d unknown (0 FP64, 1 mixed: FP32 stage states)", p.precision);
    return CSS_ERR_ARG;
  }
  if (p.do_radheat && p.precision != 0) {
    set_err("css_create: radiative diffusion runs in FP64 only");
    return CSS_ERR_ARG;
  }
  if (p.laplacian && p.precision != 0) {
    set_err("css_create: explicit viscosity runs in FP64 only (the FP32 stage states are not built for it)");
    return CSS_ERR_ARG;
  }
  const bool open_r = p.top_inout || p.bot_inout;
  if ((open_r || p.bottom_specified || p.do_entropy_rain) &&
      (p.magnetic || p.laplacian || p.do_radheat || p.precision != 0)) {
    set_err("css_create: open radial boundaries are built for hydro FP64 runs without explicit viscosity or "
            "radiative diffusion");
    return CSS_ERR_ARG;
  }
  if ((p.bottom_specified && !p.bot_inout) || (p.do_entropy_rain && !p.top_inout)) {
    set_err("css_create: bottom_specified needs bot_inout and do_entropy_rain needs top_inout");
    return CSS_ERR_ARG;
  }
  css_ctx *c = new css_ctx();
  c->p = p;
  c->nv = p.magnetic ? 8 : 5;
  c->ncell = (size_t)p.nr * p.nth * p.nphi;
  CssGeo &g = c->g;
  memset(&g, 0, sizeof g);
  g.nr = p.nr; g.nth = p.nth; g.nphi = p.nphi; g.nv = c->nv;
  g.magnetic = p.magnetic; g.non_uniform = p.non_uniform;
  g.ncell = (long long)c->ncell;
  int ns[3] = {p.nr, p.nth, p.nphi}, nn[3] = {p.nnr, p.nnt, p.nnp};
  for (int d = 0; d < 3; d++) {
    CssDir &D = g.d[d];
    D.nb = nn[d];
    if (partition(ns[d], nn[d], D.start, D.size)) {
      set_err("css_create: fewer than 9 points per block (parallel_mpi.f90:250-315)");
      css_destroy(c);
      return CSS_ERR_DECOMP;
    }
    D.maxm = 0;
    for (int b = 0; b < nn[d]; b++) {
      if (D.size[b] % 2 || D.size[b] < 10 || D.size[b] > CSS_MAXM) {
        set_err("css_create: block sizes must be even and in [10, %d] (the reference's paired sweeps read an "
                "unset row for odd sizes, derivatives.f90:755-792)", CSS_MAXM);
        css_destroy(c);
        return CSS_ERR_DECOMP;
      }
      D.maxm = D.size[b] > D.maxm ? D.size[b] : D.maxm;
      D.lphys[b] = (d < 2) && b == 0;
      D.rphys[b] = (d < 2) && b == nn[d] - 1;
    }
  }
  // host copies of the profiles
  const int nr = p.nr, nth = p.nth, nphi = p.nphi;
  std::vector<double> P(prof, prof + (size_t)CSS_NPROF * nr);
  const double *x_ind = &P[CSS_PROF_X * nr], *r_ind = &P[CSS_PROF_R * nr];
  std::vector<double> dxdr(P.begin() + CSS_PROF_DXDR * nr, P.begin() + (CSS_PROF_DXDR + 1) * nr);
  std::vector<double> d2xdr2(P.begin() + CSS_PROF_D2XDR2 * nr, P.begin() + (CSS_PROF_D2XDR2 + 1) * nr);
  if (!p.non_uniform) for (int i = 0; i < nr; i++) { dxdr[i] = 1.0; d2xdr2[i] = 1.0; }
  double dth = (p.th2 - p.th1) / (double)(nth - 1), dphi = (p.phi2 - p.phi1) / (double)nphi;
  std::vector<double> theta(nth), phi(nphi), sines(nth), cosines(nth);
  for (int i = 0; i < nth; i++) { theta[i] = dth * (double)i + p.th1; sines[i] = sin(theta[i]); cosines[i] = cos(theta[i]); }
  for (int i = 0; i < nphi; i++) phi[i] = dphi * (double)i + p.phi1;
  // block spacings (derivatives.f90:91-97)
  const std::vector<double> *coords[3] = {nullptr, &theta, &phi};
  for (int d = 0; d < 3; d++) {
    CssDir &D = g.d[d];
    for (int b = 0; b < D.nb; b++) {
      int a0 = D.start[b], a1 = D.start[b] + D.size[b] - 1;
      double v = d == 0 ? 1.0 / (x_ind[a1] - x_ind[a0]) : 1.0 / ((*coords[d])[a1] - (*coords[d])[a0]);
      D.dnum[b] = (double)(D.size[b] - 1) * v;
    }
  }
  // tables
  int maxm = std::max(g.d[0].maxm, std::max(g.d[1].maxm, g.d[2].maxm));
  g.tstride = maxm + 2;
  const int ts = g.tstride;
  std::vector<double> T;
  for (int d = 0; d < 3; d++) {
    CssDir &D = g.d[d];
    for (int b = 0; b < D.nb; b++) {
      int m = D.size[b];
      for (int order = 1; order <= 2; order++) {
        int nbd = (d == 2) ? 1 : 5;
        int off = (int)T.size();
        T.resize(T.size() + (size_t)nbd * 3 * ts, 0.0);
        for (int iv = 0; iv < nbd; iv++) {
          double *g1 = &T[off + (size_t)iv * 3 * ts], *g2 = g1 + ts, *g3 = g2 + ts;
          if (d == 2) tab_p(m, order == 1 ? 1.0 / 3.0 : 2.0 / 11.0, g1, g2, g3);
          else if (order == 1) tab_d1(m, D.lphys[b], D.rphys[b], iv, g1, g2, g3);
          else tab_d2(m, D.lphys[b], D.rphys[b], iv, g1, g2, g3);
        }
        (order == 1 ? D.tab1 : D.tab2)[b] = off;
      }
    }
  }
  // unit responses of the first-derivative system of rho to its face datum
  // on the blocks with a physical face: resp = A^-1 e_1 (low face) / A^-1
  // e_m (high face), by the same sweeps the kernels run.  Radial blocks
  // (bdry ibcr(1)) first, then theta blocks (bdry ibct(1), for the two-pass
  // stage's Density_Terms_Theta on the theta walls).
  std::vector<double> RESP((size_t)2 * (g.d[0].nb + g.d[1].nb) * ts, 0.0);
  for (int dir = 0; dir < 2; dir++) {
    const int bdry = 4;  // lbcr_rho, lbct_rho (Read_Input, mhdsph_mpi.f90:1362)
    const CssDir &D = g.d[dir];
    const size_t off0 = dir == 0 ? 0 : (size_t)2 * g.d[0].nb * ts;
    for (int b = 0; b < D.nb; b++) {
      int m = D.size[b];
      const double *g1 = &T[D.tab1[b] + (size_t)bdry * 3 * ts], *g2 = g1 + ts, *g3 = g2 + ts;
      for (int side = 0; side < 2; side++) {
        bool on = side == 0 ? (D.lphys[b] && (bdry == 2 || bdry == 4)) : (D.rphys[b] && (bdry == 3 || bdry == 4));
        if (!on) continue;
        std::vector<double> d(m + 2, 0.0), t(m + 2, 0.0), x(m + 2, 0.0);
        d[side == 0 ? 1 : m] = 1.0;
        const double a1 = -1.0 / 3.0;
        t[1] = g2[1] * d[1];
        t[2] = g2[2] * d[2] + g3[2] * t[1];
        for (int j = 3; j <= m - 2; j++) t[j] = g2[j] * (d[j] + a1 * t[j - 1]);
        t[m - 1] = g2[m - 1] * d[m - 1] + g3[m - 1] * t[m - 2];
        t[m] = g2[m] * d[m] + g3[m] * t[m - 1];
        x[m] = t[m];
        for (int j = m - 1; j >= 1; j--) x[j] = t[j] + g1[j + 1] * x[j + 1];
        double *dst = &RESP[off0 + (size_t)(2 * b + side) * ts];
        for (int j = 1; j <= m; j++) dst[j] = x[j];
      }
    }
  }
  std::vector<int> rblk(nr);
  for (int b = 0; b < g.d[0].nb; b++)
    for (int i = g.d[0].start[b]; i < g.d[0].start[b] + g.d[0].size[b]; i++) rblk[i] = b;
  // physics constants (rhs_mpi.f90:63-75)
  g.gamma = p.gamma; g.gamm1 = p.gamma - 1.0; g.cp = p.cp; g.cv = p.cp / p.gamma;
  g.invcv = 1.0 / g.cv;
  double invcp = 1.0 / p.cp;
  g.pconst = g.gamm1 * p.cp;
  g.invpconst = invcp / g.gamm1;
  g.invtconst = g.invcv / g.gamm1;
  g.omega0 = p.omega_0; g.t0 = p.t0; g.damping_time = p.damping_time; g.lumr1 = p.lumr1; g.lumr2 = p.lumr2;
  g.r1 = p.r1; g.r2 = p.r2; g.dth = dth; g.dphi = dphi; g.xi_cs = p.xi_cs;
  // entropy conduction is on under Laplacian .or. SLaplacian (rhs_mpi.f90:959,
  // :1221, :1286, :1456, :586, :618; diffusion.f90:614, :688)
  g.slaplacian = p.slaplacian || p.laplacian; g.sldiffusion = p.sldiffusion; g.set_stop = p.set_stop;
  g.top_stress_free = p.top_stress_free; g.bottom_stress_free = p.bottom_stress_free;
  g.top_constant_temp = p.top_constant_temp; g.bottom_constant_temp = p.bottom_constant_temp;
  g.theta_stress_free = p.theta_stress_free; g.theta_normal_field = p.theta_normal_field;
  g.theta_perf_conductor = p.theta_perf_conductor;
  g.top_radial_field = p.top_radial_field; g.bottom_radial_field = p.bottom_radial_field;
  g.top_perfect_cond = p.top_perfect_cond; g.bottom_perfect_cond = p.bottom_perfect_cond;
  // BC integers (Read_Input, mhdsph_mpi.f90:1317-1461)
  {
    int tn = !p.top_stress_free, bn = !p.bottom_stress_free;
    int lbcr_v = (tn && bn) ? 1 : (tn && !bn) ? 2 : (!tn && bn) ? 3 : 4;
    int tt = p.top_constant_temp, bt = p.bottom_constant_temp;
    int lbcr_s = (tt && bt) ? 1 : (tt && !bt) ? 2 : (!tt && bt) ? 3 : 4;
    int lbcr_u = p.top_inout ? 3 : 1, lbcr_rho = 4, lbcr_t = 4;  // mhdsph_mpi.f90:1355-1359
    int lbct_rho = 4, lbct_t = 0, lbct_w = 1, lbct_u = p.theta_stress_free ? 0 : 1, lbct_v = 4, lbct_s = 0;
    int lbcr_br = 0, lbcr_bt = 0, lbcr_bp = 0, lbcr_ar = 0, lbcr_at = 0, lbcr_ap = 0;
    int lbct_br = 0, lbct_bt = 0, lbct_bp = 0, lbct_ar = 0, lbct_at = 0, lbct_ap = 0;
    if (p.magnetic) {
      if (p.top_radial_field && p.bottom_radial_field) {
        lbcr_br = 4; lbcr_bt = 1; lbcr_bp = 1; lbcr_ar = 1; lbcr_at = 0; lbcr_ap = 0;
      }
      if (p.top_perfect_cond && p.bottom_perfect_cond) {
        lbcr_br = lbcr_bt = lbcr_bp = lbcr_ar = lbcr_at = lbcr_ap = 1;
      }
      if (p.theta_normal_field) { lbct_br = 1; lbct_bt = 4; lbct_bp = 1; lbct_ar = 0; lbct_at = 1; lbct_ap = 0; }
      if (p.theta_perf_conductor) { lbct_br = lbct_bt = lbct_bp = lbct_ar = lbct_at = lbct_ap = 1; }
    }
    int ir_[13] = {0, lbcr_rho, lbcr_v, lbcr_v, lbcr_u, lbcr_s, lbcr_t, lbcr_bt, lbcr_bp, lbcr_br, lbcr_at, lbcr_ap, lbcr_ar};
    int it_[13] = {0, lbct_rho, lbct_w, lbct_v, lbct_u, lbct_s, lbct_t, lbct_bt, lbct_bp, lbct_br, lbct_at, lbct_ap, lbct_ar};
    memcpy(g.ibcr, ir_, sizeof ir_);
    memcpy(g.ibct, it_, sizeof it_);
    g.lbcr_rho = lbcr_rho;
  }
  const double one_over_4pi = 1.0 / 3.1415926535897932384626433832795028841972 / 4.0;
  const double *ks = &P[CSS_PROF_KS * nr];
  g.s_flux_lo = g.s_flux_hi = 0.0;
  if (!p.bottom_constant_temp)
    g.s_flux_lo = g.slaplacian ? -p.lumr1 * one_over_4pi / (p.r1 * p.r1 * ks[0] * dxdr[0]) : 0.0 / dxdr[0];
  if (!p.top_constant_temp)
    g.s_flux_hi = g.slaplacian ? -p.lumr2 * one_over_4pi / (p.r2 * p.r2 * ks[nr - 1] * dxdr[nr - 1]) : 0.0 / dxdr[nr - 1];
  // the reports' dsdr1/dsdr2 follow SLaplacian alone (mhdsph_mpi.f90:576-584)
  c->rep_flux_lo = c->rep_flux_hi = 0.0;
  if (!p.bottom_constant_temp && p.slaplacian) c->rep_flux_lo = -p.lumr1 * one_over_4pi / (p.r1 * p.r1 * ks[0] * dxdr[0]);
  if (!p.top_constant_temp && p.slaplacian)
    c->rep_flux_hi = -p.lumr2 * one_over_4pi / (p.r2 * p.r2 * ks[nr - 1] * dxdr[nr - 1]);
  // SLD (diffusion.f90:76-114, :51-61)
  g.sld_coef = p.sld_coef; g.sld_pr = p.sld_pr; g.sld_prm = p.sld_prm;
  const double *rhor = &P[CSS_PROF_RHO * nr];
  double tv[8] = {1e-8 * rhor[nr - 1], 1e-8, 1e-8, 1e-8, 1e-8 * 1e5, 1e-8 * 1e8, 1e-8 * 1e8, 1e-8 * 1e8};
  memcpy(g.tinyvar, tv, sizeof tv);
  for (int k = 0; k < 8; k++) g.inv_tinyvar[k] = 1.0 / tv[k];  // correctly rounded, as a device division
  g.nsld = 0;
  if (p.mass_diffusion) g.varlist[g.nsld++] = 0;
  for (int i = 1; i <= 4; i++) g.varlist[g.nsld++] = i;
  if (p.magnetic && p.magnetic_diffusion) for (int i = 5; i <= 7; i++) g.varlist[g.nsld++] = i;
  g.dstype = p.dstype; g.mass_diffusion = p.mass_diffusion;
  g.do_viscous_heating = p.do_viscous_heating; g.do_ohmic_heating = p.magnetic && p.do_ohmic_heating;
  std::vector<double> dspeed(nr);
  for (int i = 0; i < nr; i++) {
    double ds = p.sld_speedh * pow(rhor[i] / rhor[nr - 1], p.sld_exp) + p.sld_speedr;
    ds = 0.5 * ds * (1.0 + tanh(p.sld_tanh_coef * (r_ind[i] - p.flux_cutoff) / (p.r2 - p.r1)));
    dspeed[i] = ds * ds;
  }
  // device copies
  int rc = setup_kernels();
  if (rc) { css_destroy(c); return rc; }
  if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    set_err("css_create: stream creation failed");
    css_destroy(c);
    return CSS_ERR_CUDA;
  }
  c->stream = c->own_stream;
  // radial profile block: r_ind r_inv dr_ind dxdr d2xdr2 rhor sr grav ks dlnks eps dspeed mur dlnmu
  std::vector<double> R((size_t)16 * nr);
  for (int i = 0; i < nr; i++) {
    R[0 * nr + i] = r_ind[i];
    R[1 * nr + i] = 1.0 / r_ind[i];
    R[2 * nr + i] = P[CSS_PROF_DR * nr + i];
    R[3 * nr + i] = dxdr[i];
    R[4 * nr + i] = d2xdr2[i];
    R[5 * nr + i] = rhor[i];
    R[6 * nr + i] = P[CSS_PROF_S * nr + i];
    R[7 * nr + i] = P[CSS_PROF_G * nr + i];
    R[8 * nr + i] = ks[i];
    R[9 * nr + i] = P[CSS_PROF_DLNKS * nr + i];
    R[10 * nr + i] = P[CSS_PROF_EPS * nr + i];
    R[11 * nr + i] = dspeed[i];
    R[12 * nr + i] = P[CSS_PROF_MUR * nr + i];
    R[13 * nr + i] = P[CSS_PROF_DLNMU * nr + i];
    R[14 * nr + i] = P[CSS_PROF_KR * nr + i];
    R[15 * nr + i] = P[CSS_PROF_DLNKR * nr + i];
  }
  if (p.laplacian) {
    // dtmaxd of Compute_Step_Size (rhs_mpi.f90:194-198; etar = ks there)
    const double *dr = &P[CSS_PROF_DR * nr], *mu = &P[CSS_PROF_MUR * nr];
    double drmin = dr[0], ksmax = ks[0], mumax = mu[0] / rhor[0];
    for (int i = 1; i < nr; i++) {
      drmin = std::min(drmin, dr[i]);
      ksmax = std::max(ksmax, ks[i]);
      mumax = std::max(mumax, mu[i] / rhor[i]);
    }
    double h = std::min(drmin, p.r1 * std::min(std::min(sines[0], sines[nth - 1]) * dphi, dth));
    c->dtd = h * h / std::max(std::max(ksmax, mumax), ksmax);
  }
  // SLD geometry tables (diffusion.f90:806-849, :1196-1247, :1316-1351),
  // the same expressions as the reference evaluates per rank
  std::vector<double> SG((size_t)5 * nth + 4 * nr);
  {
    const double *dr = &P[CSS_PROF_DR * nr];
    for (int it = 0; it < nth; it++) {
      double sphl, cphl, sphh, cphh;
      if (it == 0) { sphl = fabs(sin(theta[0] - 0.5 * dth)); cphl = cos(theta[0] - 0.5 * dth); }
      else { sphl = sin(0.5 * (theta[it] + theta[it - 1])); cphl = cos(0.5 * (theta[it] + theta[it - 1])); }
      if (it == nth - 1) { sphh = sin(theta[it] + 0.5 * dth); cphh = cos(theta[it] + 0.5 * dth); }
      else { sphh = sin(0.5 * (theta[it] + theta[it + 1])); cphh = cos(0.5 * (theta[it] + theta[it + 1])); }
      double rt, st, ct;
      if (it == 0) { rt = theta[0] - 0.5 * dth; st = cos(rt); }
      else { rt = 0.5 * (theta[it] + theta[it - 1]); st = cos(rt); }
      if (it == nth - 1) { ct = theta[it] + 0.5 * dth; rt = ct - rt; ct = cos(ct); }
      else { ct = 0.5 * (theta[it + 1] + theta[it]); rt = ct - rt; ct = cos(ct); }
      SG[it] = sphl; SG[nth + it] = cphl; SG[2 * nth + it] = sphh; SG[3 * nth + it] = cphh;
      SG[4 * nth + it] = rt / (st - ct);
    }
    double *R4 = &SG[5 * (size_t)nth];
    for (int ir = 0; ir < nr; ir++) {
      double rlo = (ir == 0) ? r_ind[0] - 0.5 * dr[0] : 0.5 * (r_ind[ir] + r_ind[ir - 1]);
      double rhi = (ir == nr - 1) ? r_ind[nr - 1] + 0.5 * dr[nr - 1] : 0.5 * (r_ind[ir + 1] + r_ind[ir]);
      R4[ir] = 3.0 / (rhi * rhi * rhi - rlo * rlo * rlo);
      R4[nr + ir] = 1.5 * (rhi * rhi - rlo * rlo) / (rhi * rhi * rhi - rlo * rlo * rlo);
      R4[2 * nr + ir] = rlo * rlo;
      R4[3 * nr + ir] = rhi * rhi;
    }
  }
  // sin, cos, theta, cot = cos/sin, csc = 1/sin (correctly rounded divisions,
  // the same values the kernels would get by dividing on the device)
  std::vector<double> TH((size_t)5 * nth);
  for (int i = 0; i < nth; i++) {
    TH[i] = sines[i]; TH[nth + i] = cosines[i]; TH[2 * nth + i] = theta[i];
    TH[3 * nth + i] = cosines[i] / sines[i]; TH[4 * nth + i] = 1.0 / sines[i];
  }
#define ALLOC(ptr, bytes)                                                                \
  do {                                                                                   \
    if (cudaMalloc(&(ptr), (bytes)) != cudaSuccess) {                                     \
      set_err("css_create: device allocation of %zu bytes failed", (size_t)(bytes));     \
      css_destroy(c);                                                                    \
      return CSS_ERR_NOMEM;                                                              \
    }                                                                                    \
  } while (0)
  ALLOC(c->tab, T.size() * 8);
  ALLOC(c->prof, R.size() * 8);
  ALLOC(c->theta_prof, TH.size() * 8);
  ALLOC(c->sld_geo, SG.size() * 8);
  ALLOC(c->resp, RESP.size() * 8);
  ALLOC(c->rblk, nr * sizeof(int));
  size_t sb = c->ncell * c->nv * sizeof(double);
  ALLOC(c->v0, sb); ALLOC(c->vA, sb); ALLOC(c->vB, sb); ALLOC(c->dv, sb); ALLOC(c->vs, sb);
  ALLOC(c->vcc, c->ncell * sizeof(double));
  ALLOC(c->tbuf, c->ncell * sizeof(double));
  if (p.magnetic) { ALLOC(c->bf, 3 * c->ncell * sizeof(double)); ALLOC(c->cda, 3 * c->ncell * sizeof(double)); }
  ALLOC(c->flag, sizeof(int));
  if (p.laplacian) {
    size_t nf = std::max((size_t)nth * nphi, (size_t)nphi * nr);
    ALLOC(c->lapbuf, 12 * c->ncell * sizeof(double));
    ALLOC(c->lapface, 6 * nf * sizeof(double));
  }
  if (p.do_radheat) {
    size_t nf = std::max((size_t)nth * nphi, (size_t)nphi * nr);
    ALLOC(c->radbuf, 10 * c->ncell * sizeof(double));
    ALLOC(c->radface, 6 * nf * sizeof(double));
  }
  if (open_r) {
    const size_t np = (size_t)nth * nphi;
    ALLOC(c->io, IO_COUNT * sizeof(double));
    ALLOC(c->io_part, std::max((size_t)8 * p.nnt * p.nnp, (size_t)2 * nr) * sizeof(double));
    ALLOC(c->rain, 2 * np * sizeof(double));
    ALLOC(c->ash_slices, 16 * np * sizeof(double));
    ALLOC(c->ashv, 4 * np * sizeof(double));
    cudaMemset(c->io, 0, IO_COUNT * sizeof(double));
    cudaMemset(c->rain, 0, 2 * np * sizeof(double));
    cudaMemset(c->ash_slices, 0, 16 * np * sizeof(double));
    cudaMemset(c->ashv, 0, 4 * np * sizeof(double));
    g.inout = c->io; g.dvel_rain = c->rain; g.dent_rain = c->rain + np; g.ashv = c->ashv;
  }
  g.top_inout = p.top_inout; g.bot_inout = p.bot_inout; g.bottom_specified = p.bottom_specified;
  g.rain = p.do_entropy_rain; g.delta_s = p.delta_s;
  cudaMemcpy(c->tab, T.data(), T.size() * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(c->prof, R.data(), R.size() * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(c->theta_prof, TH.data(), TH.size() * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(c->sld_geo, SG.data(), SG.size() * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(c->resp, RESP.data(), RESP.size() * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(c->rblk, rblk.data(), nr * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemset(c->flag, 0, sizeof(int));
  cudaMemset(c->vs, 0, sb);
  g.tab = c->tab; g.rblk = c->rblk; g.resp_r = c->resp; g.resp_t = c->resp + (size_t)2 * g.d[0].nb * ts;
  g.r_ind = c->prof; g.r_inv = c->prof + nr; g.dr_ind = c->prof + 2 * nr; g.dxdr = c->prof + 3 * nr;
  g.d2xdr2 = c->prof + 4 * nr; g.rhor = c->prof + 5 * nr; g.sr = c->prof + 6 * nr; g.grav = c->prof + 7 * nr;
  g.ks = c->prof + 8 * nr; g.dlnks = c->prof + 9 * nr; g.eps = c->prof + 10 * nr; g.dspeed = c->prof + 11 * nr;
  g.mur = c->prof + 12 * nr; g.dlnmu = c->prof + 13 * nr;
  g.kr = c->prof + 14 * nr; g.dlnkr = c->prof + 15 * nr;
  g.radheat = p.do_radheat;
  if (p.do_radheat) { g.rad_lnrho_r = c->radbuf; g.rad_dsdr = c->radbuf + c->ncell; }
  g.sines = c->theta_prof; g.cosines = c->theta_prof + nth; g.theta = c->theta_prof + 2 * nth;
  g.cot = c->theta_prof + 3 * nth; g.csc = c->theta_prof + 4 * nth;
  g.sld_th = c->sld_geo; g.sld_r = c->sld_geo + 5 * (size_t)nth;
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    set_err("css_create: %s", cudaGetErrorString(e));
    css_destroy(c);
    return CSS_ERR_CUDA;
  }
  {
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && nsm > 0)
      c->nsm = nsm;
  }
  int mag = p.magnetic;
  for (int d = 0; d < 3; d++) {
    int m0 = g.d[d].size[0], same = 1;
    for (int b = 1; b < g.d[d].nb; b++) same &= (g.d[d].size[b] == m0);
    c->mt[d] = (same && (m0 == 16 || m0 == 32)) ? m0 : 0;
  }
  auto pick = [](int mt, size_t (*f)(int, int, int), int mag, int m) {
    if (mt) return 16;
    for (int tl = 16; tl >= 1; tl /= 2)
      if (f(mag, m, tl) <= kSmemCap) return tl;
    return 1;
  };
  c->tl_theta = pick(c->mt[1], smem_theta_terms, mag, g.d[1].maxm);
  c->tl_phi = pick(c->mt[2], smem_phi_terms, mag, g.d[2].maxm);
  c->tl_r = pick(c->mt[0], smem_radial_terms, mag, g.d[0].maxm);
  // the two-pass stage (css_fused.cuh): 32-point blocks in every direction,
  // an FP64 RK4 run with closed radial faces and none of the passes that
  // sit between the sweeps (explicit viscosity, radiative diffusion, open
  // faces, prescribed bottom)
  c->fused_ok = c->mt[0] == 32 && c->mt[1] == 32 && c->mt[2] == 32 && p.precision == 0 &&
                (p.time_stepper == 4 || p.time_stepper == 0) && !p.laplacian && !p.do_radheat && !p.top_inout &&
                !p.bot_inout && !p.bottom_specified;
  if (c->fused_ok) ALLOC(c->rtw, (size_t)nr * nphi * 2 * 32 * sizeof(double));
  if (p.precision == 1) {  // backgrounds of the FP32 stage states, refreshed at every upload
    ALLOC(c->bg2, 2 * (size_t)nr * nth * sizeof(double));
    cudaMemset(c->bg2, 0, 2 * (size_t)nr * nth * sizeof(double));
    c->g.bg2 = c->bg2;
  }
  {  // cyclic phi derivative tables (css_dbydp_cyclic)
    const size_t per = 3 * (size_t)nphi + 1;
    std::vector<double> CY(2 * per);
    for (int order = 1; order <= 2; order++) cyclic_tables(nphi, order, &CY[(order - 1) * per]);
    ALLOC(c->cyc, CY.size() * sizeof(double));
    cudaMemcpy(c->cyc, CY.data(), CY.size() * sizeof(double), cudaMemcpyHostToDevice);
  }
  if (c->fused_ok && !plane_maps(c)) c->fused_ok = 0;
  c->fused = c->fused_ok;
  *out = c;
  return CSS_OK;
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
static int check_launch(css_ctx *c) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_err("kernel launch: %s", cudaGetErrorString(e));
    return CSS_ERR_CUDA;
  }
  c->launches++;
  return CSS_OK;
}

template <typename TS>
static int launch_curl(css_ctx *c, const TS *a, double *out, int apply_bc) {
  const CssGeo &g = c->g;
  int mt = g.d[1].maxm, mp = g.d[2].maxm, mr = g.d[0].maxm;
  int TL;
  int mi = -1;  // the state buffer whose A fields these are, if any
  if (std::is_same<TS, double>::value) {
    const double *ad = reinterpret_cast<const double *>(a);
    mi = ad == c->v0 + 5 * c->ncell ? 0 : (ad == c->vA + 5 * c->ncell ? 1 : (ad == c->vB + 5 * c->ncell ? 2 : -1));
    if (mi < 0 && c->vs_map && ad == c->vs + 5 * c->ncell) mi = 4;  // the SLD tendency
  }
  if (c->curl_tp == 2 && c->fused_ok && mi >= 0 && c->mt[1] == 32 && c->mt[2] == 32) {
    prof_begin(c, KI_CURL_THETA);
    // one plane buffer per CTA and three CTAs of 128 threads per SM: 1.51 ms
    // per curl on MHD 256x512x1024, against 2.13 ms for two buffers per CTA
    // and two CTAs of 256 threads (k_curl_pl<2, 256>)
    k_curl_pl<1, 128><<<3 * c->nsm, 128, CurlCfg<1, 128>::SMEM, c->stream>>>(g, out, c->pmaps[mi], c->flag);
    prof_end(c);
    if (int rc = check_launch(c)) return rc;
  } else if (c->mt[1] && c->mt[1] == c->mt[2] && c->curl_tp) {  // theta and phi in one pass
    const int M = c->mt[1];
    const size_t smem = 8 * (2 * (size_t)M * (M + 9) + 2 * (size_t)(M + 8) * (M + 1) + 2 * (size_t)M * (M + 1) +
                             2 * (size_t)M * (M + 1));
    dim3 gtp(g.d[1].nb * g.d[2].nb, g.nr);
    prof_begin(c, KI_CURL_THETA);
    if (M == 32) k_curl_tp<32, TS><<<gtp, 256, smem, c->stream>>>(g, a, out);
    else k_curl_tp<16, TS><<<gtp, 256, smem, c->stream>>>(g, a, out);
    prof_end(c);
    if (int rc = check_launch(c)) return rc;
  } else {
    TL = c->tl_theta;
    dim3 gt(g.d[1].nb * ((g.nphi + TL - 1) / TL), g.nr);
    prof_begin(c, KI_CURL_THETA);
    LAUNCH_MT(1, TL, k_curl_theta, (TS), gt, smem_theta(2, 2, mt, TL), g, a, out, TL);
    prof_end(c);
    if (int rc = check_launch(c)) return rc;
    TL = c->tl_phi;
    dim3 gp(g.d[2].nb * ((g.nth + TL - 1) / TL), g.nr);
    prof_begin(c, KI_CURL_PHI);
    LAUNCH_MT(2, TL, k_curl_phi, (TS), gp, smem_line(2, 2, 0, mp, TL), g, a, out, TL);
    prof_end(c);
    if (int rc = check_launch(c)) return rc;
  }
  if (c->curl_tp == 2 && c->fused_ok && mi >= 0 && c->mt[0] == 32 && c->mt[1] == 32) {  // radial part from TMA slabs
    prof_begin(c, KI_CURL_R);
    k_curl_rs<<<g.d[0].nb * g.d[1].nb * g.nphi, CR_NT, CR_SMEM, c->stream>>>(
        g, out, mi < 3 ? c->smaps[mi] : c->vs_slab, apply_bc, c->flag);
    prof_end(c);
    return check_launch(c);
  }
  TL = c->tl_r;
  dim3 gr(g.d[0].nb * ((g.nth + TL - 1) / TL), g.nphi);
  prof_begin(c, KI_CURL_R);
  LAUNCH_MT(0, TL, k_curl_r, (TS), gr, smem_line(2, 2, 0, mr, TL), g, a, out, TL, apply_bc);
  prof_end(c);
  return check_launch(c);
}

// RHS of one stage on `cur`; if stage > 0 also the stage update into `nx`
// the persistent phi kernel: as many CTAs as fit on the device at once
template <int MT, int TLC>
static void launch_phi_p(css_ctx *c, const double *cur) {
  const CssGeo &g = c->g;
  const int mag = g.magnetic, nh = mag ? 7 : 5, nd = mag ? 8 : 6, SR = TLC + 1;
  const size_t HS = (size_t)(MT + 8) * SR, OS = (size_t)MT * SR;
  const size_t smem = 8 * (2 * (size_t)nh * HS + (size_t)nd * OS + 2 * 3 * (MT + 2));
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_phi_terms_p<MT, TLC>, 128, smem);
  const long long ntile = (long long)g.d[2].nb * ((g.nth + TLC - 1) / TLC) * g.nr;
  const int grid = (int)std::min<long long>(ntile, (long long)std::max(per_sm, 1) * c->nsm);
  k_phi_terms_p<MT, TLC><<<grid, 128, smem, c->stream>>>(g, cur, c->bf, c->dv, c->tbuf);
}

// stage input of storage type TS, next stage state of storage type TO
// explicit viscosity (Laplacian): the viscous terms of the three sweeps and
// the cross terms, added into c->dv after the phi sweep; FP64 states only
static int launch_lap(css_ctx *c, const double *cur) {
  const CssGeo &g = c->g;
  const size_t n = c->ncell;
  const size_t nf = std::max((size_t)g.nth * g.nphi, (size_t)g.nphi * g.nr);
  double *S = c->lapbuf, *L = c->lapbuf + 6 * n, *F = c->lapface;
  const double *w = cur + n, *v = cur + 2 * n, *u = cur + 3 * n;
  const int nbp = (int)std::min<size_t>((n + 255) / 256, (size_t)c->nsm * 8);
  const int nbf = (int)std::min<size_t>((nf + 255) / 256, (size_t)c->nsm * 8);
  cudaStream_t st = c->stream;
#define LAP_D(dir, ord, x, out, lo, hi, bdry) \
  if (int rc = css_deriv_dev(c, dir, ord, x, out, lo, hi, bdry, nullptr)) return rc
  // theta sweep: d/dth and d2/dth2 of w, v (wall datum cot v), u
  k_lap_bc_theta<<<nbf, 256, 0, st>>>(g, cur, F, F + nf);
  if (int rc = check_launch(c)) return rc;
  LAP_D(1, 1, w, S, nullptr, nullptr, g.ibct[2]);
  LAP_D(1, 1, v, S + n, F, F + nf, g.ibct[3]);
  LAP_D(1, 1, u, S + 2 * n, nullptr, nullptr, g.ibct[4]);
  LAP_D(1, 2, w, S + 3 * n, nullptr, nullptr, g.ibct[2]);
  LAP_D(1, 2, v, S + 4 * n, F, F + nf, g.ibct[3]);
  LAP_D(1, 2, u, S + 5 * n, nullptr, nullptr, g.ibct[4]);
  k_lap_theta<<<nbp, 256, 0, st>>>(g, cur, S, L, c->dv);
  if (int rc = check_launch(c)) return rc;
  // phi sweep: v, w, u
  LAP_D(2, 1, v, S, nullptr, nullptr, 0);
  LAP_D(2, 1, w, S + n, nullptr, nullptr, 0);
  LAP_D(2, 1, u, S + 2 * n, nullptr, nullptr, 0);
  LAP_D(2, 2, v, S + 3 * n, nullptr, nullptr, 0);
  LAP_D(2, 2, w, S + 4 * n, nullptr, nullptr, 0);
  LAP_D(2, 2, u, S + 5 * n, nullptr, nullptr, 0);
  k_lap_phi<<<nbp, 256, 0, st>>>(g, cur, c->tbuf, S, L, c->dv);
  if (int rc = check_launch(c)) return rc;
  // radial sweep: w, v with the stress-free data, u
  k_lap_bc_r<<<nbf, 256, 0, st>>>(g, cur, F, F + nf, F + 2 * nf, F + 3 * nf);
  if (int rc = check_launch(c)) return rc;
  LAP_D(0, 1, w, S, F, F + nf, g.ibcr[2]);
  LAP_D(0, 1, v, S + n, F + 2 * nf, F + 3 * nf, g.ibcr[3]);
  LAP_D(0, 1, u, S + 2 * n, nullptr, nullptr, g.ibcr[4]);
  LAP_D(0, 2, w, S + 3 * n, F, F + nf, g.ibcr[2]);
  LAP_D(0, 2, v, S + 4 * n, F + 2 * nf, F + 3 * nf, g.ibcr[3]);
  LAP_D(0, 2, u, S + 5 * n, nullptr, nullptr, g.ibcr[4]);
  k_lap_r<<<nbp, 256, 0, st>>>(g, cur, c->tbuf, S, L, c->dv);
  if (int rc = check_launch(c)) return rc;
  // cross terms: r derivatives of r L0 (var 2), r L5 (var 4), r L2 (var 4),
  // r L3 (var 3); theta derivatives of sin L3 (var 3), sin L4 (var 2)
  k_lap_bc_cross<<<nbf, 256, 0, st>>>(g, L, F, F + nf, F + 2 * nf, F + 3 * nf);
  if (int rc = check_launch(c)) return rc;
  LAP_D(0, 1, S, L, F, nullptr, g.ibcr[2]);
  LAP_D(0, 1, S + n, L + n, nullptr, nullptr, g.ibcr[4]);
  LAP_D(0, 1, S + 2 * n, L + 2 * n, nullptr, nullptr, g.ibcr[4]);
  LAP_D(0, 1, S + 3 * n, L + 3 * n, nullptr, F + nf, g.ibcr[3]);
  LAP_D(1, 1, S + 4 * n, L + 4 * n, F + 2 * nf, F + 3 * nf, g.ibct[3]);
  LAP_D(1, 1, S + 5 * n, L + 5 * n, nullptr, nullptr, g.ibct[2]);
  k_lap_cross<<<nbp, 256, 0, st>>>(g, cur, L, c->dv);
  if (int rc = check_launch(c)) return rc;
  if (g.magnetic) {
    // resistive induction: J = curl B of c->bf (B of this stage's A)
    const int bdry_t = g.theta_normal_field ? 1 : 0;
    const double *bf = c->bf;
    k_mhd_curl_in<<<nbp, 256, 0, st>>>(g, bf, S);
    if (int rc = check_launch(c)) return rc;
    LAP_D(1, 1, S, L, nullptr, nullptr, bdry_t);
    LAP_D(1, 1, bf + 2 * n, L + n, nullptr, nullptr, bdry_t);
    LAP_D(2, 1, bf + 2 * n, L + 2 * n, nullptr, nullptr, 0);
    LAP_D(2, 1, bf, L + 3 * n, nullptr, nullptr, 0);
    LAP_D(0, 1, S + n, L + 4 * n, nullptr, nullptr, g.ibcr[7]);
    LAP_D(0, 1, S + 2 * n, L + 5 * n, nullptr, nullptr, g.ibcr[8]);
    k_mhd_resist<<<nbp, 256, 0, st>>>(g, cur, c->tbuf, L, L + 3 * n, c->dv);
    if (int rc = check_launch(c)) return rc;
  }
#undef LAP_D
  return CSS_OK;
}

// radiative diffusion: the heating of all three directions added into ds,
// after the radial kernel and before the density-theta / update kernel
static int launch_rad(css_ctx *c, const double *cur) {
  const CssGeo &g = c->g;
  const size_t n = c->ncell;
  const size_t nf = std::max((size_t)g.nth * g.nphi, (size_t)g.nphi * g.nr);
  double *S = c->radbuf + 2 * n, *F = c->radface;
  const double *rho = cur, *T = c->tbuf;
  const int nbp = (int)std::min<size_t>((n + 255) / 256, (size_t)c->nsm * 8);
  const int nbf = (int)std::min<size_t>((nf + 255) / 256, (size_t)c->nsm * 8);
  cudaStream_t st = c->stream;
  k_rad_bc<<<nbf, 256, 0, st>>>(g, cur, c->dv, T, F, F + nf, F + 2 * nf, F + 3 * nf, F + 4 * nf, F + 5 * nf);
  if (int rc = check_launch(c)) return rc;
#define RAD_D(dir, ord, x, out, lo, hi, bdry) \
  if (int rc = css_deriv_dev(c, dir, ord, x, out, lo, hi, bdry, nullptr)) return rc
  RAD_D(1, 1, rho, S, F, F + nf, g.ibct[1]);
  RAD_D(1, 1, T, S + n, F + 2 * nf, F + 3 * nf, g.ibct[6]);
  RAD_D(1, 2, T, S + 2 * n, F + 2 * nf, F + 3 * nf, g.ibct[6]);
  RAD_D(2, 1, rho, S + 3 * n, nullptr, nullptr, 0);
  RAD_D(2, 1, T, S + 4 * n, nullptr, nullptr, 0);
  RAD_D(2, 2, T, S + 5 * n, nullptr, nullptr, 0);
  RAD_D(0, 1, T, S + 6 * n, F + 4 * nf, F + 5 * nf, g.ibcr[6]);
  RAD_D(0, 2, T, S + 7 * n, F + 4 * nf, F + 5 * nf, g.ibcr[6]);
#undef RAD_D
  k_rad_point<<<nbp, 256, 0, st>>>(g, cur, T, S, c->dv);
  return check_launch(c);
}

static int launch_sld(css_ctx *c, const double *v, const double *av, double *dout, const double *tb);

// Open radial boundaries: the face sums and scalars of this RHS, after the
// mass total's refresh at the first call of every ufreq-th step
// (rhs_mpi.f90:326-353)
static int launch_inout(css_ctx *c, const double *cur) {
  const CssGeo &g = c->g;
  if (c->rhs_call == 1) {
    if (c->p.ufreq > 0 && c->istep % c->p.ufreq == 0) {
      k_plane_mass<<<g.nr, IO_NT, 0, c->stream>>>(g, cur, c->io_part);
      k_mass_finish<<<1, 32, 0, c->stream>>>(g, c->io_part, c->io, IO_MTOT, -1);
      if (int rc = check_launch(c)) return rc;
    }
    c->rhs_call = 2;  // the later stages are calls 2..4
  }
  k_inout_sums<<<g.d[1].nb * g.d[2].nb, IO_NT, 0, c->stream>>>(g, cur, c->io_part);
  k_inout_scalars<<<1, 32, 0, c->stream>>>(g, c->io_part, c->io, c->deltat, c->sim_time);
  return check_launch(c);
}

// with_sld: the step's slope-limited diffusion tendency of `cur` into c->vs,
// launched after the radial kernel (the theta kernel has left T(cur) in
// tbuf) and before the update that reads vs
template <typename TS, typename TO>
static int launch_rhs(css_ctx *c, const TS *cur, TO *nx, int stage, double dtcur, double ca = 0.0, double cb = 0.0,
                      double dsld = 0.0, bool with_sld = false) {
  const CssGeo &g = c->g;
  const int mag = g.magnetic;
  if (mag) {
    if (int rc = launch_curl(c, cur + 5 * c->ncell, c->bf, 1)) return rc;
  }
  int TL = c->tl_theta;
  dim3 gt(g.d[1].nb * ((g.nphi + TL - 1) / TL), g.nr);
  prof_begin(c, KI_THETA);
  if (mag)
    LAUNCH_MT(1, TL, k_theta_terms, (TS, 1), gt, smem_theta_terms(mag, g.d[1].maxm, TL), g, cur, c->bf, c->dv, c->tbuf,
              TL);
  else
    LAUNCH_MT(1, TL, k_theta_terms, (TS, 0), gt, smem_theta_terms(mag, g.d[1].maxm, TL), g, cur, c->bf, c->dv, c->tbuf,
              TL);
  prof_end(c);
  if (int rc = check_launch(c)) return rc;
  TL = c->tl_phi;
  dim3 gp(g.d[2].nb * ((g.nth + TL - 1) / TL), g.nr);
  prof_begin(c, KI_PHI);
  bool pers = false;
  if constexpr (sizeof(TS) == 8) {
    if (c->phi_pers) {
      pers = true;
      switch (c->mt[2] * 100 + TL) {
        case 1616: launch_phi_p<16, 16>(c, cur); break;
        case 3216: launch_phi_p<32, 16>(c, cur); break;
        case 1608: launch_phi_p<16, 8>(c, cur); break;
        case 3208: launch_phi_p<32, 8>(c, cur); break;
        default: pers = false;
      }
    }
  }
  if (!pers)
  {
    if (mag)
      LAUNCH_MT(2, TL, k_phi_terms, (TS, 1), gp, smem_phi_terms(mag, g.d[2].maxm, TL), g, cur, c->bf, c->dv, c->tbuf,
                TL);
    else
      LAUNCH_MT(2, TL, k_phi_terms, (TS, 0), gp, smem_phi_terms(mag, g.d[2].maxm, TL), g, cur, c->bf, c->dv, c->tbuf,
                TL);
  }
  prof_end(c);
  if (int rc = check_launch(c)) return rc;
  if constexpr (sizeof(TS) == 8) {
    if (c->p.laplacian)
      if (int rc = launch_lap(c, (const double *)cur)) return rc;
    if (c->io)
      if (int rc = launch_inout(c, (const double *)cur)) return rc;
  }
  TL = c->tl_r;
  const dim3 gr(g.d[0].nb * ((g.nth + TL - 1) / TL), g.nphi);
  prof_begin(c, KI_RADIAL);
  if (mag)
    LAUNCH_MT(0, TL, k_radial_terms, (TS, 2), gr, smem_radial_terms(mag, g.d[0].maxm, TL), g, cur, c->bf, c->dv, c->tbuf,
              TL);
  else if (c->io)
    LAUNCH_MT(0, TL, k_radial_terms, (TS, 1), gr, smem_radial_terms(mag, g.d[0].maxm, TL), g, cur, c->bf, c->dv, c->tbuf,
              TL);
  else
    LAUNCH_MT(0, TL, k_radial_terms, (TS, 0), gr, smem_radial_terms(mag, g.d[0].maxm, TL), g, cur, c->bf, c->dv, c->tbuf,
              TL);
  prof_end(c);
  if (int rc = check_launch(c)) return rc;
  if constexpr (sizeof(TS) == 8) {
    if (c->p.do_radheat)
      if (int rc = launch_rad(c, (const double *)cur)) return rc;
    if (with_sld)
      if (int rc = launch_sld(c, (const double *)cur, (const double *)cur + 5 * c->ncell, c->vs, c->tbuf)) return rc;
  }
  TL = c->tl_theta;
  dim3 gu(g.d[1].nb * ((g.nphi + TL - 1) / TL), g.nr);
  prof_begin(c, KI_RHOT_UPDATE);
  bool staged = false;  // RK4 stages: the stage is a template argument
  if constexpr (std::is_same<TS, double>::value && std::is_same<TO, double>::value) {
    staged = stage >= 1 && stage <= 4;
    switch (stage) {
      case 1: LAUNCH_MT(1, TL, k_rhot_update, (TS, TO, 1), gu, smem_rhot(g.d[1].maxm, TL), g, cur, c->dv, c->v0, c->vs, nx, c->tbuf, stage, dtcur,
            ca, cb, dsld, TL, c->flag); break;
      case 2: LAUNCH_MT(1, TL, k_rhot_update, (TS, TO, 2), gu, smem_rhot(g.d[1].maxm, TL), g, cur, c->dv, c->v0, c->vs, nx, c->tbuf, stage, dtcur,
            ca, cb, dsld, TL, c->flag); break;
      case 3: LAUNCH_MT(1, TL, k_rhot_update, (TS, TO, 3), gu, smem_rhot(g.d[1].maxm, TL), g, cur, c->dv, c->v0, c->vs, nx, c->tbuf, stage, dtcur,
            ca, cb, dsld, TL, c->flag); break;
      case 4: LAUNCH_MT(1, TL, k_rhot_update, (TS, TO, 4), gu, smem_rhot(g.d[1].maxm, TL), g, cur, c->dv, c->v0, c->vs, nx, c->tbuf, stage, dtcur,
            ca, cb, dsld, TL, c->flag); break;
      default: break;
    }
  } else if constexpr (std::is_same<TS, double>::value) {  // mixed, stage 1: FP64 vars0 -> FP32 U1
    if (stage == 1) { staged = true; LAUNCH_MT(1, TL, k_rhot_update, (TS, TO, 1), gu, smem_rhot(g.d[1].maxm, TL), g, cur, c->dv, c->v0, c->vs, nx, c->tbuf, stage, dtcur,
            ca, cb, dsld, TL, c->flag);; }
  } else if constexpr (std::is_same<TO, float>::value) {  // mixed, stages 2-3: FP32 -> FP32
    if (stage == 2) { staged = true; LAUNCH_MT(1, TL, k_rhot_update, (TS, TO, 2), gu, smem_rhot(g.d[1].maxm, TL), g, cur, c->dv, c->v0, c->vs, nx, c->tbuf, stage, dtcur,
            ca, cb, dsld, TL, c->flag);; }
    else if (stage == 3) { staged = true; LAUNCH_MT(1, TL, k_rhot_update, (TS, TO, 3), gu, smem_rhot(g.d[1].maxm, TL), g, cur, c->dv, c->v0, c->vs, nx, c->tbuf, stage, dtcur,
            ca, cb, dsld, TL, c->flag);; }
  } else {  // mixed, stage 4: FP32 U3 -> FP64 vars0
    if (stage == 4) { staged = true; LAUNCH_MT(1, TL, k_rhot_update, (TS, TO, 4), gu, smem_rhot(g.d[1].maxm, TL), g, cur, c->dv, c->v0, c->vs, nx, c->tbuf, stage, dtcur,
            ca, cb, dsld, TL, c->flag);; }
  }
  if (!staged)
  LAUNCH_MT(1, TL, k_rhot_update, (TS, TO), gu, smem_rhot(g.d[1].maxm, TL), g, cur, c->dv, c->v0, c->vs, nx, c->tbuf, stage, dtcur,
            ca, cb, dsld, TL, c->flag);
  prof_end(c);
  return check_launch(c);
}

// slope-limited diffusion tendency of `v` (A in av for MHD; B must be in
// c->bf) into dout
static int launch_sld(css_ctx *c, const double *v, const double *av, double *dout, const double *tb) {
  const CssGeo &g = c->g;
  int nb = 148 * 16;
  prof_begin(c, KI_SLD_VCC);
  k_sld_vcc<<<nb, 256, 0, c->stream>>>(g, v, c->bf, c->vcc);
  prof_end(c);
  if (int rc = check_launch(c)) return rc;
  prof_begin(c, KI_SLD);
  dim3 gs((g.nth + SLD_TT - 1) / SLD_TT, (g.nphi + SLD_TP - 1) / SLD_TP, (g.nr + SLD_RC - 1) / SLD_RC);
  // the diffused fields are contiguous from varlist[0]; MHD runs them in two
  // launches (the hydro fields, then A) so each carries a register window
  // of at most five fields
  // the first diffused field is a template argument: 1 without mass
  // diffusion (4 or 7 fields), 0 with it (5 or 8)
  if (g.varlist[0] != ((g.nsld == 4 || g.nsld == 7) ? 1 : 0)) {
    set_err("launch_sld: unexpected diffused-field list");
    return CSS_ERR_ARG;
  }
  const unsigned all = (1u << g.nv) - 1u;
  const int th = SLD_TT * SLD_TP;
  switch (g.nsld) {
    case 4: k_sld<4, 1><<<gs, th, sizeof(SldSmem<4>), c->stream>>>(g, v, av, c->vcc, dout, all, tb); break;
    case 5: k_sld<5, 0><<<gs, th, sizeof(SldSmem<5>), c->stream>>>(g, v, av, c->vcc, dout, all, tb); break;
    case 7:  // fields 1..7: rho is not diffused (its tendency is zero)
      k_sld<4, 1><<<gs, th, sizeof(SldSmem<4>), c->stream>>>(g, v, av, c->vcc, dout, 0x1Fu, tb);
      if (int rc = check_launch(c)) return rc;
      k_sld<3, 5><<<gs, th, sizeof(SldSmem<3>), c->stream>>>(g, v, av, c->vcc, dout, 0xE0u, tb);
      break;
    default:  // fields 0..7
      k_sld<5, 0><<<gs, th, sizeof(SldSmem<5>), c->stream>>>(g, v, av, c->vcc, dout, 0x1Fu, tb);
      if (int rc = check_launch(c)) return rc;
      k_sld<3, 5><<<gs, th, sizeof(SldSmem<3>), c->stream>>>(g, v, av, c->vcc, dout, 0xE0u, tb);
      break;
  }
  prof_end(c);
  if (int rc = check_launch(c)) return rc;
  if (g.do_ohmic_heating) {
    if (int rc = launch_curl(c, (const double *)(dout + 5 * c->ncell), c->cda, 0)) return rc;
    prof_begin(c, KI_SLD_OHMIC);
    k_sld_ohmic<<<nb, 256, 0, c->stream>>>(g, v, c->bf, c->cda, dout);
    prof_end(c);
    if (int rc = check_launch(c)) return rc;
  }
  return CSS_OK;
}

// One RK4 stage in two passes (css_fused.cuh): [curl] -> k_thph -> [SLD
// of the step's start in stage 1] -> k_rstage<stage>
static int launch_stage_fused(css_ctx *c, const double *cur, double *nx, int stage, double dtcur, bool with_sld) {
  const CssGeo &g = c->g;
  const int mag = g.magnetic;
  if (mag)
    if (int rc = launch_curl(c, cur + 5 * c->ncell, c->bf, 1)) return rc;
  // persistent kernels: one CTA per SM
  const dim3 ga(c->nsm);
  prof_begin(c, KI_THPH);
  const int mi = cur == c->v0 ? 0 : (cur == c->vA ? 1 : (cur == c->vB ? 2 : -1));
  if (mi < 0) { set_err("launch_stage_fused: stage input is not a state buffer"); return CSS_ERR_ARG; }
  const PlaneMaps &mc = c->pmaps[mi], &mb = c->pmaps[3];
  if (mag) k_thph<1><<<ga, FNT, ThphCfg<1>::SMEM, c->stream>>>(g, cur, c->bf, c->dv, c->tbuf, c->rtw, mc, mb, c->flag);
  else k_thph<0><<<ga, FNT, ThphCfg<0>::SMEM, c->stream>>>(g, cur, c->bf, c->dv, c->tbuf, c->rtw, mc, mb, c->flag);
  prof_end(c);
  if (int rc = check_launch(c)) return rc;
  if (with_sld)
    if (int rc = launch_sld(c, cur, cur + 5 * c->ncell, c->vs, c->tbuf)) return rc;
  // hydro: one tile per CTA; MHD: persistent, one CTA per SM
  const int nrtile = g.d[0].nb * g.d[1].nb * g.nphi;
  const dim3 gb(mag ? std::min(c->nsm, nrtile) : nrtile);
  prof_begin(c, KI_RSTAGE);
#define CSS_RSTAGE(M, S)                                                                                      \
  k_rstage<M, S><<<gb, RstageCfg<M>::NT, RstageCfg<M>::SMEM, c->stream>>>(g, cur, c->bf, c->dv, c->v0, c->vs, nx, c->tbuf, \
                                                              c->rtw, dtcur, c->flag, c->smaps[mi], c->smaps[3], \
                                                              c->smaps[4])
  switch (stage + (mag ? 10 : 0)) {
    case 1: CSS_RSTAGE(0, 1); break;
    case 2: CSS_RSTAGE(0, 2); break;
    case 3: CSS_RSTAGE(0, 3); break;
    case 4: CSS_RSTAGE(0, 4); break;
    case 11: CSS_RSTAGE(1, 1); break;
    case 12: CSS_RSTAGE(1, 2); break;
    case 13: CSS_RSTAGE(1, 3); break;
    case 14: CSS_RSTAGE(1, 4); break;
    default: set_err("launch_stage_fused: stage %d", stage); return CSS_ERR_ARG;
  }
#undef CSS_RSTAGE
  prof_end(c);
  return check_launch(c);
}

static int step_stages(css_ctx *c, double dt);

// the prescribed bottom fields at the clock's time (Cubic_Time_Interp)
static int ash_refresh(css_ctx *c) {
  if (!c->p.bottom_specified || !(c->ash_times[2] > c->ash_times[1])) return CSS_OK;
  const double mu = (c->sim_time - c->ash_times[1]) / (c->ash_times[2] - c->ash_times[1]);
  const size_t np = (size_t)c->p.nth * c->p.nphi;
  k_ash_interp<<<148, 256, 0, c->stream>>>(c->ash_slices, np, mu, c->ashv);
  return check_launch(c);
}

// One step with the run's clock (Program CSS2, mhdsph_mpi.f90:28-43): the
// step index advances before it and the time after it; a prescribed bottom
// interpolates its fields at the start time (Read_ASH_Inflow, ash_inflow.f90:
// 124-219) and updates the enthalpy-flux factor every ufreq steps at the end
// (step_rk4.f90:477-482)
static int step_once(css_ctx *c, double dt) {
  c->istep++;
  c->deltat = dt;
  if (c->p.bottom_specified) {
    if (!(c->sim_time < c->ash_times[2])) {
      set_err("css_step_rk4: sim_time %.17g is past the third ASH slice time %.17g; shift in the next slice "
              "first (css_set_ash_slices)", c->sim_time, c->ash_times[2]);
      c->istep--;
      return CSS_ERR_ARG;
    }
    if (int rc = ash_refresh(c)) return rc;
  }
  c->rhs_call = 1;
  int rc = step_stages(c, dt);
  c->rhs_call = 0;
  if (rc) return rc;
  if (c->p.bottom_specified && c->p.ufreq > 0 && c->istep % c->p.ufreq == 0) {
    k_ash_flux<<<1, IO_NT, 0, c->stream>>>(c->g, c->v0, c->tbuf, c->io, c->sim_time,
                                           4.0 * 3.1415926535897932384626433832795028841972);
    if (int rc2 = check_launch(c)) return rc2;
  }
  c->sim_time = c->sim_time + dt;
  return CSS_OK;
}

static int step_stages(css_ctx *c, double dt) {
  // the SLD tendency of vars0 is launched inside the first stage (with_sld)
  const bool sld = c->p.sldiffusion != 0;
  const int ts = c->p.time_stepper;
  if (ts == 2 || ts == 3) {
    // Step_RK2_TVD / Step_RK3_TVD (step_rk4.f90:31-335): vs holds the SLD
    // tendency of the step's start, added once in the last stage
    const double dsld = c->p.sldiffusion ? dt : 0.0;
    float *fA = reinterpret_cast<float *>(c->vA), *fB = reinterpret_cast<float *>(c->vB);
    const bool mixed = c->p.precision == 1;
    int rc = mixed ? launch_rhs(c, (const double *)c->v0, fA, 5, dt, 1.0, 0.0, 0.0, sld)
                   : launch_rhs(c, (const double *)c->v0, c->vA, 5, dt, 1.0, 0.0, 0.0, sld);
    if (rc) return rc;
    if (ts == 2)
      return mixed ? launch_rhs(c, (const float *)fA, c->v0, 6, 0.5 * dt, 0.5, 0.5, dsld)
                   : launch_rhs(c, (const double *)c->vA, c->v0, 6, 0.5 * dt, 0.5, 0.5, dsld);
    rc = mixed ? launch_rhs(c, (const float *)fA, fB, 5, dt / 4.0, 0.75, 0.25)
               : launch_rhs(c, (const double *)c->vA, c->vB, 5, dt / 4.0, 0.75, 0.25);
    if (rc) return rc;
    const double onethird = 1.0 / 3.0, twothirds = 2.0 / 3.0;
    return mixed ? launch_rhs(c, (const float *)fB, c->v0, 6, 2.0 * dt / 3.0, onethird, twothirds, dsld)
                 : launch_rhs(c, (const double *)c->vB, c->v0, 6, 2.0 * dt / 3.0, onethird, twothirds, dsld);
  }
  if (c->p.precision == 1) {
    // mixed: the stage states U1..U3 are FP32 (rho, s as perturbations about
    // the background); vars0, the accumulator and the tendency stay FP64
    float *fA = reinterpret_cast<float *>(c->vA), *fB = reinterpret_cast<float *>(c->vB);
    if (int rc = launch_rhs(c, (const double *)c->v0, fA, 1, dt / 2.0, 0.0, 0.0, 0.0, sld)) return rc;
    if (int rc = launch_rhs(c, (const float *)fA, fB, 2, dt / 2.0)) return rc;
    if (int rc = launch_rhs(c, (const float *)fB, fA, 3, dt)) return rc;
    if (int rc = launch_rhs(c, (const float *)fA, c->v0, 4, dt)) return rc;
    return CSS_OK;
  }
  if (c->fused) {
    if (int rc = launch_stage_fused(c, c->v0, c->vA, 1, dt / 2.0, sld)) return rc;
    if (int rc = launch_stage_fused(c, c->vA, c->vB, 2, dt / 2.0, false)) return rc;
    if (int rc = launch_stage_fused(c, c->vB, c->vA, 3, dt, false)) return rc;
    return launch_stage_fused(c, c->vA, c->v0, 4, dt, false);
  }
  if (int rc = launch_rhs(c, (const double *)c->v0, c->vA, 1, dt / 2.0, 0.0, 0.0, 0.0, sld)) return rc;
  if (int rc = launch_rhs(c, (const double *)c->vA, c->vB, 2, dt / 2.0)) return rc;
  if (int rc = launch_rhs(c, (const double *)c->vB, c->vA, 3, dt)) return rc;
  if (int rc = launch_rhs(c, (const double *)c->vA, c->v0, 4, dt)) return rc;
  return CSS_OK;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
// phi means of rho and s at every (r, theta): the backgrounds about which
// the mixed path stores its FP32 stage states (one thread per (r, theta),
// phi summed in order)
__global__ void k_phi_mean(CssGeo g, const double *__restrict__ v, double *__restrict__ bg2) {
  const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x, nrt = (size_t)g.nr * g.nth;
  if (k >= nrt) return;
  const int t = (int)(k % g.nth), r = (int)(k / g.nth);
  const size_t n = (size_t)g.ncell;
  double a = 0.0, b = 0.0;
  for (int p = 0; p < g.nphi; p++) {
    const size_t id = css_idx(g, t, p, r);
    a += __ldg(v + id);
    b += __ldg(v + 4 * n + id);
  }
  bg2[k] = a / g.nphi;
  bg2[nrt + k] = b / g.nphi;
}

extern "C" int css_upload_state(css_ctx *c, const double *vars) {
  if (!c || !vars) { set_err("css_upload_state: NULL"); return CSS_ERR_ARG; }
  CUDA_TRY(cudaMemcpyAsync(c->v0, vars, c->ncell * c->nv * 8, cudaMemcpyHostToDevice, c->stream));
  if (c->bg2) {
    const size_t nrt = (size_t)c->p.nr * c->p.nth;
    k_phi_mean<<<(unsigned)((nrt + 127) / 128), 128, 0, c->stream>>>(c->g, c->v0, c->bg2);
    if (int rc = check_launch(c)) return rc;
  }
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CSS_OK;
}

extern "C" int css_download_state(css_ctx *c, double *vars) {
  if (!c || !vars) { set_err("css_download_state: NULL"); return CSS_ERR_ARG; }
  CUDA_TRY(cudaMemcpyAsync(vars, c->v0, c->ncell * c->nv * 8, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CSS_OK;
}

extern "C" int css_download_plane(css_ctx *c, int iv, int ir, double *plane) {
  if (!c || !plane || iv < 0 || iv >= c->nv || ir < 0 || ir >= c->p.nr) {
    set_err("css_download_plane: bad argument");
    return CSS_ERR_ARG;
  }
  const size_t np = (size_t)c->p.nth * c->p.nphi;
  CUDA_TRY(cudaMemcpyAsync(plane, c->v0 + (size_t)iv * c->ncell + (size_t)ir * np, np * 8, cudaMemcpyDeviceToHost,
                           c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CSS_OK;
}

extern "C" int css_step_rk4(css_ctx *c, double dt, int nsteps) {
  if (!c || nsteps < 0 || !(dt > 0.0)) { set_err("css_step_rk4: bad argument"); return CSS_ERR_ARG; }
  CUDA_TRY(cudaMemsetAsync(c->flag, 0, sizeof(int), c->stream));
  for (int s = 0; s < nsteps; s++)
    if (int rc = step_once(c, dt)) return rc;
  int h = 0;
  CUDA_TRY(cudaMemcpyAsync(&h, c->flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (h & kFlagTimeout) {
    set_err("css_step_rk4: a tile's staged copies did not arrive within the kernel's bounded wait");
    return CSS_ERR_CUDA;
  }
  if (h) { set_err("css_step_rk4: non-finite value in the state"); return CSS_ERR_NAN; }
  return CSS_OK;
}

extern "C" int css_step_rk4_host(css_ctx *c, double *vars0, double dt, int nsteps) {
  if (int rc = css_upload_state(c, vars0)) return rc;
  int rc = css_step_rk4(c, dt, nsteps);
  if (rc && rc != CSS_ERR_NAN) return rc;
  if (int r2 = css_download_state(c, vars0)) return r2;
  return rc;
}

extern "C" int css_rhs(css_ctx *c, double *vars1, double *dvars1, int call_num) {
  if (!c || !vars1 || !dvars1) { set_err("css_rhs: NULL"); return CSS_ERR_ARG; }
  if (c->io && !(c->deltat > 0.0)) {
    set_err("css_rhs: an open radial boundary's mean-flow terms divide by the step size: set it with "
            "css_set_clock first");
    return CSS_ERR_ARG;
  }
  size_t sb = c->ncell * c->nv * 8;
  CUDA_TRY(cudaMemcpyAsync(c->vA, vars1, sb, cudaMemcpyHostToDevice, c->stream));
  c->rhs_call = call_num;
  int rc = launch_rhs(c, (const double *)c->vA, (double *)nullptr, 0, 0.0);
  c->rhs_call = 0;
  if (rc) return rc;
  CUDA_TRY(cudaMemcpyAsync(dvars1, c->dv, sb, cudaMemcpyDeviceToHost, c->stream));
  if (c->g.magnetic && call_num == 1)
    CUDA_TRY(cudaMemcpyAsync(vars1 + 5 * c->ncell, c->bf, 3 * c->ncell * 8, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CSS_OK;
}

extern "C" int css_bound(css_ctx *c, double *vars1) {
  if (!c || !vars1) { set_err("css_bound: NULL"); return CSS_ERR_ARG; }
  const size_t sb = c->ncell * c->nv * 8;
  CUDA_TRY(cudaMemcpyAsync(c->vA, vars1, sb, cudaMemcpyHostToDevice, c->stream));
  k_bound<<<c->nsm * 4, 256, 0, c->stream>>>(c->g, c->vA);
  if (int rc = check_launch(c)) return rc;
  CUDA_TRY(cudaMemcpyAsync(vars1, c->vA, sb, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CSS_OK;
}

extern "C" int css_diffusion(css_ctx *c, double *vars1, const double *avec, double *dvars1) {
  if (!c || !vars1 || !dvars1 || (c->g.magnetic && !avec)) { set_err("css_diffusion: NULL"); return CSS_ERR_ARG; }
  size_t n = c->ncell, sb = n * c->nv * 8;
  CUDA_TRY(cudaMemcpyAsync(c->vA, vars1, sb, cudaMemcpyHostToDevice, c->stream));
  if (c->g.magnetic) {
    CUDA_TRY(cudaMemcpyAsync(c->bf, vars1 + 5 * n, 3 * n * 8, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->vB, avec, 3 * n * 8, cudaMemcpyHostToDevice, c->stream));
  }
  if (int rc = launch_sld(c, c->vA, c->vB, c->dv, nullptr)) return rc;
  CUDA_TRY(cudaMemcpyAsync(dvars1, c->dv, sb, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  // the reference leaves rho and s with the mean state subtracted
  std::vector<double> rhor(c->p.nr), sr(c->p.nr);
  CUDA_TRY(cudaMemcpy(rhor.data(), c->g.rhor, c->p.nr * 8, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(sr.data(), c->g.sr, c->p.nr * 8, cudaMemcpyDeviceToHost));
  size_t plane = (size_t)c->p.nth * c->p.nphi;
  for (int ir = 0; ir < c->p.nr; ir++)
    for (size_t q = 0; q < plane; q++) {
      vars1[ir * plane + q] = vars1[ir * plane + q] - rhor[ir];
      vars1[4 * n + ir * plane + q] = vars1[4 * n + ir * plane + q] - sr[ir];
    }
  return CSS_OK;
}

extern "C" int css_deriv_dev(css_ctx *c, int dir, int order, const double *x, double *dx, const double *bc_lo,
                             const double *bc_hi, int bdry, void *stream) {
  if (!c || !x || !dx || dir < 0 || dir > 2 || order < 1 || order > 2 || bdry < 0 || bdry > 4) {
    set_err("css_deriv: bad argument");
    return CSS_ERR_ARG;
  }
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  const CssGeo &g = c->g;
  if (dir == 1) {
    int TL = c->tl_theta;
    dim3 gr(g.d[1].nb * ((g.nphi + TL - 1) / TL), g.nr);
    size_t sm = smem_theta(1, 1, g.d[1].maxm, TL);
    if (order == 1) k_deriv_theta<1, 0><<<gr, 128, sm, st>>>(g, x, dx, bc_lo, bc_hi, bdry, TL);
    else k_deriv_theta<2, 0><<<gr, 128, sm, st>>>(g, x, dx, bc_lo, bc_hi, bdry, TL);
  } else if (dir == 2) {
    int TL = c->tl_phi;
    dim3 gr(g.d[2].nb * ((g.nth + TL - 1) / TL), g.nr);
    size_t sm = smem_line(1, 1, 0, g.d[2].maxm, TL);
    if (order == 1) k_deriv_phi<1, 0><<<gr, 128, sm, st>>>(g, x, dx, TL);
    else k_deriv_phi<2, 0><<<gr, 128, sm, st>>>(g, x, dx, TL);
  } else {
    int TL = c->tl_r;
    dim3 gr(g.d[0].nb * ((g.nth + TL - 1) / TL), g.nphi);
    size_t sm = smem_line(1, 1, 0, g.d[0].maxm, TL);
    if (order == 1) k_deriv_r<1, 0><<<gr, 128, sm, st>>>(g, x, dx, bc_lo, bc_hi, bdry, TL);
    else k_deriv_r<2, 0><<<gr, 128, sm, st>>>(g, x, dx, bc_lo, bc_hi, bdry, TL);
  }
  return check_launch(c);
}

extern "C" int css_dbydp_cyclic_dev(css_ctx *c, const double *x, double *dx, int order, void *stream) {
  if (!c || !x || !dx || order < 1 || order > 2) { set_err("css_dbydp_cyclic: bad argument"); return CSS_ERR_ARG; }
  if (x == dx) { set_err("css_dbydp_cyclic: x and dx must not overlap"); return CSS_ERR_ARG; }
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  const CssGeo &g = c->g;
  const size_t nl = (size_t)g.nth * g.nr;
  const double dpi = 1.0 / c->g.dphi;
  const double *T = c->cyc + (size_t)(order - 1) * (3 * (size_t)g.nphi + 1);
  k_dbydp_cyclic<<<(unsigned)((nl + 127) / 128), 128, 0, st>>>(g, x, dx, T, order, order == 1 ? dpi : dpi * dpi);
  return check_launch(c);
}

extern "C" int css_dbydp_cyclic(css_ctx *c, const double *x, double *dx, int order) {
  if (!c || !x || !dx) { set_err("css_dbydp_cyclic: NULL"); return CSS_ERR_ARG; }
  const size_t n = c->ncell;
  CUDA_TRY(cudaMemcpyAsync(c->vA, x, n * 8, cudaMemcpyHostToDevice, c->stream));
  if (int rc = css_dbydp_cyclic_dev(c, c->vA, c->dv, order, nullptr)) return rc;
  CUDA_TRY(cudaMemcpyAsync(dx, c->dv, n * 8, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CSS_OK;
}

// dense block operators of css_deriv along dir (zero boundary data): block
// b's m x (m + 8) matrix is the solver applied, on the host, to each unit
// input of the block and its halos, with the run's tables and closures
static int adjoint_mats(css_ctx *c, int dir, int order, int bdry) {
  const int ob = dir == 2 ? 0 : bdry;
  if (c->adjM[dir][order - 1][ob]) return CSS_OK;
  const CssDir &D = c->g.d[dir];
  std::vector<double> M;
  std::vector<int> off(D.nb);
  for (int b = 0; b < D.nb; b++) {
    const int m = D.size[b], ts = m + 2, w = m + 8;
    off[b] = (int)M.size();
    M.resize(M.size() + (size_t)m * w);
    std::vector<double> T(3 * (size_t)ts, 0.0), x(w), o(m);
    double *g1 = T.data(), *g2 = g1 + ts, *g3 = g2 + ts;
    if (dir == 2) tab_p(m, order == 1 ? 1.0 / 3.0 : 2.0 / 11.0, g1, g2, g3);
    else if (order == 1) tab_d1(m, D.lphys[b], D.rphys[b], bdry, g1, g2, g3);
    else tab_d2(m, D.lphys[b], D.rphys[b], bdry, g1, g2, g3);
    const int dtype = dir == 2 ? 3 : (D.lphys[b] ? (D.rphys[b] ? 0 : 2) : (D.rphys[b] ? 1 : 3));
    const double dn = D.dnum[b], sc = order == 1 ? dn : dn * dn;
    for (int col = 0; col < w; col++) {
      std::fill(x.begin(), x.end(), 0.0);
      x[col] = 1.0;
      if (order == 1)
        line_solve_a<1>(x.data() + 4, StridedIn{1}, m, dtype, ob, 0.0, 0.0, T.data(), ts, dn, sc, dir == 2,
                        o.data(), StridedOut{1});
      else
        line_solve_a<2>(x.data() + 4, StridedIn{1}, m, dtype, ob, 0.0, 0.0, T.data(), ts, dn, sc, dir == 2,
                        o.data(), StridedOut{1});
      for (int q = 0; q < m; q++) M[(size_t)off[b] + (size_t)q * w + col] = o[q];
    }
  }
  double *dM = nullptr;
  int *dO = nullptr;
  if (cudaMalloc(&dM, M.size() * 8) != cudaSuccess || cudaMalloc(&dO, off.size() * sizeof(int)) != cudaSuccess) {
    cudaFree(dM);
    set_err("css_deriv_adjoint: device allocation failed");
    return CSS_ERR_NOMEM;
  }
  CUDA_TRY(cudaMemcpy(dM, M.data(), M.size() * 8, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(dO, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice));
  c->adjM[dir][order - 1][ob] = dM;
  c->adjOff[dir][order - 1][ob] = dO;
  return CSS_OK;
}

extern "C" int css_deriv_adjoint_dev(css_ctx *c, int dir, int order, const double *g, double *gx, int bdry,
                                     void *stream) {
  if (!c || !g || !gx || dir < 0 || dir > 2 || order < 1 || order > 2 || bdry < 0 || bdry > 4 || g == gx) {
    set_err("css_deriv_adjoint: bad argument");
    return CSS_ERR_ARG;
  }
  if (int rc = adjoint_mats(c, dir, order, bdry)) return rc;
  const int ob = dir == 2 ? 0 : bdry;
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  k_deriv_adjoint<<<(unsigned)((c->ncell + 255) / 256), 256, 0, st>>>(c->g, dir, c->adjM[dir][order - 1][ob],
                                                                       c->adjOff[dir][order - 1][ob], g, gx);
  return check_launch(c);
}

extern "C" int css_deriv(css_ctx *c, int dir, int order, const double *x, double *dx, const double *bc_lo,
                         const double *bc_hi, int bdry) {
  if (!c || !x || !dx) { set_err("css_deriv: NULL"); return CSS_ERR_ARG; }
  size_t n = c->ncell;
  size_t face = dir == 0 ? (size_t)c->p.nth * c->p.nphi : (size_t)c->p.nphi * c->p.nr;
  double *bl = c->vB, *bh = c->vB + face;  // scratch
  CUDA_TRY(cudaMemcpyAsync(c->vA, x, n * 8, cudaMemcpyHostToDevice, c->stream));
  if (bc_lo) CUDA_TRY(cudaMemcpyAsync(bl, bc_lo, face * 8, cudaMemcpyHostToDevice, c->stream));
  if (bc_hi) CUDA_TRY(cudaMemcpyAsync(bh, bc_hi, face * 8, cudaMemcpyHostToDevice, c->stream));
  if (int rc = css_deriv_dev(c, dir, order, c->vA, c->dv, bc_lo ? bl : nullptr, bc_hi ? bh : nullptr, bdry, nullptr))
    return rc;
  CUDA_TRY(cudaMemcpyAsync(dx, c->dv, n * 8, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CSS_OK;
}

// The six derivative routines by the reference's names, with its `var`
// argument (derivatives.f90:558-562): var >= 1 takes the boundary condition
// of field var from ibcr (r) or ibct (theta), var <= 0 means bdry = -var.
// Dbydp / D2bydp2 have no boundary variants and ignore var.
static int deriv_var(css_ctx *c, int dir, int order, const double *x, double *dx, const double *b1,
                     const double *b2, int var, const char *who) {
  if (!c) { set_err("%s: NULL", who); return CSS_ERR_ARG; }
  int bdry = 1;
  if (dir < 2) {
    if (var > 12) { set_err("%s: var %d beyond the 12 fields of the BC tables", who, var); return CSS_ERR_ARG; }
    bdry = var >= 1 ? (dir == 0 ? c->g.ibcr[var] : c->g.ibct[var]) : -var;
    if (bdry < 0 || bdry > 4) { set_err("%s: var %d gives no boundary variant 0..4", who, var); return CSS_ERR_ARG; }
  }
  return css_deriv(c, dir, order, x, dx, b1, b2, bdry);
}
extern "C" int css_dbydr(css_ctx *c, const double *x, double *dx, const double *b1, const double *b2, int var) {
  return deriv_var(c, 0, 1, x, dx, b1, b2, var, "css_dbydr");
}
extern "C" int css_d2bydr2(css_ctx *c, const double *x, double *dx, const double *b1, const double *b2, int var) {
  return deriv_var(c, 0, 2, x, dx, b1, b2, var, "css_d2bydr2");
}
extern "C" int css_dbydt(css_ctx *c, const double *x, double *dx, const double *b1, const double *b2, int var) {
  return deriv_var(c, 1, 1, x, dx, b1, b2, var, "css_dbydt");
}
extern "C" int css_d2bydt2(css_ctx *c, const double *x, double *dx, const double *b1, const double *b2, int var) {
  return deriv_var(c, 1, 2, x, dx, b1, b2, var, "css_d2bydt2");
}
extern "C" int css_dbydp(css_ctx *c, const double *x, double *dx, int var) {
  return deriv_var(c, 2, 1, x, dx, nullptr, nullptr, var, "css_dbydp");
}
extern "C" int css_d2bydp2(css_ctx *c, const double *x, double *dx, int var) {
  return deriv_var(c, 2, 2, x, dx, nullptr, nullptr, var, "css_d2bydp2");
}

// The reference's per-pencil calls, batched: dir 0 pencils are (theta, r)
// planes of one phi (Dbydr's x(mynth, mynr)), dir 1 / 2 pencils (theta, phi)
// planes of one radius (Dbydt's and Dbydp's x(mynth, mynphi)).  Each pencil
// goes into the field buffer at its own phi plane (dir 0) or radius (1, 2)
// -- D2bydt2 scales the Neumann datum by the radial block's dri, so a
// theta pencil's result depends on its radius -- and a pass takes pencils
// until one repeats an index.  The derivative of a plane depends on that
// plane alone, so the other planes of the buffer play no part.
extern "C" int css_deriv_pencils(css_ctx *c, int dir, int order, int npencils, const int *index, const double *x,
                                 double *dx, const double *bc_lo, const double *bc_hi, int var) {
  if (!c || !x || !dx || npencils < 0 || dir < 0 || dir > 2 || (order != 1 && order != 2)) {
    set_err("css_deriv_pencils: bad argument");
    return CSS_ERR_ARG;
  }
  int bdry = 1;
  if (dir < 2) {
    if (var > 12) { set_err("css_deriv_pencils: var %d beyond the 12 fields of the BC tables", var); return CSS_ERR_ARG; }
    bdry = var >= 1 ? (dir == 0 ? c->g.ibcr[var] : c->g.ibct[var]) : -var;
    if (bdry < 0 || bdry > 4) { set_err("css_deriv_pencils: var %d gives no boundary variant 0..4", var); return CSS_ERR_ARG; }
  }
  const size_t nth = c->p.nth, nphi = c->p.nphi, nr = c->p.nr, plane_tp = nth * nphi;
  const size_t pen = dir == 0 ? nth * nr : plane_tp;        // doubles per pencil
  const size_t bcn = dir == 0 ? nth : (dir == 1 ? nphi : 0);  // face data per pencil
  const int cap = dir == 0 ? (int)nphi : (int)nr;
  for (int p = 0; p < npencils; p++) {
    const int k = index ? index[p] : p % cap;
    if (k < 0 || k >= cap) {
      set_err("css_deriv_pencils: pencil %d has index %d outside 0..%d", p, k, cap - 1);
      return CSS_ERR_ARG;
    }
  }
  const size_t face = dir == 0 ? plane_tp : nphi * nr;
  double *bl = c->vB, *bh = c->vB + face;  // scratch
  std::vector<char> used(cap);
  for (int p0 = 0; p0 < npencils;) {
    std::fill(used.begin(), used.end(), 0);
    int p1 = p0;
    while (p1 < npencils) {
      const int k = index ? index[p1] : p1 % cap;
      if (used[k]) break;
      used[k] = 1;
      p1++;
    }
    CUDA_TRY(cudaMemsetAsync(c->vA, 0, c->ncell * 8, c->stream));
    if (bcn) CUDA_TRY(cudaMemsetAsync(bl, 0, 2 * face * 8, c->stream));
    for (int p = p0; p < p1; p++) {
      const int k = index ? index[p] : p % cap;
      const double *xs = x + (size_t)p * pen;
      if (dir == 0)  // phi plane k: nr rows of nth
        CUDA_TRY(cudaMemcpy2DAsync(c->vA + (size_t)k * nth, plane_tp * 8, xs, nth * 8, nth * 8, nr,
                                   cudaMemcpyHostToDevice, c->stream));
      else  // radius k: the field layout itself
        CUDA_TRY(cudaMemcpyAsync(c->vA + (size_t)k * plane_tp, xs, pen * 8, cudaMemcpyHostToDevice, c->stream));
      if (bcn && bc_lo)
        CUDA_TRY(cudaMemcpyAsync(bl + (size_t)k * bcn, bc_lo + (size_t)p * bcn, bcn * 8, cudaMemcpyHostToDevice,
                                 c->stream));
      if (bcn && bc_hi)
        CUDA_TRY(cudaMemcpyAsync(bh + (size_t)k * bcn, bc_hi + (size_t)p * bcn, bcn * 8, cudaMemcpyHostToDevice,
                                 c->stream));
    }
    if (int rc = css_deriv_dev(c, dir, order, c->vA, c->dv, (bcn && bc_lo) ? bl : nullptr,
                               (bcn && bc_hi) ? bh : nullptr, bdry, nullptr))
      return rc;
    for (int p = p0; p < p1; p++) {
      const int k = index ? index[p] : p % cap;
      double *ds = dx + (size_t)p * pen;
      if (dir == 0)
        CUDA_TRY(cudaMemcpy2DAsync(ds, nth * 8, c->dv + (size_t)k * nth, plane_tp * 8, nth * 8, nr,
                                   cudaMemcpyDeviceToHost, c->stream));
      else
        CUDA_TRY(cudaMemcpyAsync(ds, c->dv + (size_t)k * plane_tp, pen * 8, cudaMemcpyDeviceToHost, c->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    p0 = p1;
  }
  return CSS_OK;
}

// Lines with explicit closures; used by css_dbyd1_dt0 and css_compact_lines.
static int run_lines(const double *x, double *dx, int n, int nlines, int order, int lphys, int rphys, int bdry,
                     const double *bclo, const double *bchi, const double *hlo, const double *hhi, double dnum,
                     double scale, int dt0_quirk) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { set_err("no CUDA device"); return CSS_ERR_NODEV; }
  int ts = n + 2;
  std::vector<double> T((size_t)5 * 3 * ts, 0.0);
  for (int iv = 0; iv < 5; iv++) {
    double *g1 = &T[(size_t)iv * 3 * ts], *g2 = g1 + ts, *g3 = g2 + ts;
    if (order == 1) tab_d1(n, lphys, rphys, iv, g1, g2, g3);
    else tab_d2(n, lphys, rphys, iv, g1, g2, g3);
  }
  if (dt0_quirk && order == 1 && bdry == 2) {
    // Dbyd1_dt0 zeroes up1 before copying it into up2 (derivatives.f90:
    // 2355-2386), so for ibc = 2 its last row has no lower coefficient:
    // pivot 1/(1 - 0*c3) = 1 and no elimination term
    double *g2 = &T[(size_t)2 * 3 * ts] + ts, *g3 = g2 + ts;
    g2[n] = 1.0;
    g3[n] = 0.0;
  }
  int dtype = lphys ? (rphys ? 0 : 2) : (rphys ? 1 : 3);
  double *dT = nullptr, *dx_ = nullptr, *dy = nullptr, *work = nullptr, *dbl = nullptr, *dbh = nullptr, *dhl = nullptr,
         *dhh = nullptr;
  size_t nb = (size_t)n * nlines * 8;
  int rc = CSS_OK;
  auto fail = [&](const char *what, cudaError_t e) {
    set_err("%s: %s", what, cudaGetErrorString(e));
    rc = CSS_ERR_CUDA;
  };
  cudaError_t e;
  if ((e = cudaMalloc(&dT, T.size() * 8)) || (e = cudaMalloc(&dx_, nb)) || (e = cudaMalloc(&dy, nb)) ||
      (e = cudaMalloc(&work, (size_t)(n + 8) * nlines * 8)) || (e = cudaMalloc(&dbl, nlines * 8)) ||
      (e = cudaMalloc(&dbh, nlines * 8)) || (e = cudaMalloc(&dhl, (size_t)4 * nlines * 8)) ||
      (e = cudaMalloc(&dhh, (size_t)4 * nlines * 8))) {
    fail("lines alloc", e);
  } else {
    cudaMemcpy(dT, T.data(), T.size() * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(dx_, x, nb, cudaMemcpyHostToDevice);
    if (bclo) cudaMemcpy(dbl, bclo, nlines * 8, cudaMemcpyHostToDevice);
    if (bchi) cudaMemcpy(dbh, bchi, nlines * 8, cudaMemcpyHostToDevice);
    if (hlo) cudaMemcpy(dhl, hlo, (size_t)4 * nlines * 8, cudaMemcpyHostToDevice);
    if (hhi) cudaMemcpy(dhh, hhi, (size_t)4 * nlines * 8, cudaMemcpyHostToDevice);
    if (n <= KL_MAXN) {  // lines staged through shared memory, every global access coalesced
      const size_t smem = 2 * (size_t)KL_LINES * (n + 9) * 8;
      cudaFuncSetAttribute(k_lines_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           2 * KL_LINES * (KL_MAXN + 9) * 8);  // on the current device
      k_lines_tiled<<<(nlines + KL_LINES - 1) / KL_LINES, 128, smem>>>(
          dx_, dy, n, nlines, order, dtype, bdry, bclo ? dbl : nullptr, bchi ? dbh : nullptr, hlo ? dhl : nullptr,
          hhi ? dhh : nullptr, dT, ts, dnum, scale);
    } else {
      k_lines<<<(nlines + 127) / 128, 128>>>(dx_, dy, n, nlines, order, dtype, bdry, bclo ? dbl : nullptr,
                                             bchi ? dbh : nullptr, hlo ? dhl : nullptr, hhi ? dhh : nullptr, dT, ts,
                                             dnum, scale, work);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) fail("k_lines", e);
    else if ((e = cudaMemcpy(dx, dy, nb, cudaMemcpyDeviceToHost)) != cudaSuccess) fail("lines copy", e);
  }
  cudaFree(dT); cudaFree(dx_); cudaFree(dy); cudaFree(work); cudaFree(dbl); cudaFree(dbh); cudaFree(dhl); cudaFree(dhh);
  return rc;
}

extern "C" int css_dbyd1_dt0(const double *x, double *dxdy, const double *bdat1, const double *bdat2, int n1, int ibc,
                             int nlines) {
  if (!x || !dxdy || n1 < 14 || n1 > 100000 || ibc < 0 || ibc > 4 || nlines < 0) {
    set_err("css_dbyd1_dt0: need n1 >= 14 and ibc in 0..4");
    return CSS_ERR_ARG;
  }
  if (nlines == 0) return CSS_OK;
  // Dbyd1_dt0 takes the Neumann datum already divided by the spacing and
  // returns d/dx in grid units (the caller multiplies by 1/dx)
  return run_lines(x, dxdy, n1, nlines, 1, 1, 1, ibc, bdat1, bdat2, nullptr, nullptr, 1.0, 1.0, 1);
}

extern "C" int css_compact_lines(const double *x, double *dx, int n, int nlines, int order, int lphys, int rphys,
                                 int bdry, const double *bc_lo, const double *bc_hi, const double *halo_lo,
                                 const double *halo_hi, double dnum, double scale) {
  if (!x || !dx || n < 10 || n > 100000 || order < 1 || order > 2 || bdry < 0 || bdry > 4 || nlines < 0 ||
      (!lphys && !halo_lo) || (!rphys && !halo_hi)) {
    set_err("css_compact_lines: bad argument");
    return CSS_ERR_ARG;
  }
  if (nlines == 0) return CSS_OK;
  return run_lines(x, dx, n, nlines, order, lphys, rphys, bdry, bc_lo, bc_hi, halo_lo, halo_hi, dnum, scale, 0);
}

extern "C" int css_sync(css_ctx *c) {
  if (!c) return CSS_ERR_ARG;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CSS_OK;
}

extern "C" int css_state_device_ptr(css_ctx *c, double **dptr, long long *nelem) {
  if (!c || !dptr || !nelem) return CSS_ERR_ARG;
  *dptr = c->v0;
  *nelem = (long long)(c->ncell * c->nv);
  return CSS_OK;
}

extern "C" long long css_kernel_launches(css_ctx *c) { return c ? c->launches : 0; }

extern "C" int css_set_stream(css_ctx *c, void *stream) {
  if (!c) { set_err("css_set_stream: NULL"); return CSS_ERR_ARG; }
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return CSS_OK;
}

extern "C" int css_profile(css_ctx *c, int enable) {
  if (!c) { set_err("css_profile: NULL"); return CSS_ERR_ARG; }
  prof_collect(c);
  for (int k = 0; k < KI_COUNT; k++) { c->k_ms[k] = 0.0; c->k_count[k] = 0; }
  c->profiling = enable ? 1 : 0;
  return CSS_OK;
}

extern "C" int css_kernel_stats(css_ctx *c, int kind, const char **name, double *total_ms, long long *launches) {
  if (!c || kind < 0 || kind >= KI_COUNT) return CSS_ERR_ARG;
  prof_collect(c);
  if (name) *name = kKernelNames[kind];
  if (total_ms) *total_ms = c->k_ms[kind];
  if (launches) *launches = c->k_count[kind];
  return CSS_OK;
}

// ---------------------------------------------------------------------------
// Tile autotuner: for each sweep direction, the RHS of the resident state is
// timed with every tile height that direction's kernels have (8 or 16
// lines for the compile-time block lengths; 16, 8, 4 lines that fit for
// the generic kernels) and the fastest is kept.  Every line's arithmetic is
// the same for any tile height, so the choice changes no result bit.
// ---------------------------------------------------------------------------
extern "C" int css_autotune(css_ctx *c, int reps, int *chosen) {
  if (!c || reps < 1) { set_err("css_autotune: bad argument"); return CSS_ERR_ARG; }
  const int prof_was = c->profiling;
  c->profiling = 0;
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  int *tl[3] = {&c->tl_r, &c->tl_theta, &c->tl_phi};
  const int dirs[3] = {1, 2, 0};  // theta (theta terms, rhot, curl), phi, r
  int rc = CSS_OK;
  for (int di = 0; di < 3 && rc == CSS_OK; di++) {
    const int d = dirs[di];
    const int mag = c->g.magnetic, m = c->g.d[d].maxm;
    std::vector<int> cand;
    if (c->mt[d]) cand = {16, 8};
    else
      for (int t : {16, 8, 4}) {
        size_t need = d == 1 ? std::max(smem_theta_terms(mag, m, t), smem_rhot(m, t))
                             : (d == 2 ? smem_phi_terms(mag, m, t) : smem_radial_terms(mag, m, t));
        if (need <= kSmemCap) cand.push_back(t);
      }
    int best = *tl[d], best_pers = c->phi_pers;
    float best_ms = 1e30f;
    std::vector<std::pair<int, int>> variants;  // (tile height, persistent phi kernel)
    for (int t : cand) {
      variants.push_back({t, 0});
      if (d == 2 && c->mt[d]) variants.push_back({t, 1});
    }
    for (auto tv : variants) {
      const int t = tv.first;
      *tl[d] = t;
      if (d == 2) c->phi_pers = tv.second;
      if ((rc = launch_rhs(c, (const double *)c->v0, (double *)nullptr, 0, 0.0))) break;  // warm
      cudaEventRecord(e0, c->stream);
      for (int k = 0; k < reps && rc == CSS_OK; k++) rc = launch_rhs(c, (const double *)c->v0, (double *)nullptr, 0, 0.0);
      cudaEventRecord(e1, c->stream);
      if (rc) break;
      if (cudaEventSynchronize(e1) != cudaSuccess) { set_err("css_autotune: timing failed"); rc = CSS_ERR_CUDA; break; }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best_ms) { best_ms = ms; best = t; best_pers = tv.second; }
    }
    *tl[d] = best;
    if (d == 2) c->phi_pers = best_pers;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->profiling = prof_was;
  if (chosen) { chosen[0] = c->tl_r; chosen[1] = c->tl_theta; chosen[2] = c->tl_phi; }
  return rc;
}

// the autotuner's choices set by hand: tile heights (lines per CTA) of the
// r, theta and phi kernels and the persistent phi kernel (0/1); a height a
// direction does not offer is refused
extern "C" int css_set_fused(css_ctx *c, int on) {
  if (!c) { set_err("css_set_fused: NULL"); return CSS_ERR_ARG; }
  if (on && !c->fused_ok) {
    set_err("css_set_fused: the two-pass stage needs 32-point blocks in r, theta and phi and an FP64 RK4 run "
            "with closed radial faces, no explicit viscosity, radiative diffusion or prescribed bottom");
    return CSS_ERR_ARG;
  }
  c->fused = on ? 1 : 0;
  return CSS_OK;
}

extern "C" int css_get_fused(css_ctx *c) { return c ? c->fused : -1; }

extern "C" int css_set_tiles(css_ctx *c, int tl_r, int tl_theta, int tl_phi, int phi_persistent) {
  if (!c) { set_err("css_set_tiles: NULL"); return CSS_ERR_ARG; }
  const int tl[3] = {tl_r, tl_theta, tl_phi};
  const int mag = c->g.magnetic;
  for (int d = 0; d < 3; d++) {
    const int t = tl[d], m = c->g.d[d].maxm;
    bool ok = c->mt[d] ? (t == 8 || t == 16) : (t == 4 || t == 8 || t == 16);
    if (ok && !c->mt[d]) {
      size_t need = d == 1 ? std::max(smem_theta_terms(mag, m, t), smem_rhot(m, t))
                           : (d == 2 ? smem_phi_terms(mag, m, t) : smem_radial_terms(mag, m, t));
      ok = need <= kSmemCap;
    }
    if (!ok) { set_err("css_set_tiles: %d lines per CTA not available in direction %d", t, d); return CSS_ERR_ARG; }
  }
  if (phi_persistent && !c->mt[2]) { set_err("css_set_tiles: the persistent phi kernel needs 16- or 32-point blocks"); return CSS_ERR_ARG; }
  c->tl_r = tl_r; c->tl_theta = tl_theta; c->tl_phi = tl_phi; c->phi_pers = phi_persistent ? 1 : 0;
  return CSS_OK;
}

extern "C" int css_set_curl_pass(css_ctx *c, int mode) {
  if (!c || mode < 0 || mode > 2) { set_err("css_set_curl_pass: NULL context or mode not 0..2"); return CSS_ERR_ARG; }
  c->curl_tp = mode;
  return CSS_OK;
}

// ---------------------------------------------------------------------------
// Batched ensemble: one RK4 step of every member is captured once into a
// CUDA graph (each member's kernels on a stream of its own, forked from and
// joined to the ensemble's root stream, so small members run side by side)
// and the graph is replayed for every step.  Members keep their own state,
// parameters and tables; the graph is captured again when a time step
// changes.
// ---------------------------------------------------------------------------
struct css_ensemble {
  std::vector<css_ctx *> m;
  std::vector<cudaStream_t> ms;
  std::vector<cudaEvent_t> join;
  std::vector<double> dt;
  cudaStream_t root = nullptr;
  cudaEvent_t fork = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t t0 = nullptr, t1 = nullptr;  // around the replays of the last step call
  double last_ms = 0.0;
  long long launches_per_step = 0, launches = 0;
};

extern "C" void css_ensemble_destroy(css_ensemble *e) {
  if (!e) return;
  if (e->exec) cudaGraphExecDestroy(e->exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  for (auto s : e->ms) cudaStreamDestroy(s);
  for (auto v : e->join) cudaEventDestroy(v);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->t0) cudaEventDestroy(e->t0);
  if (e->t1) cudaEventDestroy(e->t1);
  if (e->root) cudaStreamDestroy(e->root);
  delete e;
}

extern "C" int css_ensemble_create(int nmem, css_ctx *const *members, css_ensemble **out) {
  if (!out || nmem < 1 || !members) { set_err("css_ensemble_create: bad argument"); return CSS_ERR_ARG; }
  *out = nullptr;
  for (int i = 0; i < nmem; i++) {
    if (!members[i]) { set_err("css_ensemble_create: member %d is NULL", i); return CSS_ERR_ARG; }
    if (members[i]->io) {
      set_err("css_ensemble_create: member %d has an open radial boundary, whose per-step host clock a "
              "captured step cannot carry", i);
      return CSS_ERR_ARG;
    }
  }
  css_ensemble *e = new css_ensemble();
  e->m.assign(members, members + nmem);
  e->ms.resize(nmem);
  e->join.resize(nmem);
  cudaError_t err = cudaStreamCreateWithFlags(&e->root, cudaStreamNonBlocking);
  if (!err) err = cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming);
  if (!err) err = cudaEventCreate(&e->t0);
  if (!err) err = cudaEventCreate(&e->t1);
  for (int i = 0; i < nmem && !err; i++) {
    err = cudaStreamCreateWithFlags(&e->ms[i], cudaStreamNonBlocking);
    if (!err) err = cudaEventCreateWithFlags(&e->join[i], cudaEventDisableTiming);
  }
  if (err) {
    set_err("css_ensemble_create: %s", cudaGetErrorString(err));
    css_ensemble_destroy(e);
    return CSS_ERR_CUDA;
  }
  *out = e;
  return CSS_OK;
}

static int ensemble_capture(css_ensemble *e, const double *dt) {
  if (e->exec) { cudaGraphExecDestroy(e->exec); e->exec = nullptr; }
  if (e->graph) { cudaGraphDestroy(e->graph); e->graph = nullptr; }
  const int nm = (int)e->m.size();
  CUDA_TRY(cudaStreamBeginCapture(e->root, cudaStreamCaptureModeThreadLocal));
  int rc = CSS_OK;
  long long l0 = 0, l1 = 0;
  cudaError_t err = cudaEventRecord(e->fork, e->root);
  for (int i = 0; i < nm && !rc && !err; i++) {
    css_ctx *c = e->m[i];
    err = cudaStreamWaitEvent(e->ms[i], e->fork, 0);
    if (err) break;
    cudaStream_t keep = c->stream;
    const int prof = c->profiling;
    c->stream = e->ms[i];
    c->profiling = 0;
    l0 = c->launches;
    rc = step_once(c, dt[i]);
    l1 += c->launches - l0;
    c->stream = keep;
    c->profiling = prof;
    if (!rc) err = cudaEventRecord(e->join[i], e->ms[i]);
    if (!rc && !err) err = cudaStreamWaitEvent(e->root, e->join[i], 0);
  }
  cudaGraph_t g = nullptr;
  cudaError_t end = cudaStreamEndCapture(e->root, &g);
  if (rc || err || end) {
    if (g) cudaGraphDestroy(g);
    if (!rc) {
      set_err("css_ensemble_step: capture failed: %s", cudaGetErrorString(err ? err : end));
      rc = CSS_ERR_CUDA;
    }
    return rc;
  }
  e->graph = g;
  CUDA_TRY(cudaGraphInstantiate(&e->exec, e->graph, 0));
  e->dt.assign(dt, dt + nm);
  e->launches_per_step = l1;
  return CSS_OK;
}

extern "C" int css_ensemble_step(css_ensemble *e, const double *dt, int nsteps) {
  if (!e || !dt || nsteps < 0) { set_err("css_ensemble_step: bad argument"); return CSS_ERR_ARG; }
  const int nm = (int)e->m.size();
  for (int i = 0; i < nm; i++)
    if (!(dt[i] > 0.0)) { set_err("css_ensemble_step: dt[%d] must be positive", i); return CSS_ERR_ARG; }
  bool same = e->exec != nullptr;
  for (int i = 0; i < nm && same; i++) same = (e->dt[i] == dt[i]);
  // order after whatever each member's own stream has queued (uploads)
  for (int i = 0; i < nm; i++) {
    CUDA_TRY(cudaEventRecord(e->join[i], e->m[i]->stream));
    CUDA_TRY(cudaStreamWaitEvent(e->root, e->join[i], 0));
  }
  if (!same)
    if (int rc = ensemble_capture(e, dt)) return rc;
  for (int i = 0; i < nm; i++) CUDA_TRY(cudaMemsetAsync(e->m[i]->flag, 0, sizeof(int), e->root));
  CUDA_TRY(cudaEventRecord(e->t0, e->root));
  for (int s = 0; s < nsteps; s++) CUDA_TRY(cudaGraphLaunch(e->exec, e->root));
  CUDA_TRY(cudaEventRecord(e->t1, e->root));
  e->launches += e->launches_per_step * nsteps;
  std::vector<int> h(nm, 0);
  for (int i = 0; i < nm; i++)
    CUDA_TRY(cudaMemcpyAsync(&h[i], e->m[i]->flag, sizeof(int), cudaMemcpyDeviceToHost, e->root));
  CUDA_TRY(cudaStreamSynchronize(e->root));
  float ms = 0.f;
  CUDA_TRY(cudaEventElapsedTime(&ms, e->t0, e->t1));
  e->last_ms = ms;
  for (int i = 0; i < nm; i++)
    if (h[i] & kFlagTimeout) {
      set_err("css_ensemble_step: member %d: a tile's staged copies did not arrive within the kernel's bounded wait", i);
      return CSS_ERR_CUDA;
    }
  for (int i = 0; i < nm; i++)
    if (h[i]) { set_err("css_ensemble_step: non-finite value in member %d", i); return CSS_ERR_NAN; }
  return CSS_OK;
}

extern "C" double css_ensemble_last_ms(css_ensemble *e) { return e ? e->last_ms : -1.0; }

extern "C" long long css_ensemble_launches(css_ensemble *e) { return e ? e->launches : -1; }

// ---------------------------------------------------------------------------
// Diagnostics of the current state (vars0): Scalar_Output, Compute_Step_Size,
// Shell_Average_Output and the (theta, phi) spectrum.  Between steps the
// stage buffers are free, so they hold the scratch: vA = ds/dr, vB = face
// data and spectrum tables, vs = reduction partials and per-radius results,
// dv = spectrum line sums, bf = B.
// ---------------------------------------------------------------------------
__global__ void k_fill2(double *a, size_t n, double x, double y) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < 2 * n; i += (size_t)gridDim.x * blockDim.x)
    a[i] = i < n ? x : y;
}

static int stats_chunks(const css_ctx *c) {
  const size_t np = (size_t)c->p.nth * c->p.nphi;
  int nchunk = (4 * 148 + c->p.nr - 1) / c->p.nr;  // about four CTAs per SM over all radii
  nchunk = std::max(1, std::min(nchunk, 64));
  while (nchunk > 1 && np / (size_t)nchunk < 256) nchunk--;
  return nchunk;
}

// per-radius accumulators res[ir*SA_N + a] of the current state
static int run_stats(css_ctx *c, int need_dsdr, std::vector<double> &res) {
  const CssGeo &g = c->g;
  const size_t n = c->ncell, np = (size_t)g.nth * g.nphi;
  const int nr = g.nr, nchunk = stats_chunks(c);
  if ((size_t)nr * nchunk * SA_NPASS1 + (size_t)nr * SA_N > (size_t)c->nv * n) {
    set_err("diagnostics: grid too small for the reduction scratch");
    return CSS_ERR_ARG;
  }
  cudaStream_t st = c->stream;
  if (g.magnetic)
    if (int rc = launch_curl(c, (const double *)(c->v0 + 5 * n), c->bf, 1)) return rc;  // Compute_B(0)
  const double *dsdr = nullptr;
  if (need_dsdr) {
    // Compute_Derivatives (report_mpi.f90:288-318): d s/d r with the
    // constant-flux datum dsdr1/dxdr(1), dsdr2/dxdr(nr) at the faces
    k_fill2<<<256, 256, 0, st>>>(c->vB, np, c->rep_flux_lo, c->rep_flux_hi);
    if (int rc = check_launch(c)) return rc;
    if (int rc = css_deriv_dev(c, 0, 1, c->v0 + 4 * n, c->vA, c->vB, c->vB + np, g.ibcr[5], nullptr)) return rc;
    dsdr = c->vA;
  }
  double *part = c->vs, *resd = c->vs + (size_t)nr * nchunk * SA_NPASS1;
  k_stats_pass1<<<dim3(nchunk, nr), 256, 0, st>>>(g, c->v0, c->bf, dsdr, part);
  if (int rc = check_launch(c)) return rc;
  k_stats_combine<<<nr, 32, 0, st>>>(part, nchunk, SA_NPASS1, 0, resd);
  if (int rc = check_launch(c)) return rc;
  k_stats_pass2<<<dim3(nchunk, nr), 256, 0, st>>>(g, c->v0, resd, part);
  if (int rc = check_launch(c)) return rc;
  k_stats_combine<<<nr, 32, 0, st>>>(part, nchunk, SA_NPASS2, SA_NPASS1, resd);
  if (int rc = check_launch(c)) return rc;
  res.assign((size_t)nr * SA_N, 0.0);
  CUDA_TRY(cudaMemcpyAsync(res.data(), resd, res.size() * 8, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return CSS_OK;
}

extern "C" int css_scalars(css_ctx *c, double *out) {
  if (!c || !out) { set_err("css_scalars: NULL argument"); return CSS_ERR_ARG; }
  std::vector<double> res;
  if (int rc = run_stats(c, 0, res)) return rc;
  const int nr = c->p.nr;
  const double ntot = (double)c->ncell;
  double s[SA_N] = {0};
  double umax = -INFINITY, bmax2 = -INFINITY;
  for (int ir = 0; ir < nr; ir++) {
    const double *r = &res[(size_t)ir * SA_N];
    for (int a : {SA_RU2, SA_RW2, SA_RV2, SA_RUSQ, SA_BSQ}) s[a] += r[a];
    umax = std::max(umax, r[SA_UMACH]);
    bmax2 = std::max(bmax2, r[SA_BMAX2]);
  }
  const double cke = s[SA_RU2] / (2.0 * ntot);
  out[0] = s[SA_RUSQ] / (2.0 * ntot);                                // kinener
  out[1] = cke;                                                      // cke
  out[2] = cke + s[SA_RW2] / (2.0 * ntot);                           // mcke
  out[3] = s[SA_RV2] / (2.0 * ntot);                                 // drke
  out[4] = sqrt(umax);                                               // umach
  out[5] = c->p.magnetic ? s[SA_BSQ] / (8.0 * M_PI * ntot) : 0.0;    // magener
  out[6] = c->p.magnetic ? sqrt(bmax2) * 2.0 * sqrt(2.0 * M_PI) : 0.0;  // bmax
  return CSS_OK;
}

extern "C" int css_step_size(css_ctx *c, double cfl_safety, double *out) {
  if (!c || !out) { set_err("css_step_size: NULL argument"); return CSS_ERR_ARG; }
  std::vector<double> res;
  if (int rc = run_stats(c, 0, res)) return rc;
  double dtc = 1e4, dtb = 1e4, e = 0.0, l = 0.0, m = 0.0, mrs = 0.0;
  for (int ir = 0; ir < c->p.nr; ir++) {
    const double *r = &res[(size_t)ir * SA_N];
    dtc = std::min(dtc, r[SA_DTC]);
    if (c->p.magnetic) dtb = std::min(dtb, r[SA_DTB]);
    e += r[SA_E];
    l += r[SA_L];
    m += r[SA_M];
    mrs += r[SA_MRS];
  }
  const double dtd = c->dtd;  // 1e10 unless explicit viscosity is on
  out[0] = std::min(std::min(dtb, dtc), dtd) * cfl_safety;
  out[1] = e;
  out[2] = l;
  out[3] = m;
  out[4] = mrs;
  return CSS_OK;
}

extern "C" int css_shell_averages(css_ctx *c, const int *quantities, int nq, const double *k0, double *out) {
  if (!c || !quantities || !out || nq < 1) { set_err("css_shell_averages: bad argument"); return CSS_ERR_ARG; }
  int need_dsdr = 0;
  for (int iq = 0; iq < nq; iq++) {
    const int q = quantities[iq];
    if (q < 1 || q > 18) {
      set_err("css_shell_averages: quantity %d not supported (1..18; 19 needs the SLD flux output)", q);
      return CSS_ERR_ARG;
    }
    if (q == 15 && c->p.do_radheat) {
      set_err("css_shell_averages: F_ks of a radiative-diffusion run (the kr T^3 dT/dr term) is not built");
      return CSS_ERR_ARG;
    }
    if (q >= 10 && q <= 14 && !c->p.magnetic) {
      set_err("css_shell_averages: quantity %d needs a magnetic run", q);
      return CSS_ERR_ARG;
    }
    if (q == 9 || q == 15) need_dsdr = 1;
  }
  std::vector<double> res;
  if (int rc = run_stats(c, need_dsdr, res)) return rc;
  const int nr = c->p.nr;
  const double inv = 1.0 / ((double)c->p.nth * c->p.nphi);
  const double gamm1 = c->p.gamma - 1.0, cv = c->p.cp / c->p.gamma;
  std::vector<double> ksh(nr);
  CUDA_TRY(cudaMemcpy(ksh.data(), c->g.ks, nr * 8, cudaMemcpyDeviceToHost));
  static const int kMap[19] = {-1, SA_RHO, SA_T, SA_S, SA_RHOT, SA_VR, SA_VT, SA_VP, SA_KE, SA_DSDR,
                               SA_BR, SA_BT, SA_BP, SA_ME, SA_BPOL, SA_DSDR, SA_FEN, SA_FKE, SA_FAC};
  for (int iq = 0; iq < nq; iq++) {
    const int q = quantities[iq];
    for (int ir = 0; ir < nr; ir++) {
      const double sum = res[(size_t)ir * SA_N + kMap[q]];
      double v;
      if (q == 4) v = gamm1 * cv * sum * inv;
      else if (q == 15) {  // F_ks: conduction by the SLaplacian ks plus the prescribed flux k0
        const double k0r = k0 ? k0[ir] : 0.0;
        v = c->g.slaplacian ? -ksh[ir] * sum * inv + k0r : k0r;
      } else if (q == 16) v = c->p.cp * sum * inv;
      else v = sum * inv;
      out[(size_t)iq * nr + ir] = v;
    }
  }
  return CSS_OK;
}

extern "C" int css_spectrum(css_ctx *c, int kind, double *out) {
  if (!c || !out) { set_err("css_spectrum: NULL argument"); return CSS_ERR_ARG; }
  const int nth = c->p.nth, nphi = c->p.nphi, nr = c->p.nr;
  if (nth % 2 || nphi % 2 || nth < 4 || nphi < 4) {
    set_err("css_spectrum: nth and nphi must be even");
    return CSS_ERR_ARG;
  }
  if (kind < 0 || kind > 1 + c->nv || (kind == 1 && !c->p.magnetic)) {
    set_err("css_spectrum: kind %d not available (0 KE, 1 ME (magnetic), 2+iv variable iv)", kind);
    return CSS_ERR_ARG;
  }
  const size_t n = c->ncell;
  cudaStream_t st = c->stream;
  if (kind == 1)
    if (int rc = launch_curl(c, (const double *)(c->v0 + 5 * n), c->bf, 1)) return rc;
  // theta weights: apodisation 1 - cos(pi (theta - theta_1)/(theta_n - theta_1))^64 and
  // W(t) = sum_{kt=1}^{nth/2-1} exp(-2 pi i kt t / nth); phi twiddles cos|sin(2 pi j / nphi)
  std::vector<double> tab(3 * (size_t)nth + 2 * (size_t)nphi);
  const double dth = (c->p.th2 - c->p.th1) / (double)(nth - 1);
  const double th0 = c->p.th1, thn = dth * (double)(nth - 1) + c->p.th1;
  for (int t = 0; t < nth; t++) {
    const double th = dth * (double)t + c->p.th1;
    const double apod = 1.0 - pow(cos(M_PI * (th - th0) / (thn - th0)), 64);
    double wr = 0.0, wi = 0.0;
    for (int kt = 1; kt < nth / 2; kt++) {
      const double ang = 2.0 * M_PI * (double)(((long long)kt * t) % nth) / (double)nth;
      wr += cos(ang);
      wi -= sin(ang);
    }
    tab[t] = apod;
    tab[nth + t] = apod * wr;
    tab[2 * nth + t] = apod * wi;
  }
  for (int j = 0; j < nphi; j++) {
    const double ang = 2.0 * M_PI * (double)j / (double)nphi;
    tab[3 * nth + j] = cos(ang);
    tab[3 * nth + nphi + j] = sin(ang);
  }
  CUDA_TRY(cudaMemcpyAsync(c->vB, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice, st));
  k_spec_theta<<<dim3((nphi + 7) / 8, nr), 256, 0, st>>>(c->g, c->v0, c->bf, kind, c->vB, c->dv);
  if (int rc = check_launch(c)) return rc;
  const size_t sm = (size_t)3 * nphi * 8;
  if (sm > 48 * 1024) CUDA_TRY(cudaFuncSetAttribute(k_spec_phi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  k_spec_phi<<<nr, 256, sm, st>>>(c->dv, c->vB + 3 * nth, nth, nphi, c->vA);
  if (int rc = check_launch(c)) return rc;
  CUDA_TRY(cudaMemcpyAsync(out, c->vA, (size_t)nr * (nphi / 2) * 8, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return CSS_OK;
}

// ---------------------------------------------------------------------------
// Learned subgrid closure.  A fine state is box-filtered into coarse fields
// and the twelve subgrid targets; 3x3x3 stencil features of the coarse
// fields feed an MLP (in 135 -> 128 -> 128 -> 128 -> 12, GELU (tanh form), BF16 weights
// and activations, FP32 accumulation) whose matrix products run on the
// tensor cores in the fused inference kernel or, for training and the
// per-layer path, in k_gemm_bf16; its predicted subgrid velocity variance
// becomes the per-cell SLD speed^2 of a coarse run, in place of the
// prescribed radial profile (diffusion.f90:19-63).
// ---------------------------------------------------------------------------
extern "C" int css_set_sld_speed2(css_ctx *c, const double *speed2) {
  if (!c) { set_err("css_set_sld_speed2: NULL context"); return CSS_ERR_ARG; }
  c->g.speed2 = speed2;
  return CSS_OK;
}

extern "C" int css_box_filter(css_ctx *c, int f, double *fields, double *targets) {
  if (!c || !fields || !targets || f < 1 || c->p.nr % f || c->p.nth % f || c->p.nphi % f) {
    set_err("css_box_filter: bad argument (the factor must divide nr, nth and nphi)");
    return CSS_ERR_ARG;
  }
  const size_t n = c->ncell;
  if (c->g.magnetic)
    if (int rc = launch_curl(c, (const double *)(c->v0 + 5 * n), c->bf, 1)) return rc;
  k_box_filter<<<148 * 8, 256, 0, c->stream>>>(c->g, c->v0, c->g.magnetic ? c->bf : nullptr, f, c->p.nth / f,
                                                c->p.nphi / f, c->p.nr / f, fields, targets);
  if (int rc = check_launch(c)) return rc;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CSS_OK;
}

extern "C" int css_closure_scales(int nct, int ncp, int ncr, const double *fields, const double *targets,
                                  float *scales) {
  if (!fields || !scales || nct < 1 || ncp < 1 || ncr < 1) { set_err("css_closure_scales: bad argument"); return CSS_ERR_ARG; }
  const int nb = 148 * 2, nk = CL_NQ + CL_NTARGET;
  double *part = nullptr;
  CUDA_TRY(cudaMalloc(&part, (size_t)nb * nk * 8));
  k_closure_sumsq<<<nb, 256>>>(fields, targets, nct, ncp, ncr, part);
  std::vector<double> h((size_t)nb * nk);
  cudaError_t e = cudaGetLastError();
  if (!e) e = cudaMemcpy(h.data(), part, h.size() * 8, cudaMemcpyDeviceToHost);
  cudaFree(part);
  if (e) { set_err("css_closure_scales: %s", cudaGetErrorString(e)); return CSS_ERR_CUDA; }
  const double nc = (double)nct * ncp * ncr;
  for (int k = 0; k < nk; k++) {
    double s = 0.0;
    for (int b = 0; b < nb; b++) s += h[(size_t)b * nk + k];
    const double rms = sqrt(s / nc);
    scales[k] = (float)(rms > 0.0 ? rms : 1.0);
  }
  return CSS_OK;
}

extern "C" int css_closure_features(int nct, int ncp, int ncr, const double *fields, const float *scale, void *x) {
  if (!fields || !scale || !x || nct < 1 || ncp < 1 || ncr < 1) { set_err("css_closure_features: bad argument"); return CSS_ERR_ARG; }
  k_closure_features<<<148 * 8, 128>>>(fields, nct, ncp, ncr, scale, (__nv_bfloat16 *)x);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaDeviceSynchronize());
  return CSS_OK;
}

extern "C" int css_closure_targets(long long nc, const double *targets, const float *tscale, float *tn) {
  if (!targets || !tscale || !tn || nc < 1) { set_err("css_closure_targets: bad argument"); return CSS_ERR_ARG; }
  k_closure_targets<<<148 * 8, 256>>>(targets, (size_t)nc, tscale, tn);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaDeviceSynchronize());
  return CSS_OK;
}

extern "C" int css_closure_speed2(long long nc, const float *y, const float *tscale, double *speed2) {
  if (!y || !tscale || !speed2 || nc < 1) { set_err("css_closure_speed2: bad argument"); return CSS_ERR_ARG; }
  k_closure_speed2<<<148 * 8, 256>>>(y, (size_t)nc, tscale, speed2);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaDeviceSynchronize());
  return CSS_OK;
}

extern "C" int css_closure_speed2_shaped(css_ctx *c, const float *y, const float *tscale, double *speed2) {
  if (!c || !y || !tscale || !speed2) { set_err("css_closure_speed2_shaped: bad argument"); return CSS_ERR_ARG; }
  k_closure_speed2_shaped<<<c->p.nr, 256, 0, c->stream>>>(c->g, y, tscale, speed2);
  if (int rc = check_launch(c)) return rc;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CSS_OK;
}

// the two grids of a restriction / prolongation: same variables, the fine
// one f times the coarse one in every direction
static bool grid_pair(const css_ctx *fine, const css_ctx *coarse, int f) {
  return fine && coarse && f >= 1 && fine->nv == coarse->nv && coarse->p.nr * f == fine->p.nr &&
         coarse->p.nth * f == fine->p.nth && coarse->p.nphi * f == fine->p.nphi;
}

extern "C" int css_restrict_state(css_ctx *fine, const double *fine_base, int f, css_ctx *coarse,
                                  const double *coarse_base) {
  if (!grid_pair(fine, coarse, f)) {
    set_err("css_restrict_state: the fine grid must be f times the coarse grid in every direction, same variables");
    return CSS_ERR_ARG;
  }
  CUDA_TRY(cudaStreamSynchronize(coarse->stream));
  k_restrict_state<<<148 * 8, 256, 0, fine->stream>>>(fine->v0, fine_base, fine->p.nth, fine->p.nphi, fine->p.nr, f,
                                                       fine->nv, coarse_base, coarse->v0);
  if (int rc = check_launch(fine)) return rc;
  CUDA_TRY(cudaStreamSynchronize(fine->stream));
  if (coarse->bg2) {
    const size_t nrt = (size_t)coarse->p.nr * coarse->p.nth;
    k_phi_mean<<<(unsigned)((nrt + 127) / 128), 128, 0, coarse->stream>>>(coarse->g, coarse->v0, coarse->bg2);
    if (int rc = check_launch(coarse)) return rc;
    CUDA_TRY(cudaStreamSynchronize(coarse->stream));
  }
  return CSS_OK;
}

extern "C" int css_prolong_add(css_ctx *coarse, const double *coarse_base, int f, css_ctx *fine) {
  if (!grid_pair(fine, coarse, f)) {
    set_err("css_prolong_add: the fine grid must be f times the coarse grid in every direction, same variables");
    return CSS_ERR_ARG;
  }
  CUDA_TRY(cudaStreamSynchronize(coarse->stream));
  k_prolong_add<<<148 * 8, 256, 0, fine->stream>>>(coarse->v0, coarse_base, coarse->p.nth, coarse->p.nphi,
                                                    coarse->p.nr, f, fine->nv, fine->v0);
  if (int rc = check_launch(fine)) return rc;
  if (fine->bg2) {
    const size_t nrt = (size_t)fine->p.nr * fine->p.nth;
    k_phi_mean<<<(unsigned)((nrt + 127) / 128), 128, 0, fine->stream>>>(fine->g, fine->v0, fine->bg2);
    if (int rc = check_launch(fine)) return rc;
  }
  CUDA_TRY(cudaStreamSynchronize(fine->stream));
  return CSS_OK;
}

struct css_mlp {
  int dims[5];          // padded widths: input, hidden x3, output
  int nreal_in, nreal_out;
  size_t cap;           // rows per pass
  float *W[4] = {}, *B[4] = {}, *gW[4] = {}, *gB[4] = {}, *mW[4] = {}, *vW[4] = {}, *mB[4] = {}, *vB[4] = {};
  __nv_bfloat16 *Wb[4] = {};
  __nv_bfloat16 *WbT[4] = {};   // Wb transposed (out x in), for the forward products
  bool wt_ok = false;
  float *Z[4] = {};             // pre-activations; Z[3] is the output
  __nv_bfloat16 *H[4] = {};     // H[1..3] activations; H[0] is the caller's input
  float *dH = nullptr;          // FP32 gradient scratch
  __nv_bfloat16 *dZb = nullptr; // BF16 gradient
  double *part = nullptr;
  int adam_t = 0;
  float *gpart = nullptr;       // row-chunk partials of the weight gradients
  cudaStream_t st = nullptr, own_st = nullptr;
  unsigned char *packed = nullptr;  // weights for the fused forward kernel
  bool packed_ok = false;
  int fused = 2;                    // 0 per-layer GEMMs, 1 fused mma.sync kernel, 2 fused tcgen05 kernel
  int *flag = nullptr;              // set by the tcgen05 kernel when its bounded wait runs out
};

// the products of a pass, on k_gemm_bf16 (row-major; see css_closure.cuh)
#define GM_NSPLIT 64
// Z = X W with W read as its transpose WT (out x in): the same access
// pattern as dH = dZ W^T, so both run the row-contiguous form of the kernel
static int gemm_fwd(css_mlp *m, const __nv_bfloat16 *X, const __nv_bfloat16 *WT, float *Z, size_t rows, int K, int M) {
  dim3 grid((unsigned)((rows + GM_TP - 1) / GM_TP), (M + GM_TQ - 1) / GM_TQ);
  k_gemm_bf16<GM_DIN><<<grid, 128, 0, m->st>>>(X, WT, Z, (int)rows, M, K, K, K, 0);
  CUDA_TRY(cudaGetLastError());
  return CSS_OK;
}
static int gemm_din(css_mlp *m, const __nv_bfloat16 *D, const __nv_bfloat16 *W, float *dH, size_t rows, int K, int M) {
  dim3 grid((unsigned)((rows + GM_TP - 1) / GM_TP), (K + GM_TQ - 1) / GM_TQ);
  k_gemm_bf16<GM_DIN><<<grid, 128, 0, m->st>>>(D, W, dH, (int)rows, K, M, M, M, 0);
  CUDA_TRY(cudaGetLastError());
  return CSS_OK;
}
static int gemm_dw(css_mlp *m, const __nv_bfloat16 *X, const __nv_bfloat16 *D, float *gW, size_t rows, int K, int M) {
  long long chunk = ((long long)rows + GM_NSPLIT - 1) / GM_NSPLIT;
  chunk = std::max(256LL, (chunk + 15) / 16 * 16);
  const int nsplit = (int)(((long long)rows + chunk - 1) / chunk);
  dim3 grid((K + GM_TP - 1) / GM_TP, (M + GM_TQ - 1) / GM_TQ, nsplit);
  k_gemm_bf16<GM_DW><<<grid, 128, 0, m->st>>>(X, D, m->gpart, K, M, (long long)rows, K, M, chunk);
  CUDA_TRY(cudaGetLastError());
  k_sum_partials<<<64, 256, 0, m->st>>>(m->gpart, nsplit, K * M, gW);
  CUDA_TRY(cudaGetLastError());
  return CSS_OK;
}

__global__ void k_to_bf16(const float *__restrict__ a, __nv_bfloat16 *__restrict__ b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = __float2bfloat16_rn(a[i]);
}

extern "C" void css_mlp_destroy(css_mlp *m) {
  if (!m) return;
  for (int l = 0; l < 4; l++) {
    cudaFree(m->W[l]); cudaFree(m->B[l]); cudaFree(m->gW[l]); cudaFree(m->gB[l]);
    cudaFree(m->mW[l]); cudaFree(m->vW[l]); cudaFree(m->mB[l]); cudaFree(m->vB[l]); cudaFree(m->Wb[l]); cudaFree(m->WbT[l]);
    cudaFree(m->Z[l]); cudaFree(m->H[l]);
  }
  cudaFree(m->dH); cudaFree(m->dZb); cudaFree(m->part); cudaFree(m->gpart); cudaFree(m->packed);
  cudaFree(m->flag);
  if (m->own_st) cudaStreamDestroy(m->own_st);
  else if (m->st) cudaStreamDestroy(m->st);
  delete m;
}

extern "C" int css_mlp_create(int n_in, int width, int n_out, int max_rows, unsigned long long seed, css_mlp **out) {
  if (!out || n_in < 1 || width < 16 || width % 16 || n_out < 1 || max_rows < 1) {
    set_err("css_mlp_create: bad argument (width a multiple of 16)");
    return CSS_ERR_ARG;
  }
  *out = nullptr;
  css_mlp *m = new css_mlp();
  auto pad16 = [](int x) { return (x + 15) / 16 * 16; };
  m->nreal_in = n_in;
  m->nreal_out = n_out;
  m->dims[0] = pad16(n_in);
  m->dims[1] = m->dims[2] = m->dims[3] = width;
  m->dims[4] = pad16(n_out);
  m->cap = (size_t)max_rows;
  cudaError_t e = cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking);
  const int wmax = std::max(std::max(m->dims[0], width), m->dims[4]);
  if (!e) e = cudaMalloc(&m->gpart, (size_t)GM_NSPLIT * wmax * wmax * 4);
  for (int l = 0; l < 4 && !e; l++) {
    const size_t K = m->dims[l], M = m->dims[l + 1];
    float **f4[] = {&m->W[l], &m->gW[l], &m->mW[l], &m->vW[l]};
    for (auto pp : f4)
      if (!e) e = cudaMalloc(pp, K * M * 4);
    float **b4[] = {&m->B[l], &m->gB[l], &m->mB[l], &m->vB[l]};
    for (auto pp : b4)
      if (!e) e = cudaMalloc(pp, M * 4);
    if (!e) e = cudaMalloc(&m->Wb[l], K * M * 2);
    if (!e) e = cudaMalloc(&m->WbT[l], K * M * 2);
    if (!e) e = cudaMalloc(&m->Z[l], m->cap * M * 4);
    if (!e && l > 0) e = cudaMalloc(&m->H[l], m->cap * K * 2);
  }
  if (!e) e = cudaMalloc(&m->dH, m->cap * wmax * 4);
  if (!e) e = cudaMalloc(&m->dZb, m->cap * wmax * 2);
  if (!e) e = cudaMalloc(&m->part, 1024 * 8);
  if (!e) e = cudaMalloc(&m->packed, FM_PARAM_BYTES);
  if (e) {
    set_err("css_mlp_create: %s", cudaGetErrorString(e));
    css_mlp_destroy(m);
    return e == cudaErrorMemoryAllocation ? CSS_ERR_NOMEM : CSS_ERR_CUDA;
  }
  // Glorot-uniform weights from a SplitMix64 stream, zero biases; the rows
  // of padded inputs and the columns of padded outputs are zero
  unsigned long long x = seed;
  auto next = [&x]() {
    unsigned long long z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  };
  for (int l = 0; l < 4 && !e; l++) {
    const int K = m->dims[l], M = m->dims[l + 1];
    const int kr = l == 0 ? n_in : K, mr = l == 3 ? n_out : M;
    const double a = sqrt(6.0 / (double)(kr + mr));
    std::vector<float> w((size_t)K * M, 0.0f), z((size_t)K * M, 0.0f), zb(M, 0.0f);
    for (int k = 0; k < K; k++)
      for (int j = 0; j < M; j++) {
        const double u = next();
        if (k < kr && j < mr) w[(size_t)k * M + j] = (float)(a * (2.0 * u - 1.0));
      }
    if (!e) e = cudaMemcpy(m->W[l], w.data(), w.size() * 4, cudaMemcpyHostToDevice);
    for (float *p : {m->mW[l], m->vW[l]})
      if (!e) e = cudaMemcpy(p, z.data(), z.size() * 4, cudaMemcpyHostToDevice);
    for (float *p : {m->B[l], m->mB[l], m->vB[l]})
      if (!e) e = cudaMemcpy(p, zb.data(), zb.size() * 4, cudaMemcpyHostToDevice);
    if (!e) {
      k_to_bf16<<<64, 256, 0, m->st>>>(m->W[l], m->Wb[l], (size_t)K * M);
      e = cudaGetLastError();
    }
  }
  if (!e) e = cudaStreamSynchronize(m->st);
  if (e) {
    set_err("css_mlp_create: %s", cudaGetErrorString(e));
    css_mlp_destroy(m);
    return CSS_ERR_CUDA;
  }
  *out = m;
  return CSS_OK;
}

extern "C" int css_mlp_dims(css_mlp *m, int *dims) {
  if (!m || !dims) return CSS_ERR_ARG;
  for (int k = 0; k < 5; k++) dims[k] = m->dims[k];
  return CSS_OK;
}

// forward pass of n <= cap rows: Z[3] holds the outputs (row-major n x dims[4])
static int mlp_forward_rows(css_mlp *m, const __nv_bfloat16 *x, size_t n) {
  if (!m->wt_ok) {
    for (int l = 0; l < 4; l++) {
      k_transpose_bf16<<<64, 256, 0, m->st>>>(m->Wb[l], m->dims[l], m->dims[l + 1], m->WbT[l]);
      CUDA_TRY(cudaGetLastError());
    }
    m->wt_ok = true;
  }
  const __nv_bfloat16 *in = x;
  for (int l = 0; l < 4; l++) {
    const int K = m->dims[l], M = m->dims[l + 1];
    if (int rc = gemm_fwd(m, in, m->WbT[l], m->Z[l], n, K, M)) return rc;
    __nv_bfloat16 *next = l < 3 ? m->H[l + 1] : nullptr;
    k_bias_gelu<<<148 * 4, 256, 0, m->st>>>(m->Z[l], m->B[l], next, M, n);
    CUDA_TRY(cudaGetLastError());
    in = next;
  }
  return CSS_OK;
}

static bool mlp_fusable(const css_mlp *m) {
  return m->dims[0] == FM_IN && m->dims[1] == FM_W && m->dims[2] == FM_W && m->dims[3] == FM_W &&
         m->dims[4] == FM_OUT;
}

// transposed, padded BF16 weights and FP32 biases in one block for k_mlp_fused
static int mlp_pack(css_mlp *m) {
  const int kp[4] = {FM_KP0, FM_KP, FM_KP, FM_KP};
  const size_t off[4] = {0, FM_OFF_W1, FM_OFF_W2, FM_OFF_W3};
  for (int l = 0; l < 4; l++) {
    k_pack_wt<<<64, 256, 0, m->st>>>(m->Wb[l], m->dims[l], m->dims[l + 1], kp[l],
                                      reinterpret_cast<__nv_bfloat16 *>(m->packed + off[l]));
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(m->packed + FM_OFF_B + (size_t)l * FM_W * 4, m->B[l], (size_t)m->dims[l + 1] * 4,
                             cudaMemcpyDeviceToDevice, m->st));
  }
  m->packed_ok = true;
  return CSS_OK;
}

// 1: forward passes use the fused kernel (the default when the widths are
// 144/128/128/128/16); 0: the per-layer GEMM path
extern "C" int css_mlp_set_fused(css_mlp *m, int on) {
  if (!m || on < 0 || on > 2) { set_err("css_mlp_set_fused: bad argument"); return CSS_ERR_ARG; }
  m->fused = on;
  return CSS_OK;
}

extern "C" int css_mlp_forward(css_mlp *m, const void *x, long long n, float *y) {
  if (!m || !x || !y || n < 1) { set_err("css_mlp_forward: bad argument"); return CSS_ERR_ARG; }
  const int K0 = m->dims[0], MO = m->dims[4];
  if (m->fused == 2 && mlp_fusable(m)) {
    static bool attr_tc = false;
    if (!attr_tc) {
      CUDA_TRY(cudaFuncSetAttribute(k_mlp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM_BYTES));
      attr_tc = true;
    }
    if (!m->packed_ok)
      if (int rc = mlp_pack(m)) return rc;
    if (!m->flag) {
      CUDA_TRY(cudaMalloc(&m->flag, sizeof(int)));
    }
    CUDA_TRY(cudaMemsetAsync(m->flag, 0, sizeof(int), m->st));
    const long long ntiles = (n + TC_ROWS - 1) / TC_ROWS;
    int dev = 0, nsm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int grid = (int)std::min<long long>(nsm, ntiles);
    k_mlp_tc<<<grid, TC_NT, TC_SMEM_BYTES, m->st>>>((const __nv_bfloat16 *)x, n, m->packed, y, m->flag);
    CUDA_TRY(cudaGetLastError());
    int h = 0;
    CUDA_TRY(cudaMemcpyAsync(&h, m->flag, sizeof(int), cudaMemcpyDeviceToHost, m->st));
    CUDA_TRY(cudaStreamSynchronize(m->st));
    if (h) { set_err("css_mlp_forward: tensor-core products did not complete within the kernel's bounded wait"); return CSS_ERR_CUDA; }
    return CSS_OK;
  }
  if (m->fused && mlp_fusable(m)) {
    static bool attr_done = false;
    if (!attr_done) {
      CUDA_TRY(cudaFuncSetAttribute(k_mlp_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, FM_SMEM_BYTES));
      attr_done = true;
    }
    if (!m->packed_ok)
      if (int rc = mlp_pack(m)) return rc;
    const long long ntiles = (n + 15) / 16;
    const int grid = (int)std::min<long long>(148, (ntiles + FM_WARPS - 1) / FM_WARPS);
    k_mlp_fused<<<grid, FM_WARPS * 32, FM_SMEM_BYTES, m->st>>>((const __nv_bfloat16 *)x, n, m->packed, y);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(m->st));
    return CSS_OK;
  }
  for (long long r0 = 0; r0 < n; r0 += (long long)m->cap) {
    const size_t rows = (size_t)std::min<long long>((long long)m->cap, n - r0);
    if (int rc = mlp_forward_rows(m, (const __nv_bfloat16 *)x + (size_t)r0 * K0, rows)) return rc;
    CUDA_TRY(cudaMemcpyAsync(y + (size_t)r0 * MO, m->Z[3], rows * MO * 4, cudaMemcpyDeviceToDevice, m->st));
  }
  CUDA_TRY(cudaStreamSynchronize(m->st));
  return CSS_OK;
}

extern "C" int css_mlp_train_step(css_mlp *m, const void *x, const float *t, long long n, float lr, float *loss) {
  if (!m || !x || !t || n < 1 || (size_t)n > m->cap) {
    set_err("css_mlp_train_step: bad argument (at most %zu rows per step)", m ? m->cap : (size_t)0);
    return CSS_ERR_ARG;
  }
  const size_t rows = (size_t)n;
  const __nv_bfloat16 *xb = (const __nv_bfloat16 *)x;
  if (int rc = mlp_forward_rows(m, xb, rows)) return rc;
  const int nb = 256;
  k_mse<<<nb, 256, 0, m->st>>>(m->Z[3], t, rows, m->nreal_out, m->dH, m->dZb, m->part);
  CUDA_TRY(cudaGetLastError());
  for (int l = 3; l >= 0; l--) {
    const int K = m->dims[l], M = m->dims[l + 1];
    const __nv_bfloat16 *in = l == 0 ? xb : m->H[l];
    // dW = dZ^T-contracted input, db = column sums of dZ
    if (int rc = gemm_dw(m, in, m->dZb, m->gW[l], rows, K, M)) return rc;
    k_colsum<<<M, 256, 0, m->st>>>(m->dH, M, rows, m->gB[l]);
    CUDA_TRY(cudaGetLastError());
    if (l > 0) {
      if (int rc = gemm_din(m, m->dZb, m->Wb[l], m->dH, rows, K, M)) return rc;
      k_gelu_back<<<148 * 4, 256, 0, m->st>>>(m->dH, m->Z[l - 1], m->dZb, (size_t)K * rows);
      CUDA_TRY(cudaGetLastError());
    }
  }
  m->adam_t++;
  m->packed_ok = false;
  m->wt_ok = false;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.0f - powf(b1, (float)m->adam_t), c2 = 1.0f - powf(b2, (float)m->adam_t);
  for (int l = 0; l < 4; l++) {
    const size_t K = m->dims[l], M = m->dims[l + 1];
    k_adam<<<148, 256, 0, m->st>>>(m->W[l], m->gW[l], m->mW[l], m->vW[l], m->Wb[l], K * M, lr, b1, b2, eps, c1, c2);
    k_adam<<<4, 256, 0, m->st>>>(m->B[l], m->gB[l], m->mB[l], m->vB[l], nullptr, M, lr, b1, b2, eps, c1, c2);
  }
  CUDA_TRY(cudaGetLastError());
  std::vector<double> h(nb);
  CUDA_TRY(cudaMemcpyAsync(h.data(), m->part, nb * 8, cudaMemcpyDeviceToHost, m->st));
  CUDA_TRY(cudaStreamSynchronize(m->st));
  double s = 0.0;
  for (double v : h) s += v;
  if (loss) *loss = (float)(s / ((double)rows * m->nreal_out));
  return CSS_OK;
}

// run the network's work on the caller's stream (NULL: its own)
extern "C" int css_mlp_set_stream(css_mlp *m, void *stream) {
  if (!m) { set_err("css_mlp_set_stream: NULL"); return CSS_ERR_ARG; }
  if (!m->own_st) m->own_st = m->st;
  m->st = stream ? (cudaStream_t)stream : m->own_st;
  return CSS_OK;
}

// host copies of layer l's FP32 weights (row-major dims[l] x dims[l+1]) and
// biases; set = 1 writes them (and refreshes the BF16 copy)
extern "C" int css_mlp_params(css_mlp *m, int l, float *w, float *b, int set) {
  if (!m || l < 0 || l > 3) { set_err("css_mlp_params: bad argument"); return CSS_ERR_ARG; }
  const size_t K = m->dims[l], M = m->dims[l + 1];
  if (set) {
    if (w) CUDA_TRY(cudaMemcpy(m->W[l], w, K * M * 4, cudaMemcpyHostToDevice));
    if (b) CUDA_TRY(cudaMemcpy(m->B[l], b, M * 4, cudaMemcpyHostToDevice));
    k_to_bf16<<<64, 256, 0, m->st>>>(m->W[l], m->Wb[l], K * M);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(m->st));
    m->packed_ok = false;
    m->wt_ok = false;
  } else {
    if (w) CUDA_TRY(cudaMemcpy(w, m->W[l], K * M * 4, cudaMemcpyDeviceToHost));
    if (b) CUDA_TRY(cudaMemcpy(b, m->B[l], M * 4, cudaMemcpyDeviceToHost));
  }
  return CSS_OK;
}

// the last train step's gradients of layer l (host, same layout)
extern "C" int css_mlp_grads(css_mlp *m, int l, float *gw, float *gb) {
  if (!m || l < 0 || l > 3) { set_err("css_mlp_grads: bad argument"); return CSS_ERR_ARG; }
  const size_t K = m->dims[l], M = m->dims[l + 1];
  CUDA_TRY(cudaStreamSynchronize(m->st));
  if (gw) CUDA_TRY(cudaMemcpy(gw, m->gW[l], K * M * 4, cudaMemcpyDeviceToHost));
  if (gb) CUDA_TRY(cudaMemcpy(gb, m->gB[l], M * 4, cudaMemcpyDeviceToHost));
  return CSS_OK;
}

// ---------------------------------------------------------------------------
// Checkpoints in the reference's layout (Checkpoint_Output / Checkpoint_Input,
// checkpoint.f90:146-423): a directory holding a text `header` -- line 1
// nr, nth, nphi, nv, istep as (5i9), line 2 deltat, sim_time, r1, r2, th1,
// th2, phi1, phi2 as (8e14.7) -- and one file `checkpoint.<name>` per field
// (rho w v u s bt bp br; for MHD the last three hold the vector potential,
// as vars0 does) with the raw FP64 array (nth, nphi, nr) in Fortran order,
// which is the library's own layout of a field.
// ---------------------------------------------------------------------------
static const char *kCkptNames[8] = {"rho", "w", "v", "u", "s", "bt", "bp", "br"};

// Fortran E14.7: [-]0.dddddddE+xx right-justified in 14 columns
static void fortran_e14_7(double x, char *out) {
  char m[64];
  if (x == 0.0 || !std::isfinite(x)) {
    if (x == 0.0) snprintf(out, 15, "%14s", std::signbit(x) ? "-0.0000000E+00" : "0.0000000E+00");
    else snprintf(out, 15, "%14s", std::isnan(x) ? "NaN" : (x > 0 ? "Infinity" : "-Infinity"));
    return;
  }
  snprintf(m, sizeof m, "%.6E", fabs(x));  // d.ddddddE+xx: the 7 significant digits
  const int e10 = atoi(m + 9) + 1;           // exponent of the 0.d form
  char digits[8] = {m[0], m[2], m[3], m[4], m[5], m[6], m[7], 0};
  char buf[32];
  if (e10 > 99 || e10 < -99) snprintf(buf, sizeof buf, "%s0.%s%+04d", x < 0 ? "-" : "", digits, e10);
  else snprintf(buf, sizeof buf, "%s0.%sE%+03d", x < 0 ? "-" : "", digits, e10);
  size_t len = strlen(buf);  // at most 14: -0.dddddddE+xx or -0.ddddddd+xxx
  if (len > 14) len = 14;
  memset(out, ' ', 14 - len);
  memcpy(out + 14 - len, buf, len);
  out[14] = 0;
}

extern "C" int css_checkpoint_write(css_ctx *c, const char *dir, int istep, double deltat, double sim_time) {
  if (!c || !dir) { set_err("css_checkpoint_write: NULL argument"); return CSS_ERR_ARG; }
  mkdir(dir, 0755);  // as Make_Checkpoint_Filename; an existing directory is fine
  std::string d(dir);
  if (d.empty() || d.back() != '/') d += '/';
  const css_params &p = c->p;
  FILE *f = fopen((d + "header").c_str(), "w");
  if (!f) { set_err("css_checkpoint_write: cannot create %sheader", d.c_str()); return CSS_ERR_ARG; }
  fprintf(f, "%9d%9d%9d%9d%9d\n", p.nr, p.nth, p.nphi, c->nv, istep);
  const double h2[8] = {deltat, sim_time, p.r1, p.r2, p.th1, p.th2, p.phi1, p.phi2};
  for (int k = 0; k < 8; k++) {
    char e[16];
    fortran_e14_7(h2[k], e);
    fputs(e, f);
  }
  fputs("\n", f);
  fclose(f);
  std::vector<double> h((size_t)c->nv * c->ncell);
  if (int rc = css_download_state(c, h.data())) return rc;
  for (int iv = 0; iv < c->nv; iv++) {
    FILE *g = fopen((d + "checkpoint." + kCkptNames[iv]).c_str(), "wb");
    if (!g) { set_err("css_checkpoint_write: cannot create %scheckpoint.%s", d.c_str(), kCkptNames[iv]); return CSS_ERR_ARG; }
    const size_t w = fwrite(h.data() + (size_t)iv * c->ncell, 8, c->ncell, g);
    fclose(g);
    if (w != c->ncell) { set_err("css_checkpoint_write: short write of checkpoint.%s", kCkptNames[iv]); return CSS_ERR_ARG; }
  }
  return CSS_OK;
}

extern "C" int css_checkpoint_read(css_ctx *c, const char *dir, int *istep, double *deltat, double *sim_time) {
  if (!c || !dir) { set_err("css_checkpoint_read: NULL argument"); return CSS_ERR_ARG; }
  std::string d(dir);
  if (d.empty() || d.back() != '/') d += '/';
  FILE *f = fopen((d + "header").c_str(), "r");
  if (!f) { set_err("css_checkpoint_read: cannot open %sheader", d.c_str()); return CSS_ERR_ARG; }
  int nr = 0, nth = 0, nphi = 0, nv = 0, step = 0;
  double h2[8] = {0};
  int got = fscanf(f, "%d %d %d %d %d", &nr, &nth, &nphi, &nv, &step);
  for (int k = 0; k < 8 && got == 5 + k; k++) got += fscanf(f, "%lf", &h2[k]);
  fclose(f);
  if (got != 13) { set_err("css_checkpoint_read: malformed header in %s", d.c_str()); return CSS_ERR_ARG; }
  if (nr != c->p.nr || nth != c->p.nth || nphi != c->p.nphi) {
    // the reference interpolates horizontally (Checkpoint_Interpolate); not here
    set_err("css_checkpoint_read: checkpoint is %dx%dx%d, the run %dx%dx%d", nr, nth, nphi, c->p.nr, c->p.nth,
            c->p.nphi);
    return CSS_ERR_ARG;
  }
  std::vector<double> h((size_t)c->nv * c->ncell);
  if (int rc = css_download_state(c, h.data())) return rc;  // fields the file lacks keep their values
  for (int iv = 0; iv < std::min(c->nv, nv); iv++) {
    FILE *g = fopen((d + "checkpoint." + kCkptNames[iv]).c_str(), "rb");
    if (!g) { set_err("css_checkpoint_read: cannot open %scheckpoint.%s", d.c_str(), kCkptNames[iv]); return CSS_ERR_ARG; }
    const size_t r = fread(h.data() + (size_t)iv * c->ncell, 8, c->ncell, g);
    fclose(g);
    if (r != c->ncell) { set_err("css_checkpoint_read: checkpoint.%s is short", kCkptNames[iv]); return CSS_ERR_ARG; }
  }
  if (int rc = css_upload_state(c, h.data())) return rc;
  if (istep) *istep = step;
  if (deltat) *deltat = h2[0];
  if (sim_time) *sim_time = h2[1];
  return CSS_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free compact lines.
//
// Some callers cannot allocate device memory at the moment they want a
// derivative: a code that has handed all device memory to its own pool or
// to a framework's caching allocator at start-up (cudaMalloc then fails or
// evicts their cache), or one that must not stall, because cudaMalloc and
// cudaFree synchronize the whole device.  css_compact_lines_noalloc serves
// them: the caller passes device buffers for the inputs and outputs, and
// the LU tables and the halo-padded copies of the lines live in one
// file-scope device array of fixed size that every GPU loading this library
// holds until the process exits.  Nothing is allocated, on the device or
// on the host.
// ---------------------------------------------------------------------------
#define CSS_NOALLOC_DOUBLES (1 << 18)  // 2 MiB of scratch per device
static __device__ __align__(256) double g_noalloc_scratch[CSS_NOALLOC_DOUBLES];
// device address of the array, per device: published with release order
// once it has been looked up, so a host thread that sees it non-null also
// sees a finished lookup; the lookup itself runs under g_noalloc_mu
static std::atomic<double *> g_noalloc_addr[64];
static std::mutex g_noalloc_mu;

// The array's device address on the current device.  The first lookup on a
// device loads this library's device code there (under lazy module loading
// that is when the array itself is placed in device memory), so it must run
// before the caller hands its device memory to a pool and before any stream
// capture.
static int noalloc_scratch(double **out) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) { set_err("css_compact_lines_noalloc: device index %d out of range", dev); return CSS_ERR_ARG; }
  double *p = g_noalloc_addr[dev].load(std::memory_order_acquire);
  if (!p) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    p = g_noalloc_addr[dev].load(std::memory_order_relaxed);
    if (!p) {
      CUDA_TRY(cudaGetSymbolAddress((void **)&p, g_noalloc_scratch));
      g_noalloc_addr[dev].store(p, std::memory_order_release);
    }
  }
  *out = p;
  return CSS_OK;
}

// LU tables of one (n, lphys, rphys) line for bdry 0..4, written on the
// device with the same correctly rounded steps as the host's tab_d1/tab_d2
// (no contraction), so they equal the tables css_compact_lines uses.
__global__ void k_noalloc_tables(double *T, int n, int lphys, int rphys, int order) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int ts = n + 2;
  for (int k = 0; k < 15 * ts; k++) T[k] = 0.0;
  for (int iv = 0; iv < 5; iv++) {
    double *g1 = T + (size_t)iv * 3 * ts, *g2 = g1 + ts, *g3 = g2 + ts;
    double alpha, a2, g2c, up1, up2;
    if (order == 1) {
      alpha = 1.0 / 3.0; a2 = 0.75; g2c = 0.125;
      double cn = __ddiv_rn(1.0, __dsub_rn(a2, __dmul_rn(3.0, g2c)));
      up1 = __dmul_rn(__dsub_rn(__dmul_rn(6.0, a2), 3.0), cn);
      up2 = ((iv != 1) && (iv != 2)) ? 0.0 : up1;
      if (iv % 2 == 0) up1 = 0.0;
    } else {
      const double U1[5] = {707.0 / 193.0, 137.0 / 13.0, 707.0 / 193.0, 137.0 / 13.0, 707.0 / 193.0};
      const double U2[5] = {707.0 / 193.0, 137.0 / 13.0, 137.0 / 13.0, 707.0 / 193.0, 707.0 / 193.0};
      alpha = 2.0 / 11.0; a2 = -0.35; g2c = 0.1; up1 = U1[iv]; up2 = U2[iv];
    }
    double c1 = 1.0, c2 = 1.0, c3;
    g1[1] = g2[1] = g3[1] = c2;
    if (lphys) {
      c3 = (order == 1) ? __dmul_rn(up1, c2) : up1;
      g1[2] = c3; c2 = __ddiv_rn(c1, __dsub_rn(c1, __dmul_rn(g2c, c3))); g2[2] = c2;
      c3 = __dmul_rn(a2, c2); g1[3] = c3; c2 = __ddiv_rn(c1, __dsub_rn(c1, __dmul_rn(alpha, c3))); g2[3] = c2;
      g3[2] = __dmul_rn(-g2c, g2[2]);
    } else {
      c3 = __dmul_rn(alpha, c2); g1[2] = c3; c2 = __ddiv_rn(c1, __dsub_rn(c1, __dmul_rn(alpha, c3))); g2[2] = c2;
      g3[2] = __dmul_rn(-alpha, g2[2]);
      c3 = __dmul_rn(alpha, c2); g1[3] = c3; c2 = __ddiv_rn(c1, __dsub_rn(c1, __dmul_rn(alpha, c3))); g2[3] = c2;
    }
    for (int i = 4; i <= n - 2; i++) {
      c3 = __dmul_rn(alpha, c2); g1[i] = c3; c2 = __ddiv_rn(c1, __dsub_rn(c1, __dmul_rn(alpha, c3))); g2[i] = c2;
    }
    for (int i = 3; i <= n - 2; i++) g3[i] = __dmul_rn(-alpha, g2[i]);
    // row n-1 of a physical upper end mirrors row 2: lower coefficient a2,
    // upper coefficient g2c (tab_d1; tab_d2 swaps its two names, same values)
    const double rl = a2, ru = g2c;
    if (rphys) {
      c3 = __dmul_rn(alpha, c2); g1[n - 1] = c3; c2 = __ddiv_rn(c1, __dsub_rn(c1, __dmul_rn(rl, c3))); g2[n - 1] = c2;
      c3 = __dmul_rn(ru, c2); g1[n] = c3; c2 = __ddiv_rn(c1, __dsub_rn(c1, __dmul_rn(up2, c3))); g2[n] = c2;
      g3[n - 1] = __dmul_rn(-rl, g2[n - 1]);
      g3[n] = __dmul_rn(-up2, g2[n]);
    } else {
      c3 = __dmul_rn(alpha, c2); g1[n - 1] = c3; c2 = __ddiv_rn(c1, __dsub_rn(c1, __dmul_rn(alpha, c3))); g2[n - 1] = c2;
      c3 = __dmul_rn(alpha, c2); g1[n] = c3; c2 = __ddiv_rn(c1, __dsub_rn(c1, __dmul_rn(alpha, c3))); g2[n] = c2;
      g3[n - 1] = __dmul_rn(-alpha, g2[n - 1]);
      g3[n] = __dmul_rn(-alpha, g2[n]);
    }
    for (int j = 1; j <= n; j++) g1[j] = -g1[j];
  }
}

extern "C" int css_compact_lines_noalloc(const double *x, double *dx, int n, int nlines, int order, int lphys,
                                         int rphys, int bdry, const double *bc_lo, const double *bc_hi,
                                         const double *halo_lo, const double *halo_hi, double dnum, double scale,
                                         void *stream) {
  if (!x || !dx || n < 10 || order < 1 || order > 2 || bdry < 0 || bdry > 4 || nlines < 0 ||
      (!lphys && !halo_lo) || (!rphys && !halo_hi)) {
    set_err("css_compact_lines_noalloc: bad argument");
    return CSS_ERR_ARG;
  }
  const size_t ts = (size_t)n + 2, need = 15 * ts + (size_t)nlines * ((size_t)n + 8);
  if (need > (size_t)CSS_NOALLOC_DOUBLES) {
    set_err("css_compact_lines_noalloc: %zu doubles of scratch needed, the fixed device array holds %d "
            "(15*(n+2) + nlines*(n+8) must fit); split the lines into smaller batches",
            need, CSS_NOALLOC_DOUBLES);
    return CSS_ERR_ARG;
  }
  // the set-up comes first, so a call with nlines == 0 on each device at
  // start-up does it without launching anything
  double *T = nullptr;
  if (int rc = noalloc_scratch(&T)) return rc;
  if (nlines == 0) return CSS_OK;
  double *work = T + 15 * ts;
  cudaStream_t st = (cudaStream_t)stream;
  k_noalloc_tables<<<1, 1, 0, st>>>(T, n, lphys, rphys, order);
  CUDA_TRY(cudaGetLastError());
  int dtype = lphys ? (rphys ? 0 : 2) : (rphys ? 1 : 3);
  k_lines<<<(nlines + 127) / 128, 128, 0, st>>>(x, dx, n, nlines, order, dtype, bdry, bc_lo, bc_hi, halo_lo, halo_hi,
                                                T, (int)ts, dnum, scale, work);
  CUDA_TRY(cudaGetLastError());
  return CSS_OK;
}

// ---------------------------------------------------------------------------
// Open radial boundaries: clock, mass bookkeeping, rain and ASH inputs
// ---------------------------------------------------------------------------
extern "C" int css_set_clock(css_ctx *c, long long istep, double sim_time, double deltat) {
  if (!c) { set_err("css_set_clock: NULL"); return CSS_ERR_ARG; }
  c->istep = istep;
  c->sim_time = sim_time;
  c->deltat = deltat;
  if (c->io) return ash_refresh(c);
  return CSS_OK;
}

extern "C" int css_get_clock(css_ctx *c, long long *istep, double *sim_time) {
  if (!c) { set_err("css_get_clock: NULL"); return CSS_ERR_ARG; }
  if (istep) *istep = c->istep;
  if (sim_time) *sim_time = c->sim_time;
  return CSS_OK;
}

static int need_open(css_ctx *c, const char *who) {
  if (!c) { set_err("%s: NULL", who); return CSS_ERR_ARG; }
  if (!c->io) { set_err("%s: the run has no open radial boundary (top_inout / bot_inout)", who); return CSS_ERR_ARG; }
  return CSS_OK;
}

// m0 and vol of the resident state (mhdsph_mpi.f90:863-947) and mtot
// (:979-999; for a closed bottom the start-up leaves mtot = m0)
extern "C" int css_inout_init(css_ctx *c) {
  if (int rc = need_open(c, "css_inout_init")) return rc;
  const CssGeo &g = c->g;
  k_plane_mass<<<g.nr, IO_NT, 0, c->stream>>>(g, c->v0, c->io_part);
  k_mass_finish<<<1, 32, 0, c->stream>>>(g, c->io_part, c->io, IO_M0, IO_VOL);
  k_mass_finish<<<1, 32, 0, c->stream>>>(g, c->io_part, c->io, IO_MTOT, -1);
  if (int rc = check_launch(c)) return rc;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CSS_OK;
}

extern "C" int css_inout_state(css_ctx *c, double *out) {
  if (int rc = need_open(c, "css_inout_state")) return rc;
  if (!out) { set_err("css_inout_state: NULL"); return CSS_ERR_ARG; }
  double io[IO_COUNT];
  CUDA_TRY(cudaMemcpyAsync(io, c->io, sizeof io, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  out[0] = io[IO_M0]; out[1] = io[IO_VOL]; out[2] = io[IO_MTOT]; out[3] = io[IO_ASH_FEN_MOD];
  return CSS_OK;
}

extern "C" int css_set_rain_fields(css_ctx *c, const double *dvel_rain, const double *dent_rain) {
  if (int rc = need_open(c, "css_set_rain_fields")) return rc;
  if (!dvel_rain || !dent_rain) { set_err("css_set_rain_fields: NULL"); return CSS_ERR_ARG; }
  const size_t np = (size_t)c->p.nth * c->p.nphi;
  CUDA_TRY(cudaMemcpyAsync(c->rain, dvel_rain, np * 8, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(cudaMemcpyAsync(c->rain + np, dent_rain, np * 8, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CSS_OK;
}

extern "C" int css_get_rain_fields(css_ctx *c, double *dvel_rain, double *dent_rain) {
  if (int rc = need_open(c, "css_get_rain_fields")) return rc;
  if (!dvel_rain || !dent_rain) { set_err("css_get_rain_fields: NULL"); return CSS_ERR_ARG; }
  const size_t np = (size_t)c->p.nth * c->p.nphi;
  CUDA_TRY(cudaMemcpyAsync(dvel_rain, c->rain, np * 8, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaMemcpyAsync(dent_rain, c->rain + np, np * 8, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CSS_OK;
}

// squalls: 6 per squall (theta_loc, phi_loc, size, scaling, vel, dels); the
// grid point of each centre follows Find_Position (entropy_rain.f90:817-824)
static int build_squalls(css_ctx *c, int sstruct, int nsq, const double *squalls, int add);
extern "C" int css_build_squalls(css_ctx *c, int sstruct, int nsq, const double *squalls) {
  if (int rc = need_open(c, "css_build_squalls")) return rc;
  return build_squalls(c, sstruct, nsq, squalls, 0);
}
extern "C" int css_add_squalls(css_ctx *c, int sstruct, int nsq, const double *squalls) {
  if (int rc = need_open(c, "css_add_squalls")) return rc;
  return build_squalls(c, sstruct, nsq, squalls, 1);
}

extern "C" int css_voronoi(int n, const double *x, const double *y, int *degree, int *start, int *face, int *nvert,
                           double *vxy) {
  if (n < 3 || !x || !y || !degree || !start || !face || !nvert || !vxy) {
    set_err("css_voronoi: bad argument (at least 3 sites)");
    return CSS_ERR_ARG;
  }
  std::vector<int> deg, st, fc;
  std::vector<double> v;
  if (vor_cells(n, x, y, deg, st, fc, v)) {
    set_err("css_voronoi: coincident or degenerate sites (no unique Delaunay triangulation)");
    return CSS_ERR_ARG;
  }
  for (int g = 0; g < n; g++) { degree[g] = deg[g]; start[g] = st[g]; }
  std::copy(fc.begin(), fc.end(), face);
  *nvert = (int)(v.size() / 2);
  std::copy(v.begin(), v.end(), vxy);
  return CSS_OK;
}

extern "C" int css_build_lanes(css_ctx *c, int ncells, const double *cells, double meansize, double meanvel,
                               double meands) {
  if (int rc = need_open(c, "css_build_lanes")) return rc;
  if (ncells < 1 || !cells || !(meansize > 0.0)) {
    set_err("css_build_lanes: bad argument (ncells >= 1, cells, meansize > 0)");
    return CSS_ERR_ARG;
  }
  const css_params &p = c->p;
  const double dth = (p.th2 - p.th1) / (double)(p.nth - 1), dphi = (p.phi2 - p.phi1) / (double)p.nphi;
  // the sites and their periodic copies one domain width left and right
  // (Initialize_Rain_Squalls / Update_Rain_Squalls, entropy_rain.f90:80-89, :374-385)
  const int n3 = 3 * ncells;
  std::vector<double> x(n3), y(n3), sc(n3);
  for (int k = 0; k < ncells; k++) {
    const double *q = cells + 3 * k;
    if (!(q[2] >= 0.0)) { set_err("css_build_lanes: cell %d has scaling %g (must be >= 0)", k, q[2]); return CSS_ERR_ARG; }
    for (int cpy = 0; cpy < 3; cpy++) {
      const int i = k + cpy * ncells;
      x[i] = cpy == 0 ? q[0] : cpy == 1 ? q[0] - (p.phi2 - p.phi1) : (p.phi2 - p.phi1) + q[0];
      y[i] = q[1];
      sc[i] = q[2];
    }
  }
  std::vector<int> deg, st, fc;
  std::vector<double> v;
  if (vor_cells(n3, x.data(), y.data(), deg, st, fc, v)) {
    set_err("css_build_lanes: coincident or degenerate cell sites");
    return CSS_ERR_ARG;
  }
  // the points along every cell edge (Build_Downflow_Lanes, entropy_rain.f90:667-703)
  const int nmax = (int)std::sqrt((double)p.nth * p.nth + (double)p.nphi * p.nphi);
  std::vector<double> smp;
  for (int ic = 0; ic < n3; ic++)
    for (int ie = 0; ie < deg[ic]; ie++) {
      const int a = fc[st[ic] + ie], b = fc[st[ic] + (ie + 1 < deg[ic] ? ie + 1 : 0)];
      const double x1 = v[2 * a], y1 = v[2 * a + 1];
      const double dvx = v[2 * b] - x1, dvy = v[2 * b + 1] - y1;
      const double gx = dvx / dphi, gy = dvy / dth;
      const double len = std::sqrt(gx * gx + gy * gy);
      const int my = len >= (double)nmax ? nmax : (int)len;
      for (int k = 0; k < my; k++) {
        const double t = (double)k / (double)my;
        smp.push_back(x1 + dvx * t);
        smp.push_back(y1 + dvy * t);
        smp.push_back(sc[ic]);
      }
    }
  const int ns = (int)(smp.size() / 3);
  const size_t need = smp.size() + 1;
  if (need > c->lane_cap) {
    cudaFree(c->lanes);
    c->lanes = nullptr;
    c->lane_cap = 0;
    CUDA_TRY(cudaMalloc(&c->lanes, need * sizeof(double)));
    c->lane_cap = need;
  }
  unsigned long long *maxbits = reinterpret_cast<unsigned long long *>(c->lanes + smp.size());
  if (ns > 0) CUDA_TRY(cudaMemcpyAsync(c->lanes, smp.data(), smp.size() * 8, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(cudaMemsetAsync(maxbits, 0, 8, c->stream));
  // isz_max (Initialize_Rain_Squalls, entropy_rain.f90:58): the window margin in cells
  double smin = 1.0;
  for (int it = 0; it < p.nth; it++) smin = std::min(smin, std::sin(dth * (double)it + p.th1));
  const int isz = (int)std::ceil(meansize * std::sqrt(-std::log(1e-5)) / (p.r2 * std::min(dth, dphi * smin)));
  const double rtmp = (p.r2 / meansize) * (p.r2 / meansize);
  const size_t np = (size_t)p.nth * p.nphi;
  k_lanes<<<(unsigned)((np + 255) / 256), 256, 0, c->stream>>>(c->g, c->lanes, ns, p.phi1, isz * dphi, isz * dth,
                                                               rtmp, c->rain, maxbits);
  if (int rc = check_launch(c)) return rc;
  k_lanes_scale<<<(unsigned)((np + 255) / 256), 256, 0, c->stream>>>(np, maxbits, meanvel, meands, c->rain,
                                                                     c->rain + np);
  if (int rc = check_launch(c)) return rc;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CSS_OK;
}

static int build_squalls(css_ctx *c, int sstruct, int nsq, const double *squalls, int add) {
  if (nsq < 0 || (nsq > 0 && !squalls) || (sstruct != 0 && sstruct != 1)) {
    set_err("css_build_squalls: bad argument");
    return CSS_ERR_ARG;
  }
  const css_params &p = c->p;
  const double dth = (p.th2 - p.th1) / (double)(p.nth - 1), dphi = (p.phi2 - p.phi1) / (double)p.nphi;
  std::vector<double> sq((size_t)8 * std::max(nsq, 1));
  for (int i = 0; i < nsq; i++) {
    const double *q = squalls + 6 * i;
    if (!(q[2] > 0.0)) { set_err("css_build_squalls: squall %d has size %g", i, q[2]); return CSS_ERR_ARG; }
    for (int k = 0; k < 6; k++) sq[8 * i + k] = q[k];
    const double ft = floor((q[0] - p.th1) / dth) + 1.0, fp = floor((q[1] - p.phi1) / dphi) + 1.0;
    sq[8 * i + 6] = std::max(std::min(ft, (double)p.nth), 1.0);
    sq[8 * i + 7] = std::max(std::min(fp, (double)p.nphi), 1.0);
  }
  if (nsq > c->squall_cap) {
    cudaFree(c->squalls);
    c->squalls = nullptr;
    c->squall_cap = 0;
    CUDA_TRY(cudaMalloc(&c->squalls, (size_t)8 * nsq * sizeof(double)));
    c->squall_cap = nsq;
  }
  if (nsq > 0) CUDA_TRY(cudaMemcpyAsync(c->squalls, sq.data(), (size_t)8 * nsq * 8, cudaMemcpyHostToDevice, c->stream));
  const size_t np = (size_t)p.nth * p.nphi;
  k_squalls<<<(unsigned)((np + 255) / 256), 256, 0, c->stream>>>(c->g, c->squalls, nsq, sstruct == 0, p.phi1, p.phi2,
                                                                    add, c->rain, c->rain + np);
  if (int rc = check_launch(c)) return rc;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CSS_OK;
}

extern "C" int css_set_ash_slices(css_ctx *c, const double *slices, const double *times, double ash_fen_mod) {
  if (int rc = need_open(c, "css_set_ash_slices")) return rc;
  if (!slices || !times) { set_err("css_set_ash_slices: NULL"); return CSS_ERR_ARG; }
  if (!(times[2] > times[1])) { set_err("css_set_ash_slices: times[2] must exceed times[1]"); return CSS_ERR_ARG; }
  const size_t np = (size_t)c->p.nth * c->p.nphi;
  CUDA_TRY(cudaMemcpyAsync(c->ash_slices, slices, 16 * np * 8, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(cudaMemcpyAsync(c->io + IO_ASH_FEN_MOD, &ash_fen_mod, 8, cudaMemcpyHostToDevice, c->stream));
  for (int k = 0; k < 4; k++) c->ash_times[k] = times[k];
  if (int rc = ash_refresh(c)) return rc;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CSS_OK;
}
