// css_closure.cuh -- the learned subgrid closure: box filtering of a fine
// state into coarse fields and subgrid targets, the 3x3x3 stencil features,
// and the elementwise parts of the MLP (bias + GELU and its derivative,
// loss, bias gradients, Adam), and k_gemm_bf16: the MLP's matrix products
// for training and the per-layer forward pass, BF16 operands with FP32
// accumulation on the tensor cores (mma.sync m16n8k16), issued from
// css_api.cu.
#pragma once
#include <cuda_bf16.h>

#include "css_geo.cuh"

namespace css {

#define CL_NFIELD 7    // coarse fields: u_theta, u_phi, u_r, s', B_theta, B_phi, B_r
#define CL_NTARGET 12  // tau_tt tau_tp tau_tr tau_pp tau_pr tau_rr, q_t q_p q_r, emf_t emf_p emf_r
#define CL_NQ 5        // stencil quantities: u_theta, u_phi, u_r, |B|, ds'/dr
#define CL_NFEAT 135   // 27 stencil points x 5 quantities
#define CL_XPAD 144    // feature row length (zero padded to a multiple of 16)
#define CL_YPAD 16     // output row length (12 targets, zero padded)

// Box filter by the factor f in every direction: coarse cell (it, ip, ir)
// averages the f^3 fine cells f*it.., f*ip.., f*ir...  fields[k*nc + c],
// targets[k*nc + c]; c = it + nct*(ip + ncp*ir).  s' = s - sr(r); B from bf
// (NULL for hydro: B and the EMF are zero).
__global__ void k_box_filter(CssGeo g, const double *__restrict__ v, const double *__restrict__ bf, int f, int nct,
                             int ncp, int ncr, double *__restrict__ fields, double *__restrict__ targets) {
  const size_t nc = (size_t)nct * ncp * ncr, n = (size_t)g.ncell;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
    const int it = (int)(c % nct), ip = (int)((c / nct) % ncp), ir = (int)(c / ((size_t)nct * ncp));
    double m[19];
#pragma unroll
    for (int k = 0; k < 19; k++) m[k] = 0.0;
    for (int dr = 0; dr < f; dr++) {
      const int fr = f * ir + dr;
      const double sbar = g.sr[fr];
      for (int dp = 0; dp < f; dp++)
        for (int dt = 0; dt < f; dt++) {
          const size_t id = css_idx(g, f * it + dt, f * ip + dp, fr);
          const double ut = v[n + id], up = v[2 * n + id], ur = v[3 * n + id], sp = v[4 * n + id] - sbar;
          double bt = 0.0, bp = 0.0, br = 0.0;
          if (bf) { bt = bf[id]; bp = bf[n + id]; br = bf[2 * n + id]; }
          m[0] += ut; m[1] += up; m[2] += ur; m[3] += sp; m[4] += bt; m[5] += bp; m[6] += br;
          m[7] += ut * ut; m[8] += ut * up; m[9] += ut * ur; m[10] += up * up; m[11] += up * ur; m[12] += ur * ur;
          m[13] += ut * sp; m[14] += up * sp; m[15] += ur * sp;
          m[16] += up * br - ur * bp; m[17] += ur * bt - ut * br; m[18] += ut * bp - up * bt;
        }
    }
    const double w = 1.0 / ((double)f * f * f);
#pragma unroll
    for (int k = 0; k < 19; k++) m[k] *= w;
    const double ut = m[0], up = m[1], ur = m[2], sp = m[3], bt = m[4], bp = m[5], br = m[6];
#pragma unroll
    for (int k = 0; k < CL_NFIELD; k++) fields[k * nc + c] = m[k];
    targets[0 * nc + c] = m[7] - ut * ut;
    targets[1 * nc + c] = m[8] - ut * up;
    targets[2 * nc + c] = m[9] - ut * ur;
    targets[3 * nc + c] = m[10] - up * up;
    targets[4 * nc + c] = m[11] - up * ur;
    targets[5 * nc + c] = m[12] - ur * ur;
    targets[6 * nc + c] = m[13] - ut * sp;
    targets[7 * nc + c] = m[14] - up * sp;
    targets[8 * nc + c] = m[15] - ur * sp;
    targets[9 * nc + c] = m[16] - (up * br - ur * bp);
    targets[10 * nc + c] = m[17] - (ur * bt - ut * br);
    targets[11 * nc + c] = m[18] - (ut * bp - up * bt);
  }
}

// the five stencil quantities of coarse cell (it, ip, ir)
__device__ __forceinline__ void cl_quantities(const double *__restrict__ F, int nct, int ncp, int ncr, int it, int ip,
                                              int ir, double q[CL_NQ]) {
  const size_t nc = (size_t)nct * ncp * ncr;
  const size_t c = it + (size_t)nct * (ip + (size_t)ncp * ir);
  q[0] = F[c];
  q[1] = F[nc + c];
  q[2] = F[2 * nc + c];
  const double bt = F[4 * nc + c], bp = F[5 * nc + c], br = F[6 * nc + c];
  q[3] = sqrt(bt * bt + bp * bp + br * br);
  // ds'/dr in coarse index units: central inside, one-sided at the ends
  const int lo = ir > 0 ? ir - 1 : ir, hi = ir < ncr - 1 ? ir + 1 : ir;
  const size_t cl = it + (size_t)nct * (ip + (size_t)ncp * lo), ch = it + (size_t)nct * (ip + (size_t)ncp * hi);
  q[4] = (F[3 * nc + ch] - F[3 * nc + cl]) / (double)(hi - lo);
}

// features: row c of X (CL_XPAD bf16) = the 27 neighbours (r, theta clamped
// at the ends, phi periodic; order (dr, dt, dp) with dp fastest) x the five
// quantities divided by scale[q], then zeros
__global__ void k_closure_features(const double *__restrict__ F, int nct, int ncp, int ncr,
                                   const float *__restrict__ scale, __nv_bfloat16 *__restrict__ X) {
  const size_t nc = (size_t)nct * ncp * ncr;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
    const int it = (int)(c % nct), ip = (int)((c / nct) % ncp), ir = (int)(c / ((size_t)nct * ncp));
    __nv_bfloat16 *row = X + c * CL_XPAD;
    int col = 0;
    for (int dr = -1; dr <= 1; dr++)
      for (int dt = -1; dt <= 1; dt++)
        for (int dp = -1; dp <= 1; dp++) {
          const int jr = min(max(ir + dr, 0), ncr - 1), jt = min(max(it + dt, 0), nct - 1);
          const int jp = (ip + dp + ncp) % ncp;
          double q[CL_NQ];
          cl_quantities(F, nct, ncp, ncr, jt, jp, jr, q);
#pragma unroll
          for (int k = 0; k < CL_NQ; k++) row[col++] = __float2bfloat16_rn((float)(q[k] / (double)scale[k]));
        }
    for (; col < CL_XPAD; col++) row[col] = __float2bfloat16_rn(0.0f);
  }
}

// root mean square of the five stencil quantities and of the twelve targets:
// part[(blk)*17 + k] partial sums of squares (grid-stride, one block row each)
__global__ void k_closure_sumsq(const double *__restrict__ F, const double *__restrict__ T, int nct, int ncp, int ncr,
                                double *__restrict__ part) {
  __shared__ double red[256];
  const size_t nc = (size_t)nct * ncp * ncr;
  double acc[CL_NQ + CL_NTARGET];
#pragma unroll
  for (int k = 0; k < CL_NQ + CL_NTARGET; k++) acc[k] = 0.0;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
    const int it = (int)(c % nct), ip = (int)((c / nct) % ncp), ir = (int)(c / ((size_t)nct * ncp));
    double q[CL_NQ];
    cl_quantities(F, nct, ncp, ncr, it, ip, ir, q);
#pragma unroll
    for (int k = 0; k < CL_NQ; k++) acc[k] += q[k] * q[k];
    if (T)
#pragma unroll
      for (int k = 0; k < CL_NTARGET; k++) acc[CL_NQ + k] += T[k * nc + c] * T[k * nc + c];
  }
  for (int k = 0; k < CL_NQ + CL_NTARGET; k++) {
    red[threadIdx.x] = acc[k];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) part[(size_t)blockIdx.x * (CL_NQ + CL_NTARGET) + k] = red[0];
    __syncthreads();
  }
}

// training targets: Tn[c*CL_YPAD + k] = T[k*nc + c] / tscale[k] (FP32), pad zero
__global__ void k_closure_targets(const double *__restrict__ T, size_t nc, const float *__restrict__ tscale,
                                  float *__restrict__ Tn) {
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x)
    for (int k = 0; k < CL_YPAD; k++)
      Tn[c * CL_YPAD + k] = k < CL_NTARGET ? (float)(T[k * nc + c] / (double)tscale[k]) : 0.0f;
}

// GELU in its tanh form (Hendrycks & Gimpel): 0.5 x (1 + tanh(u)),
// u = sqrt(2/pi) (x + 0.044715 x^3), with the hardware tanh approximation
// (relative error about 2^-11, below the BF16 rounding of the activations);
// the derivative is 0.5 (1 + t) + 0.5 x (1 - t^2) du/dx
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu_f(float x) {
  const float u = 0.7978845608028654f * fmaf(0.044715f * x, x * x, x);
  return 0.5f * x * (1.0f + tanh_hw(u));
}
// Packed FP32x2 arithmetic (add/mul/fma .f32x2, sm_100): two lanes per
// instruction, each rounded as its scalar form.
typedef unsigned long long f32x2_t;
__device__ __forceinline__ f32x2_t f2_pack(float a, float b) {
  f32x2_t r;
  asm("mov.b64 %0, {%1,%2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void f2_unpack(f32x2_t v, float &a, float &b) {
  asm("mov.b64 {%0,%1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ f32x2_t f2_add(f32x2_t a, f32x2_t b) {
  f32x2_t r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f32x2_t f2_mul(f32x2_t a, f32x2_t b) {
  f32x2_t r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f32x2_t f2_fma(f32x2_t a, f32x2_t b, f32x2_t c) {
  f32x2_t r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
// gelu_f of (z + bias) for two values, the same operations in the same
// order (so the same roundings) in packed arithmetic, rounded to BF16x2
__device__ __forceinline__ uint32_t gelu2_bf16(f32x2_t z, f32x2_t bias) {
  const f32x2_t x = f2_add(z, bias);
  const f32x2_t u = f2_mul(f2_pack(0.7978845608028654f, 0.7978845608028654f),
                           f2_fma(f2_mul(f2_pack(0.044715f, 0.044715f), x), f2_mul(x, x), x));
  float u0, u1;
  f2_unpack(u, u0, u1);
  const f32x2_t t = f2_add(f2_pack(1.0f, 1.0f), f2_pack(tanh_hw(u0), tanh_hw(u1)));
  float g0, g1;
  f2_unpack(f2_mul(f2_mul(f2_pack(0.5f, 0.5f), x), t), g0, g1);
  const __nv_bfloat162 h = __floats2bfloat162_rn(g0, g1);
  return *reinterpret_cast<const uint32_t *>(&h);
}
__device__ __forceinline__ float gelu_df(float x) {
  const float u = 0.7978845608028654f * fmaf(0.044715f * x, x * x, x);
  const float t = tanh_hw(u);
  const float du = 0.7978845608028654f * fmaf(3.0f * 0.044715f, x * x, 1.0f);
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * du;
}

// Z (col-major M x n: Z[r*M + j]) += b[j]; H = bf16(GELU(Z)) when H != NULL
__global__ void k_bias_gelu(float *__restrict__ Z, const float *__restrict__ b, __nv_bfloat16 *__restrict__ H,
                            int M, size_t n) {
  const size_t tot = (size_t)M * n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < tot; i += (size_t)gridDim.x * blockDim.x) {
    const float z = Z[i] + b[i % M];
    Z[i] = z;
    if (H) H[i] = __float2bfloat16_rn(gelu_f(z));
  }
}

// loss and output gradient: D = Y - T over the first nreal of CL_YPAD
// columns; dY = 2 D / (n nreal) (FP32 and BF16), pad columns zero;
// part[block] = partial sum of D^2
__global__ void k_mse(const float *__restrict__ Y, const float *__restrict__ T, size_t n, int nreal,
                      float *__restrict__ dY, __nv_bfloat16 *__restrict__ dYb, double *__restrict__ part) {
  __shared__ double red[256];
  const size_t tot = n * CL_YPAD;
  const float sc = 2.0f / ((float)n * (float)nreal);
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < tot; i += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(i % CL_YPAD);
    float d = 0.0f;
    if (k < nreal) {
      d = Y[i] - T[i];
      acc += (double)d * d;
    }
    dY[i] = sc * d;
    dYb[i] = __float2bfloat16_rn(sc * d);
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// back through GELU: dZ = dH * GELU'(Z) (FP32 in place of dH, and BF16)
__global__ void k_gelu_back(float *__restrict__ dH, const float *__restrict__ Z, __nv_bfloat16 *__restrict__ dZb,
                            size_t tot) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < tot; i += (size_t)gridDim.x * blockDim.x) {
    const float d = dH[i] * gelu_df(Z[i]);
    dH[i] = d;
    dZb[i] = __float2bfloat16_rn(d);
  }
}

// bias gradient: db[j] = sum over the n rows of dZ[r*M + j]; grid = M
// blocks, each sums its column in a fixed order (deterministic)
__global__ void k_colsum(const float *__restrict__ dZ, int M, size_t n, float *__restrict__ db) {
  __shared__ double red[256];
  const int j = blockIdx.x;
  double acc = 0.0;
  for (size_t r = threadIdx.x; r < n; r += blockDim.x) acc += dZ[r * M + j];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[j] = (float)red[0];
}

// Adam (bias-corrected) on FP32 master parameters, refreshing the BF16 copy
__global__ void k_adam(float *__restrict__ w, const float *__restrict__ gr, float *__restrict__ m,
                       float *__restrict__ v2, __nv_bfloat16 *__restrict__ wb, size_t cnt, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cnt; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = gr[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v2[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v2[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
  }
}

// Fine -> coarse restriction of the whole state (the evaluation of a coarse
// run starts from the filtered fine state): vc[iv][c] = base_c[iv][c] + the
// f x f x f box average of vf - base_f over the fine cells of coarse cell c,
// summed in (r, phi, theta) order (a NULL base is zero).  The perturbation
// about each grid's own background is what is filtered, so the coarse
// state stays in its own grid's hydrostatic balance.  Layout
// [iv][r][phi][theta] on both grids.
__global__ void k_restrict_state(const double *__restrict__ vf, const double *__restrict__ base_f, int nthf,
                                 int nphif, int nrf, int f, int nv, const double *__restrict__ base_c,
                                 double *__restrict__ vc) {
  const int nct = nthf / f, ncp = nphif / f, ncr = nrf / f;
  const size_t nc = (size_t)nct * ncp * ncr, nf = (size_t)nthf * nphif * nrf;
  const double w = 1.0 / ((double)f * f * f);
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nc * nv; k += (size_t)gridDim.x * blockDim.x) {
    const int iv = (int)(k / nc);
    const size_t c = k - (size_t)iv * nc;
    const int it = (int)(c % nct), ip = (int)((c / nct) % ncp), ir = (int)(c / ((size_t)nct * ncp));
    double s = 0.0;
    for (int dr = 0; dr < f; dr++)
      for (int dp = 0; dp < f; dp++) {
        const size_t row = (size_t)iv * nf + (size_t)(f * it) +
                           (size_t)nthf * ((size_t)(f * ip + dp) + (size_t)nphif * (f * ir + dr));
        for (int dt = 0; dt < f; dt++) s += base_f ? vf[row + dt] - base_f[row + dt] : vf[row + dt];
      }
    vc[k] = (base_c ? base_c[k] : 0.0) + s * w;
  }
}

// linear interpolation weights of fine index i from a grid f times coarser
// (cell-centred: fine i sits at coarse coordinate (i + 0.5) / f - 0.5);
// clamped at the ends, or periodic
__device__ __forceinline__ void prolong_w(int i, int f, int nc, bool periodic, int &i0, int &i1, double &w) {
  const double x = (i + 0.5) / f - 0.5;
  int j = (int)floor(x);
  w = x - j;
  if (periodic) {
    i0 = (j % nc + nc) % nc;
    i1 = (i0 + 1) % nc;
  } else if (j < 0) {
    i0 = i1 = 0;
    w = 0.0;
  } else if (j >= nc - 1) {
    i0 = i1 = nc - 1;
    w = 0.0;
  } else {
    i0 = j;
    i1 = j + 1;
  }
}

// Coarse -> fine: vf += P(vc - base), P trilinear in index space (theta and
// r clamped, phi periodic); base NULL means zero.  A state developed on the
// coarse grid is carried to the fine grid as a perturbation of the fine
// grid's own state.
__global__ void k_prolong_add(const double *__restrict__ vc, const double *__restrict__ base, int nct, int ncp,
                              int ncr, int f, int nv, double *__restrict__ vf) {
  const int nthf = nct * f, nphif = ncp * f, nrf = ncr * f;
  const size_t nf = (size_t)nthf * nphif * nrf, nc = (size_t)nct * ncp * ncr;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nf * nv; k += (size_t)gridDim.x * blockDim.x) {
    const int iv = (int)(k / nf);
    const size_t id = k - (size_t)iv * nf;
    const int it = (int)(id % nthf), ip = (int)((id / nthf) % nphif), ir = (int)(id / ((size_t)nthf * nphif));
    int t0, t1, p0, p1, r0, r1;
    double wt, wp, wr;
    prolong_w(it, f, nct, false, t0, t1, wt);
    prolong_w(ip, f, ncp, true, p0, p1, wp);
    prolong_w(ir, f, ncr, false, r0, r1, wr);
    const double *c = vc + (size_t)iv * nc;
    const double *b = base ? base + (size_t)iv * nc : nullptr;
    auto at = [&](int t, int p, int r) {
      const size_t q = (size_t)t + (size_t)nct * ((size_t)p + (size_t)ncp * r);
      return b ? c[q] - b[q] : c[q];
    };
    const double v00 = (1.0 - wt) * at(t0, p0, r0) + wt * at(t1, p0, r0);
    const double v10 = (1.0 - wt) * at(t0, p1, r0) + wt * at(t1, p1, r0);
    const double v01 = (1.0 - wt) * at(t0, p0, r1) + wt * at(t1, p0, r1);
    const double v11 = (1.0 - wt) * at(t0, p1, r1) + wt * at(t1, p1, r1);
    vf[k] += (1.0 - wr) * ((1.0 - wp) * v00 + wp * v10) + wr * ((1.0 - wp) * v01 + wp * v11);
  }
}

// closure -> SLD speed^2 shaped by the prescribed profile: the predicted
// subgrid variance k = tau_tt + tau_pp + tau_rr of each cell, divided by its
// shell mean and multiplied by the prescribed speed^2 of that radius, so a
// shell keeps the prescribed mean diffusion speed^2 and the network moves it
// to where the subgrid motions are.  One CTA per radius; the shell sum is a
// fixed-order block reduction.  -1 (the prescribed profile) where the output
// is not finite or the shell mean is not positive.
__global__ void __launch_bounds__(256) k_closure_speed2_shaped(CssGeo g, const float *__restrict__ Y,
                                                               const float *__restrict__ tscale,
                                                               double *__restrict__ speed2) {
  __shared__ double red[2][8];
  const int ir = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const size_t np = (size_t)g.nth * g.nphi, c0 = (size_t)ir * np;
  double sum = 0.0, cnt = 0.0;
  for (size_t q = threadIdx.x; q < np; q += blockDim.x) {
    const float *y = Y + (c0 + q) * CL_YPAD;
    const double tr = (double)y[0] * tscale[0] + (double)y[3] * tscale[3] + (double)y[5] * tscale[5];
    if (isfinite(tr)) { sum += fmax(tr, 0.0); cnt += 1.0; }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sum += __shfl_down_sync(0xffffffffu, sum, o);
    cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  }
  if (lane == 0) { red[0][warp] = sum; red[1][warp] = cnt; }
  __syncthreads();
  double tot = 0.0, n = 0.0;
  for (int w = 0; w < 8; w++) { tot += red[0][w]; n += red[1][w]; }
  const double mean = n > 0.0 ? tot / n : 0.0;
  const double prof = g.dspeed[ir];
  for (size_t q = threadIdx.x; q < np; q += blockDim.x) {
    const float *y = Y + (c0 + q) * CL_YPAD;
    const double tr = (double)y[0] * tscale[0] + (double)y[3] * tscale[3] + (double)y[5] * tscale[5];
    speed2[c0 + q] = (isfinite(tr) && mean > 0.0) ? prof * fmax(tr, 0.0) / mean : -1.0;
  }
}

// closure -> SLD speed^2 of each coarse cell: the subgrid velocity variance
// tau_tt + tau_pp + tau_rr (network outputs times their target scales),
// floored at zero; -1 (the prescribed profile is used) where the output is
// not finite
__global__ void k_closure_speed2(const float *__restrict__ Y, size_t nc, const float *__restrict__ tscale,
                                 double *__restrict__ speed2) {
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
    const float *y = Y + c * CL_YPAD;
    const double tr = (double)y[0] * tscale[0] + (double)y[3] * tscale[3] + (double)y[5] * tscale[5];
    speed2[c] = isfinite(tr) ? fmax(tr, 0.0) : -1.0;
  }
}

}  // namespace css

namespace css {

// ---------------------------------------------------------------------------
// Fused forward pass of the closure network (in 144 -> 128 -> 128 -> 128 ->
// 16, GELU after the hidden layers).  A persistent CTA of 8 warps copies the
// BF16 weights (stored transposed, n-major with k contiguous and rows padded
// by 8 so fragment loads hit distinct banks) and the FP32 biases into shared
// memory once; each warp then takes 16 rows at a time: the feature rows are
// staged in shared memory by asynchronous 16-byte copies, the four layers
// run as BF16 tensor-core MMAs (m16n8k16, FP32 accumulate), and each
// layer's accumulator fragments, after bias and GELU, are rounded to BF16
// and reused in registers as the next layer's A fragments.  Only the
// features are read and only the outputs written.
// ---------------------------------------------------------------------------
#define FM_IN 144
#define FM_W 128
#define FM_OUT 16
#define FM_KP0 (FM_IN + 8)   // padded row of the first layer's transposed weights
#define FM_KP (FM_W + 8)     // padded row of the other layers
#define FM_XS (FM_IN + 8)    // padded feature row in shared memory
#define FM_WARPS 8
// packed parameter block (bytes): W0t | W1t | W2t | W3t | b0 b1 b2 b3 (FP32)
#define FM_OFF_W1 (FM_W * FM_KP0 * 2)
#define FM_OFF_W2 (FM_OFF_W1 + FM_W * FM_KP * 2)
#define FM_OFF_W3 (FM_OFF_W2 + FM_W * FM_KP * 2)
#define FM_OFF_B (FM_OFF_W3 + FM_OUT * FM_KP * 2)
#define FM_PARAM_BYTES (FM_OFF_B + (3 * FM_W + FM_OUT) * 4)
#define FM_SMEM_BYTES (FM_PARAM_BYTES + FM_WARPS * 16 * FM_XS * 2)

// dst[n*KP + k] = W[k*M + n] (k < K), zero in the padding
__global__ void k_pack_wt(const __nv_bfloat16 *__restrict__ W, int K, int M, int KP, __nv_bfloat16 *__restrict__ dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M * KP; i += gridDim.x * blockDim.x) {
    const int nn = i / KP, k = i - nn * KP;
    dst[i] = k < K ? W[(size_t)k * M + nn] : __float2bfloat16_rn(0.0f);
  }
}

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ unsigned pack_bf16x2(float lo, float hi) {
  __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<unsigned *>(&h);
}

// one hidden layer: acc (16 n-tiles of 8 columns) = A (KSTEPS k-steps) x Wt
template <int KSTEPS, int KPAD>
__device__ __forceinline__ void fm_layer(const unsigned (&a)[KSTEPS][4], const __nv_bfloat16 *__restrict__ Wt,
                                         int g, int t, float (&acc)[16][4]) {
#pragma unroll
  for (int nt = 0; nt < 16; nt++)
#pragma unroll
    for (int q = 0; q < 4; q++) acc[nt][q] = 0.0f;
#pragma unroll
  for (int j = 0; j < KSTEPS; j++)
#pragma unroll
    for (int nt = 0; nt < 16; nt++) {
      const __nv_bfloat16 *wr = Wt + (size_t)(nt * 8 + g) * KPAD + 16 * j + 2 * t;
      const unsigned b0 = *reinterpret_cast<const unsigned *>(wr);
      const unsigned b1 = *reinterpret_cast<const unsigned *>(wr + 8);
      mma_bf16_16816(acc[nt], a[j], b0, b1);
    }
}

// bias + GELU on the accumulators, rounded to BF16 A fragments of the next layer
__device__ __forceinline__ void fm_activate(const float (&acc)[16][4], const float *__restrict__ b, int t,
                                            unsigned (&a)[8][4]) {
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const int c0 = 16 * j + 2 * t, c1 = c0 + 8;
    const float *lo = acc[2 * j], *hi = acc[2 * j + 1];
    a[j][0] = pack_bf16x2(gelu_f(lo[0] + b[c0]), gelu_f(lo[1] + b[c0 + 1]));
    a[j][1] = pack_bf16x2(gelu_f(lo[2] + b[c0]), gelu_f(lo[3] + b[c0 + 1]));
    a[j][2] = pack_bf16x2(gelu_f(hi[0] + b[c1]), gelu_f(hi[1] + b[c1 + 1]));
    a[j][3] = pack_bf16x2(gelu_f(hi[2] + b[c1]), gelu_f(hi[3] + b[c1 + 1]));
  }
}

__global__ void __launch_bounds__(FM_WARPS * 32, 1) k_mlp_fused(const __nv_bfloat16 *__restrict__ X, long long n,
                                                               const unsigned char *__restrict__ params,
                                                               float *__restrict__ Y) {
  extern __shared__ __align__(16) unsigned char fm_sm[];
  // parameters -> shared memory (16-byte words; FM_PARAM_BYTES is a multiple of 16)
  for (int i = threadIdx.x; i < FM_PARAM_BYTES / 16; i += blockDim.x)
    reinterpret_cast<uint4 *>(fm_sm)[i] = reinterpret_cast<const uint4 *>(params)[i];
  __syncthreads();
  const __nv_bfloat16 *W0 = reinterpret_cast<const __nv_bfloat16 *>(fm_sm);
  const __nv_bfloat16 *W1 = reinterpret_cast<const __nv_bfloat16 *>(fm_sm + FM_OFF_W1);
  const __nv_bfloat16 *W2 = reinterpret_cast<const __nv_bfloat16 *>(fm_sm + FM_OFF_W2);
  const __nv_bfloat16 *W3 = reinterpret_cast<const __nv_bfloat16 *>(fm_sm + FM_OFF_W3);
  const float *bias = reinterpret_cast<const float *>(fm_sm + FM_OFF_B);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  __nv_bfloat16 *Xs = reinterpret_cast<__nv_bfloat16 *>(fm_sm + FM_PARAM_BYTES) + (size_t)warp * 16 * FM_XS;
  const long long ntiles = (n + 15) / 16;
  for (long long tile = (long long)blockIdx.x * FM_WARPS + warp; tile < ntiles;
       tile += (long long)gridDim.x * FM_WARPS) {
    const long long r0 = tile * 16;
    // stage 16 feature rows (18 x 16 bytes each); rows past n are zero
    for (int k = lane; k < 16 * (FM_IN / 8); k += 32) {
      const int row = k / (FM_IN / 8), ch = k - row * (FM_IN / 8);
      const bool in = r0 + row < n;
      const __nv_bfloat16 *src = in ? X + (size_t)(r0 + row) * FM_IN + ch * 8 : X;
      cp_async16(Xs + row * FM_XS + ch * 8, src, in ? 16 : 0);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncwarp();
    unsigned a0[FM_IN / 16][4];
#pragma unroll
    for (int j = 0; j < FM_IN / 16; j++) {
      a0[j][0] = *reinterpret_cast<const unsigned *>(Xs + g * FM_XS + 16 * j + 2 * t);
      a0[j][1] = *reinterpret_cast<const unsigned *>(Xs + (g + 8) * FM_XS + 16 * j + 2 * t);
      a0[j][2] = *reinterpret_cast<const unsigned *>(Xs + g * FM_XS + 16 * j + 8 + 2 * t);
      a0[j][3] = *reinterpret_cast<const unsigned *>(Xs + (g + 8) * FM_XS + 16 * j + 8 + 2 * t);
    }
    __syncwarp();  // the staging buffer is free for the next tile
    float acc[16][4];
    unsigned a[8][4];
    fm_layer<FM_IN / 16, FM_KP0>(a0, W0, g, t, acc);
    fm_activate(acc, bias, t, a);
    fm_layer<8, FM_KP>(a, W1, g, t, acc);
    fm_activate(acc, bias + FM_W, t, a);
    fm_layer<8, FM_KP>(a, W2, g, t, acc);
    fm_activate(acc, bias + 2 * FM_W, t, a);
    // output layer: 2 n-tiles
    float out[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll
    for (int j = 0; j < 8; j++)
#pragma unroll
      for (int nt = 0; nt < 2; nt++) {
        const __nv_bfloat16 *wr = W3 + (size_t)(nt * 8 + g) * FM_KP + 16 * j + 2 * t;
        mma_bf16_16816(out[nt], a[j], *reinterpret_cast<const unsigned *>(wr),
                       *reinterpret_cast<const unsigned *>(wr + 8));
      }
    const float *b3 = bias + 3 * FM_W;
#pragma unroll
    for (int nt = 0; nt < 2; nt++) {
      const int c = nt * 8 + 2 * t;
      if (r0 + g < n)
        *reinterpret_cast<float2 *>(Y + (size_t)(r0 + g) * FM_OUT + c) =
            make_float2(out[nt][0] + b3[c], out[nt][1] + b3[c + 1]);
      if (r0 + g + 8 < n)
        *reinterpret_cast<float2 *>(Y + (size_t)(r0 + g + 8) * FM_OUT + c) =
            make_float2(out[nt][2] + b3[c], out[nt][3] + b3[c + 1]);
    }
  }
}

// ---------------------------------------------------------------------------
// The fused forward pass on the 5th-generation tensor cores (tcgen05): a
// persistent CTA per SM keeps all four layers' BF16 weights in shared memory
// in the UMMA K-major core-matrix layout (8 rows x 16 bytes per core matrix:
// the canonical no-swizzle layout; leading byte offset = the distance
// between the two K halves of one K=16 step, stride byte offset = 128
// between 8-row groups).  Its three warpgroups each take 128-row tiles in
// turn, with a shared-memory slot, 128 tensor-memory columns and an
// mbarrier of their own, so one group's products run on the tensor core
// while the other applies its activations:
//   features -> the slot (16-byte copies, the same layout) -> one thread
//   issues the layer's tcgen05.mma (M 128, N 128 or 16, K 16 each; BF16 x
//   BF16 -> FP32 accumulators in tensor memory) and commits them to the
//   mbarrier -> each thread reads its row's accumulators (tcgen05.ld), adds
//   the bias, applies GELU, rounds to BF16 and writes the next layer's A
//   operand into the slot (the features are consumed by then).
// Waits are bounded: a group whose products never complete sets `flag` and
// stops; the tensor memory is released before the CTA exits.
// ---------------------------------------------------------------------------
#define TC_ROWS 128
#define TC_GROUPS 3               // warpgroups, each with its own tile, slot, accumulator and mbarrier
#define TC_NT (128 * TC_GROUPS)
// shared layout (bytes): W0 (128 x 144) | W1 | W2 (128 x 128) | W3 (16 x 128) | a slot per group (128 x 144
// each) | biases (FP32) | an mbarrier per group | tensor-memory address
#define TC_OFF_W1 (FM_W * FM_IN * 2)
#define TC_OFF_W2 (TC_OFF_W1 + FM_W * FM_W * 2)
#define TC_OFF_W3 (TC_OFF_W2 + FM_W * FM_W * 2)
#define TC_OFF_S (TC_OFF_W3 + FM_OUT * FM_W * 2)
#define TC_SLOT (TC_ROWS * FM_IN * 2)
#define TC_OFF_B (TC_OFF_S + TC_GROUPS * TC_SLOT)
#define TC_OFF_BAR (TC_OFF_B + (3 * FM_W + FM_OUT) * 4)
#define TC_SMEM_BYTES (TC_OFF_BAR + 8 * TC_GROUPS + 8)

// byte offset of element (row r, k) of an R-row K-major operand tile in the
// core-matrix layout: core matrix (k/8, r/8) at ((k/8) * R/8 + r/8) * 128
__host__ __device__ __forceinline__ unsigned tc_off(int r, int k, int R) {
  return (unsigned)(((k >> 3) * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// UMMA shared-memory descriptor: no swizzle, version 1 (sm_100)
__device__ __forceinline__ uint64_t tc_desc(unsigned saddr, unsigned lbo, unsigned sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // version
  return d;               // base offset 0, layout type 0 (no swizzle)
}
// instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 D
__host__ __device__ constexpr uint32_t tc_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, int acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   (unsigned)__cvta_generic_to_shared(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_proxy() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// 16 FP32 accumulator columns of this thread's lane (no wait)
__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tc_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }
__device__ __forceinline__ bool tc_wait(uint64_t *bar, unsigned parity) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  const long long t0 = clock64();
  for (;;) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > 4000000000ll) return false;
  }
}
// barrier of one warpgroup (named barrier 1 + group, 128 threads)
__device__ __forceinline__ void tc_group_sync(int grp) {
  asm volatile("bar.sync %0, 128;\n" ::"r"(1 + grp) : "memory");
}
// the same barrier, returning whether any of the group's threads passed pred
__device__ __forceinline__ bool tc_group_any(int grp, bool pred) {
  unsigned r;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 q, %1, 0;\n barrier.red.or.pred p, %2, 128, q;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(r)
      : "r"((unsigned)pred), "r"(1 + grp)
      : "memory");
  return r != 0;
}

// a group stages a 128-row feature tile (rows past n zero) into its slot
__device__ __forceinline__ void tc_stage_x(const __nv_bfloat16 *__restrict__ X, long long n, long long r0,
                                           unsigned char *xs, int gt) {
  for (int k = gt; k < TC_ROWS * (FM_IN / 8); k += 128) {
    const int r = k / (FM_IN / 8), kc = k - r * (FM_IN / 8);
    const bool in = r0 + r < n;
    const __nv_bfloat16 *src = in ? X + (size_t)(r0 + r) * FM_IN + kc * 8 : X;
    cp_async16(xs + tc_off(r, kc * 8, TC_ROWS), src, in ? 16 : 0);
  }
  cp_async_commit();
}

__global__ void __launch_bounds__(TC_NT, 1) k_mlp_tc(const __nv_bfloat16 *__restrict__ X, long long n,
                                                    const unsigned char *__restrict__ params, float *__restrict__ Y,
                                                    int *flag) {
  extern __shared__ __align__(128) unsigned char tc_sm[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int grp = warp >> 2, gt = tid & 127;  // warpgroup and its thread
  uint64_t *bars = reinterpret_cast<uint64_t *>(tc_sm + TC_OFF_BAR);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(tc_sm + TC_OFF_BAR + 8 * TC_GROUPS);
  // weights: packed rows (transposed, k contiguous, padded) -> core-matrix layout
  {
    const int Kl[4] = {FM_IN, FM_W, FM_W, FM_W}, Nl[4] = {FM_W, FM_W, FM_W, FM_OUT};
    const int KPl[4] = {FM_KP0, FM_KP, FM_KP, FM_KP};
    const size_t srco[4] = {0, FM_OFF_W1, FM_OFF_W2, FM_OFF_W3};
    const unsigned dsto[4] = {0, TC_OFF_W1, TC_OFF_W2, TC_OFF_W3};
#pragma unroll
    for (int l = 0; l < 4; l++) {
      const int nch = Kl[l] / 8;
      for (int k = tid; k < Nl[l] * nch; k += TC_NT) {
        const int r = k / nch, kc = k - r * nch;
        *reinterpret_cast<uint4 *>(tc_sm + dsto[l] + tc_off(r, kc * 8, Nl[l])) =
            __ldg(reinterpret_cast<const uint4 *>(params + srco[l] + ((size_t)r * KPl[l] + kc * 8) * 2));
      }
    }
    for (int k = tid; k < 3 * FM_W + FM_OUT; k += TC_NT)
      reinterpret_cast<float *>(tc_sm + TC_OFF_B)[k] = reinterpret_cast<const float *>(params + FM_OFF_B)[k];
  }
  if (warp == 0) {  // 512 tensor-memory columns (a power of two): a 128 x 128 FP32 accumulator per group
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;\n" ::"r"(
                     (unsigned)__cvta_generic_to_shared(tslot))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) {
    for (int b = 0; b < TC_GROUPS; b++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"((unsigned)__cvta_generic_to_shared(bars + b))
                   : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  tc_fence_proxy();  // the weights, written here, are read by the tensor core
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot + (uint32_t)(grp * 128);
  const unsigned sbase = (unsigned)__cvta_generic_to_shared(tc_sm);
  const float *bias = reinterpret_cast<const float *>(tc_sm + TC_OFF_B);
  unsigned char *slot = tc_sm + TC_OFF_S + grp * TC_SLOT;
  const unsigned slot_s = sbase + TC_OFF_S + grp * TC_SLOT;
  uint64_t *bar = bars + grp;
  const long long ntiles = (n + TC_ROWS - 1) / TC_ROWS;
  unsigned phase = 0;
  bool failed = false;
  // this thread's row: lane quarter (warp % 4) of its group's accumulator
  const int row = (warp & 3) * 32 + lane;
  const uint32_t trow = tmem + ((uint32_t)((warp & 3) * 32) << 16);
  for (long long tile = blockIdx.x + (long long)grp * gridDim.x; tile < ntiles && !failed;
       tile += (long long)TC_GROUPS * gridDim.x) {
    const long long r0 = tile * TC_ROWS;
    tc_stage_x(X, n, r0, slot, gt);
    cp_async_wait<0>();
    tc_fence_proxy();
    tc_fence_before();
    tc_group_sync(grp);
    for (int l = 0; l < 4; l++) {
      const int K = l == 0 ? FM_IN : FM_W, N = l == 3 ? FM_OUT : FM_W;
      if (gt == 0) {
        tc_fence_after();
        const unsigned b0 = sbase + (l == 0 ? 0u : l == 1 ? (unsigned)TC_OFF_W1 : l == 2 ? (unsigned)TC_OFF_W2 : (unsigned)TC_OFF_W3);
        const uint32_t idesc = tc_idesc(TC_ROWS, N);
        for (int kk = 0; kk < K / 16; kk++) {
          const uint64_t da = tc_desc(slot_s + kk * 2 * (TC_ROWS / 8) * 128, (TC_ROWS / 8) * 128, 128);
          const uint64_t db = tc_desc(b0 + kk * 2 * (N / 8) * 128, (N / 8) * 128, 128);
          tc_mma(tmem, da, db, idesc, kk > 0);
        }
        tc_commit(bar);
      }
      const bool ok = tc_wait(bar, phase);
      phase ^= 1u;
      if (tc_group_any(grp, !ok)) {  // the whole group stops together
        failed = true;
        break;
      }
      tc_fence_after();
      if (l < 3) {
        const float *b = bias + l * FM_W;
#pragma unroll
        for (int half = 0; half < 2; half++) {
          uint32_t r[4][16];
#pragma unroll
          for (int q = 0; q < 4; q++) tc_ld16(trow + half * 64 + q * 16, r[q]);
          tc_ld_wait();
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const int c0 = half * 64 + q * 16;
            const f32x2_t *b2 = reinterpret_cast<const f32x2_t *>(b + c0);
            uint32_t hv[8];
#pragma unroll
            for (int e = 0; e < 8; e++)
              hv[e] = gelu2_bf16(((f32x2_t)r[q][2 * e + 1] << 32) | r[q][2 * e], b2[e]);
            *reinterpret_cast<uint4 *>(slot + tc_off(row, c0, TC_ROWS)) = make_uint4(hv[0], hv[1], hv[2], hv[3]);
            *reinterpret_cast<uint4 *>(slot + tc_off(row, c0 + 8, TC_ROWS)) = make_uint4(hv[4], hv[5], hv[6], hv[7]);
          }
        }
        tc_fence_proxy();
      } else {
        uint32_t r[16];
        tc_ld16(trow, r);
        tc_ld_wait();
        const float *b3 = bias + 3 * FM_W;
        if (r0 + row < n) {
          float4 *y = reinterpret_cast<float4 *>(Y + (size_t)(r0 + row) * FM_OUT);
#pragma unroll
          for (int q = 0; q < 4; q++)
            y[q] = make_float4(__uint_as_float(r[4 * q]) + b3[4 * q], __uint_as_float(r[4 * q + 1]) + b3[4 * q + 1],
                               __uint_as_float(r[4 * q + 2]) + b3[4 * q + 2],
                               __uint_as_float(r[4 * q + 3]) + b3[4 * q + 3]);
        }
      }
      tc_fence_before();
      tc_group_sync(grp);
    }
  }
  if (failed) atomicOr(flag, 1);
  cp_async_wait<0>();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;\n" ::"r"(*tslot) : "memory");
}

// ---------------------------------------------------------------------------
// The products of a training step on the tensor cores: BF16 mma.sync
// m16n8k16 with FP32 accumulation, row-major operands.
//   GM_FWD: C[n][i] = sum_k X[n][k] W[k][i]             (Z = X W)
//   GM_DIN: C[n][j] = sum_i D[n][i] W[j][i]             (dH = dZ W^T)
//   GM_DW:  C[z][j][i] = sum_{n in chunk z} X[n][j] D[n][i]   (dW = X^T dZ,
//           split over row chunks; k_sum_partials adds the chunks in order)
// A CTA of 4 warps computes a 32 (p) x 64 (q) tile of C; the reduction runs
// in 16-wide steps through shared memory, zero-filled outside the operands.
// ---------------------------------------------------------------------------
enum { GM_FWD = 0, GM_DIN = 1, GM_DW = 2 };
#define GM_TP 32
#define GM_TQ 64
#define GM_KS 64              // reduction width of one shared-memory stage
#define GM_RS (GM_KS + 8)     // shared row stride in BF16: 144 B, rows stay 16-byte aligned

// 8 consecutive BF16 from p (n of them valid, the rest zero): one 16-byte
// load when all 8 are valid (p is then 16-byte aligned: every leading
// dimension here is a multiple of 8 elements)
__device__ __forceinline__ uint4 gm_ld8(const __nv_bfloat16 *__restrict__ p, int n) {
  if (n >= 8) return __ldg(reinterpret_cast<const uint4 *>(p));
  __align__(16) __nv_bfloat16 v[8];
#pragma unroll
  for (int e = 0; e < 8; e++) v[e] = e < n ? p[e] : __float2bfloat16_rn(0.0f);
  return *reinterpret_cast<uint4 *>(v);
}

// scatter 8 BF16 down a column of a [row][GM_RS] shared tile
__device__ __forceinline__ void gm_st8_col(__nv_bfloat16 (*T)[GM_RS], int row0, int col, uint4 v) {
  const __nv_bfloat16 *e = reinterpret_cast<const __nv_bfloat16 *>(&v);
#pragma unroll
  for (int k = 0; k < 8; k++) T[row0 + k][col] = e[k];
}

template <int MODE>
__global__ void __launch_bounds__(128) k_gemm_bf16(const __nv_bfloat16 *__restrict__ X,
                                                   const __nv_bfloat16 *__restrict__ Y, float *__restrict__ C,
                                                   int P, int Q, long long R, int ldx, int ldy, long long chunk) {
  __shared__ __align__(16) __nv_bfloat16 As[GM_TP][GM_RS];
  __shared__ __align__(16) __nv_bfloat16 Bs[GM_TQ][GM_RS];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, g = lane >> 2, t = lane & 3;
  const int p0 = blockIdx.x * GM_TP, q0 = blockIdx.y * GM_TQ;
  long long r0 = 0, r1 = R;
  if (MODE == GM_DW) {
    r0 = (long long)blockIdx.z * chunk;
    r1 = r0 + chunk < R ? r0 + chunk : R;
    C += (size_t)blockIdx.z * P * Q;
  }
  const int wp = (w & 1) * 16, wq = (w >> 1) * 32;
  float acc[4][4];
#pragma unroll
  for (int nt = 0; nt < 4; nt++)
#pragma unroll
    for (int c = 0; c < 4; c++) acc[nt][c] = 0.0f;
  for (long long rb = r0; rb < r1; rb += GM_KS) {
    const long long rleft = r1 - rb;
    // A tile (32 p x 64 r): 256 vectors of 8, two per thread
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int v = tid + h * 128;
      if (MODE == GM_DW) {  // A(p, r) = X[r * ldx + p]: vectors along p
        const int rr = v >> 2, p8 = (v & 3) * 8;
        const int p = p0 + p8;
        const int n = (rr < rleft) ? (P - p < 8 ? P - p : 8) : 0;
        gm_st8_col(As, p8, rr, gm_ld8(X + (rb + rr) * ldx + p, n));
      } else {  // A(p, r) = X[p * ldx + r]: vectors along r
        const int pp = v >> 3, r8 = (v & 7) * 8;
        const int p = p0 + pp;
        const long long rl = rleft - r8;
        const int n = (p < P) ? (int)(rl < 8 ? (rl > 0 ? rl : 0) : 8) : 0;
        *reinterpret_cast<uint4 *>(&As[pp][r8]) = gm_ld8(X + (long long)p * ldx + rb + r8, n);
      }
    }
    // B tile (64 q x 64 r), stored [q][r]: 512 vectors of 8, four per thread
#pragma unroll
    for (int h = 0; h < 4; h++) {
      const int v = tid + h * 128;
      if (MODE == GM_DIN) {  // B(r, q) = Y[q * ldy + r]: vectors along r
        const int qq = v >> 3, r8 = (v & 7) * 8;
        const int q = q0 + qq;
        const long long rl = rleft - r8;
        const int n = (q < Q) ? (int)(rl < 8 ? (rl > 0 ? rl : 0) : 8) : 0;
        *reinterpret_cast<uint4 *>(&Bs[qq][r8]) = gm_ld8(Y + (long long)q * ldy + rb + r8, n);
      } else {  // B(r, q) = Y[r * ldy + q]: vectors along q
        const int rr = v >> 3, q8 = (v & 7) * 8;
        const int q = q0 + q8;
        const int n = (rr < rleft) ? (Q - q < 8 ? (Q - q > 0 ? Q - q : 0) : 8) : 0;
        gm_st8_col(Bs, q8, rr, gm_ld8(Y + (rb + rr) * ldy + (n > 0 ? q : 0), n));
      }
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < GM_KS; ks += 16) {
      unsigned a[4];
      a[0] = *reinterpret_cast<const unsigned *>(&As[wp + g][ks + 2 * t]);
      a[1] = *reinterpret_cast<const unsigned *>(&As[wp + g + 8][ks + 2 * t]);
      a[2] = *reinterpret_cast<const unsigned *>(&As[wp + g][ks + 2 * t + 8]);
      a[3] = *reinterpret_cast<const unsigned *>(&As[wp + g + 8][ks + 2 * t + 8]);
#pragma unroll
      for (int nt = 0; nt < 4; nt++) {
        const __nv_bfloat16 *br = &Bs[wq + nt * 8 + g][ks + 2 * t];
        mma_bf16_16816(acc[nt], a, *reinterpret_cast<const unsigned *>(br),
                       *reinterpret_cast<const unsigned *>(br + 8));
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int nt = 0; nt < 4; nt++)
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int p = p0 + wp + g + (c >= 2 ? 8 : 0), q = q0 + wq + nt * 8 + 2 * t + (c & 1);
      if (p < P && q < Q) C[(size_t)p * Q + q] = acc[nt][c];
    }
}

// dst (M x K) = src (K x M) transposed, BF16
__global__ void k_transpose_bf16(const __nv_bfloat16 *__restrict__ src, int K, int M, __nv_bfloat16 *__restrict__ dst) {
  const int n = K * M;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int q = i / K, k = i - q * K;
    dst[i] = src[(size_t)k * M + q];
  }
}

// out[i] = sum over z in order of part[z * count + i]
__global__ void k_sum_partials(const float *__restrict__ part, int nsplit, int count, float *__restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int z = 0; z < nsplit; z++) s += part[(size_t)z * count + i];
    out[i] = s;
  }
}

}  // namespace css

