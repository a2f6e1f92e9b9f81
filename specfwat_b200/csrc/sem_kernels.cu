// CUDA kernels of the elastic SEM time loop (sm_100a).
//
// Wavefields use the lane-interleaved layout [point][component][lane]: a
// lane is one event.  With one event (the plain path) this is the usual
// point-major xyz layout of the reference's displ(3,NGLOB); with many events
// consecutive lanes of one point/component are contiguous, so a warp's
// gather and scatter-add of one point touch whole 32-byte sectors and the
// element data (ibool, kappa, mu) is read once for all lanes of a block.
//
// One step = k_forces (element stiffness + assembly, strain products for
// the kernels), k_stacey (absorbing traction / boundary store save and
// replay), k_points (moment-tensor source, receivers, adjoint sources) and
// k_update (Newmark corrector of this step fused with the predictor of the
// next, plus the density-kernel product).

#include <algorithm>
#include <cstdio>

#include "sem_gll.cuh"
#include "sem_internal.cuh"

namespace sem {

__constant__ float c_D[25];    // D[i][l] = l_l'(xi_i), index i*5+l
__constant__ float c_DWt[25];  // DWt[i][l] = w_l * D[l][i], index i*5+l
__constant__ float c_w[5];

void set_gll_constants(const float* D, const float* DWt, const float* w) {
  cudaMemcpyToSymbol(c_D, D, 25 * sizeof(float));
  cudaMemcpyToSymbol(c_DWt, DWt, 25 * sizeof(float));
  cudaMemcpyToSymbol(c_w, w, 5 * sizeof(float));
}

// ---------------------------------------------------------------------------
// element kernel
// ---------------------------------------------------------------------------

// Displacement gradient at GLL point (i,j,k) of one lane.  b holds the
// element's displacement as [c][125][LB]; g[c][d] = d u_c / d x_d.
template <int LB>
__device__ __forceinline__ void grad_point(const float* __restrict__ b, int i, int j, int k,
                                           int lane, const float* __restrict__ sD, float xix,
                                           float g[3][3]) {
  float di[5], dj[5], dk[5];
#pragma unroll
  for (int l = 0; l < 5; ++l) {
    di[l] = sD[i * 5 + l];
    dj[l] = sD[j * 5 + l];
    dk[l] = sD[k * 5 + l];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float* bc = b + c * NGLL3 * LB;
    float s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      s1 = fmaf(di[l], bc[(l + 5 * j + 25 * k) * LB + lane], s1);
      s2 = fmaf(dj[l], bc[(i + 5 * l + 25 * k) * LB + lane], s2);
      s3 = fmaf(dk[l], bc[(i + 5 * j + 25 * l) * LB + lane], s3);
    }
    g[c][0] = xix * s1;
    g[c][1] = xix * s2;
    g[c][2] = xix * s3;
  }
}

// Isotropic stress times jacobian*xix: sig = {xx, yy, zz, xy, xz, yz}.
__device__ __forceinline__ void stress_point(const float g[3][3], float kap, float mu, float fac,
                                             float sig[6]) {
  const float l2m = kap + (4.0f / 3.0f) * mu;
  const float lam = l2m - 2.0f * mu;
  sig[0] = fac * (l2m * g[0][0] + lam * (g[1][1] + g[2][2]));
  sig[1] = fac * (l2m * g[1][1] + lam * (g[0][0] + g[2][2]));
  sig[2] = fac * (l2m * g[2][2] + lam * (g[0][0] + g[1][1]));
  sig[3] = fac * (mu * (g[0][1] + g[1][0]));
  sig[4] = fac * (mu * (g[0][2] + g[2][0]));
  sig[5] = fac * (mu * (g[1][2] + g[2][1]));
}

// General element (per-point mapping G = xix, xiy, xiz, etax, etay, etaz,
// gammax, gammay, gammaz, jacobian): physical gradient from the reference
// derivatives r[c][d] (d = xi, eta, gamma), and the fluxes of each
// component through the three reference directions,
// F[c*3+d] = jacobian * sum_a sigma_{c,a} d(xi_d)/d(x_a).
__device__ __forceinline__ void map_gradient(const float r[3][3], const float* G, float g[3][3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int a = 0; a < 3; ++a) g[c][a] = r[c][0] * G[a] + r[c][1] * G[3 + a] + r[c][2] * G[6 + a];
}
__device__ __forceinline__ void map_flux(const float sig[6], const float* G, float F[9]) {
  const float sc[3][3] = {{sig[0], sig[3], sig[4]}, {sig[3], sig[1], sig[5]},
                          {sig[4], sig[5], sig[2]}};
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int d = 0; d < 3; ++d)
      F[c * 3 + d] = G[9] * (sc[c][0] * G[3 * d] + sc[c][1] * G[3 * d + 1] + sc[c][2] * G[3 * d + 2]);
}

// Divergence from the nine fluxes F[c*3+d] staged per point.
template <int LB>
__device__ __forceinline__ void div_point_gen(const float* __restrict__ b, int i, int j, int k,
                                              int lane, const float* __restrict__ sDWt,
                                              const float* __restrict__ sw, float f[3]) {
  float a[3] = {0.f, 0.f, 0.f}, bb[3] = {0.f, 0.f, 0.f}, cc[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int l = 0; l < 5; ++l) {
    const float wi = sDWt[i * 5 + l], wj = sDWt[j * 5 + l], wk = sDWt[k * 5 + l];
    const int qi = (l + 5 * j + 25 * k) * LB + lane;
    const int qj = (i + 5 * l + 25 * k) * LB + lane;
    const int qk = (i + 5 * j + 25 * l) * LB + lane;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      a[c] = fmaf(wi, b[(c * 3 + 0) * NGLL3 * LB + qi], a[c]);
      bb[c] = fmaf(wj, b[(c * 3 + 1) * NGLL3 * LB + qj], bb[c]);
      cc[c] = fmaf(wk, b[(c * 3 + 2) * NGLL3 * LB + qk], cc[c]);
    }
  }
  const float wjk = sw[j] * sw[k], wik = sw[i] * sw[k], wij = sw[i] * sw[j];
#pragma unroll
  for (int c = 0; c < 3; ++c) f[c] = -(wjk * a[c] + wik * bb[c] + wij * cc[c]);
}

// Weak-form divergence at (i,j,k): f_c = -sum_d w w sum_l DW * sig_{c,d}.
template <int LB>
__device__ __forceinline__ void div_point(const float* __restrict__ b, int i, int j, int k,
                                          int lane, const float* __restrict__ sDWt,
                                          const float* __restrict__ sw, float f[3]) {
  const float* Sxx = b;
  const float* Syy = b + 1 * NGLL3 * LB;
  const float* Szz = b + 2 * NGLL3 * LB;
  const float* Sxy = b + 3 * NGLL3 * LB;
  const float* Sxz = b + 4 * NGLL3 * LB;
  const float* Syz = b + 5 * NGLL3 * LB;
  float ax = 0.f, ay = 0.f, az = 0.f, bx = 0.f, by = 0.f, bz = 0.f, cx = 0.f, cy = 0.f,
        cz = 0.f;
#pragma unroll
  for (int l = 0; l < 5; ++l) {
    const float wi = sDWt[i * 5 + l], wj = sDWt[j * 5 + l], wk = sDWt[k * 5 + l];
    const int qi = (l + 5 * j + 25 * k) * LB + lane;
    const int qj = (i + 5 * l + 25 * k) * LB + lane;
    const int qk = (i + 5 * j + 25 * l) * LB + lane;
    ax = fmaf(wi, Sxx[qi], ax);
    ay = fmaf(wi, Sxy[qi], ay);
    az = fmaf(wi, Sxz[qi], az);
    bx = fmaf(wj, Sxy[qj], bx);
    by = fmaf(wj, Syy[qj], by);
    bz = fmaf(wj, Syz[qj], bz);
    cx = fmaf(wk, Sxz[qk], cx);
    cy = fmaf(wk, Syz[qk], cy);
    cz = fmaf(wk, Szz[qk], cz);
  }
  const float wjk = sw[j] * sw[k], wik = sw[i] * sw[k], wij = sw[i] * sw[j];
  f[0] = -(wjk * ax + wik * bx + wij * cx);
  f[1] = -(wjk * ay + wik * by + wij * cy);
  f[2] = -(wjk * az + wik * bz + wij * cz);
}

// One block = one element x LB lanes.  ADJ: lanes in the adjoint phase also
// carry the backward field (f2) and accumulate the mu/kappa kernels.
template <int LB, int NT, bool ADJ, bool GEN = false>
__global__ void __launch_bounds__(NT) k_forces(StepArgs A) {
  constexpr int G = NT / LB;
  constexpr int P = (NGLL3 + G - 1) / G;
  constexpr int NQ = GEN ? 9 : 6;   // staged values per point: fluxes or stresses
  extern __shared__ float sm[];
  __shared__ int s_ib[NGLL3];
  __shared__ float s_kap[NGLL3], s_mu[NGLL3];
  __shared__ float s_D[25], s_DWt[25], s_w[5];
  float* b1 = sm;
  float* b2 = sm + NQ * NGLL3 * LB;

  const int e = A.m.order[blockIdx.x];
  const int lane = threadIdx.x % LB;
  const int pg = threadIdx.x / LB;
  const int lg = blockIdx.y * LB + lane;
  const int nev = A.nev;
  bool act1 = false, act2 = false, scat2 = false;
  if (lg < nev) {
    const LaneDesc* L = A.lanes + lg;
    const int it = L->it0 + A.s;
    const int ph = L->phase;
    if (ph != PH_IDLE && it < L->nstep) {
      act1 = true;
      if (ADJ && ph == PH_ADJ) {
        act2 = true;
        scat2 = it > 0;
      }
    }
  }
  if (!__syncthreads_or(act1)) return;

  for (int p = threadIdx.x; p < NGLL3; p += NT) {
    const size_t ep = (size_t)e * NGLL3 + p;
    s_ib[p] = A.m.ibool[ep];
    s_kap[p] = A.m.kappa[ep];
    s_mu[p] = A.m.mu[ep];
  }
  if (threadIdx.x < 25) {
    s_D[threadIdx.x] = c_D[threadIdx.x];
    s_DWt[threadIdx.x] = c_DWt[threadIdx.x];
  }
  if (threadIdx.x < 5) s_w[threadIdx.x] = c_w[threadIdx.x];
  __syncthreads();

#pragma unroll
  for (int t = 0; t < P; ++t) {
    const int p = pg + t * G;
    if (p < NGLL3) {
      const size_t ig = (size_t)s_ib[p];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const size_t q = act1 || act2 ? A.fi(ig, c, lg) : 0;
        b1[(c * NGLL3 + p) * LB + lane] = act1 ? A.f1.u[q] : 0.f;
        if (ADJ) b2[(c * NGLL3 + p) * LB + lane] = act2 ? A.f2.u[q] : 0.f;
      }
    }
  }
  __syncthreads();

  const float xix = A.m.xix;
  const float fac = A.m.jac * A.m.xix;
  // general elements: this element's mapping, or the regular one
  const float* geo = nullptr;
  if (GEN) {
    const int ir = A.m.irreg[e];
    if (ir >= 0) geo = A.m.geo + (size_t)ir * NGLL3 * 10;
  }
  float sg1[P][NQ];
  float sg2[ADJ ? P : 1][NQ];
#pragma unroll
  for (int t = 0; t < P; ++t) {
    const int p = pg + t * G;
    if (p < NGLL3) {
      const int i = p % 5, j = (p / 5) % 5, k = p / 25;
      float Gp[10];
      if (GEN && geo) {
#pragma unroll
        for (int q = 0; q < 10; ++q) Gp[q] = geo[p * 10 + q];
      }
      float g1[3][3];
      if (GEN && geo) {
        float r1[3][3];
        grad_point<LB>(b1, i, j, k, lane, s_D, 1.0f, r1);
        map_gradient(r1, Gp, g1);
        float sg[6];
        stress_point(g1, s_kap[p], s_mu[p], 1.0f, sg);
        map_flux(sg, Gp, sg1[t]);
      } else {
        grad_point<LB>(b1, i, j, k, lane, s_D, xix, g1);
        if (GEN) {
          float sg[6];
          stress_point(g1, s_kap[p], s_mu[p], fac, sg);
          const float F[9] = {sg[0], sg[3], sg[4], sg[3], sg[1], sg[5], sg[4], sg[5], sg[2]};
#pragma unroll
          for (int q = 0; q < NQ; ++q) sg1[t][q] = F[q];
        } else {
          stress_point(g1, s_kap[p], s_mu[p], fac, sg1[t]);
        }
      }
      if (ADJ) {
        float g2[3][3];
        if (GEN && geo) {
          float r2[3][3];
          grad_point<LB>(b2, i, j, k, lane, s_D, 1.0f, r2);
          map_gradient(r2, Gp, g2);
          float sg[6];
          stress_point(g2, s_kap[p], s_mu[p], 1.0f, sg);
          map_flux(sg, Gp, sg2[t]);
        } else {
          grad_point<LB>(b2, i, j, k, lane, s_D, xix, g2);
          if (GEN) {
            float sg[6];
            stress_point(g2, s_kap[p], s_mu[p], fac, sg);
            const float F[9] = {sg[0], sg[3], sg[4], sg[3], sg[1], sg[5], sg[4], sg[5], sg[2]};
#pragma unroll
            for (int q = 0; q < NQ; ++q) sg2[t][q] = F[q];
          } else {
            stress_point(g2, s_kap[p], s_mu[p], fac, sg2[t]);
          }
        }
        if (act2) {
          // deviatoric strain products (adjoint x backward) and traces
          const float tr1 = g1[0][0] + g1[1][1] + g1[2][2];
          const float tr2 = g2[0][0] + g2[1][1] + g2[2][2];
          const float a_xx = g1[0][0] - tr1 * (1.0f / 3.0f);
          const float a_yy = g1[1][1] - tr1 * (1.0f / 3.0f);
          const float b_xx = g2[0][0] - tr2 * (1.0f / 3.0f);
          const float b_yy = g2[1][1] - tr2 * (1.0f / 3.0f);
          const float a_xy = 0.5f * (g1[0][1] + g1[1][0]);
          const float a_xz = 0.5f * (g1[0][2] + g1[2][0]);
          const float a_yz = 0.5f * (g1[1][2] + g1[2][1]);
          const float b_xy = 0.5f * (g2[0][1] + g2[1][0]);
          const float b_xz = 0.5f * (g2[0][2] + g2[2][0]);
          const float b_yz = 0.5f * (g2[1][2] + g2[2][1]);
          const float dd = a_xx * b_xx + a_yy * b_yy + (a_xx + a_yy) * (b_xx + b_yy) +
                           2.0f * (a_xy * b_xy + a_xz * b_xz + a_yz * b_yz);
          const size_t q = A.ei((size_t)e * NGLL3 + p, lg);
          A.k.mu[q] += A.dt * dd;
          A.k.kappa[q] += A.dt * (tr1 * tr2);
        }
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int t = 0; t < P; ++t) {
    const int p = pg + t * G;
    if (p < NGLL3) {
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        b1[(q * NGLL3 + p) * LB + lane] = sg1[t][q];
        if (ADJ) b2[(q * NGLL3 + p) * LB + lane] = sg2[t][q];
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int t = 0; t < P; ++t) {
    const int p = pg + t * G;
    if (p < NGLL3) {
      const int i = p % 5, j = (p / 5) % 5, k = p / 25;
      const size_t ig = (size_t)s_ib[p];
      if (act1) {
        float f[3];
        if (GEN)
          div_point_gen<LB>(b1, i, j, k, lane, s_DWt, s_w, f);
        else
          div_point<LB>(b1, i, j, k, lane, s_DWt, s_w, f);
#pragma unroll
        for (int c = 0; c < 3; ++c) atomicAdd(&A.f1.a[A.fi(ig, c, lg)], f[c]);
      }
      if (ADJ && scat2) {
        float f[3];
        if (GEN)
          div_point_gen<LB>(b2, i, j, k, lane, s_DWt, s_w, f);
        else
          div_point<LB>(b2, i, j, k, lane, s_DWt, s_w, f);
#pragma unroll
        for (int c = 0; c < 3; ++c) atomicAdd(&A.f2.a[A.fi(ig, c, lg)], f[c]);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// element kernel, thread per GLL point, xi contractions by warp shuffles
// ---------------------------------------------------------------------------
//
// Warp w holds GLL rows r = 6w .. 6w+5 (row r is (j,k) = (r%5, r/5)); lane l
// is point i = l%5 of row 6w + l/5, and lanes 30, 31 idle, so the five
// points of a row sit in five consecutive lanes of one warp.  The
// xi-derivatives and the xi part of the divergence read the row through
// __shfl_sync; the eta and gamma directions go through shared memory as in
// the thread-per-point kernel.  One lane per block (grid.y = lane).

template <bool ADJ>
__global__ void __launch_bounds__(160) k_forces_shfl(StepArgs A) {
  constexpr int NF = ADJ ? 2 : 1;
  __shared__ float sU[NF][3][NGLL3];
  __shared__ float sS[NF][6][NGLL3];
  __shared__ float sD[25], sDWt[25], sW[5];
  const int e = A.m.order[blockIdx.x];
  const int lg = blockIdx.y;
  const int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
  const int r = 6 * w + ln / 5;
  const bool act = ln < 30 && r < 25;
  const int rr = act ? r : 0;
  const int i = act ? ln % 5 : 0, j = rr % 5, k = rr / 5;
  const int p = i + 5 * rr;
  const int base = (ln / 5) * 5;
  bool act1 = false, act2 = false, scat2 = false;
  {
    const LaneDesc* L = A.lanes + lg;
    const int it = L->it0 + A.s;
    if (L->phase != PH_IDLE && it < L->nstep) {
      act1 = true;
      if (ADJ && L->phase == PH_ADJ) {
        act2 = true;
        scat2 = it > 0;
      }
    }
  }
  if (threadIdx.x < 25) {
    sD[threadIdx.x] = c_D[threadIdx.x];
    sDWt[threadIdx.x] = c_DWt[threadIdx.x];
  }
  if (threadIdx.x < 5) sW[threadIdx.x] = c_w[threadIdx.x];
  if (!__syncthreads_or(act1)) return;

  const size_t ep = (size_t)e * NGLL3 + p;
  const int ig = A.m.ibool[ep];
  const float kp = A.m.kappa[ep], mu = A.m.mu[ep];
  float u[NF][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const size_t q = A.fi((size_t)ig, c, lg);
    u[0][c] = act1 ? A.f1.u[q] : 0.f;
    if (ADJ) u[NF - 1][c] = act2 ? A.f2.u[q] : 0.f;
  }
  if (act)
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int c = 0; c < 3; ++c) sU[f][c][p] = u[f][c];
  __syncthreads();

  const float xix = A.m.xix;
  const float fac = A.m.jac * A.m.xix;
  float di[5], dj[5], dk[5];
#pragma unroll
  for (int l = 0; l < 5; ++l) {
    di[l] = sD[i * 5 + l];
    dj[l] = sD[j * 5 + l];
    dk[l] = sD[k * 5 + l];
  }
  float sig[NF][6];
  float g[NF][3][3];
#pragma unroll
  for (int f = 0; f < NF; ++f) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float a = 0.f, b = 0.f, cc = 0.f;
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        a = fmaf(di[l], __shfl_sync(0xffffffffu, u[f][c], base + l), a);
        b = fmaf(dj[l], sU[f][c][i + 5 * l + 25 * k], b);
        cc = fmaf(dk[l], sU[f][c][i + 5 * j + 25 * l], cc);
      }
      g[f][c][0] = a * xix;
      g[f][c][1] = b * xix;
      g[f][c][2] = cc * xix;
    }
    stress_point(g[f], kp, mu, fac, sig[f]);
  }
  if (ADJ && act2 && act) {
    const float tr1 = g[0][0][0] + g[0][1][1] + g[0][2][2];
    const float tr2 = g[1][0][0] + g[1][1][1] + g[1][2][2];
    const float a_xx = g[0][0][0] - tr1 * (1.0f / 3.0f), a_yy = g[0][1][1] - tr1 * (1.0f / 3.0f);
    const float b_xx = g[1][0][0] - tr2 * (1.0f / 3.0f), b_yy = g[1][1][1] - tr2 * (1.0f / 3.0f);
    const float a_xy = 0.5f * (g[0][0][1] + g[0][1][0]), a_xz = 0.5f * (g[0][0][2] + g[0][2][0]);
    const float a_yz = 0.5f * (g[0][1][2] + g[0][2][1]);
    const float b_xy = 0.5f * (g[1][0][1] + g[1][1][0]), b_xz = 0.5f * (g[1][0][2] + g[1][2][0]);
    const float b_yz = 0.5f * (g[1][1][2] + g[1][2][1]);
    const float dd = a_xx * b_xx + a_yy * b_yy + (a_xx + a_yy) * (b_xx + b_yy) +
                     2.0f * (a_xy * b_xy + a_xz * b_xz + a_yz * b_yz);
    const size_t q = A.ei(ep, lg);
    A.k.mu[q] += A.dt * dd;
    A.k.kappa[q] += A.dt * (tr1 * tr2);
  }
  __syncthreads();  // every eta/gamma read of sU is done
  if (act)
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int q = 0; q < 6; ++q) sS[f][q][p] = sig[f][q];
  __syncthreads();
#pragma unroll
  for (int l = 0; l < 5; ++l) {
    di[l] = sDWt[i * 5 + l];
    dj[l] = sDWt[j * 5 + l];
    dk[l] = sDWt[k * 5 + l];
  }
  const float wjk = sW[j] * sW[k], wik = sW[i] * sW[k], wij = sW[i] * sW[j];
  // flux components: xi direction sigma_{c,x} = (xx, xy, xz), eta
  // sigma_{c,y} = (xy, yy, yz), gamma sigma_{c,z} = (xz, yz, zz)
  constexpr int QX[3] = {0, 3, 4}, QY[3] = {3, 1, 5}, QZ[3] = {4, 5, 2};
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    float fo[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float a = 0.f, b = 0.f, cc = 0.f;
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        a = fmaf(di[l], __shfl_sync(0xffffffffu, sig[f][QX[c]], base + l), a);
        b = fmaf(dj[l], sS[f][QY[c]][i + 5 * l + 25 * k], b);
        cc = fmaf(dk[l], sS[f][QZ[c]][i + 5 * j + 25 * l], cc);
      }
      fo[c] = -(wjk * a + wik * b + wij * cc);
    }
    const bool on = f == 0 ? act1 : scat2;
    if (act && on) {
      float* acc = f == 0 ? A.f1.a : A.f2.a;
#pragma unroll
      for (int c = 0; c < 3; ++c) atomicAdd(&acc[A.fi((size_t)ig, c, lg)], fo[c]);
    }
  }
}

template <bool ADJ>
static int forces_shfl_cfg(const StepArgs& a, cudaStream_t st) {
  dim3 grid(a.m.nspec, a.nev);
  k_forces_shfl<ADJ><<<grid, 160, 0, st>>>(a);
  return 1;
}

// ---------------------------------------------------------------------------
// element kernel, pencil decomposition
// ---------------------------------------------------------------------------
//
// Each element is worked by 25 "pencil" threads per lane.  Thread t takes
// three roles: owner of the xi-pencil (j,k) = (t%5, t/5), of the eta-pencil
// (i,k) and of the gamma-pencil (i,j).  Along its own pencil every
// contraction is register-local with the GLL matrices as immediates; the
// other two directions are exchanged through shared memory, so one element
// costs about 235 shared accesses per pencil thread instead of the ~130 per
// GLL point of a thread-per-point kernel (~3x fewer per element).
//
//   gather        u -> U                      (cooperative, coalesced)
//   eta/gamma     U -> d_eta, d_gamma -> A
//   xi            U, A -> gradient -> stress -> B (sigma for eta/gamma),
//                 f_xi in registers, strain products (adjoint)
//   eta/gamma     B -> f_eta, f_gamma -> A
//   xi            A + f_xi -> scatter-add into accel

// Per-lane base offsets of the lane-group layout with the group width known
// at compile time (LWLOG 0: one event, 3: groups of 8): a field value is
// base(lg) + (ig*3 + c) << LWLOG, a per-point value base(lg) + i << LWLOG.
template <int LWLOG>
__device__ __forceinline__ size_t fbase(const StepArgs& A, int lg) {
  return (((size_t)(lg >> LWLOG) * (size_t)A.m.nglob * 3) << LWLOG) + (lg & ((1 << LWLOG) - 1));
}
template <int LWLOG>
__device__ __forceinline__ size_t ebase(const StepArgs& A, int lg) {
  return (((size_t)(lg >> LWLOG) * (size_t)A.m.nspec * NGLL3) << LWLOG) +
         (lg & ((1 << LWLOG) - 1));
}
template <int LWLOG>
__device__ __forceinline__ size_t foff(int ig, int c) {
  return ((size_t)ig * 3 + c) << LWLOG;
}

// shared floats per (field, element, lane): U/B region then A region
constexpr int PR_U = 640;  // >= 625 (B: 5 sigma components)
constexpr int PR_A = 768;  // >= 750 (6 derivative / divergence components)
constexpr int PR_F = PR_U + PR_A;

template <int LB>
struct PencilBuf {
  float* ub;  // U/B region of this (field, element), lane offset applied
  float* ab;  // A region
  __device__ __forceinline__ float& U(int c, int p) const { return ub[(c * 125 + p) * LB]; }
  __device__ __forceinline__ float& B(int q, int p) const { return ub[(q * 125 + p) * LB]; }
  __device__ __forceinline__ float& Ar(int q, int p) const { return ab[(q * 125 + p) * LB]; }
};

// eta / gamma derivative roles of thread t (pencils (i,k) and (i,j)).
// Derivatives are left in reference coordinates; the regular-element
// factor xix is folded into the stress and strain-product scalings.
template <int LB>
__device__ __forceinline__ void pencil_grad_eg(const PencilBuf<LB>& b, int t) {
  const int pi = t % 5, pq = t / 5;
  // eta-pencil (i = pi, k = pq): d/d eta at (pi, j, pq)
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float v[5];
#pragma unroll
    for (int l = 0; l < 5; ++l) v[l] = b.U(c, pi + 5 * l + 25 * pq);
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      float s = 0.f;
#pragma unroll
      for (int l = 0; l < 5; ++l) s = cfma(gD(j, l), v[l], s);
      b.Ar(c, pi + 5 * j + 25 * pq) = s;
    }
  }
  // gamma-pencil (i = pi, j = pq): d/d gamma at (pi, pq, k)
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float v[5];
#pragma unroll
    for (int l = 0; l < 5; ++l) v[l] = b.U(c, pi + 5 * pq + 25 * l);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      float s = 0.f;
#pragma unroll
      for (int l = 0; l < 5; ++l) s = cfma(gD(k, l), v[l], s);
      b.Ar(3 + c, pi + 5 * pq + 25 * k) = s;
    }
  }
}

// xi role of thread t: full gradient on its xi-pencil (j,k) = (t%5, t/5).
// g[i][c][d] = d u_c / d xi_d at (i, j, k) (times xix: d u_c / d x_d).
template <int LB>
__device__ __forceinline__ void pencil_grad_xi(const PencilBuf<LB>& b, int t, float g[5][3][3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float v[5];
#pragma unroll
    for (int l = 0; l < 5; ++l) v[l] = b.U(c, l + 5 * t);
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      float s = 0.f;
#pragma unroll
      for (int l = 0; l < 5; ++l) s = cfma(gD(i, l), v[l], s);
      g[i][c][0] = s;
      g[i][c][1] = b.Ar(c, i + 5 * t);
      g[i][c][2] = b.Ar(3 + c, i + 5 * t);
    }
  }
}

// Stress on the xi-pencil, sigma components for the other roles into B
// (xy, yy, yz, xz, zz) and the xi part of the divergence in registers.
template <int LB>
__device__ __forceinline__ void pencil_stress(const PencilBuf<LB>& b, int t, const float g[5][3][3],
                                              const float* s_kap, const float* s_mu, float fac,
                                              float fx[5][3]) {
  float sxx[5], sxy[5], sxz[5];
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    const int p = i + 5 * t;
    float sig[6];
    stress_point(g[i], s_kap[p], s_mu[p], fac, sig);
    sxx[i] = sig[0];
    sxy[i] = sig[3];
    sxz[i] = sig[4];
    b.B(0, p) = sig[3];  // xy
    b.B(1, p) = sig[1];  // yy
    b.B(2, p) = sig[5];  // yz
    b.B(3, p) = sig[4];  // xz
    b.B(4, p) = sig[2];  // zz
  }
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    float ax = 0.f, ay = 0.f, az = 0.f;
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      ax = cfma(gDWt(i, l), sxx[l], ax);
      ay = cfma(gDWt(i, l), sxy[l], ay);
      az = cfma(gDWt(i, l), sxz[l], az);
    }
    fx[i][0] = ax;
    fx[i][1] = ay;
    fx[i][2] = az;
  }
}

// eta / gamma divergence roles: B -> A.
template <int LB>
__device__ __forceinline__ void pencil_div_eg(const PencilBuf<LB>& b, int t) {
  const int pi = t % 5, pq = t / 5;
  {  // eta-pencil (i = pi, k = pq): sigma_{c,y} = (xy, yy, yz) = B0, B1, B2
    float v[3][5];
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      const int p = pi + 5 * l + 25 * pq;
      v[0][l] = b.B(0, p);
      v[1][l] = b.B(1, p);
      v[2][l] = b.B(2, p);
    }
#pragma unroll
    for (int j = 0; j < 5; ++j)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float s = 0.f;
#pragma unroll
        for (int l = 0; l < 5; ++l) s = cfma(gDWt(j, l), v[c][l], s);
        b.Ar(c, pi + 5 * j + 25 * pq) = s;
      }
  }
  {  // gamma-pencil (i = pi, j = pq): sigma_{c,z} = (xz, yz, zz) = B3, B2, B4
    float v[3][5];
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      const int p = pi + 5 * pq + 25 * l;
      v[0][l] = b.B(3, p);
      v[1][l] = b.B(2, p);
      v[2][l] = b.B(4, p);
    }
#pragma unroll
    for (int k = 0; k < 5; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float s = 0.f;
#pragma unroll
        for (int l = 0; l < 5; ++l) s = cfma(gDWt(k, l), v[c][l], s);
        b.Ar(3 + c, pi + 5 * pq + 25 * k) = s;
      }
  }
}

// xi role: total force on the xi-pencil and scatter-add.
template <int LB>
__device__ __forceinline__ void pencil_scatter(const PencilBuf<LB>& b, int t, const float fx[5][3],
                                               const int* s_ib, float* accb) {
  constexpr int LWLOG = LB == 1 ? 0 : 3;
  const int pj = t % 5, pk = t / 5;
  float wj = 0.f, wk = 0.f;
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    if (q == pj) wj = gW(q);
    if (q == pk) wk = gW(q);
  }
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    const int p = i + 5 * t;
    const size_t ig = (size_t)s_ib[p];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float f = -(wj * wk * fx[i][c] + gW(i) * wk * b.Ar(c, p) + gW(i) * wj * b.Ar(3 + c, p));
      atomicAdd(&accb[foff<LWLOG>((int)ig, c)], f);
    }
  }
}

template <int LB, int EPB, bool ADJ>
__global__ void __launch_bounds__(EPB * 25 * LB) k_forces_pencil(StepArgs A) {
  constexpr int NT = EPB * 25 * LB;
  constexpr int NF = ADJ ? 2 : 1;
  extern __shared__ float sm[];
  __shared__ int s_ib[EPB * NGLL3];
  __shared__ float s_kap[EPB * NGLL3], s_mu[EPB * NGLL3];
  __shared__ unsigned char s_act[2][LB];

  const int tid = threadIdx.x;
  const int lane = tid % LB;
  const int t = (tid / LB) % 25;
  const int el = tid / (25 * LB);
  const int eslot = blockIdx.x * EPB + el;
  const int e = eslot < A.m.nspec ? A.m.order[eslot] : A.m.nspec;
  const int lg = blockIdx.y * LB + lane;
  const int nev = A.nev;

  bool any = false;
  if (tid < LB) {
    bool a1 = false, a2 = false;
    const int l2 = blockIdx.y * LB + tid;
    if (l2 < nev) {
      const LaneDesc* L = A.lanes + l2;
      const int it = L->it0 + A.s;
      if (L->phase != PH_IDLE && it < L->nstep) {
        a1 = true;
        // at it == 0 of the adjoint phase the backward strain is still
        // needed (kernels); only its scatter is skipped
        a2 = ADJ && L->phase == PH_ADJ;
      }
    }
    s_act[0][tid] = a1;
    s_act[1][tid] = a2;
    any = a1;
  }
  if (!__syncthreads_or(any)) return;
  bool scat2 = false;
  if (ADJ && lg < nev) {
    const LaneDesc* L = A.lanes + lg;
    scat2 = s_act[1][lane] && (L->it0 + A.s) > 0;
  }

  for (int idx = tid; idx < EPB * NGLL3; idx += NT) {
    const int s2 = blockIdx.x * EPB + idx / NGLL3;
    if (s2 < A.m.nspec) {
      const size_t ep = (size_t)A.m.order[s2] * NGLL3 + idx % NGLL3;
      s_ib[idx] = A.m.ibool[ep];
      s_kap[idx] = A.m.kappa[ep];
      s_mu[idx] = A.m.mu[ep];
    } else {
      s_ib[idx] = -1;
      s_kap[idx] = 0.f;
      s_mu[idx] = 0.f;
    }
  }
  __syncthreads();
  // cooperative gather of the displacement of every (field, element, lane)
#pragma unroll 1
  for (int f = 0; f < NF; ++f) {
    const float* src = f == 0 ? A.f1.u : A.f2.u;
    for (int idx = tid; idx < EPB * NGLL3 * 3 * LB; idx += NT) {
      const int ln = idx % LB;
      const int r = idx / LB;
      const int c = r % 3;
      const int r2 = r / 3;
      const int p = r2 % NGLL3;
      const int e2 = r2 / NGLL3;
      const int ig = s_ib[e2 * NGLL3 + p];
      const int l2 = blockIdx.y * LB + ln;
      float v = 0.f;
      if (ig >= 0 && s_act[f][ln]) v = src[A.fi((size_t)ig, c, l2)];
      sm[((f * EPB + e2) * PR_F + c * NGLL3 + p) * LB + ln] = v;
    }
  }
  __syncthreads();

  // gradients stay in reference coordinates: stress scale jac*xix*xix,
  // strain products scale xix^2
  const float fac = A.m.jac * A.m.xix * A.m.xix;
  const float dtk = A.dt * A.m.xix * A.m.xix;
  float* f1b = sm + ((0 * EPB + el) * PR_F) * LB + lane;
  float* f2b = sm + ((1 * EPB + el) * PR_F) * LB + lane;
  PencilBuf<LB> b1{f1b, f1b + PR_U * LB};
  PencilBuf<LB> b2{f2b, f2b + PR_U * LB};
  pencil_grad_eg<LB>(b1, t);
  if (ADJ) pencil_grad_eg<LB>(b2, t);
  __syncthreads();

  const float* kap = s_kap + el * NGLL3;
  const float* mu = s_mu + el * NGLL3;
  float fx1[5][3], fx2[ADJ ? 5 : 1][3];
  if (ADJ) {
    float g2[5][3][3];
    pencil_grad_xi<LB>(b2, t, g2);
    float e2v[5][6];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      const float tr = g2[i][0][0] + g2[i][1][1] + g2[i][2][2];
      e2v[i][0] = g2[i][0][0] - tr * (1.0f / 3.0f);
      e2v[i][1] = g2[i][1][1] - tr * (1.0f / 3.0f);
      e2v[i][2] = 0.5f * (g2[i][0][1] + g2[i][1][0]);
      e2v[i][3] = 0.5f * (g2[i][0][2] + g2[i][2][0]);
      e2v[i][4] = 0.5f * (g2[i][1][2] + g2[i][2][1]);
      e2v[i][5] = tr;
    }
    pencil_stress<LB>(b2, t, g2, kap, mu, fac, fx2);
    float g1[5][3][3];
    pencil_grad_xi<LB>(b1, t, g1);
    if (s_act[1][lane] && e < A.m.nspec) {
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        const float tr1 = g1[i][0][0] + g1[i][1][1] + g1[i][2][2];
        const float a_xx = g1[i][0][0] - tr1 * (1.0f / 3.0f);
        const float a_yy = g1[i][1][1] - tr1 * (1.0f / 3.0f);
        const float a_xy = 0.5f * (g1[i][0][1] + g1[i][1][0]);
        const float a_xz = 0.5f * (g1[i][0][2] + g1[i][2][0]);
        const float a_yz = 0.5f * (g1[i][1][2] + g1[i][2][1]);
        const float* bv = e2v[i];
        const float dd = a_xx * bv[0] + a_yy * bv[1] + (a_xx + a_yy) * (bv[0] + bv[1]) +
                         2.0f * (a_xy * bv[2] + a_xz * bv[3] + a_yz * bv[4]);
        const size_t q = A.ei((size_t)e * NGLL3 + i + 5 * t, lg);
        A.k.mu[q] += dtk * dd;
        A.k.kappa[q] += dtk * (tr1 * bv[5]);
      }
    }
    pencil_stress<LB>(b1, t, g1, kap, mu, fac, fx1);
  } else {
    float g1[5][3][3];
    pencil_grad_xi<LB>(b1, t, g1);
    pencil_stress<LB>(b1, t, g1, kap, mu, fac, fx1);
  }
  __syncthreads();
  pencil_div_eg<LB>(b1, t);
  if (ADJ) pencil_div_eg<LB>(b2, t);
  __syncthreads();
  if (e < A.m.nspec) {
    const int* ib = s_ib + el * NGLL3;
    constexpr int LWL = LB == 1 ? 0 : 3;
    if (s_act[0][lane]) pencil_scatter<LB>(b1, t, fx1, ib, A.f1.a + fbase<LWL>(A, lg));
    if (ADJ && scat2) pencil_scatter<LB>(b2, t, fx2, ib, A.f2.a + fbase<LWL>(A, lg));
  }
}

// ---------------------------------------------------------------------------
// element kernel, pencil decomposition, persistent and software-pipelined
// ---------------------------------------------------------------------------
//
// Persistent blocks walk element groups g, g + gridDim.x, ...  While group
// k is computed, cp.async (LDGSTS) copies already bring the displacement
// gather, kappa/mu and (adjoint) kernel accumulators of group k+1 and the
// ibool of group k+2 into shared memory, so the gather latency that stalls
// a one-shot element kernel overlaps the arithmetic of the previous group.

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
// Read-only global load into registers that were zeroed first, issued as
// a predicated load: nothing depends on the loaded value until it is used,
// so a prefetch made one work item ahead does not stall at the load.
__device__ __forceinline__ void ldg_pred(float& x, const float* g, bool ok) {
  x = 0.f;
  asm volatile(
      "{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %1, 0;\n\t@q ld.global.nc.f32 %0, [%2];\n\t}\n"
      : "+f"(x)
      : "r"((int)ok), "l"(g));
}
__device__ __forceinline__ void ldg_pred(float2& x, const float* g, bool ok) {
  x = make_float2(0.f, 0.f);
  asm volatile(
      "{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q ld.global.nc.v2.f32 {%0, %1}, "
      "[%3];\n\t}\n"
      : "+f"(x.x), "+f"(x.y)
      : "r"((int)ok), "l"(g));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// shared floats of the pipelined kernel per (field, element, lane)
constexpr int PP_U = 625;  // U (3 comps) then B (5 sigma comps)
constexpr int PP_A = 750;  // d_eta/d_gamma, then f_eta/f_gamma

// Region offsets are rounded up to 4 floats so that every region starts on
// a 16-byte boundary (float2 / float4 accesses and 16-byte cp.async).
constexpr int al4(int x) { return (x + 3) & ~3; }

template <int LB, int EPB, int TPE, bool ADJ>
struct PipeLayout {
  static constexpr int NF = ADJ ? 2 : 1;
  static constexpr int NE = EPB * NGLL3;                          // element points per group
  static constexpr int OFF_IB = 0;                                // int [3][NE]
  static constexpr int OFF_KM = al4(OFF_IB + 3 * NE);             // float [2][2][NE] kappa, mu
  static constexpr int OFF_U = al4(OFF_KM + 4 * NE);              // [2][NF][EPB][PP_U*LB]
  static constexpr int OFF_A = al4(OFF_U + 2 * NF * EPB * PP_U * LB);   // [NF][EPB][PP_A*LB]
  static constexpr int OFF_K = al4(OFF_A + NF * EPB * PP_A * LB);  // [2][2][NE*LB] mu/kappa acc
  static constexpr int TOTAL = OFF_K + (ADJ ? 4 * NE * LB : 0);
  static constexpr size_t BYTES = (size_t)TOTAL * 4;
};

// SMs a persistent element kernel of this run may fill: the run's share
// (sem_set_sm_share) or the whole device, so that runs of other meshes on
// other streams find room beside it.
__host__ __forceinline__ int sm_share(const StepArgs& a, int sms) {
  return (a.sm_limit > 0 && a.sm_limit < sms) ? a.sm_limit : sms;
}

// Work items are (lane chunk, element group) pairs walked chunk-major, so
// all resident blocks sweep the mesh for one group of event lanes at a
// time and the working set of shared GLL points stays in L2; the sub-chunks
// of one 32-byte sector of lanes (LB < 8) take adjacent items.
// With `gmap` (serving: only some 8-lane groups hold running events) the
// sector groups walked are gmap[0..nsg-1]; otherwise 0..nsg-1.
struct PipeItems {
  int ngroups, nchunk, spg;
  int nsg;              // sector groups walked
  const int* gmap;      // device list of active sector groups, or null
  int spg_log;          // spg = 1 << spg_log
  float inv_per;        // 1 / (ngroups * spg)
  __device__ __forceinline__ void decode(int w, int& chunk, int& g) const {
    // w / per by a float reciprocal, corrected to the exact quotient
    const int per = ngroups << spg_log;
    int k = __float2int_rz((float)w * inv_per);
    int rem = w - k * per;
    while (rem < 0) {
      --k;
      rem += per;
    }
    while (rem >= per) {
      ++k;
      rem -= per;
    }
    g = rem >> spg_log;
    const int sg = gmap ? gmap[k] : k;
    chunk = (sg << spg_log) + (rem & (spg - 1));
  }
  __host__ __device__ __forceinline__ int count() const { return nsg * spg * ngroups; }
};

// Work items of a launch: lane chunks of LB lanes, grouped by the 8-lane
// (32-byte) sector groups of the lane-group layout.
template <int LB>
static PipeItems make_items(const StepArgs& a, int ngroups) {
  PipeItems it;
  it.ngroups = ngroups;
  it.nchunk = (a.nev + LB - 1) / LB;
  const int lw = 1 << a.lm.lwlog;
  it.spg = (lw > LB && a.nev > LB) ? lw / LB : 1;
  const int nsg_all = (it.nchunk + it.spg - 1) / it.spg;
  it.gmap = a.gmap;
  it.nsg = a.gmap ? a.ngmap : nsg_all;
  it.spg_log = it.spg == 1 ? 0 : it.spg == 2 ? 1 : it.spg == 4 ? 2 : 3;
  it.inv_per = 1.0f / (float)(it.ngroups * it.spg);
  return it;
}

// The work items a persistent block has in flight, in shared memory: slot
// j & 3 holds item w + j * gridDim.x as (element, lane chunk).  One thread
// decodes an item three iterations before it is computed and fetches its
// element id from the traversal order by cp.async, so the copies that need
// the id are addressed without a dependent global load on the way.
struct ItemRing {
  int* e;  // [4] element; nspec past the end of the items
  int* c;  // [4] lane chunk; items.nchunk past the end
  __device__ __forceinline__ void fill(const PipeItems& items, const int* order, int nspec, int w,
                                       int slot) const {
    if (w < items.count()) {
      int chunk, g;
      items.decode(w, chunk, g);  // g < items.ngroups, the length of order
      c[slot] = chunk;
      cp_async4(e + slot, order + g);
    } else {
      c[slot] = items.nchunk;
      e[slot] = nspec;
    }
  }
};

template <int LB, int EPB, int TPE, bool ADJ>
__global__ void __launch_bounds__(EPB * TPE * LB) k_forces_piped(StepArgs A, PipeItems items) {
  using LY = PipeLayout<LB, EPB, TPE, ADJ>;
  constexpr int NT = EPB * TPE * LB;
  constexpr int NE = LY::NE;
  constexpr int NF = LY::NF;
  extern __shared__ float sm[];
  int* sIB = (int*)(sm + LY::OFF_IB);
  float* sKM = sm + LY::OFF_KM;
  float* sU = sm + LY::OFF_U;
  float* sA = sm + LY::OFF_A;
  float* sK = sm + LY::OFF_K;

  const int tid = threadIdx.x;
  const int lane = tid % LB;
  const int t = (tid / LB) % TPE;
  const int el = tid / (TPE * LB);
  const bool pen = t < 25;
  const int nev = A.nev;
  const int nspec = A.m.nspec;
  const int nitems = items.count();

  // whole launch idle (every lane finished or parked): nothing to do
  bool any = false;
  for (int l = tid; l < nev; l += NT) {
    const LaneDesc* L = A.lanes + l;
    any |= L->phase != PH_IDLE && L->it0 + A.s < L->nstep;
  }
  if (!__syncthreads_or(any)) return;

  constexpr int LWLOG = LB == 1 ? 0 : 3;
  if (A.lm.lwlog != LWLOG) return;  // launched only with the matching layout

  // lane state of this thread for item w: bit0 active, bit1 adjoint field,
  // bit2 adjoint scatter; cached per lane chunk (fixed within a launch)
  int c_chunk = -1, c_flag = 0;
  auto flags = [&](int w, int& lg, int& g) -> int {
    int chunk;
    items.decode(w, chunk, g);
    lg = chunk * LB + lane;
    if (chunk == c_chunk) return c_flag;
    int f = 0;
    if (chunk < items.nchunk && lg < nev) {
      const LaneDesc* L = A.lanes + lg;
      const int it = L->it0 + A.s;
      if (L->phase != PH_IDLE && it < L->nstep) {
        f = 1;
        if (ADJ && L->phase == PH_ADJ) f |= 2 | (it > 0 ? 4 : 0);
      }
    }
    c_chunk = chunk;
    c_flag = f;
    return f;
  };
  auto issue_ib = [&](int w, int slot) {
    int* dst = sIB + slot * NE;
    int chunk = 0, g = 0;
    if (w < nitems) items.decode(w, chunk, g);
    for (int i = tid; i < NE; i += NT) {
      const int es = g * EPB + i / NGLL3;
      if (w < nitems && es < nspec)
        cp_async4(dst + i, A.m.ibool + (size_t)A.m.order[es] * NGLL3 + i % NGLL3);
      else
        dst[i] = -1;
    }
  };
  auto issue_data = [&](int w, int ibslot, int buf) {
    if (w >= nitems) return;
    int lg, g;
    const int fl = flags(w, lg, g);
    const int* ib = sIB + ibslot * NE;
    float* km = sKM + buf * 2 * NE;
    for (int i = tid; i < NE; i += NT) {
      const int es = g * EPB + i / NGLL3;
      if (es < nspec) {
        const size_t ep = (size_t)A.m.order[es] * NGLL3 + i % NGLL3;
        cp_async4(km + i, A.m.kappa + ep);
        cp_async4(km + NE + i, A.m.mu + ep);
      }
    }
    if (pen) {
      const size_t fb = fbase<LWLOG>(A, lg);
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const bool act = f == 0 ? (fl & 1) : (fl & 2);
        const float* src = (f == 0 ? A.f1.u : A.f2.u) + fb;
        float* ub = sU + (((buf * NF + f) * EPB + el) * PP_U) * LB + lane;
#pragma unroll
        for (int r = 0; r < 5; ++r) {
          const int p = t + 25 * r;
          const int ig = ib[el * NGLL3 + p];
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            float* d = ub + (c * NGLL3 + p) * LB;
            if (act && ig >= 0)
              cp_async4(d, src + foff<LWLOG>(ig, c));
            else
              *d = 0.f;
          }
        }
      }
      if (ADJ && (fl & 2)) {
        const int es = g * EPB + el;
        float* kb = sK + buf * 2 * NE * LB;
        if (es < nspec) {
          const size_t eb = ebase<LWLOG>(A, lg) + (((size_t)A.m.order[es] * NGLL3) << LWLOG);
#pragma unroll
          for (int r = 0; r < 5; ++r) {
            const int p = t + 25 * r;
            const size_t q = eb + ((size_t)p << LWLOG);
            cp_async4(kb + (el * NGLL3 + p) * LB + lane, A.k.mu + q);
            cp_async4(kb + (NE + el * NGLL3 + p) * LB + lane, A.k.kappa + q);
          }
        }
      }
    }
  };

  // ---- prologue --------------------------------------------------------------
  int w = blockIdx.x;
  issue_ib(w, 0);
  cp_commit();
  cp_wait_all();
  __syncthreads();
  issue_data(w, 0, 0);
  issue_ib(w + gridDim.x, 1);
  cp_commit();

  // gradients stay in reference coordinates: stress scale jac*xix*xix,
  // strain products scale xix^2
  const float fac = A.m.jac * A.m.xix * A.m.xix;
  const float dtk = A.dt * A.m.xix * A.m.xix;
  for (int k = 0; w < nitems; ++k, w += gridDim.x) {
    const int buf = k & 1;
    const int ibs = k % 3;
    cp_wait_all();
    __syncthreads();
    // prefetch the next item while this one is computed
    issue_data(w + gridDim.x, (k + 1) % 3, buf ^ 1);
    issue_ib(w + 2 * gridDim.x, (k + 2) % 3);
    cp_commit();

    int lg, g;
    const int fl = flags(w, lg, g);
    const bool act1 = fl & 1, act2 = ADJ && (fl & 2), scat2 = ADJ && (fl & 4);
    const int es = g * EPB + el;
    const int e = es < nspec ? A.m.order[es] : nspec;
    const float* kap = sKM + buf * 2 * NE + el * NGLL3;
    const float* mu = kap + NE;
    float* u1 = sU + (((buf * NF + 0) * EPB + el) * PP_U) * LB + lane;
    float* u2 = sU + (((buf * NF + (NF - 1)) * EPB + el) * PP_U) * LB + lane;
    float* a1 = sA + ((0 * EPB + el) * PP_A) * LB + lane;
    float* a2 = sA + (((NF - 1) * EPB + el) * PP_A) * LB + lane;
    PencilBuf<LB> b1{u1, a1};
    PencilBuf<LB> b2{u2, a2};
    if (pen) {
      pencil_grad_eg<LB>(b1, t);
      if (ADJ) pencil_grad_eg<LB>(b2, t);
    }
    __syncthreads();
    float fx1[5][3], fx2[ADJ ? 5 : 1][3];
    if (pen) {
      if (ADJ) {
        float g2[5][3][3];
        pencil_grad_xi<LB>(b2, t, g2);
        float e2v[5][6];
#pragma unroll
        for (int i = 0; i < 5; ++i) {
          const float tr = g2[i][0][0] + g2[i][1][1] + g2[i][2][2];
          e2v[i][0] = g2[i][0][0] - tr * (1.0f / 3.0f);
          e2v[i][1] = g2[i][1][1] - tr * (1.0f / 3.0f);
          e2v[i][2] = 0.5f * (g2[i][0][1] + g2[i][1][0]);
          e2v[i][3] = 0.5f * (g2[i][0][2] + g2[i][2][0]);
          e2v[i][4] = 0.5f * (g2[i][1][2] + g2[i][2][1]);
          e2v[i][5] = tr;
        }
        pencil_stress<LB>(b2, t, g2, kap, mu, fac, fx2);
        float g1[5][3][3];
        pencil_grad_xi<LB>(b1, t, g1);
        if (act2 && e < nspec) {
          const float* kb = sK + buf * 2 * NE * LB;
#pragma unroll
          for (int i = 0; i < 5; ++i) {
            const float tr1 = g1[i][0][0] + g1[i][1][1] + g1[i][2][2];
            const float a_xx = g1[i][0][0] - tr1 * (1.0f / 3.0f);
            const float a_yy = g1[i][1][1] - tr1 * (1.0f / 3.0f);
            const float a_xy = 0.5f * (g1[i][0][1] + g1[i][1][0]);
            const float a_xz = 0.5f * (g1[i][0][2] + g1[i][2][0]);
            const float a_yz = 0.5f * (g1[i][1][2] + g1[i][2][1]);
            const float* bv = e2v[i];
            const float dd = a_xx * bv[0] + a_yy * bv[1] + (a_xx + a_yy) * (bv[0] + bv[1]) +
                             2.0f * (a_xy * bv[2] + a_xz * bv[3] + a_yz * bv[4]);
            const int p = i + 5 * t;
            const size_t q = ebase<LWLOG>(A, lg) + (((size_t)e * NGLL3 + p) << LWLOG);
            A.k.mu[q] = kb[(el * NGLL3 + p) * LB + lane] + dtk * dd;
            A.k.kappa[q] = kb[(NE + el * NGLL3 + p) * LB + lane] + dtk * (tr1 * bv[5]);
          }
        }
        pencil_stress<LB>(b1, t, g1, kap, mu, fac, fx1);
      } else {
        float g1[5][3][3];
        pencil_grad_xi<LB>(b1, t, g1);
        pencil_stress<LB>(b1, t, g1, kap, mu, fac, fx1);
      }
    }
    __syncthreads();
    if (pen) {
      pencil_div_eg<LB>(b1, t);
      if (ADJ) pencil_div_eg<LB>(b2, t);
    }
    __syncthreads();
    if (pen && e < nspec) {
      const int* ib = sIB + ibs * NE + el * NGLL3;
      if (act1) pencil_scatter<LB>(b1, t, fx1, ib, A.f1.a + fbase<LWLOG>(A, lg));
      if (ADJ && scat2) pencil_scatter<LB>(b2, t, fx2, ib, A.f2.a + fbase<LWLOG>(A, lg));
    }
  }
  cp_wait_all();
}

template <int LB, int EPB, int TPE, bool ADJ>
static void forces_piped_cfg(const StepArgs& a, cudaStream_t st) {
  using LY = PipeLayout<LB, EPB, TPE, ADJ>;
  constexpr int NT = EPB * TPE * LB;
  static int blocks_per_sm = 0, sms = 0;
  if (!blocks_per_sm) {
    cudaFuncSetAttribute(k_forces_piped<LB, EPB, TPE, ADJ>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LY::BYTES);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm,
                                                  k_forces_piped<LB, EPB, TPE, ADJ>, NT,
                                                  LY::BYTES);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (blocks_per_sm < 1) blocks_per_sm = 1;
  }
  PipeItems items = make_items<LB>(a, (a.m.nspec + EPB - 1) / EPB);
  if (items.count() == 0) return;
  int gx = blocks_per_sm * sm_share(a, sms);
  if (gx > items.count()) gx = items.count();
  if (gx < 1) gx = 1;
  k_forces_piped<LB, EPB, TPE, ADJ><<<gx, NT, LY::BYTES, st>>>(a, items);
}

template <int LB, int EPB, bool ADJ>
static void forces_pencil_cfg(const StepArgs& a, cudaStream_t st) {
  const size_t shm = (size_t)(ADJ ? 2 : 1) * EPB * PR_F * LB * sizeof(float);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_forces_pencil<LB, EPB, ADJ>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    attr = true;
  }
  dim3 grid((a.m.nspec + EPB - 1) / EPB, (a.nev + LB - 1) / LB);
  k_forces_pencil<LB, EPB, ADJ><<<grid, EPB * 25 * LB, shm, st>>>(a);
}

template <int LB, int NT, bool ADJ, bool GEN = false>
static void forces_cfg(const StepArgs& a, cudaStream_t st) {
  const size_t shm = (size_t)(ADJ ? 2 : 1) * (GEN ? 9 : 6) * NGLL3 * LB * sizeof(float);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_forces<LB, NT, ADJ, GEN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)shm);
    attr = true;
  }
  dim3 grid(a.m.nspec, (a.nev + LB - 1) / LB);
  k_forces<LB, NT, ADJ, GEN><<<grid, NT, shm, st>>>(a);
}

// ---------------------------------------------------------------------------
// element kernel, pencil decomposition with NL event lanes per thread
// ---------------------------------------------------------------------------
//
// As k_forces_piped, but each thread carries NL adjacent event lanes of its
// pencil: shared-memory traffic moves as float2/float4 (one LDS/STS per NL
// values), the gather as NL*4-byte cp.async, the scatter as vector atomics,
// and every index computation is shared by the NL lanes.  The xi role also
// fuses gradient and stress point by point so that only one point's nine
// derivatives are live at a time.  In the adjoint phase the backward
// field's strain is parked in its own A region (the xi role reads and
// rewrites only its own pencil there) until the adjoint field's strain
// at the same point is ready for the kernel products.

template <int NL>
struct LV {
  float v[NL];
};

template <int NL>
__device__ __forceinline__ LV<NL> lds_v(const float* p) {
  LV<NL> r;
  if constexpr (NL == 1) {
    r.v[0] = *p;
  } else if constexpr (NL == 2) {
    const float2 t = *reinterpret_cast<const float2*>(p);
    r.v[0] = t.x;
    r.v[1] = t.y;
  } else {
    const float4 t = *reinterpret_cast<const float4*>(p);
    r.v[0] = t.x;
    r.v[1] = t.y;
    r.v[2] = t.z;
    r.v[3] = t.w;
  }
  return r;
}

template <int NL>
__device__ __forceinline__ void sts_v(float* p, const LV<NL>& x) {
  if constexpr (NL == 1) {
    *p = x.v[0];
  } else if constexpr (NL == 2) {
    *reinterpret_cast<float2*>(p) = make_float2(x.v[0], x.v[1]);
  } else {
    *reinterpret_cast<float4*>(p) = make_float4(x.v[0], x.v[1], x.v[2], x.v[3]);
  }
}

template <int NL>
__device__ __forceinline__ void cp_async_v(float* smem, const float* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if constexpr (NL == 1)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
  else if constexpr (NL == 2)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

template <int NL>
__device__ __forceinline__ void red_v(float* g, const LV<NL>& x) {
  if constexpr (NL == 1) {
    atomicAdd(g, x.v[0]);
  } else if constexpr (NL == 2) {
    atomicAdd(reinterpret_cast<float2*>(g), make_float2(x.v[0], x.v[1]));
  } else {
    atomicAdd(reinterpret_cast<float4*>(g), make_float4(x.v[0], x.v[1], x.v[2], x.v[3]));
  }
}

// Packed FP32x2 arithmetic (Blackwell f32x2): two values that share a GLL
// coefficient - two events of one thread, or the adjoint and backward
// fields of one event - advance with one instruction issue.  fma.rn on
// each half, so the results are those of the scalar FMAs.
__device__ __forceinline__ float2 p2(const LV<2>& x) { return make_float2(x.v[0], x.v[1]); }
__device__ __forceinline__ LV<2> lv2(float2 x) {
  LV<2> r;
  r.v[0] = x.x;
  r.v[1] = x.y;
  return r;
}
__device__ __forceinline__ float2 splat(float c) { return make_float2(c, c); }
// a + c x for a compile-time GLL coefficient c (c = 0: no instruction)
__device__ __forceinline__ float2 cfma2(float c, float2 x, float2 a) {
  return c == 0.0f ? a : __ffma2_rn(splat(c), x, a);
}
// Isotropic stress times fac of two gradients sharing kappa and mu:
// sig = {xx, yy, zz, xy, xz, yz}.
__device__ __forceinline__ void stress_point2(const float2 g[3][3], float kap, float mu,
                                              float fac, float2 sig[6]) {
  const float l2m = kap + (4.0f / 3.0f) * mu;
  const float lam = l2m - 2.0f * mu;
  const float2 L = splat(l2m), M = splat(lam), F = splat(fac), MU = splat(fac * mu);
  sig[0] = __fmul2_rn(F, __ffma2_rn(L, g[0][0], __fmul2_rn(M, __fadd2_rn(g[1][1], g[2][2]))));
  sig[1] = __fmul2_rn(F, __ffma2_rn(L, g[1][1], __fmul2_rn(M, __fadd2_rn(g[0][0], g[2][2]))));
  sig[2] = __fmul2_rn(F, __ffma2_rn(L, g[2][2], __fmul2_rn(M, __fadd2_rn(g[0][0], g[1][1]))));
  sig[3] = __fmul2_rn(MU, __fadd2_rn(g[0][1], g[1][0]));
  sig[4] = __fmul2_rn(MU, __fadd2_rn(g[0][2], g[2][0]));
  sig[5] = __fmul2_rn(MU, __fadd2_rn(g[1][2], g[2][1]));
}

// Mapping of GLL point p of a general element: xix, xiy, xiz, etax, etay,
// etaz, gammax, gammay, gammaz, jacobian (geo_e = the element's row of the
// mesh's per-point mapping, 8-byte aligned), or the regular element's
// diagonal mapping when geo_e is null.
__device__ __forceinline__ void load_geo(const float* geo_e, int p, float xix, float jac,
                                         float G[10]) {
  if (geo_e) {
    const float2* q = reinterpret_cast<const float2*>(geo_e + p * 10);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      const float2 v = __ldg(q + k);
      G[2 * k] = v.x;
      G[2 * k + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int k = 0; k < 9; ++k) G[k] = (k % 4 == 0) ? xix : 0.f;
    G[9] = jac;
  }
}

// Shared block of one (field, element): U/B region then A region, each
// value a run of LB lanes; `ub`/`ab` already include the thread's lane
// offset.
template <int LB>
struct PBuf {
  float* ub;
  float* ab;
  __device__ __forceinline__ float* U(int q, int p) const { return ub + (q * 125 + p) * LB; }
  __device__ __forceinline__ float* Ar(int q, int p) const { return ab + (q * 125 + p) * LB; }
};

// eta / gamma derivative roles (pencils (i,k) and (i,j) of thread t);
// GAMMA false: the eta role only (the gamma role taken from registers by
// grad_gamma_regs).
template <int LB, int NL, bool GAMMA = true>
__device__ __forceinline__ void v_grad_eg(const PBuf<LB>& b, int pi, int pq) {
  if constexpr (NL == 2) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float2 v[5];
#pragma unroll
      for (int l = 0; l < 5; ++l) v[l] = p2(lds_v<2>(b.U(c, pi + 5 * l + 25 * pq)));
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        float2 a = make_float2(0.f, 0.f);
#pragma unroll
        for (int l = 0; l < 5; ++l) a = cfma2(gD(j, l), v[l], a);
        sts_v<2>(b.Ar(c, pi + 5 * j + 25 * pq), lv2(a));
      }
    }
    if constexpr (GAMMA) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float2 v[5];
#pragma unroll
      for (int l = 0; l < 5; ++l) v[l] = p2(lds_v<2>(b.U(c, pi + 5 * pq + 25 * l)));
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        float2 a = make_float2(0.f, 0.f);
#pragma unroll
        for (int l = 0; l < 5; ++l) a = cfma2(gD(k, l), v[l], a);
        sts_v<2>(b.Ar(3 + c, pi + 5 * pq + 25 * k), lv2(a));
      }
    }
    }
  } else {
    static_assert(GAMMA, "the eta-only role is packed (NL == 2)");
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      LV<NL> v[5];
#pragma unroll
      for (int l = 0; l < 5; ++l) v[l] = lds_v<NL>(b.U(c, pi + 5 * l + 25 * pq));
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        LV<NL> s;
#pragma unroll
        for (int n = 0; n < NL; ++n) {
          float a = 0.f;
#pragma unroll
          for (int l = 0; l < 5; ++l) a = cfma(gD(j, l), v[l].v[n], a);
          s.v[n] = a;
        }
        sts_v<NL>(b.Ar(c, pi + 5 * j + 25 * pq), s);
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      LV<NL> v[5];
#pragma unroll
      for (int l = 0; l < 5; ++l) v[l] = lds_v<NL>(b.U(c, pi + 5 * pq + 25 * l));
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        LV<NL> s;
#pragma unroll
        for (int n = 0; n < NL; ++n) {
          float a = 0.f;
#pragma unroll
          for (int l = 0; l < 5; ++l) a = cfma(gD(k, l), v[l].v[n], a);
          s.v[n] = a;
        }
        sts_v<NL>(b.Ar(3 + c, pi + 5 * pq + 25 * k), s);
      }
    }
  }
}

// Gamma derivative role from registers: thread t's gamma pencil (points
// t + 25 l, l = 0..4) is the displacement it gathered itself, v[l][c], so
// its derivatives need no shared-memory loads.
template <int LB>
__device__ __forceinline__ void grad_gamma_regs(const PBuf<LB>& b, int t, const float2 v[5][3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      float2 a = make_float2(0.f, 0.f);
#pragma unroll
      for (int l = 0; l < 5; ++l) a = cfma2(gD(k, l), v[l][c], a);
      sts_v<2>(b.Ar(3 + c, t + 25 * k), lv2(a));
    }
}

// eta / gamma divergence roles: B -> A.
template <int LB, int NL, bool GEN = false>
__device__ __forceinline__ void v_div_eg(const PBuf<LB>& b, int pi, int pq) {
  if constexpr (NL == 2) {
    {
      float2 v[3][5];
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        const int p = pi + 5 * l + 25 * pq;
        v[0][l] = p2(lds_v<2>(b.U(0, p)));
        v[1][l] = p2(lds_v<2>(b.U(1, p)));
        v[2][l] = p2(lds_v<2>(b.U(2, p)));
      }
#pragma unroll
      for (int j = 0; j < 5; ++j)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float2 a = make_float2(0.f, 0.f);
#pragma unroll
          for (int l = 0; l < 5; ++l) a = cfma2(gDWt(j, l), v[c][l], a);
          sts_v<2>(b.Ar(c, pi + 5 * j + 25 * pq), lv2(a));
        }
    }
    {
      float2 v[3][5];
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        const int p = pi + 5 * pq + 25 * l;
        v[0][l] = p2(lds_v<2>(b.U(3, p)));
        v[1][l] = p2(lds_v<2>(b.U(GEN ? 4 : 2, p)));
        v[2][l] = p2(lds_v<2>(b.U(GEN ? 5 : 4, p)));
      }
#pragma unroll
      for (int k = 0; k < 5; ++k)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float2 a = make_float2(0.f, 0.f);
#pragma unroll
          for (int l = 0; l < 5; ++l) a = cfma2(gDWt(k, l), v[c][l], a);
          sts_v<2>(b.Ar(3 + c, pi + 5 * pq + 25 * k), lv2(a));
        }
    }
  } else {
    {
      // eta pencil: sigma_{c,y} = (xy, yy, yz) = B0, B1, B2
      LV<NL> v[3][5];
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        const int p = pi + 5 * l + 25 * pq;
        v[0][l] = lds_v<NL>(b.U(0, p));
        v[1][l] = lds_v<NL>(b.U(1, p));
        v[2][l] = lds_v<NL>(b.U(2, p));
      }
#pragma unroll
      for (int j = 0; j < 5; ++j)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          LV<NL> s;
#pragma unroll
          for (int n = 0; n < NL; ++n) {
            float a = 0.f;
#pragma unroll
            for (int l = 0; l < 5; ++l) a = cfma(gDWt(j, l), v[c][l].v[n], a);
            s.v[n] = a;
          }
          sts_v<NL>(b.Ar(c, pi + 5 * j + 25 * pq), s);
        }
    }
    {
      // gamma pencil: sigma_{c,z} = (xz, yz, zz) = B3, B2, B4; general
      // elements: the gamma fluxes of the three components, B3, B4, B5
      LV<NL> v[3][5];
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        const int p = pi + 5 * pq + 25 * l;
        v[0][l] = lds_v<NL>(b.U(3, p));
        v[1][l] = lds_v<NL>(b.U(GEN ? 4 : 2, p));
        v[2][l] = lds_v<NL>(b.U(GEN ? 5 : 4, p));
      }
#pragma unroll
      for (int k = 0; k < 5; ++k)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          LV<NL> s;
#pragma unroll
          for (int n = 0; n < NL; ++n) {
            float a = 0.f;
#pragma unroll
            for (int l = 0; l < 5; ++l) a = cfma(gDWt(k, l), v[c][l].v[n], a);
            s.v[n] = a;
          }
          sts_v<NL>(b.Ar(3 + c, pi + 5 * pq + 25 * k), s);
        }
    }
  }
}

// xi role on pencil t (points p = i + 5t): gradient and stress point by
// point; sigma for the other roles into B; f_xi into fx.
// MODE 0: plain.  MODE 1: backward field of the adjoint phase; its
// deviatoric strain and trace are parked in its own A region at the
// pencil's points.  MODE 2: adjoint field; the products with the parked
// backward strain (read from `park`) are returned in kmu / kka.
// GEN: general elements.  The derivatives are mapped with the point's
// mapping, the stress is formed without scale, and the xi role keeps the
// xi fluxes J sigma_c . grad(xi) while the eta and gamma fluxes of the
// three components go to B0..B2 and B3..B5; the strains of MODE 1 / 2 are
// the physical ones (the caller's kernel-product scale is dt alone).
template <int LB, int NL, int MODE, bool GEN = false>
__device__ __forceinline__ void v_xi(const PBuf<LB>& b, const PBuf<LB>& park, int t,
                                     const float* kap, const float* mu, float fac,
                                     LV<NL> fx[5][3], LV<NL> kmu[5], LV<NL> kka[5],
                                     const float* geo_e = nullptr, float xix = 0.f,
                                     float jac = 0.f) {
  if constexpr (NL == 2 && MODE == 0 && !GEN) {
    float2 u[3][5];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int l = 0; l < 5; ++l) u[c][l] = p2(lds_v<2>(b.U(c, l + 5 * t)));
    float2 sx[3][5];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      const int p = i + 5 * t;
      float2 g[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float2 a = make_float2(0.f, 0.f);
#pragma unroll
        for (int l = 0; l < 5; ++l) a = cfma2(gD(i, l), u[c][l], a);
        g[c][0] = a;
        g[c][1] = p2(lds_v<2>(b.Ar(c, p)));
        g[c][2] = p2(lds_v<2>(b.Ar(3 + c, p)));
      }
      float2 sig[6];
      stress_point2(g, kap[p], mu[p], fac, sig);
      sx[0][i] = sig[0];
      sx[1][i] = sig[3];
      sx[2][i] = sig[4];
      sts_v<2>(b.U(0, p), lv2(sig[3]));
      sts_v<2>(b.U(1, p), lv2(sig[1]));
      sts_v<2>(b.U(2, p), lv2(sig[5]));
      sts_v<2>(b.U(3, p), lv2(sig[4]));
      sts_v<2>(b.U(4, p), lv2(sig[2]));
    }
#pragma unroll
    for (int i = 0; i < 5; ++i)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float2 a = make_float2(0.f, 0.f);
#pragma unroll
        for (int l = 0; l < 5; ++l) a = cfma2(gDWt(i, l), sx[c][l], a);
        fx[i][c] = lv2(a);
      }
  } else {
    LV<NL> u[3][5];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int l = 0; l < 5; ++l) u[c][l] = lds_v<NL>(b.U(c, l + 5 * t));
    LV<NL> sx[3][5];  // sigma_xx, sigma_xy, sigma_xz along the pencil
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      const int p = i + 5 * t;
      LV<NL> de[3], dg[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        de[c] = lds_v<NL>(b.Ar(c, p));
        dg[c] = lds_v<NL>(b.Ar(3 + c, p));
      }
      LV<NL> pk[6];
      if (MODE == 2) {
#pragma unroll
        for (int q = 0; q < 6; ++q) pk[q] = lds_v<NL>(park.Ar(q, p));
      }
      constexpr int NO = GEN ? 6 : 5;
      LV<NL> o[NO];
      const float kp = kap[p], m = mu[p];
      float G[10];
      if (GEN) load_geo(geo_e, p, xix, jac, G);
#pragma unroll
      for (int n = 0; n < NL; ++n) {
        float g[3][3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float a = 0.f;
#pragma unroll
          for (int l = 0; l < 5; ++l) a = cfma(gD(i, l), u[c][l].v[n], a);
          g[c][0] = a;
          g[c][1] = de[c].v[n];
          g[c][2] = dg[c].v[n];
        }
        if constexpr (GEN) {
          float r[3][3];
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int d = 0; d < 3; ++d) r[c][d] = g[c][d];
          map_gradient(r, G, g);
          float sig[6], F[9];
          stress_point(g, kp, m, 1.0f, sig);
          map_flux(sig, G, F);
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            sx[c][i].v[n] = F[c * 3 + 0];
            o[c].v[n] = F[c * 3 + 1];
            o[3 + c].v[n] = F[c * 3 + 2];
          }
        } else {
          float sig[6];
          stress_point(g, kp, m, fac, sig);
          sx[0][i].v[n] = sig[0];
          sx[1][i].v[n] = sig[3];
          sx[2][i].v[n] = sig[4];
          o[0].v[n] = sig[3];
          o[1].v[n] = sig[1];
          o[2].v[n] = sig[5];
          o[3].v[n] = sig[4];
          o[4].v[n] = sig[2];
        }
        if (MODE != 0) {
          const float tr = g[0][0] + g[1][1] + g[2][2];
          const float xx = g[0][0] - tr * (1.0f / 3.0f);
          const float yy = g[1][1] - tr * (1.0f / 3.0f);
          const float xy = 0.5f * (g[0][1] + g[1][0]);
          const float xz = 0.5f * (g[0][2] + g[2][0]);
          const float yz = 0.5f * (g[1][2] + g[2][1]);
          if (MODE == 1) {
            pk[0].v[n] = xx;
            pk[1].v[n] = yy;
            pk[2].v[n] = xy;
            pk[3].v[n] = xz;
            pk[4].v[n] = yz;
            pk[5].v[n] = tr;
          } else {
            const float bxx = pk[0].v[n], byy = pk[1].v[n];
            kmu[i].v[n] = xx * bxx + yy * byy + (xx + yy) * (bxx + byy) +
                          2.0f * (xy * pk[2].v[n] + xz * pk[3].v[n] + yz * pk[4].v[n]);
            kka[i].v[n] = tr * pk[5].v[n];
          }
        }
      }
#pragma unroll
      for (int q = 0; q < NO; ++q) sts_v<NL>(b.U(q, p), o[q]);
      if (MODE == 1) {
#pragma unroll
        for (int q = 0; q < 6; ++q) sts_v<NL>(b.Ar(q, p), pk[q]);
      }
    }
#pragma unroll
    for (int i = 0; i < 5; ++i)
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int n = 0; n < NL; ++n) {
          float a = 0.f;
#pragma unroll
          for (int l = 0; l < 5; ++l) a = cfma(gDWt(i, l), sx[c][l].v[n], a);
          fx[i][c].v[n] = a;
        }
  }
}

// xi role: total force on the pencil and vector scatter-add.
// Plain read-modify-write of NL consecutive floats, for colour-ordered
// launches in which no other thread touches the same point.
template <int NL>
__device__ __forceinline__ void rmw_v(float* g, const LV<NL>& x) {
  if constexpr (NL == 1) {
    *g += x.v[0];
  } else if constexpr (NL == 2) {
    float2* q = reinterpret_cast<float2*>(g);
    float2 o = *q;
    o.x += x.v[0];
    o.y += x.v[1];
    *q = o;
  } else {
    float4* q = reinterpret_cast<float4*>(g);
    float4 o = *q;
    o.x += x.v[0];
    o.y += x.v[1];
    o.z += x.v[2];
    o.w += x.v[3];
    *q = o;
  }
}

template <int LB, int NL, bool ATOMIC = true>
__device__ __forceinline__ void v_scatter(const PBuf<LB>& b, int t, const LV<NL> fx[5][3],
                                          const int* ib, float* accb, const int* fl, int bit) {
  const int pj = t % 5, pk = t / 5;
  float wj = 0.f, wk = 0.f;
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    if (q == pj) wj = gW(q);
    if (q == pk) wk = gW(q);
  }
  const float wjk = wj * wk;
  if constexpr (NL == 2) {
    const float2 njk = splat(-wjk);
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      const int p = i + 5 * t;
      const size_t ig = (size_t)ib[p];
      const float2 nik = splat(-(gW(i) * wk)), nij = splat(-(gW(i) * wj));
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float2 e1 = p2(lds_v<2>(b.Ar(c, p)));
        const float2 e2 = p2(lds_v<2>(b.Ar(3 + c, p)));
        float2 v = __ffma2_rn(nij, e2, __ffma2_rn(nik, e1, __fmul2_rn(njk, p2(fx[i][c]))));
        // lanes not in this phase add nothing
        LV<2> f;
        f.v[0] = (fl[0] & bit) ? v.x : 0.f;
        f.v[1] = (fl[1] & bit) ? v.y : 0.f;
        if constexpr (ATOMIC)
          red_v<2>(&accb[foff<3>((int)ig, c)], f);
        else
          rmw_v<2>(&accb[foff<3>((int)ig, c)], f);
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      const int p = i + 5 * t;
      const size_t ig = (size_t)ib[p];
      const float wik = gW(i) * wk, wij = gW(i) * wj;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const LV<NL> e1 = lds_v<NL>(b.Ar(c, p));
        const LV<NL> e2 = lds_v<NL>(b.Ar(3 + c, p));
        LV<NL> f;
#pragma unroll
        for (int n = 0; n < NL; ++n) {
          const float v = -(wjk * fx[i][c].v[n] + wik * e1.v[n] + wij * e2.v[n]);
          f.v[n] = (fl[n] & bit) ? v : 0.f;  // lanes not in this phase add nothing
        }
        if constexpr (ATOMIC)
          red_v<NL>(&accb[foff<3>((int)ig, c)], f);
        else
          rmw_v<NL>(&accb[foff<3>((int)ig, c)], f);
      }
    }
  }
}

// One block = one element x LB lanes, 25 * LB / NL threads (pencil t,
// lane group of NL).  Persistent and cp.async-pipelined like
// k_forces_piped, with the same chunk-major work items.
template <int LB, int NL, bool ADJ>
__global__ void __launch_bounds__(25 * LB / NL) k_forces_vec(StepArgs A, PipeItems items) {
  constexpr int NT = 25 * LB / NL;
  constexpr int NF = ADJ ? 2 : 1;
  using LY = PipeLayout<LB, 1, 25, ADJ>;
  constexpr int NE = LY::NE;
  extern __shared__ float sm[];
  int* sIB = (int*)(sm + LY::OFF_IB);
  float* sKM = sm + LY::OFF_KM;
  float* sU = sm + LY::OFF_U;
  float* sA = sm + LY::OFF_A;
  float* sK = sm + LY::OFF_K;

  const int tid = threadIdx.x;
  const int lq = tid % (LB / NL);      // lane group within the block
  const int t = tid / (LB / NL);       // pencil 0..24
  const int lane = lq * NL;            // first lane of the group
  const int pi = t % 5, pq = t / 5;
  const int nev = A.nev;
  const int nspec = A.m.nspec;
  const int nitems = items.count();

  bool any = false;
  for (int l = tid; l < nev; l += NT) {
    const LaneDesc* L = A.lanes + l;
    any |= L->phase != PH_IDLE && L->it0 + A.s < L->nstep;
  }
  if (!__syncthreads_or(any)) return;

  // Lane flags are per NL-group: lanes of a group share a phase in
  // lock-step runs; in mixed batches a group is active if its first
  // lane is, and per-lane activity masks the writes.
  auto lane_flag = [&](int lg) -> int {
    if (lg >= nev) return 0;
    const LaneDesc* L = A.lanes + lg;
    const int it = L->it0 + A.s;
    if (L->phase == PH_IDLE || it >= L->nstep) return 0;
    int f = 1;
    if (ADJ && L->phase == PH_ADJ) f |= 2 | (it > 0 ? 4 : 0);
    return f;
  };
  constexpr int LWLOG = 3;
  if (A.lm.lwlog != LWLOG) return;  // batched layout only
  int c_chunk = -1, c_any = 0, c_fl[NL];
#pragma unroll
  for (int n = 0; n < NL; ++n) c_fl[n] = 0;
  // flags of the NL lanes of item w, cached per lane chunk
  auto group_flags = [&](int w, int& lg0, int& g, int fl[NL]) {
    int chunk;
    items.decode(w, chunk, g);
    lg0 = chunk * LB + lane;
    if (chunk != c_chunk) {
      c_any = 0;
#pragma unroll
      for (int n = 0; n < NL; ++n) {
        c_fl[n] = (chunk < items.nchunk) ? lane_flag(lg0 + n) : 0;
        c_any |= c_fl[n];
      }
      c_chunk = chunk;
    }
#pragma unroll
    for (int n = 0; n < NL; ++n) fl[n] = c_fl[n];
    return c_any;
  };
  auto issue_ib = [&](int w, int slot) {
    int* dst = sIB + slot * NE;
    int chunk = 0, g = 0;
    if (w < nitems) items.decode(w, chunk, g);
    for (int i = tid; i < NE; i += NT) {
      if (w < nitems && g < nspec)
        cp_async4(dst + i, A.m.ibool + (size_t)A.m.order[g] * NGLL3 + i);
      else
        dst[i] = -1;
    }
  };
  auto issue_data = [&](int w, int ibslot, int buf) {
    if (w >= nitems) return;
    int lg0, g, fl[NL];
    const int anyf = group_flags(w, lg0, g, fl);
    const int* ib = sIB + ibslot * NE;
    float* km = sKM + buf * 2 * NE;
    const int e = g < nspec ? A.m.order[g] : 0;
    for (int i = tid; i < NE; i += NT) {
      if (g < nspec) {
        const size_t ep = (size_t)e * NGLL3 + i;
        cp_async4(km + i, A.m.kappa + ep);
        cp_async4(km + NE + i, A.m.mu + ep);
      }
    }
    const size_t fb = fbase<LWLOG>(A, lg0);
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      const bool act = f == 0 ? (anyf & 1) : (anyf & 2);
      const float* src = (f == 0 ? A.f1.u : A.f2.u) + fb;
      float* ub = sU + ((buf * NF + f) * PP_U) * LB + lane;
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        const int p = t + 25 * r;
        const int ig = ib[p];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float* d = ub + (c * NGLL3 + p) * LB;
          if (act && ig >= 0) {
            cp_async_v<NL>(d, src + foff<LWLOG>(ig, c));
          } else {
            LV<NL> z;
#pragma unroll
            for (int n = 0; n < NL; ++n) z.v[n] = 0.f;
            sts_v<NL>(d, z);
          }
        }
      }
    }
    if (ADJ && (anyf & 2) && g < nspec) {
      float* kb = sK + buf * 2 * NE * LB;
      const size_t eb = ebase<LWLOG>(A, lg0) + (((size_t)e * NGLL3) << LWLOG);
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        const int p = t + 25 * r;
        const size_t q = eb + ((size_t)p << LWLOG);
        cp_async_v<NL>(kb + p * LB + lane, A.k.mu + q);
        cp_async_v<NL>(kb + (NE + p) * LB + lane, A.k.kappa + q);
      }
    }
  };

  int w = blockIdx.x;
  issue_ib(w, 0);
  cp_commit();
  cp_wait_all();
  __syncthreads();
  issue_data(w, 0, 0);
  issue_ib(w + gridDim.x, 1);
  cp_commit();

  const float fac = A.m.jac * A.m.xix * A.m.xix;
  const float dtk = A.dt * A.m.xix * A.m.xix;
  for (int k = 0; w < nitems; ++k, w += gridDim.x) {
    const int buf = k & 1;
    const int ibs = k % 3;
    cp_wait_all();
    __syncthreads();
    issue_data(w + gridDim.x, (k + 1) % 3, buf ^ 1);
    issue_ib(w + 2 * gridDim.x, (k + 2) % 3);
    cp_commit();

    int lg0, g, fl[NL];
    const int anyf = group_flags(w, lg0, g, fl);
    const int e = g < nspec ? A.m.order[g] : nspec;
    const float* kap = sKM + buf * 2 * NE;
    const float* mu = kap + NE;
    float* u1 = sU + ((buf * NF + 0) * PP_U) * LB + lane;
    float* u2 = sU + ((buf * NF + (NF - 1)) * PP_U) * LB + lane;
    float* a1 = sA + (0 * PP_A) * LB + lane;
    float* a2 = sA + ((NF - 1) * PP_A) * LB + lane;
    PBuf<LB> b1{u1, a1};
    PBuf<LB> b2{u2, a2};
    v_grad_eg<LB, NL>(b1, pi, pq);
    if (ADJ) v_grad_eg<LB, NL>(b2, pi, pq);
    __syncthreads();
    LV<NL> fx1[5][3], fx2[ADJ ? 5 : 1][3];
    if (ADJ) {
      LV<NL> km[5], kk[5];
      v_xi<LB, NL, 1>(b2, b2, t, kap, mu, fac, fx2, km, kk);
      v_xi<LB, NL, 2>(b1, b2, t, kap, mu, fac, fx1, km, kk);
      if ((anyf & 2) && e < nspec) {
        const float* kb = sK + buf * 2 * NE * LB;
#pragma unroll
        for (int i = 0; i < 5; ++i) {
          const int p = i + 5 * t;
          const LV<NL> m0 = lds_v<NL>(kb + p * LB + lane);
          const LV<NL> k0 = lds_v<NL>(kb + (NE + p) * LB + lane);
          LV<NL> mo, ko;
#pragma unroll
          for (int n = 0; n < NL; ++n) {
            const bool on = fl[n] & 2;
            mo.v[n] = on ? m0.v[n] + dtk * km[i].v[n] : m0.v[n];
            ko.v[n] = on ? k0.v[n] + dtk * kk[i].v[n] : k0.v[n];
          }
          const size_t q = ebase<LWLOG>(A, lg0) + (((size_t)e * NGLL3 + p) << LWLOG);
          sts_v<NL>(A.k.mu + q, mo);
          sts_v<NL>(A.k.kappa + q, ko);
        }
      }
    } else {
      LV<NL> km[1], kk[1];
      v_xi<LB, NL, 0>(b1, b1, t, kap, mu, fac, fx1, km, kk);
    }
    __syncthreads();
    v_div_eg<LB, NL>(b1, pi, pq);
    if (ADJ) v_div_eg<LB, NL>(b2, pi, pq);
    __syncthreads();
    if (e < nspec) {
      const int* ib = sIB + ibs * NE;
      const size_t fb = fbase<LWLOG>(A, lg0);
      if (anyf & 1) v_scatter<LB, NL>(b1, t, fx1, ib, A.f1.a + fb, fl, 1);
      if (ADJ && (anyf & 4)) v_scatter<LB, NL>(b2, t, fx2, ib, A.f2.a + fb, fl, 4);
    }
  }
  cp_wait_all();
}

// ---------------------------------------------------------------------------
// adjoint-phase element kernel: (adjoint, backward) field pair as a float2
// ---------------------------------------------------------------------------
//
// In the adjoint phase every event carries two fields on the same element
// with the same kappa and mu.  Here they are the two values of one float2:
// shared memory holds "virtual lanes" (event, field), a thread works one
// event's pencil for both fields with float2 shared traffic, and the
// strain products for the mu/kappa kernels are formed in registers at each
// point, with no parking in shared memory.

// GEN: general elements, as v_xi (six fluxes to B, physical strains).
template <int VL, bool GEN = false>
__device__ __forceinline__ void pair_xi(const PBuf<VL>& b, int t, const float* kap, const float* mu,
                                        float fac, LV<2> fx[5][3], float kmu[5], float kka[5],
                                        const float* geo_e = nullptr, float xix = 0.f,
                                        float jac = 0.f) {
  if constexpr (!GEN) {
    // the adjoint (x) and backward (y) fields as one packed pair
    float2 u[3][5];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int l = 0; l < 5; ++l) u[c][l] = p2(lds_v<2>(b.U(c, l + 5 * t)));
    float2 sx[3][5];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      const int p = i + 5 * t;
      float2 g[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float2 a = make_float2(0.f, 0.f);
#pragma unroll
        for (int l = 0; l < 5; ++l) a = cfma2(gD(i, l), u[c][l], a);
        g[c][0] = a;
        g[c][1] = p2(lds_v<2>(b.Ar(c, p)));
        g[c][2] = p2(lds_v<2>(b.Ar(3 + c, p)));
      }
      float2 sig[6];
      stress_point2(g, kap[p], mu[p], fac, sig);
      sx[0][i] = sig[0];
      sx[1][i] = sig[3];
      sx[2][i] = sig[4];
      // deviatoric strains and traces of both fields, then the adjoint x
      // backward products
      const float2 tr = __fadd2_rn(__fadd2_rn(g[0][0], g[1][1]), g[2][2]);
      const float2 m3 = splat(-1.0f / 3.0f), h = splat(0.5f);
      const float2 exx = __ffma2_rn(tr, m3, g[0][0]);
      const float2 eyy = __ffma2_rn(tr, m3, g[1][1]);
      const float2 exy = __fmul2_rn(h, __fadd2_rn(g[0][1], g[1][0]));
      const float2 exz = __fmul2_rn(h, __fadd2_rn(g[0][2], g[2][0]));
      const float2 eyz = __fmul2_rn(h, __fadd2_rn(g[1][2], g[2][1]));
      kmu[i] = exx.x * exx.y + eyy.x * eyy.y + (exx.x + eyy.x) * (exx.y + eyy.y) +
               2.0f * (exy.x * exy.y + exz.x * exz.y + eyz.x * eyz.y);
      kka[i] = tr.x * tr.y;
      sts_v<2>(b.U(0, p), lv2(sig[3]));
      sts_v<2>(b.U(1, p), lv2(sig[1]));
      sts_v<2>(b.U(2, p), lv2(sig[5]));
      sts_v<2>(b.U(3, p), lv2(sig[4]));
      sts_v<2>(b.U(4, p), lv2(sig[2]));
    }
#pragma unroll
    for (int i = 0; i < 5; ++i)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float2 a = make_float2(0.f, 0.f);
#pragma unroll
        for (int l = 0; l < 5; ++l) a = cfma2(gDWt(i, l), sx[c][l], a);
        fx[i][c] = lv2(a);
      }
  } else {
    LV<2> u[3][5];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int l = 0; l < 5; ++l) u[c][l] = lds_v<2>(b.U(c, l + 5 * t));
    LV<2> sx[3][5];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      const int p = i + 5 * t;
      LV<2> de[3], dg[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        de[c] = lds_v<2>(b.Ar(c, p));
        dg[c] = lds_v<2>(b.Ar(3 + c, p));
      }
      constexpr int NO = GEN ? 6 : 5;
      LV<2> o[NO];
      float ev[2][6];
      const float kp = kap[p], m = mu[p];
      float G[10];
      if (GEN) load_geo(geo_e, p, xix, jac, G);
#pragma unroll
      for (int n = 0; n < 2; ++n) {
        float g[3][3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float a = 0.f;
#pragma unroll
          for (int l = 0; l < 5; ++l) a = cfma(gD(i, l), u[c][l].v[n], a);
          g[c][0] = a;
          g[c][1] = de[c].v[n];
          g[c][2] = dg[c].v[n];
        }
        if constexpr (GEN) {
          float r[3][3];
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int d = 0; d < 3; ++d) r[c][d] = g[c][d];
          map_gradient(r, G, g);
          float sig[6], F[9];
          stress_point(g, kp, m, 1.0f, sig);
          map_flux(sig, G, F);
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            sx[c][i].v[n] = F[c * 3 + 0];
            o[c].v[n] = F[c * 3 + 1];
            o[3 + c].v[n] = F[c * 3 + 2];
          }
        } else {
          float sig[6];
          stress_point(g, kp, m, fac, sig);
          sx[0][i].v[n] = sig[0];
          sx[1][i].v[n] = sig[3];
          sx[2][i].v[n] = sig[4];
          o[0].v[n] = sig[3];
          o[1].v[n] = sig[1];
          o[2].v[n] = sig[5];
          o[3].v[n] = sig[4];
          o[4].v[n] = sig[2];
        }
        const float tr = g[0][0] + g[1][1] + g[2][2];
        ev[n][0] = g[0][0] - tr * (1.0f / 3.0f);
        ev[n][1] = g[1][1] - tr * (1.0f / 3.0f);
        ev[n][2] = 0.5f * (g[0][1] + g[1][0]);
        ev[n][3] = 0.5f * (g[0][2] + g[2][0]);
        ev[n][4] = 0.5f * (g[1][2] + g[2][1]);
        ev[n][5] = tr;
      }
      // adjoint (n = 0) x backward (n = 1) deviatoric products and traces
      kmu[i] = ev[0][0] * ev[1][0] + ev[0][1] * ev[1][1] +
               (ev[0][0] + ev[0][1]) * (ev[1][0] + ev[1][1]) +
               2.0f * (ev[0][2] * ev[1][2] + ev[0][3] * ev[1][3] + ev[0][4] * ev[1][4]);
      kka[i] = ev[0][5] * ev[1][5];
#pragma unroll
      for (int q = 0; q < NO; ++q) sts_v<2>(b.U(q, p), o[q]);
    }
#pragma unroll
    for (int i = 0; i < 5; ++i)
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int n = 0; n < 2; ++n) {
          float a = 0.f;
#pragma unroll
          for (int l = 0; l < 5; ++l) a = cfma(gDWt(i, l), sx[c][l].v[n], a);
          fx[i][c].v[n] = a;
        }
  }
}

template <int VL>
__device__ __forceinline__ void pair_scatter(const PBuf<VL>& b, int t, const LV<2> fx[5][3],
                                             const int* ib, float* accb1, float* accb2, bool on1,
                                             bool on2) {
  const int pj = t % 5, pk = t / 5;
  float wj = 0.f, wk = 0.f;
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    if (q == pj) wj = gW(q);
    if (q == pk) wk = gW(q);
  }
  const float2 njk = splat(-(wj * wk));
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    const int p = i + 5 * t;
    const int ig = ib[p];
    const float2 nik = splat(-(gW(i) * wk)), nij = splat(-(gW(i) * wj));
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float2 e1 = p2(lds_v<2>(b.Ar(c, p)));
      const float2 e2 = p2(lds_v<2>(b.Ar(3 + c, p)));
      const float2 v = __ffma2_rn(nij, e2, __ffma2_rn(nik, e1, __fmul2_rn(njk, p2(fx[i][c]))));
      const size_t q = foff<3>(ig, c);
      if (on1) atomicAdd(&accb1[q], v.x);
      if (on2) atomicAdd(&accb2[q], v.y);
    }
  }
}

template <int LB>
struct PairLayout {
  using LY = PipeLayout<2 * LB, 1, 25, false>;
  static constexpr int OFF_K = al4(LY::TOTAL);                     // [2][2][125][LB]
  static constexpr int TOTAL = OFF_K + 4 * NGLL3 * LB;
  static constexpr size_t BYTES = (size_t)TOTAL * 4;
};

template <int LB>
__global__ void __launch_bounds__(25 * LB) k_forces_adjpair(StepArgs A, PipeItems items) {
  constexpr int VL = 2 * LB;
  constexpr int NT = 25 * LB;
  using LY = typename PairLayout<LB>::LY;
  constexpr int NE = LY::NE;
  constexpr int LWLOG = 3;
  extern __shared__ float sm[];
  int* sIB = (int*)(sm + LY::OFF_IB);
  float* sKM = sm + LY::OFF_KM;
  float* sU = sm + LY::OFF_U;
  float* sA = sm + LY::OFF_A;
  float* sK = sm + PairLayout<LB>::OFF_K;

  const int tid = threadIdx.x;
  const int lq = tid % LB;
  const int t = tid / LB;
  const int pi = t % 5, pq = t / 5;
  const int nev = A.nev;
  const int nspec = A.m.nspec;
  const int nitems = items.count();

  bool any = false;
  for (int l = tid; l < nev; l += NT) {
    const LaneDesc* L = A.lanes + l;
    any |= L->phase != PH_IDLE && L->it0 + A.s < L->nstep;
  }
  if (!__syncthreads_or(any)) return;
  if (A.lm.lwlog != LWLOG) return;  // batched layout only

  int c_chunk = -1, c_flag = 0;
  auto flags = [&](int w, int& lg, int& g) -> int {
    int chunk;
    items.decode(w, chunk, g);
    lg = chunk * LB + lq;
    if (chunk == c_chunk) return c_flag;
    int f = 0;
    if (chunk < items.nchunk && lg < nev) {
      const LaneDesc* L = A.lanes + lg;
      const int it = L->it0 + A.s;
      if (L->phase != PH_IDLE && it < L->nstep) {
        f = 1;
        if (L->phase == PH_ADJ) f |= 2 | (it > 0 ? 4 : 0);
      }
    }
    c_chunk = chunk;
    c_flag = f;
    return f;
  };
  auto issue_ib = [&](int w, int slot) {
    int* dst = sIB + slot * NE;
    int chunk = 0, g = 0;
    if (w < nitems) items.decode(w, chunk, g);
    for (int i = tid; i < NE; i += NT) {
      if (w < nitems && g < nspec)
        cp_async4(dst + i, A.m.ibool + (size_t)A.m.order[g] * NGLL3 + i);
      else
        dst[i] = -1;
    }
  };
  auto issue_data = [&](int w, int ibslot, int buf) {
    if (w >= nitems) return;
    int lg, g;
    const int fl = flags(w, lg, g);
    const int* ib = sIB + ibslot * NE;
    float* km = sKM + buf * 2 * NE;
    const int e = g < nspec ? A.m.order[g] : 0;
    for (int i = tid; i < NE; i += NT) {
      if (g < nspec) {
        const size_t ep = (size_t)e * NGLL3 + i;
        cp_async4(km + i, A.m.kappa + ep);
        cp_async4(km + NE + i, A.m.mu + ep);
      }
    }
    const size_t fb = fbase<LWLOG>(A, lg);
    float* ub = sU + (buf * PP_U) * VL + 2 * lq;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      const int p = t + 25 * r;
      const int ig = ib[p];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float* d = ub + (c * NGLL3 + p) * VL;
        if ((fl & 1) && ig >= 0)
          cp_async4(d, A.f1.u + fb + foff<LWLOG>(ig, c));
        else
          d[0] = 0.f;
        if ((fl & 2) && ig >= 0)
          cp_async4(d + 1, A.f2.u + fb + foff<LWLOG>(ig, c));
        else
          d[1] = 0.f;
      }
    }
    if ((fl & 2) && g < nspec) {
      float* kb = sK + buf * 2 * NGLL3 * LB;
      const size_t eb = ebase<LWLOG>(A, lg) + (((size_t)e * NGLL3) << LWLOG);
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        const int p = t + 25 * r;
        const size_t q = eb + ((size_t)p << LWLOG);
        cp_async4(kb + p * LB + lq, A.k.mu + q);
        cp_async4(kb + (NGLL3 + p) * LB + lq, A.k.kappa + q);
      }
    }
  };

  int w = blockIdx.x;
  issue_ib(w, 0);
  cp_commit();
  cp_wait_all();
  __syncthreads();
  issue_data(w, 0, 0);
  issue_ib(w + gridDim.x, 1);
  cp_commit();

  const float fac = A.m.jac * A.m.xix * A.m.xix;
  const float dtk = A.dt * A.m.xix * A.m.xix;
  for (int k = 0; w < nitems; ++k, w += gridDim.x) {
    const int buf = k & 1;
    const int ibs = k % 3;
    cp_wait_all();
    __syncthreads();
    issue_data(w + gridDim.x, (k + 1) % 3, buf ^ 1);
    issue_ib(w + 2 * gridDim.x, (k + 2) % 3);
    cp_commit();

    int lg, g;
    const int fl = flags(w, lg, g);
    const int e = g < nspec ? A.m.order[g] : nspec;
    const float* kap = sKM + buf * 2 * NE;
    const float* mu = kap + NE;
    PBuf<VL> b{sU + (buf * PP_U) * VL + 2 * lq, sA + 2 * lq};
    v_grad_eg<VL, 2>(b, pi, pq);
    __syncthreads();
    LV<2> fx[5][3];
    float kmu[5], kka[5];
    pair_xi<VL>(b, t, kap, mu, fac, fx, kmu, kka);
    if ((fl & 2) && e < nspec) {
      const float* kb = sK + buf * 2 * NGLL3 * LB;
      const size_t eb = ebase<LWLOG>(A, lg) + (((size_t)e * NGLL3) << LWLOG);
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        const int p = i + 5 * t;
        const size_t q = eb + ((size_t)p << LWLOG);
        A.k.mu[q] = kb[p * LB + lq] + dtk * kmu[i];
        A.k.kappa[q] = kb[(NGLL3 + p) * LB + lq] + dtk * kka[i];
      }
    }
    __syncthreads();
    v_div_eg<VL, 2>(b, pi, pq);
    __syncthreads();
    if (e < nspec && (fl & 1)) {
      const size_t fb = fbase<LWLOG>(A, lg);
      pair_scatter<VL>(b, t, fx, sIB + ibs * NE, A.f1.a + fb, A.f2.a + fb, true, (fl & 4) != 0);
    }
  }
  cp_wait_all();
}

// As k_forces_adjpair, but the next element's displacement gather is
// prefetched into registers (plain loads issued before the current element
// is computed, stored to shared memory once the current element's stresses
// have been read), so the displacement region is single-buffered: 40 KB
// less shared memory per 8 events, twice the resident blocks.  Four block
// barriers per element: the gather store shares the top barrier with the
// copies of the next items, and the items come from an ItemRing.
template <int LB, bool GEN = false>
struct PairRLayout {
  static constexpr int VL = 2 * LB;
  static constexpr int NE = NGLL3;
  static constexpr int PPU = GEN ? 6 * NGLL3 : PP_U;               // U, then 5 (6) values
  static constexpr int OFF_IB = 0;                                  // int [3][NE]
  static constexpr int OFF_IT = al4(OFF_IB + 3 * NE);               // int [2][4] item ring
  static constexpr int OFF_KM = al4(OFF_IT + 8);                    // [2][2][NE]
  static constexpr int OFF_U = al4(OFF_KM + 4 * NE);                // [PPU][VL]
  static constexpr int OFF_A = al4(OFF_U + PPU * VL);               // [PP_A][VL]
  static constexpr int TOTAL = OFF_A + PP_A * VL;
  static constexpr size_t BYTES = (size_t)TOTAL * 4;
};

template <int LB, bool GEN = false>
__global__ void __launch_bounds__(25 * LB, LB == 8 ? 2 : 4) k_forces_adjpair_r(StepArgs A, PipeItems items) {
  constexpr int VL = 2 * LB;
  constexpr int NT = 25 * LB;
  using LY = PairRLayout<LB, GEN>;
  constexpr int NE = NGLL3;
  constexpr int LWLOG = 3;
  extern __shared__ float sm[];
  int* sIB = (int*)(sm + LY::OFF_IB);
  const ItemRing ring{(int*)(sm + LY::OFF_IT), (int*)(sm + LY::OFF_IT) + 4};
  float* sKM = sm + LY::OFF_KM;
  float* sU = sm + LY::OFF_U;
  float* sA = sm + LY::OFF_A;

  const int tid = threadIdx.x;
  const int lq = tid % LB;
  const int t = tid / LB;
  const int pi = t % 5, pq = t / 5;
  const int nev = A.nev;
  const int nspec = A.m.nspec;
  const int nitems = items.count();
  const int G = gridDim.x;

  bool any = false;
  for (int l = tid; l < nev; l += NT) {
    const LaneDesc* L = A.lanes + l;
    any |= L->phase != PH_IDLE && L->it0 + A.s < L->nstep;
  }
  if (!__syncthreads_or(any)) return;
  if (A.lm.lwlog != LWLOG) return;  // batched layout only

  // this thread's lane of a chunk and its flags: 1 running, 2 adjoint
  // phase, 4 adjoint phase past its first step
  int c_chunk = -1, c_flag = 0;
  auto flags = [&](int chunk, int& lg) -> int {
    lg = chunk * LB + lq;
    if (chunk == c_chunk) return c_flag;
    int f = 0;
    if (chunk < items.nchunk && lg < nev) {
      const LaneDesc* L = A.lanes + lg;
      const int it = L->it0 + A.s;
      if (L->phase != PH_IDLE && it < L->nstep) {
        f = 1;
        if (L->phase == PH_ADJ) f |= 2 | (it > 0 ? 4 : 0);
      }
    }
    c_chunk = chunk;
    c_flag = f;
    return f;
  };
  // ibool row of element e into slot `slot` (-1 past the end)
  auto issue_ib = [&](int e, int slot) {
    int* dst = sIB + slot * NE;
    for (int i = tid; i < NE; i += NT) {
      if (e < nspec)
        cp_async4(dst + i, A.m.ibool + (size_t)e * NGLL3 + i);
      else
        dst[i] = -1;
    }
  };
  // kappa and mu of element e into buffer buf
  auto issue_km = [&](int e, int buf) {
    if (e >= nspec) return;
    float* km = sKM + buf * 2 * NE;
    for (int i = tid; i < NE; i += NT) {
      const size_t ep = (size_t)e * NGLL3 + i;
      cp_async4(km + i, A.m.kappa + ep);
      cp_async4(km + NE + i, A.m.mu + ep);
    }
  };
  // displacement gather of an item into registers (ibool from slot ibslot)
  // (adjoint, backward) displacement of points t + 25 r: the thread's
  // gamma pencil
  float2 pre[5][3];
  auto load_u = [&](int chunk, int ibslot) {
    int lg;
    const int fl = flags(chunk, lg);
    const int* ib = sIB + ibslot * NE;
    const size_t fb = fbase<LWLOG>(A, lg);
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      const int ig = ib[t + 25 * r];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        ldg_pred(pre[r][c].x, A.f1.u + fb + foff<LWLOG>(ig, c), (fl & 1) && ig >= 0);
        ldg_pred(pre[r][c].y, A.f2.u + fb + foff<LWLOG>(ig, c), (fl & 2) && ig >= 0);
      }
    }
  };
  auto store_u = [&]() {
    float* ub = sU + 2 * lq;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      const int p = t + 25 * r;
#pragma unroll
      for (int c = 0; c < 3; ++c) sts_v<2>(ub + (c * NGLL3 + p) * VL, lv2(pre[r][c]));
    }
  };

  int w = blockIdx.x;
  if (tid == 0)
    for (int j = 0; j < 3; ++j) ring.fill(items, A.m.order, nspec, w + j * G, j);
  cp_commit();
  cp_wait_all();
  __syncthreads();
  issue_ib(ring.e[0], 0);
  cp_commit();
  cp_wait_all();
  __syncthreads();
  issue_km(ring.e[0], 0);
  issue_ib(ring.e[1], 1);
  cp_commit();
  load_u(ring.c[0], 0);
  store_u();

  const float fac = A.m.jac * A.m.xix * A.m.xix;
  // kernel products: raw reference derivatives (times xix^2) or, for
  // general elements, physical strains
  const float dtk = GEN ? A.dt : A.dt * A.m.xix * A.m.xix;
  for (int k = 0; w < nitems; ++k, w += G) {
    const int buf = k & 1;
    const int ibs = k % 3;
    cp_wait_all();
    __syncthreads();  // U holds this item's displacement, its copies landed, the last scatter is done
    PBuf<VL> b{sU + 2 * lq, sA + 2 * lq};
    grad_gamma_regs<VL>(b, t, pre);  // before the next gather replaces pre
    if (tid == 0) ring.fill(items, A.m.order, nspec, w + 3 * G, (k + 3) & 3);
    issue_km(ring.e[(k + 1) & 3], buf ^ 1);
    issue_ib(ring.e[(k + 2) & 3], (k + 2) % 3);
    cp_commit();
    load_u(ring.c[(k + 1) & 3], (k + 1) % 3);  // next item's gather, stored after this item's divergence

    int lg;
    const int fl = flags(ring.c[k & 3], lg);
    const int e = ring.e[k & 3];
    const float* kap = sKM + buf * 2 * NE;
    const float* mu = kap + NE;
    v_grad_eg<VL, 2, false>(b, pi, pq);
    __syncthreads();
    LV<2> fx[5][3];
    float kmu[5], kka[5];
    const float* geo_e = nullptr;
    if (GEN && e < nspec) {
      const int ir = A.m.irreg[e];
      if (ir >= 0) geo_e = A.m.geo + (size_t)ir * NGLL3 * 10;
    }
    pair_xi<VL, GEN>(b, t, kap, mu, fac, fx, kmu, kka, geo_e, A.m.xix, A.m.jac);
    if ((fl & 2) && e < nspec) {
      // mu/kappa kernel products: one writer per element point and lane in
      // a launch, added in L2 without a round trip through the SM
      const size_t eb = ebase<LWLOG>(A, lg) + (((size_t)e * NGLL3) << LWLOG);
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        const int p = i + 5 * t;
        const size_t q = eb + ((size_t)p << LWLOG);
        atomicAdd(&A.k.mu[q], dtk * kmu[i]);
        atomicAdd(&A.k.kappa[q], dtk * kka[i]);
      }
    }
    __syncthreads();
    v_div_eg<VL, 2, GEN>(b, pi, pq);
    __syncthreads();  // U's stresses read: it takes the next displacement
    store_u();
    if (e < nspec && (fl & 1)) {
      const size_t fb = fbase<LWLOG>(A, lg);
      pair_scatter<VL>(b, t, fx, sIB + ibs * NE, A.f1.a + fb, A.f2.a + fb, true, (fl & 4) != 0);
    }
  }
  cp_wait_all();
}

template <int LB, bool GEN = false>
static void forces_adjpair_r_cfg(const StepArgs& a, cudaStream_t st) {
  constexpr int NT = 25 * LB;
  constexpr size_t BYTES = PairRLayout<LB, GEN>::BYTES;
  static int blocks_per_sm = 0, sms = 0;
  if (!blocks_per_sm) {
    cudaFuncSetAttribute(k_forces_adjpair_r<LB, GEN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)BYTES);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_forces_adjpair_r<LB, GEN>, NT,
                                                  BYTES);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (blocks_per_sm < 1) blocks_per_sm = 1;
  }
  PipeItems items = make_items<LB>(a, a.m.nspec);
  if (items.count() == 0) return;
  int gx = blocks_per_sm * sm_share(a, sms);
  if (gx > items.count()) gx = items.count();
  if (gx < 1) gx = 1;
  k_forces_adjpair_r<LB, GEN><<<gx, NT, BYTES, st>>>(a, items);
}

// Adjoint element kernel sized for three blocks per SM (variant 14; regular
// elements, 8 lanes x 2 fields per block).  Same arithmetic as
// k_forces_adjpair_r, in 72.8 KB of shared memory instead of 91.5 KB:
// - the displacement takes 3 planes; the stress planes 0-2 overwrite them
//   at the xi owner's points, planes 3-4 overwrite the eta-derivative slots
//   0-1 of those points once the owner has read them;
// - the divergence is summed in shared memory: the xi owner writes
//   -wjk f_xi into planes A2..A4 of its points, the eta and gamma owners
//   add -wik f_eta and -wij f_gamma there in two more passes, and the xi
//   owner scatters the sums, so no flux registers live to the scatter;
// - kappa/mu are single-buffered, fetched for the next element once this
//   element's stress is formed.
struct PairR3Layout {
  static constexpr int VL = 16;
  static constexpr int NE = NGLL3;
  static constexpr int OFF_IB = 0;                          // int [3][NE]
  static constexpr int OFF_KM = al4(OFF_IB + 3 * NE);       // [2][NE] kappa, mu
  static constexpr int OFF_U = al4(OFF_KM + 2 * NE);        // [3][NE][VL]
  static constexpr int OFF_A = al4(OFF_U + 3 * NE * VL);    // [6][NE][VL]
  static constexpr int TOTAL = OFF_A + 6 * NE * VL;
  static constexpr size_t BYTES = (size_t)TOTAL * 4;
};

// xi role of variant 14: gradient, stress and strain products at the
// pencil's points (as pair_xi), stress components to U0..U2 and A0..A1,
// and -wjk times the xi divergence to A2..A4.
__device__ __forceinline__ void pair_xi3(const PBuf<16>& b, int t, const float* kap,
                                         const float* mu, float fac, float kmu[5], float kka[5]) {
  float2 u[3][5];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int l = 0; l < 5; ++l) u[c][l] = p2(lds_v<2>(b.U(c, l + 5 * t)));
  float2 sx[3][5];
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    const int p = i + 5 * t;
    float2 g[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float2 a = make_float2(0.f, 0.f);
#pragma unroll
      for (int l = 0; l < 5; ++l) a = cfma2(gD(i, l), u[c][l], a);
      g[c][0] = a;
      g[c][1] = p2(lds_v<2>(b.Ar(c, p)));
      g[c][2] = p2(lds_v<2>(b.Ar(3 + c, p)));
    }
    float2 sig[6];
    stress_point2(g, kap[p], mu[p], fac, sig);
    sx[0][i] = sig[0];
    sx[1][i] = sig[3];
    sx[2][i] = sig[4];
    const float2 tr = __fadd2_rn(__fadd2_rn(g[0][0], g[1][1]), g[2][2]);
    const float2 m3 = splat(-1.0f / 3.0f), h = splat(0.5f);
    const float2 exx = __ffma2_rn(tr, m3, g[0][0]);
    const float2 eyy = __ffma2_rn(tr, m3, g[1][1]);
    const float2 exy = __fmul2_rn(h, __fadd2_rn(g[0][1], g[1][0]));
    const float2 exz = __fmul2_rn(h, __fadd2_rn(g[0][2], g[2][0]));
    const float2 eyz = __fmul2_rn(h, __fadd2_rn(g[1][2], g[2][1]));
    kmu[i] = exx.x * exx.y + eyy.x * eyy.y + (exx.x + eyy.x) * (exx.y + eyy.y) +
             2.0f * (exy.x * exy.y + exz.x * exz.y + eyz.x * eyz.y);
    kka[i] = tr.x * tr.y;
    // sigma for the eta pencils: xy, yy, yz; for the gamma pencils xz, yz, zz
    sts_v<2>(b.U(0, p), lv2(sig[3]));
    sts_v<2>(b.U(1, p), lv2(sig[1]));
    sts_v<2>(b.U(2, p), lv2(sig[5]));
    sts_v<2>(b.Ar(0, p), lv2(sig[4]));
    sts_v<2>(b.Ar(1, p), lv2(sig[2]));
  }
  const int pj = t % 5, pk = t / 5;
  float wj = 0.f, wk = 0.f;
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    if (q == pj) wj = gW(q);
    if (q == pk) wk = gW(q);
  }
  const float2 njk = splat(-(wj * wk));
#pragma unroll
  for (int i = 0; i < 5; ++i)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float2 a = make_float2(0.f, 0.f);
#pragma unroll
      for (int l = 0; l < 5; ++l) a = cfma2(gDWt(i, l), sx[c][l], a);
      sts_v<2>(b.Ar(2 + c, i + 5 * t), lv2(__fmul2_rn(njk, a)));
    }
}

// eta (DIR 1) or gamma (DIR 2) role of variant 14 on the pencil (pi, pq):
// the divergence along the pencil of the three components' fluxes, times
// -w w of the other two directions, added to A2..A4 at the pencil's points.
template <int DIR, int VL = 16>
__device__ __forceinline__ void div_add3(const PBuf<VL>& b, int pi, int pq) {
  // point l of the pencil
  auto pt = [&](int l) { return DIR == 1 ? pi + 5 * l + 25 * pq : pi + 5 * pq + 25 * l; };
  float2 v[3][5];
#pragma unroll
  for (int l = 0; l < 5; ++l) {
    const int p = pt(l);
    if (DIR == 1) {                       // sigma_{c,y} = xy, yy, yz
      v[0][l] = p2(lds_v<2>(b.U(0, p)));
      v[1][l] = p2(lds_v<2>(b.U(1, p)));
      v[2][l] = p2(lds_v<2>(b.U(2, p)));
    } else {                              // sigma_{c,z} = xz, yz, zz
      v[0][l] = p2(lds_v<2>(b.Ar(0, p)));
      v[1][l] = p2(lds_v<2>(b.U(2, p)));
      v[2][l] = p2(lds_v<2>(b.Ar(1, p)));
    }
  }
  float wa = 0.f, wb = 0.f;
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    if (q == pi) wa = gW(q);
    if (q == pq) wb = gW(q);
  }
  const float2 nw = splat(-(wa * wb));
#pragma unroll
  for (int j = 0; j < 5; ++j)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float2 a = make_float2(0.f, 0.f);
#pragma unroll
      for (int l = 0; l < 5; ++l) a = cfma2(gDWt(j, l), v[c][l], a);
      float* d = b.Ar(2 + c, pt(j));
      sts_v<2>(d, lv2(__ffma2_rn(nw, a, p2(lds_v<2>(d)))));
    }
}

__global__ void __maxnreg__(96) k_forces_adjpair_r3(StepArgs A, PipeItems items) {
  constexpr int LB = 8;
  constexpr int VL = 2 * LB;
  constexpr int NT = 25 * LB;
  using LY = PairR3Layout;
  constexpr int NE = NGLL3;
  constexpr int LWLOG = 3;
  extern __shared__ float sm[];
  int* sIB = (int*)(sm + LY::OFF_IB);
  float* sKM = sm + LY::OFF_KM;
  float* sU = sm + LY::OFF_U;
  float* sA = sm + LY::OFF_A;

  const int tid = threadIdx.x;
  const int lq = tid % LB;
  const int t = tid / LB;
  const int pi = t % 5, pq = t / 5;
  const int nev = A.nev;
  const int nspec = A.m.nspec;
  const int nitems = items.count();

  bool any = false;
  for (int l = tid; l < nev; l += NT) {
    const LaneDesc* L = A.lanes + l;
    any |= L->phase != PH_IDLE && L->it0 + A.s < L->nstep;
  }
  if (!__syncthreads_or(any)) return;
  if (A.lm.lwlog != LWLOG) return;  // batched layout only

  int c_chunk = -1, c_flag = 0;
  auto flags = [&](int w, int& lg, int& g) -> int {
    int chunk;
    items.decode(w, chunk, g);
    lg = chunk * LB + lq;
    if (chunk == c_chunk) return c_flag;
    int f = 0;
    if (chunk < items.nchunk && lg < nev) {
      const LaneDesc* L = A.lanes + lg;
      const int it = L->it0 + A.s;
      if (L->phase != PH_IDLE && it < L->nstep) {
        f = 1;
        if (L->phase == PH_ADJ) f |= 2 | (it > 0 ? 4 : 0);
      }
    }
    c_chunk = chunk;
    c_flag = f;
    return f;
  };
  auto issue_ib = [&](int w, int slot) {
    int* dst = sIB + slot * NE;
    int chunk = 0, g = 0;
    if (w < nitems) items.decode(w, chunk, g);
    for (int i = tid; i < NE; i += NT) {
      if (w < nitems && g < nspec)
        cp_async4(dst + i, A.m.ibool + (size_t)A.m.order[g] * NGLL3 + i);
      else
        dst[i] = -1;
    }
  };
  auto issue_km = [&](int w) {
    if (w >= nitems) return;
    int chunk, g;
    items.decode(w, chunk, g);
    if (g >= nspec) return;
    const int e = A.m.order[g];
    for (int i = tid; i < NE; i += NT) {
      const size_t ep = (size_t)e * NGLL3 + i;
      cp_async4(sKM + i, A.m.kappa + ep);
      cp_async4(sKM + NE + i, A.m.mu + ep);
    }
  };
  float pre[2][5][3];
  auto load_u = [&](int w, int ibslot) {
    int lg = 0, g = 0, fl = 0;
    if (w < nitems) fl = flags(w, lg, g);
    const int* ib = sIB + ibslot * NE;
    const size_t fb = fbase<LWLOG>(A, lg);
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      const int ig = (w < nitems) ? ib[t + 25 * r] : -1;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        ldg_pred(pre[0][r][c], A.f1.u + fb + foff<LWLOG>(ig, c), (fl & 1) && ig >= 0);
        ldg_pred(pre[1][r][c], A.f2.u + fb + foff<LWLOG>(ig, c), (fl & 2) && ig >= 0);
      }
    }
  };

  int w = blockIdx.x;
  issue_ib(w, 0);
  cp_commit();
  cp_wait_all();
  __syncthreads();
  issue_km(w);
  issue_ib(w + gridDim.x, 1);
  cp_commit();
  load_u(w, 0);

  const float fac = A.m.jac * A.m.xix * A.m.xix;
  const float dtk = A.dt * A.m.xix * A.m.xix;
  for (int k = 0; w < nitems; ++k, w += gridDim.x) {
    const int ibs = k % 3;
    cp_wait_all();
    __syncthreads();  // previous element done with U/A; this one's kappa/mu landed
    {
      float* ub = sU + 2 * lq;
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        const int p = t + 25 * r;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          LV<2> v;
          v.v[0] = pre[0][r][c];
          v.v[1] = pre[1][r][c];
          sts_v<2>(ub + (c * NGLL3 + p) * VL, v);
        }
      }
    }
    issue_ib(w + 2 * gridDim.x, (k + 2) % 3);
    cp_commit();
    __syncthreads();  // U complete
    load_u(w + gridDim.x, (k + 1) % 3);

    int lg, g;
    const int fl = flags(w, lg, g);
    const int e = g < nspec ? A.m.order[g] : nspec;
    PBuf<VL> b{sU + 2 * lq, sA + 2 * lq};
    v_grad_eg<VL, 2>(b, pi, pq);
    __syncthreads();
    float kmu[5], kka[5];
    pair_xi3(b, t, sKM, sKM + NE, fac, kmu, kka);
    if ((fl & 2) && e < nspec) {
      const size_t eb = ebase<LWLOG>(A, lg) + (((size_t)e * NGLL3) << LWLOG);
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        const size_t q = eb + ((size_t)(i + 5 * t) << LWLOG);
        atomicAdd(&A.k.mu[q], dtk * kmu[i]);
        atomicAdd(&A.k.kappa[q], dtk * kka[i]);
      }
    }
    __syncthreads();  // stress and xi sums complete; kappa/mu free
    issue_km(w + gridDim.x);
    cp_commit();
    div_add3<1>(b, pi, pq);
    __syncthreads();
    div_add3<2>(b, pi, pq);
    __syncthreads();
    if (e < nspec && (fl & 1)) {
      const int* ib = sIB + ibs * NE;
      const size_t fb = fbase<LWLOG>(A, lg);
      const bool on2 = (fl & 4) != 0;
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        const int p = i + 5 * t;
        const int ig = ib[p];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float2 v = p2(lds_v<2>(b.Ar(2 + c, p)));
          const size_t q = fb + foff<LWLOG>(ig, c);
          atomicAdd(&A.f1.a[q], v.x);
          if (on2) atomicAdd(&A.f2.a[q], v.y);
        }
      }
    }
  }
  cp_wait_all();
}

static void forces_adjpair_r3_cfg(const StepArgs& a, cudaStream_t st) {
  constexpr int NT = 200;
  constexpr size_t BYTES = PairR3Layout::BYTES;
  static int blocks_per_sm = 0, sms = 0;
  if (!blocks_per_sm) {
    cudaFuncSetAttribute(k_forces_adjpair_r3, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)BYTES);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_forces_adjpair_r3, NT, BYTES);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (blocks_per_sm < 1) blocks_per_sm = 1;
  }
  PipeItems items = make_items<8>(a, a.m.nspec);
  if (items.count() == 0) return;
  int gx = blocks_per_sm * sm_share(a, sms);
  if (gx > items.count()) gx = items.count();
  if (gx < 1) gx = 1;
  k_forces_adjpair_r3<<<gx, NT, BYTES, st>>>(a, items);
}

// Forward element kernel sized for five blocks per SM (variant 15; regular
// elements, 8 lanes, 2 events per thread, 100 threads): the shared-memory
// plan of variant 14 for one field - displacement in 3 planes, stress
// planes 3-4 in the derivative slots of the owner's points, the
// divergence summed in 3 planes by the xi, eta and gamma owners in turn,
// single-buffered kappa/mu - 38.5 KB instead of 47.5 KB.
struct FwdR5Layout {
  static constexpr int LB = 8;
  static constexpr int NE = NGLL3;
  static constexpr int OFF_IB = 0;                          // int [3][NE]
  static constexpr int OFF_KM = al4(OFF_IB + 3 * NE);       // [2][NE] kappa, mu
  static constexpr int OFF_U = al4(OFF_KM + 2 * NE);        // [3][NE][LB]
  static constexpr int OFF_A = al4(OFF_U + 3 * NE * LB);    // [6][NE][LB]
  static constexpr int TOTAL = OFF_A + 6 * NE * LB;
  static constexpr size_t BYTES = (size_t)TOTAL * 4;
};

// xi role of variant 15: gradient and stress of two events at the pencil's
// points, stress components to U0..U2 and A0..A1, -wjk f_xi to A2..A4.
__device__ __forceinline__ void fwd_xi5(const PBuf<8>& b, int t, const float* kap,
                                        const float* mu, float fac) {
  float2 u[3][5];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int l = 0; l < 5; ++l) u[c][l] = p2(lds_v<2>(b.U(c, l + 5 * t)));
  float2 sx[3][5];
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    const int p = i + 5 * t;
    float2 g[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float2 a = make_float2(0.f, 0.f);
#pragma unroll
      for (int l = 0; l < 5; ++l) a = cfma2(gD(i, l), u[c][l], a);
      g[c][0] = a;
      g[c][1] = p2(lds_v<2>(b.Ar(c, p)));
      g[c][2] = p2(lds_v<2>(b.Ar(3 + c, p)));
    }
    float2 sig[6];
    stress_point2(g, kap[p], mu[p], fac, sig);
    sx[0][i] = sig[0];
    sx[1][i] = sig[3];
    sx[2][i] = sig[4];
    sts_v<2>(b.U(0, p), lv2(sig[3]));
    sts_v<2>(b.U(1, p), lv2(sig[1]));
    sts_v<2>(b.U(2, p), lv2(sig[5]));
    sts_v<2>(b.Ar(0, p), lv2(sig[4]));
    sts_v<2>(b.Ar(1, p), lv2(sig[2]));
  }
  const int pj = t % 5, pk = t / 5;
  float wj = 0.f, wk = 0.f;
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    if (q == pj) wj = gW(q);
    if (q == pk) wk = gW(q);
  }
  const float2 njk = splat(-(wj * wk));
#pragma unroll
  for (int i = 0; i < 5; ++i)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float2 a = make_float2(0.f, 0.f);
#pragma unroll
      for (int l = 0; l < 5; ++l) a = cfma2(gDWt(i, l), sx[c][l], a);
      sts_v<2>(b.Ar(2 + c, i + 5 * t), lv2(__fmul2_rn(njk, a)));
    }
}

__global__ void __maxnreg__(96) k_forces_fwd_r5(StepArgs A, PipeItems items) {
  constexpr int LB = 8;
  constexpr int NL = 2;
  constexpr int NT = 25 * LB / NL;
  using LY = FwdR5Layout;
  constexpr int NE = NGLL3;
  constexpr int LWLOG = 3;
  extern __shared__ float sm[];
  int* sIB = (int*)(sm + LY::OFF_IB);
  float* sKM = sm + LY::OFF_KM;
  float* sU = sm + LY::OFF_U;
  float* sA = sm + LY::OFF_A;

  const int tid = threadIdx.x;
  const int lq = tid % (LB / NL);
  const int t = tid / (LB / NL);
  const int lane = lq * NL;
  const int pi = t % 5, pq = t / 5;
  const int nev = A.nev;
  const int nspec = A.m.nspec;
  const int nitems = items.count();

  bool any = false;
  for (int l = tid; l < nev; l += NT) {
    const LaneDesc* L = A.lanes + l;
    any |= L->phase != PH_IDLE && L->it0 + A.s < L->nstep;
  }
  if (!__syncthreads_or(any)) return;
  if (A.lm.lwlog != LWLOG) return;  // batched layout only

  int c_chunk = -1, c_fl[NL] = {0, 0};
  auto flags = [&](int w, int& lg0, int& g, int fl[NL]) -> int {
    int chunk;
    items.decode(w, chunk, g);
    lg0 = chunk * LB + lane;
    if (chunk != c_chunk) {
#pragma unroll
      for (int n = 0; n < NL; ++n) {
        int f = 0;
        const int lg = lg0 + n;
        if (chunk < items.nchunk && lg < nev) {
          const LaneDesc* L = A.lanes + lg;
          const int it = L->it0 + A.s;
          if (L->phase != PH_IDLE && it < L->nstep) f = 1;
        }
        c_fl[n] = f;
      }
      c_chunk = chunk;
    }
    fl[0] = c_fl[0];
    fl[1] = c_fl[1];
    return fl[0] | fl[1];
  };
  auto issue_ib = [&](int w, int slot) {
    int* dst = sIB + slot * NE;
    int chunk = 0, g = 0;
    if (w < nitems) items.decode(w, chunk, g);
    for (int i = tid; i < NE; i += NT) {
      if (w < nitems && g < nspec)
        cp_async4(dst + i, A.m.ibool + (size_t)A.m.order[g] * NGLL3 + i);
      else
        dst[i] = -1;
    }
  };
  auto issue_km = [&](int w) {
    if (w >= nitems) return;
    int chunk, g;
    items.decode(w, chunk, g);
    if (g >= nspec) return;
    const int e = A.m.order[g];
    for (int i = tid; i < NE; i += NT) {
      const size_t ep = (size_t)e * NGLL3 + i;
      cp_async4(sKM + i, A.m.kappa + ep);
      cp_async4(sKM + NE + i, A.m.mu + ep);
    }
  };
  float2 pre[5][3];
  auto load_u = [&](int w, int ibslot) {
    int lg0 = 0, g = 0, fl[NL] = {0, 0}, anyf = 0;
    if (w < nitems) anyf = flags(w, lg0, g, fl);
    const int* ib = sIB + ibslot * NE;
    const float* src = A.f1.u + fbase<LWLOG>(A, lg0);
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      const int ig = (w < nitems) ? ib[t + 25 * r] : -1;
#pragma unroll
      for (int c = 0; c < 3; ++c)
        ldg_pred(pre[r][c], src + foff<LWLOG>(ig, c), anyf && ig >= 0);
    }
  };

  int w = blockIdx.x;
  issue_ib(w, 0);
  cp_commit();
  cp_wait_all();
  __syncthreads();
  issue_km(w);
  issue_ib(w + gridDim.x, 1);
  cp_commit();
  load_u(w, 0);

  const float fac = A.m.jac * A.m.xix * A.m.xix;
  for (int k = 0; w < nitems; ++k, w += gridDim.x) {
    const int ibs = k % 3;
    cp_wait_all();
    __syncthreads();  // previous element done with U/A; this one's kappa/mu landed
    {
      float* ub = sU + lane;
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        const int p = t + 25 * r;
#pragma unroll
        for (int c = 0; c < 3; ++c)
          *reinterpret_cast<float2*>(ub + (c * NGLL3 + p) * LB) = pre[r][c];
      }
    }
    issue_ib(w + 2 * gridDim.x, (k + 2) % 3);
    cp_commit();
    __syncthreads();  // U complete
    load_u(w + gridDim.x, (k + 1) % 3);

    int lg0, g, fl[NL];
    const int anyf = flags(w, lg0, g, fl);
    const bool valid = g < nspec;
    PBuf<LB> b{sU + lane, sA + lane};
    v_grad_eg<LB, NL>(b, pi, pq);
    __syncthreads();
    fwd_xi5(b, t, sKM, sKM + NE, fac);
    __syncthreads();  // stress and xi sums complete; kappa/mu free
    issue_km(w + gridDim.x);
    cp_commit();
    div_add3<1, LB>(b, pi, pq);
    __syncthreads();
    div_add3<2, LB>(b, pi, pq);
    __syncthreads();
    if (valid && anyf) {
      const int* ib = sIB + ibs * NE;
      float* accb = A.f1.a + fbase<LWLOG>(A, lg0);
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        const int p = i + 5 * t;
        const int ig = ib[p];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          LV<2> f = lds_v<2>(b.Ar(2 + c, p));
          if (!(fl[0] & 1)) f.v[0] = 0.f;   // lanes not running add nothing
          if (!(fl[1] & 1)) f.v[1] = 0.f;
          red_v<2>(&accb[foff<3>(ig, c)], f);
        }
      }
    }
  }
  cp_wait_all();
}

static int forces_fwd_r5_cfg(const StepArgs& a, cudaStream_t st) {
  constexpr int NT = 100;
  constexpr size_t BYTES = FwdR5Layout::BYTES;
  static int blocks_per_sm = 0, sms = 0;
  if (!blocks_per_sm) {
    cudaFuncSetAttribute(k_forces_fwd_r5, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BYTES);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_forces_fwd_r5, NT, BYTES);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (blocks_per_sm < 1) blocks_per_sm = 1;
  }
  PipeItems items = make_items<8>(a, a.m.nspec);
  if (items.count() == 0) return 0;
  int gx = blocks_per_sm * sm_share(a, sms);
  if (gx > items.count()) gx = items.count();
  if (gx < 1) gx = 1;
  k_forces_fwd_r5<<<gx, NT, BYTES, st>>>(a, items);
  return 1;
}

// Forward-phase element kernel with 2 events per thread and the next
// element's gather prefetched into registers (single-buffered shared
// displacement, stored once the current element's stresses have been
// read), LB events per block.  LB is at most the 8-lane sector group, so a
// work item never spans two groups of a group map.  Four block barriers per
// element, items from an ItemRing.
template <int LB, bool GEN = false>
struct FwdRLayout {
  static constexpr int NE = NGLL3;
  static constexpr int PPU = GEN ? 6 * NGLL3 : PP_U;   // U, then 5 (6) values
  static constexpr int OFF_IB = 0;                      // int [3][NE]
  static constexpr int OFF_IT = al4(OFF_IB + 3 * NE);   // int [2][4] item ring
  static constexpr int OFF_KM = al4(OFF_IT + 8);        // [2][2][NE]
  static constexpr int OFF_U = al4(OFF_KM + 4 * NE);    // [PPU][LB]
  static constexpr int OFF_A = al4(OFF_U + PPU * LB);   // [PP_A][LB]
  static constexpr int TOTAL = OFF_A + PP_A * LB;
  static constexpr size_t BYTES = (size_t)TOTAL * 4;
};

template <int LB, bool COLOURED, bool GEN = false>
__global__ void __launch_bounds__(25 * LB / 2) k_forces_fwd_r(StepArgs A, PipeItems items) {
  constexpr int NL = 2;
  constexpr int NT = 25 * LB / NL;
  using LY = FwdRLayout<LB, GEN>;
  constexpr int NE = NGLL3;
  constexpr int LWLOG = 3;
  extern __shared__ float sm[];
  int* sIB = (int*)(sm + LY::OFF_IB);
  const ItemRing ring{(int*)(sm + LY::OFF_IT), (int*)(sm + LY::OFF_IT) + 4};
  float* sKM = sm + LY::OFF_KM;
  float* sU = sm + LY::OFF_U;
  float* sA = sm + LY::OFF_A;

  const int tid = threadIdx.x;
  const int lq = tid % (LB / NL);
  const int t = tid / (LB / NL);
  const int lane = lq * NL;
  const int pi = t % 5, pq = t / 5;
  const int nev = A.nev;
  // element ids index the mesh arrays (with colouring, `order` is this
  // colour's part of the colour order); nspec marks an item past the end
  const int nel = A.m.nspec;
  const int nitems = items.count();
  const int G = gridDim.x;

  bool any = false;
  for (int l = tid; l < nev; l += NT) {
    const LaneDesc* L = A.lanes + l;
    any |= L->phase != PH_IDLE && L->it0 + A.s < L->nstep;
  }
  if (!__syncthreads_or(any)) return;
  if (A.lm.lwlog != LWLOG) return;  // batched layout only

  // running flags of this thread's two lanes of a chunk
  int c_chunk = -1, c_fl[NL] = {0, 0};
  auto flags = [&](int chunk, int& lg0, int fl[NL]) -> int {
    lg0 = chunk * LB + lane;
    if (chunk != c_chunk) {
#pragma unroll
      for (int n = 0; n < NL; ++n) {
        int f = 0;
        const int lg = lg0 + n;
        if (chunk < items.nchunk && lg < nev) {
          const LaneDesc* L = A.lanes + lg;
          const int it = L->it0 + A.s;
          if (L->phase != PH_IDLE && it < L->nstep) f = 1;
        }
        c_fl[n] = f;
      }
      c_chunk = chunk;
    }
    fl[0] = c_fl[0];
    fl[1] = c_fl[1];
    return fl[0] | fl[1];
  };
  // ibool row of element e into slot `slot` (-1 past the end)
  auto issue_ib = [&](int e, int slot) {
    int* dst = sIB + slot * NE;
    for (int i = tid; i < NE; i += NT) {
      if (e < nel)
        cp_async4(dst + i, A.m.ibool + (size_t)e * NGLL3 + i);
      else
        dst[i] = -1;
    }
  };
  // kappa and mu of element e into buffer buf
  auto issue_km = [&](int e, int buf) {
    if (e >= nel) return;
    float* km = sKM + buf * 2 * NE;
    for (int i = tid; i < NE; i += NT) {
      const size_t ep = (size_t)e * NGLL3 + i;
      cp_async4(km + i, A.m.kappa + ep);
      cp_async4(km + NE + i, A.m.mu + ep);
    }
  };
  float2 pre[5][3];
  auto load_u = [&](int chunk, int ibslot) {
    int lg0, fl[NL];
    const int anyf = flags(chunk, lg0, fl);
    const int* ib = sIB + ibslot * NE;
    const float* src = A.f1.u + fbase<LWLOG>(A, lg0);
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      const int ig = ib[t + 25 * r];
#pragma unroll
      for (int c = 0; c < 3; ++c)
        ldg_pred(pre[r][c], src + foff<LWLOG>(ig, c), anyf && ig >= 0);
    }
  };
  auto store_u = [&]() {
    float* ub = sU + lane;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      const int p = t + 25 * r;
#pragma unroll
      for (int c = 0; c < 3; ++c)
        *reinterpret_cast<float2*>(ub + (c * NGLL3 + p) * LB) = pre[r][c];
    }
  };

  int w = blockIdx.x;
  if (tid == 0)
    for (int j = 0; j < 3; ++j) ring.fill(items, A.m.order, nel, w + j * G, j);
  cp_commit();
  cp_wait_all();
  __syncthreads();
  issue_ib(ring.e[0], 0);
  cp_commit();
  cp_wait_all();
  __syncthreads();
  issue_km(ring.e[0], 0);
  issue_ib(ring.e[1], 1);
  cp_commit();
  load_u(ring.c[0], 0);
  store_u();

  const float fac = A.m.jac * A.m.xix * A.m.xix;
  for (int k = 0; w < nitems; ++k, w += G) {
    const int buf = k & 1;
    const int ibs = k % 3;
    cp_wait_all();
    __syncthreads();  // U holds this item's displacement, its copies landed, the last scatter is done
    PBuf<LB> b{sU + lane, sA + lane};
    grad_gamma_regs<LB>(b, t, pre);  // before the next gather replaces pre
    if (tid == 0) ring.fill(items, A.m.order, nel, w + 3 * G, (k + 3) & 3);
    issue_km(ring.e[(k + 1) & 3], buf ^ 1);
    issue_ib(ring.e[(k + 2) & 3], (k + 2) % 3);
    cp_commit();
    load_u(ring.c[(k + 1) & 3], (k + 1) % 3);

    int lg0, fl[NL];
    const int anyf = flags(ring.c[k & 3], lg0, fl);
    const int e = ring.e[k & 3];
    const bool valid = e < nel;
    const float* geo_e = nullptr;
    if (GEN && valid) {
      const int ir = A.m.irreg[e];
      if (ir >= 0) geo_e = A.m.geo + (size_t)ir * NGLL3 * 10;
    }
    const float* kap = sKM + buf * 2 * NE;
    const float* mu = kap + NE;
    v_grad_eg<LB, NL, false>(b, pi, pq);
    __syncthreads();
    LV<NL> fx[5][3], km[1], kk[1];
    v_xi<LB, NL, 0, GEN>(b, b, t, kap, mu, fac, fx, km, kk, geo_e, A.m.xix, A.m.jac);
    __syncthreads();
    v_div_eg<LB, NL, GEN>(b, pi, pq);
    __syncthreads();  // U's stresses read: it takes the next displacement
    store_u();
    if (valid && anyf)
      v_scatter<LB, NL, !COLOURED>(b, t, fx, sIB + ibs * NE, A.f1.a + fbase<LWLOG>(A, lg0), fl, 1);
  }
  cp_wait_all();
}

template <int LB, bool COLOURED, bool GEN = false>
static int forces_fwd_r_cfg(const StepArgs& a, cudaStream_t st) {
  constexpr int NT = 25 * LB / 2;
  constexpr size_t BYTES = FwdRLayout<LB, GEN>::BYTES;
  static int blocks_per_sm = 0, sms = 0;
  if (!blocks_per_sm) {
    cudaFuncSetAttribute(k_forces_fwd_r<LB, COLOURED, GEN>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BYTES);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm,
                                                  k_forces_fwd_r<LB, COLOURED, GEN>, NT, BYTES);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (blocks_per_sm < 1) blocks_per_sm = 1;
  }
  auto launch = [&](const StepArgs& ac, int nel) {
    PipeItems items = make_items<LB>(ac, nel);
    if (items.count() == 0) return 0;
    int gx = blocks_per_sm * sm_share(a, sms);
    if (gx > items.count()) gx = items.count();
    if (gx < 1) gx = 1;
    k_forces_fwd_r<LB, COLOURED, GEN><<<gx, NT, BYTES, st>>>(ac, items);
    return 1;
  };
  if (!COLOURED) return launch(a, a.m.nspec);
  // one launch per colour: within a colour no two elements share a point,
  // so the scatter is a plain read-modify-write
  int n = 0;
  for (int c = 0; c < a.m.ncolour; ++c) {
    StepArgs ac = a;
    ac.m.order = a.m.corder + a.m.cstart[c];
    n += launch(ac, a.m.cstart[c + 1] - a.m.cstart[c]);
  }
  return n;
}

template <int LB>
static void forces_adjpair_cfg(const StepArgs& a, cudaStream_t st) {
  constexpr int NT = 25 * LB;
  constexpr size_t BYTES = PairLayout<LB>::BYTES;
  static int blocks_per_sm = 0, sms = 0;
  if (!blocks_per_sm) {
    cudaFuncSetAttribute(k_forces_adjpair<LB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)BYTES);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_forces_adjpair<LB>, NT, BYTES);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (blocks_per_sm < 1) blocks_per_sm = 1;
  }
  PipeItems items = make_items<LB>(a, a.m.nspec);
  if (items.count() == 0) return;
  int gx = blocks_per_sm * sm_share(a, sms);
  if (gx > items.count()) gx = items.count();
  if (gx < 1) gx = 1;
  k_forces_adjpair<LB><<<gx, NT, BYTES, st>>>(a, items);
}

template <int LB, int NL, bool ADJ>
static void forces_vec_cfg(const StepArgs& a, cudaStream_t st) {
  using LY = PipeLayout<LB, 1, 25, ADJ>;
  constexpr int NT = 25 * LB / NL;
  static int blocks_per_sm = 0, sms = 0;
  if (!blocks_per_sm) {
    cudaFuncSetAttribute(k_forces_vec<LB, NL, ADJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)LY::BYTES);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_forces_vec<LB, NL, ADJ>, NT,
                                                  LY::BYTES);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (blocks_per_sm < 1) blocks_per_sm = 1;
  }
  PipeItems items = make_items<LB>(a, a.m.nspec);
  if (items.count() == 0) return;
  int gx = blocks_per_sm * sm_share(a, sms);
  if (gx > items.count()) gx = items.count();
  if (gx < 1) gx = 1;
  k_forces_vec<LB, NL, ADJ><<<gx, NT, LY::BYTES, st>>>(a, items);
}

// Element-kernel variants (StepArgs::variant):
//   0 thread-per-point, 1 pencil, 2 pencil pipelined (lanes per block by
//   event count), 3 pencil pipelined with 2 lanes per block, 4 pencil
//   pipelined with 2 lanes per thread, 5 as 4 with more lanes per block,
//   6 / 7 adjoint phase with the (adjoint, backward) field pair of an
//   event as a float2, 4 / 8 events per block, 8 / 9 the same with the
//   displacement prefetched into registers, 10 forward phase with 2 events
//   per thread and register prefetch (8 events per block).
int launch_forces(const StepArgs& a, bool adj, cudaStream_t st) {
  // the kernel follows the wavefield layout, not the lane count: a lane
  // group of a batch (lane-group layout) that holds one event still takes
  // the batch's kernels, whose lanes past the batch are idle
  const bool batched = a.lm.lwlog != 0;
  if (a.m.geo) {
    // a mesh with irregular elements: the register-prefetch kernels with
    // the general mapping (variant 10, batched), else the thread-per-point
    // kernel with the general mapping
    if (a.variant == 10 && batched) {
      if (!adj) return forces_fwd_r_cfg<8, false, true>(a, st);
      forces_adjpair_r_cfg<8, true>(a, st);
      return 1;
    }
    if (!batched) {
      if (adj)
        forces_cfg<1, 128, true, true>(a, st);
      else
        forces_cfg<1, 128, false, true>(a, st);
    } else {
      if (adj)
        forces_cfg<8, 256, true, true>(a, st);
      else
        forces_cfg<8, 256, false, true>(a, st);
    }
    return 1;
  }
  if (a.variant == 12 && !a.gmap) return adj ? forces_shfl_cfg<true>(a, st) : forces_shfl_cfg<false>(a, st);
  if (a.variant == 10 && batched) {
    if (!adj) return forces_fwd_r_cfg<8, false>(a, st);
    forces_adjpair_r_cfg<8>(a, st);
    return 1;
  }
  if (a.variant == 11 && batched) {
    if (!adj) return a.m.ncolour > 0 ? forces_fwd_r_cfg<8, true>(a, st)
                                     : forces_fwd_r_cfg<8, false>(a, st);
    forces_adjpair_r_cfg<8>(a, st);
    return 1;
  }
  if (a.variant == 13 && batched) {
    if (!adj) return forces_fwd_r_cfg<8, false>(a, st);
    forces_adjpair_r3_cfg(a, st);
    return 1;
  }
  if (a.variant == 14 && batched) {
    if (!adj) return forces_fwd_r5_cfg(a, st);
    forces_adjpair_r_cfg<8>(a, st);
    return 1;
  }
  if ((a.variant >= 6 && a.variant <= 9) && batched) {
    if (!adj)
      forces_vec_cfg<8, 2, false>(a, st);
    else if (a.variant == 6)
      forces_adjpair_cfg<4>(a, st);
    else if (a.variant == 7)
      forces_adjpair_cfg<8>(a, st);
    else if (a.variant == 8)
      forces_adjpair_r_cfg<4>(a, st);
    else
      forces_adjpair_r_cfg<8>(a, st);
    return 1;
  }
  if (a.variant == 4 && batched) {
    if (adj)
      forces_vec_cfg<4, 2, true>(a, st);
    else
      forces_vec_cfg<8, 2, false>(a, st);
    return 1;
  }
  if (a.variant == 5 && batched) {
    if (adj)
      forces_vec_cfg<8, 2, true>(a, st);
    else
      forces_vec_cfg<8, 4, false>(a, st);
    return 1;
  }
  if (a.variant == 3 && batched) {
    if (adj)
      forces_piped_cfg<2, 2, 25, true>(a, st);
    else
      forces_piped_cfg<2, 2, 25, false>(a, st);
    return 1;
  }
  if (a.variant == 2 || a.variant == 3) {
    if (!batched) {
      if (adj)
        forces_piped_cfg<1, 4, 32, true>(a, st);
      else
        forces_piped_cfg<1, 4, 32, false>(a, st);
    } else if (a.nev <= 4) {
      if (adj)
        forces_piped_cfg<4, 1, 25, true>(a, st);
      else
        forces_piped_cfg<4, 1, 25, false>(a, st);
    } else {
      if (adj)
        forces_piped_cfg<4, 1, 25, true>(a, st);
      else
        forces_piped_cfg<8, 1, 25, false>(a, st);
    }
    return 1;
  }
  if (a.variant == 1) {
    if (!batched) {
      if (adj)
        forces_pencil_cfg<1, 5, true>(a, st);
      else
        forces_pencil_cfg<1, 5, false>(a, st);
    } else if (a.nev <= 4) {
      if (adj)
        forces_pencil_cfg<4, 1, true>(a, st);
      else
        forces_pencil_cfg<4, 1, false>(a, st);
    } else {
      if (adj)
        forces_pencil_cfg<8, 1, true>(a, st);
      else
        forces_pencil_cfg<8, 1, false>(a, st);
    }
    return 1;
  }
  if (!batched) {
    if (adj)
      forces_cfg<1, 128, true>(a, st);
    else
      forces_cfg<1, 128, false>(a, st);
  } else {
    if (adj)
      forces_cfg<8, 256, true>(a, st);
    else
      forces_cfg<8, 256, false>(a, st);
  }
  return 1;
}

// ---------------------------------------------------------------------------
// Stacey absorbing faces: traction, boundary store save / replay
// ---------------------------------------------------------------------------

// Incident velocity and traction of face point fp at step it: the 4-point
// Lagrange interpolant of the samples at it / inj_np (exact when inj_np
// divides it), sample indices clamped to the stored range.
__device__ __forceinline__ void injected(const LaneDesc* L, int it, int fp, int npt, float vi[3],
                                         float ti[3]) {
  const int i1 = it / L->inj_np - L->inj_k0;
  const float x = (float)(it % L->inj_np) / (float)L->inj_np;
  float w[4];
  w[0] = -x * (x - 1.f) * (x - 2.f) * (1.f / 6.f);
  w[1] = (x + 1.f) * (x - 1.f) * (x - 2.f) * 0.5f;
  w[2] = -(x + 1.f) * x * (x - 2.f) * 0.5f;
  w[3] = (x + 1.f) * x * (x - 1.f) * (1.f / 6.f);
#pragma unroll
  for (int c = 0; c < 3; ++c) vi[c] = ti[c] = 0.f;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    if (q != 1 && x == 0.f) continue;
    const int k = min(max(i1 - 1 + q, 0), L->inj_nt - 1);
    const size_t b = ((size_t)k * npt + fp) * 3;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      vi[c] = fmaf(w[q], L->inj_v[b + c], vi[c]);
      ti[c] = fmaf(w[q], L->inj_t[b + c], ti[c]);
    }
  }
}

// Block of 128 threads = FPB faces x (32 point slots x LBB lanes).
// INJ: lanes may carry an FK injection (a separate instantiation, so that
// runs without one keep the plain kernel's registers).
template <int LBB, bool INJ>
__global__ void __launch_bounds__(128) k_stacey(StepArgs A) {
  constexpr int FPB = 128 / (32 * LBB);
  __shared__ unsigned s_max[FPB * LBB];
  const int t = threadIdx.x;
  const int fl = t / (32 * LBB);
  const int r = t % (32 * LBB);
  const int lane = r % LBB;
  const int p = r / LBB;
  const int f = blockIdx.x * FPB + fl;
  const int lg = blockIdx.y * LBB + lane;
  const int nf = A.m.nf;
  const int nev = A.nev;
  if (t < FPB * LBB) s_max[t] = 0u;
  __syncthreads();

  bool absorb = false, save = false, replay = false;
  int it = 0, nstep = 1;
  const LaneDesc* L = nullptr;
  if (lg < nev) {
    L = A.lanes + lg;
    it = L->it0 + A.s;
    nstep = L->nstep;
    if (L->phase != PH_IDLE && it < nstep) {
      absorb = true;
      save = (L->phase == PH_FWD) && L->save;
      replay = (L->phase == PH_ADJ) && it > 0;
    }
  }
  const bool valid = (f < nf) && (p < NGLL2) && (lg < nev);
  float sv[3] = {0.f, 0.f, 0.f};
  size_t ig = 0;
  if (valid) {
    const int fp = f * NGLL2 + p;
    ig = (size_t)A.m.f_iglob[fp];
    if (absorb) {
      const float nx = A.m.f_n[fp * 3 + 0], ny = A.m.f_n[fp * 3 + 1], nz = A.m.f_n[fp * 3 + 2];
      float vi[3] = {0.f, 0.f, 0.f}, ti[3] = {0.f, 0.f, 0.f};
      if (INJ && L->phase == PH_FWD && L->inj_v) injected(L, it, fp, nf * NGLL2, vi, ti);
      // FK injection: Stacey on the velocity relative to the incident field,
      // plus the incident traction
      const float vx = A.f1.v[A.fi(ig, 0, lg)] - vi[0];
      const float vy = A.f1.v[A.fi(ig, 1, lg)] - vi[1];
      const float vz = A.f1.v[A.fi(ig, 2, lg)] - vi[2];
      const float vn = vx * nx + vy * ny + vz * nz;
      const float rvp = A.m.f_rvp[fp], rvs = A.m.f_rvs[fp];
      const float jw = A.m.f_jw[fp];
      sv[0] = (rvp * vn * nx + rvs * (vx - vn * nx) - ti[0]) * jw;
      sv[1] = (rvp * vn * ny + rvs * (vy - vn * ny) - ti[1]) * jw;
      sv[2] = (rvp * vn * nz + rvs * (vz - vn * nz) - ti[2]) * jw;
#pragma unroll
      for (int c = 0; c < 3; ++c) atomicAdd(&A.f1.a[A.fi(ig, c, lg)], -sv[c]);
      if (save && A.store_fp16) {
        const float m = fmaxf(fabsf(sv[0]), fmaxf(fabsf(sv[1]), fabsf(sv[2])));
        atomicMax(&s_max[fl * LBB + lane], __float_as_uint(m));
      }
    }
  }
  if (A.store_fp16) __syncthreads();
  // row of record n in the lane's store (resident: n; ring: its chunk's
  // device slot, slots ring_nev * ring_c rows apart)
  auto row_of = [&](int n) -> size_t {
    if (L->ring_c <= 0) return (size_t)n;
    const int c = L->ring_c;
    return (size_t)((n / c) % L->ring_d) * (size_t)A.ring_nev * c + (size_t)(n % c);
  };
  if (valid && save) {
    const size_t row = row_of(it);
    const size_t base = (row * nf + f) * 75 + p * 3;
    if (A.store_fp16) {
      const float mx = __uint_as_float(s_max[fl * LBB + lane]);
      const float inv = mx > 0.f ? 32768.0f / mx : 0.f;
      __half* st = (__half*)L->store;
#pragma unroll
      for (int c = 0; c < 3; ++c) st[base + c] = __float2half_rn(sv[c] * inv);
      if (p == 0) L->scale[row * nf + f] = mx * (1.0f / 32768.0f);
    } else {
      float* st = (float*)L->store;
#pragma unroll
      for (int c = 0; c < 3; ++c) st[base + c] = sv[c];
    }
  }
  if (valid && replay) {
    const size_t row = row_of(nstep - 1 - it);
    const size_t base = (row * nf + f) * 75 + p * 3;
    float val[3];
    if (A.store_fp16) {
      const float sc = L->scale[row * nf + f];
      const __half* st = (const __half*)L->store;
#pragma unroll
      for (int c = 0; c < 3; ++c) val[c] = __half2float(st[base + c]) * sc;
    } else {
      const float* st = (const float*)L->store;
#pragma unroll
      for (int c = 0; c < 3; ++c) val[c] = st[base + c];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) atomicAdd(&A.f2.a[A.fi(ig, c, lg)], -val[c]);
  }
}

int launch_boundary(const StepArgs& a, bool adj, cudaStream_t st) {
  (void)adj;
  int n = 0;
  if (a.m.nf > 0) {
    if (a.nev == 1) {
      dim3 grid((a.m.nf + 3) / 4, 1);
      if (a.inject)
        k_stacey<1, true><<<grid, 128, 0, st>>>(a);
      else
        k_stacey<1, false><<<grid, 128, 0, st>>>(a);
    } else if (a.nev == 2) {
      dim3 grid((a.m.nf + 1) / 2, 1);
      if (a.inject)
        k_stacey<2, true><<<grid, 128, 0, st>>>(a);
      else
        k_stacey<2, false><<<grid, 128, 0, st>>>(a);
    } else {
      dim3 grid(a.m.nf, (a.nev + 3) / 4);
      if (a.inject)
        k_stacey<4, true><<<grid, 128, 0, st>>>(a);
      else
        k_stacey<4, false><<<grid, 128, 0, st>>>(a);
    }
    ++n;
  }
  return n;
}

// ---------------------------------------------------------------------------
// point sources, receivers and adjoint sources
// ---------------------------------------------------------------------------

// blocks [0, nev): moment-tensor source of one lane (forward field in the
// forward phase, backward field in the adjoint phase).
// blocks [nev, ...): one warp per (receiver, lane): record the forward
// displacement, or inject the adjoint source into the adjoint field.
__global__ void __launch_bounds__(128) k_points(StepArgs A) {
  const int nev = A.nev;
  if ((int)blockIdx.x < nev) {
    const int lg = blockIdx.x;
    const LaneDesc* L = A.lanes + lg;
    const int it = L->it0 + A.s;
    if (L->phase == PH_IDLE || it >= L->nstep || L->src_ispec < 0) return;
    float* acc;
    float s;
    if (L->phase == PH_FWD) {
      acc = A.f1.a;
      s = L->stf[it];
    } else {
      if (it == 0) return;
      acc = A.f2.a;
      s = L->stf[L->nstep - 1 - it];
    }
    const int p = threadIdx.x;
    if (p < NGLL3) {
      const size_t ig = (size_t)A.m.ibool[(size_t)L->src_ispec * NGLL3 + p];
#pragma unroll
      for (int c = 0; c < 3; ++c)
        atomicAdd(&acc[A.fi(ig, c, lg)], L->srcarr[p * 3 + c] * s);
    }
    return;
  }
  const int warp = threadIdx.x >> 5, ln = threadIdx.x & 31;
  const int pair = ((int)blockIdx.x - nev) * 4 + warp;
  const int r = pair / nev, lg = pair - r * nev;
  if (r >= A.nrec_max) return;
  const LaneDesc* L = A.lanes + lg;
  const int it = L->it0 + A.s;
  if (L->phase == PH_IDLE || it >= L->nstep || r >= L->nrec) return;
  const int e = L->rec_ispec[r];
  const float* w = L->rec_w + (size_t)r * NGLL3;
  if (L->phase == PH_FWD) {
    float s0 = 0.f, s1 = 0.f, s2 = 0.f;
    for (int p = ln; p < NGLL3; p += 32) {
      const size_t ig = (size_t)A.m.ibool[(size_t)e * NGLL3 + p];
      const float wp = w[p];
      s0 = fmaf(wp, A.f1.u[A.fi(ig, 0, lg)], s0);
      s1 = fmaf(wp, A.f1.u[A.fi(ig, 1, lg)], s1);
      s2 = fmaf(wp, A.f1.u[A.fi(ig, 2, lg)], s2);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s0 += __shfl_xor_sync(0xffffffffu, s0, o);
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if (ln == 0) {
      const size_t ns = (size_t)L->nstep;
      L->seis[((size_t)r * 3 + 0) * ns + it] = s0;
      L->seis[((size_t)r * 3 + 1) * ns + it] = s1;
      L->seis[((size_t)r * 3 + 2) * ns + it] = s2;
    }
  } else {
    const size_t ns = (size_t)L->nstep;
    const int n = L->nstep - 1 - it;
    const float a0 = L->adj[((size_t)r * 3 + 0) * ns + n];
    const float a1 = L->adj[((size_t)r * 3 + 1) * ns + n];
    const float a2 = L->adj[((size_t)r * 3 + 2) * ns + n];
    for (int p = ln; p < NGLL3; p += 32) {
      const size_t ig = (size_t)A.m.ibool[(size_t)e * NGLL3 + p];
      const float wp = w[p];
      atomicAdd(&A.f1.a[A.fi(ig, 0, lg)], wp * a0);
      atomicAdd(&A.f1.a[A.fi(ig, 1, lg)], wp * a1);
      atomicAdd(&A.f1.a[A.fi(ig, 2, lg)], wp * a2);
    }
  }
}

// ---------------------------------------------------------------------------
// Newmark corrector (this step) + predictor (next step)
// ---------------------------------------------------------------------------

// One thread per (point, lane), lanes of a group fastest, in 128-thread
// blocks.  HESS: also accumulate the approximate Hessian (a separate
// instantiation, so that the plain adjoint update keeps its code).
constexpr int kUpdThreads = 128;

template <bool ADJ, bool HESS = false>
__global__ void __launch_bounds__(kUpdThreads) k_update(StepArgs A) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int nev = A.nev;
  const int lwlog = A.lm.lwlog;
  const size_t nglob = (size_t)A.m.nglob;
  const size_t ngroups = A.gmap ? (size_t)A.ngmap : ((size_t)nev + (1u << lwlog) - 1) >> lwlog;
  if (idx >= (ngroups * nglob) << lwlog) return;
  const size_t kg = idx / (nglob << lwlog);
  const size_t rem = idx - kg * (nglob << lwlog);
  const size_t grp = A.gmap ? (size_t)A.gmap[kg] : kg;
  const size_t ig = rem >> lwlog;
  const int lg = (int)((grp << lwlog) + (rem & ((1u << lwlog) - 1)));
  if (lg >= nev) return;
  const LaneDesc* L = A.lanes + lg;
  const int it = L->it0 + A.s;
  const int ph = L->phase;
  if (ph == PH_IDLE || it >= L->nstep) return;
  const bool pred = it + 1 < L->nstep;
  const float dt = A.dt, dt2 = 0.5f * A.dt, dtsq2 = 0.5f * A.dt * A.dt;
  float u[3], v[3], a[3], mi[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const size_t q = A.fi(ig, c, lg);
    mi[c] = A.minv[ig * 3 + c];
    a[c] = A.f1.a[q] * mi[c];
    v[c] = A.f1.v[q] + dt2 * a[c];
    u[c] = A.f1.u[q];
  }
  if (ADJ && ph == PH_ADJ) {
    float bu[3], bv[3], ba[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t q = A.fi(ig, c, lg);
      bu[c] = A.f2.u[q];
      bv[c] = A.f2.v[q];
      ba[c] = A.f2.a[q];
      if (it > 0) {
        ba[c] = ba[c] * mi[c];
        bv[c] = bv[c] - dt2 * ba[c];
      }
    }
    A.k.rho_glob[A.gi(ig, lg)] += dt * (a[0] * bu[0] + a[1] * bu[1] + a[2] * bu[2]);
    // approximate Hessian: adjoint acceleration . backward acceleration
    if (HESS) A.k.hess_glob[A.gi(ig, lg)] += dt * (a[0] * ba[0] + a[1] * ba[1] + a[2] * ba[2]);
    if (pred) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        bu[c] = bu[c] - dt * bv[c] + dtsq2 * ba[c];
        bv[c] = bv[c] - dt2 * ba[c];
        ba[c] = 0.f;
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t q = A.fi(ig, c, lg);
      A.f2.u[q] = bu[c];
      A.f2.v[q] = bv[c];
      A.f2.a[q] = ba[c];
    }
  }
  if (pred) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      u[c] = u[c] + dt * v[c] + dtsq2 * a[c];
      v[c] = v[c] + dt2 * a[c];
      a[c] = 0.f;
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const size_t q = A.fi(ig, c, lg);
    A.f1.u[q] = u[c];
    A.f1.v[q] = v[c];
    A.f1.a[q] = a[c];
  }
}

int launch_update(const StepArgs& a, bool adj, cudaStream_t st) {
  const int lw = 1 << a.lm.lwlog;
  const size_t ng = a.gmap ? (size_t)a.ngmap : (size_t)((a.nev + lw - 1) / lw);
  const size_t n = (size_t)a.m.nglob * ng * lw;
  if (n == 0) return 0;
  // 128-thread blocks fit beside two resident blocks of the adjoint element
  // kernel, so the update of one lane group can run under another group's
  // element kernel
  const unsigned blocks = (unsigned)((n + kUpdThreads - 1) / kUpdThreads);
  if (adj && a.k.hess_glob)
    k_update<true, true><<<blocks, kUpdThreads, 0, st>>>(a);
  else if (adj)
    k_update<true><<<blocks, kUpdThreads, 0, st>>>(a);
  else
    k_update<false><<<blocks, kUpdThreads, 0, st>>>(a);
  return 1;
}

int launch_points(const StepArgs& a, cudaStream_t st) {
  const int blocks = a.nev + (a.nrec_max * a.nev + 3) / 4;
  k_points<<<blocks, 128, 0, st>>>(a);
  return 1;
}

__global__ void k_advance(LaneDesc* lanes, int nev, int k) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l < nev) lanes[l].it0 += k;
}

int launch_advance(LaneDesc* lanes, int nev, int k, cudaStream_t st) {
  k_advance<<<(nev + 127) / 128, 128, 0, st>>>(lanes, nev, k);
  return 1;
}

// ---------------------------------------------------------------------------
// kernels: final scaling (FP64) and cross-event FP64 sum
// ---------------------------------------------------------------------------

__global__ void k_finalize(MeshView m, const float* __restrict__ rho, KernAcc k, LaneMap lm,
                           int lane, double* __restrict__ out6, double* __restrict__ sum6) {
  const size_t ne = (size_t)m.nspec * NGLL3;
  const size_t ep = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ep >= ne) return;
  const double r = rho[ep], mu = m.mu[ep], kap = m.kappa[ep];
  const double rk = -r * (double)k.rho_glob[lm.p((size_t)m.ibool[ep], lane, (size_t)m.nglob)];
  const double mk = -2.0 * mu * (double)k.mu[lm.p(ep, lane, ne)];
  const double kk = -kap * (double)k.kappa[lm.p(ep, lane, ne)];
  const double v6[6] = {rk, mk, kk, rk + kk + mk, 2.0 * (mk - 4.0 / 3.0 * mu / kap * kk),
                        2.0 * (1.0 + 4.0 / 3.0 * mu / kap) * kk};
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    if (out6) out6[q * ne + ep] = v6[q];
    if (sum6) sum6[q * ne + ep] += v6[q];
  }
}

int launch_finalize_kernels(const MeshView& m, const float* rho, const KernAcc& k, LaneMap lm,
                            int lane, double* out6, double* sum6, cudaStream_t st) {
  const size_t ne = (size_t)m.nspec * NGLL3;
  k_finalize<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(m, rho, k, lm, lane, out6, sum6);
  return 1;
}

// hess_kernel: twice the accumulated sum, mapped from global to element
// points (the factor 2 of the approximate Hessian's scaling; a positive
// factor cancels in the preconditioner's normalisations).
__global__ void k_finalize_hess(MeshView m, const float* __restrict__ hess_glob, LaneMap lm,
                                int lane, double* __restrict__ out, double* __restrict__ sum,
                                int abs_each) {
  const size_t ne = (size_t)m.nspec * NGLL3;
  const size_t ep = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ep >= ne) return;
  const double h = 2.0 * (double)hess_glob[lm.p((size_t)m.ibool[ep], lane, (size_t)m.nglob)];
  if (out) out[ep] = h;
  if (sum) sum[ep] += abs_each ? fabs(h) : h;
}

int launch_finalize_hessian(const MeshView& m, const float* hess_glob, LaneMap lm, int lane,
                            double* out, double* sum, int abs_each, cudaStream_t st) {
  const size_t ne = (size_t)m.nspec * NGLL3;
  k_finalize_hess<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(m, hess_glob, lm, lane, out, sum,
                                                                 abs_each);
  return 1;
}

// ---------------------------------------------------------------------------
// L2 waveform misfit and adjoint source in FP64
// ---------------------------------------------------------------------------

// One block per (receiver, component) series.
__global__ void __launch_bounds__(256) k_measure_l2(const float* __restrict__ seis,
                                                    const double* __restrict__ obs,
                                                    const double* __restrict__ taper,
                                                    const double* __restrict__ simpw, int nstep,
                                                    float* __restrict__ adj,
                                                    double* __restrict__ misfit_rc) {
  __shared__ double red[256];
  const size_t base = (size_t)blockIdx.x * nstep;
  double acc = 0.0;
  for (int i = threadIdx.x; i < nstep; i += blockDim.x) {
    const double w = taper[i];
    const double r = (double)seis[base + i] * w - obs[base + i] * w;
    adj[base + i] = (float)(r * w);
    acc += simpw[i] * r * r;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) misfit_rc[blockIdx.x] = 0.5 * red[0];
}

int launch_measure_l2(const float* seis, const double* obs, const double* taper,
                      const double* simpw, int nrec, int nstep, float* adj_out,
                      double* misfit_rc, cudaStream_t st) {
  k_measure_l2<<<nrec * 3, 256, 0, st>>>(seis, obs, taper, simpw, nstep, adj_out, misfit_rc);
  return 1;
}

// ---------------------------------------------------------------------------
// lane utilities (phase transitions) and health check
// ---------------------------------------------------------------------------

__global__ void k_lane_copy(Fields s, Fields d, int nglob, LaneMap lm, int lane) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)nglob * 3) return;
  const size_t q = lm.f(i / 3, (int)(i % 3), lane, (size_t)nglob);
  d.u[q] = s.u[q];
  d.v[q] = s.v[q];
  d.a[q] = s.a[q];
}

__global__ void k_lane_zero(Fields f, int nglob, LaneMap lm, int lane) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)nglob * 3) return;
  const size_t q = lm.f(i / 3, (int)(i % 3), lane, (size_t)nglob);
  f.u[q] = 0.f;
  f.v[q] = 0.f;
  f.a[q] = 0.f;
}

int launch_lane_copy(const Fields& src, const Fields& dst, int nglob, LaneMap lm, int lane,
                     cudaStream_t st) {
  const size_t n = (size_t)nglob * 3;
  k_lane_copy<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(src, dst, nglob, lm, lane);
  return 1;
}

// One lane's values of the given per-point arrays (u, v, a of a field, or
// per-point records with rec values each) moved to another lane of the
// same run.
__global__ void k_lane_move(float* __restrict__ x0, float* __restrict__ x1, float* __restrict__ x2,
                            size_t npts, int rec, LaneMap lm, int from, int to) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts * rec) return;
  const size_t pnt = i / rec;
  const int c = (int)(i % rec);
  // lm.f() with `rec` values per point in place of 3
  const size_t lw = (size_t)1 << lm.lwlog;
  const size_t qf = ((((size_t)(from >> lm.lwlog)) * npts + pnt) * rec + c) * lw +
                    (from & (lw - 1));
  const size_t qt = ((((size_t)(to >> lm.lwlog)) * npts + pnt) * rec + c) * lw + (to & (lw - 1));
  x0[qt] = x0[qf];
  if (x1) x1[qt] = x1[qf];
  if (x2) x2[qt] = x2[qf];
}

int launch_lane_move(float* x0, float* x1, float* x2, size_t npts, int rec, LaneMap lm, int from,
                     int to, cudaStream_t st) {
  const size_t n = npts * rec;
  k_lane_move<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x0, x1, x2, npts, rec, lm, from, to);
  return 1;
}

int launch_lane_zero(const Fields& f, int nglob, LaneMap lm, int lane, cudaStream_t st) {
  const size_t n = (size_t)nglob * 3;
  k_lane_zero<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(f, nglob, lm, lane);
  return 1;
}

__global__ void k_lane_zero_acc(KernAcc k, int nglob, size_t ne, LaneMap lm, int lane) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < (size_t)nglob) {
    k.rho_glob[lm.p(i, lane, (size_t)nglob)] = 0.f;
    if (k.hess_glob) k.hess_glob[lm.p(i, lane, (size_t)nglob)] = 0.f;
  }
  if (i < ne) {
    k.mu[lm.p(i, lane, ne)] = 0.f;
    k.kappa[lm.p(i, lane, ne)] = 0.f;
  }
}

int launch_lane_zero_acc(const KernAcc& k, int nglob, size_t ne, LaneMap lm, int lane,
                         cudaStream_t st) {
  const size_t n = std::max((size_t)nglob, ne);
  k_lane_zero_acc<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(k, nglob, ne, lm, lane);
  return 1;
}

// Sum of n per-series misfits in series order (the order of a host loop)
// into *out.
__global__ void k_sum_series(const double* __restrict__ part, int n, double* out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double t = 0.0;
  for (int k = 0; k < n; ++k) t += part[k];
  *out = t;
}

int launch_sum_series(const double* part, int n, double* out, cudaStream_t st) {
  k_sum_series<<<1, 1, 0, st>>>(part, n, out);
  return 1;
}

// Periodic stability check of a run's wavefield u ([group][point][3][LW]):
// flags[lane] |= 1 for every running lane that holds a non-finite value.
// per_group = values per lane group (nglob * 3 * LW).
__global__ void k_check_lanes(const float* __restrict__ u, size_t n, size_t per_group, int lwlog,
                              const LaneDesc* __restrict__ lanes, int nev, int* flags) {
  const size_t lwm = ((size_t)1 << lwlog) - 1;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    if (!isfinite(u[i])) {
      const int lane = (int)(((i / per_group) << lwlog) + (i & lwm));
      if (lane < nev && lanes[lane].phase != PH_IDLE && !flags[lane]) atomicOr(&flags[lane], 1);
    }
  }
}

// Stops the flagged lanes: phase idle, so the remaining launches of the run
// skip them, and the step reached when the flag was first seen
// (it0 + s_off, at most the lane's nstep) in halt_step.
__global__ void k_halt_lanes(LaneDesc* lanes, int nev, const int* __restrict__ flags,
                             int* halt_step, int s_off) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nev; e += gridDim.x * blockDim.x) {
    LaneDesc& L = lanes[e];
    if (flags[e] && L.phase != PH_IDLE) {
      if (halt_step[e] < 0) halt_step[e] = min(L.it0 + s_off, L.nstep);
      L.phase = PH_IDLE;
    }
  }
}

int launch_check_lanes(const float* u, size_t nglob, int lwlog, int nevp, LaneDesc* lanes,
                       int nev, int* flags, cudaStream_t st) {
  const size_t per_group = nglob * 3 * ((size_t)1 << lwlog);
  k_check_lanes<<<148 * 4, 256, 0, st>>>(u, per_group * (size_t)(nevp >> lwlog), per_group,
                                         lwlog, lanes, nev, flags);
  return 1;
}

int launch_halt_lanes(LaneDesc* lanes, int nev, const int* flags, int* halt_step, int s_off,
                      cudaStream_t st) {
  k_halt_lanes<<<(nev + 127) / 128, 128, 0, st>>>(lanes, nev, flags, halt_step, s_off);
  return 1;
}

}  // namespace sem
