// PDE smoothing of element fields (kernels, Hessians) on the device.
//
// Reference: smooth_sem_pde (src/postproc/smooth.f90:7-437) and its GPU
// form smooth_pde_cuda_ (src/postproc/smooth_sem_pde.cu:298-478).  The
// smoother integrates an anisotropic diffusion equation explicitly:
//   project      dat_glob = sum_e(dat * rvol_local) / sum_e(rvol_local)
//   each step    ddat = -K dat_glob;  dat_glob += ddat / M;  CPML points = 0
//   output       dat(e) = dat_glob(ibool(e))
// with K the stiffness of the flux ((cv-ch) r (r.grad) + ch grad) and M
// the lumped volume, and cv, ch and the step count from the smoothing
// lengths and the minimum GLL point distance (smooth.f90:99-109).
//
// B200 layout: up to 4 fields are smoothed together, interleaved per global
// point ([nglob][F]); one launch per step sweeps all elements in Morton
// order (one 128-thread block per element, thread = GLL point), so a point
// record is one 4-16 byte vector and the fields share every ibool load.  At
// F = 4 on a 2.1M-point mesh the two point arrays (67 MB), ibool and the
// volume fit the 126 MB L2, so a step runs from L2.  Steps are replayed from
// a CUDA graph of 16 steps.
//
// Irregular (deformed) elements take their stored mapping terms and
// Jacobian at every GLL point, in the fluxes and in the lumped volume
// rvol_local = jacobian * w_i w_j w_k (smooth.f90:142-164 and its
// ispec_irreg branch :255-268; smooth_sem_pde.cu:149-160).  For regular
// elements `mapping` selects the mapping terms: the reference's regular
// branch sets all nine (xix .. gammaz) to xix_regular (smooth.f90:269-279,
// smooth_sem_pde.cu:161-170), which makes the operator a diffusion along
// (1,1,1) with coefficient 3(cv + 2ch), several times the stability bound
// that the step count assumes; SEM_SMOOTH_MAP_CUBE uses the cube's diagonal
// mapping (xix = etay = gammaz = xix_regular).

#include <cmath>
#include <cstdio>
#include <vector>

#include "sem_b200.h"
#include "sem_internal.cuh"

namespace sem {
namespace {

// GLL tables of the smoother: D[i][l] = l_l'(xi_i), DWt[i][l] = w_l D[l][i],
// w (double-precision values rounded to float, set once per process).
__constant__ float c_smooth_D[25];
__constant__ float c_smooth_DWt[25];
__constant__ float c_smooth_w[5];
__constant__ double c_smooth_w3[125];  // w_i w_j w_k in FP64, point i + 5j + 25k

struct SmoothArgs {
  int nspec, nglob;
  const int* ibool;   // [nspec*125]
  const int* order;   // [nspec]
  float M[3][3];      // mapping terms of a regular element: row xi/eta/gamma, column x/y/z
  float cv, ch, jac;
  const float* rot;   // [nglob][3] radial unit vector, or null (Cartesian)
  const int* irreg;   // [nspec] -1 or row of geo; null: all regular
  const float* geo;   // [nirr][125][10] xix..gammaz, jacobian
};

// rvol_local of element point q (element q / 125): real(dble(jacobian) *
// w_i w_j w_k) with the point's own Jacobian in an irregular element.
__device__ __forceinline__ float smooth_rvl(const int* __restrict__ irreg,
                                            const float* __restrict__ geo, float jac, size_t q) {
  const int p = (int)(q % NGLL3);
  float j = jac;
  if (irreg) {
    const int ir = irreg[q / NGLL3];
    if (ir >= 0) j = geo[((size_t)ir * NGLL3 + p) * 10 + 9];
  }
  return (float)((double)j * c_smooth_w3[p]);
}

template <int F>
struct Vec;
template <>
struct Vec<1> {
  using T = float;
};
template <>
struct Vec<2> {
  using T = float2;
};
template <>
struct Vec<4> {
  using T = float4;
};

template <int F>
__device__ __forceinline__ void vload(const float* p, float v[F]) {
  if constexpr (F == 1) {
    v[0] = *p;
  } else if constexpr (F == 2) {
    const float2 t = *reinterpret_cast<const float2*>(p);
    v[0] = t.x;
    v[1] = t.y;
  } else {
    const float4 t = *reinterpret_cast<const float4*>(p);
    v[0] = t.x;
    v[1] = t.y;
    v[2] = t.z;
    v[3] = t.w;
  }
}

template <int F>
__device__ __forceinline__ void vred(float* p, const float v[F]) {
  if constexpr (F == 1)
    atomicAdd(p, v[0]);
  else if constexpr (F == 2)
    atomicAdd(reinterpret_cast<float2*>(p), make_float2(v[0], v[1]));
  else
    atomicAdd(reinterpret_cast<float4*>(p), make_float4(v[0], v[1], v[2], v[3]));
}

// One element per block, thread p = GLL point (i + 5j + 25k), F fields.
// Gradient with D (hprime_xxT), fluxes, divergence with the weighted
// transpose (hprimewgll) and the wgllwgll face weights, scatter -sum.
template <int F>
__global__ void __launch_bounds__(128) k_smooth_elem(SmoothArgs A, const float* __restrict__ dat,
                                                     float* __restrict__ ddat) {
  __shared__ float su[F][NGLL3];
  __shared__ float sf[3][F][NGLL3];
  __shared__ float sD[25], sDW[25], sW[5];
  const int e = A.order[blockIdx.x];
  const int p = threadIdx.x;
  if (p < 25) {
    sD[p] = c_smooth_D[p];
    sDW[p] = c_smooth_DWt[p];
    if (p < 5) sW[p] = c_smooth_w[p];
  }
  const bool act = p < NGLL3;
  const int pp = act ? p : NGLL3 - 1;
  const int i = pp % 5, j = (pp / 5) % 5, k = pp / 25;
  const int ig = A.ibool[(size_t)e * NGLL3 + pp];
  // mapping terms and Jacobian at this point
  float M[3][3], jac = A.jac;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) M[r][c] = A.M[r][c];
  if (A.irreg) {
    const int ir = A.irreg[e];
    if (ir >= 0) {
      const float* G = A.geo + ((size_t)ir * NGLL3 + pp) * 10;
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) M[r][c] = G[3 * r + c];
      jac = G[9];
    }
  }
  {
    float v[F];
    vload<F>(dat + (size_t)ig * F, v);
    if (act)
#pragma unroll
      for (int f = 0; f < F; ++f) su[f][p] = v[f];
  }
  float r0 = 0.f, r1 = 0.f, r2 = 0.f;
  if (A.rot) {
    r0 = A.rot[(size_t)ig * 3 + 0];
    r1 = A.rot[(size_t)ig * 3 + 1];
    r2 = A.rot[(size_t)ig * 3 + 2];
  }
  __syncthreads();
#pragma unroll
  for (int f = 0; f < F; ++f) {
    // reference derivatives: hprime_xxT(l,i) = D[i][l]
    float t1 = 0.f, t2 = 0.f, t3 = 0.f;
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      t1 = fmaf(su[f][l + 5 * j + 25 * k], sD[i * 5 + l], t1);
      t2 = fmaf(su[f][i + 5 * l + 25 * k], sD[j * 5 + l], t2);
      t3 = fmaf(su[f][i + 5 * j + 25 * l], sD[k * 5 + l], t3);
    }
    const float dx = t1 * M[0][0] + t2 * M[1][0] + t3 * M[2][0];
    const float dy = t1 * M[0][1] + t2 * M[1][1] + t3 * M[2][1];
    const float dz = t1 * M[0][2] + t2 * M[1][2] + t3 * M[2][2];
    const float rg = r0 * dx + r1 * dy + r2 * dz;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float g = M[a][0] * dx + M[a][1] * dy + M[a][2] * dz;
      float s;
      if (A.rot)
        s = ((A.cv - A.ch) * (r0 * M[a][0] + r1 * M[a][1] + r2 * M[a][2]) * rg + A.ch * g) * jac;
      else
        s = ((A.cv - A.ch) * M[a][2] * dz + A.ch * g) * jac;
      if (act) sf[a][f][p] = s;
    }
  }
  __syncthreads();
  if (!act) return;
  const float wjk = sW[j] * sW[k], wik = sW[i] * sW[k], wij = sW[i] * sW[j];
  float out[F];
#pragma unroll
  for (int f = 0; f < F; ++f) {
    // divergence: hprimewgll_xx(l,i) = w_l D[l][i] = DWt[i][l]
    float n1 = 0.f, n2 = 0.f, n3 = 0.f;
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      n1 = fmaf(sf[0][f][l + 5 * j + 25 * k], sDW[i * 5 + l], n1);
      n2 = fmaf(sf[1][f][i + 5 * l + 25 * k], sDW[j * 5 + l], n2);
      n3 = fmaf(sf[2][f][i + 5 * j + 25 * l], sDW[k * 5 + l], n3);
    }
    out[f] = -(wjk * n1 + wik * n2 + wij * n3);
  }
  vred<F>(ddat + (size_t)ig * F, out);
}

// dat += ddat / M; ddat = 0; points of CPML elements reset to 0.
template <int F>
__global__ void k_smooth_update(float* __restrict__ dat, float* __restrict__ ddat,
                                const float* __restrict__ rvol, const unsigned char* __restrict__ cpml,
                                int nglob) {
  const int ig = blockIdx.x * blockDim.x + threadIdx.x;
  if (ig >= nglob) return;
  using V = typename Vec<F>::T;
  float a[F], d[F];
  vload<F>(dat + (size_t)ig * F, a);
  vload<F>(ddat + (size_t)ig * F, d);
  const float rv = rvol[ig];
  const bool zero = cpml && cpml[ig];
#pragma unroll
  for (int f = 0; f < F; ++f) a[f] = zero ? 0.f : a[f] + d[f] * rv;
  if constexpr (F == 1) {
    dat[ig] = a[0];
    ddat[ig] = 0.f;
  } else if constexpr (F == 2) {
    reinterpret_cast<V*>(dat)[ig] = make_float2(a[0], a[1]);
    reinterpret_cast<V*>(ddat)[ig] = make_float2(0.f, 0.f);
  } else {
    reinterpret_cast<V*>(dat)[ig] = make_float4(a[0], a[1], a[2], a[3]);
    reinterpret_cast<V*>(ddat)[ig] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

// Lumped volume: rvol(iglob) += rvol_local over element points.
__global__ void k_smooth_volume(const int* __restrict__ ibool, int nspec, const int* irreg,
                                const float* geo, float jac, float* vol) {
  const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (size_t)nspec * NGLL3) return;
  atomicAdd(&vol[ibool[q]], smooth_rvl(irreg, geo, jac, q));
}

__global__ void k_smooth_invert(float* v, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = 1.0f / v[i];
}

// Projection of F element fields (field f at din + f*ne) onto the points.
template <int F>
__global__ void k_smooth_project(const int* __restrict__ ibool, int nspec, const float* __restrict__ din,
                                 size_t ne, int nf_live, const int* irreg, const float* geo,
                                 float jac, float* __restrict__ dat) {
  const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (size_t)nspec * NGLL3) return;
  const int ig = ibool[q];
  const float w = smooth_rvl(irreg, geo, jac, q);
  float v[F];
#pragma unroll
  for (int f = 0; f < F; ++f) v[f] = f < nf_live ? din[f * ne + q] * w : 0.f;
  vred<F>(dat + (size_t)ig * F, v);
}

template <int F>
__global__ void k_smooth_scale(float* __restrict__ dat, const float* __restrict__ rvol, int nglob) {
  const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (size_t)nglob * F) return;
  dat[q] *= rvol[q / F];
}

template <int F>
__global__ void k_smooth_gather(const int* __restrict__ ibool, int nspec, const float* __restrict__ dat,
                                int nf_live, size_t ne, float* __restrict__ dout) {
  const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (size_t)nspec * NGLL3) return;
  const int ig = ibool[q];
#pragma unroll
  for (int f = 0; f < F; ++f)
    if (f < nf_live) dout[f * ne + q] = dat[(size_t)ig * F + f];
}

template <int F>
void launch_step(const SmoothArgs& a, float* dat, float* ddat, const float* rvol,
                 const unsigned char* cpml, cudaStream_t st) {
  k_smooth_elem<F><<<a.nspec, 128, 0, st>>>(a, dat, ddat);
  k_smooth_update<F><<<(a.nglob + 255) / 256, 256, 0, st>>>(dat, ddat, rvol, cpml, a.nglob);
}

template <int F>
void launch_project(const SmoothArgs& a, const float* din, size_t ne, int nf_live, float* dat,
                    const float* rvol, cudaStream_t st) {
  const size_t n = (size_t)a.nspec * NGLL3;
  k_smooth_project<F><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
      a.ibool, a.nspec, din, ne, nf_live, a.irreg, a.geo, a.jac, dat);
  k_smooth_scale<F><<<(unsigned)(((size_t)a.nglob * F + 255) / 256), 256, 0, st>>>(dat, rvol, a.nglob);
}

template <int F>
void launch_gather(const SmoothArgs& a, const float* dat, int nf_live, size_t ne, float* dout,
                   cudaStream_t st) {
  const size_t n = (size_t)a.nspec * NGLL3;
  k_smooth_gather<F><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a.ibool, a.nspec, dat, nf_live, ne,
                                                                  dout);
}

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

// Smoothing parameters in FP32 as the reference computes them (CUSTOM_REAL,
// smooth.f90:99-109).
void smooth_params(double sigma_h, double sigma_v, double dmin, float* cv, float* ch, double* nstep) {
  const float sh = (float)sigma_h, sv = (float)sigma_v, d = (float)dmin;
  const float cmax = d * d / 9.0f;
  if (sv >= sh) {
    *cv = cmax;
    *ch = *cv * (sh * sh) / (sv * sv);
  } else {
    *ch = cmax;
    *cv = *ch * (sv * sv) / (sh * sh);
  }
  const float mx = sh > sv ? sh : sv;
  *nstep = std::ceil((double)(mx * mx / (2.0f * cmax)));
}

}  // namespace
}  // namespace sem

using namespace sem;

#define SCK(call)                                                                        \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      cudaGetLastError();                                                                \
      if (graph) cudaGraphDestroy(graph);                                                \
      if (gexec) cudaGraphExecDestroy(gexec);                                            \
      if (st) cudaStreamDestroy(st);                                                     \
      if (ev0) cudaEventDestroy(ev0);                                                    \
      if (ev1) cudaEventDestroy(ev1);                                                    \
      return report_error(SEM_ERR_CUDA, "smoothing: %s: %s", #call, cudaGetErrorString(e_)); \
    }                                                                                    \
  } while (0)

extern "C" int sem_smooth_pde(sem_mesh* mesh, const sem_smooth_cfg* cfg, int nfield,
                              const float* dat_in, const int* is_cpml, float* dat_out,
                              sem_smooth_stats* stats) {
  NvtxPhase ph("sem_smooth_pde");
  if (!mesh || !cfg || !dat_in || !dat_out) return report_error(SEM_ERR_ARG, "null argument");
  if (nfield < 1) return report_error(SEM_ERR_ARG, "nfield must be >= 1");
  if (!(cfg->sigma_h >= 0.0) || !(cfg->sigma_v >= 0.0))
    return report_error(SEM_ERR_ARG, "sigma_h and sigma_v must be >= 0");
  if (cfg->mapping != SEM_SMOOTH_MAP_REFERENCE && cfg->mapping != SEM_SMOOTH_MAP_CUBE)
    return report_error(SEM_ERR_ARG, "mapping must be SEM_SMOOTH_MAP_REFERENCE or _CUBE");
  SmoothMeshView mv{};
  int rc = mesh_smooth_view(mesh, &mv);
  if (rc) return rc;
  // minimum GLL point distance: of a regular element (xi_1 - xi_0) / xix;
  // with irregular elements, the smallest distance between neighbouring
  // GLL points along the element's index lines over the whole mesh
  double dmin = cfg->distance_min;
  if (!(dmin > 0.0)) {
    if (mv.irreg) {
      double d2 = 1e300;
      for (int e = 0; e < mv.nspec; ++e) {
        const int* ib = mv.h_ibool + (size_t)e * NGLL3;
        for (int p = 0; p < NGLL3; ++p) {
          const int i = p % 5, j = (p / 5) % 5, k = p / 25;
          const int nb[3] = {i < 4 ? p + 1 : -1, j < 4 ? p + 5 : -1, k < 4 ? p + 25 : -1};
          for (int q : nb) {
            if (q < 0) continue;
            const double dx = (double)mv.x[ib[q]] - mv.x[ib[p]];
            const double dy = (double)mv.y[ib[q]] - mv.y[ib[p]];
            const double dz = (double)mv.z[ib[q]] - mv.z[ib[p]];
            d2 = std::min(d2, dx * dx + dy * dy + dz * dz);
          }
        }
      }
      dmin = std::sqrt(d2);
    } else {
      dmin = (1.0 - std::sqrt(3.0 / 7.0)) / (double)mv.xix;
    }
  }
  float cv = 0.f, ch = 0.f;
  double nstep_d = 0.0;
  smooth_params(cfg->sigma_h, cfg->sigma_v, dmin, &cv, &ch, &nstep_d);
  if (cfg->nstep > 0) nstep_d = cfg->nstep;
  if (!(nstep_d >= 0.0) || nstep_d > 1e7)
    return report_error(SEM_ERR_ARG, "smoothing step count %.0f outside [0, 1e7]", nstep_d);
  const int nstep = (int)nstep_d;

  SmoothArgs a{};
  a.nspec = mv.nspec;
  a.nglob = mv.nglob;
  a.ibool = mv.ibool;
  a.order = mv.order;
  a.cv = cv;
  a.ch = ch;
  a.jac = mv.jac;
  a.irreg = mv.irreg;
  a.geo = mv.geo;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      a.M[r][c] = (cfg->mapping == SEM_SMOOTH_MAP_REFERENCE || r == c) ? mv.xix : 0.f;

  // host-side set-up: element-point volumes, radial vectors, CPML points
  const double xg[5] = {-1.0, -std::sqrt(3.0 / 7.0), 0.0, std::sqrt(3.0 / 7.0), 1.0};
  const double wg[5] = {0.1, 49.0 / 90.0, 32.0 / 45.0, 49.0 / 90.0, 0.1};
  double w3[NGLL3];
  for (int k = 0; k < 5; ++k)
    for (int j = 0; j < 5; ++j)
      for (int i = 0; i < 5; ++i) w3[i + 5 * j + 25 * k] = wg[i] * wg[j] * wg[k];
  {
    // D[i][l] = derivative of the l-th Lagrange polynomial at node i
    float hD[25], hDW[25], hW[5];
    double Dd[5][5];
    for (int i = 0; i < 5; ++i)
      for (int l = 0; l < 5; ++l) {
        double sum = 0.0;
        for (int m = 0; m < 5; ++m) {
          if (m == l) continue;
          double prod = 1.0 / (xg[l] - xg[m]);
          for (int n = 0; n < 5; ++n)
            if (n != l && n != m) prod *= (xg[i] - xg[n]) / (xg[l] - xg[n]);
          sum += prod;
        }
        Dd[i][l] = sum;
      }
    for (int i = 0; i < 5; ++i) {
      hW[i] = (float)wg[i];
      for (int l = 0; l < 5; ++l) {
        hD[i * 5 + l] = (float)Dd[i][l];
        hDW[i * 5 + l] = (float)(wg[l] * Dd[l][i]);
      }
    }
    cudaError_t e1 = cudaMemcpyToSymbol(c_smooth_D, hD, sizeof(hD));
    if (e1 == cudaSuccess) e1 = cudaMemcpyToSymbol(c_smooth_DWt, hDW, sizeof(hDW));
    if (e1 == cudaSuccess) e1 = cudaMemcpyToSymbol(c_smooth_w, hW, sizeof(hW));
    if (e1 == cudaSuccess) e1 = cudaMemcpyToSymbol(c_smooth_w3, w3, sizeof(w3));
    if (e1 != cudaSuccess) {
      cudaGetLastError();
      return report_error(SEM_ERR_CUDA, "smoothing tables: %s", cudaGetErrorString(e1));
    }
  }
  std::vector<float> rot;
  if (cfg->is_sph) {
    rot.resize((size_t)mv.nglob * 3);
    for (int g = 0; g < mv.nglob; ++g) {
      const float x = mv.x[g], y = mv.y[g], z = mv.z[g];
      const float rl = std::sqrt(x * x + y * y + z * z);
      if (!(rl > 0.f))
        return report_error(SEM_ERR_ARG, "is_sph: mesh point %d is at the origin", g);
      rot[(size_t)g * 3 + 0] = x / rl;
      rot[(size_t)g * 3 + 1] = y / rl;
      rot[(size_t)g * 3 + 2] = z / rl;
    }
  }
  std::vector<unsigned char> cpml;
  if (is_cpml) {
    cpml.assign(mv.nglob, 0);
    for (int e = 0; e < mv.nspec; ++e)
      if (is_cpml[e])
        for (int p = 0; p < NGLL3; ++p) cpml[mv.h_ibool[(size_t)e * NGLL3 + p]] = 1;
  }

  cudaStream_t st = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  const int F = nfield >= 3 ? 4 : (nfield == 2 ? 2 : 1);
  const size_t ne = (size_t)mv.nspec * NGLL3;
  DevBuf b_dat, b_ddat, b_rvol, b_rot, b_cpml, b_din;
  SCK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  SCK(cudaEventCreate(&ev0));
  SCK(cudaEventCreate(&ev1));
  SCK(cudaMalloc(&b_dat.p, (size_t)mv.nglob * F * sizeof(float)));
  SCK(cudaMalloc(&b_ddat.p, (size_t)mv.nglob * F * sizeof(float)));
  SCK(cudaMalloc(&b_rvol.p, (size_t)mv.nglob * sizeof(float)));
  SCK(cudaMalloc(&b_din.p, ne * F * sizeof(float)));
  float* dat = (float*)b_dat.p;
  float* ddat = (float*)b_ddat.p;
  float* rvol = (float*)b_rvol.p;
  float* din = (float*)b_din.p;
  const unsigned char* dcpml = nullptr;
  if (!rot.empty()) {
    SCK(cudaMalloc(&b_rot.p, rot.size() * sizeof(float)));
    SCK(cudaMemcpyAsync(b_rot.p, rot.data(), rot.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    a.rot = (const float*)b_rot.p;
  }
  if (!cpml.empty()) {
    SCK(cudaMalloc(&b_cpml.p, cpml.size()));
    SCK(cudaMemcpyAsync(b_cpml.p, cpml.data(), cpml.size(), cudaMemcpyHostToDevice, st));
    dcpml = (const unsigned char*)b_cpml.p;
  }
  SCK(cudaMemsetAsync(rvol, 0, (size_t)mv.nglob * sizeof(float), st));
  k_smooth_volume<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(a.ibool, a.nspec, a.irreg, a.geo,
                                                                 a.jac, rvol);
  k_smooth_invert<<<(mv.nglob + 255) / 256, 256, 0, st>>>(rvol, mv.nglob);
  SCK(cudaGetLastError());

  constexpr int kGraphSteps = 16;
  auto step = [&](int nsteps) {
    for (int s = 0; s < nsteps; ++s) {
      if (F == 4)
        launch_step<4>(a, dat, ddat, rvol, dcpml, st);
      else if (F == 2)
        launch_step<2>(a, dat, ddat, rvol, dcpml, st);
      else
        launch_step<1>(a, dat, ddat, rvol, dcpml, st);
    }
  };
  const bool use_graph = nstep >= 2 * kGraphSteps;
  if (use_graph) {
    SCK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    step(kGraphSteps);
    SCK(cudaStreamEndCapture(st, &graph));
    SCK(cudaGraphInstantiate(&gexec, graph, 0));
  }
  double step_ms = 0.0;
  for (int f0 = 0; f0 < nfield; f0 += F) {
    const int live = nfield - f0 < F ? nfield - f0 : F;
    SCK(cudaMemcpyAsync(din, dat_in + (size_t)f0 * ne, (size_t)live * ne * sizeof(float),
                        cudaMemcpyHostToDevice, st));
    SCK(cudaMemsetAsync(dat, 0, (size_t)mv.nglob * F * sizeof(float), st));
    SCK(cudaMemsetAsync(ddat, 0, (size_t)mv.nglob * F * sizeof(float), st));
    if (F == 4)
      launch_project<4>(a, din, ne, live, dat, rvol, st);
    else if (F == 2)
      launch_project<2>(a, din, ne, live, dat, rvol, st);
    else
      launch_project<1>(a, din, ne, live, dat, rvol, st);
    SCK(cudaEventRecord(ev0, st));
    int left = nstep;
    if (use_graph)
      for (; left >= kGraphSteps; left -= kGraphSteps) SCK(cudaGraphLaunch(gexec, st));
    step(left);
    SCK(cudaEventRecord(ev1, st));
    if (F == 4)
      launch_gather<4>(a, dat, live, ne, din, st);
    else if (F == 2)
      launch_gather<2>(a, dat, live, ne, din, st);
    else
      launch_gather<1>(a, dat, live, ne, din, st);
    SCK(cudaGetLastError());
    SCK(cudaMemcpyAsync(dat_out + (size_t)f0 * ne, din, (size_t)live * ne * sizeof(float),
                        cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    float ms = 0.f;
    SCK(cudaEventElapsedTime(&ms, ev0, ev1));
    step_ms += ms;
  }
  if (stats) {
    stats->nstep = nstep;
    stats->cv = cv;
    stats->ch = ch;
    stats->distance_min = dmin;
    stats->fields_per_pass = F;
    stats->step_ms = step_ms;
  }
  if (gexec) cudaGraphExecDestroy(gexec);
  if (graph) cudaGraphDestroy(graph);
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  cudaStreamDestroy(st);
  return SEM_OK;
}
