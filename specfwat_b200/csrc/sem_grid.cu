// Kernels on the model grid, on the device:
//  - gll2grid: element fields projected onto a regular grid
//    (src/grid/model_grid_data.f90:183-198; compute_interpolation_coeff_FD_SEM
//    and Project_model_SEM2FD_grid, src/shared/projection_on_FD_grid_mod_fwat.f90:
//    186-596, with locate_point_in_element :935-1125);
//  - taper_kernel_grid: the grid kernels times a 3-D boundary taper
//    (src/postproc/post_processing.f90:283-325, taper_cls in
//    src/postproc/taper_3D_mod.f90, the trilinear interp3 of
//    src/shared/utils.f90:1089-1159);
//  - zprecond_grid: the depth preconditioner on the grid
//    (src/postproc/zprecond.f90:73-100).
//
// The projection follows the reference loop's rule that the first element
// whose candidate range holds a grid point takes it: every element writes
// its index into the points of its range with atomicMin, and a second
// kernel evaluates each point from the element left there.  All of it is
// FP64; the projected values are rounded to FP32 as the reference's
// CUSTOM_REAL grid.

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "sem_b200.h"
#include "sem_internal.cuh"

namespace sem {
namespace {

struct GridGeom {
  double x0[3], h[3];
  int n[3];
};

// Separable taper: 1-D windows w[d][0..n[d]) on the points xmin[d] + i h[d]
struct TaperGeom {
  double xmin[3], h[3];
  int n[3];
  const double* w[3];
};

__device__ __forceinline__ double gll_node(int i) {
  const double a = sqrt(3.0 / 7.0);
  return i == 0 ? -1.0 : i == 1 ? -a : i == 2 ? 0.0 : i == 3 ? a : 1.0;
}

// GLL Lagrange polynomials h_0..h_4 at x, each a running product of the
// factors (x - x_m) / (x_i - x_m)
__device__ void lagrange5(double x, double h[5]) {
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    double v = 1.0;
#pragma unroll
    for (int m = 0; m < 5; ++m)
      if (m != i) v *= (x - gll_node(m)) / (gll_node(i) - gll_node(m));
    h[i] = v;
  }
}

__device__ __forceinline__ double clamp1(double v) { return fmin(fmax(v, -1.0), 1.0); }

// Fortran integer assignment of a real: truncation toward zero
__device__ __forceinline__ int trunc_int(double v) {
  v = fmin(fmax(v, -2.0e9), 2.0e9);
  return (int)v;
}

// Per element (one block of 128 threads): the bounding box of its 125 GLL
// points and its grid candidates, index ranges [1 + (lo - x0) / h] - 1 ..
// [1 + (hi - x0) / h] - 1 truncated and cut to the grid; every candidate
// keeps the smallest element index, the first element of the reference's
// loop that takes it.
__global__ void __launch_bounds__(128) k_grid_claim(const int* __restrict__ ibool,
                                                    const float* __restrict__ x,
                                                    const float* __restrict__ y,
                                                    const float* __restrict__ z, GridGeom g,
                                                    double* __restrict__ box,
                                                    int* __restrict__ owner) {
  __shared__ double s_part[6][4];
  __shared__ int s_rng[6];
  const int e = blockIdx.x;
  const int t = threadIdx.x;
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  if (t < NGLL3) {
    const int ig = ibool[(size_t)e * NGLL3 + t];
    const double c[3] = {(double)x[ig], (double)y[ig], (double)z[ig]};
#pragma unroll
    for (int d = 0; d < 3; ++d) lo[d] = hi[d] = c[d];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
  if ((t & 31) == 0)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      s_part[d][t >> 5] = lo[d];
      s_part[3 + d][t >> 5] = hi[d];
    }
  __syncthreads();
  if (t == 0) {
    for (int d = 0; d < 3; ++d) {
      double l = s_part[d][0], u = s_part[3 + d][0];
      for (int w = 1; w < 4; ++w) {
        l = fmin(l, s_part[d][w]);
        u = fmax(u, s_part[3 + d][w]);
      }
      box[(size_t)e * 6 + d] = l;
      box[(size_t)e * 6 + 3 + d] = u;
      const int i0 = trunc_int(1.0 + (l - g.x0[d]) / g.h[d]) - 1;
      const int i1 = trunc_int(1.0 + (u - g.x0[d]) / g.h[d]) - 1;
      s_rng[d] = max(i0, 0);
      s_rng[3 + d] = min(i1, g.n[d] - 1);
    }
  }
  __syncthreads();
  const int ax = s_rng[0], ay = s_rng[1], az = s_rng[2];
  const int bx = s_rng[3], by = s_rng[4], bz = s_rng[5];
  if (bx < ax || by < ay || bz < az) return;
  const long long ny = by - ay + 1, nz = bz - az + 1;
  const long long cnt = (long long)(bx - ax + 1) * ny * nz;
  for (long long q = t; q < cnt; q += blockDim.x) {
    const int iz = az + (int)(q % nz);
    const long long r = q / nz;
    const int iy = ay + (int)(r % ny);
    const int ix = ax + (int)(r / ny);
    atomicMin(owner + ((size_t)ix * g.n[1] + iy) * g.n[2] + iz, e);
  }
}

// 1-D shape functions of the anchor nodes, on m = 2 ([-1, 1]) or 3
// ([-1, 0, 1]) nodes: values l and derivatives dl at u
__device__ __forceinline__ void anchor_shape(double u, int m, double l[3], double dl[3]) {
  if (m == 2) {
    l[0] = 0.5 * (1.0 - u);
    l[1] = 0.5 * (1.0 + u);
    dl[0] = -0.5;
    dl[1] = 0.5;
    l[2] = dl[2] = 0.0;
  } else {
    l[0] = 0.5 * u * (u - 1.0);
    l[1] = 1.0 - u * u;
    l[2] = 0.5 * u * (u + 1.0);
    dl[0] = u - 0.5;
    dl[1] = -2.0 * u;
    dl[2] = u + 0.5;
  }
}

// locate_point_in_element for one target: the initial guess at the nearest
// of the element's 27 interior GLL nodes (the first in k, j, i order), then
// NUM_ITER = 4 Newton steps on the mapping of the ngnod anchor nodes (8:
// corners; 27: corners, edge, face and centre GLL nodes), each step's
// coordinates clamped to [-1, 1].
__device__ void locate(const int* __restrict__ ib, const float* __restrict__ x,
                       const float* __restrict__ y, const float* __restrict__ z,
                       const double tp[3], int ngnod, double ref[3]) {
  double best = INFINITY;
  int bi = 1, bj = 1, bk = 1;
  for (int k = 1; k < 4; ++k)
    for (int j = 1; j < 4; ++j)
      for (int i = 1; i < 4; ++i) {
        const int ig = ib[i + 5 * j + 25 * k];
        const double dx = tp[0] - (double)x[ig], dy = tp[1] - (double)y[ig],
                     dz = tp[2] - (double)z[ig];
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < best) {
          best = d2;
          bi = i;
          bj = j;
          bk = k;
        }
      }
  ref[0] = gll_node(bi);
  ref[1] = gll_node(bj);
  ref[2] = gll_node(bk);
  const int m = ngnod == 8 ? 2 : 3;
  const int sel[3] = {0, m == 2 ? 4 : 2, 4};
  double anc[3][3][3][3];  // [c][b][a][coordinate]
  for (int c = 0; c < m; ++c)
    for (int b = 0; b < m; ++b)
      for (int a = 0; a < m; ++a) {
        const int ig = ib[sel[a] + 5 * sel[b] + 25 * sel[c]];
        anc[c][b][a][0] = (double)x[ig];
        anc[c][b][a][1] = (double)y[ig];
        anc[c][b][a][2] = (double)z[ig];
      }
  for (int it = 0; it < 4; ++it) {
    double la[3], da[3], lb[3], db[3], lc[3], dc[3];
    anchor_shape(ref[0], m, la, da);
    anchor_shape(ref[1], m, lb, db);
    anchor_shape(ref[2], m, lc, dc);
    double xm[3] = {0.0, 0.0, 0.0}, J[3][3] = {{0.0}};
    for (int c = 0; c < m; ++c)
      for (int b = 0; b < m; ++b)
        for (int a = 0; a < m; ++a) {
          const double w = la[a] * lb[b] * lc[c];
          const double wx = da[a] * lb[b] * lc[c];
          const double wy = la[a] * db[b] * lc[c];
          const double wz = la[a] * lb[b] * dc[c];
          for (int d = 0; d < 3; ++d) {
            const double v = anc[c][b][a][d];
            xm[d] += w * v;
            J[d][0] += wx * v;
            J[d][1] += wy * v;
            J[d][2] += wz * v;
          }
        }
    // J dr = tp - xm by Gaussian elimination with partial pivoting
    double A[3][4];
    for (int d = 0; d < 3; ++d) {
      A[d][0] = J[d][0];
      A[d][1] = J[d][1];
      A[d][2] = J[d][2];
      A[d][3] = tp[d] - xm[d];
    }
    for (int col = 0; col < 3; ++col) {
      int piv = col;
      for (int r = col + 1; r < 3; ++r)
        if (fabs(A[r][col]) > fabs(A[piv][col])) piv = r;
      if (piv != col)
        for (int q = 0; q < 4; ++q) {
          const double tmp = A[col][q];
          A[col][q] = A[piv][q];
          A[piv][q] = tmp;
        }
      for (int r = col + 1; r < 3; ++r) {
        const double f = A[r][col] / A[col][col];
        for (int q = col; q < 4; ++q) A[r][q] -= f * A[col][q];
      }
    }
    double dr[3];
    for (int r = 2; r >= 0; --r) {
      double s = A[r][3];
      for (int q = r + 1; q < 3; ++q) s -= A[r][q] * dr[q];
      dr[r] = s / A[r][r];
    }
    for (int d = 0; d < 3; ++d) ref[d] = clamp1(ref[d] + dr[d]);
  }
}

// Per grid point: the value of the owner element's 5x5x5 interpolant at
// the point's reference coordinates (affine elements: the linear
// coordinates in the element's box, clamped to it, which is where the
// locator's Newton steps land; irregular elements: the locator itself),
// or 0 where no element took the point.
__global__ void __launch_bounds__(128) k_grid_eval(
    const float* __restrict__ fields, int nfield, size_t nfe, const int* __restrict__ owner,
    const double* __restrict__ box, const int* __restrict__ irreg, const int* __restrict__ ibool,
    const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z,
    int nspec, GridGeom g, int ngnod, float* __restrict__ out, size_t ngrid) {
  for (size_t gp = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gp < ngrid;
       gp += (size_t)gridDim.x * blockDim.x) {
    const int e = owner[gp];
    if (e < 0 || e >= nspec) {
      for (int f = 0; f < nfield; ++f) out[(size_t)f * ngrid + gp] = 0.f;
      continue;
    }
    const int iz = (int)(gp % (size_t)g.n[2]);
    const size_t r = gp / (size_t)g.n[2];
    const int iy = (int)(r % (size_t)g.n[1]);
    const int ix = (int)(r / (size_t)g.n[1]);
    const double tp[3] = {g.x0[0] + (double)ix * g.h[0], g.x0[1] + (double)iy * g.h[1],
                          g.x0[2] + (double)iz * g.h[2]};
    double ref[3];
    if (irreg && irreg[e] >= 0) {
      locate(ibool + (size_t)e * NGLL3, x, y, z, tp, ngnod, ref);
    } else {
      for (int d = 0; d < 3; ++d) {
        const double lo = box[(size_t)e * 6 + d], hi = box[(size_t)e * 6 + 3 + d];
        ref[d] = clamp1(2.0 * (tp[d] - lo) / (hi - lo) - 1.0);
      }
    }
    double hx[5], hy[5], hz[5];
    lagrange5(ref[0], hx);
    lagrange5(ref[1], hy);
    lagrange5(ref[2], hz);
    for (int f = 0; f < nfield; ++f) {
      const float* ge = fields + (size_t)f * nfe + (size_t)e * NGLL3;
      double v = 0.0;
      for (int k = 0; k < 5; ++k)
        for (int j = 0; j < 5; ++j)
          for (int i = 0; i < 5; ++i)
            v += hx[i] * hy[j] * hz[k] * (double)ge[i + 5 * j + 25 * k];
      out[(size_t)f * ngrid + gp] = (float)v;
    }
  }
}

// Smallest and largest distance between neighbouring GLL points along the
// element's three index directions, per element
__global__ void k_elem_dist(const int* __restrict__ ibool, const float* __restrict__ x,
                            const float* __restrict__ y, const float* __restrict__ z, int nspec,
                            double* __restrict__ dmin, double* __restrict__ dmax) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nspec) return;
  const int* ib = ibool + (size_t)e * NGLL3;
  double lo = INFINITY, hi = 0.0;
  for (int p = 0; p < NGLL3; ++p) {
    const int i = p % 5, j = (p / 5) % 5, k = p / 25;
    const int nb[3] = {i < 4 ? p + 1 : -1, j < 4 ? p + 5 : -1, k < 4 ? p + 25 : -1};
    for (int q : nb) {
      if (q < 0) continue;
      const double dx = (double)x[ib[q]] - (double)x[ib[p]];
      const double dy = (double)y[ib[q]] - (double)y[ib[p]];
      const double dz = (double)z[ib[q]] - (double)z[ib[p]];
      const double d = sqrt(dx * dx + dy * dy + dz * dz);
      lo = fmin(lo, d);
      hi = fmax(hi, d);
    }
  }
  dmin[e] = lo;
  dmax[e] = hi;
}

// index of the last point xmin + k h at or below v, cut to [0, n-2]
// (locate_bissection with the bracket clamped)
__device__ __forceinline__ int taper_cell(double v, double xmin, double h, int n) {
  int k = (int)floor(fmin(fmax((v - xmin) / h, -2.0), (double)n + 1.0));
  while (k + 1 < n && xmin + (double)(k + 1) * h <= v) ++k;
  while (k >= 0 && xmin + (double)k * h > v) --k;
  return min(max(k, 0), n - 2);
}

// The grid kernels times the taper at their points: the trilinear value of
// the separable mask, 0 outside the mask's box (interp3)
__global__ void __launch_bounds__(128) k_grid_taper(float* __restrict__ grid, int nfield,
                                                    size_t ngrid, GridGeom g, TaperGeom tg,
                                                    double* __restrict__ mask_out) {
  for (size_t gp = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gp < ngrid;
       gp += (size_t)gridDim.x * blockDim.x) {
    const int iz = (int)(gp % (size_t)g.n[2]);
    const size_t r = gp / (size_t)g.n[2];
    const int iy = (int)(r % (size_t)g.n[1]);
    const int ix = (int)(r / (size_t)g.n[1]);
    const double p[3] = {g.x0[0] + (double)ix * g.h[0], g.x0[1] + (double)iy * g.h[1],
                         g.x0[2] + (double)iz * g.h[2]};
    bool inside = true;
    int kc[3];
    double fc[3];
    for (int d = 0; d < 3; ++d) {
      const double c0 = tg.xmin[d], c1 = tg.xmin[d] + (double)(tg.n[d] - 1) * tg.h[d];
      inside = inside && p[d] >= c0 && p[d] <= c1;
      kc[d] = taper_cell(p[d], tg.xmin[d], tg.h[d], tg.n[d]);
      const double a = tg.xmin[d] + (double)kc[d] * tg.h[d];
      const double b = tg.xmin[d] + (double)(kc[d] + 1) * tg.h[d];
      fc[d] = (p[d] - a) / (b - a);
    }
    double m = 0.0;
    if (inside) {
      for (int a = 0; a < 2; ++a) {
        const double wa = a ? fc[0] : 1.0 - fc[0];
        for (int b = 0; b < 2; ++b) {
          const double wb = b ? fc[1] : 1.0 - fc[1];
          for (int c = 0; c < 2; ++c) {
            const double wc = c ? fc[2] : 1.0 - fc[2];
            const double t = tg.w[0][kc[0] + a] * tg.w[1][kc[1] + b] * tg.w[2][kc[2] + c];
            m = m + wa * wb * wc * t;
          }
        }
      }
    }
    for (int f = 0; f < nfield; ++f) {
      float* q = grid + (size_t)f * ngrid + gp;
      *q = (float)((double)*q * m);
    }
    if (mask_out) mask_out[gp] = m;
  }
}

// zprecond_grid's depth profile: 1e-8 above the surface, z + 1e-8 below,
// 1/|z| (type 2) or 1/sqrt|z| (type 3), times nevents, normalised by the
// largest magnitude, inverted and normalised again (one block)
__global__ void k_grid_zprofile(const double* __restrict__ zlev, int nz, int ptype, int nevents,
                                double* __restrict__ prof) {
  __shared__ double s_m[32];
  const int t = threadIdx.x;
  auto block_max = [&](double v) -> double {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((t & 31) == 0) s_m[t >> 5] = v;
    __syncthreads();
    double r = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmax(r, s_m[w]);
    __syncthreads();
    return r;
  };
  double m = 0.0;
  for (int k = t; k < nz; k += blockDim.x) {
    const double z = zlev[k];
    const double zl = z > 0.0 ? 1e-8 : z + 1e-8;
    const double v = (ptype == 2 ? 1.0 / sqrt(zl * zl) : 1.0 / sqrt(sqrt(zl * zl))) *
                     (double)nevents;
    prof[k] = v;
    m = fmax(m, fabs(v));
  }
  const double m1 = block_max(m);
  m = 0.0;
  for (int k = t; k < nz; k += blockDim.x) {
    const double v = 1.0 / (prof[k] / m1);
    prof[k] = v;
    m = fmax(m, fabs(v));
  }
  const double m2 = block_max(m);
  for (int k = t; k < nz; k += blockDim.x) prof[k] = prof[k] / m2;
}

__global__ void k_grid_broadcast(const double* __restrict__ prof, int nz, size_t n,
                                 float* __restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = (float)prof[i % (size_t)nz];
}

// Device buffer released at scope exit
template <class T>
struct Buf {
  T* p = nullptr;
  size_t n = 0;
  int alloc(size_t count) {
    n = count;
    return cudaMalloc((void**)&p, std::max<size_t>(count, 1) * sizeof(T)) == cudaSuccess ? 0 : -1;
  }
  ~Buf() {
    if (p) cudaFree(p);
  }
};

int check_grid(const sem_grid_desc* g, GridGeom* out, size_t* ngrid) {
  if (!g) return report_error(SEM_ERR_ARG, "null grid");
  size_t n = 1;
  for (int d = 0; d < 3; ++d) {
    if (g->n[d] < 1) return report_error(SEM_ERR_ARG, "grid sizes must be >= 1");
    if (!(g->h[d] > 0.0) || !std::isfinite(g->h[d]) || !std::isfinite(g->x0[d]))
      return report_error(SEM_ERR_ARG, "grid spacing must be > 0 and the origin finite");
    out->x0[d] = g->x0[d];
    out->h[d] = g->h[d];
    out->n[d] = g->n[d];
    n *= (size_t)g->n[d];
  }
  if (n > ((size_t)1 << 34)) return report_error(SEM_ERR_ARG, "grid too large");
  *ngrid = n;
  return SEM_OK;
}

#define GK(call)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return report_error(SEM_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));       \
  } while (0)

int upload_coords(const SmoothMeshView& mv, Buf<float>& xyz) {
  const size_t ng = (size_t)mv.nglob;
  if (xyz.alloc(3 * ng)) return report_error(SEM_ERR_NOMEM, "grid: coordinates");
  GK(cudaMemcpy(xyz.p, mv.x, ng * 4, cudaMemcpyHostToDevice));
  GK(cudaMemcpy(xyz.p + ng, mv.y, ng * 4, cudaMemcpyHostToDevice));
  GK(cudaMemcpy(xyz.p + 2 * ng, mv.z, ng * 4, cudaMemcpyHostToDevice));
  return SEM_OK;
}

unsigned blocks_for(size_t n) { return (unsigned)std::min<size_t>((n + 127) / 128, 148 * 64); }

// coswin: the rising (opt 1) or falling half of a 2n+1-point Hann window,
// without its centre
void coswin(int n, int opt, double* out) {
  const int nn = 2 * n + 1;
  for (int i = 0; i < n; ++i) {
    const int q = opt == 1 ? i : n + 1 + i;
    out[i] = 0.5 - 0.5 * std::cos(2.0 * 3.1415926535 * (double)q / (double)(nn - 1));
  }
}

// create_taper's window along one axis of n points of spacing h: zero for
// t1 from each end (both) or the low end only, a half cosine over the next
// t2, one inside
int taper_window(int n, double h, double t1, double t2, bool both, std::vector<double>& w) {
  w.assign((size_t)n, 0.0);
  if (t1 / h > (double)n || t2 / h > (double)n)
    return report_error(SEM_ERR_ARG, "taper widths (%g + %g m) exceed the mesh", t1, t2);
  const long long nh1 = (long long)std::floor(t1 / h), nh2 = (long long)std::floor(t2 / h);
  const long long a = nh1, b = nh1 + nh2;
  const long long c = both ? (long long)n - nh1 - nh2 : (long long)n;
  if (nh1 < 0 || nh2 < 0 || b > c)
    return report_error(SEM_ERR_ARG, "taper widths (%g + %g m) exceed the mesh", t1, t2);
  std::vector<double> up((size_t)nh2), down((size_t)nh2);
  coswin((int)nh2, 1, up.data());
  coswin((int)nh2, 0, down.data());
  for (long long i = 0; i < nh2; ++i) w[(size_t)(a + i)] = up[(size_t)i];
  if (both)
    for (long long i = 0; i < nh2; ++i) w[(size_t)(c + i)] = down[(size_t)i];
  for (long long i = b; i < c; ++i) w[(size_t)i] = 1.0;
  return SEM_OK;
}

}  // namespace
}  // namespace sem

using namespace sem;

extern "C" int sem_grid_project(sem_mesh* mesh, const sem_grid_desc* grid, int nfield,
                                const float* fields, float* out) {
  NvtxPhase ph("sem_grid_project");
  if (!mesh || !fields || !out) return report_error(SEM_ERR_ARG, "null argument");
  if (nfield < 1 || nfield > 64) return report_error(SEM_ERR_ARG, "nfield must be in [1, 64]");
  GridGeom g{};
  size_t ngrid = 0;
  int rc = check_grid(grid, &g, &ngrid);
  if (rc) return rc;
  if (grid->ngnod != 8 && grid->ngnod != 27)
    return report_error(SEM_ERR_ARG, "ngnod must be 8 or 27");
  SmoothMeshView mv{};
  rc = mesh_smooth_view(mesh, &mv);
  if (rc) return rc;
  const size_t nfe = (size_t)mv.nspec * NGLL3;
  Buf<float> xyz, f, o;
  Buf<int> owner;
  Buf<double> box;
  rc = upload_coords(mv, xyz);
  if (rc) return rc;
  if (f.alloc(nfe * nfield) || o.alloc(ngrid * nfield) || owner.alloc(ngrid) ||
      box.alloc((size_t)mv.nspec * 6))
    return report_error(SEM_ERR_NOMEM, "grid: device buffers");
  GK(cudaMemcpy(f.p, fields, nfe * nfield * 4, cudaMemcpyHostToDevice));
  GK(cudaMemset(owner.p, 0x7f, ngrid * sizeof(int)));  // 0x7f7f7f7f: no owner
  const size_t ng = (size_t)mv.nglob;
  k_grid_claim<<<mv.nspec, 128>>>(mv.ibool, xyz.p, xyz.p + ng, xyz.p + 2 * ng, g, box.p,
                                  owner.p);
  GK(cudaGetLastError());
  k_grid_eval<<<blocks_for(ngrid), 128>>>(f.p, nfield, nfe, owner.p, box.p, mv.irreg, mv.ibool,
                                          xyz.p, xyz.p + ng, xyz.p + 2 * ng, mv.nspec, g,
                                          grid->ngnod, o.p, ngrid);
  GK(cudaGetLastError());
  GK(cudaMemcpy(out, o.p, ngrid * nfield * 4, cudaMemcpyDeviceToHost));
  return SEM_OK;
}

extern "C" int sem_grid_taper(sem_mesh* mesh, const sem_grid_desc* grid,
                              const sem_grid_taper_cfg* taper, int nfield, float* grid_fields,
                              double* mask) {
  NvtxPhase ph("sem_grid_taper");
  if (!mesh || !taper || (!grid_fields && nfield > 0) || (!mask && nfield == 0))
    return report_error(SEM_ERR_ARG, "null argument");
  if (nfield < 0 || nfield > 64) return report_error(SEM_ERR_ARG, "nfield must be in [0, 64]");
  GridGeom g{};
  size_t ngrid = 0;
  int rc = check_grid(grid, &g, &ngrid);
  if (rc) return rc;
  const double tw[4] = {taper->h_suppress, taper->h_buffer, taper->v_suppress, taper->v_buffer};
  for (double v : tw)
    if (!(v >= 0.0) || !std::isfinite(v))
      return report_error(SEM_ERR_ARG, "taper widths must be finite and >= 0");
  SmoothMeshView mv{};
  rc = mesh_smooth_view(mesh, &mv);
  if (rc) return rc;
  Buf<float> xyz;
  rc = upload_coords(mv, xyz);
  if (rc) return rc;
  // mask spacing: the mean of the smallest and largest GLL point distance
  const size_t ng = (size_t)mv.nglob;
  Buf<double> dmin, dmax;
  if (dmin.alloc((size_t)mv.nspec) || dmax.alloc((size_t)mv.nspec))
    return report_error(SEM_ERR_NOMEM, "grid: distances");
  k_elem_dist<<<(mv.nspec + 127) / 128, 128>>>(mv.ibool, xyz.p, xyz.p + ng, xyz.p + 2 * ng,
                                               mv.nspec, dmin.p, dmax.p);
  GK(cudaGetLastError());
  std::vector<double> hmin((size_t)mv.nspec), hmax((size_t)mv.nspec);
  GK(cudaMemcpy(hmin.data(), dmin.p, hmin.size() * 8, cudaMemcpyDeviceToHost));
  GK(cudaMemcpy(hmax.data(), dmax.p, hmax.size() * 8, cudaMemcpyDeviceToHost));
  double lo = INFINITY, hi = 0.0;
  for (size_t e = 0; e < hmin.size(); ++e) {
    lo = std::min(lo, hmin[e]);
    hi = std::max(hi, hmax[e]);
  }
  const double dh = 0.5 * (hi + lo);
  // the mask's grid over the mesh's extent
  const float* cs[3] = {mv.x, mv.y, mv.z};
  TaperGeom tg{};
  std::vector<double> w[3];
  Buf<double> wd[3];
  for (int d = 0; d < 3; ++d) {
    const float* c = cs[d];
    float cmin = c[0], cmax = c[0];
    for (size_t i = 1; i < ng; ++i) {
      cmin = std::min(cmin, c[i]);
      cmax = std::max(cmax, c[i]);
    }
    const int n = (int)std::floor(((double)cmax - (double)cmin) / dh + 1.0);
    if (n < 2) return report_error(SEM_ERR_ARG, "mesh extent below two taper cells");
    tg.xmin[d] = (double)cmin;
    tg.h[d] = dh;
    tg.n[d] = n;
    rc = d < 2 ? taper_window(n, dh, tw[0], tw[1], true, w[d])
               : taper_window(n, dh, tw[2], tw[3], false, w[d]);
    if (rc) return rc;
    if (wd[d].alloc((size_t)n)) return report_error(SEM_ERR_NOMEM, "grid: taper windows");
    GK(cudaMemcpy(wd[d].p, w[d].data(), (size_t)n * 8, cudaMemcpyHostToDevice));
    tg.w[d] = wd[d].p;
  }
  Buf<float> gd;
  Buf<double> md;
  if (gd.alloc(ngrid * (size_t)nfield) || (mask && md.alloc(ngrid)))
    return report_error(SEM_ERR_NOMEM, "grid: device buffers");
  if (nfield > 0)
    GK(cudaMemcpy(gd.p, grid_fields, ngrid * nfield * 4, cudaMemcpyHostToDevice));
  k_grid_taper<<<blocks_for(ngrid), 128>>>(gd.p, nfield, ngrid, g, tg, mask ? md.p : nullptr);
  GK(cudaGetLastError());
  if (nfield > 0)
    GK(cudaMemcpy(grid_fields, gd.p, ngrid * nfield * 4, cudaMemcpyDeviceToHost));
  if (mask) GK(cudaMemcpy(mask, md.p, ngrid * 8, cudaMemcpyDeviceToHost));
  return SEM_OK;
}

extern "C" int sem_grid_zprecond(const sem_grid_desc* grid, const double* zlev, int precond_type,
                                 int nevents, float* out) {
  if (!out) return report_error(SEM_ERR_ARG, "null argument");
  if (precond_type != 2 && precond_type != 3)
    return report_error(SEM_ERR_ARG, "the depth forms are PRECOND_TYPE 2 and 3");
  if (nevents < 1) return report_error(SEM_ERR_ARG, "nevents must be >= 1");
  GridGeom g{};
  size_t ngrid = 0;
  int rc = check_grid(grid, &g, &ngrid);
  if (rc) return rc;
  const int nz = g.n[2];
  std::vector<double> z((size_t)nz);
  for (int k = 0; k < nz; ++k) z[(size_t)k] = zlev ? zlev[k] : g.x0[2] + (double)k * g.h[2];
  Buf<double> zd, prof;
  Buf<float> od;
  if (zd.alloc((size_t)nz) || prof.alloc((size_t)nz) || od.alloc(ngrid))
    return report_error(SEM_ERR_NOMEM, "grid: device buffers");
  GK(cudaMemcpy(zd.p, z.data(), (size_t)nz * 8, cudaMemcpyHostToDevice));
  k_grid_zprofile<<<1, 256>>>(zd.p, nz, precond_type, nevents, prof.p);
  GK(cudaGetLastError());
  k_grid_broadcast<<<blocks_for(ngrid), 128>>>(prof.p, nz, ngrid, od.p);
  GK(cudaGetLastError());
  GK(cudaMemcpy(out, od.p, ngrid * 4, cudaMemcpyDeviceToHost));
  return SEM_OK;
}
