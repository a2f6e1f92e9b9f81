// Kernel preconditioners of the post-processing, on the device.
//
//  - Approximate-Hessian preconditioner, PostFlow%apply_precond with
//    PRECOND_TYPE 0 or 1 (src/postproc/post_processing.f90:164-197): the
//    event sum of hess_kernel (PRECOND_TYPE 1: of |hess|; 0: |sum|),
//    inverted by invert_hess (post_processing.f90:333-372):
//        h = h / max|h|         (h = 1 when max|h| < 1e-18)
//        h = 1 / h              where |h| > THRESHOLD_HESS, else 1 / THRESHOLD_HESS
//        h = h / max|h|
//    with THRESHOLD_HESS = 1e-3 (src/shared/config.f90:42).
//  - Depth preconditioner zprecond_gll, PRECOND_TYPE 2 or 3
//    (src/postproc/zprecond.f90:11-71): a 1-D profile on the model grid's
//    depth levels, 1/|z| (2) or 1/sqrt|z| (3) with z = 1e-8 above the
//    surface and z + 1e-8 below, linearly interpolated to every GLL point
//    (interp1, src/shared/utils.f90:889-910), times the event count, then
//        h = h / max|h|,  h = 1 / h,  h = h / max|h|.
//
// Values are computed in FP64 and returned as FP32 (the reference's
// CUSTOM_REAL).  Three grid-stride passes: the first maximum, the inverted
// values' maximum, the output.  The maxima of non-negative doubles are
// combined with an integer atomicMax on their bit patterns, so the result
// does not depend on the order of the blocks.

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "sem_b200.h"
#include "sem_internal.cuh"

namespace sem {
namespace {

constexpr double kThresholdHess = 1e-3;  // THRESHOLD_HESS

// Where the values to invert come from: a summed Hessian, or the depth
// profile interpolated at the GLL points.
struct PrecondSrc {
  const double* hess;   // [n] or null (depth form)
  int take_abs;         // PRECOND_TYPE 0: |sum hess|
  const int* ibool;     // depth form: [n] element point -> global point
  const float* zg;      // [nglob] z of the global points
  const double* zlev;   // [nz] ascending depth levels
  const double* vlev;   // [nz] profile at the levels
  int nz;
  double scale;         // the event count
  double threshold;     // inversion threshold (0: plain 1/h)
  int zero_guard;       // h = 1 when the first maximum is below 1e-18
};

__device__ double src_value(const PrecondSrc& s, size_t i) {
  if (s.hess) {
    const double h = s.hess[i];
    return s.take_abs ? fabs(h) : h;
  }
  const double z = (double)s.zg[s.ibool[i]];
  const int top = s.nz - 1;
  if (z >= s.zlev[top]) return s.vlev[top] * s.scale;
  if (z <= s.zlev[0]) return s.vlev[0] * s.scale;
  // zlev[lo] <= z < zlev[hi], hi = lo + 1
  int lo = 0, hi = top;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (s.zlev[mid] <= z)
      lo = mid;
    else
      hi = mid;
  }
  const double v = (s.vlev[lo] * (s.zlev[hi] - z) + s.vlev[hi] * (z - s.zlev[lo])) /
                   fabs(s.zlev[hi] - s.zlev[lo]);
  return v * s.scale;
}

// Inverted value of point i given the first maximum m1.
__device__ double inv_value(const PrecondSrc& s, size_t i, double m1) {
  double h = src_value(s, i);
  h = (s.zero_guard && m1 < 1e-18) ? 1.0 : h / m1;
  if (s.threshold > 0.0) return fabs(h) > s.threshold ? 1.0 / h : 1.0 / s.threshold;
  return 1.0 / h;
}

__device__ void block_max_to(double v, unsigned long long* dst) {
  __shared__ double red[256];
  red[threadIdx.x] = v;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicMax(dst, (unsigned long long)__double_as_longlong(red[0]));
}

// pass 0: m[0] = max|h|; pass 1: m[1] = max|inv|; pass 2: out = inv / m[1]
template <int PASS>
__global__ void __launch_bounds__(256) k_precond(PrecondSrc s, size_t n, unsigned long long* m,
                                                 float* __restrict__ out) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  double mx = 0.0;
  const double m1 = PASS > 0 ? __longlong_as_double((long long)m[0]) : 0.0;
  const double m2 = PASS > 1 ? __longlong_as_double((long long)m[1]) : 1.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    if constexpr (PASS == 0) {
      mx = fmax(mx, fabs(src_value(s, i)));
    } else if constexpr (PASS == 1) {
      mx = fmax(mx, fabs(inv_value(s, i, m1)));
    } else {
      out[i] = (float)(inv_value(s, i, m1) / m2);
    }
  }
  if constexpr (PASS < 2) block_max_to(mx, m + PASS);
}

int run_precond(const PrecondSrc& s, size_t n, unsigned long long* m, float* out,
                cudaStream_t st) {
  const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 8);
  k_precond<0><<<blocks, 256, 0, st>>>(s, n, m, out);
  k_precond<1><<<blocks, 256, 0, st>>>(s, n, m, out);
  k_precond<2><<<blocks, 256, 0, st>>>(s, n, m, out);
  return 3;
}

// Device buffers of one call, freed on every return path.
struct Bufs {
  std::vector<void*> p;
  ~Bufs() {
    for (void* q : p) cudaFree(q);
  }
  template <typename T>
  cudaError_t get(T** out, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
    if (e == cudaSuccess) p.push_back(q);
    *out = (T*)q;
    return e;
  }
};

#define PCK(call)                                                                   \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      cudaGetLastError();                                                           \
      if (st) cudaStreamDestroy(st);                                                \
      return report_error(SEM_ERR_CUDA, "preconditioner: %s: %s", #call,            \
                          cudaGetErrorString(e_));                                  \
    }                                                                               \
  } while (0)

// Runs the three passes on fresh device copies and copies the result back.
int precond_call(PrecondSrc s, size_t n, const double* h_hess, const float* h_z, size_t nglob,
                 const double* h_zlev, const double* h_vlev, float* h_out) {
  cudaStream_t st = nullptr;
  Bufs b;
  unsigned long long* m = nullptr;
  float* out = nullptr;
  PCK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  PCK(b.get(&m, 2));
  PCK(b.get(&out, n));
  PCK(cudaMemsetAsync(m, 0, 2 * sizeof(unsigned long long), st));
  if (h_hess) {
    double* d = nullptr;
    PCK(b.get(&d, n));
    PCK(cudaMemcpyAsync(d, h_hess, n * 8, cudaMemcpyHostToDevice, st));
    s.hess = d;
  } else {
    float* z = nullptr;
    double *zl = nullptr, *vl = nullptr;
    PCK(b.get(&z, nglob));
    PCK(b.get(&zl, s.nz));
    PCK(b.get(&vl, s.nz));
    PCK(cudaMemcpyAsync(z, h_z, nglob * 4, cudaMemcpyHostToDevice, st));
    PCK(cudaMemcpyAsync(zl, h_zlev, s.nz * 8, cudaMemcpyHostToDevice, st));
    PCK(cudaMemcpyAsync(vl, h_vlev, s.nz * 8, cudaMemcpyHostToDevice, st));
    s.zg = z;
    s.zlev = zl;
    s.vlev = vl;
  }
  run_precond(s, n, m, out, st);
  PCK(cudaGetLastError());
  PCK(cudaMemcpyAsync(h_out, out, n * 4, cudaMemcpyDeviceToHost, st));
  PCK(cudaStreamSynchronize(st));
  cudaStreamDestroy(st);
  return SEM_OK;
}

}  // namespace
}  // namespace sem

using namespace sem;

extern "C" int sem_hessian_precond(const double* hess_sum, long long n, int precond_type,
                                   float* precond) {
  if (!hess_sum || !precond) return report_error(SEM_ERR_ARG, "null argument");
  if (n < 1) return report_error(SEM_ERR_ARG, "n must be >= 1");
  if (precond_type != 0 && precond_type != 1)
    return report_error(SEM_ERR_ARG, "precond_type %d: the Hessian forms are 0 and 1",
                        precond_type);
  PrecondSrc s{};
  s.take_abs = precond_type == 0;
  s.threshold = kThresholdHess;
  s.zero_guard = 1;
  return precond_call(s, (size_t)n, hess_sum, nullptr, 0, nullptr, nullptr, precond);
}

extern "C" int sem_depth_precond(sem_mesh* mesh, const double* zlev, int nz, int precond_type,
                                 int nevents, float* precond) {
  if (!mesh || !zlev || !precond) return report_error(SEM_ERR_ARG, "null argument");
  if (nz < 2) return report_error(SEM_ERR_ARG, "nz must be >= 2");
  if (precond_type != 2 && precond_type != 3)
    return report_error(SEM_ERR_ARG, "precond_type %d: the depth forms are 2 and 3",
                        precond_type);
  if (nevents < 1) return report_error(SEM_ERR_ARG, "nevents must be >= 1");
  for (int i = 1; i < nz; ++i)
    if (!(zlev[i] > zlev[i - 1]))
      return report_error(SEM_ERR_ARG, "depth levels must be strictly ascending (level %d)", i);
  SmoothMeshView mv{};
  int rc = mesh_smooth_view(mesh, &mv);
  if (rc) return rc;
  // get_1d_precond (zprecond.f90:11-32)
  std::vector<double> vlev(nz);
  for (int i = 0; i < nz; ++i) {
    const double zl = zlev[i] > 0.0 ? 1e-8 : zlev[i] + 1e-8;
    vlev[i] = precond_type == 2 ? 1.0 / std::sqrt(zl * zl) : 1.0 / std::sqrt(std::sqrt(zl * zl));
  }
  PrecondSrc s{};
  s.ibool = mv.ibool;
  s.nz = nz;
  s.scale = (double)nevents;
  s.threshold = 0.0;
  s.zero_guard = 0;
  return precond_call(s, (size_t)mv.nspec * NGLL3, nullptr, mv.z, (size_t)mv.nglob, zlev,
                      vlev.data(), precond);
}
