// L2 waveform misfit for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: code running inside another
// framework's memory pool or under a fixed device-memory budget, and
// Fortran hosts that only hand over buffers they already own.  For them
// sem_measure_l2_noalloc computes the same FP64 L2 misfit and adjoint
// sources as sem_measure_l2, but on caller-owned device buffers and with
// its working memory in one file-scope device array of fixed size, so the
// call itself allocates nothing.
//
// The array lives on every GPU that loads this library until the process
// exits.  Every call shares it and it keeps the last call's contents; each
// call overwrites the parts it reads (weights and per-series partial
// misfits) before using them, so nothing has to start at zero.  Calls that
// overlap on the GPU (different streams, or different host threads, at the
// same time) race on the array and must not be issued.
//
// Set-up: the first call in a CUDA context (the first on a device, and the
// first after the context was torn down and recreated, e.g. by
// cudaDeviceReset) looks up the array's device address.  CUDA loads device
// code lazily, so that first call is also when the driver loads this file's
// device code and places the array (about 608 KiB) on the GPU; on a device
// with no memory left it fails with SEM_ERR_CUDA.  A caller under a fixed
// budget makes one small call at start-up, before the budget applies.  Make
// the first call before any stream capture.  The address is cached per
// device together with the context's id, so a recreated context is set up
// again instead of reusing an address from the old one.

#include <cuda.h>  // CUcontext / CUresult types of the two driver calls below

#include <cmath>
#include <cstdio>
#include <mutex>

#include "sem_b200.h"
#include "sem_internal.cuh"

namespace {

constexpr int kMaxSteps = SEM_L2_NOALLOC_MAX_STEPS;
constexpr int kMaxSeries = 3 * SEM_L2_NOALLOC_MAX_RECEIVERS;
// taper weights, Simpson weights, per-series partial misfits
constexpr size_t kScratchDoubles = 2 * (size_t)kMaxSteps + (size_t)kMaxSeries;

static __device__ __align__(256) double g_l2_scratch[kScratchDoubles];

constexpr int kMaxDevices = 128;
std::mutex g_mu;
struct ScratchSlot {
  unsigned long long ctx_id;  // context the address belongs to
  double* addr;
};
ScratchSlot g_slot[kMaxDevices] = {};

// Unique id of the calling thread's current CUDA context (cuCtxGetId),
// through the runtime's driver entry points, so the library needs no link
// to libcuda.
int current_context_id(unsigned long long* id) {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  if (!get_current || !get_id) {
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2) {
      cudaGetLastError();
      return sem::report_error(SEM_ERR_CUDA, "driver context queries are not available");
    }
    get_current = (GetCurrent)f1;
    get_id = (GetId)f2;
  }
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, id) != CUDA_SUCCESS)
    return sem::report_error(SEM_ERR_CUDA, "no current CUDA context");
  return SEM_OK;
}

// Device address of g_l2_scratch in the current context (the host-side name
// of the array is only a stand-in), looked up once per device and context.
int scratch_for_current_device(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return sem::report_error(SEM_ERR_NODEVICE, "no CUDA device: %s", cudaGetErrorString(e));
  }
  if (dev < 0 || dev >= kMaxDevices)
    return sem::report_error(SEM_ERR_UNSUPPORTED, "device ordinal %d above %d", dev, kMaxDevices);
  // makes the device's primary context current if no context is yet
  e = cudaSetDevice(dev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return sem::report_error(SEM_ERR_CUDA, "cudaSetDevice(%d) failed: %s", dev,
                             cudaGetErrorString(e));
  }
  unsigned long long ctx = 0;
  int rc = current_context_id(&ctx);
  if (rc) return rc;
  std::lock_guard<std::mutex> lock(g_mu);
  ScratchSlot& s = g_slot[dev];
  if (!s.addr || s.ctx_id != ctx) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_l2_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return sem::report_error(SEM_ERR_CUDA, "cudaGetSymbolAddress of the L2 scratch failed: %s",
                               cudaGetErrorString(e));
    }
    s.addr = (double*)p;
    s.ctx_id = ctx;
  }
  *out = s.addr;
  return SEM_OK;
}

// Taper weights of src/shared/signal.f90:419-491 and the Simpson weights of
// src/shared/utils.f90:1635-1663 (including the weight 1 + 2 its even-count
// branch gives sample n-1), accumulated in the same order as the host code
// of sem_measure_l2.
__global__ void k_l2_weights(double* taper, double* simpw, int n, int frac, double dx,
                             int type) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double w = 1.0;
  if (frac > 0) {
    const double den = 2.0 * frac - 1.0;
    double x = -1.0;
    if (i < frac)
      x = (double)i;
    else if (i >= n - frac)
      x = (double)(frac + i - (n - frac));
    if (x >= 0.0) {
      double tw;
      switch (type) {
        case 1: tw = 0.5 - 0.5 * cos(2.0 * M_PI * x / den); break;
        case 2: tw = 0.54 - 0.46 * cos(2.0 * M_PI * x / den); break;
        case 3: tw = cos(M_PI * x / den - M_PI / 2.0); break;
        default: tw = 1.0 - pow(cos(M_PI * x / den), 10.0); break;
      }
      w *= tw;
    }
  }
  taper[i] = w;
  double s = 0.0;
  if (n >= 2) {
    if (n % 2 == 0) {
      if (i == 0) s += dx / 3.0;
      if (i == n - 2) s += dx / 3.0;
      if ((i & 1) && i >= 1 && i <= n - 3) s += 4.0 * dx / 3.0;
      if (!(i & 1) && i >= 2 && i <= n - 2) s += 2.0 * dx / 3.0;
      if (i == n - 2) s += 0.5 * dx;
      if (i == n - 1) s += 0.5 * dx;
    } else {
      if (i == 0) s += dx / 3.0;
      if (i == n - 1) s += dx / 3.0;
      if ((i & 1) && i >= 1 && i <= n - 2) s += 4.0 * dx / 3.0;
      if (!(i & 1) && i >= 2 && i <= n - 3) s += 2.0 * dx / 3.0;
    }
  }
  simpw[i] = s;
}

// Sum of the per-series misfits in series order (the order the host sum of
// sem_measure_l2 uses), written to the caller's output.
__global__ void k_l2_total(const double* part, int nseries, double* out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double t = 0.0;
  for (int k = 0; k < nseries; ++k) t += part[k];
  *out = t;
}

}  // namespace

extern "C" int sem_measure_l2_noalloc(const float* seis_dev, const double* obs_dev, int nrec,
                                      int nstep, double dt, double taper_pct, int taper_type,
                                      float* adj_dev, double* misfit_dev, void* stream) {
  if (!seis_dev || !obs_dev || !adj_dev || !misfit_dev)
    return sem::report_error(SEM_ERR_ARG, "null device buffer");
  if (nrec < 1 || nstep < 1) return sem::report_error(SEM_ERR_ARG, "nrec and nstep must be >= 1");
  if (nrec > SEM_L2_NOALLOC_MAX_RECEIVERS)
    return sem::report_error(SEM_ERR_ARG,
                             "nrec %d above the %d receivers the static scratch holds", nrec,
                             SEM_L2_NOALLOC_MAX_RECEIVERS);
  if (nstep > SEM_L2_NOALLOC_MAX_STEPS)
    return sem::report_error(SEM_ERR_ARG, "nstep %d above the %d samples the static scratch holds",
                             nstep, SEM_L2_NOALLOC_MAX_STEPS);
  if (!(dt > 0.0)) return sem::report_error(SEM_ERR_ARG, "dt must be > 0");
  if (!(taper_pct >= 0.0 && taper_pct <= 1.0))
    return sem::report_error(SEM_ERR_ARG, "taper_percentage must be in [0, 1]");
  if (taper_type < 1 || taper_type > 4)
    return sem::report_error(SEM_ERR_ARG, "taper type must be 1..4");
  double* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  double* taper = scratch;
  double* simpw = scratch + kMaxSteps;
  double* part = scratch + 2 * (size_t)kMaxSteps;
  const int frac = (taper_pct == 0.0 || taper_pct == 1.0) ? (int)(nstep * taper_pct / 2.0)
                                                          : (int)(nstep * taper_pct / 2.0 + 0.5);
  cudaStream_t st = (cudaStream_t)stream;
  k_l2_weights<<<(nstep + 255) / 256, 256, 0, st>>>(taper, simpw, nstep, frac, dt, taper_type);
  sem::launch_measure_l2(seis_dev, obs_dev, taper, simpw, nrec, nstep, adj_dev, part, st);
  k_l2_total<<<1, 1, 0, st>>>(part, 3 * nrec, misfit_dev);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return sem::report_error(SEM_ERR_CUDA, "L2 measurement launch failed: %s",
                             cudaGetErrorString(e));
  return SEM_OK;
}
