// Internal types shared by the CUDA kernels and the host engine.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstddef>
#include <cstdint>

#include "sem_b200.h"

namespace sem {

constexpr int NGLL = 5;
constexpr int NGLL2 = 25;
constexpr int NGLL3 = 125;

// Phase of an event lane.  A lane is one event's wavefield column in the
// lane-interleaved layout [point][component][lane].
enum Phase : int { PH_IDLE = 0, PH_FWD = 1, PH_ADJ = 3 };

// Per-lane state read by every kernel of a step.  `it0` is the step index
// at graph step s = 0; the kernel's step is it0 + s.  In the adjoint phase
// the step index is the adjoint iteration j (adjoint source sample
// nstep-1-j, backward state nstep-1-j).
struct LaneDesc {
  int phase;
  int it0;
  int nstep;
  int save;          // forward phase: write the boundary store
  int src_ispec;
  int nrec;
  // boundary store ring (host spill): 0 when the whole store is resident;
  // else records of ring_c steps per chunk in ring_d device slots, record
  // `it` at row ((it / ring_c) % ring_d) * nev * ring_c + it % ring_c
  int ring_c, ring_d;
  const float* stf;      // [nstep]      source time function samples
  const float* srcarr;   // [125][3]     moment tensor : grad(phi_abc)
  const int* rec_ispec;  // [nrec]
  const float* rec_w;    // [nrec][125]  Lagrange interpolation weights
  float* seis;           // [nrec][3][nstep]
  const float* adj;      // [nrec][3][nstep] adjoint sources, forward time
  void* store;           // [nstep][nf][25][3] float or half
  float* scale;          // [nstep][nf] per-face FP16 scale
  // incident wavefield on the absorbing faces (forward phase), or null:
  // [inj_nt][nf*25][3] velocity and traction, sample k at time
  // (k + inj_k0) * inj_np * DT
  const float* inj_v;
  const float* inj_t;
  int inj_nt, inj_np, inj_k0, inj_pad;
};

struct MeshView {
  int nspec, nglob, nf;
  float xix, jac;
  const int* ibool;      // [nspec*125]
  const int* order;      // [nspec] element traversal order (Morton curve)
  const float* kappa;    // [nspec*125]
  const float* mu;       // [nspec*125]
  const int* f_iglob;    // [nf*25]
  const float* f_rvp;    // [nf*25] rho*vp at the face point
  const float* f_rvs;    // [nf*25] rho*vs
  const float* f_jw;     // [nf*25] jacobian2D * weights
  const float* f_n;      // [nf*25*3]
  // element colouring for assembly without atomics: colour c's elements
  // are corder[cstart[c] .. cstart[c+1]), no two of them share a point
  static constexpr int kMaxColours = 32;
  int ncolour;           // 0: not coloured (more than kMaxColours needed)
  const int* corder;     // [nspec]
  int cstart[kMaxColours + 1];
  // irregular elements: irreg[e] = -1 or the row of geo [nirr][125][10]
  // (xix, xiy, xiz, etax, etay, etaz, gammax, gammay, gammaz, jacobian);
  // both null when every element is regular
  const int* irreg;
  const float* geo;
};

struct Fields {
  float* u;
  float* v;
  float* a;
};

struct KernAcc {
  float* rho_glob;   // [nglob][nev]
  float* mu;         // [nspec*125][nev]
  float* kappa;      // [nspec*125][nev]
  float* hess_glob;  // [nglob][nev] approximate Hessian, or null (not accumulated)
};

// Per-event arrays use a lane-group layout: event lanes are grouped by
// LW = 2^lwlog (1 for a single event, 8 otherwise) and an array of
// per-point records is stored [group][point][record][LW], so one group's
// data is contiguous and a warp of a group reads whole 32-byte sectors.
struct LaneMap {
  int lwlog;
  // field value (point ig, component c) of lane lg; nglob points
  __host__ __device__ __forceinline__ size_t f(size_t ig, int c, int lg, size_t nglob) const {
    return ((((size_t)(lg >> lwlog)) * nglob + ig) * 3 + c) * ((size_t)1 << lwlog) +
           (lg & ((1 << lwlog) - 1));
  }
  // one value per point (or element point) i of n
  __host__ __device__ __forceinline__ size_t p(size_t i, int lg, size_t n) const {
    return (((size_t)(lg >> lwlog)) * n + i) * ((size_t)1 << lwlog) + (lg & ((1 << lwlog) - 1));
  }
};

struct StepArgs {
  MeshView m;
  Fields f1;             // forward field, or adjoint field in PH_ADJ
  Fields f2;             // backward (reconstructed) field, PH_ADJ only
  KernAcc k;
  const LaneDesc* lanes; // [nev]
  const float* minv;     // [nglob*3] 1/(M + dt/2 C)
  int nev;
  int s;                 // graph step
  float dt;
  int store_fp16;
  int nrec_max;
  int variant;           // element kernel: 0 thread-per-point, 1 pencil
  LaneMap lm;            // lane-group layout of the per-event arrays
  const int* gmap;       // serving: active 8-lane groups (device), or null
  int ngmap;
  int inject;            // some lane has an FK injection (LaneDesc::inj_v)
  int sm_limit;          // SMs the persistent element kernels may fill (0: all)
  int ring_nev;          // lanes of the whole run: the boundary-store ring's slot pitch
  __device__ __forceinline__ size_t fi(size_t ig, int c, int lg) const {
    return lm.f(ig, c, lg, (size_t)m.nglob);
  }
  __device__ __forceinline__ size_t ei(size_t ep, int lg) const {
    return lm.p(ep, lg, (size_t)m.nspec * NGLL3);
  }
  __device__ __forceinline__ size_t gi(size_t ig, int lg) const {
    return lm.p(ig, lg, (size_t)m.nglob);
  }
};

// Launch helpers (defined in sem_kernels.cu).  Each returns the number of
// kernels launched.
int launch_forces(const StepArgs& a, bool adj, cudaStream_t st);
int launch_boundary(const StepArgs& a, bool adj, cudaStream_t st);
int launch_update(const StepArgs& a, bool adj, cudaStream_t st);
int launch_points(const StepArgs& a, cudaStream_t st);
int launch_advance(LaneDesc* lanes, int nev, int k, cudaStream_t st);
int launch_finalize_kernels(const MeshView& m, const float* rho,
                            const KernAcc& k, LaneMap lm, int lane,
                            double* out6, double* sum6, cudaStream_t st);
// hess_kernel of one lane in element layout: out[ep] = 2 hess_glob[ibool[ep]]
// (written when out is not null), sum[ep] += that value or its magnitude
int launch_finalize_hessian(const MeshView& m, const float* hess_glob, LaneMap lm, int lane,
                            double* out, double* sum, int abs_each, cudaStream_t st);
int launch_measure_l2(const float* seis, const double* obs, const double* taper,
                      const double* simpw, int nrec, int nstep, float* adj_out,
                      double* misfit_rc, cudaStream_t st);
int launch_lane_copy(const Fields& src, const Fields& dst, int nglob, LaneMap lm,
                     int lane, cudaStream_t st);
int launch_lane_zero(const Fields& f, int nglob, LaneMap lm, int lane,
                     cudaStream_t st);
// Lane `from`'s values of up to three arrays laid out [group][npts][rec][LW]
// copied to lane `to` (x1, x2 may be null).
int launch_lane_move(float* x0, float* x1, float* x2, size_t npts, int rec, LaneMap lm, int from,
                     int to, cudaStream_t st);
// Periodic stability check: flags[lane] |= 1 for running lanes of u (a
// field of nevp lanes) with a non-finite value; then halt the flagged lanes
// (phase idle, halt_step = it0 + s_off at the first flag).
int launch_check_lanes(const float* u, size_t nglob, int lwlog, int nevp, LaneDesc* lanes,
                       int nev, int* flags, cudaStream_t st);
int launch_halt_lanes(LaneDesc* lanes, int nev, const int* flags, int* halt_step, int s_off,
                      cudaStream_t st);
// *out = part[0] + ... + part[n-1], summed in that order
int launch_sum_series(const double* part, int n, double* out, cudaStream_t st);
int launch_lane_zero_acc(const KernAcc& k, int nglob, size_t ne, LaneMap lm, int lane,
                         cudaStream_t st);

void set_gll_constants(const float* D, const float* DWt, const float* w);

// Waveform measurement (sem_measure.cu): Butterworth band-pass sections
// (b0, b1, b2, a1, a2 with a0 = 1) per band and the launch parameters.
constexpr int kMeasMaxBands = 4;
constexpr int kMeasMaxSections = 10;
struct MeasBand {
  int nsect;
  double b0[kMeasMaxSections], b1[kMeasMaxSections], b2[kMeasMaxSections];
  double a1[kMeasMaxSections], a2[kMeasMaxSections];
};
struct MeasParams {
  int nrec, nstep, obs_npts, nband, passes, win_taper_type, rotate, adj_norm;
  double dt, t0, obs_tbeg, obs_dt, pre_taper, win_taper, weight;
  MeasBand band[kMeasMaxBands];
};
int design_bandpass(int order, double flo, double fhi, double dt, MeasBand* out);
// Checks a configuration (and host windows, when given) and fills p.
int check_measure_params(const sem_meas_cfg* c, int nrec, int nstep, double dt,
                         const double* windows_host, MeasParams* p);
size_t measure_scratch_doubles(const MeasParams& p);
int launch_measure_waveform(const MeasParams& p, const float* seis, const double* obs,
                            const double* win, const double* baz, double* scratch, float* adj,
                            double* mis, cudaStream_t st);

// What the kernel smoother reads from a prepared mesh (defined in
// sem_api.cu, where the mesh type lives).
struct SmoothMeshView {
  int nspec, nglob;
  float xix, jac;
  const int* ibool;       // device [nspec*125], 0-based
  const int* order;       // device [nspec] element traversal order
  const int* h_ibool;     // host copy of ibool
  const float *x, *y, *z; // host [nglob] coordinates
  // irregular elements (both null when all are regular): device irreg[e] =
  // -1 or the row of geo [nirr][125][10] (xix..gammaz, jacobian)
  const int* irreg;
  const float* geo;
};
int mesh_smooth_view(const ::sem_mesh_s* m, SmoothMeshView* out);

// Sets the per-thread error message returned by sem_last_error().
int report_error(int code, const char* fmt, ...);

// NVTX range over one C-ABI call (what a profiler's timeline shows as the
// phase: forward run, measurement, kernel sum, smoothing, ...); a no-op
// unless a profiler is attached.
struct NvtxPhase {
  explicit NvtxPhase(const char* name) { nvtxRangePushA(name); }
  ~NvtxPhase() { nvtxRangePop(); }
  NvtxPhase(const NvtxPhase&) = delete;
  NvtxPhase& operator=(const NvtxPhase&) = delete;
};

}  // namespace sem
