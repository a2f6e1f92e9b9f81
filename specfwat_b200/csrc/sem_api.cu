// Host engine and C ABI (include/sem_b200.h) of the B200 SEM time loop.
//
// The reference drives its solver through argument-free Fortran entry
// points acting on module globals (src/preproc/prepare_fwd.f90:328-368);
// here the same sequence is a handle API: a resident mesh (the database of
// read_mesh_databases_fwat), a run (prepare_timerun_fwat: mass matrix with
// the Stacey term for this dt, wavefields, boundary store), sources and
// receivers (setup_sources_receivers_fwat), the time loop (iterate_time for
// SIMULATION_TYPE 1 and 3) and the kernels (save_adjoint_kernels).
//
// Device work of a run is queued on the run's stream.  The step loop is
// either launched step by step or replayed as CUDA graphs of `graph_steps`
// steps; per-lane step counters live in device memory (LaneDesc::it0) and
// are advanced by a kernel at the end of each graph, so the graph needs no
// parameter updates between replays.

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "sem_b200.h"
#include "sem_internal.cuh"

using namespace sem;

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CK(x)                                                                   \
  do {                                                                          \
    cudaError_t e_ = (x);                                                       \
    if (e_ != cudaSuccess)                                                      \
      return fail(SEM_ERR_CUDA, "%s failed: %s", #x, cudaGetErrorString(e_));   \
  } while (0)

#define CKM(x, what)                                                            \
  do {                                                                          \
    cudaError_t e_ = (x);                                                       \
    if (e_ != cudaSuccess) {                                                    \
      cudaGetLastError();                                                       \
      return fail(SEM_ERR_NOMEM, "device allocation of %s failed: %s", what,   \
                  cudaGetErrorString(e_));                                      \
    }                                                                           \
  } while (0)

// ----------------------------------------------------------------------------
// GLL quadrature of degree 4 (closed form) and Lagrange interpolants
// ----------------------------------------------------------------------------

struct GllTables {
  double xi[5], w[5], D[5][5];
};

const GllTables& gll() {
  static GllTables t = [] {
    GllTables g{};
    const double s = std::sqrt(3.0 / 7.0);
    const double xi[5] = {-1.0, -s, 0.0, s, 1.0};
    const double w[5] = {0.1, 49.0 / 90.0, 32.0 / 45.0, 49.0 / 90.0, 0.1};
    for (int i = 0; i < 5; ++i) {
      g.xi[i] = xi[i];
      g.w[i] = w[i];
    }
    // D[i][l] = derivative of the l-th Lagrange polynomial at node i:
    // off-diagonal (pi_i / pi_l) / (x_i - x_l) with pi_m = prod_{n!=m}
    // (x_m - x_n); diagonal = sum_{n!=i} 1/(x_i - x_n).
    double pi[5];
    for (int m = 0; m < 5; ++m) {
      pi[m] = 1.0;
      for (int n = 0; n < 5; ++n)
        if (n != m) pi[m] *= (xi[m] - xi[n]);
    }
    for (int i = 0; i < 5; ++i)
      for (int l = 0; l < 5; ++l) {
        if (i != l) {
          g.D[i][l] = pi[i] / (pi[l] * (xi[i] - xi[l]));
        } else {
          double sum = 0.0;
          for (int n = 0; n < 5; ++n)
            if (n != i) sum += 1.0 / (xi[i] - xi[n]);
          g.D[i][l] = sum;
        }
      }
    return g;
  }();
  return t;
}

void lagrange_all(double x, double h[5], double hd[5]) {
  const GllTables& g = gll();
  for (int a = 0; a < 5; ++a) {
    double p = 1.0;
    for (int m = 0; m < 5; ++m)
      if (m != a) p *= (x - g.xi[m]) / (g.xi[a] - g.xi[m]);
    h[a] = p;
    double s = 0.0;
    for (int m = 0; m < 5; ++m) {
      if (m == a) continue;
      double prod = 1.0 / (g.xi[a] - g.xi[m]);
      for (int n = 0; n < 5; ++n) {
        if (n == a || n == m) continue;
        prod *= (x - g.xi[n]) / (g.xi[a] - g.xi[n]);
      }
      s += prod;
    }
    hd[a] = s;
  }
}

bool invert3(const double A[3][3], double B[3][3]) {
  const double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                     A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                     A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
  if (!(std::fabs(det) > 0.0)) return false;
  B[0][0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]) / det;
  B[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) / det;
  B[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) / det;
  B[1][0] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) / det;
  B[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) / det;
  B[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) / det;
  B[2][0] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) / det;
  B[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) / det;
  B[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) / det;
  return true;
}

double ricker(double t, double f0) {
  const double a = M_PI * M_PI * f0 * f0;
  return (1.0 - 2.0 * a * t * t) * std::exp(-a * t * t);
}

template <typename T>
struct DevArray {
  T* p = nullptr;
  size_t n = 0;
  DevArray() = default;
  DevArray(const DevArray&) = delete;
  DevArray& operator=(const DevArray&) = delete;
  ~DevArray() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t alloc(size_t count) {
    reset();
    if (count == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc((void**)&p, count * sizeof(T));
    if (e == cudaSuccess) n = count;
    return e;
  }
  size_t bytes() const { return n * sizeof(T); }
};

int check_device() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(SEM_ERR_NODEVICE, "no CUDA device: %s", cudaGetErrorString(e));
  }
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, dev);
  if (e != cudaSuccess) return fail(SEM_ERR_NODEVICE, "%s", cudaGetErrorString(e));
  if (prop.major != 10)
    return fail(SEM_ERR_NODEVICE, "device %s is sm_%d%d; this library is built for sm_100a",
                prop.name, prop.major, prop.minor);
  return SEM_OK;
}

}  // namespace

namespace sem {
// Records an error for sem_last_error from the other translation units.
int report_error(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}
}  // namespace sem

// ----------------------------------------------------------------------------
// mesh
// ----------------------------------------------------------------------------

struct sem_mesh_s {
  int nspec = 0, nglob = 0, nf = 0;
  float xix = 0.f, jac = 0.f;
  DevArray<int> ibool;
  DevArray<int> order;
  DevArray<int> corder;          // elements grouped by colour
  int ncolour = 0;
  std::vector<int> cstart;       // [ncolour + 1]
  DevArray<float> kappa, mu, rho;
  DevArray<int> f_iglob;
  DevArray<float> f_rvp, f_rvs, f_jw, f_n;
  // host copies used for set-up work
  std::vector<int> h_ibool;
  std::vector<float> h_rmass;
  std::vector<int> h_f_iglob;
  std::vector<float> h_f_rvp, h_f_rvs, h_f_jw, h_f_n;
  std::vector<float> h_x, h_y, h_z;  // point coordinates
  std::vector<int> h_irreg;          // [nspec] -1 or row of geo; empty: all regular
  DevArray<int> irreg;
  DevArray<float> geo;               // [nirreg][125][10] xix..gammaz, jacobian
  std::vector<double> centre;  // [nspec][3]
  std::vector<double> half;    // [nspec][3]
  int live_runs = 0;

  MeshView view() const {
    MeshView v{};
    v.nspec = nspec;
    v.nglob = nglob;
    v.nf = nf;
    v.xix = xix;
    v.jac = jac;
    v.ibool = ibool.p;
    v.order = order.p;
    v.corder = corder.p;
    v.irreg = irreg.p;
    v.geo = geo.p;
    v.ncolour = ncolour;
    for (int c = 0; c <= MeshView::kMaxColours; ++c)
      v.cstart[c] = c <= ncolour && ncolour > 0 ? cstart[c] : 0;
    v.kappa = kappa.p;
    v.mu = mu.p;
    v.f_iglob = f_iglob.p;
    v.f_rvp = f_rvp.p;
    v.f_rvs = f_rvs.p;
    v.f_jw = f_jw.p;
    v.f_n = f_n.p;
    return v;
  }
  size_t device_bytes() const {
    return ibool.bytes() + order.bytes() + corder.bytes() + irreg.bytes() + geo.bytes() +
           kappa.bytes() + mu.bytes() + rho.bytes() + f_iglob.bytes() +
           f_rvp.bytes() + f_rvs.bytes() + f_jw.bytes() + f_n.bytes();
  }

  // GLL interpolant of element e's coordinates at xi and its derivatives
  // dX[a][d] = dx_a / dxi_d.
  void element_map(int e, const double xi[3], double X[3], double dX[3][3]) const {
    double l[3][5], dl[3][5];
    for (int d = 0; d < 3; ++d) lagrange_all(xi[d], l[d], dl[d]);
    for (int a = 0; a < 3; ++a) {
      X[a] = 0.0;
      for (int d = 0; d < 3; ++d) dX[a][d] = 0.0;
    }
    const float* cs[3] = {h_x.data(), h_y.data(), h_z.data()};
    for (int k = 0; k < 5; ++k)
      for (int j = 0; j < 5; ++j)
        for (int i = 0; i < 5; ++i) {
          const int ig = h_ibool[(size_t)e * NGLL3 + i + 5 * j + 25 * k];
          const double w0 = l[0][i] * l[1][j] * l[2][k];
          const double wd[3] = {dl[0][i] * l[1][j] * l[2][k], l[0][i] * dl[1][j] * l[2][k],
                                l[0][i] * l[1][j] * dl[2][k]};
          for (int a = 0; a < 3; ++a) {
            const double c = (double)cs[a][ig];
            X[a] += w0 * c;
            for (int d = 0; d < 3; ++d) dX[a][d] += wd[d] * c;
          }
        }
  }

  // d xi_d / d x_a at xi in element e: xix_regular on the diagonal for a
  // regular element, else the inverse of the interpolated mapping Jacobian.
  void dxi_dx(int e, const double xi[3], double B[3][3]) const {
    for (int d = 0; d < 3; ++d)
      for (int a = 0; a < 3; ++a) B[d][a] = d == a ? (double)xix : 0.0;
    if (h_irreg.empty() || h_irreg[e] < 0) return;
    double X[3], A[3][3];
    element_map(e, xi, X, A);
    invert3(A, B);
  }

  // Newton iteration for point p in element e, xi clamped to [-1, 1];
  // returns the distance of the mapped point from p.
  double newton(int e, const double p[3], double xi[3]) const {
    xi[0] = xi[1] = xi[2] = 0.0;
    double X[3], A[3][3], B[3][3];
    for (int it = 0; it < 30; ++it) {
      element_map(e, xi, X, A);
      if (!invert3(A, B)) break;
      double step = 0.0;
      for (int d = 0; d < 3; ++d) {
        double dd = 0.0;
        for (int a = 0; a < 3; ++a) dd += B[d][a] * (p[a] - X[a]);
        xi[d] = std::min(1.5, std::max(-1.5, xi[d] + dd));
        step = std::max(step, std::fabs(dd));
      }
      if (step < 1e-13) break;
    }
    for (int d = 0; d < 3; ++d) xi[d] = std::min(1.0, std::max(-1.0, xi[d]));
    element_map(e, xi, X, A);
    return std::sqrt((X[0] - p[0]) * (X[0] - p[0]) + (X[1] - p[1]) * (X[1] - p[1]) +
                     (X[2] - p[2]) * (X[2] - p[2]));
  }

  // Element holding the point and the reference coordinates in it.  All
  // regular: the element whose centre is nearest (ties: lowest index),
  // coordinates from its axis-aligned extent, clamped to [-1, 1].  With
  // irregular elements: of the 12 nearest centres, the lowest-numbered
  // element containing the point (Newton iteration; a point on a shared
  // face, edge or corner lies in several, whose source arrays differ), else
  // the element whose located point lies closest.
  int locate(double px, double py, double pz, double xi3[3]) const {
    if (!h_irreg.empty()) {
      std::vector<std::pair<double, int>> cand((size_t)nspec);
      for (int e = 0; e < nspec; ++e) {
        const double* c = &centre[(size_t)e * 3];
        cand[e] = {(px - c[0]) * (px - c[0]) + (py - c[1]) * (py - c[1]) +
                       (pz - c[2]) * (pz - c[2]),
                   e};
      }
      const size_t nc = std::min<size_t>(12, cand.size());
      std::partial_sort(cand.begin(), cand.begin() + nc, cand.end());
      const double p[3] = {px, py, pz};
      int best = -1;
      double bd = 1e300;
      bool inside = false;
      for (size_t q = 0; q < nc; ++q) {
        const int e = cand[q].second;
        double xi[3];
        const double d = newton(e, p, xi);
        const bool in = d <= 1e-6 * 2.0 * half[(size_t)e * 3];
        const bool better = in ? (!inside || e < best) : (!inside && d < bd);
        if (better) {
          inside = inside || in;
          bd = d;
          best = e;
          for (int k = 0; k < 3; ++k) xi3[k] = xi[k];
        }
      }
      return best;
    }
    int best = -1;
    double bd = 1e300;
    for (int e = 0; e < nspec; ++e) {
      const double* c = &centre[(size_t)e * 3];
      const double d =
          (px - c[0]) * (px - c[0]) + (py - c[1]) * (py - c[1]) + (pz - c[2]) * (pz - c[2]);
      if (d < bd) {
        bd = d;
        best = e;
      }
    }
    const double* c = &centre[(size_t)best * 3];
    const double* h = &half[(size_t)best * 3];
    const double p[3] = {px, py, pz};
    for (int d = 0; d < 3; ++d) {
      double v = (p[d] - c[d]) / h[d];
      xi3[d] = v < -1.0 ? -1.0 : (v > 1.0 ? 1.0 : v);
    }
    return best;
  }
};

// ----------------------------------------------------------------------------
// run
// ----------------------------------------------------------------------------

struct sem_run_s {
  sem_mesh_s* mesh = nullptr;
  sem_run_cfg cfg{};
  int nev = 1, nstep = 0, nrec_max = 1;
  int nevp = 1;        // lanes allocated: nev rounded up to the lane-group width
  LaneMap lm{0};       // lane-group layout of the per-event arrays
  double dt = 0.0;
  cudaStream_t stream = nullptr;      // stream work is queued on
  cudaStream_t own_stream = nullptr;  // the run's own stream
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  DevArray<float> minv;
  DevArray<float> u1, v1, a1, u2, v2, a2;
  DevArray<LaneDesc> lanes;
  std::vector<LaneDesc> h_lanes;
  DevArray<float> stf, srcarr, rec_w, seis, adj;
  DevArray<int> rec_ispec;
  DevArray<unsigned char> store;
  DevArray<float> scale;
  // boundary store host spill (sem_set_store_spill): the store is cut into
  // chunks of ring_c steps (one graph launch); chunk k lives in device slot
  // k % ring_d; chunks 0 .. ring_n - ring_d - 1 are copied to pinned host
  // memory during the forward run and fetched back, one launch ahead,
  // during the adjoint run.  ring_d == 0: the whole store is resident.
  long long spill_budget = 0;     // device bytes for the store; 0 = resident, < 0 = auto
  int ring_c = 0, ring_d = 0, ring_n = 0;
  unsigned char* h_spill = nullptr;   // [ring_n - ring_d] chunks, pinned
  float* h_spill_scale = nullptr;
  size_t h_spill_bytes = 0;
  cudaStream_t copy_stream = nullptr;
  std::vector<cudaEvent_t> ev_chunk, ev_launch;  // per chunk / per launch
  DevArray<float> k_rho, k_mu, k_kappa;
  DevArray<float> k_hess;          // approximate Hessian [nglob][nevp]
  bool hess_on = false;            // accumulate it in adjoint runs
  bool hess_done = false;          // the last adjoint run accumulated it
  DevArray<double> kout, ksum;
  DevArray<double> obs, taper, simpw, misfit_rc, obs_ev;
  double taper_pct_cached = -1.0;
  int taper_type_cached = -1;
  int taper_ns_cached = -1;
  // serving: per-lane boundary stores (stream-ordered allocations)
  std::vector<void*> lane_store;
  std::vector<float*> lane_scale;
  std::vector<char> lane_saved;   // lane finished a forward with saved store
  bool lanes_mode = false;        // run driven through the sem_lane_* calls
  DevArray<int> gmap;             // serving: active 8-lane groups
  // periodic stability check (cfg.check_every > 0): per-lane non-finite
  // flags and the step each flagged lane was stopped at (device), their
  // pinned host copies for lane-driven runs, and the lane state on the host
  DevArray<int> lflags, halt_step;
  int* h_lflags = nullptr;
  int* h_halt = nullptr;
  cudaEvent_t check_ev = nullptr;
  bool check_pending = false;     // a check's flags are on their way to h_lflags
  int steps_since_check = 0;
  std::vector<char> lane_failed;
  std::vector<int> lane_fail_step;
  // lane-driven runs: pinned host staging, so that a lane's set-up and the
  // lane table reach the device without draining the stream (a copy from
  // pageable host memory first waits for all queued work)
  static constexpr int kStage = 8;
  unsigned char* h_stage_tab = nullptr;      // [kStage][lane table, group map]
  size_t stage_tab_bytes = 0;
  cudaEvent_t stage_ev[kStage] = {};
  long long stage_next = 0;
  std::vector<unsigned char*> h_lane_stage;  // per lane: set-up or observed data
  size_t lane_stage_bytes = 0;
  std::vector<cudaEvent_t> lane_ev;          // per lane: its staged copies have left
  std::vector<cudaEvent_t> lane_res_ev;      // per lane: its queued results have landed
  DevArray<double> lane_misfit;              // [nev] misfit of each lane's last measurement
  // completion marks (sem_mark): a ring of timing events on the run's stream
  static constexpr int kMarks = 16;
  cudaEvent_t mark_ev[kMarks] = {};
  long long mark_next = 0;        // token of the next mark
  std::vector<int> src_ispec, nrec;
  std::vector<char> have_src, have_rec, have_adj;
  // FK injection per event: one device allocation holding the velocity and
  // traction samples, and its shape
  struct Injection {
    float* buf = nullptr;
    int nt = 0, np = 1, k0 = 0;
  };
  std::vector<Injection> inj;
  bool fwd_saved = false, adj_done = false;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  // graph branches of the lane groups past the first: one stream each, and
  // the events that fork them from `stream` and join them back
  std::vector<cudaStream_t> chain_st;
  std::vector<cudaEvent_t> chain_ev;
  int variant[2] = {-1, -1};  // element-kernel variant per phase (fwd, adj)
  double last_ms = 0.0;
  long long last_launches = 0;
  int sm_limit = 0;   // SMs its persistent element kernels may fill (0: all)

  ~sem_run_s() {
    for (auto& j : inj)
      if (j.buf) cudaFree(j.buf);
    for (size_t l = 0; l < lane_store.size(); ++l) {
      if (lane_store[l]) cudaFreeAsync(lane_store[l], stream);
      if (lane_scale[l]) cudaFreeAsync(lane_scale[l], stream);
    }
    if (stream) cudaStreamSynchronize(stream);
    for (auto& g : gexec)
      if (g) cudaGraphExecDestroy(g);
    for (auto c : chain_st) cudaStreamDestroy(c);
    for (auto e : chain_ev) cudaEventDestroy(e);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (check_ev) cudaEventDestroy(check_ev);
    for (auto e : mark_ev)
      if (e) cudaEventDestroy(e);
    for (auto e : stage_ev)
      if (e) cudaEventDestroy(e);
    for (auto e : lane_ev)
      if (e) cudaEventDestroy(e);
    for (auto e : lane_res_ev)
      if (e) cudaEventDestroy(e);
    if (h_stage_tab) cudaFreeHost(h_stage_tab);
    for (auto p : h_lane_stage)
      if (p) cudaFreeHost(p);
    if (copy_stream) cudaStreamSynchronize(copy_stream);
    for (auto e : ev_chunk) cudaEventDestroy(e);
    for (auto e : ev_launch) cudaEventDestroy(e);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    if (h_spill) cudaFreeHost(h_spill);
    if (h_spill_scale) cudaFreeHost(h_spill_scale);
    if (h_lflags) cudaFreeHost(h_lflags);
    if (h_halt) cudaFreeHost(h_halt);
    if (own_stream) cudaStreamDestroy(own_stream);
    if (mesh) mesh->live_runs--;
  }

  size_t store_elem() const { return cfg.store_kind == SEM_STORE_FP16 ? 2 : 4; }
  size_t store_bytes_per_event() const {
    return (size_t)nstep * mesh->nf * 75 * store_elem();
  }
  bool ring() const { return ring_d > 0; }
  // one chunk of ring_c records of all events: store bytes and scale floats
  size_t chunk_store_bytes() const { return (size_t)nev * ring_c * mesh->nf * 75 * store_elem(); }
  size_t chunk_scale_floats() const {
    return cfg.store_kind == SEM_STORE_FP16 ? (size_t)nev * ring_c * mesh->nf : 0;
  }

  StepArgs args(bool adjoint) const {
    StepArgs a{};
    a.m = mesh->view();
    a.f1 = {u1.p, v1.p, a1.p};
    a.f2 = adjoint ? Fields{u2.p, v2.p, a2.p} : Fields{nullptr, nullptr, nullptr};
    a.k = {k_rho.p, k_mu.p, k_kappa.p, hess_on ? k_hess.p : nullptr};
    a.lanes = lanes.p;
    a.minv = minv.p;
    a.nev = nev;
    a.s = 0;
    a.dt = (float)dt;
    a.store_fp16 = cfg.store_kind == SEM_STORE_FP16;
    a.nrec_max = nrec_max;
    a.lm = lm;
    a.inject = 0;
    for (const auto& j : inj) a.inject |= j.buf != nullptr;
    a.sm_limit = sm_limit;
    a.ring_nev = nev;
    // public 1 = thread-per-point, 2 = pencil, 3 = pencil pipelined;
    // 0 = chosen by the autotuner per phase
    const int v = variant[adjoint ? 1 : 0];
    a.variant = cfg.kernel_variant > 0 ? cfg.kernel_variant - 1 : (v >= 0 ? v : 2);
    return a;
  }

  void fill_lanes(int phase, int save) {
    h_lanes.assign(nev, LaneDesc{});
    const size_t ns = (size_t)nstep;
    for (int e = 0; e < nev; ++e) {
      LaneDesc& L = h_lanes[e];
      L.phase = phase;
      L.it0 = 0;
      L.nstep = nstep;
      L.save = save;
      L.src_ispec = src_ispec[e];
      L.nrec = nrec[e];
      L.stf = stf.p + (size_t)e * ns;
      L.srcarr = srcarr.p + (size_t)e * 375;
      L.rec_ispec = rec_ispec.p + (size_t)e * nrec_max;
      L.rec_w = rec_w.p + (size_t)e * nrec_max * 125;
      L.seis = seis.p + (size_t)e * nrec_max * 3 * ns;
      L.adj = adj.p + (size_t)e * nrec_max * 3 * ns;
      if (ring()) {
        // lane e's rows of slot 0; slot s starts nev * ring_c rows further
        L.store = store.p ? store.p + (size_t)e * ring_c * mesh->nf * 75 * store_elem() : nullptr;
        L.scale = scale.p ? scale.p + (size_t)e * ring_c * mesh->nf : nullptr;
        L.ring_c = ring_c;
        L.ring_d = ring_d;
      } else {
        L.store = store.p ? store.p + (size_t)e * store_bytes_per_event() : nullptr;
        L.scale = scale.p ? scale.p + (size_t)e * ns * mesh->nf : nullptr;
      }
      if (e < (int)inj.size() && inj[e].buf) {
        const size_t npt3 = (size_t)mesh->nf * 25 * 3;
        L.inj_v = inj[e].buf;
        L.inj_t = inj[e].buf + (size_t)inj[e].nt * npt3;
        L.inj_nt = inj[e].nt;
        L.inj_np = inj[e].np;
        L.inj_k0 = inj[e].k0;
      }
    }
  }
};

namespace sem {
int mesh_smooth_view(const sem_mesh_s* m, SmoothMeshView* out) {
  if (!m || !out) return fail(SEM_ERR_ARG, "null mesh");
  out->nspec = m->nspec;
  out->nglob = m->nglob;
  out->xix = m->xix;
  out->jac = m->jac;
  out->ibool = m->ibool.p;
  out->order = m->order.p;
  out->h_ibool = m->h_ibool.data();
  out->x = m->h_x.data();
  out->y = m->h_y.data();
  out->z = m->h_z.data();
  out->irreg = m->irreg.p;
  out->geo = m->geo.p;
  return SEM_OK;
}
}  // namespace sem

// ----------------------------------------------------------------------------
// C ABI
// ----------------------------------------------------------------------------

extern "C" {

int sem_abi_version(void) { return SEM_ABI_VERSION; }

const char* sem_last_error(void) { return g_err.c_str(); }

int sem_device_info(int* sm_count, long long* hbm_bytes, int* cc_major, int* cc_minor) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(SEM_ERR_NODEVICE, "no CUDA device: %s", cudaGetErrorString(e));
  }
  cudaDeviceProp p;
  CK(cudaGetDeviceProperties(&p, dev));
  if (sm_count) *sm_count = p.multiProcessorCount;
  if (hbm_bytes) *hbm_bytes = (long long)p.totalGlobalMem;
  if (cc_major) *cc_major = p.major;
  if (cc_minor) *cc_minor = p.minor;
  return SEM_OK;
}

int sem_prepare_mesh(const sem_mesh_desc* d, sem_mesh** out) {
  NvtxPhase ph("sem_prepare_mesh");
  if (!d || !out) return fail(SEM_ERR_ARG, "null argument");
  *out = nullptr;
  if (d->nspec <= 0 || d->nglob <= 0) return fail(SEM_ERR_ARG, "nspec and nglob must be > 0");
  if (d->index_base != 0 && d->index_base != 1)
    return fail(SEM_ERR_ARG, "index_base must be 0 or 1");
  if (!d->ibool || !d->xstore || !d->ystore || !d->zstore || !d->kappastore || !d->mustore ||
      !d->rhostore || !d->rmass || !d->rho_vp || !d->rho_vs)
    return fail(SEM_ERR_ARG, "missing mesh array");
  const int nf = d->num_abs_boundary_faces;
  if (nf < 0) return fail(SEM_ERR_ARG, "num_abs_boundary_faces < 0");
  if (nf > 0 && (!d->abs_boundary_ispec || !d->abs_boundary_ijk ||
                 !d->abs_boundary_jacobian2Dw || !d->abs_boundary_normal))
    return fail(SEM_ERR_ARG, "missing absorbing-boundary array");
  if (!(d->xix_regular > 0.f) || !(d->jacobian_regular > 0.f))
    return fail(SEM_ERR_ARG, "xix_regular and jacobian_regular must be > 0");
  bool any_irregular = false;
  if (d->irregular_element_number)
    for (int e = 0; e < d->nspec; ++e) {
      const int k = d->irregular_element_number[e];
      if (k < 0 || k > d->nspec_irregular)
        return fail(SEM_ERR_ARG, "irregular_element_number[%d] = %d outside [0, %d]", e, k,
                    d->nspec_irregular);
      any_irregular |= k > 0;
    }
  const float* const geo_in[10] = {d->xixstore,    d->xiystore,    d->xizstore,   d->etaxstore,
                                   d->etaystore,   d->etazstore,   d->gammaxstore, d->gammaystore,
                                   d->gammazstore, d->jacobianstore};
  if (any_irregular)
    for (int q = 0; q < 10; ++q)
      if (!geo_in[q]) return fail(SEM_ERR_ARG, "irregular elements need all ten mapping arrays");
  int rc = check_device();
  if (rc) return rc;

  auto m = new sem_mesh_s();
  std::unique_ptr<sem_mesh_s> guard(m);
  m->nspec = d->nspec;
  m->nglob = d->nglob;
  m->nf = nf;
  m->xix = d->xix_regular;
  m->jac = d->jacobian_regular;
  const size_t ne = (size_t)d->nspec * NGLL3;
  m->h_ibool.resize(ne);
  for (size_t i = 0; i < ne; ++i) {
    const int g = d->ibool[i] - d->index_base;
    if (g < 0 || g >= d->nglob)
      return fail(SEM_ERR_ARG, "ibool[%zu] = %d outside [0, nglob)", i, d->ibool[i]);
    m->h_ibool[i] = g;
  }
  for (size_t i = 0; i < ne; ++i) {
    const float k = d->kappastore[i], mu = d->mustore[i], r = d->rhostore[i];
    if (!std::isfinite(k) || !std::isfinite(mu) || !std::isfinite(r) || !(r > 0.f) ||
        mu < 0.f || !(k > 0.f))
      return fail(SEM_ERR_ARG, "invalid material at element point %zu", i);
  }
  m->h_rmass.assign(d->rmass, d->rmass + d->nglob);
  if (any_irregular) {
    const size_t nirr = (size_t)d->nspec_irregular;
    m->h_irreg.assign(d->nspec, -1);
    for (int e = 0; e < d->nspec; ++e)
      if (d->irregular_element_number[e] > 0) m->h_irreg[e] = d->irregular_element_number[e] - 1;
    std::vector<float> hg(nirr * NGLL3 * 10);
    for (size_t r = 0; r < nirr; ++r)
      for (int p = 0; p < NGLL3; ++p)
        for (int q = 0; q < 10; ++q) {
          const float v = geo_in[q][r * NGLL3 + p];
          if (!std::isfinite(v) || (q == 9 && !(v > 0.f)))
            return fail(SEM_ERR_ARG, "irregular element row %zu point %d: invalid mapping", r, p);
          hg[(r * NGLL3 + p) * 10 + q] = v;
        }
    CKM(m->irreg.alloc(d->nspec), "irregular element map");
    CKM(m->geo.alloc(hg.size()), "irregular element mapping");
    CK(cudaMemcpy(m->irreg.p, m->h_irreg.data(), d->nspec * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(m->geo.p, hg.data(), hg.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  m->h_x.assign(d->xstore, d->xstore + d->nglob);
  m->h_y.assign(d->ystore, d->ystore + d->nglob);
  m->h_z.assign(d->zstore, d->zstore + d->nglob);
  for (int g = 0; g < d->nglob; ++g)
    if (!(m->h_rmass[g] > 0.f) || !std::isfinite(m->h_rmass[g]))
      return fail(SEM_ERR_ARG, "mass matrix is not positive at point %d", g);
  // element centres and half widths for locating points
  m->centre.resize((size_t)d->nspec * 3);
  m->half.resize((size_t)d->nspec * 3);
  for (int e = 0; e < d->nspec; ++e) {
    const int g0 = m->h_ibool[(size_t)e * NGLL3 + 0];
    const int g7 = m->h_ibool[(size_t)e * NGLL3 + 124];
    const float* c[3] = {d->xstore, d->ystore, d->zstore};
    for (int k = 0; k < 3; ++k) {
      m->centre[(size_t)e * 3 + k] = 0.5 * ((double)c[k][g0] + (double)c[k][g7]);
      m->half[(size_t)e * 3 + k] = 0.5 * ((double)c[k][g7] - (double)c[k][g0]);
      if (!(m->half[(size_t)e * 3 + k] > 0.0))
        return fail(SEM_ERR_ARG, "element %d has non-positive extent along axis %d", e, k);
    }
  }
  // Element traversal order: Morton (Z-curve) order of the element centres
  // on a 1024^3 lattice over the mesh bounding box, so that the elements in
  // flight at one time form a compact 3-D region whose shared GLL points
  // stay in L2 across all event lanes.
  std::vector<int> order(d->nspec);
  {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int e = 0; e < d->nspec; ++e)
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], m->centre[(size_t)e * 3 + k]);
        hi[k] = std::max(hi[k], m->centre[(size_t)e * 3 + k]);
      }
    std::vector<std::pair<unsigned long long, int>> key(d->nspec);
    for (int e = 0; e < d->nspec; ++e) {
      unsigned q[3];
      for (int k = 0; k < 3; ++k) {
        const double span = hi[k] - lo[k];
        const double v = span > 0 ? (m->centre[(size_t)e * 3 + k] - lo[k]) / span : 0.0;
        q[k] = (unsigned)std::min(1023.0, std::max(0.0, std::floor(v * 1023.0 + 0.5)));
      }
      unsigned long long code = 0;
      for (int b = 9; b >= 0; --b)
        for (int k = 2; k >= 0; --k) code = (code << 1) | ((q[k] >> b) & 1u);
      key[e] = {code, e};
    }
    std::sort(key.begin(), key.end());
    for (int e = 0; e < d->nspec; ++e) order[e] = key[e].second;
  }
  // absorbing faces: per face point global index and coefficients
  m->h_f_iglob.resize((size_t)nf * NGLL2);
  m->h_f_rvp.resize((size_t)nf * NGLL2);
  m->h_f_rvs.resize((size_t)nf * NGLL2);
  m->h_f_jw.resize((size_t)nf * NGLL2);
  m->h_f_n.resize((size_t)nf * NGLL2 * 3);
  for (int f = 0; f < nf; ++f) {
    const int e = d->abs_boundary_ispec[f] - d->index_base;
    if (e < 0 || e >= d->nspec) return fail(SEM_ERR_ARG, "abs_boundary_ispec[%d] out of range", f);
    for (int p = 0; p < NGLL2; ++p) {
      const size_t fp = (size_t)f * NGLL2 + p;
      int ijk[3];
      for (int k = 0; k < 3; ++k) {
        ijk[k] = d->abs_boundary_ijk[fp * 3 + k] - d->index_base;
        if (ijk[k] < 0 || ijk[k] >= NGLL)
          return fail(SEM_ERR_ARG, "abs_boundary_ijk of face %d point %d out of range", f, p);
      }
      const size_t lp = (size_t)e * NGLL3 + ijk[0] + NGLL * ijk[1] + NGLL2 * ijk[2];
      m->h_f_iglob[fp] = m->h_ibool[lp];
      m->h_f_rvp[fp] = d->rho_vp[lp];
      m->h_f_rvs[fp] = d->rho_vs[lp];
      m->h_f_jw[fp] = d->abs_boundary_jacobian2Dw[fp];
      for (int k = 0; k < 3; ++k) m->h_f_n[fp * 3 + k] = d->abs_boundary_normal[fp * 3 + k];
    }
  }
  CKM(m->ibool.alloc(ne), "ibool");
  CKM(m->order.alloc(d->nspec), "element order");
  CKM(m->kappa.alloc(ne), "kappastore");
  CKM(m->mu.alloc(ne), "mustore");
  CKM(m->rho.alloc(ne), "rhostore");
  CKM(m->f_iglob.alloc((size_t)nf * NGLL2), "face index");
  CKM(m->f_rvp.alloc((size_t)nf * NGLL2), "face rho_vp");
  CKM(m->f_rvs.alloc((size_t)nf * NGLL2), "face rho_vs");
  CKM(m->f_jw.alloc((size_t)nf * NGLL2), "face jacobian2Dw");
  CKM(m->f_n.alloc((size_t)nf * NGLL2 * 3), "face normal");
  CK(cudaMemcpy(m->ibool.p, m->h_ibool.data(), ne * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(m->order.p, order.data(), d->nspec * sizeof(int), cudaMemcpyHostToDevice));
  {
    // Greedy colouring in traversal order: an element takes the first
    // colour none of whose elements shares a point with it.  Within a colour
    // the elements keep the Morton order.  A structured hexahedral mesh
    // needs 8 colours.
    std::vector<int> col(d->nspec, -1);
    std::vector<std::vector<char>> used;
    int ncol = 0;
    for (int q = 0; q < d->nspec && ncol <= MeshView::kMaxColours; ++q) {
      const int e = order[q];
      const int* ib = &m->h_ibool[(size_t)e * NGLL3];
      int c = 0;
      for (;; ++c) {
        if (c == ncol) {
          used.emplace_back(d->nglob, 0);
          ++ncol;
        }
        bool ok = true;
        for (int p = 0; p < NGLL3 && ok; ++p) ok = !used[c][ib[p]];
        if (ok) break;
      }
      col[e] = c;
      for (int p = 0; p < NGLL3; ++p) used[c][ib[p]] = 1;
    }
    if (ncol <= MeshView::kMaxColours) {
      m->ncolour = ncol;
      m->cstart.assign(ncol + 1, 0);
      for (int e = 0; e < d->nspec; ++e) m->cstart[col[e] + 1]++;
      for (int c = 0; c < ncol; ++c) m->cstart[c + 1] += m->cstart[c];
      std::vector<int> pos(m->cstart.begin(), m->cstart.end() - 1), corder(d->nspec);
      for (int q = 0; q < d->nspec; ++q) corder[pos[col[order[q]]]++] = order[q];
      CKM(m->corder.alloc(d->nspec), "colour order");
      CK(cudaMemcpy(m->corder.p, corder.data(), d->nspec * sizeof(int), cudaMemcpyHostToDevice));
    }
  }
  CK(cudaMemcpy(m->kappa.p, d->kappastore, ne * sizeof(float), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(m->mu.p, d->mustore, ne * sizeof(float), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(m->rho.p, d->rhostore, ne * sizeof(float), cudaMemcpyHostToDevice));
  if (nf > 0) {
    CK(cudaMemcpy(m->f_iglob.p, m->h_f_iglob.data(), m->f_iglob.bytes(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(m->f_rvp.p, m->h_f_rvp.data(), m->f_rvp.bytes(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(m->f_rvs.p, m->h_f_rvs.data(), m->f_rvs.bytes(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(m->f_jw.p, m->h_f_jw.data(), m->f_jw.bytes(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(m->f_n.p, m->h_f_n.data(), m->f_n.bytes(), cudaMemcpyHostToDevice));
  }
  // GLL derivative tables for the element kernel
  const GllTables& g = gll();
  float D[25], DWt[25], w[5];
  for (int i = 0; i < 5; ++i) {
    w[i] = (float)g.w[i];
    for (int l = 0; l < 5; ++l) {
      D[i * 5 + l] = (float)g.D[i][l];
      DWt[i * 5 + l] = (float)(g.w[l] * g.D[l][i]);
    }
  }
  set_gll_constants(D, DWt, w);
  CK(cudaGetLastError());
  *out = guard.release();
  return SEM_OK;
}

int sem_release_mesh(sem_mesh* m) {
  if (!m) return fail(SEM_ERR_ARG, "null mesh");
  if (m->live_runs > 0) return fail(SEM_ERR_STATE, "mesh still has %d live runs", m->live_runs);
  delete m;
  return SEM_OK;
}

int sem_mesh_info(const sem_mesh* m, int* nspec, int* nglob, int* nfaces,
                  long long* device_bytes) {
  if (!m) return fail(SEM_ERR_ARG, "null mesh");
  if (nspec) *nspec = m->nspec;
  if (nglob) *nglob = m->nglob;
  if (nfaces) *nfaces = m->nf;
  if (device_bytes) *device_bytes = (long long)m->device_bytes();
  return SEM_OK;
}

static int validate_cfg(const sem_run_cfg* c) {
  if (!c) return fail(SEM_ERR_ARG, "null cfg");
  if (c->nev < 1 || c->nev > 4096) return fail(SEM_ERR_ARG, "nev must be in [1, 4096]");
  if (c->nstep < 1) return fail(SEM_ERR_ARG, "nstep must be >= 1");
  if (!(c->dt > 0.0) || !std::isfinite(c->dt)) return fail(SEM_ERR_ARG, "dt must be > 0");
  if (c->store_kind != SEM_STORE_FP32 && c->store_kind != SEM_STORE_FP16)
    return fail(SEM_ERR_ARG, "unknown store_kind %d", c->store_kind);
  if (c->max_receivers < 1 || c->max_receivers > 100000)
    return fail(SEM_ERR_ARG, "max_receivers must be in [1, 100000]");
  if (c->graph_steps < 0) return fail(SEM_ERR_ARG, "graph_steps must be >= 0");
  if (c->kernel_variant < 0 || c->kernel_variant > 15)
    return fail(SEM_ERR_ARG, "kernel_variant must be 0..15");

  return SEM_OK;
}

long long sem_run_bytes(const sem_mesh* m, const sem_run_cfg* c) {
  if (!m || validate_cfg(c)) return -1;
  const size_t ng = m->nglob, ne = (size_t)m->nspec * NGLL3, ns = c->nstep;
  const size_t nev = c->nev > 1 ? (size_t)((c->nev + 7) / 8) * 8 : 1;
  const size_t nr = c->max_receivers;
  size_t b = ng * 3 * 4;                         // minv
  b += 6 * ng * 3 * nev * 4;                     // two fields
  b += nev * (ns + 375) * 4;                     // stf + source arrays
  b += nev * nr * (4 + 125 * 4);                 // receivers
  b += 2 * nev * nr * 3 * ns * 4;                // seismograms + adjoint sources
  b += nev * ns * (size_t)m->nf * 75 * (c->store_kind == SEM_STORE_FP16 ? 2 : 4);
  if (c->store_kind == SEM_STORE_FP16) b += nev * ns * (size_t)m->nf * 4;
  b += (ng + 2 * ne) * nev * 4;                  // kernel accumulators
  b += 2 * 6 * ne * 8;                           // kernel output + sum
  b += nr * 3 * ns * 8 + 2 * ns * 8 + nr * 3 * 8;  // measurement
  return (long long)b;
}

int sem_prepare_timerun(sem_mesh* m, const sem_run_cfg* c, sem_run** out) {
  NvtxPhase ph("sem_prepare_timerun");
  if (!m || !out) return fail(SEM_ERR_ARG, "null argument");
  *out = nullptr;
  int rc = validate_cfg(c);
  if (rc) return rc;
  if (!m->h_irreg.empty() && c->kernel_variant > 1 && c->kernel_variant != 11)
    return fail(SEM_ERR_UNSUPPORTED,
                "kernel_variant %d needs regular elements; this mesh has irregular ones "
                "(use 0, 1 or 11)",
                c->kernel_variant);
  auto r = new sem_run_s();
  std::unique_ptr<sem_run_s> guard(r);
  r->mesh = m;
  m->live_runs++;
  r->cfg = *c;
  if (r->cfg.graph_steps == 0) r->cfg.graph_steps = 50;
  r->nev = c->nev;
  r->lm.lwlog = c->nev > 1 ? 3 : 0;
  r->nevp = ((c->nev + (1 << r->lm.lwlog) - 1) >> r->lm.lwlog) << r->lm.lwlog;
  r->nstep = c->nstep;
  r->dt = c->dt;
  r->nrec_max = c->max_receivers;
  // SEM_FORCE_VARIANTS="f,a" pins the autotuned element-kernel variants
  // (public numbering 1..15) for the forward and adjoint phases, so that a
  // profiler run replays the choice made by an unprofiled run.
  if (c->kernel_variant == 0) {
    const char* fv = std::getenv("SEM_FORCE_VARIANTS");
    int vf = 0, va = 0;
    if (fv && std::sscanf(fv, "%d,%d", &vf, &va) == 2 && vf >= 1 && vf <= 15 && va >= 1 &&
        va <= 15) {
      r->variant[0] = vf - 1;
      r->variant[1] = va - 1;
    }
  }
  CK(cudaStreamCreateWithFlags(&r->own_stream, cudaStreamNonBlocking));
  r->stream = r->own_stream;
  CK(cudaEventCreate(&r->e0));
  CK(cudaEventCreate(&r->e1));

  // 1/(M + dt/2 C): Stacey's diagonal damping folded into the mass so the
  // absorbing term is implicit in the corrector velocity.
  const size_t ng = m->nglob;
  std::vector<double> mx(ng * 3);
  for (size_t g = 0; g < ng; ++g)
    for (int k = 0; k < 3; ++k) mx[g * 3 + k] = (double)m->h_rmass[g];
  for (int f = 0; f < m->nf; ++f)
    for (int p = 0; p < NGLL2; ++p) {
      const size_t fp = (size_t)f * NGLL2 + p;
      const size_t g = (size_t)m->h_f_iglob[fp];
      const double rvp = m->h_f_rvp[fp], rvs = m->h_f_rvs[fp], jw = m->h_f_jw[fp];
      for (int k = 0; k < 3; ++k) {
        const double n = m->h_f_n[fp * 3 + k];
        mx[g * 3 + k] += 0.5 * c->dt * jw * (rvp * n * n + rvs * (1.0 - n * n));
      }
    }
  std::vector<float> mi(ng * 3);
  for (size_t i = 0; i < mi.size(); ++i) mi[i] = (float)(1.0 / mx[i]);
  CKM(r->minv.alloc(ng * 3), "inverse mass");
  CK(cudaMemcpy(r->minv.p, mi.data(), r->minv.bytes(), cudaMemcpyHostToDevice));

  const size_t nev = r->nev, ns = r->nstep, nr = r->nrec_max, ne = (size_t)m->nspec * NGLL3;
  const size_t nf3 = ng * 3 * (size_t)r->nevp;
  CKM(r->u1.alloc(nf3), "displ");
  CKM(r->v1.alloc(nf3), "veloc");
  CKM(r->a1.alloc(nf3), "accel");
  CKM(r->lanes.alloc(nev), "lane table");
  CKM(r->stf.alloc(nev * ns), "source time functions");
  CKM(r->srcarr.alloc(nev * 375), "source arrays");
  CKM(r->rec_ispec.alloc(nev * nr), "receiver elements");
  CKM(r->rec_w.alloc(nev * nr * 125), "receiver weights");
  CKM(r->seis.alloc(nev * nr * 3 * ns), "seismograms");
  CKM(r->adj.alloc(nev * nr * 3 * ns), "adjoint sources");
  CK(cudaMemsetAsync(r->seis.p, 0, r->seis.bytes(), r->stream));
  CK(cudaMemsetAsync(r->adj.p, 0, r->adj.bytes(), r->stream));
  (void)ne;
  r->src_ispec.assign(nev, -1);
  r->nrec.assign(nev, 0);
  r->have_src.assign(nev, 0);
  r->inj.assign(nev, sem_run_s::Injection{});
  r->have_rec.assign(nev, 0);
  r->have_adj.assign(nev, 0);
  CK(cudaStreamSynchronize(r->stream));
  *out = guard.release();
  return SEM_OK;
}

int sem_release_run(sem_run* r) {
  if (!r) return fail(SEM_ERR_ARG, "null run");
  cudaStreamSynchronize(r->stream);
  delete r;
  return SEM_OK;
}

int sem_set_sources(sem_run* r, int nev, const sem_source* src) {
  if (!r || !src) return fail(SEM_ERR_ARG, "null argument");
  if (nev != r->nev) return fail(SEM_ERR_ARG, "nev %d != run nev %d", nev, r->nev);
  const size_t ns = r->nstep;
  std::vector<float> stf((size_t)nev * ns), sa((size_t)nev * 375);
  for (int e = 0; e < nev; ++e) {
    const sem_source& s = src[e];
    if (!(s.f0 > 0.0) || !std::isfinite(s.x + s.y + s.z))
      return fail(SEM_ERR_ARG, "source %d: invalid position or f0", e);
    double xi3[3];
    const int ispec = r->mesh->locate(s.x, s.y, s.z, xi3);
    r->src_ispec[e] = ispec;
    // CMT (r, theta, phi) -> x=E, y=N, z=Up (locate_source_fwat.f90:215-228)
    const double Mzz = s.Mrr, Myy = s.Mtt, Mxx = s.Mpp;
    const double Myz = -s.Mrt, Mxz = s.Mrp, Mxy = -s.Mtp;
    const double M[3][3] = {{Mxx, Mxy, Mxz}, {Mxy, Myy, Myz}, {Mxz, Myz, Mzz}};
    double hx[5], hxd[5], hy[5], hyd[5], hz[5], hzd[5];
    lagrange_all(xi3[0], hx, hxd);
    lagrange_all(xi3[1], hy, hyd);
    lagrange_all(xi3[2], hz, hzd);
    double B[3][3];
    r->mesh->dxi_dx(ispec, xi3, B);
    for (int c = 0; c < 5; ++c)
      for (int b = 0; b < 5; ++b)
        for (int a = 0; a < 5; ++a) {
          // gradient of the interpolant phi_abc at the source
          const double dr[3] = {hxd[a] * hy[b] * hz[c], hx[a] * hyd[b] * hz[c],
                                hx[a] * hy[b] * hzd[c]};
          double gr[3];
          for (int k = 0; k < 3; ++k) gr[k] = B[0][k] * dr[0] + B[1][k] * dr[1] + B[2][k] * dr[2];
          const int p = a + 5 * b + 25 * c;
          for (int k = 0; k < 3; ++k)
            sa[(size_t)e * 375 + p * 3 + k] =
                (float)(M[k][0] * gr[0] + M[k][1] * gr[1] + M[k][2] * gr[2]);
        }
    const double t0 = 1.2 / s.f0 + s.tshift;
    for (size_t it = 0; it < ns; ++it)
      stf[(size_t)e * ns + it] = (float)ricker((double)it * r->dt - t0, s.f0);
    r->have_src[e] = 1;
  }
  CK(cudaMemcpyAsync(r->stf.p, stf.data(), r->stf.bytes(), cudaMemcpyHostToDevice, r->stream));
  CK(cudaMemcpyAsync(r->srcarr.p, sa.data(), r->srcarr.bytes(), cudaMemcpyHostToDevice,
                     r->stream));
  CK(cudaStreamSynchronize(r->stream));
  return SEM_OK;
}

// Receiver elements and Lagrange weights of nrec receivers into isp
// [nrec_max] and w [nrec_max][125] (entries past nrec zero).
static int receivers_host(sem_run* r, int nrec, const double* xyz, int* isp, float* w) {
  std::fill(isp, isp + r->nrec_max, 0);
  std::fill(w, w + (size_t)r->nrec_max * 125, 0.f);
  for (int k = 0; k < nrec; ++k) {
    if (!std::isfinite(xyz[k * 3] + xyz[k * 3 + 1] + xyz[k * 3 + 2]))
      return fail(SEM_ERR_ARG, "receiver %d position is not finite", k);
    double xi3[3];
    isp[k] = r->mesh->locate(xyz[k * 3], xyz[k * 3 + 1], xyz[k * 3 + 2], xi3);
    double hx[5], hy[5], hz[5], d[5];
    lagrange_all(xi3[0], hx, d);
    lagrange_all(xi3[1], hy, d);
    lagrange_all(xi3[2], hz, d);
    for (int c = 0; c < 5; ++c)
      for (int b = 0; b < 5; ++b)
        for (int a = 0; a < 5; ++a)
          w[(size_t)k * 125 + a + 5 * b + 25 * c] = (float)(hx[a] * hy[b] * hz[c]);
  }
  return SEM_OK;
}

int sem_set_receivers(sem_run* r, int ev, int nrec, const double* xyz) {
  if (!r || (!xyz && nrec > 0)) return fail(SEM_ERR_ARG, "null argument");
  if (nrec < 0 || nrec > r->nrec_max)
    return fail(SEM_ERR_ARG, "nrec %d outside [0, max_receivers=%d]", nrec, r->nrec_max);
  if (ev < -1 || ev >= r->nev) return fail(SEM_ERR_ARG, "event %d out of range", ev);
  std::vector<int> isp(r->nrec_max, 0);
  std::vector<float> w((size_t)r->nrec_max * 125, 0.f);
  int rrc = receivers_host(r, nrec, xyz, isp.data(), w.data());
  if (rrc) return rrc;
  const int e0 = ev < 0 ? 0 : ev, e1 = ev < 0 ? r->nev : ev + 1;
  for (int e = e0; e < e1; ++e) {
    CK(cudaMemcpyAsync(r->rec_ispec.p + (size_t)e * r->nrec_max, isp.data(),
                       isp.size() * sizeof(int), cudaMemcpyHostToDevice, r->stream));
    CK(cudaMemcpyAsync(r->rec_w.p + (size_t)e * r->nrec_max * 125, w.data(),
                       w.size() * sizeof(float), cudaMemcpyHostToDevice, r->stream));
    r->nrec[e] = nrec;
    r->have_rec[e] = 1;
  }
  CK(cudaStreamSynchronize(r->stream));
  return SEM_OK;
}

static int ensure_adjoint_buffers(sem_run* r) {
  const size_t ng = r->mesh->nglob, nev = r->nevp, ne = (size_t)r->mesh->nspec * NGLL3;
  if (!r->u2.p) {
    CKM(r->u2.alloc(ng * 3 * nev), "backward displ");
    CKM(r->v2.alloc(ng * 3 * nev), "backward veloc");
    CKM(r->a2.alloc(ng * 3 * nev), "backward accel");
  }
  if (!r->k_rho.p) {
    CKM(r->k_rho.alloc(ng * nev), "rho kernel");
    CKM(r->k_mu.alloc(ne * nev), "mu kernel");
    CKM(r->k_kappa.alloc(ne * nev), "kappa kernel");
  }
  if (r->hess_on && !r->k_hess.p) {
    CKM(r->k_hess.alloc(ng * nev), "Hessian kernel");
    CK(cudaMemsetAsync(r->k_hess.p, 0, r->k_hess.bytes(), r->stream));
  }
  return SEM_OK;
}

// Device bytes reserved beside the store in the automatic spill budget:
// the FP64 kernel output and sum (6 values per element point each), the
// measurement buffers and 1 GiB of slack.
static size_t spill_reserve(const sem_run* r) {
  const size_t ne = (size_t)r->mesh->nspec * NGLL3;
  return 2 * 6 * ne * 8 + (size_t)r->nrec_max * 3 * r->nstep * 8 * 2 + ((size_t)1 << 30);
}

static void release_ring(sem_run* r) {
  if (r->copy_stream) cudaStreamSynchronize(r->copy_stream);
  if (r->h_spill) cudaFreeHost(r->h_spill);
  if (r->h_spill_scale) cudaFreeHost(r->h_spill_scale);
  r->h_spill = nullptr;
  r->h_spill_scale = nullptr;
  r->h_spill_bytes = 0;
  for (auto e : r->ev_chunk) cudaEventDestroy(e);
  for (auto e : r->ev_launch) cudaEventDestroy(e);
  r->ev_chunk.clear();
  r->ev_launch.clear();
  r->ring_c = r->ring_d = r->ring_n = 0;
}

static int ensure_store(sem_run* r) {
  if (r->mesh->nf == 0 || r->store.p) return SEM_OK;
  release_ring(r);
  const size_t full = r->store_bytes_per_event() * r->nev +
                      (r->cfg.store_kind == SEM_STORE_FP16
                           ? (size_t)r->nev * r->nstep * r->mesh->nf * 4 : 0);
  if (r->spill_budget != 0) {
    long long budget = r->spill_budget;
    if (budget < 0) {
      size_t fr = 0, tot = 0;
      CK(cudaMemGetInfo(&fr, &tot));
      budget = (long long)fr - (long long)spill_reserve(r);
    }
    r->ring_c = r->cfg.graph_steps;
    r->ring_n = (r->nstep + r->ring_c - 1) / r->ring_c;
    const size_t slot = r->chunk_store_bytes() + r->chunk_scale_floats() * 4;
    const long long d = budget > 0 ? budget / (long long)slot : 0;
    if ((size_t)budget >= full || d >= r->ring_n) {
      r->ring_c = r->ring_n = 0;  // fits: resident
    } else if (d < 2) {
      r->ring_c = r->ring_n = 0;
      return fail(SEM_ERR_NOMEM,
                  "boundary store spill: a device budget of %lld bytes holds %lld chunk slots "
                  "of %zu bytes; at least 2 are needed",
                  budget, d, slot);
    } else {
      r->ring_d = (int)d;
    }
  }
  if (r->ring()) {
    const int spilled = r->ring_n - r->ring_d;
    CKM(r->store.alloc(r->chunk_store_bytes() * r->ring_d), "boundary store ring");
    if (r->cfg.store_kind == SEM_STORE_FP16)
      CKM(r->scale.alloc(r->chunk_scale_floats() * r->ring_d), "boundary store ring scales");
    r->h_spill_bytes = r->chunk_store_bytes() * spilled;
    cudaError_t e = cudaHostAlloc((void**)&r->h_spill, r->h_spill_bytes, cudaHostAllocDefault);
    if (e == cudaSuccess && r->chunk_scale_floats())
      e = cudaHostAlloc((void**)&r->h_spill_scale, r->chunk_scale_floats() * 4 * spilled,
                        cudaHostAllocDefault);
    if (e != cudaSuccess) {
      cudaGetLastError();
      const size_t want = r->h_spill_bytes;
      release_ring(r);
      r->store.reset();
      r->scale.reset();
      return fail(SEM_ERR_NOMEM, "pinned host memory for the spilled boundary store (%zu bytes): %s",
                  want, cudaGetErrorString(e));
    }
    if (!r->copy_stream) CK(cudaStreamCreateWithFlags(&r->copy_stream, cudaStreamNonBlocking));
    r->ev_chunk.assign(r->ring_n, nullptr);
    r->ev_launch.assign(r->ring_n, nullptr);
    for (auto& ev : r->ev_chunk) CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    for (auto& ev : r->ev_launch) CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    return SEM_OK;
  }
  CKM(r->store.alloc(r->store_bytes_per_event() * r->nev), "boundary store");
  if (r->cfg.store_kind == SEM_STORE_FP16)
    CKM(r->scale.alloc((size_t)r->nev * r->nstep * r->mesh->nf), "boundary store scales");
  return SEM_OK;
}

// Autotuner: time each element-kernel variant of a phase over a few steps
// of the current run (its own event count, lanes per block and mesh) and
// keep the fastest.  Runs on scratch state before the forward run: the
// forward zeroes its wavefields and the adjoint run rebuilds its own.
static int autotune_phase(sem_run* r, bool adj) {
  const int cands_multi[] = {0, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 13, 14};
  const int cands_single[] = {0, 2, 12};
  const int* cands = r->nev > 1 ? cands_multi : cands_single;
  const int ncand = r->nev > 1 ? 13 : 3;
  const int nsteps = std::max(1, std::min(8, r->nstep - 2));
  r->fill_lanes(adj ? PH_ADJ : PH_FWD, 0);
  for (auto& L : r->h_lanes) L.it0 = 1;
  CK(cudaMemcpyAsync(r->lanes.p, r->h_lanes.data(), r->lanes.bytes(), cudaMemcpyHostToDevice,
                     r->stream));
  cudaEvent_t t0, t1;
  CK(cudaEventCreate(&t0));
  CK(cudaEventCreate(&t1));
  double best = 1e300;
  int bestv = 2;
  for (int ci = 0; ci < ncand; ++ci) {
    r->variant[adj ? 1 : 0] = cands[ci];
    StepArgs a = r->args(adj);
    a.s = 0;
    launch_forces(a, adj, r->stream);  // warm-up (first-launch set-up)
    CK(cudaEventRecord(t0, r->stream));
    for (int s = 0; s < nsteps; ++s) {
      a.s = s;
      launch_forces(a, adj, r->stream);
    }
    CK(cudaEventRecord(t1, r->stream));
    CK(cudaGetLastError());
    CK(cudaEventSynchronize(t1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, t0, t1));
    if (ms < best) {
      best = ms;
      bestv = cands[ci];
    }
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  r->variant[adj ? 1 : 0] = bestv;
  return SEM_OK;
}

static int ensure_tuned(sem_run* r) {
  if (r->cfg.kernel_variant != 0 || (r->variant[0] >= 0 && r->variant[1] >= 0)) return SEM_OK;
  if (!r->mesh->h_irreg.empty()) {
    // irregular elements: the register-prefetch kernels for batches, the
    // thread-per-point kernel for one event
    r->variant[0] = r->variant[1] = r->nev > 1 ? 10 : 0;
    return SEM_OK;
  }
  if (r->nstep < 3) {
    r->variant[0] = r->variant[1] = 2;
    return SEM_OK;
  }
  int rc = ensure_adjoint_buffers(r);
  if (rc) return rc;
  CK(cudaMemsetAsync(r->u2.p, 0, r->u2.bytes(), r->stream));
  CK(cudaMemsetAsync(r->v2.p, 0, r->v2.bytes(), r->stream));
  CK(cudaMemsetAsync(r->a2.p, 0, r->a2.bytes(), r->stream));
  rc = autotune_phase(r, false);
  if (rc) return rc;
  rc = autotune_phase(r, true);
  if (rc) return rc;
  // discard the kernel products accumulated while timing
  CK(cudaMemsetAsync(r->k_mu.p, 0, r->k_mu.bytes(), r->stream));
  CK(cudaMemsetAsync(r->k_kappa.p, 0, r->k_kappa.bytes(), r->stream));
  return SEM_OK;
}

// Periodic stability check (cfg.check_every > 0).  The per-lane flags and
// halt steps start cleared (flags 0, halt step -1) for every lane.
static int ensure_check_buffers(sem_run* r) {
  if (r->lflags.p) return SEM_OK;
  CKM(r->lflags.alloc((size_t)r->nev), "stability flags");
  CKM(r->halt_step.alloc((size_t)r->nev), "stability halt steps");
  CK(cudaMallocHost((void**)&r->h_lflags, (size_t)r->nev * sizeof(int)));
  CK(cudaMallocHost((void**)&r->h_halt, (size_t)r->nev * sizeof(int)));
  CK(cudaEventCreateWithFlags(&r->check_ev, cudaEventDisableTiming));
  CK(cudaMemsetAsync(r->lflags.p, 0, r->lflags.bytes(), r->stream));
  CK(cudaMemsetAsync(r->halt_step.p, 0xff, r->halt_step.bytes(), r->stream));
  r->lane_failed.assign(r->nev, 0);
  r->lane_fail_step.assign(r->nev, -1);
  return SEM_OK;
}

// Queue a scan of the run's fields (the backward field too once it exists)
// and stop the lanes found non-finite; s_off = steps the kernels have done
// beyond each lane's device it0.
static void queue_check(sem_run* r, bool both, int s_off) {
  launch_check_lanes(r->u1.p, r->mesh->nglob, r->lm.lwlog, r->nevp, r->lanes.p, r->nev,
                     r->lflags.p, r->stream);
  if (both && r->u2.p)
    launch_check_lanes(r->u2.p, r->mesh->nglob, r->lm.lwlog, r->nevp, r->lanes.p, r->nev,
                       r->lflags.p, r->stream);
  launch_halt_lanes(r->lanes.p, r->nev, r->lflags.p, r->halt_step.p, s_off, r->stream);
}

// Boundary store ring: the stream work around launch unit g (steps
// [g K, (g+1) K) of the phase, K = ring_c).  Forward (saving): the unit
// writes chunk g into slot g % D once the spill of chunk g - D, the slot's
// previous chunk, has left; chunks below N - D are then spilled to the host
// on the copy stream.  Adjoint: unit g replays records nstep-1-j for its j,
// i.e. chunks lo..hi; a spilled chunk k is fetched into slot k % D right
// after the unit that replays the last record of chunk k + D (the slot's
// occupant), at least (D - 1) K + 1 steps before chunk k is first needed.
static int ring_before(sem_run* r, bool adjoint, int g, bool save) {
  const int K = r->ring_c, D = r->ring_d, N = r->ring_n;
  if (!adjoint) {
    if (save && g >= D && g - D < N - D) CK(cudaStreamWaitEvent(r->stream, r->ev_chunk[g - D], 0));
    return SEM_OK;
  }
  const int ns = r->nstep;
  const int jhi = std::min((g + 1) * K, ns) - 1;
  const int lo = (ns - 1 - jhi) / K, hi = (ns - 1 - g * K) / K;
  for (int k = lo; k <= hi && k < N - D; ++k)
    CK(cudaStreamWaitEvent(r->stream, r->ev_chunk[k], 0));
  return SEM_OK;
}

static int ring_after(sem_run* r, bool adjoint, int g, bool save) {
  const int K = r->ring_c, D = r->ring_d, N = r->ring_n;
  const size_t cs = r->chunk_store_bytes(), cf = r->chunk_scale_floats();
  if (!adjoint) {
    if (!save || g >= N - D) return SEM_OK;
    CK(cudaEventRecord(r->ev_launch[g], r->stream));
    CK(cudaStreamWaitEvent(r->copy_stream, r->ev_launch[g], 0));
    const int slot = g % D;
    CK(cudaMemcpyAsync(r->h_spill + (size_t)g * cs, r->store.p + (size_t)slot * cs, cs,
                       cudaMemcpyDeviceToHost, r->copy_stream));
    if (cf)
      CK(cudaMemcpyAsync(r->h_spill_scale + (size_t)g * cf, r->scale.p + (size_t)slot * cf,
                         cf * 4, cudaMemcpyDeviceToHost, r->copy_stream));
    CK(cudaEventRecord(r->ev_chunk[g], r->copy_stream));
    return SEM_OK;
  }
  bool recorded = false;
  for (int k = 0; k < N - D; ++k) {
    // unit replaying record (k + D) K, the last one of chunk k + D
    const int last_use = (r->nstep - 1 - (k + D) * K) / K;
    if (last_use != g) continue;
    if (!recorded) {
      CK(cudaEventRecord(r->ev_launch[g], r->stream));
      CK(cudaStreamWaitEvent(r->copy_stream, r->ev_launch[g], 0));
      recorded = true;
    }
    const int slot = k % D;
    CK(cudaMemcpyAsync(r->store.p + (size_t)slot * cs, r->h_spill + (size_t)k * cs, cs,
                       cudaMemcpyHostToDevice, r->copy_stream));
    if (cf)
      CK(cudaMemcpyAsync(r->scale.p + (size_t)slot * cf, r->h_spill_scale + (size_t)k * cf,
                         cf * 4, cudaMemcpyHostToDevice, r->copy_stream));
    CK(cudaEventRecord(r->ev_chunk[k], r->copy_stream));
  }
  return SEM_OK;
}

// Step arguments of lane group g (lanes 8g .. 8g+7) of a batched run as a
// run of its own: every per-lane array starts at the group's block of the
// lane-group layout, so the kernels see lanes 0..7 of one group.
static StepArgs group_args(const sem_run* r, const StepArgs& a, int g) {
  StepArgs ag = a;
  const int lw = 1 << a.lm.lwlog;
  const size_t fg = (size_t)g * r->mesh->nglob * 3 * lw;   // field values of a group
  const size_t pg = (size_t)g * r->mesh->nglob * lw;       // per-point values
  const size_t eg = (size_t)g * r->mesh->nspec * 125 * lw; // per element point
  auto off = [](float* p, size_t o) { return p ? p + o : p; };
  ag.f1 = {off(a.f1.u, fg), off(a.f1.v, fg), off(a.f1.a, fg)};
  ag.f2 = {off(a.f2.u, fg), off(a.f2.v, fg), off(a.f2.a, fg)};
  ag.k = {off(a.k.rho_glob, pg), off(a.k.mu, eg), off(a.k.kappa, eg), off(a.k.hess_glob, pg)};
  ag.lanes = a.lanes + (size_t)g * lw;
  ag.nev = std::min(lw, a.nev - g * lw);
  ag.gmap = nullptr;
  ag.ngmap = 0;
  return ag;
}

// Lane groups captured as separate graph branches: the groups' events are
// independent, so one group's update (HBM-bound) can run while another
// group's element kernel (bound by shared memory and latency) holds the SMs.
static int chain_groups(const sem_run* r) {
  if (r->lm.lwlog != 3 || r->nev <= 8 || r->mesh->nglob == 0) return 1;
  return (r->nev + 7) / 8;
}

static int ensure_chains(sem_run* r, int G) {
  while ((int)r->chain_st.size() < G - 1) {
    cudaStream_t c;
    CK(cudaStreamCreateWithFlags(&c, cudaStreamNonBlocking));
    r->chain_st.push_back(c);
  }
  while ((int)r->chain_ev.size() < G) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    r->chain_ev.push_back(e);
  }
  return SEM_OK;
}

// Queue the step loop of one phase (graphs or per-step launches).
static int run_loop(sem_run* r, bool adjoint) {
  long long launches = 0;
  StepArgs a = r->args(adjoint);
  const bool save = !adjoint && !r->h_lanes.empty() && r->h_lanes[0].save;
  CK(cudaEventRecord(r->e0, r->stream));
  if (r->cfg.use_graph) {
    const int K = r->cfg.graph_steps;
    cudaGraphExec_t& gx = r->gexec[adjoint ? 1 : 0];
    if (!gx) {
      cudaGraph_t g;
      const int G = chain_groups(r);
      if (G > 1) {
        int rc = ensure_chains(r, G);
        if (rc) return rc;
      }
      CK(cudaStreamBeginCapture(r->stream, cudaStreamCaptureModeThreadLocal));
      if (G > 1) {
        CK(cudaEventRecord(r->chain_ev[0], r->stream));
        for (int c = 1; c < G; ++c) CK(cudaStreamWaitEvent(r->chain_st[c - 1], r->chain_ev[0], 0));
      }
      for (int c = 0; c < G; ++c) {
        cudaStream_t st = c == 0 ? r->stream : r->chain_st[c - 1];
        StepArgs ac = G > 1 ? group_args(r, a, c) : a;
        for (int s = 0; s < K; ++s) {
          ac.s = s;
          launch_forces(ac, adjoint, st);
          launch_boundary(ac, adjoint, st);
          launch_points(ac, st);
          launch_update(ac, adjoint, st);
        }
      }
      if (G > 1)
        for (int c = 1; c < G; ++c) {
          CK(cudaEventRecord(r->chain_ev[c], r->chain_st[c - 1]));
          CK(cudaStreamWaitEvent(r->stream, r->chain_ev[c], 0));
        }
      launch_advance(r->lanes.p, r->nev, K, r->stream);
      cudaError_t ce = cudaStreamEndCapture(r->stream, &g);
      if (ce != cudaSuccess) return fail(SEM_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
      ce = cudaGraphInstantiate(&gx, g, 0);
      cudaGraphDestroy(g);
      if (ce != cudaSuccess)
        return fail(SEM_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
    }
    const int nlaunch = (r->nstep + K - 1) / K;
    const int per_step = (r->mesh->nf > 0 ? 4 : 3) * chain_groups(r);
    const int ce = r->cfg.check_every;
    const bool ring = r->ring() && (adjoint || save);
    for (int g = 0; g < nlaunch; ++g) {
      if (ring) {
        int rc = ring_before(r, adjoint, g, save);
        if (rc) return rc;
      }
      CK(cudaGraphLaunch(gx, r->stream));
      launches += (long long)K * per_step + 1;
      if (ring) {
        int rc = ring_after(r, adjoint, g, save);
        if (rc) return rc;
      }
      // stability check at the first graph boundary at or after every
      // check_every steps, and after the last graph (each graph advances
      // the lanes' device it0 by K)
      if (ce > 0 && (g == nlaunch - 1 || (long long)(g + 1) * K / ce > (long long)g * K / ce)) {
        queue_check(r, adjoint, 0);
        launches += adjoint ? 3 : 2;
      }
    }
  } else {
    const int ce = r->cfg.check_every;
    const bool ring = r->ring() && (adjoint || save);
    const int K = ring ? r->ring_c : r->nstep;
    for (int s = 0; s < r->nstep; ++s) {
      if (ring && s % K == 0) {
        int rc = ring_before(r, adjoint, s / K, save);
        if (rc) return rc;
      }
      a.s = s;
      launches += launch_forces(a, adjoint, r->stream);
      launches += launch_boundary(a, adjoint, r->stream);
      launches += launch_points(a, r->stream);
      launches += launch_update(a, adjoint, r->stream);
      if (ring && ((s + 1) % K == 0 || s == r->nstep - 1)) {
        int rc = ring_after(r, adjoint, s / K, save);
        if (rc) return rc;
      }
      if (ce > 0 && ((s + 1) % ce == 0 || s == r->nstep - 1)) {
        queue_check(r, adjoint, s + 1);
        launches += adjoint ? 3 : 2;
      }
    }
  }
  if (r->copy_stream && r->ring()) {
    // the phase ends when its copies have too
    CK(cudaEventRecord(r->ev_launch[0], r->copy_stream));
    CK(cudaStreamWaitEvent(r->stream, r->ev_launch[0], 0));
  }
  CK(cudaGetLastError());
  CK(cudaEventRecord(r->e1, r->stream));
  r->last_launches = launches;
  return SEM_OK;
}

int sem_iterate_time(sem_run* r, int sim_type, int save_forward) {
  NvtxPhase ph(sim_type == 3 ? "sem_iterate_time adjoint" : "sem_iterate_time forward");
  if (!r) return fail(SEM_ERR_ARG, "null run");
  if (r->lanes_mode)
    return fail(SEM_ERR_STATE, "run is driven lane by lane (sem_lane_*); use sem_advance");
  const size_t n3 = (size_t)r->mesh->nglob * 3 * r->nevp;
  if (r->cfg.check_every > 0 && (sim_type == 1 || sim_type == 3)) {
    int rc = ensure_check_buffers(r);
    if (rc) return rc;
    CK(cudaMemsetAsync(r->lflags.p, 0, r->lflags.bytes(), r->stream));
    CK(cudaMemsetAsync(r->halt_step.p, 0xff, r->halt_step.bytes(), r->stream));
  }
  if (sim_type == 1) {
    for (int e = 0; e < r->nev; ++e)
      if (!(r->have_src[e] || r->inj[e].buf) || !r->have_rec[e])
        return fail(SEM_ERR_STATE, "event %d has no source, injection or receivers", e);
    int trc = ensure_tuned(r);
    if (trc) return trc;
    if (save_forward) {
      int rc = ensure_store(r);
      if (rc) return rc;
    }
    CK(cudaMemsetAsync(r->u1.p, 0, n3 * 4, r->stream));
    CK(cudaMemsetAsync(r->v1.p, 0, n3 * 4, r->stream));
    CK(cudaMemsetAsync(r->a1.p, 0, n3 * 4, r->stream));
    r->fill_lanes(PH_FWD, save_forward ? 1 : 0);
    CK(cudaMemcpyAsync(r->lanes.p, r->h_lanes.data(), r->lanes.bytes(), cudaMemcpyHostToDevice,
                       r->stream));
    int rc = run_loop(r, false);
    if (rc) return rc;
    r->fwd_saved = save_forward != 0;
    r->adj_done = false;
  } else if (sim_type == 3) {
    if (!r->fwd_saved)
      return fail(SEM_ERR_STATE, "sim_type 3 needs a previous sim_type 1 with save_forward");
    for (int e = 0; e < r->nev; ++e)
      if (!r->have_adj[e]) return fail(SEM_ERR_STATE, "event %d has no adjoint sources", e);
    int rc = ensure_adjoint_buffers(r);
    if (rc) return rc;
    // backward field starts from the final forward state; adjoint at rest
    CK(cudaMemcpyAsync(r->u2.p, r->u1.p, n3 * 4, cudaMemcpyDeviceToDevice, r->stream));
    CK(cudaMemcpyAsync(r->v2.p, r->v1.p, n3 * 4, cudaMemcpyDeviceToDevice, r->stream));
    CK(cudaMemcpyAsync(r->a2.p, r->a1.p, n3 * 4, cudaMemcpyDeviceToDevice, r->stream));
    CK(cudaMemsetAsync(r->u1.p, 0, n3 * 4, r->stream));
    CK(cudaMemsetAsync(r->v1.p, 0, n3 * 4, r->stream));
    CK(cudaMemsetAsync(r->a1.p, 0, n3 * 4, r->stream));
    CK(cudaMemsetAsync(r->k_rho.p, 0, r->k_rho.bytes(), r->stream));
    CK(cudaMemsetAsync(r->k_mu.p, 0, r->k_mu.bytes(), r->stream));
    CK(cudaMemsetAsync(r->k_kappa.p, 0, r->k_kappa.bytes(), r->stream));
    if (r->hess_on) CK(cudaMemsetAsync(r->k_hess.p, 0, r->k_hess.bytes(), r->stream));
    r->hess_done = r->hess_on;
    r->fill_lanes(PH_ADJ, 0);
    CK(cudaMemcpyAsync(r->lanes.p, r->h_lanes.data(), r->lanes.bytes(), cudaMemcpyHostToDevice,
                       r->stream));
    rc = run_loop(r, true);
    if (rc) return rc;
    r->fwd_saved = false;  // the final state has been consumed
    r->adj_done = true;
  } else {
    return fail(SEM_ERR_ARG, "sim_type must be 1 or 3");
  }
  if (r->cfg.check_every > 0) {
    // the checks ran inside the loop; a flagged event stopped at its check
    std::vector<int> fl(r->nev), hs(r->nev);
    CK(cudaMemcpyAsync(fl.data(), r->lflags.p, r->lflags.bytes(), cudaMemcpyDeviceToHost,
                       r->stream));
    CK(cudaMemcpyAsync(hs.data(), r->halt_step.p, r->halt_step.bytes(), cudaMemcpyDeviceToHost,
                       r->stream));
    CK(cudaStreamSynchronize(r->stream));
    int nbad = 0, first = -1;
    for (int e = 0; e < r->nev; ++e)
      if (fl[e]) {
        if (first < 0) first = e;
        ++nbad;
      }
    if (nbad) {
      r->fwd_saved = false;
      r->adj_done = false;
      return fail(SEM_ERR_NUMERIC,
                  "non-finite wavefield in event %d (%d of %d events) found at step %d of %d "
                  "(sim_type %d, checked every %d steps); those events stopped there",
                  first, nbad, r->nev, hs[first], r->nstep, sim_type, r->cfg.check_every);
    }
  }
  return SEM_OK;
}

int sem_synchronize(sem_run* r) {
  if (!r) return fail(SEM_ERR_ARG, "null run");
  CK(cudaStreamSynchronize(r->stream));
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, r->e0, r->e1) == cudaSuccess) r->last_ms = ms;
  cudaGetLastError();
  return SEM_OK;
}

int sem_get_seismograms(sem_run* r, int ev, float* out) {
  if (!r || !out) return fail(SEM_ERR_ARG, "null argument");
  if (ev < 0 || ev >= r->nev) return fail(SEM_ERR_ARG, "event %d out of range", ev);
  const size_t n = (size_t)r->nrec[ev] * 3 * r->nstep;
  CK(cudaMemcpyAsync(out, r->seis.p + (size_t)ev * r->nrec_max * 3 * r->nstep, n * 4,
                     cudaMemcpyDeviceToHost, r->stream));
  CK(cudaStreamSynchronize(r->stream));
  return SEM_OK;
}

int sem_set_adjoint_sources(sem_run* r, int ev, const double* adj) {
  if (!r || !adj) return fail(SEM_ERR_ARG, "null argument");
  if (ev < 0 || ev >= r->nev) return fail(SEM_ERR_ARG, "event %d out of range", ev);
  const size_t n = (size_t)r->nrec[ev] * 3 * r->nstep;
  std::vector<float> f(n);
  for (size_t i = 0; i < n; ++i) f[i] = (float)adj[i];
  CK(cudaMemcpyAsync(r->adj.p + (size_t)ev * r->nrec_max * 3 * r->nstep, f.data(), n * 4,
                     cudaMemcpyHostToDevice, r->stream));
  CK(cudaStreamSynchronize(r->stream));
  r->have_adj[ev] = 1;
  return SEM_OK;
}

// Taper (src/shared/signal.f90:419-491) and Simpson weights
// (src/shared/utils.f90:1635-1663, as written there) for ns samples of dt.
static void measure_weights(int ns, double dx, double taper_pct, int taper_type, double* w,
                            double* sw) {
  for (int i = 0; i < ns; ++i) w[i] = 1.0;
  const int frac = (taper_pct == 0.0 || taper_pct == 1.0) ? (int)(ns * taper_pct / 2.0)
                                                          : (int)(ns * taper_pct / 2.0 + 0.5);
  if (frac > 0) {
    const double den = 2.0 * frac - 1.0;
    auto tw = [&](double x) {
      switch (taper_type) {
        case 1: return 0.5 - 0.5 * std::cos(2.0 * M_PI * x / den);
        case 2: return 0.54 - 0.46 * std::cos(2.0 * M_PI * x / den);
        case 3: return std::cos(M_PI * x / den - M_PI / 2.0);
        default: return 1.0 - std::pow(std::cos(M_PI * x / den), 10.0);
      }
    };
    for (int i = 0; i < frac; ++i) {
      w[i] *= tw(i);
      w[ns - frac + i] *= tw(frac + i);
    }
  }
  // The even-count branch weights sample n-1 (1-based) by 1 + 2: the
  // initial sum holds y(n-1) and the loop adds 2 y(i+1) up to i+1 = n-1.
  for (int i = 0; i < ns; ++i) sw[i] = 0.0;
  if (ns >= 2) {
    if (ns % 2 == 0) {
      sw[0] += dx / 3.0;
      sw[ns - 2] += dx / 3.0;
      for (int i = 2; i <= ns - 2; i += 2) {  // 1-based loop index
        sw[i - 1] += 4.0 * dx / 3.0;
        sw[i] += 2.0 * dx / 3.0;
      }
      sw[ns - 2] += 0.5 * dx;
      sw[ns - 1] += 0.5 * dx;
    } else {
      sw[0] += dx / 3.0;
      sw[ns - 1] += dx / 3.0;
      for (int i = 2; i <= ns - 1; i += 2) sw[i - 1] += 4.0 * dx / 3.0;
      for (int i = 3; i <= ns - 2; i += 2) sw[i - 1] += 2.0 * dx / 3.0;
    }
  }
}

static int prepare_measure_buffers(sem_run* r) {
  if (!r->taper.p) {
    CKM(r->taper.alloc(r->nstep), "taper");
    CKM(r->simpw.alloc(r->nstep), "simpson weights");
    CKM(r->misfit_rc.alloc((size_t)r->nrec_max * 3), "misfits");
  }
  return SEM_OK;
}

static int prepare_measure(sem_run* r, double taper_pct, int taper_type, int ns) {
  int rc = prepare_measure_buffers(r);
  if (rc) return rc;
  if (taper_pct == r->taper_pct_cached && taper_type == r->taper_type_cached &&
      ns == r->taper_ns_cached)
    return SEM_OK;
  std::vector<double> w(ns), sw(ns);
  measure_weights(ns, r->dt, taper_pct, taper_type, w.data(), sw.data());
  CK(cudaMemcpyAsync(r->taper.p, w.data(), ns * 8, cudaMemcpyHostToDevice, r->stream));
  CK(cudaMemcpyAsync(r->simpw.p, sw.data(), ns * 8, cudaMemcpyHostToDevice, r->stream));
  CK(cudaStreamSynchronize(r->stream));
  r->taper_pct_cached = taper_pct;
  r->taper_type_cached = taper_type;
  r->taper_ns_cached = ns;
  return SEM_OK;
}

int sem_set_observed(sem_run* r, int ev, const double* obs) {
  if (!r || !obs) return fail(SEM_ERR_ARG, "null argument");
  if (ev < 0 || ev >= r->nev) return fail(SEM_ERR_ARG, "event %d out of range", ev);
  const size_t per = (size_t)r->nrec_max * 3 * r->nstep;
  if (!r->obs_ev.p) CKM(r->obs_ev.alloc(per * r->nev), "observed data");
  CK(cudaMemcpyAsync(r->obs_ev.p + per * ev, obs, (size_t)r->nrec[ev] * 3 * r->nstep * 8,
                     cudaMemcpyHostToDevice, r->stream));
  CK(cudaStreamSynchronize(r->stream));
  return SEM_OK;
}

int sem_measure_l2(sem_run* r, int ev, const double* obs, double taper_pct, int taper_type,
                   double* misfit) {
  NvtxPhase ph("sem_measure_l2");
  if (!r) return fail(SEM_ERR_ARG, "null run");
  if (ev < 0 || ev >= r->nev) return fail(SEM_ERR_ARG, "event %d out of range", ev);
  if (!(taper_pct >= 0.0 && taper_pct <= 1.0))
    return fail(SEM_ERR_ARG, "taper_percentage must be in [0, 1]");
  if (taper_type < 1 || taper_type > 4) return fail(SEM_ERR_ARG, "taper type must be 1..4");
  const int ns = r->nstep, nr = r->nrec[ev];
  if (nr == 0) return fail(SEM_ERR_STATE, "event %d has no receivers", ev);
  if (!obs && !r->obs_ev.p) return fail(SEM_ERR_STATE, "no observed data for event %d", ev);
  int rc = prepare_measure(r, taper_pct, taper_type, ns);
  if (rc) return rc;
  const size_t per = (size_t)r->nrec_max * 3 * ns;
  const double* dobs;
  if (obs) {
    if (!r->obs.p) CKM(r->obs.alloc(per), "observed data");
    CK(cudaMemcpyAsync(r->obs.p, obs, (size_t)nr * 3 * ns * 8, cudaMemcpyHostToDevice,
                       r->stream));
    dobs = r->obs.p;
  } else {
    dobs = r->obs_ev.p + per * ev;
  }
  const size_t off = (size_t)ev * per;
  launch_measure_l2(r->seis.p + off, dobs, r->taper.p, r->simpw.p, nr, ns, r->adj.p + off,
                    r->misfit_rc.p, r->stream);
  CK(cudaGetLastError());
  r->have_adj[ev] = 1;
  if (misfit) {
    std::vector<double> m((size_t)nr * 3);
    CK(cudaMemcpyAsync(m.data(), r->misfit_rc.p, m.size() * 8, cudaMemcpyDeviceToHost,
                       r->stream));
    CK(cudaStreamSynchronize(r->stream));
    double total = 0.0;
    for (double v : m) total += v;
    *misfit = total;
  }
  return SEM_OK;
}

int sem_measure_waveform(sem_run* r, int ev, const sem_meas_cfg* cfg, const double* obs,
                         const double* windows, const double* baz, double* misfit_band,
                         double* misfit_trace) {
  NvtxPhase ph("sem_measure_waveform");
  if (!r || !cfg || !obs || !windows) return fail(SEM_ERR_ARG, "null argument");
  if (ev < 0 || ev >= r->nev) return fail(SEM_ERR_ARG, "event %d out of range", ev);
  if (cfg->rotate && !baz) return fail(SEM_ERR_ARG, "rotate needs the back-azimuths");
  const int ns = r->nstep, nr = r->nrec[ev];
  if (nr == 0) return fail(SEM_ERR_STATE, "event %d has no receivers", ev);
  MeasParams p;
  int rc = check_measure_params(cfg, nr, ns, r->dt, windows, &p);
  if (rc) return rc;
  const int nb = p.nband > 0 ? p.nband : 1;
  const size_t n_obs = (size_t)nr * 3 * p.obs_npts, n_win = (size_t)nb * nr * 3 * 2;
  const size_t n_mis = (size_t)nb * nr * 3, n_scr = measure_scratch_doubles(p);
  double* buf = nullptr;
  const size_t total = n_obs + n_win + nr + n_mis + n_scr;
  cudaError_t e = cudaMallocAsync((void**)&buf, total * sizeof(double), r->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(SEM_ERR_NOMEM, "measurement buffers (%zu MB): %s", total * 8 >> 20,
                cudaGetErrorString(e));
  }
  double* d_obs = buf;
  double* d_win = d_obs + n_obs;
  double* d_baz = d_win + n_win;
  double* d_mis = d_baz + nr;
  double* d_scr = d_mis + n_mis;
  std::vector<double> mis(n_mis);
  auto run = [&]() -> cudaError_t {
    cudaError_t err = cudaMemcpyAsync(d_obs, obs, n_obs * 8, cudaMemcpyHostToDevice, r->stream);
    if (err == cudaSuccess)
      err = cudaMemcpyAsync(d_win, windows, n_win * 8, cudaMemcpyHostToDevice, r->stream);
    if (err == cudaSuccess && baz)
      err = cudaMemcpyAsync(d_baz, baz, (size_t)nr * 8, cudaMemcpyHostToDevice, r->stream);
    if (err != cudaSuccess) return err;
    const size_t per = (size_t)r->nrec_max * 3 * ns;
    launch_measure_waveform(p, r->seis.p + per * ev, d_obs, d_win, d_baz, d_scr,
                            r->adj.p + per * ev, d_mis, r->stream);
    err = cudaGetLastError();
    if (err == cudaSuccess)
      err = cudaMemcpyAsync(mis.data(), d_mis, n_mis * 8, cudaMemcpyDeviceToHost, r->stream);
    return err;
  };
  e = run();
  cudaFreeAsync(buf, r->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(SEM_ERR_CUDA, "waveform measurement: %s", cudaGetErrorString(e));
  }
  r->have_adj[ev] = 1;
  if (misfit_band)
    for (int b = 0; b < nb; ++b) {
      double t = 0.0;
      for (int q = 0; q < nr * 3; ++q) t += mis[(size_t)b * nr * 3 + q];
      misfit_band[b] = t;
    }
  if (misfit_trace) std::copy(mis.begin(), mis.end(), misfit_trace);
  return SEM_OK;
}

int sem_save_adjoint_kernels(sem_run* r, int ev, double* out) {
  if (!r || !out) return fail(SEM_ERR_ARG, "null argument");
  if (ev < 0 || ev >= r->nev) return fail(SEM_ERR_ARG, "event %d out of range", ev);
  if (!r->adj_done) return fail(SEM_ERR_STATE, "no adjoint run has completed");
  const size_t ne = (size_t)r->mesh->nspec * NGLL3;
  if (!r->kout.p) CKM(r->kout.alloc(6 * ne), "kernel output");
  launch_finalize_kernels(r->mesh->view(), r->mesh->rho.p, {r->k_rho.p, r->k_mu.p, r->k_kappa.p},
                          r->lm, ev, r->kout.p, nullptr, r->stream);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, r->kout.p, 6 * ne * 8, cudaMemcpyDeviceToHost, r->stream));
  CK(cudaStreamSynchronize(r->stream));
  return SEM_OK;
}

int sem_sum_kernels(sem_run* r, double* out) {
  NvtxPhase ph("sem_sum_kernels");
  if (!r || !out) return fail(SEM_ERR_ARG, "null argument");
  if (!r->adj_done) return fail(SEM_ERR_STATE, "no adjoint run has completed");
  const size_t ne = (size_t)r->mesh->nspec * NGLL3;
  if (!r->ksum.p) CKM(r->ksum.alloc(6 * ne), "kernel sum");
  CK(cudaMemsetAsync(r->ksum.p, 0, r->ksum.bytes(), r->stream));
  for (int e = 0; e < r->nev; ++e)
    launch_finalize_kernels(r->mesh->view(), r->mesh->rho.p,
                            {r->k_rho.p, r->k_mu.p, r->k_kappa.p}, r->lm, e, nullptr,
                            r->ksum.p, r->stream);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, r->ksum.p, 6 * ne * 8, cudaMemcpyDeviceToHost, r->stream));
  CK(cudaStreamSynchronize(r->stream));
  return SEM_OK;
}

int sem_sum_kernels_device(sem_run* r, double* dev_out) {
  NvtxPhase ph("sem_sum_kernels_device");
  if (!r || !dev_out) return fail(SEM_ERR_ARG, "null argument");
  if (!r->adj_done) return fail(SEM_ERR_STATE, "no adjoint run has completed");
  const size_t ne = (size_t)r->mesh->nspec * NGLL3;
  CK(cudaMemsetAsync(dev_out, 0, 6 * ne * 8, r->stream));
  for (int e = 0; e < r->nev; ++e)
    launch_finalize_kernels(r->mesh->view(), r->mesh->rho.p,
                            {r->k_rho.p, r->k_mu.p, r->k_kappa.p}, r->lm, e, nullptr, dev_out,
                            r->stream);
  CK(cudaGetLastError());
  return SEM_OK;
}

// A captured step graph holds the kernel instantiations and the step
// arguments of its capture (the Hessian update and accumulator, the
// injecting Stacey kernel); a switch that changes them drops the graphs,
// and the next run of each phase captures its graph again.
static int drop_graphs(sem_run* r) {
  if (!r->gexec[0] && !r->gexec[1]) return SEM_OK;
  CK(cudaStreamSynchronize(r->stream));
  for (auto& g : r->gexec)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  return SEM_OK;
}

static bool any_injection(const sem_run* r) {
  for (const auto& j : r->inj)
    if (j.buf) return true;
  return false;
}

int sem_set_approximate_hessian(sem_run* r, int enable) {
  if (!r) return fail(SEM_ERR_ARG, "null run");
  const bool was = r->hess_on;
  r->hess_on = enable != 0;
  if (r->hess_on && r->k_rho.p) {
    // adjoint buffers exist already (an earlier adjoint run or lane start)
    int rc = ensure_adjoint_buffers(r);
    if (rc) return rc;
  }
  return was != r->hess_on ? drop_graphs(r) : SEM_OK;
}

int sem_save_hessian_kernel(sem_run* r, int ev, double* out) {
  if (!r || !out) return fail(SEM_ERR_ARG, "null argument");
  if (ev < 0 || ev >= r->nev) return fail(SEM_ERR_ARG, "event %d out of range", ev);
  if (!r->adj_done || !r->hess_done)
    return fail(SEM_ERR_STATE, "no adjoint run with the approximate Hessian has completed");
  const size_t ne = (size_t)r->mesh->nspec * NGLL3;
  if (!r->kout.p) CKM(r->kout.alloc(6 * ne), "kernel output");
  launch_finalize_hessian(r->mesh->view(), r->k_hess.p, r->lm, ev, r->kout.p, nullptr, 0,
                          r->stream);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, r->kout.p, ne * 8, cudaMemcpyDeviceToHost, r->stream));
  CK(cudaStreamSynchronize(r->stream));
  return SEM_OK;
}

int sem_sum_hessian(sem_run* r, int abs_each, double* out) {
  if (!r || !out) return fail(SEM_ERR_ARG, "null argument");
  if (!r->adj_done || !r->hess_done)
    return fail(SEM_ERR_STATE, "no adjoint run with the approximate Hessian has completed");
  const size_t ne = (size_t)r->mesh->nspec * NGLL3;
  if (!r->ksum.p) CKM(r->ksum.alloc(6 * ne), "kernel sum");
  CK(cudaMemsetAsync(r->ksum.p, 0, ne * 8, r->stream));
  for (int e = 0; e < r->nev; ++e)
    launch_finalize_hessian(r->mesh->view(), r->k_hess.p, r->lm, e, nullptr, r->ksum.p,
                            abs_each != 0, r->stream);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, r->ksum.p, ne * 8, cudaMemcpyDeviceToHost, r->stream));
  CK(cudaStreamSynchronize(r->stream));
  return SEM_OK;
}

int sem_set_injection(sem_run* r, int ev, const float* veloc, const float* tract, int nt,
                      int np_resamp, int k0) {
  if (!r) return fail(SEM_ERR_ARG, "null run");
  if (ev < 0 || ev >= r->nev) return fail(SEM_ERR_ARG, "event %d out of range", ev);
  if (r->lanes_mode) return fail(SEM_ERR_STATE, "run is driven lane by lane (sem_lane_*)");
  auto& j = r->inj[ev];
  const bool before = any_injection(r);
  if (!veloc) {
    if (j.buf) {
      CK(cudaStreamSynchronize(r->stream));
      cudaFree(j.buf);
    }
    j = sem_run_s::Injection{};
    return before != any_injection(r) ? drop_graphs(r) : SEM_OK;
  }
  if (!tract) return fail(SEM_ERR_ARG, "null traction");
  if (r->mesh->nf == 0) return fail(SEM_ERR_STATE, "the mesh has no absorbing faces");
  if (nt < 1 || np_resamp < 1) return fail(SEM_ERR_ARG, "nt and np_resamp must be >= 1");
  const size_t npt3 = (size_t)r->mesh->nf * 25 * 3;
  const size_t n = (size_t)nt * npt3;
  for (const float* a : {veloc, tract})
    for (size_t i = 0; i < n; ++i)
      if (!std::isfinite(a[i])) return fail(SEM_ERR_ARG, "non-finite injected value at %zu", i);
  if (j.buf && j.nt != nt) {
    CK(cudaStreamSynchronize(r->stream));
    cudaFree(j.buf);
    j.buf = nullptr;
  }
  if (!j.buf) {
    cudaError_t e = cudaMalloc((void**)&j.buf, 2 * n * sizeof(float));
    if (e != cudaSuccess) {
      cudaGetLastError();
      j.buf = nullptr;
      return fail(SEM_ERR_NOMEM, "device allocation of the injected field failed: %s",
                  cudaGetErrorString(e));
    }
  }
  j.nt = nt;
  j.np = np_resamp;
  j.k0 = k0;
  CK(cudaMemcpyAsync(j.buf, veloc, n * 4, cudaMemcpyHostToDevice, r->stream));
  CK(cudaMemcpyAsync(j.buf + n, tract, n * 4, cudaMemcpyHostToDevice, r->stream));
  CK(cudaStreamSynchronize(r->stream));
  return before ? SEM_OK : drop_graphs(r);
}

int sem_set_stream(sem_run* r, void* stream) {
  if (!r) return fail(SEM_ERR_ARG, "null run");
  CK(cudaStreamSynchronize(r->stream));
  r->stream = stream ? (cudaStream_t)stream : r->own_stream;
  return SEM_OK;
}

int sem_mark(sem_run* r, long long* token) {
  if (!r || !token) return fail(SEM_ERR_ARG, "null argument");
  const int slot = (int)(r->mark_next % sem_run_s::kMarks);
  if (!r->mark_ev[slot]) CK(cudaEventCreate(&r->mark_ev[slot]));
  CK(cudaEventRecord(r->mark_ev[slot], r->stream));
  *token = r->mark_next++;
  return SEM_OK;
}

// A mark whose slot has been recorded again is older than every mark in
// flight; the stream runs in order, so it has completed.
static bool mark_recycled(const sem_run* r, long long token) {
  return token < r->mark_next - sem_run_s::kMarks;
}

int sem_mark_done(sem_run* r, long long token, int wait) {
  if (!r || token < 0 || token >= r->mark_next) return fail(SEM_ERR_ARG, "unknown mark %lld", token);
  if (mark_recycled(r, token)) return 1;
  cudaEvent_t e = r->mark_ev[token % sem_run_s::kMarks];
  if (wait) {
    CK(cudaEventSynchronize(e));
    return 1;
  }
  const cudaError_t q = cudaEventQuery(e);
  if (q == cudaSuccess) return 1;
  if (q == cudaErrorNotReady) {
    cudaGetLastError();
    return 0;
  }
  return fail(SEM_ERR_CUDA, "mark %lld: %s", token, cudaGetErrorString(q));
}

int sem_mark_elapsed(sem_run* r, long long t0, long long t1, double* ms) {
  if (!r || !ms) return fail(SEM_ERR_ARG, "null argument");
  if (t0 < 0 || t1 < t0 || t1 >= r->mark_next || mark_recycled(r, t0))
    return fail(SEM_ERR_ARG, "marks %lld..%lld are not both in the ring", t0, t1);
  float f = 0.f;
  CK(cudaEventElapsedTime(&f, r->mark_ev[t0 % sem_run_s::kMarks],
                          r->mark_ev[t1 % sem_run_s::kMarks]));
  *ms = f;
  return SEM_OK;
}

int sem_set_store_spill(sem_run* r, long long device_store_bytes) {
  if (!r) return fail(SEM_ERR_ARG, "null run");
  if (r->lanes_mode)
    return fail(SEM_ERR_STATE, "lane-driven runs keep their boundary stores resident");
  if (device_store_bytes == r->spill_budget) return SEM_OK;
  CK(cudaStreamSynchronize(r->stream));
  release_ring(r);
  r->store.reset();
  r->scale.reset();
  r->spill_budget = device_store_bytes;
  r->fwd_saved = false;  // a saved store of the old layout is gone
  return SEM_OK;
}

int sem_store_info(sem_run* r, int* chunk_steps, int* device_slots, int* chunks,
                   long long* device_bytes, long long* host_bytes) {
  if (!r) return fail(SEM_ERR_ARG, "null run");
  const size_t dev = r->store.bytes() + r->scale.bytes();
  const size_t host = r->h_spill_bytes + (r->h_spill_scale ? r->chunk_scale_floats() * 4 *
                                                                 (r->ring_n - r->ring_d) : 0);
  if (chunk_steps) *chunk_steps = r->ring_c;
  if (device_slots) *device_slots = r->ring_d;
  if (chunks) *chunks = r->ring_n;
  if (device_bytes) *device_bytes = (long long)dev;
  if (host_bytes) *host_bytes = (long long)host;
  return SEM_OK;
}

int sem_set_sm_share(sem_run* r, int sm_limit, int high_priority) {
  if (!r || sm_limit < 0) return fail(SEM_ERR_ARG, "bad argument");
  r->sm_limit = sm_limit;
  if (r->stream != r->own_stream) return SEM_OK;  // a caller's stream keeps its priority
  int lo = 0, hi = 0;
  CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
  int cur = 0;
  CK(cudaStreamGetPriority(r->own_stream, &cur));
  const int want = high_priority ? hi : lo;
  if (cur == want) return SEM_OK;
  cudaStream_t s2 = nullptr;
  CK(cudaStreamCreateWithPriority(&s2, cudaStreamNonBlocking, want));
  // the new stream starts after everything queued on the old one
  cudaEvent_t e = nullptr;
  CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  CK(cudaEventRecord(e, r->own_stream));
  CK(cudaStreamWaitEvent(s2, e, 0));
  CK(cudaEventDestroy(e));
  CK(cudaStreamSynchronize(r->own_stream));
  CK(cudaStreamDestroy(r->own_stream));
  r->own_stream = s2;
  r->stream = s2;
  return SEM_OK;
}

int sem_time_kernels(sem_run* r, int sim_type, int nsteps, double* ms4) {
  if (!r || !ms4) return fail(SEM_ERR_ARG, "null argument");
  if (sim_type != 1 && sim_type != 3) return fail(SEM_ERR_ARG, "sim_type must be 1 or 3");
  if (nsteps < 1 || nsteps >= r->nstep) return fail(SEM_ERR_ARG, "nsteps must be in [1, nstep)");
  const bool adj = sim_type == 3;
  if (adj && (!r->u2.p || !r->k_rho.p))
    return fail(SEM_ERR_STATE, "sim_type 3 timing needs a completed adjoint run");
  if (!adj && !r->have_src[0]) return fail(SEM_ERR_STATE, "sources not set");
  if (r->mesh->nf > 0 && !r->store.p) {
    int rc = ensure_store(r);
    if (rc) return rc;
  }
  // lanes at step 1 so that every kernel does its full work (backward
  // scatter, store replay and source are skipped at step 0)
  r->fill_lanes(adj ? PH_ADJ : PH_FWD, adj ? 0 : 1);
  for (auto& L : r->h_lanes) L.it0 = 1;
  CK(cudaMemcpyAsync(r->lanes.p, r->h_lanes.data(), r->lanes.bytes(), cudaMemcpyHostToDevice,
                     r->stream));
  std::vector<cudaEvent_t> ev(5 * nsteps);
  for (auto& e : ev) CK(cudaEventCreate(&e));
  StepArgs a = r->args(adj);
  for (int s = 0; s < nsteps; ++s) {
    a.s = s;
    cudaEvent_t* E = &ev[5 * s];
    CK(cudaEventRecord(E[0], r->stream));
    launch_forces(a, adj, r->stream);
    CK(cudaEventRecord(E[1], r->stream));
    launch_boundary(a, adj, r->stream);
    CK(cudaEventRecord(E[2], r->stream));
    launch_points(a, r->stream);
    CK(cudaEventRecord(E[3], r->stream));
    launch_update(a, adj, r->stream);
    CK(cudaEventRecord(E[4], r->stream));
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(r->stream));
  double acc[4] = {0, 0, 0, 0};
  for (int s = 0; s < nsteps; ++s)
    for (int k = 0; k < 4; ++k) {
      float f = 0.f;
      CK(cudaEventElapsedTime(&f, ev[5 * s + k], ev[5 * s + k + 1]));
      acc[k] += f;
    }
  for (auto& e : ev) cudaEventDestroy(e);
  for (int k = 0; k < 4; ++k) ms4[k] = acc[k] / nsteps;
  return SEM_OK;
}

// ----------------------------------------------------------------------------
// serving primitives: one event per lane, lanes advance independently
// ----------------------------------------------------------------------------

// Event marking that a lane's queued results (async finish, misfit) have
// landed.
static int lane_result_event(sem_run* r, int lane, cudaEvent_t* out) {
  if (r->lane_res_ev.empty()) r->lane_res_ev.assign(r->nev, nullptr);
  if (!r->lane_res_ev[lane])
    CK(cudaEventCreateWithFlags(&r->lane_res_ev[lane], cudaEventDisableTiming));
  *out = r->lane_res_ev[lane];
  return SEM_OK;
}

// Pinned staging area of a lane, at least `bytes`, once the lane's earlier
// staged copies have left it.
static int lane_stage(sem_run* r, int lane, size_t bytes, unsigned char** out) {
  if (r->h_lane_stage.empty()) {
    r->h_lane_stage.assign(r->nev, nullptr);
    r->lane_ev.assign(r->nev, nullptr);
  }
  if (!r->lane_ev[lane])
    CK(cudaEventCreateWithFlags(&r->lane_ev[lane], cudaEventDisableTiming));
  else
    CK(cudaEventSynchronize(r->lane_ev[lane]));
  // every lane's area has the largest size any lane needs
  const size_t need = std::max(bytes, r->lane_stage_bytes);
  if (need > r->lane_stage_bytes) {
    for (int l = 0; l < r->nev; ++l)
      if (r->h_lane_stage[l]) {
        if (r->lane_ev[l]) CK(cudaEventSynchronize(r->lane_ev[l]));
        cudaFreeHost(r->h_lane_stage[l]);
        r->h_lane_stage[l] = nullptr;
      }
    r->lane_stage_bytes = need;
  }
  if (!r->h_lane_stage[lane])
    CK(cudaMallocHost((void**)&r->h_lane_stage[lane], r->lane_stage_bytes));
  *out = r->h_lane_stage[lane];
  return SEM_OK;
}

static void lane_defaults(sem_run* r, int e) {
  const size_t ns = (size_t)r->nstep;  // per-lane regions are sized for the run's nstep
  LaneDesc& L = r->h_lanes[e];
  L.stf = r->stf.p + (size_t)e * ns;
  L.srcarr = r->srcarr.p + (size_t)e * 375;
  L.rec_ispec = r->rec_ispec.p + (size_t)e * r->nrec_max;
  L.rec_w = r->rec_w.p + (size_t)e * r->nrec_max * 125;
  L.seis = r->seis.p + (size_t)e * r->nrec_max * 3 * ns;
  L.adj = r->adj.p + (size_t)e * r->nrec_max * 3 * ns;
}

static int enter_lanes_mode(sem_run* r) {
  if (r->lanes_mode) return SEM_OK;
  int rc = ensure_tuned(r);
  if (rc) return rc;
  rc = ensure_adjoint_buffers(r);
  if (rc) return rc;
  const size_t n3 = (size_t)r->mesh->nglob * 3 * r->nevp;
  CK(cudaMemsetAsync(r->u1.p, 0, n3 * 4, r->stream));
  CK(cudaMemsetAsync(r->v1.p, 0, n3 * 4, r->stream));
  CK(cudaMemsetAsync(r->a1.p, 0, n3 * 4, r->stream));
  CK(cudaMemsetAsync(r->u2.p, 0, n3 * 4, r->stream));
  CK(cudaMemsetAsync(r->v2.p, 0, n3 * 4, r->stream));
  CK(cudaMemsetAsync(r->a2.p, 0, n3 * 4, r->stream));
  r->h_lanes.assign(r->nev, LaneDesc{});
  for (int e = 0; e < r->nev; ++e) {
    r->h_lanes[e].phase = PH_IDLE;
    lane_defaults(r, e);
  }
  r->lane_store.assign(r->nev, nullptr);
  r->lane_scale.assign(r->nev, nullptr);
  r->lane_saved.assign(r->nev, 0);
  if (r->variant[0] < 0) r->variant[0] = 2;
  if (r->variant[1] < 0) r->variant[1] = 2;
  r->lanes_mode = true;
  return SEM_OK;
}

static size_t lane_store_bytes(const sem_run* r, int nstep) {
  const size_t per = (size_t)nstep * r->mesh->nf * 75 * r->store_elem();
  return per + (r->cfg.store_kind == SEM_STORE_FP16 ? (size_t)nstep * r->mesh->nf * 4 : 0);
}

long long sem_lane_store_bytes(const sem_run* r, int nstep) {
  if (!r || nstep < 1) return -1;
  return (long long)lane_store_bytes(r, nstep);
}

int sem_lane_start_forward(sem_run* r, int lane, const sem_source* src, int nrec,
                           const double* xyz, int nstep, int save_forward) {
  if (!r || !src) return fail(SEM_ERR_ARG, "null argument");
  if (lane < 0 || lane >= r->nev) return fail(SEM_ERR_ARG, "lane %d out of range", lane);
  if (nstep < 1 || nstep > r->nstep)
    return fail(SEM_ERR_ARG, "nstep %d outside [1, run nstep %d]", nstep, r->nstep);
  int rc = enter_lanes_mode(r);
  if (rc) return rc;
  if (r->h_lanes[lane].phase != PH_IDLE) return fail(SEM_ERR_STATE, "lane %d is busy", lane);
  // source and receivers of this lane (same set-up as sem_set_sources for
  // one event; the time function covers the lane's own nstep)
  const sem_source& s = *src;
  if (!(s.f0 > 0.0) || !std::isfinite(s.x + s.y + s.z))
    return fail(SEM_ERR_ARG, "invalid source position or f0");
  double xi3[3];
  r->src_ispec[lane] = r->mesh->locate(s.x, s.y, s.z, xi3);
  const double Mzz = s.Mrr, Myy = s.Mtt, Mxx = s.Mpp;
  const double Myz = -s.Mrt, Mxz = s.Mrp, Mxy = -s.Mtp;
  const double M[3][3] = {{Mxx, Mxy, Mxz}, {Mxy, Myy, Myz}, {Mxz, Myz, Mzz}};
  double hx[5], hxd[5], hy[5], hyd[5], hz[5], hzd[5];
  lagrange_all(xi3[0], hx, hxd);
  lagrange_all(xi3[1], hy, hyd);
  lagrange_all(xi3[2], hz, hzd);
  double B[3][3];
  r->mesh->dxi_dx(r->src_ispec[lane], xi3, B);
  if (nrec < 0 || nrec > r->nrec_max || (!xyz && nrec > 0))
    return fail(SEM_ERR_ARG, "nrec %d outside [0, max_receivers=%d]", nrec, r->nrec_max);
  // source array, time function and receivers staged in pinned memory, so
  // that the lane starts without waiting for the work queued on the run
  const size_t nr = r->nrec_max;
  unsigned char* stage = nullptr;
  rc = lane_stage(r, lane, (375 + (size_t)r->nstep + nr * 125) * 4 + nr * 4, &stage);
  if (rc) return rc;
  float* sa = (float*)stage;
  float* stf = sa + 375;
  float* rw = stf + r->nstep;
  int* isp = (int*)(rw + nr * 125);
  for (int c = 0; c < 5; ++c)
    for (int b = 0; b < 5; ++b)
      for (int a = 0; a < 5; ++a) {
        const double dr[3] = {hxd[a] * hy[b] * hz[c], hx[a] * hyd[b] * hz[c],
                              hx[a] * hy[b] * hzd[c]};
        double gr[3];
        for (int k = 0; k < 3; ++k) gr[k] = B[0][k] * dr[0] + B[1][k] * dr[1] + B[2][k] * dr[2];
        const int p = a + 5 * b + 25 * c;
        for (int k = 0; k < 3; ++k)
          sa[p * 3 + k] = (float)(M[k][0] * gr[0] + M[k][1] * gr[1] + M[k][2] * gr[2]);
      }
  const double t0 = 1.2 / s.f0 + s.tshift;
  for (int it = 0; it < nstep; ++it) stf[it] = (float)ricker((double)it * r->dt - t0, s.f0);
  rc = receivers_host(r, nrec, xyz, isp, rw);
  if (rc) return rc;
  CK(cudaMemcpyAsync(r->srcarr.p + (size_t)lane * 375, sa, 375 * 4, cudaMemcpyHostToDevice,
                     r->stream));
  CK(cudaMemcpyAsync(r->stf.p + (size_t)lane * r->nstep, stf, (size_t)nstep * 4,
                     cudaMemcpyHostToDevice, r->stream));
  CK(cudaMemcpyAsync(r->rec_ispec.p + (size_t)lane * nr, isp, nr * sizeof(int),
                     cudaMemcpyHostToDevice, r->stream));
  CK(cudaMemcpyAsync(r->rec_w.p + (size_t)lane * nr * 125, rw, nr * 125 * sizeof(float),
                     cudaMemcpyHostToDevice, r->stream));
  CK(cudaEventRecord(r->lane_ev[lane], r->stream));
  r->have_src[lane] = 1;
  r->nrec[lane] = nrec;
  r->have_rec[lane] = 1;
  // boundary store for the later adjoint run
  if (r->lane_store[lane]) {
    CK(cudaFreeAsync(r->lane_store[lane], r->stream));
    r->lane_store[lane] = nullptr;
  }
  if (r->lane_scale[lane]) {
    CK(cudaFreeAsync(r->lane_scale[lane], r->stream));
    r->lane_scale[lane] = nullptr;
  }
  if (save_forward && r->mesh->nf > 0) {
    cudaError_t e = cudaMallocAsync(&r->lane_store[lane],
                                    (size_t)nstep * r->mesh->nf * 75 * r->store_elem(), r->stream);
    if (e == cudaSuccess && r->cfg.store_kind == SEM_STORE_FP16)
      e = cudaMallocAsync((void**)&r->lane_scale[lane], (size_t)nstep * r->mesh->nf * 4,
                          r->stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(SEM_ERR_NOMEM, "boundary store of lane %d (%d steps): %s", lane, nstep,
                  cudaGetErrorString(e));
    }
  }
  launch_lane_zero({r->u1.p, r->v1.p, r->a1.p}, r->mesh->nglob, r->lm, lane, r->stream);
  CK(cudaGetLastError());
  if (r->cfg.check_every > 0) {
    rc = ensure_check_buffers(r);
    if (rc) return rc;
    CK(cudaMemsetAsync(r->lflags.p + lane, 0, sizeof(int), r->stream));
    CK(cudaMemsetAsync(r->halt_step.p + lane, 0xff, sizeof(int), r->stream));
    r->lane_failed[lane] = 0;
    r->lane_fail_step[lane] = -1;
  }
  LaneDesc& L = r->h_lanes[lane];
  lane_defaults(r, lane);
  L.phase = PH_FWD;
  L.it0 = 0;
  L.nstep = nstep;
  L.save = save_forward ? 1 : 0;
  L.src_ispec = r->src_ispec[lane];
  L.nrec = nrec;
  L.store = r->lane_store[lane];
  L.scale = r->lane_scale[lane];
  r->lane_saved[lane] = 0;
  return SEM_OK;
}

int sem_lane_start_adjoint(sem_run* r, int lane, const double* obs, double taper_pct,
                           int taper_type, double* misfit) {
  if (!r || !obs) return fail(SEM_ERR_ARG, "null argument");
  if (!r->lanes_mode || lane < 0 || lane >= r->nev)
    return fail(SEM_ERR_ARG, "lane %d is not a serving lane", lane);
  LaneDesc& L = r->h_lanes[lane];
  if (L.phase != PH_FWD || L.it0 < L.nstep || !L.save)
    return fail(SEM_ERR_STATE, "lane %d has no completed forward run with a saved store", lane);
  if (!(taper_pct >= 0.0 && taper_pct <= 1.0) || taper_type < 1 || taper_type > 4)
    return fail(SEM_ERR_ARG, "invalid taper");
  const int ns = L.nstep, nr = L.nrec;
  int rc = prepare_measure_buffers(r);
  if (rc) return rc;
  if (!r->obs.p) CKM(r->obs.alloc((size_t)r->nrec_max * 3 * r->nstep), "observed data");
  if (!r->lane_misfit.p) CKM(r->lane_misfit.alloc((size_t)r->nev), "lane misfits");
  // observed data and this record's weights staged in pinned memory, so
  // that the switch does not wait for the work queued on the run; the
  // device buffers are shared, and every use is stream-ordered
  unsigned char* stage = nullptr;
  rc = lane_stage(r, lane, ((size_t)nr * 3 * ns + 2 * (size_t)ns) * 8, &stage);
  if (rc) return rc;
  double* hobs = (double*)stage;
  double* hw = hobs + (size_t)nr * 3 * ns;
  double* hsw = hw + ns;
  std::memcpy(hobs, obs, (size_t)nr * 3 * ns * 8);
  measure_weights(ns, r->dt, taper_pct, taper_type, hw, hsw);
  CK(cudaMemcpyAsync(r->obs.p, hobs, (size_t)nr * 3 * ns * 8, cudaMemcpyHostToDevice,
                     r->stream));
  CK(cudaMemcpyAsync(r->taper.p, hw, (size_t)ns * 8, cudaMemcpyHostToDevice, r->stream));
  CK(cudaMemcpyAsync(r->simpw.p, hsw, (size_t)ns * 8, cudaMemcpyHostToDevice, r->stream));
  CK(cudaEventRecord(r->lane_ev[lane], r->stream));
  r->taper_ns_cached = -1;  // the shared weights now hold this record's
  launch_measure_l2(L.seis, r->obs.p, r->taper.p, r->simpw.p, nr, ns, (float*)L.adj,
                    r->misfit_rc.p, r->stream);
  launch_sum_series(r->misfit_rc.p, 3 * nr, r->lane_misfit.p + lane, r->stream);
  // backward field starts from this lane's final forward state
  const Fields f1{r->u1.p, r->v1.p, r->a1.p}, f2{r->u2.p, r->v2.p, r->a2.p};
  launch_lane_copy(f1, f2, r->mesh->nglob, r->lm, lane, r->stream);
  launch_lane_zero(f1, r->mesh->nglob, r->lm, lane, r->stream);
  launch_lane_zero_acc({r->k_rho.p, r->k_mu.p, r->k_kappa.p, r->hess_on ? r->k_hess.p : nullptr},
                       r->mesh->nglob,
                       (size_t)r->mesh->nspec * NGLL3, r->lm, lane, r->stream);
  CK(cudaGetLastError());
  if (misfit) {
    CK(cudaMemcpyAsync(misfit, r->lane_misfit.p + lane, sizeof(double), cudaMemcpyDeviceToHost,
                       r->stream));
    CK(cudaStreamSynchronize(r->stream));
  }
  L.phase = PH_ADJ;
  L.it0 = 0;
  L.save = 0;
  return SEM_OK;
}

int sem_lane_misfit(sem_run* r, int lane, double* misfit) {
  if (!r || !misfit || !r->lanes_mode || lane < 0 || lane >= r->nev)
    return fail(SEM_ERR_ARG, "lane %d is not a serving lane", lane);
  if (!r->lane_misfit.p) return fail(SEM_ERR_STATE, "no lane has been measured");
  cudaEvent_t done = nullptr;
  int rc = lane_result_event(r, lane, &done);
  if (rc) return rc;
  CK(cudaMemcpyAsync(misfit, r->lane_misfit.p + lane, sizeof(double), cudaMemcpyDeviceToHost,
                     r->stream));
  CK(cudaEventRecord(done, r->stream));
  return SEM_OK;
}

// Lane-driven runs: take in the flags of the last stability check once its
// copy has landed (without waiting).  A flagged running lane is marked
// failed and complete, so no further launch works it; sem_lane_status and
// sem_lane_finish report it.
static void consume_check(sem_run* r) {
  if (!r->check_pending || cudaEventQuery(r->check_ev) != cudaSuccess) {
    cudaGetLastError();  // cudaErrorNotReady is not an error here
    return;
  }
  r->check_pending = false;
  for (int l = 0; l < r->nev; ++l) {
    LaneDesc& L = r->h_lanes[l];
    if (r->h_lflags[l] && !r->lane_failed[l] && L.phase != PH_IDLE) {
      r->lane_failed[l] = 1;
      r->lane_fail_step[l] = r->h_halt[l];
      L.it0 = L.nstep;
    }
  }
}

int sem_advance(sem_run* r, int nsteps) {
  NvtxPhase ph("sem_advance");
  if (!r || nsteps < 1) return fail(SEM_ERR_ARG, "bad argument");
  if (!r->lanes_mode) return fail(SEM_ERR_STATE, "no lane has been started");
  if (r->cfg.check_every > 0) consume_check(r);
  // 8-lane groups with running events, split by phase: a group with any
  // adjoint lane goes to the two-field kernels, an all-forward group to the
  // one-field kernels
  const int lw = 1 << r->lm.lwlog;
  const int ngr = r->nevp / lw;
  std::vector<int> has(ngr, 0);
  bool any = false;
  for (int e = 0; e < r->nev; ++e) {
    const LaneDesc& L = r->h_lanes[e];
    if (L.phase != PH_IDLE && L.it0 < L.nstep) {
      any = true;
      has[e / lw] |= (L.phase == PH_ADJ) ? 2 : 1;
    }
  }
  if (!any) return SEM_OK;
  std::vector<int> gmap;  // [fwd groups..., adj groups...]
  for (int g = 0; g < ngr; ++g)
    if (has[g] == 1) gmap.push_back(g);
  const int nf = (int)gmap.size();
  for (int g = 0; g < ngr; ++g)
    if (has[g] & 2) gmap.push_back(g);
  const int na = (int)gmap.size() - nf;
  if (!r->gmap.p) CKM(r->gmap.alloc((size_t)std::max(1, ngr)), "group map");
  // lane table and group map through a ring of pinned slots, so that the
  // launches queue behind the work in flight instead of waiting for it
  if (!r->h_stage_tab) {
    r->stage_tab_bytes = r->lanes.bytes() + (size_t)std::max(1, ngr) * sizeof(int);
    CK(cudaMallocHost((void**)&r->h_stage_tab, r->stage_tab_bytes * sem_run_s::kStage));
    for (auto& e : r->stage_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  {
    const int slot = (int)(r->stage_next++ % sem_run_s::kStage);
    CK(cudaEventSynchronize(r->stage_ev[slot]));
    unsigned char* tab = r->h_stage_tab + (size_t)slot * r->stage_tab_bytes;
    std::memcpy(tab, r->h_lanes.data(), r->lanes.bytes());
    std::memcpy(tab + r->lanes.bytes(), gmap.data(), gmap.size() * sizeof(int));
    CK(cudaMemcpyAsync(r->lanes.p, tab, r->lanes.bytes(), cudaMemcpyHostToDevice, r->stream));
    CK(cudaMemcpyAsync(r->gmap.p, tab + r->lanes.bytes(), gmap.size() * sizeof(int),
                       cudaMemcpyHostToDevice, r->stream));
    CK(cudaEventRecord(r->stage_ev[slot], r->stream));
  }
  StepArgs af = r->args(false), aa = r->args(true), ab = r->args(na > 0);
  if (lw > 1) {
    af.gmap = r->gmap.p;
    af.ngmap = nf;
    aa.gmap = r->gmap.p + nf;
    aa.ngmap = na;
    // the persistent element kernels are the ones that walk a group map
    if (af.variant < 2) af.variant = 2;
    if (aa.variant < 2) aa.variant = 2;
  }
  long long launches = 0;
  for (int s = 0; s < nsteps; ++s) {
    af.s = aa.s = ab.s = s;
    if (lw == 1) {
      launches += launch_forces(ab, na > 0, r->stream);
    } else {
      if (nf) launches += launch_forces(af, false, r->stream);
      if (na) launches += launch_forces(aa, true, r->stream);
    }
    launches += launch_boundary(ab, na > 0, r->stream);
    launches += launch_points(ab, r->stream);
    if (lw == 1) {
      launches += launch_update(ab, na > 0, r->stream);
    } else {
      if (nf) launches += launch_update(af, false, r->stream);
      if (na) launches += launch_update(aa, true, r->stream);
    }
  }
  CK(cudaGetLastError());
  if (r->cfg.check_every > 0) {
    r->steps_since_check += nsteps;
    // one check in flight at a time; a due check waits for the previous one
    if (r->steps_since_check >= r->cfg.check_every && !r->check_pending) {
      queue_check(r, true, nsteps);
      launches += 3;
      CK(cudaMemcpyAsync(r->h_lflags, r->lflags.p, r->lflags.bytes(), cudaMemcpyDeviceToHost,
                         r->stream));
      CK(cudaMemcpyAsync(r->h_halt, r->halt_step.p, r->halt_step.bytes(),
                         cudaMemcpyDeviceToHost, r->stream));
      CK(cudaEventRecord(r->check_ev, r->stream));
      r->check_pending = true;
      r->steps_since_check = 0;
    }
  }
  for (auto& L : r->h_lanes)
    if (L.phase != PH_IDLE) L.it0 = std::min(L.nstep, L.it0 + nsteps);
  r->last_launches = launches;
  return SEM_OK;
}

int sem_lane_status(sem_run* r, int lane, int* phase, int* step, int* nstep) {
  if (!r || lane < 0 || lane >= r->nev) return fail(SEM_ERR_ARG, "bad lane");
  if (!r->lanes_mode) {
    if (phase) *phase = PH_IDLE;
    if (step) *step = 0;
    if (nstep) *nstep = 0;
    return SEM_OK;
  }
  if (r->cfg.check_every > 0) consume_check(r);
  const LaneDesc& L = r->h_lanes[lane];
  if (phase) *phase = L.phase;
  if (step) *step = L.it0;
  if (nstep) *nstep = L.nstep;
  if (r->cfg.check_every > 0 && r->lane_failed[lane])
    return fail(SEM_ERR_NUMERIC,
                "lane %d: non-finite wavefield found at step %d of its %s run (checked every "
                "%d steps); the lane stopped there, sem_lane_finish releases it",
                lane, r->lane_fail_step[lane], L.phase == PH_ADJ ? "adjoint" : "forward",
                r->cfg.check_every);
  return SEM_OK;
}

int sem_lane_finish(sem_run* r, int lane, float* seis, double* kernels6, double* ksum_dev) {
  if (!r || !r->lanes_mode || lane < 0 || lane >= r->nev)
    return fail(SEM_ERR_ARG, "lane %d is not a serving lane", lane);
  LaneDesc& L = r->h_lanes[lane];
  if (L.phase == PH_IDLE || L.it0 < L.nstep)
    return fail(SEM_ERR_STATE, "lane %d has not completed a run", lane);
  if (r->cfg.check_every > 0) {
    // take in the check in flight, then scan the lane's final state, so that
    // no result leaves a lane unchecked and no flag outlives its request
    if (r->check_pending) {
      CK(cudaEventSynchronize(r->check_ev));
      consume_check(r);
    }
    if (!r->lane_failed[lane]) {
      queue_check(r, true, 0);
      CK(cudaMemcpyAsync(r->h_lflags, r->lflags.p, r->lflags.bytes(), cudaMemcpyDeviceToHost,
                         r->stream));
      CK(cudaMemcpyAsync(r->h_halt, r->halt_step.p, r->halt_step.bytes(),
                         cudaMemcpyDeviceToHost, r->stream));
      CK(cudaEventRecord(r->check_ev, r->stream));
      r->check_pending = true;
      CK(cudaEventSynchronize(r->check_ev));
      consume_check(r);
    }
  }
  if (r->cfg.check_every > 0 && r->lane_failed[lane]) {
    // a lane stopped by the stability check: release it, no results
    if (r->lane_store[lane]) CK(cudaFreeAsync(r->lane_store[lane], r->stream));
    if (r->lane_scale[lane]) CK(cudaFreeAsync(r->lane_scale[lane], r->stream));
    r->lane_store[lane] = nullptr;
    r->lane_scale[lane] = nullptr;
    const int at = r->lane_fail_step[lane];
    const bool adj = L.phase == PH_ADJ;
    L.phase = PH_IDLE;
    r->lane_failed[lane] = 0;
    CK(cudaStreamSynchronize(r->stream));
    return fail(SEM_ERR_NUMERIC, "lane %d: non-finite wavefield at step %d of its %s run; lane "
                "released without results", lane, at, adj ? "adjoint" : "forward");
  }
  if (seis && L.phase == PH_FWD)
    CK(cudaMemcpyAsync(seis, L.seis, (size_t)L.nrec * 3 * L.nstep * 4, cudaMemcpyDeviceToHost,
                       r->stream));
  if (L.phase == PH_ADJ && (kernels6 || ksum_dev)) {
    const size_t ne = (size_t)r->mesh->nspec * NGLL3;
    if (kernels6 && !r->kout.p) CKM(r->kout.alloc(6 * ne), "kernel output");
    launch_finalize_kernels(r->mesh->view(), r->mesh->rho.p,
                            {r->k_rho.p, r->k_mu.p, r->k_kappa.p}, r->lm, lane,
                            kernels6 ? r->kout.p : nullptr, ksum_dev, r->stream);
    CK(cudaGetLastError());
    if (kernels6)
      CK(cudaMemcpyAsync(kernels6, r->kout.p, 6 * ne * 8, cudaMemcpyDeviceToHost, r->stream));
  }
  const bool keep_store = L.phase == PH_FWD && L.save;
  if (!keep_store) {
    if (r->lane_store[lane]) CK(cudaFreeAsync(r->lane_store[lane], r->stream));
    if (r->lane_scale[lane]) CK(cudaFreeAsync(r->lane_scale[lane], r->stream));
    r->lane_store[lane] = nullptr;
    r->lane_scale[lane] = nullptr;
    L.phase = PH_IDLE;
  }
  CK(cudaStreamSynchronize(r->stream));
  return SEM_OK;
}

int sem_lane_move(sem_run* r, int from, int to) {
  if (!r || !r->lanes_mode || from < 0 || from >= r->nev || to < 0 || to >= r->nev || from == to)
    return fail(SEM_ERR_ARG, "lanes %d -> %d are not two serving lanes of this run", from, to);
  LaneDesc& F = r->h_lanes[from];
  LaneDesc& T = r->h_lanes[to];
  if (F.phase == PH_IDLE) return fail(SEM_ERR_STATE, "lane %d holds no request", from);
  if (T.phase != PH_IDLE || r->lane_store[to] || r->lane_scale[to])
    return fail(SEM_ERR_STATE, "lane %d is not free", to);
  if (r->cfg.check_every > 0 && r->lane_failed[from])
    return fail(SEM_ERR_STATE, "lane %d was stopped by the stability check", from);
  // wavefields, kernel accumulators and the per-event arrays, queued behind
  // the work already on the stream
  const size_t ng = r->mesh->nglob, ne = (size_t)r->mesh->nspec * NGLL3;
  launch_lane_move(r->u1.p, r->v1.p, r->a1.p, ng, 3, r->lm, from, to, r->stream);
  if (F.phase == PH_ADJ) {
    launch_lane_move(r->u2.p, r->v2.p, r->a2.p, ng, 3, r->lm, from, to, r->stream);
    launch_lane_move(r->k_rho.p, r->hess_on ? r->k_hess.p : nullptr, nullptr, ng, 1, r->lm, from,
                     to, r->stream);
    launch_lane_move(r->k_mu.p, r->k_kappa.p, nullptr, ne, 1, r->lm, from, to, r->stream);
  }
  const size_t ns = r->nstep, nr = r->nrec_max;
  auto d2d = [&](float* base, size_t per) -> cudaError_t {
    return cudaMemcpyAsync(base + (size_t)to * per, base + (size_t)from * per, per * 4,
                           cudaMemcpyDeviceToDevice, r->stream);
  };
  CK(d2d(r->stf.p, ns));
  CK(d2d(r->srcarr.p, 375));
  CK(d2d(r->rec_w.p, nr * 125));
  CK(d2d(r->seis.p, nr * 3 * ns));
  CK(d2d(r->adj.p, nr * 3 * ns));
  CK(cudaMemcpyAsync(r->rec_ispec.p + (size_t)to * nr, r->rec_ispec.p + (size_t)from * nr,
                     nr * sizeof(int), cudaMemcpyDeviceToDevice, r->stream));
  if (r->lane_misfit.p)
    CK(cudaMemcpyAsync(r->lane_misfit.p + to, r->lane_misfit.p + from, sizeof(double),
                       cudaMemcpyDeviceToDevice, r->stream));
  if (r->cfg.check_every > 0 && r->lflags.p) {
    // the target starts with a clear stability flag
    CK(cudaMemsetAsync(r->lflags.p + to, 0, sizeof(int), r->stream));
    CK(cudaMemsetAsync(r->halt_step.p + to, 0xff, sizeof(int), r->stream));
    r->lane_failed[to] = 0;
    r->lane_fail_step[to] = -1;
  }
  CK(cudaGetLastError());
  // host state: the lane descriptor with the target's array regions
  const LaneDesc f = F;
  lane_defaults(r, to);
  T.phase = f.phase;
  T.it0 = f.it0;
  T.nstep = f.nstep;
  T.save = f.save;
  T.src_ispec = f.src_ispec;
  T.nrec = f.nrec;
  T.store = f.store;
  T.scale = f.scale;
  r->lane_store[to] = r->lane_store[from];
  r->lane_scale[to] = r->lane_scale[from];
  r->lane_store[from] = nullptr;
  r->lane_scale[from] = nullptr;
  r->lane_saved[to] = r->lane_saved[from];
  r->lane_saved[from] = 0;
  r->src_ispec[to] = r->src_ispec[from];
  r->nrec[to] = r->nrec[from];
  r->have_src[to] = r->have_src[from];
  r->have_rec[to] = r->have_rec[from];
  F = LaneDesc{};
  F.phase = PH_IDLE;
  lane_defaults(r, from);
  return SEM_OK;
}

int sem_lane_finish_async(sem_run* r, int lane, float* seis, double* kernels6,
                          double* ksum_dev) {
  if (!r || !r->lanes_mode || lane < 0 || lane >= r->nev)
    return fail(SEM_ERR_ARG, "lane %d is not a serving lane", lane);
  // with the stability check on, a lane's last steps are scanned before
  // its results leave: the blocking form does that
  if (r->cfg.check_every > 0) return sem_lane_finish(r, lane, seis, kernels6, ksum_dev);
  LaneDesc& L = r->h_lanes[lane];
  if (L.phase == PH_IDLE || L.it0 < L.nstep)
    return fail(SEM_ERR_STATE, "lane %d has not completed a run", lane);
  cudaEvent_t done = nullptr;
  int rc = lane_result_event(r, lane, &done);
  if (rc) return rc;
  if (seis && L.phase == PH_FWD)
    CK(cudaMemcpyAsync(seis, L.seis, (size_t)L.nrec * 3 * L.nstep * 4, cudaMemcpyDeviceToHost,
                       r->stream));
  if (L.phase == PH_ADJ && (kernels6 || ksum_dev)) {
    const size_t ne = (size_t)r->mesh->nspec * NGLL3;
    if (kernels6 && !r->kout.p) CKM(r->kout.alloc(6 * ne), "kernel output");
    launch_finalize_kernels(r->mesh->view(), r->mesh->rho.p,
                            {r->k_rho.p, r->k_mu.p, r->k_kappa.p}, r->lm, lane,
                            kernels6 ? r->kout.p : nullptr, ksum_dev, r->stream);
    CK(cudaGetLastError());
    if (kernels6)
      CK(cudaMemcpyAsync(kernels6, r->kout.p, 6 * ne * 8, cudaMemcpyDeviceToHost, r->stream));
  }
  CK(cudaEventRecord(done, r->stream));
  const bool keep_store = L.phase == PH_FWD && L.save;
  if (!keep_store) {
    if (r->lane_store[lane]) CK(cudaFreeAsync(r->lane_store[lane], r->stream));
    if (r->lane_scale[lane]) CK(cudaFreeAsync(r->lane_scale[lane], r->stream));
    r->lane_store[lane] = nullptr;
    r->lane_scale[lane] = nullptr;
    L.phase = PH_IDLE;
  }
  return SEM_OK;
}

int sem_lane_ready(sem_run* r, int lane, int wait) {
  if (!r || lane < 0 || lane >= r->nev) return fail(SEM_ERR_ARG, "bad lane");
  if (r->lane_res_ev.empty() || !r->lane_res_ev[lane]) return 1;
  if (wait) {
    CK(cudaEventSynchronize(r->lane_res_ev[lane]));
    return 1;
  }
  const cudaError_t q = cudaEventQuery(r->lane_res_ev[lane]);
  if (q == cudaSuccess) return 1;
  if (q == cudaErrorNotReady) {
    cudaGetLastError();
    return 0;
  }
  return fail(SEM_ERR_CUDA, "lane %d: %s", lane, cudaGetErrorString(q));
}

int sem_kernel_variants(sem_run* r, int* fwd, int* adj) {
  if (!r) return fail(SEM_ERR_ARG, "null run");
  // internal 0..3 -> public 1..4
  auto pub = [&](int ph) {
    if (r->cfg.kernel_variant != 0) return r->cfg.kernel_variant;
    return r->variant[ph] < 0 ? -1 : r->variant[ph] + 1;
  };
  if (fwd) *fwd = pub(0);
  if (adj) *adj = pub(1);
  return SEM_OK;
}

int sem_last_loop_ms(sem_run* r, double* ms) {
  if (!r || !ms) return fail(SEM_ERR_ARG, "null argument");
  CK(cudaStreamSynchronize(r->stream));
  float f = 0.f;
  CK(cudaEventElapsedTime(&f, r->e0, r->e1));
  *ms = f;
  return SEM_OK;
}

int sem_last_launch_count(sem_run* r, long long* count) {
  if (!r || !count) return fail(SEM_ERR_ARG, "null argument");
  *count = r->last_launches;
  return SEM_OK;
}

}  // extern "C"
