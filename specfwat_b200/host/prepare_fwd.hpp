// C++ host side above the C ABI: the per-event driver in the shape of the
// reference's PrepareFWD (src/preproc/prepare_fwd.f90:28-35), for a C++ or
// Fortran-replacing caller that runs forward, measurement and adjoint
// passes of a batch of events on one resident mesh.
//
//   reference (prepare_fwd.f90)          here
//   -----------------------------------  ---------------------------------
//   init(this)             :39-96        PrepareFWD(mesh, cfg, run_mode, nev)
//   prepare_for_event      :167-233      prepare_for_event(events)
//   simulation             :297-326      simulation()
//   run_simulation(run_opt):328-368      run_simulation(1 | 3)   (private)
//   measure_adj            :258-295      measure_adj()           (private)
//   postproc_adjoint       :370-384      postproc_adjoint()      (private)
//   destroy                :127-140      destroy() / destructor
//   obj_func                             obj_func()
//
//   xfwat_post_proc for an isotropic model (src/postproc/fwat_post_proc.f90:
//   29-46; PostFlow%apply_precond, pde_smooth, taper_kernel_grid of
//   post_processing.f90:164-325)         gradient_on_grid(mesh, kernels, ...)
//
// read_mesh_databases_fwat (+ the mesh part of prepare_GPU) is Mesh, built
// from the database arrays the reference reads (sem_mesh_desc).  The run
// modes are the reference's (src/shared/config.f90:52-56).  Where the
// reference aborts through exit_MPI, these calls throw SemError with the
// library's status and message; the device state stays usable.
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "sem_b200.h"

namespace specfwat {

enum RunMode : int {
  FORWARD_ONLY = 1,     // forward, seismograms
  FORWARD_MEASADJ = 2,  // forward, misfit and adjoint sources
  FORWARD_ADJOINT = 3,  // forward (saved), misfit, adjoint, kernels
  FORWARD_SAVE = 4,     // forward with the state kept for a later adjoint
  ADJOINT_ONLY = 5      // adjoint of the saved forward, kernels
};

// A refused or failed C-ABI call: its sem_status and sem_last_error().
class SemError : public std::runtime_error {
 public:
  SemError(int status, const std::string& what) : std::runtime_error(what), status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

// Device-resident mesh database.
class Mesh {
 public:
  explicit Mesh(const sem_mesh_desc& desc);
  ~Mesh();
  Mesh(const Mesh&) = delete;
  Mesh& operator=(const Mesh&) = delete;
  sem_mesh* handle() const { return h_; }
  int nspec() const { return nspec_; }

 private:
  sem_mesh* h_ = nullptr;
  int nspec_ = 0;
};

// One event of the acquisition: CMT source, stations (x, y, z in metres,
// [nrec][3]) and, for the measurement run modes, the observed data
// [nrec][3][nstep] on the synthetics' time axis.
struct EventData {
  sem_source source{};
  std::vector<double> stations;
  std::vector<double> observed;
};

class PrepareFWD {
 public:
  struct Config {
    int nstep = 0;
    double dt = 0.0;
    int store_kind = SEM_STORE_FP16;  // boundary store of the forward run
    bool use_graph = true;            // step loop replayed as CUDA graphs
    int graph_steps = 50;
    int max_receivers = 128;
    double taper_pct = 0.05;          // L2 measurement taper (fraction)
    int taper_type = 1;
  };

  // init: the run's device state for nev events sharing the mesh
  PrepareFWD(const Mesh& mesh, const Config& cfg, RunMode run_mode, int nev);
  ~PrepareFWD();
  PrepareFWD(const PrepareFWD&) = delete;
  PrepareFWD& operator=(const PrepareFWD&) = delete;

  // sources and stations of the batch (setup_sources_receivers_fwat), and
  // the observed data the measurement needs
  void prepare_for_event(const std::vector<EventData>& events);
  // one pass of the run mode: forward, measurement, adjoint, kernels
  void simulation();
  // releases the device state (also done by the destructor)
  void destroy();

  // adjoint sources of event ev in forward time order [nrec][3][nstep],
  // for ADJOINT_ONLY passes whose sources come from elsewhere
  void set_adjoint_sources(int ev, const std::vector<double>& adj);
  // the mode of the next pass: a FORWARD_SAVE pass keeps the forward state
  // on the device, and an ADJOINT_ONLY pass of the same object runs the
  // adjoint of it (the reference does the two in separate runs through
  // save_forward_arrays.bin and absorb_field.bin)
  void set_run_mode(RunMode mode);

  // results of the last pass
  double obj_func() const { return obj_func_; }                     // sum of the misfits
  const std::vector<double>& misfits() const { return misfits_; }   // per event
  std::vector<float> seismograms(int ev) const;                     // [nrec][3][nstep]
  const std::vector<double>& event_kernels(int ev) const;           // [6][nspec][125]
  const std::vector<double>& sum_kernels() const { return sum_; }   // [6][nspec][125], FP64

  int nev() const { return nev_; }
  RunMode run_mode() const { return mode_; }

 private:
  void run_simulation(int sim_type);
  void measure_adj();
  void postproc_adjoint();

  sem_run* run_ = nullptr;
  const Mesh* mesh_;
  Config cfg_;
  RunMode mode_;
  int nev_;
  bool saved_ = false;  // a forward state is kept for an adjoint run
  std::vector<int> nrec_;
  std::vector<std::vector<double>> observed_;
  std::vector<double> misfits_;
  double obj_func_ = 0.0;
  std::vector<std::vector<double>> kernels_;
  std::vector<double> sum_;
};

// The model-grid gradient of fwat_post_proc: the KERNEL_ISO kernels
// (alpha, beta, rhop; src/shared/config.f90:35) of summed kernels
// [6][nspec][125] (rho, mu, kappa, rhop, beta, alpha), times the
// preconditioner [nspec][125] when given (apply_precond), each smoothed
// (pde_smooth: sem_smooth_pde, the cube mapping), projected onto the grid
// (gll2grid: sem_grid_project); with rho_scaling the rhop grid is the beta
// grid times 0.33 (USE_RHO_SCALING, post_processing.f90:262-264); then
// tapered when `taper` is set (taper_kernel_grid: sem_grid_taper).
// Returns [3][nx][ny][nz] in KERNEL_ISO order.
struct GradientConfig {
  sem_grid_desc grid{};
  double sigma_h = 0.0, sigma_v = 0.0;
  bool rho_scaling = false;
  bool taper = false;
  sem_grid_taper_cfg taper_widths{};
};

std::vector<float> gradient_on_grid(const Mesh& mesh, const std::vector<double>& kernels,
                                    const std::vector<float>* precond,
                                    const GradientConfig& cfg);

}  // namespace specfwat
