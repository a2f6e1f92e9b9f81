// PrepareFWD over the C ABI (see prepare_fwd.hpp for the reference map).
#include "prepare_fwd.hpp"

#include <string>
#include <vector>

namespace specfwat {
namespace {

void check(int rc, const char* call) {
  if (rc != SEM_OK) {
    const char* msg = sem_last_error();
    throw SemError(rc, std::string(call) + ": " + (msg ? msg : ""));
  }
}

void require(bool ok, const std::string& what) {
  if (!ok) throw SemError(SEM_ERR_ARG, what);
}

}  // namespace

Mesh::Mesh(const sem_mesh_desc& desc) : nspec_(desc.nspec) {
  check(sem_prepare_mesh(&desc, &h_), "sem_prepare_mesh");
}

Mesh::~Mesh() {
  if (h_) sem_release_mesh(h_);
}

PrepareFWD::PrepareFWD(const Mesh& mesh, const Config& cfg, RunMode run_mode, int nev)
    : mesh_(&mesh), cfg_(cfg), mode_(run_mode), nev_(nev) {
  require(run_mode >= FORWARD_ONLY && run_mode <= ADJOINT_ONLY, "run_mode must be 1..5");
  require(nev >= 1, "nev must be >= 1");
  sem_run_cfg c{};
  c.nev = nev;
  c.nstep = cfg.nstep;
  c.dt = cfg.dt;
  c.store_kind = cfg.store_kind;
  c.use_graph = cfg.use_graph ? 1 : 0;
  c.graph_steps = cfg.graph_steps;
  c.max_receivers = cfg.max_receivers;
  c.check_every = 0;
  c.kernel_variant = 0;  // autotuned
  check(sem_prepare_timerun(mesh.handle(), &c, &run_), "sem_prepare_timerun");
  nrec_.assign((size_t)nev, 0);
  observed_.assign((size_t)nev, {});
  misfits_.assign((size_t)nev, 0.0);
  kernels_.assign((size_t)nev, {});
}

PrepareFWD::~PrepareFWD() { destroy(); }

void PrepareFWD::destroy() {
  if (run_) {
    sem_release_run(run_);
    run_ = nullptr;
  }
}

void PrepareFWD::prepare_for_event(const std::vector<EventData>& events) {
  require(run_ != nullptr, "the run was destroyed");
  require((int)events.size() == nev_, "one EventData per event of the batch");
  const bool measure = mode_ == FORWARD_MEASADJ || mode_ == FORWARD_ADJOINT;
  std::vector<sem_source> src((size_t)nev_);
  for (int e = 0; e < nev_; ++e) src[(size_t)e] = events[(size_t)e].source;
  check(sem_set_sources(run_, nev_, src.data()), "sem_set_sources");
  for (int e = 0; e < nev_; ++e) {
    const EventData& ev = events[(size_t)e];
    require(!ev.stations.empty() && ev.stations.size() % 3 == 0,
            "stations are [nrec][3] coordinates");
    const int nrec = (int)(ev.stations.size() / 3);
    check(sem_set_receivers(run_, e, nrec, ev.stations.data()), "sem_set_receivers");
    nrec_[(size_t)e] = nrec;
    if (measure) {
      require(ev.observed.size() == (size_t)nrec * 3 * (size_t)cfg_.nstep,
              "observed data are [nrec][3][nstep]");
      observed_[(size_t)e] = ev.observed;
    }
  }
}

void PrepareFWD::set_adjoint_sources(int ev, const std::vector<double>& adj) {
  require(run_ != nullptr, "the run was destroyed");
  require(ev >= 0 && ev < nev_, "event out of range");
  require(adj.size() == (size_t)nrec_[(size_t)ev] * 3 * (size_t)cfg_.nstep,
          "adjoint sources are [nrec][3][nstep]");
  check(sem_set_adjoint_sources(run_, ev, adj.data()), "sem_set_adjoint_sources");
}

void PrepareFWD::set_run_mode(RunMode mode) {
  require(mode >= FORWARD_ONLY && mode <= ADJOINT_ONLY, "run_mode must be 1..5");
  mode_ = mode;
}

void PrepareFWD::simulation() {
  require(run_ != nullptr, "the run was destroyed");
  if (mode_ <= FORWARD_SAVE) run_simulation(1);
  if (mode_ == FORWARD_MEASADJ || mode_ == FORWARD_ADJOINT) measure_adj();
  if (mode_ == FORWARD_ADJOINT || mode_ == ADJOINT_ONLY) {
    if (!saved_)
      throw SemError(SEM_ERR_STATE, "the adjoint run needs a saved forward run "
                                    "(FORWARD_ADJOINT, or FORWARD_SAVE before ADJOINT_ONLY)");
    run_simulation(3);
    postproc_adjoint();
  }
}

void PrepareFWD::run_simulation(int sim_type) {
  // SAVE_FORWARD for the run modes that keep the forward state
  const int save = (sim_type == 1 && (mode_ == FORWARD_ADJOINT || mode_ == FORWARD_SAVE)) ? 1 : 0;
  check(sem_iterate_time(run_, sim_type, save), "sem_iterate_time");
  check(sem_synchronize(run_), "sem_synchronize");
  if (sim_type == 1) saved_ = save != 0;
}

void PrepareFWD::measure_adj() {
  obj_func_ = 0.0;
  for (int e = 0; e < nev_; ++e) {
    double m = 0.0;
    check(sem_measure_l2(run_, e, observed_[(size_t)e].data(), cfg_.taper_pct, cfg_.taper_type,
                         &m),
          "sem_measure_l2");
    misfits_[(size_t)e] = m;
    obj_func_ += m;
  }
}

void PrepareFWD::postproc_adjoint() {
  const size_t n = (size_t)6 * (size_t)mesh_->nspec() * 125;
  for (int e = 0; e < nev_; ++e) {
    kernels_[(size_t)e].assign(n, 0.0);
    check(sem_save_adjoint_kernels(run_, e, kernels_[(size_t)e].data()),
          "sem_save_adjoint_kernels");
  }
  sum_.assign(n, 0.0);
  check(sem_sum_kernels(run_, sum_.data()), "sem_sum_kernels");
}

std::vector<float> PrepareFWD::seismograms(int ev) const {
  require(run_ != nullptr, "the run was destroyed");
  require(ev >= 0 && ev < nev_, "event out of range");
  std::vector<float> out((size_t)nrec_[(size_t)ev] * 3 * (size_t)cfg_.nstep);
  check(sem_get_seismograms(run_, ev, out.data()), "sem_get_seismograms");
  return out;
}

const std::vector<double>& PrepareFWD::event_kernels(int ev) const {
  require(ev >= 0 && ev < nev_, "event out of range");
  return kernels_[(size_t)ev];
}

std::vector<float> gradient_on_grid(const Mesh& mesh, const std::vector<double>& kernels,
                                    const std::vector<float>* precond,
                                    const GradientConfig& cfg) {
  const size_t ne = (size_t)mesh.nspec() * 125;
  require(kernels.size() == 6 * ne, "kernels are [6][nspec][125]");
  require(!precond || precond->size() == ne, "the preconditioner is [nspec][125]");
  const int iso[3] = {5, 4, 3};  // alpha, beta, rhop in rho, mu, kappa, rhop, beta, alpha
  const int nsm = cfg.rho_scaling ? 2 : 3;
  std::vector<float> in((size_t)nsm * ne), sm((size_t)nsm * ne);
  for (int f = 0; f < nsm; ++f)
    for (size_t i = 0; i < ne; ++i) {
      double v = kernels[(size_t)iso[f] * ne + i];
      if (precond) v *= (double)(*precond)[i];
      in[(size_t)f * ne + i] = (float)v;
    }
  sem_smooth_cfg sc{};
  sc.sigma_h = cfg.sigma_h;
  sc.sigma_v = cfg.sigma_v;
  sc.mapping = SEM_SMOOTH_MAP_CUBE;
  check(sem_smooth_pde(mesh.handle(), &sc, nsm, in.data(), nullptr, sm.data(), nullptr),
        "sem_smooth_pde");
  const size_t ng = (size_t)cfg.grid.n[0] * cfg.grid.n[1] * cfg.grid.n[2];
  std::vector<float> grid(3 * ng);
  check(sem_grid_project(mesh.handle(), &cfg.grid, nsm, sm.data(), grid.data()),
        "sem_grid_project");
  if (cfg.rho_scaling)
    for (size_t i = 0; i < ng; ++i) grid[2 * ng + i] = grid[ng + i] * 0.33f;
  if (cfg.taper)
    check(sem_grid_taper(mesh.handle(), &cfg.grid, &cfg.taper_widths, 3, grid.data(), nullptr),
          "sem_grid_taper");
  return grid;
}

}  // namespace specfwat
