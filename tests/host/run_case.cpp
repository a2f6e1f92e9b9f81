// Test driver of the C++ host side: reads a case directory written by
// tests/test_gpu_host_cpp.py, runs one PrepareFWD pass and writes the
// results beside the inputs.
//
// case.txt: nspec nglob nf nev nrec nstep dt xix jac run_mode taper_pct
// arrays (little-endian, C order): ibool.i32 [nspec*125], x/y/z.f32
// [nglob], kappa/mu/rho/rho_vp/rho_vs.f32 [nspec*125], rmass.f32 [nglob],
// f_ispec.i32 [nf], f_ijk.i32 [nf*75], f_jw.f32 [nf*25], f_n.f32 [nf*75],
// sources.f64 [nev][11] (sem_source fields), stations.f64 [nrec][3],
// obs.f64 [nev][nrec][3][nstep].
// Writes misfits.f64, kernels.f64 [nev][6][nspec*125], sum.f64,
// seis.f32 [nev][nrec][3][nstep] and errors.txt (the status of a refused
// call).  With a second argument "save-adjoint" the pass is FORWARD_SAVE,
// then ADJOINT_ONLY with the adjoint sources synthetics - observed.
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "case_mesh.hpp"
#include "prepare_fwd.hpp"

int main(int argc, char** argv) {
  if (argc != 2 && argc != 3) {
    std::cerr << "usage: run_case <case dir> [save-adjoint]\n";
    return 2;
  }
  const std::string dir = argv[1];
  const bool two_pass = argc == 3 && std::string(argv[2]) == "save-adjoint";
  try {
    std::ifstream h(dir + "/case.txt");
    int nspec, nglob, nf, nev, nrec, nstep, mode;
    double dt, xix, jac, taper;
    if (!(h >> nspec >> nglob >> nf >> nev >> nrec >> nstep >> dt >> xix >> jac >> mode >> taper))
      throw std::runtime_error("bad case.txt");
    CaseMesh cm(dir, nspec, nglob, nf, xix, jac);
    auto srcs = load_array<double>(dir, "sources.f64", (size_t)nev * 11);
    auto sta = load_array<double>(dir, "stations.f64", (size_t)nrec * 3);
    const size_t per = (size_t)nrec * 3 * nstep;
    auto obs = load_array<double>(dir, "obs.f64", (size_t)nev * per);
    const sem_mesh_desc& d = cm.desc;
    specfwat::Mesh mesh(d);

    specfwat::PrepareFWD::Config cfg;
    cfg.nstep = nstep;
    cfg.dt = dt;
    cfg.max_receivers = nrec;
    cfg.taper_pct = taper;
    specfwat::PrepareFWD fwd(mesh, cfg, (specfwat::RunMode)mode, nev);
    std::vector<specfwat::EventData> events((size_t)nev);
    for (int e = 0; e < nev; ++e) {
      const double* s = srcs.data() + (size_t)e * 11;
      events[(size_t)e].source = sem_source{s[0], s[1], s[2], s[3], s[4], s[5],
                                            s[6], s[7], s[8], s[9], s[10]};
      events[(size_t)e].stations = sta;
      events[(size_t)e].observed.assign(obs.begin() + (long)(e * per),
                                        obs.begin() + (long)((e + 1) * per));
    }
    fwd.prepare_for_event(events);
    if (two_pass) {
      // an adjoint pass before any saved forward is refused
      fwd.set_run_mode(specfwat::ADJOINT_ONLY);
      int early = 0;
      try {
        fwd.simulation();
      } catch (const specfwat::SemError& e) {
        early = e.status();
      }
      if (early != SEM_ERR_STATE) throw std::runtime_error("adjoint before forward not refused");
      fwd.set_run_mode(specfwat::FORWARD_SAVE);
      fwd.simulation();
      for (int e = 0; e < nev; ++e) {
        const auto s = fwd.seismograms(e);
        std::vector<double> adj(per);
        for (size_t i = 0; i < per; ++i) adj[i] = (double)s[i] - events[(size_t)e].observed[i];
        fwd.set_adjoint_sources(e, adj);
      }
      fwd.set_run_mode(specfwat::ADJOINT_ONLY);
    }
    fwd.simulation();

    save_array(dir, "misfits.f64", fwd.misfits());
    std::vector<float> seis;
    std::vector<double> kern;
    for (int e = 0; e < nev; ++e) {
      auto s = fwd.seismograms(e);
      seis.insert(seis.end(), s.begin(), s.end());
      const auto& k = fwd.event_kernels(e);
      kern.insert(kern.end(), k.begin(), k.end());
    }
    save_array(dir, "seis.f32", seis);
    save_array(dir, "kernels.f64", kern);
    save_array(dir, "sum.f64", fwd.sum_kernels());

    // a refused call reaches the caller as SemError with the status
    int status = 0;
    try {
      fwd.set_adjoint_sources(nev, std::vector<double>(per, 0.0));
    } catch (const specfwat::SemError& e) {
      status = e.status();
    }
    std::ofstream out(dir + "/errors.txt");
    out.precision(17);
    out << status << " " << fwd.obj_func() << "\n";
  } catch (const specfwat::SemError& e) {
    std::cerr << "SemError " << e.status() << ": " << e.what() << "\n";
    return 3;
  } catch (const std::exception& e) {
    std::cerr << e.what() << "\n";
    return 4;
  }
  return 0;
}
