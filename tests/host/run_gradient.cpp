// Test driver of the C++ gradient_on_grid: reads a case directory written by
// tests/test_gpu_host_cpp.py and writes the gradient grid.
//
// case.txt: nspec nglob nf xix jac  x0 y0 z0  hx hy hz  nx ny nz
//           sigma_h sigma_v rho_scaling taper h_suppress h_buffer v_suppress
//           v_buffer
// mesh arrays as for run_case, kernels.f64 [6][nspec*125], precond.f32
// [nspec*125].  Writes grad.f32 [3][nx][ny][nz].
#include <iostream>
#include <string>
#include <vector>

#include "case_mesh.hpp"
#include "prepare_fwd.hpp"

int main(int argc, char** argv) {
  if (argc != 2) {
    std::cerr << "usage: run_gradient <case dir>\n";
    return 2;
  }
  const std::string dir = argv[1];
  try {
    std::ifstream h(dir + "/case.txt");
    int nspec, nglob, nf, rho_scaling, taper;
    double xix, jac;
    specfwat::GradientConfig cfg;
    if (!(h >> nspec >> nglob >> nf >> xix >> jac))
      throw std::runtime_error("bad case.txt");
    for (int d = 0; d < 3; ++d) h >> cfg.grid.x0[d];
    for (int d = 0; d < 3; ++d) h >> cfg.grid.h[d];
    for (int d = 0; d < 3; ++d) h >> cfg.grid.n[d];
    cfg.grid.ngnod = 8;
    if (!(h >> cfg.sigma_h >> cfg.sigma_v >> rho_scaling >> taper >>
          cfg.taper_widths.h_suppress >> cfg.taper_widths.h_buffer >>
          cfg.taper_widths.v_suppress >> cfg.taper_widths.v_buffer))
      throw std::runtime_error("bad case.txt");
    cfg.rho_scaling = rho_scaling != 0;
    cfg.taper = taper != 0;
    CaseMesh cm(dir, nspec, nglob, nf, xix, jac);
    const size_t ne = (size_t)nspec * 125;
    auto kernels = load_array<double>(dir, "kernels.f64", 6 * ne);
    auto precond = load_array<float>(dir, "precond.f32", ne);
    specfwat::Mesh mesh(cm.desc);
    auto grad = specfwat::gradient_on_grid(mesh, kernels, &precond, cfg);
    save_array(dir, "grad.f32", grad);
  } catch (const specfwat::SemError& e) {
    std::cerr << "SemError " << e.status() << ": " << e.what() << "\n";
    return 3;
  } catch (const std::exception& e) {
    std::cerr << e.what() << "\n";
    return 4;
  }
  return 0;
}
