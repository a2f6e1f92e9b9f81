// Mesh arrays of a test case directory (written by tests/test_gpu_host_cpp.py)
// and the sem_mesh_desc over them.
#pragma once

#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "sem_b200.h"

template <class T>
std::vector<T> load_array(const std::string& dir, const std::string& name, size_t n) {
  std::vector<T> v(n);
  std::ifstream f(dir + "/" + name, std::ios::binary);
  if (!f || !f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(n * sizeof(T))))
    throw std::runtime_error("cannot read " + name);
  return v;
}

template <class T>
void save_array(const std::string& dir, const std::string& name, const std::vector<T>& v) {
  std::ofstream f(dir + "/" + name, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(T)));
}

struct CaseMesh {
  std::vector<int> ibool, fisp, fijk;
  std::vector<float> x, y, z, kappa, mu, rho, rvp, rvs, rmass, fjw, fn;
  sem_mesh_desc desc{};

  CaseMesh(const std::string& dir, int nspec, int nglob, int nf, double xix, double jac) {
    const size_t ne = (size_t)nspec * 125;
    ibool = load_array<int>(dir, "ibool.i32", ne);
    x = load_array<float>(dir, "x.f32", nglob);
    y = load_array<float>(dir, "y.f32", nglob);
    z = load_array<float>(dir, "z.f32", nglob);
    kappa = load_array<float>(dir, "kappa.f32", ne);
    mu = load_array<float>(dir, "mu.f32", ne);
    rho = load_array<float>(dir, "rho.f32", ne);
    rvp = load_array<float>(dir, "rho_vp.f32", ne);
    rvs = load_array<float>(dir, "rho_vs.f32", ne);
    rmass = load_array<float>(dir, "rmass.f32", nglob);
    fisp = load_array<int>(dir, "f_ispec.i32", nf);
    fijk = load_array<int>(dir, "f_ijk.i32", (size_t)nf * 75);
    fjw = load_array<float>(dir, "f_jw.f32", (size_t)nf * 25);
    fn = load_array<float>(dir, "f_n.f32", (size_t)nf * 75);
    desc.nspec = nspec;
    desc.nglob = nglob;
    desc.index_base = 0;
    desc.ibool = ibool.data();
    desc.xstore = x.data();
    desc.ystore = y.data();
    desc.zstore = z.data();
    desc.xix_regular = (float)xix;
    desc.jacobian_regular = (float)jac;
    desc.kappastore = kappa.data();
    desc.mustore = mu.data();
    desc.rhostore = rho.data();
    desc.rmass = rmass.data();
    desc.rho_vp = rvp.data();
    desc.rho_vs = rvs.data();
    desc.num_abs_boundary_faces = nf;
    desc.abs_boundary_ispec = fisp.data();
    desc.abs_boundary_ijk = fijk.data();
    desc.abs_boundary_jacobian2Dw = fjw.data();
    desc.abs_boundary_normal = fn.data();
  }
};
