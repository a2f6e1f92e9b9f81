// CPU oracle for the isotropic-elastic SEM forward/adjoint time loop.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA solver
// is compared against; it is never linked into the product library and the
// product never calls it.  Only the tests, the smoke check and the CPU
// baseline leg of the benchmark load it.
//
// Parity status: UNPINNED against the reference.  The reference's solver
// (SPECFEM3D Cartesian, git submodule src/specfem3d, .gitmodules:1-4) is not
// in the reference tree, so its numbers cannot be reproduced here.  This
// restatement follows the published spectral-element formulation
// (Komatitsch & Tromp 1999/2002: GLL quadrature, diagonal mass, explicit
// Newmark; Clayton-Engquist/Stacey first-order absorbing traction; adjoint
// kernels and backward reconstruction after Tromp, Tape & Liu 2005 and
// Liu & Tromp 2006) and the conventions the reference tree fixes:
//   * array layouts            src/specfem_interface/read_mesh_databases.f90:158-193
//   * run modes                src/preproc/prepare_fwd.f90:98-125,333-349
//   * CMT -> xyz mapping       src/specfem_interface/locate_source_fwat.f90:215-228
//   * Ricker t0 = 1.2/f0       src/specfem_interface/locate_source_fwat.f90:499-506
//   * kernel names/derivation  src/postproc/post_processing.f90:417-422
// It is pinned by physics instead: energy conservation, exact time
// reversibility of the backward reconstruction, the analytic full-space
// moment-tensor Green's function and a finite-difference gradient test,
// on regular meshes and on meshes of irregular (deformed) elements, whose
// per-point mapping (xixstore .. jacobianstore, read_mesh_databases.f90:
// 172-181) enters the gradient and the fluxes of the weak form.
//
// Time stepping convention (shared with the CUDA solver):
//   step it (0-based) = predictor, forces on the predicted displacement,
//   Stacey traction from the predicted velocity, source stf(it*dt),
//   a *= 1/(M + dt/2 C), corrector.  Afterwards (u,v,a) represent time
//   it*dt and seismogram sample it is recorded from u.
//   Backward step reconstructing forward state n uses stf(n*dt) and the
//   stored boundary term of forward step n.  The adjoint field after
//   adjoint step j (adjoint source sample N-1-j) is paired with the
//   backward state N-1-j for kernel accumulation.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#include <xmmintrin.h>
#endif

namespace {

constexpr int NG = 5;
constexpr int NG2 = 25;
constexpr int NG3 = 125;

struct Gll {
  double xi[NG], w[NG], D[NG][NG];  // D[i][l] = l_l'(xi_i)
};

// Legendre P_n(x) and its derivative by the three-term recurrence.
void legendre(int n, double x, double* p, double* dp) {
  double p0 = 1.0, p1 = x;
  if (n == 0) { *p = 1.0; *dp = 0.0; return; }
  for (int k = 2; k <= n; ++k) {
    double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
    p0 = p1;
    p1 = p2;
  }
  *p = p1;
  *dp = (std::fabs(x) < 1.0) ? n * (p0 - x * p1) / (1.0 - x * x)
                             : 0.5 * n * (n + 1.0) * std::pow(x, n + 1);
}

// GLL nodes: +-1 and the roots of P_4'(x) by Newton iteration on
// P_4'(x) = 0 (derivative computed by finite recurrence), weights
// 2/(N(N+1) P_N(x)^2).
Gll make_gll() {
  Gll g{};
  const int N = NG - 1;
  g.xi[0] = -1.0;
  g.xi[N] = 1.0;
  for (int i = 1; i < N; ++i) {
    double x = -std::cos(M_PI * i / N);
    for (int it = 0; it < 200; ++it) {
      // f(x) = P_N'(x); f'(x) from the Legendre ODE:
      // (1-x^2) P'' = 2x P' - N(N+1) P
      double p, dp;
      legendre(N, x, &p, &dp);
      double d2p = (2.0 * x * dp - N * (N + 1.0) * p) / (1.0 - x * x);
      double dx = dp / d2p;
      x -= dx;
      if (std::fabs(dx) < 1e-17) break;
    }
    g.xi[i] = x;
  }
  for (int i = 0; i < NG; ++i) {
    double p, dp;
    legendre(N, g.xi[i], &p, &dp);
    g.w[i] = 2.0 / (N * (N + 1.0) * p * p);
  }
  for (int i = 0; i < NG; ++i)
    for (int l = 0; l < NG; ++l) {
      // derivative of Lagrange polynomial l at node i
      double s = 0.0;
      for (int m = 0; m < NG; ++m) {
        if (m == l) continue;
        double prod = 1.0 / (g.xi[l] - g.xi[m]);
        for (int n = 0; n < NG; ++n) {
          if (n == l || n == m) continue;
          prod *= (g.xi[i] - g.xi[n]) / (g.xi[l] - g.xi[n]);
        }
        s += prod;
      }
      g.D[i][l] = s;
    }
  return g;
}

double lagrange(const Gll& g, int a, double x) {
  double p = 1.0;
  for (int m = 0; m < NG; ++m)
    if (m != a) p *= (x - g.xi[m]) / (g.xi[a] - g.xi[m]);
  return p;
}

double lagrange_d(const Gll& g, int a, double x) {
  double s = 0.0;
  for (int m = 0; m < NG; ++m) {
    if (m == a) continue;
    double prod = 1.0 / (g.xi[a] - g.xi[m]);
    for (int n = 0; n < NG; ++n) {
      if (n == a || n == m) continue;
      prod *= (x - g.xi[n]) / (g.xi[a] - g.xi[n]);
    }
    s += prod;
  }
  return s;
}

double ricker(double t, double f0) {
  double a = M_PI * M_PI * f0 * f0;
  return (1.0 - 2.0 * a * t * t) * std::exp(-a * t * t);
}

}  // namespace

extern "C" {

struct oracle_mesh {
  int nspec, nglob;
  const int* ibool;  // [nspec][125], 0-based
  const float *x, *y, *z;
  double xix, jac;   // regular element mapping
  const float *kappa, *mu, *rho, *rmass, *rho_vp, *rho_vs;
  int nf;
  const int* f_ispec;   // [nf]
  const int* f_ijk;     // [nf][25][3]
  const float* f_jw;    // [nf][25]
  const float* f_n;     // [nf][25][3]
  // irregular elements (may be null): irreg[e] = -1 for a regular element,
  // else its row in geo [nirreg][125][10] = xix, xiy, xiz, etax, etay,
  // etaz, gammax, gammay, gammaz, jacobian at each GLL point
  const int* irreg;
  const float* geo;
};

struct oracle_source {
  double x, y, z;
  double mt[6];  // Mrr, Mtt, Mpp, Mrt, Mrp, Mtp (N m)
  double f0, tshift;
};

}  // extern "C"

namespace {

struct Located {
  int ispec;
  double xi, eta, gam;
};

// Coordinates of the element's GLL interpolant at (xi, eta, gamma) and
// their derivatives dX[a][d] = dx_a / dxi_d.
void element_map(const oracle_mesh& m, const Gll& g, int e, const double xi[3], double X[3],
                 double dX[3][3]) {
  double l[3][NG], dl[3][NG];
  for (int d = 0; d < 3; ++d)
    for (int a = 0; a < NG; ++a) {
      l[d][a] = lagrange(g, a, xi[d]);
      dl[d][a] = lagrange_d(g, a, xi[d]);
    }
  for (int a = 0; a < 3; ++a) {
    X[a] = 0.0;
    for (int d = 0; d < 3; ++d) dX[a][d] = 0.0;
  }
  const float* cs[3] = {m.x, m.y, m.z};
  for (int k = 0; k < NG; ++k)
    for (int j = 0; j < NG; ++j)
      for (int i = 0; i < NG; ++i) {
        const int ig = m.ibool[(size_t)e * NG3 + i + NG * j + NG2 * k];
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

// Newton iteration for the reference coordinates of point p in element e;
// returns the distance of the mapped (clamped) point from p.
double newton_xi(const oracle_mesh& m, const Gll& g, int e, const double p[3], double xi[3]) {
  xi[0] = xi[1] = xi[2] = 0.0;
  double X[3], dX[3][3], inv[3][3];
  for (int it = 0; it < 30; ++it) {
    element_map(m, g, e, xi, X, dX);
    if (!invert3(dX, inv)) break;
    double step = 0.0;
    for (int d = 0; d < 3; ++d) {
      double dd = 0.0;
      for (int a = 0; a < 3; ++a) dd += inv[d][a] * (p[a] - X[a]);
      xi[d] += dd;
      if (xi[d] > 1.5) xi[d] = 1.5;
      if (xi[d] < -1.5) xi[d] = -1.5;
      step = std::max(step, std::fabs(dd));
    }
    if (step < 1e-13) break;
  }
  for (int d = 0; d < 3; ++d) xi[d] = xi[d] < -1.0 ? -1.0 : (xi[d] > 1.0 ? 1.0 : xi[d]);
  element_map(m, g, e, xi, X, dX);
  return std::sqrt((X[0] - p[0]) * (X[0] - p[0]) + (X[1] - p[1]) * (X[1] - p[1]) +
                   (X[2] - p[2]) * (X[2] - p[2]));
}

Located locate_regular(const oracle_mesh& m, double px, double py, double pz);

// On a mesh with irregular elements: of the 12 elements with the nearest
// centres, the lowest-numbered one containing the point (Newton iteration),
// else the one whose located point lies closest.
Located locate(const oracle_mesh& m, double px, double py, double pz) {
  if (!m.irreg) return locate_regular(m, px, py, pz);
  static const Gll g = make_gll();
  std::vector<std::pair<double, int>> cand;
  cand.reserve(m.nspec);
  for (int e = 0; e < m.nspec; ++e) {
    double c[3] = {0, 0, 0};
    const int corner[8] = {0, 4, 20, 24, 100, 104, 120, 124};
    const float* cs[3] = {m.x, m.y, m.z};
    for (int q = 0; q < 8; ++q) {
      const int ig = m.ibool[(size_t)e * NG3 + corner[q]];
      for (int a = 0; a < 3; ++a) c[a] += 0.125 * (double)cs[a][ig];
    }
    const double d = (px - c[0]) * (px - c[0]) + (py - c[1]) * (py - c[1]) + (pz - c[2]) * (pz - c[2]);
    cand.push_back({d, e});
  }
  const size_t nc = std::min<size_t>(12, cand.size());
  std::partial_sort(cand.begin(), cand.begin() + nc, cand.end());
  // a point on a face, edge or corner lies in several elements, whose
  // source arrays differ: take the lowest-numbered element containing it
  // (distance below 1e-6 of the element size), else the closest
  Located best{-1, 0, 0, 0};
  double bd = 1e300;
  bool inside = false;
  const double p[3] = {px, py, pz};
  for (size_t q = 0; q < nc; ++q) {
    const int e = cand[q].second;
    double xi[3];
    const double d = newton_xi(m, g, e, p, xi);
    const int g0 = m.ibool[(size_t)e * NG3], g7 = m.ibool[(size_t)e * NG3 + 124];
    const double size = std::fabs((double)m.x[g7] - (double)m.x[g0]);
    const bool in = d <= 1e-6 * size;
    const bool better = in ? (!inside || e < best.ispec) : (!inside && d < bd);
    if (better) {
      inside = inside || in;
      bd = d;
      best = {e, xi[0], xi[1], xi[2]};
    }
  }
  return best;
}

// Element whose centre is nearest (ties: lowest index), reference
// coordinates from the element's axis-aligned extent.
Located locate_regular(const oracle_mesh& m, double px, double py, double pz) {
  Located best{-1, 0, 0, 0};
  double bd = 1e300;
  for (int e = 0; e < m.nspec; ++e) {
    int g0 = m.ibool[e * NG3 + 0];
    int g7 = m.ibool[e * NG3 + 124];
    double cx = 0.5 * ((double)m.x[g0] + (double)m.x[g7]);
    double cy = 0.5 * ((double)m.y[g0] + (double)m.y[g7]);
    double cz = 0.5 * ((double)m.z[g0] + (double)m.z[g7]);
    double d = (px - cx) * (px - cx) + (py - cy) * (py - cy) + (pz - cz) * (pz - cz);
    if (d < bd) {
      bd = d;
      double hx = 0.5 * ((double)m.x[g7] - (double)m.x[g0]);
      double hy = 0.5 * ((double)m.y[g7] - (double)m.y[g0]);
      double hz = 0.5 * ((double)m.z[g7] - (double)m.z[g0]);
      best = {e, (px - cx) / hx, (py - cy) / hy, (pz - cz) / hz};
    }
  }
  auto clamp = [](double v) { return v < -1.0 ? -1.0 : (v > 1.0 ? 1.0 : v); };
  best.xi = clamp(best.xi);
  best.eta = clamp(best.eta);
  best.gam = clamp(best.gam);
  return best;
}

template <typename T>
struct Solver {
  oracle_mesh m;
  Gll g;
  int nthreads;
  T D[NG][NG], DW[NG][NG], w[NG];
  T xix, jac;
  std::vector<T> kappa, mu, rho_vp, rho_vs, jw, nrm;
  std::vector<int> colour_start, colour_elems;

  // run state
  double dt = 0.0;
  int nstep = 0;
  std::vector<T> minv;               // [nglob*3]
  std::vector<T> u, v, a;            // forward or adjoint field
  std::vector<T> bu, bv, ba;         // backward field
  std::vector<T> store;              // [nstep][nf][25][3]
  std::vector<T> fin_u, fin_v, fin_a;
  bool have_forward = false;
  // source
  oracle_source src{};
  int src_ispec = -1;
  std::vector<T> srcarr;             // [125][3]
  std::vector<T> stf;                // [nstep]
  // kernels
  std::vector<T> rho_kl_glob, mu_kl, kappa_kl;
  // approximate Hessian sum_j DT a_adj . a_bwd per global point
  // (APPROXIMATE_HESS_KL; read as hess_kernel by post_processing.f90:175)
  std::vector<T> hess_kl_glob;
  // FK injection (forward runs): [inj_nt][nf*25][3] incident velocity and
  // traction, sample k at time (k + inj_k0) * inj_np * dt
  std::vector<double> inj_v, inj_t;
  int inj_nt = 0, inj_np = 1, inj_k0 = 0;

  explicit Solver(const oracle_mesh& mm, int nth) : m(mm), nthreads(nth) {
    g = make_gll();
    for (int i = 0; i < NG; ++i) {
      w[i] = (T)g.w[i];
      for (int l = 0; l < NG; ++l) {
        D[i][l] = (T)g.D[i][l];
        DW[i][l] = (T)(g.w[i] * g.D[i][l]);
      }
    }
    xix = (T)m.xix;
    jac = (T)m.jac;
    size_t ne = (size_t)m.nspec * NG3;
    kappa.assign(m.kappa, m.kappa + ne);
    mu.assign(m.mu, m.mu + ne);
    rho_vp.assign(m.rho_vp, m.rho_vp + ne);
    rho_vs.assign(m.rho_vs, m.rho_vs + ne);
    jw.assign(m.f_jw, m.f_jw + (size_t)m.nf * NG2);
    nrm.assign(m.f_n, m.f_n + (size_t)m.nf * NG2 * 3);
    colour();
  }

  // Greedy element colouring so that elements of one colour share no point:
  // each colour is assembled in parallel without races, deterministically.
  void colour() {
    std::vector<int> col(m.nspec, -1);
    std::vector<std::vector<char>> used;  // per colour: point taken
    int ncol = 0;
    for (int e = 0; e < m.nspec; ++e) {
      int c = 0;
      for (;; ++c) {
        if (c == ncol) {
          used.emplace_back(m.nglob, 0);
          ++ncol;
        }
        bool ok = true;
        for (int p = 0; p < NG3 && ok; ++p)
          if (used[c][m.ibool[e * NG3 + p]]) ok = false;
        if (ok) break;
      }
      col[e] = c;
      for (int p = 0; p < NG3; ++p) used[c][m.ibool[e * NG3 + p]] = 1;
    }
    colour_start.assign(ncol + 1, 0);
    for (int e = 0; e < m.nspec; ++e) colour_start[col[e] + 1]++;
    for (int c = 0; c < ncol; ++c) colour_start[c + 1] += colour_start[c];
    colour_elems.resize(m.nspec);
    std::vector<int> pos(colour_start.begin(), colour_start.end() - 1);
    for (int e = 0; e < m.nspec; ++e) colour_elems[pos[col[e]]++] = e;
  }

  void set_dt(double d) {
    dt = d;
    // M + dt/2 * C_diag, C from the Stacey faces (n axis components)
    std::vector<double> mx((size_t)m.nglob * 3);
    for (int ig = 0; ig < m.nglob; ++ig)
      for (int c = 0; c < 3; ++c) mx[(size_t)ig * 3 + c] = (double)m.rmass[ig];
    for (int f = 0; f < m.nf; ++f) {
      int e = m.f_ispec[f];
      for (int p = 0; p < NG2; ++p) {
        const int* ijk = &m.f_ijk[((size_t)f * NG2 + p) * 3];
        int lp = ijk[0] + NG * ijk[1] + NG2 * ijk[2];
        int ig = m.ibool[e * NG3 + lp];
        double rvp = (double)m.rho_vp[(size_t)e * NG3 + lp];
        double rvs = (double)m.rho_vs[(size_t)e * NG3 + lp];
        double jwd = (double)m.f_jw[(size_t)f * NG2 + p];
        for (int c = 0; c < 3; ++c) {
          double n = (double)m.f_n[((size_t)f * NG2 + p) * 3 + c];
          mx[(size_t)ig * 3 + c] += 0.5 * d * jwd * (rvp * n * n + rvs * (1.0 - n * n));
        }
      }
    }
    minv.resize(mx.size());
    for (size_t i = 0; i < mx.size(); ++i) minv[i] = (T)(1.0 / mx[i]);
  }

  // Element loop: acc -= K u.  Optionally returns strain pieces per element
  // point: eps[e*125+p] = {dev_xx, dev_yy, dev_xy, dev_xz, dev_yz, trace}.
  void forces(const std::vector<T>& uu, std::vector<T>& acc, std::vector<T>* eps) {
    int ncol = (int)colour_start.size() - 1;
    for (int c = 0; c < ncol; ++c) {
#pragma omp parallel for schedule(static) num_threads(nthreads)
      for (int q = colour_start[c]; q < colour_start[c + 1]; ++q) {
        int e = colour_elems[q];
        element(e, uu, acc, eps);
      }
    }
  }

  void element(int e, const std::vector<T>& uu, std::vector<T>& acc, std::vector<T>* eps) {
    const float* gen =
        (m.irreg && m.irreg[e] >= 0) ? m.geo + (size_t)m.irreg[e] * NG3 * 10 : nullptr;
    T ul[3][NG3];
    const int* ib = &m.ibool[(size_t)e * NG3];
    for (int p = 0; p < NG3; ++p)
      for (int c = 0; c < 3; ++c) ul[c][p] = uu[(size_t)ib[p] * 3 + c];
    T t1[3][NG3], t2[3][NG3], t3[3][NG3];
    const T four3 = (T)(4.0 / 3.0);
    for (int k = 0; k < NG; ++k)
      for (int j = 0; j < NG; ++j)
        for (int i = 0; i < NG; ++i) {
          int p = i + NG * j + NG2 * k;
          T dxi[3], det[3], dga[3];
          for (int c = 0; c < 3; ++c) {
            T s1 = 0, s2 = 0, s3 = 0;
            for (int l = 0; l < NG; ++l) {
              s1 += D[i][l] * ul[c][l + NG * j + NG2 * k];
              s2 += D[j][l] * ul[c][i + NG * l + NG2 * k];
              s3 += D[k][l] * ul[c][i + NG * j + NG2 * l];
            }
            dxi[c] = s1;
            det[c] = s2;
            dga[c] = s3;
          }
          T duxdx, duxdy, duxdz, duydx, duydy, duydz, duzdx, duzdy, duzdz;
          const float* G = gen ? gen + (size_t)p * 10 : nullptr;
          if (!G) {
            duxdx = xix * dxi[0], duxdy = xix * det[0], duxdz = xix * dga[0];
            duydx = xix * dxi[1], duydy = xix * det[1], duydz = xix * dga[1];
            duzdx = xix * dxi[2], duzdy = xix * det[2], duzdz = xix * dga[2];
          } else {
            // du_c/dx = xix dxi + etax deta + gammax dgamma, and likewise
            // for y (xiy, etay, gammay) and z (xiz, etaz, gammaz)
            T du[3][3];
            for (int c = 0; c < 3; ++c)
              for (int d = 0; d < 3; ++d)
                du[c][d] = (T)G[d] * dxi[c] + (T)G[3 + d] * det[c] + (T)G[6 + d] * dga[c];
            duxdx = du[0][0], duxdy = du[0][1], duxdz = du[0][2];
            duydx = du[1][0], duydy = du[1][1], duydz = du[1][2];
            duzdx = du[2][0], duzdy = du[2][1], duzdz = du[2][2];
          }
          size_t ep = (size_t)e * NG3 + p;
          T kap = kappa[ep], mul = mu[ep];
          T l2m = kap + four3 * mul;
          T lam = l2m - (T)2 * mul;
          T sxx = l2m * duxdx + lam * (duydy + duzdz);
          T syy = l2m * duydy + lam * (duxdx + duzdz);
          T szz = l2m * duzdz + lam * (duxdx + duydy);
          T sxy = mul * (duxdy + duydx);
          T sxz = mul * (duxdz + duzdx);
          T syz = mul * (duydz + duzdy);
          if (!G) {
            T fac = jac * xix;
            t1[0][p] = fac * sxx; t2[0][p] = fac * sxy; t3[0][p] = fac * sxz;
            t1[1][p] = fac * sxy; t2[1][p] = fac * syy; t3[1][p] = fac * syz;
            t1[2][p] = fac * sxz; t2[2][p] = fac * syz; t3[2][p] = fac * szz;
          } else {
            // flux of component c through the xi, eta, gamma directions:
            // jacobian * sigma_c . (xix, xiy, xiz) etc.
            const T jl = (T)G[9];
            const T sc[3][3] = {{sxx, sxy, sxz}, {sxy, syy, syz}, {sxz, syz, szz}};
            for (int c = 0; c < 3; ++c) {
              t1[c][p] = jl * (sc[c][0] * (T)G[0] + sc[c][1] * (T)G[1] + sc[c][2] * (T)G[2]);
              t2[c][p] = jl * (sc[c][0] * (T)G[3] + sc[c][1] * (T)G[4] + sc[c][2] * (T)G[5]);
              t3[c][p] = jl * (sc[c][0] * (T)G[6] + sc[c][1] * (T)G[7] + sc[c][2] * (T)G[8]);
            }
          }
          if (eps) {
            T tr = duxdx + duydy + duzdz;
            T tr3 = tr / (T)3;
            T* o = &(*eps)[ep * 6];
            o[0] = duxdx - tr3;
            o[1] = duydy - tr3;
            o[2] = (T)0.5 * (duxdy + duydx);
            o[3] = (T)0.5 * (duxdz + duzdx);
            o[4] = (T)0.5 * (duydz + duzdy);
            o[5] = tr;
          }
        }
    for (int k = 0; k < NG; ++k)
      for (int j = 0; j < NG; ++j)
        for (int i = 0; i < NG; ++i) {
          int p = i + NG * j + NG2 * k;
          for (int c = 0; c < 3; ++c) {
            T s1 = 0, s2 = 0, s3 = 0;
            for (int l = 0; l < NG; ++l) {
              s1 += DW[l][i] * t1[c][l + NG * j + NG2 * k];
              s2 += DW[l][j] * t2[c][i + NG * l + NG2 * k];
              s3 += DW[l][k] * t3[c][i + NG * j + NG2 * l];
            }
            T f = -(w[j] * w[k] * s1 + w[i] * w[k] * s2 + w[i] * w[j] * s3);
            acc[(size_t)ib[p] * 3 + c] += f;
          }
        }
  }

  // Stacey traction from velocity vel; acc -= jw t.  mode 0: absorb,
  // mode 1: absorb and save record `rec`, mode 2: subtract stored record.
  // Incident velocity and traction of face point fp at step it: the 4-point
  // Lagrange interpolant in time of the stored samples, indices clamped.
  void injected(int it, size_t fp, T vi[3], T ti[3]) const {
    const size_t npt = (size_t)m.nf * NG2;
    const int i1 = it / inj_np - inj_k0;
    const double x = (double)(it % inj_np) / inj_np;
    const double w[4] = {-x * (x - 1) * (x - 2) / 6, (x + 1) * (x - 1) * (x - 2) / 2,
                         -(x + 1) * x * (x - 2) / 2, (x + 1) * x * (x - 1) / 6};
    double sv[3] = {0, 0, 0}, st[3] = {0, 0, 0};
    for (int q = 0; q < 4; ++q) {
      const int k = std::min(std::max(i1 - 1 + q, 0), inj_nt - 1);
      for (int c = 0; c < 3; ++c) {
        sv[c] += w[q] * inj_v[((size_t)k * npt + fp) * 3 + c];
        st[c] += w[q] * inj_t[((size_t)k * npt + fp) * 3 + c];
      }
    }
    for (int c = 0; c < 3; ++c) {
      vi[c] = (T)sv[c];
      ti[c] = (T)st[c];
    }
  }

  // Stacey faces.  mode 0: absorb; 1: absorb and save the boundary term
  // in store[rec]; 2: subtract store[rec].  it_inj >= 0: the forward step
  // whose incident field is injected (absorb the velocity relative to it,
  // add its traction).
  void stacey(const std::vector<T>& vel, std::vector<T>& acc, int mode, int rec,
              int it_inj = -1) {
    const bool inject = it_inj >= 0 && !inj_v.empty();
    for (int f = 0; f < m.nf; ++f) {
      int e = m.f_ispec[f];
      for (int p = 0; p < NG2; ++p) {
        const int* ijk = &m.f_ijk[((size_t)f * NG2 + p) * 3];
        int lp = ijk[0] + NG * ijk[1] + NG2 * ijk[2];
        size_t ig = (size_t)m.ibool[e * NG3 + lp];
        T* st = store.empty() ? nullptr
                              : &store[(((size_t)rec * m.nf + f) * NG2 + p) * 3];
        if (mode == 2) {
          for (int c = 0; c < 3; ++c) acc[ig * 3 + c] -= st[c];
          continue;
        }
        const T* n = &nrm[((size_t)f * NG2 + p) * 3];
        T vi[3] = {0, 0, 0}, ti[3] = {0, 0, 0};
        if (inject) injected(it_inj, (size_t)f * NG2 + p, vi, ti);
        T vx = vel[ig * 3 + 0] - vi[0], vy = vel[ig * 3 + 1] - vi[1], vz = vel[ig * 3 + 2] - vi[2];
        T vn = vx * n[0] + vy * n[1] + vz * n[2];
        T rvp = rho_vp[(size_t)e * NG3 + lp], rvs = rho_vs[(size_t)e * NG3 + lp];
        T tx = rvp * vn * n[0] + rvs * (vx - vn * n[0]) - ti[0];
        T ty = rvp * vn * n[1] + rvs * (vy - vn * n[1]) - ti[1];
        T tz = rvp * vn * n[2] + rvs * (vz - vn * n[2]) - ti[2];
        T wgt = jw[(size_t)f * NG2 + p];
        T sx = tx * wgt, sy = ty * wgt, sz = tz * wgt;
        acc[ig * 3 + 0] -= sx;
        acc[ig * 3 + 1] -= sy;
        acc[ig * 3 + 2] -= sz;
        if (mode == 1) {
          st[0] = sx;
          st[1] = sy;
          st[2] = sz;
        }
      }
    }
  }

  void setup_source(const oracle_source& s) {
    src = s;
    Located L = locate(m, s.x, s.y, s.z);
    src_ispec = L.ispec;
    // CMT (r,theta,phi) -> (x=E, y=N, z=Up)
    double Mzz = s.mt[0], Myy = s.mt[1], Mxx = s.mt[2];
    double Myz = -s.mt[3], Mxz = s.mt[4], Mxy = -s.mt[5];
    double M[3][3] = {{Mxx, Mxy, Mxz}, {Mxy, Myy, Myz}, {Mxz, Myz, Mzz}};
    srcarr.assign(NG3 * 3, (T)0);
    // d(xi_d)/dx_a at the source: the regular element's xix on the
    // diagonal, or the inverse of the interpolated mapping's Jacobian
    double dxi[3][3] = {{m.xix, 0, 0}, {0, m.xix, 0}, {0, 0, m.xix}};
    if (m.irreg && m.irreg[L.ispec] >= 0) {
      const double xi3[3] = {L.xi, L.eta, L.gam};
      double X[3], dX[3][3];
      element_map(m, g, L.ispec, xi3, X, dX);
      invert3(dX, dxi);
    }
    for (int c3 = 0; c3 < NG; ++c3)
      for (int b = 0; b < NG; ++b)
        for (int a3 = 0; a3 < NG; ++a3) {
          double la = lagrange(g, a3, L.xi), lb = lagrange(g, b, L.eta),
                 lc = lagrange(g, c3, L.gam);
          const double dr[3] = {lagrange_d(g, a3, L.xi) * lb * lc,
                                la * lagrange_d(g, b, L.eta) * lc,
                                la * lb * lagrange_d(g, c3, L.gam)};
          double grad[3];
          for (int a = 0; a < 3; ++a)
            grad[a] = dxi[0][a] * dr[0] + dxi[1][a] * dr[1] + dxi[2][a] * dr[2];
          int p = a3 + NG * b + NG2 * c3;
          for (int r = 0; r < 3; ++r)
            srcarr[p * 3 + r] =
                (T)(M[r][0] * grad[0] + M[r][1] * grad[1] + M[r][2] * grad[2]);
        }
    stf.resize(nstep);
    for (int it = 0; it < nstep; ++it)
      stf[it] = (T)ricker(it * dt - 1.2 / s.f0 - s.tshift, s.f0);
  }

  void add_source(std::vector<T>& acc, int it) {
    T s = stf[it];
    const int* ib = &m.ibool[(size_t)src_ispec * NG3];
    for (int p = 0; p < NG3; ++p)
      for (int c = 0; c < 3; ++c) acc[(size_t)ib[p] * 3 + c] += srcarr[p * 3 + c] * s;
  }

  struct Recv {
    int ispec;
    T wgt[NG3];
  };
  std::vector<Recv> recs;

  void setup_receivers(int nrec, const double* xyz) {
    recs.resize(nrec);
    for (int r = 0; r < nrec; ++r) {
      Located L = locate(m, xyz[r * 3], xyz[r * 3 + 1], xyz[r * 3 + 2]);
      recs[r].ispec = L.ispec;
      for (int c = 0; c < NG; ++c)
        for (int b = 0; b < NG; ++b)
          for (int a3 = 0; a3 < NG; ++a3)
            recs[r].wgt[a3 + NG * b + NG2 * c] =
                (T)(lagrange(g, a3, L.xi) * lagrange(g, b, L.eta) * lagrange(g, c, L.gam));
    }
  }

  void record(const std::vector<T>& uu, double* seis, int it) {
    for (size_t r = 0; r < recs.size(); ++r) {
      const int* ib = &m.ibool[(size_t)recs[r].ispec * NG3];
      for (int c = 0; c < 3; ++c) {
        T s = 0;
        for (int p = 0; p < NG3; ++p) s += recs[r].wgt[p] * uu[(size_t)ib[p] * 3 + c];
        seis[((size_t)r * 3 + c) * nstep + it] = (double)s;
      }
    }
  }

  void predictor(std::vector<T>& uu, std::vector<T>& vv, std::vector<T>& aa, double d) {
    T dtt = (T)d, dt2 = (T)(0.5 * d), dtsq2 = (T)(0.5 * d * d);
    size_t n = uu.size();
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (size_t i = 0; i < n; ++i) {
      uu[i] = uu[i] + dtt * vv[i] + dtsq2 * aa[i];
      vv[i] = vv[i] + dt2 * aa[i];
      aa[i] = 0;
    }
  }

  void corrector(std::vector<T>& vv, std::vector<T>& aa, double d) {
    T dt2 = (T)(0.5 * d);
    size_t n = vv.size();
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (size_t i = 0; i < n; ++i) {
      aa[i] = aa[i] * minv[i];
      vv[i] = vv[i] + dt2 * aa[i];
    }
  }

  int forward(double d, int ns, const oracle_source& s, int nrec, const double* rxyz,
              double* seis, int save) {
    nstep = ns;
    set_dt(d);
    setup_source(s);
    setup_receivers(nrec, rxyz);
    size_t n3 = (size_t)m.nglob * 3;
    u.assign(n3, 0);
    v.assign(n3, 0);
    a.assign(n3, 0);
    store.clear();
    if (save) store.assign((size_t)nstep * m.nf * NG2 * 3, (T)0);
    for (int it = 0; it < nstep; ++it) {
      predictor(u, v, a, dt);
      forces(u, a, nullptr);
      stacey(v, a, save ? 1 : 0, it, it);
      add_source(a, it);
      corrector(v, a, dt);
      if (seis) record(u, seis, it);
    }
    fin_u = u;
    fin_v = v;
    fin_a = a;
    have_forward = save != 0;
    return 0;
  }

  // adjoint + backward with kernel accumulation.  adj: [nrec][3][nstep]
  // (forward-time order), receivers are the adjoint sources.
  int adjoint(int nrec, const double* rxyz, const double* adj, double* kern,
              double* bseis, double* aseis) {
    if (!have_forward) return 3;
    setup_receivers(nrec, rxyz);
    size_t n3 = (size_t)m.nglob * 3;
    size_t ne = (size_t)m.nspec * NG3;
    u.assign(n3, 0);
    v.assign(n3, 0);
    a.assign(n3, 0);
    bu = fin_u;
    bv = fin_v;
    ba = fin_a;
    rho_kl_glob.assign(m.nglob, 0);
    hess_kl_glob.assign(m.nglob, 0);
    mu_kl.assign(ne, 0);
    kappa_kl.assign(ne, 0);
    std::vector<T> eps_a(ne * 6), eps_b(ne * 6), scratch(n3);
    const int N = nstep;
    const T tdt = (T)dt;
    for (int j = 0; j < N; ++j) {
      // adjoint step j
      predictor(u, v, a, dt);
      forces(u, a, &eps_a);
      stacey(v, a, 0, 0);
      for (int r = 0; r < nrec; ++r) {
        const int* ib = &m.ibool[(size_t)recs[r].ispec * NG3];
        for (int c = 0; c < 3; ++c) {
          T s = (T)adj[((size_t)r * 3 + c) * N + (N - 1 - j)];
          for (int p = 0; p < NG3; ++p) a[(size_t)ib[p] * 3 + c] += recs[r].wgt[p] * s;
        }
      }
      corrector(v, a, dt);
      if (aseis) record(u, aseis, j);
      // strain of the backward state N-1-j (forces discarded)
      std::fill(scratch.begin(), scratch.end(), (T)0);
      forces(bu, scratch, &eps_b);
      if (bseis) record(bu, bseis, N - 1 - j);
      // kernel accumulation
#pragma omp parallel for schedule(static) num_threads(nthreads)
      for (int ig = 0; ig < m.nglob; ++ig) {
        size_t q = (size_t)ig * 3;
        rho_kl_glob[ig] += tdt * (a[q] * bu[q] + a[q + 1] * bu[q + 1] + a[q + 2] * bu[q + 2]);
        hess_kl_glob[ig] += tdt * (a[q] * ba[q] + a[q + 1] * ba[q + 1] + a[q + 2] * ba[q + 2]);
      }
#pragma omp parallel for schedule(static) num_threads(nthreads)
      for (size_t ep = 0; ep < ne; ++ep) {
        const T* ea = &eps_a[ep * 6];
        const T* eb = &eps_b[ep * 6];
        T dd = ea[0] * eb[0] + ea[1] * eb[1] + (ea[0] + ea[1]) * (eb[0] + eb[1]) +
               (T)2 * (ea[2] * eb[2] + ea[3] * eb[3] + ea[4] * eb[4]);
        mu_kl[ep] += tdt * dd;
        kappa_kl[ep] += tdt * (ea[5] * eb[5]);
      }
      // backward step reconstructing state N-2-j
      if (j < N - 1) {
        int n = N - 2 - j;
        predictor(bu, bv, ba, -dt);
        forces(bu, ba, nullptr);
        if (!store.empty()) stacey(bv, ba, 2, n);
        {
          T s = stf[n];
          const int* ib = &m.ibool[(size_t)src_ispec * NG3];
          for (int p = 0; p < NG3; ++p)
            for (int c = 0; c < 3; ++c) ba[(size_t)ib[p] * 3 + c] += srcarr[p * 3 + c] * s;
        }
        corrector(bv, ba, -dt);
      }
    }
    finalize_kernels(kern);
    return 0;
  }

  // rho/mu/kappa scaled as in Tromp, Tape & Liu (2005) and the derived
  // rhop/beta/alpha kernels; layout kern[6][nspec*125].
  void finalize_kernels(double* kern) {
    size_t ne = (size_t)m.nspec * NG3;
    for (size_t ep = 0; ep < ne; ++ep) {
      double rho = m.rho[ep], muv = m.mu[ep], kap = m.kappa[ep];
      double rk = -rho * (double)rho_kl_glob[m.ibool[ep]];
      double mk = -2.0 * muv * (double)mu_kl[ep];
      double kk = -kap * (double)kappa_kl[ep];
      kern[0 * ne + ep] = rk;
      kern[1 * ne + ep] = mk;
      kern[2 * ne + ep] = kk;
      kern[3 * ne + ep] = rk + kk + mk;
      kern[4 * ne + ep] = 2.0 * (mk - 4.0 / 3.0 * muv / kap * kk);
      kern[5 * ne + ep] = 2.0 * (1.0 + 4.0 / 3.0 * muv / kap) * kk;
    }
  }

  // kinetic + strain energy of the current forward field (uses M, not the
  // Stacey-augmented mass)
  double energy() {
    size_t n3 = (size_t)m.nglob * 3;
    std::vector<T> f(n3, 0);
    forces(u, f, nullptr);
    double ek = 0, ep = 0;
    for (int ig = 0; ig < m.nglob; ++ig)
      for (int c = 0; c < 3; ++c) {
        size_t q = (size_t)ig * 3 + c;
        ek += 0.5 * (double)m.rmass[ig] * (double)v[q] * (double)v[q];
        ep -= 0.5 * (double)u[q] * (double)f[q];
      }
    return ek + ep;
  }
};

// ---------------------------------------------------------------------------
// PDE smoothing of element fields: the CPU branch of smooth_sem_pde
// (src/postproc/smooth.f90:7-437) restated in precision T.
//
// Steps, in the reference's order:
//   * rotate_r = x/|x| at every element point                (smooth.f90:81-94)
//   * cmax = dmin^2/9, cv/ch from sigma_v/sigma_h, ntstep     (smooth.f90:99-109)
//     (always in FP32, CUSTOM_REAL, so both precisions take the same steps)
//   * rvol_local = real(dble(jac) * w_i w_j w_k); rvol = 1 / sum (smooth.f90:142-164)
//   * project: dat_glob = sum(dat * rvol_local) * rvol        (smooth.f90:193-214)
//   * per step: ddat = 0; per element the gradient with hprime_xxT, the
//     fluxes stemp1..3, the divergence with hprimewgll and wgllwgll
//     weights, ddat -= ...; then ddat *= rvol, dat_glob += ddat, and
//     points of CPML elements reset to dat_bak = 0 (ZERO_PML)   (smooth.f90:244-370)
//   * output dat(e) = dat_glob(ibool(e))
// Irregular elements (m.irreg[e] >= 0) take their nine mapping terms and
// Jacobian at each point from m.geo, in the fluxes and in rvol_local
// (smooth.f90:142-164 and the ispec_irreg branch :255-268).  For regular
// elements, mapping 1 reproduces the reference's regular branch, where all
// nine derivative terms (xix .. gammaz) are xix_regular (smooth.f90:269-279,
// get_gradient_element_regular :648-689); mapping 0 uses the cube's
// diagonal mapping (xix = etay = gammaz = xix_regular, zero off the
// diagonal).
// ---------------------------------------------------------------------------

struct SmoothParams {
  float cv, ch, cmax;
  int nstep;
};

SmoothParams smooth_params(double sigma_h, double sigma_v, double dmin, int nstep_override) {
  SmoothParams q{};
  const float sh = (float)sigma_h, sv = (float)sigma_v, d = (float)dmin;
  q.cmax = d * d / 9.0f;
  if (sv >= sh) {
    q.cv = q.cmax;
    q.ch = q.cv * (sh * sh) / (sv * sv);
  } else {
    q.ch = q.cmax;
    q.cv = q.ch * (sv * sv) / (sh * sh);
  }
  const float mx = sh > sv ? sh : sv;
  q.nstep = (int)std::ceil(mx * mx / (2.0f * q.cmax));
  if (nstep_override > 0) q.nstep = nstep_override;
  return q;
}

template <typename T>
void smooth_run(const oracle_mesh& m, int nfield, const float* dat_in, const int* is_cpml,
                const SmoothParams& q, int is_sph, int mapping, double* out) {
  const Gll g = make_gll();
  T D[NG][NG], DWt[NG][NG];
  for (int i = 0; i < NG; ++i) {
    for (int l = 0; l < NG; ++l) {
      D[i][l] = (T)g.D[i][l];              // hprime_xxT(l,i) = hprime_xx(i,l)
      DWt[i][l] = (T)(g.w[l] * g.D[l][i]); // hprimewgll_xx(l,i)
    }
  }
  const T xix = (T)(float)m.xix, jac_reg = (T)(float)m.jac;
  const T cv = (T)q.cv, ch = (T)q.ch;
  // mapping rows of a regular element: derivative terms of xi, eta, gamma
  // along x, y, z
  T Mreg[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) Mreg[a][b] = (mapping == 1 || a == b) ? xix : (T)0;
  const size_t ne = (size_t)m.nspec * NG3;
  // mapping row of an irregular element, or null
  auto geo_of = [&](int e) -> const float* {
    return (m.irreg && m.irreg[e] >= 0) ? m.geo + (size_t)m.irreg[e] * NG3 * 10 : nullptr;
  };
  std::vector<T> rvol_local(ne), rvol(m.nglob, (T)0);
  for (int e = 0; e < m.nspec; ++e) {
    const float* G = geo_of(e);
    for (int k = 0; k < NG; ++k)
      for (int j = 0; j < NG; ++j)
        for (int i = 0; i < NG; ++i) {
          const int p = i + NG * j + NG2 * k;
          const double weight = g.w[i] * g.w[j] * g.w[k];
          const float jacobianl = G ? G[p * 10 + 9] : (float)m.jac;
          rvol_local[(size_t)e * NG3 + p] = (T)((double)jacobianl * weight);
        }
  }
  for (int e = 0; e < m.nspec; ++e)
    for (int p = 0; p < NG3; ++p) rvol[m.ibool[e * NG3 + p]] += rvol_local[(size_t)e * NG3 + p];
  for (int ig = 0; ig < m.nglob; ++ig) rvol[ig] = (T)1 / rvol[ig];
  std::vector<char> cpml_pt(m.nglob, 0);
  if (is_cpml)
    for (int e = 0; e < m.nspec; ++e)
      if (is_cpml[e])
        for (int p = 0; p < NG3; ++p) cpml_pt[m.ibool[e * NG3 + p]] = 1;
  std::vector<T> rx, ry, rz;
  if (is_sph) {
    rx.resize(m.nglob);
    ry.resize(m.nglob);
    rz.resize(m.nglob);
    for (int ig = 0; ig < m.nglob; ++ig) {
      const T xl = (T)m.x[ig], yl = (T)m.y[ig], zl = (T)m.z[ig];
      const T rl = std::sqrt(xl * xl + yl * yl + zl * zl);
      rx[ig] = xl / rl;
      ry[ig] = yl / rl;
      rz[ig] = zl / rl;
    }
  }
  std::vector<T> dat_glob(m.nglob), ddat(m.nglob);
  for (int f = 0; f < nfield; ++f) {
    const float* din = dat_in + (size_t)f * ne;
    std::fill(dat_glob.begin(), dat_glob.end(), (T)0);
    for (int e = 0; e < m.nspec; ++e)
      for (int p = 0; p < NG3; ++p)
        dat_glob[m.ibool[e * NG3 + p]] +=
            (T)din[(size_t)e * NG3 + p] * rvol_local[(size_t)e * NG3 + p];
    for (int ig = 0; ig < m.nglob; ++ig) dat_glob[ig] = dat_glob[ig] * rvol[ig];
    for (int it = 0; it < q.nstep; ++it) {
      std::fill(ddat.begin(), ddat.end(), (T)0);
      for (int e = 0; e < m.nspec; ++e) {
        const int* ib = &m.ibool[(size_t)e * NG3];
        const float* G = geo_of(e);
        T s[NG3], st1[NG3], st2[NG3], st3[NG3];
        for (int p = 0; p < NG3; ++p) s[p] = dat_glob[ib[p]];
        for (int k = 0; k < NG; ++k)
          for (int j = 0; j < NG; ++j)
            for (int i = 0; i < NG; ++i) {
              T M[3][3];
              T jac = jac_reg;
              const int pq = i + NG * j + NG2 * k;
              for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b)
                  M[a][b] = G ? (T)G[pq * 10 + 3 * a + b] : Mreg[a][b];
              if (G) jac = (T)G[pq * 10 + 9];
              T t1 = 0, t2 = 0, t3 = 0;
              for (int l = 0; l < NG; ++l) t1 += s[l + NG * j + NG2 * k] * D[i][l];
              for (int l = 0; l < NG; ++l) t2 += s[i + NG * l + NG2 * k] * D[j][l];
              for (int l = 0; l < NG; ++l) t3 += s[i + NG * j + NG2 * l] * D[k][l];
              const T dx = t1 * M[0][0] + t2 * M[1][0] + t3 * M[2][0];
              const T dy = t1 * M[0][1] + t2 * M[1][1] + t3 * M[2][1];
              const T dz = t1 * M[0][2] + t2 * M[1][2] + t3 * M[2][2];
              const int p = i + NG * j + NG2 * k;
              T* st[3] = {st1, st2, st3};
              for (int a = 0; a < 3; ++a) {
                T v;
                if (is_sph) {
                  const T r0 = rx[ib[p]], r1 = ry[ib[p]], r2 = rz[ib[p]];
                  v = ((cv - ch) * (r0 * M[a][0] + r1 * M[a][1] + r2 * M[a][2]) *
                           (r0 * dx + r1 * dy + r2 * dz) +
                       ch * (M[a][0] * dx + M[a][1] * dy + M[a][2] * dz)) *
                      jac;
                } else {
                  v = ((cv - ch) * M[a][2] * dz + ch * (M[a][0] * dx + M[a][1] * dy + M[a][2] * dz)) *
                      jac;
                }
                st[a][p] = v;
              }
            }
        for (int k = 0; k < NG; ++k)
          for (int j = 0; j < NG; ++j)
            for (int i = 0; i < NG; ++i) {
              T n1 = 0, n2 = 0, n3 = 0;
              for (int l = 0; l < NG; ++l) {
                n1 += st1[l + NG * j + NG2 * k] * DWt[i][l];
                n2 += st2[i + NG * l + NG2 * k] * DWt[j][l];
                n3 += st3[i + NG * j + NG2 * l] * DWt[k][l];
              }
              // wgllwgll_yz(j,k), wgllwgll_xz(i,k), wgllwgll_xy(i,j)
              const T fac1 = (T)(g.w[j] * g.w[k]), fac2 = (T)(g.w[i] * g.w[k]),
                      fac3 = (T)(g.w[i] * g.w[j]);
              const int p = i + NG * j + NG2 * k;
              ddat[ib[p]] -= fac1 * n1 + fac2 * n2 + fac3 * n3;
            }
      }
      for (int ig = 0; ig < m.nglob; ++ig) {
        dat_glob[ig] += ddat[ig] * rvol[ig];
        if (cpml_pt[ig]) dat_glob[ig] = (T)0;
      }
    }
    double* o = out + (size_t)f * ne;
    for (size_t i = 0; i < ne; ++i) o[i] = (double)dat_glob[m.ibool[i]];
  }
}

struct Handle {
  int prec;
  std::unique_ptr<Solver<float>> s32;
  std::unique_ptr<Solver<double>> s64;
  int nthreads = 1;
  int flush = 0;  // flush subnormals to zero during runs (x86 FTZ + DAZ)
};

// Subnormal FP32 values (below 1.2e-38: the numerical tail ahead of a
// wavefront, products of two small strains) make x86 cores 10-100x slower.
// A scope that sets FTZ and DAZ on the calling thread and on the OpenMP
// pool's threads for the duration of one run, and restores them after.
// It changes nothing above 1.2e-38, i.e. nothing a relative L2 norm of a
// seismogram or kernel can see; the FP64 oracle never needs it.
struct FlushScope {
  int nthreads;
  bool on;
  FlushScope(bool on_, int nt) : nthreads(nt), on(on_) {
    if (on) set(true);
  }
  ~FlushScope() {
    if (on) set(false);
  }
  void set(bool v) const {
#pragma omp parallel num_threads(nthreads)
    {
      unsigned c = _mm_getcsr();
      _mm_setcsr(v ? (c | 0x8040u) : (c & ~0x8040u));
    }
    unsigned c = _mm_getcsr();
    _mm_setcsr(v ? (c | 0x8040u) : (c & ~0x8040u));
  }
};

}  // namespace

extern "C" {

void* oracle_create(const oracle_mesh* m, int precision, int nthreads) {
  if (!m || (precision != 4 && precision != 8)) return nullptr;
  if (nthreads <= 0) nthreads = 1;
  auto* h = new Handle{precision, nullptr, nullptr};
  h->nthreads = nthreads;
  if (precision == 4)
    h->s32.reset(new Solver<float>(*m, nthreads));
  else
    h->s64.reset(new Solver<double>(*m, nthreads));
  return h;
}

void oracle_destroy(void* p) { delete (Handle*)p; }

// Flush FP32 subnormals to zero in this handle's runs (speed only; see
// FlushScope).
int oracle_set_flush_subnormals(void* p, int on) {
  auto* h = (Handle*)p;
  if (!h) return 1;
  h->flush = on ? 1 : 0;
  return 0;
}

int oracle_forward(void* p, double dt, int nstep, const oracle_source* s, int nrec,
                   const double* rxyz, double* seis, int save_forward) {
  auto* h = (Handle*)p;
  if (!h || !s || nstep <= 0) return 1;
  FlushScope fs(h->flush != 0, h->nthreads);
  return h->prec == 4 ? h->s32->forward(dt, nstep, *s, nrec, rxyz, seis, save_forward)
                      : h->s64->forward(dt, nstep, *s, nrec, rxyz, seis, save_forward);
}

int oracle_adjoint(void* p, int nrec, const double* rxyz, const double* adj, double* kern,
                   double* bseis, double* aseis) {
  auto* h = (Handle*)p;
  if (!h || !adj || !kern) return 1;
  FlushScope fs(h->flush != 0, h->nthreads);
  return h->prec == 4 ? h->s32->adjoint(nrec, rxyz, adj, kern, bseis, aseis)
                      : h->s64->adjoint(nrec, rxyz, adj, kern, bseis, aseis);
}

// hess_kernel of the last adjoint run, out[nspec*125]: twice the
// accumulated sum at each element point (the approximate Hessian's scaling
// by 2; a positive factor cancels in the preconditioner).
int oracle_get_hessian(void* p, double* out) {
  auto* h = (Handle*)p;
  if (!h || !out) return 1;
  auto copy = [&](auto& s) {
    if (s.hess_kl_glob.empty()) return 2;
    const size_t ne = (size_t)s.m.nspec * 125;
    for (size_t ep = 0; ep < ne; ++ep) out[ep] = 2.0 * (double)s.hess_kl_glob[s.m.ibool[ep]];
    return 0;
  };
  return h->prec == 4 ? copy(*h->s32) : copy(*h->s64);
}

// FK injection for the next forward runs: [nt][nf*25][3] velocity and
// traction, sample k at time (k + k0) * np_resamp * dt; veloc = null clears.
int oracle_set_injection(void* p, int nt, int np_resamp, int k0, const double* veloc,
                         const double* tract) {
  auto* h = (Handle*)p;
  if (!h) return 1;
  auto set = [&](auto& s) {
    if (!veloc) {
      s.inj_v.clear();
      s.inj_t.clear();
      return 0;
    }
    if (!tract || nt < 1 || np_resamp < 1) return 2;
    const size_t n = (size_t)nt * s.m.nf * 25 * 3;
    s.inj_v.assign(veloc, veloc + n);
    s.inj_t.assign(tract, tract + n);
    s.inj_nt = nt;
    s.inj_np = np_resamp;
    s.inj_k0 = k0;
    return 0;
  };
  return h->prec == 4 ? set(*h->s32) : set(*h->s64);
}

double oracle_energy(void* p) {
  auto* h = (Handle*)p;
  return h->prec == 4 ? h->s32->energy() : h->s64->energy();
}

// which: 0..2 = forward/adjoint u,v,a; 3..5 = backward u,v,a; 6 = minv
int oracle_get_field(void* p, int which, double* out) {
  auto* h = (Handle*)p;
  auto copy = [&](auto& s) {
    const auto* src = which == 0 ? &s.u : which == 1 ? &s.v : which == 2 ? &s.a
                    : which == 3 ? &s.bu : which == 4 ? &s.bv : which == 5 ? &s.ba
                    : &s.minv;
    for (size_t i = 0; i < src->size(); ++i) out[i] = (double)(*src)[i];
    return (int)src->size();
  };
  return h->prec == 4 ? copy(*h->s32) : copy(*h->s64);
}

// Forward run that also returns the energy after every `every` steps
// (energy[k] after step (k+1)*every - 1).
int oracle_forward_energy(void* p, double dt, int nstep, const oracle_source* s, int every,
                          double* energy) {
  auto* h = (Handle*)p;
  auto run = [&](auto& S) {
    S.nstep = nstep;
    S.set_dt(dt);
    S.setup_source(*s);
    size_t n3 = (size_t)S.m.nglob * 3;
    S.u.assign(n3, 0);
    S.v.assign(n3, 0);
    S.a.assign(n3, 0);
    S.store.clear();
    int k = 0;
    for (int it = 0; it < nstep; ++it) {
      S.predictor(S.u, S.v, S.a, dt);
      S.forces(S.u, S.a, nullptr);
      S.stacey(S.v, S.a, 0, it);
      S.add_source(S.a, it);
      S.corrector(S.v, S.a, dt);
      if ((it + 1) % every == 0) energy[k++] = S.energy();
    }
    return 0;
  };
  return h->prec == 4 ? run(*h->s32) : run(*h->s64);
}

int oracle_source_element(void* p, double x, double y, double z, double* xi3) {
  auto* h = (Handle*)p;
  const oracle_mesh& m = h->prec == 4 ? h->s32->m : h->s64->m;
  Located L = locate(m, x, y, z);
  xi3[0] = L.xi;
  xi3[1] = L.eta;
  xi3[2] = L.gam;
  return L.ispec;
}

// PDE smoothing (see smooth_run): dat_in/out are [nfield][nspec][125];
// is_cpml may be null.  Returns the step count, or -1 on bad arguments.
int oracle_smooth_pde(const oracle_mesh* m, int precision, int nfield, const float* dat_in,
                      const int* is_cpml, double sigma_h, double sigma_v, double dmin,
                      int is_sph, int mapping, int nstep_override, double* out, double* cvch) {
  if (!m || !dat_in || !out || nfield < 1 || !(dmin > 0.0)) return -1;
  const SmoothParams q = smooth_params(sigma_h, sigma_v, dmin, nstep_override);
  if (cvch) {
    cvch[0] = q.cv;
    cvch[1] = q.ch;
  }
  if (precision == 4)
    smooth_run<float>(*m, nfield, dat_in, is_cpml, q, is_sph, mapping, out);
  else
    smooth_run<double>(*m, nfield, dat_in, is_cpml, q, is_sph, mapping, out);
  return q.nstep;
}

}  // extern "C"
