// Waveform measurement with the reference's pre-processing, on the device.
//
// Replaces LEQData%measure_adj for the waveform (L2) misfit
// (src/preproc/leq_data.f90:48-188) with one window per trace and band:
//   obs  interpolate onto the synthetic axis   signal.f90:85-125
//        detrend, demean                         signal.f90:382-417
//        Hann taper taper_per                    signal.f90:419-491, config.f90:69
//        Butterworth band-pass                   signal.f90:7-36 (xapiir)
//   syn  rotation E,N -> R,T by back-azimuth     syn_data.f90:64-66, common.f90:136-152
//        Hann taper, band-pass
//   L2   tapered window cut, misfit 0.5 simpson((s-d)^2), adjoint taper(s-d)
//                                                waveform_misfit.f90:15-64
//        band-pass of the adjoint source, cut and taper to the window
//                                                adjoint_source.f90:92-114
//        times src_weight                        leq_data.f90:156-164
//   sum (or normalised sum) over bands, rotation Z,R,T -> Z,N,E
//                                                noise_data.f90:213-252, common.f90:272-291
// Everything runs in FP64.  The reference band-passes in FP32 (bandpass_dp
// converts to single precision for xapiir); its Butterworth design (analog
// prototype, tangent-warped edges, low-pass to band-pass transform, gain 1
// at the band centre, bilinear transform) is restated here in FP64 and the
// sections run in FP64, which removes the FP32 rounding the low band edge
// amplifies (poles within 1e-3 of z = 1 at 50 s periods and 0.02 s steps).
//
// Layout: one thread per (band, trace) runs the trace's whole chain
// sequentially (the IIR recurrences are serial in time); traces are
// [band][trace][3][nstep] FP64 in scratch.  A second kernel, one thread per
// (receiver, sample), combines the bands, rotates back and writes the FP32
// adjoint source the time loop injects.

#include <cmath>
#include <complex>
#include <cstdio>
#include <vector>

#include "sem_b200.h"
#include "sem_internal.cuh"

static_assert(sem::kMeasMaxBands == SEM_MEAS_MAX_BANDS, "band count of the C ABI");

namespace sem {

int design_bandpass(int order, double flo, double fhi, double dt, MeasBand* out) {
  if (order < 1 || order > 10) return report_error(SEM_ERR_ARG, "band-pass order must be 1..10");
  if (!(flo > 0.0) || !(fhi > flo) || !(fhi * dt < 0.5))
    return report_error(SEM_ERR_ARG,
                        "band %g-%g Hz is not inside (0, Nyquist %g Hz) with low < high", flo,
                        fhi, 0.5 / dt);
  using cd = std::complex<double>;
  const double pi = M_PI;
  std::vector<cd> poles;
  std::vector<int> real_pole;
  const int half = order / 2;
  if (2 * half < order) {
    poles.push_back(cd(-1.0, 0.0));
    real_pole.push_back(1);
  }
  for (int k = 1; k <= half; ++k) {
    const double ang = pi * (0.5 + (2.0 * k - 1.0) / (2.0 * order));
    poles.push_back(cd(std::cos(ang), std::sin(ang)));
    real_pole.push_back(0);
  }
  // band edges warped for the bilinear map s = (1 - z^-1)/(1 + z^-1)
  const double flw = std::tan(pi * flo * dt) / (2.0 * pi);
  const double fhw = std::tan(pi * fhi * dt) / (2.0 * pi);
  const double A = 4.0 * pi * pi * flw * fhw;
  const double B = 2.0 * pi * (fhw - flw);
  // analog sections: numerator n0 + n1 s + n2 s^2, denominator likewise
  std::vector<double> sn, sd;
  for (size_t i = 0; i < poles.size(); ++i) {
    if (!real_pole[i]) {
      const cd bp = B * poles[i];
      const cd c = std::sqrt(bp * bp - 4.0 * A);
      const cd q[2] = {0.5 * (bp + c), 0.5 * (bp - c)};
      for (const cd& qq : q) {
        sn.insert(sn.end(), {0.0, B, 0.0});
        sd.insert(sd.end(), {std::norm(qq), -2.0 * qq.real(), 1.0});
      }
    } else {
      sn.insert(sn.end(), {0.0, B, 0.0});
      sd.insert(sd.end(), {A, -B * poles[i].real(), 1.0});
    }
  }
  const int ns = (int)sn.size() / 3;
  if (ns > kMeasMaxSections) return report_error(SEM_ERR_ARG, "too many filter sections");
  // unit gain at the geometric band centre s = i sqrt(A)
  const cd s(0.0, std::sqrt(A));
  cd h(1.0, 0.0);
  for (int j = 0; j < ns; ++j)
    h *= ((sn[3 * j + 2] * s + sn[3 * j + 1]) * s + sn[3 * j]) /
         ((sd[3 * j + 2] * s + sd[3 * j + 1]) * s + sd[3 * j]);
  const double scale = 1.0 / std::abs(h);
  for (int k = 0; k < 3; ++k) sn[k] *= scale;
  out->nsect = ns;
  for (int j = 0; j < ns; ++j) {
    const double a0 = sd[3 * j], a1 = sd[3 * j + 1], a2 = sd[3 * j + 2];
    const double b0 = sn[3 * j], b1 = sn[3 * j + 1], b2 = sn[3 * j + 2];
    const double sc = a2 + a1 + a0;
    out->b0[j] = (b2 + b1 + b0) / sc;
    out->b1[j] = 2.0 * (b0 - b2) / sc;
    out->b2[j] = (b2 - b1 + b0) / sc;
    out->a1[j] = 2.0 * (a0 - a2) / sc;
    out->a2[j] = (a2 - a1 + a0) / sc;
  }
  return SEM_OK;
}

namespace {

// window_taper weight of sample k (0-based) of an n-sample trace
__device__ double taper_weight(int k, int n, double pct, int type) {
  const int frac = (pct == 0.0 || pct == 1.0) ? (int)(n * pct / 2.0) : (int)(n * pct / 2.0 + 0.5);
  if (frac <= 0) return 1.0;
  double x;
  if (k < frac)
    x = (double)k;
  else if (k >= n - frac)
    x = (double)(frac + k - (n - frac));
  else
    return 1.0;
  const double den = 2.0 * frac - 1.0;
  switch (type) {
    case 1: return 0.5 - 0.5 * cos(2.0 * M_PI * x / den);
    case 2: return 0.54 - 0.46 * cos(2.0 * M_PI * x / den);
    case 3: return cos(M_PI * x / den - M_PI / 2.0);
    default: return 1.0 - pow(cos(M_PI * x / den), 10.0);
  }
}

// weight of sample k in simpson(y, dx) of utils.f90:1635-1663, including
// the weight 1 + 2 its even-count branch gives sample n-2 (0-based)
__device__ double simpson_weight(int k, int n, double dx) {
  double s = 0.0;
  if (n < 2) return 0.0;
  if (n % 2 == 0) {
    if (k == 0) s += dx / 3.0;
    if (k == n - 2) s += dx / 3.0;
    if ((k & 1) && k >= 1 && k <= n - 3) s += 4.0 * dx / 3.0;
    if (!(k & 1) && k >= 2 && k <= n - 2) s += 2.0 * dx / 3.0;
    if (k == n - 2) s += 0.5 * dx;
    if (k == n - 1) s += 0.5 * dx;
  } else {
    if (k == 0) s += dx / 3.0;
    if (k == n - 1) s += dx / 3.0;
    if ((k & 1) && k >= 1 && k <= n - 2) s += 4.0 * dx / 3.0;
    if (!(k & 1) && k >= 2 && k <= n - 3) s += 2.0 * dx / 3.0;
  }
  return s;
}

// Cascade of second-order sections over x[0..n), forward then (passes 2)
// backward; per sample the sections run in turn, which gives the same
// values as running each section over the whole trace.
__device__ void iir(double* x, int n, const MeasBand& b, int passes) {
  for (int pass = 0; pass < passes; ++pass) {
    double x1[kMeasMaxSections], x2[kMeasMaxSections], y1[kMeasMaxSections], y2[kMeasMaxSections];
#pragma unroll
    for (int j = 0; j < kMeasMaxSections; ++j) x1[j] = x2[j] = y1[j] = y2[j] = 0.0;
    for (int q = 0; q < n; ++q) {
      const int i = pass == 0 ? q : n - 1 - q;
      double v = x[i];
#pragma unroll
      for (int j = 0; j < kMeasMaxSections; ++j) {
        if (j < b.nsect) {
          double o = b.b0[j] * v + b.b1[j] * x1[j] + b.b2[j] * x2[j];
          o = o - (b.a1[j] * y1[j] + b.a2[j] * y2[j]);
          y2[j] = y1[j];
          y1[j] = o;
          x2[j] = x1[j];
          x1[j] = v;
          v = o;
        }
      }
      x[i] = v;
    }
  }
}

__global__ void __launch_bounds__(64) k_meas_trace(MeasParams P, const float* __restrict__ seis,
                                                   const double* __restrict__ obs,
                                                   const double* __restrict__ win,
                                                   const double* __restrict__ baz, double* scratch,
                                                   double* amax, double* mis) {
  __shared__ MeasBand sband[kMeasMaxBands];
  if (threadIdx.x < kMeasMaxBands) sband[threadIdx.x] = P.band[threadIdx.x];
  __syncthreads();
  const int ntr = P.nrec * 3;
  const int nb = P.nband > 0 ? P.nband : 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nb * ntr) return;
  const int band = t / ntr, tr = t - band * ntr;
  const int rec = tr / 3, comp = tr - rec * 3;
  const int n = P.nstep;
  double* d = scratch + (size_t)t * 3 * n;
  double* s = d + n;
  double* a = s + n;
  // observed: interpolation onto the synthetic axis, detrend, demean
  const double* ob = obs + (size_t)tr * P.obs_npts;
  const double t1 = P.obs_tbeg, dt1 = P.obs_dt, t2 = -P.t0;
  const double tend = t1 + (P.obs_npts - 1) * dt1;
  double ds1 = 0.0, ds2 = 0.0;
  for (int i = 0; i < n; ++i) {
    const double time = t2 + i * P.dt;
    double v = 0.0;
    if (time > t1 && time < tend) {
      int ii = (int)floor((time - t1) / dt1);
      if (ii > P.obs_npts - 2) ii = P.obs_npts - 2;
      if (ii < 0) ii = 0;
      const double tt = time - (ii * dt1 + t1);
      v = (ob[ii + 1] - ob[ii]) * tt / dt1 + ob[ii];
    }
    d[i] = v;
    ds1 += v;
    ds2 += ds1;
  }
  const double dan = (double)n;
  const double davei = 0.5 * (dan + 1.0), davex = ds1 / dan;
  const double dslope = -12.0 * (ds2 - davei * ds1) / (dan * (dan * dan - 1.0));
  double sum = 0.0;
  for (int i = 0; i < n; ++i) {
    const double v = d[i] - davex - dslope * ((double)i - davei);
    d[i] = v;
    sum += v;
  }
  const double mean = sum / dan;
  // synthetic, rotated to Z, R, T when asked
  const float* sr = seis + (size_t)rec * 3 * n;
  double sb = 0.0, cb = 0.0;
  if (P.rotate) {
    const double b = baz[rec] * (M_PI / 180.0);
    sb = sin(b);
    cb = cos(b);
  }
  for (int i = 0; i < n; ++i) {
    const double w = taper_weight(i, n, P.pre_taper, 1);
    d[i] = (d[i] - mean) * w;
    double v;
    if (!P.rotate) {
      v = (double)sr[(size_t)comp * n + i];
    } else {
      const double e = sr[i], nn = sr[(size_t)n + i], z = sr[(size_t)2 * n + i];
      v = comp == 0 ? z : (comp == 1 ? -e * sb - nn * cb : -e * cb + nn * sb);
    }
    s[i] = v * w;
  }
  if (P.nband > 0) {
    iir(d, n, sband[band], P.passes);
    iir(s, n, sband[band], P.passes);
  }
  // window of this trace and band
  const double* wv = win + ((size_t)band * ntr + tr) * 2;
  const int wb = (int)((wv[0] + P.t0) / P.dt);      // nb - 1
  const int we = (int)((wv[1] + P.t0) / P.dt);      // ne
  const int nw = we - wb;
  double m = 0.0;
  for (int i = 0; i < n; ++i) a[i] = 0.0;
  if (!(wv[0] + P.t0 >= 0.0) || nw < 1 || we > n) {
    // a window the host could not check (device-buffer form): no
    // contribution, and a NaN misfit that tells the caller
    mis[t] = NAN;
    amax[t] = 0.0;
    return;
  }
  for (int k = 0; k < nw; ++k) {
    const double w = taper_weight(k, nw, P.win_taper, P.win_taper_type);
    const double r = s[wb + k] * w - d[wb + k] * w;
    m += simpson_weight(k, nw, P.dt) * r * r;
    a[wb + k] = r * w;
  }
  if (P.nband > 0) iir(a, n, sband[band], P.passes);
  double mx = 0.0;
  for (int i = 0; i < n; ++i) {
    const int k = i - wb;
    const double v = (k >= 0 && k < nw) ? a[i] * taper_weight(k, nw, P.win_taper, P.win_taper_type) *
                                              P.weight
                                        : 0.0;
    a[i] = v;
    mx = fmax(mx, fabs(v));
  }
  mis[t] = 0.5 * m * P.weight;
  amax[t] = mx;
}

__global__ void k_meas_combine(MeasParams P, const double* __restrict__ scratch,
                               const double* __restrict__ amax, const double* __restrict__ baz,
                               float* __restrict__ adj) {
  const int n = P.nstep;
  const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (size_t)P.nrec * n) return;
  const int rec = (int)(q / n), i = (int)(q - (size_t)rec * n);
  const int ntr = P.nrec * 3;
  const int nb = P.nband > 0 ? P.nband : 1;
  double v[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int tr = rec * 3 + c;
    double acc = 0.0;
    if (P.adj_norm && nb > 1) {
      double mall = 0.0;
      for (int b = 0; b < nb; ++b) mall = fmax(mall, amax[b * ntr + tr]);
      for (int b = 0; b < nb; ++b) {
        const double mb = amax[b * ntr + tr];
        if (mb == 0.0) continue;
        acc += scratch[((size_t)(b * ntr + tr) * 3 + 2) * n + i] / mb * mall;
      }
    } else {
      for (int b = 0; b < nb; ++b) acc += scratch[((size_t)(b * ntr + tr) * 3 + 2) * n + i];
    }
    v[c] = acc;
  }
  if (P.rotate) {
    const double b = baz[rec] * (M_PI / 180.0);
    const double sb = sin(b), cb = cos(b);
    const double z = v[0], r = v[1], t = v[2];
    v[0] = -r * sb - t * cb;   // E
    v[1] = -r * cb + t * sb;   // N
    v[2] = z;
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) adj[((size_t)rec * 3 + c) * n + i] = (float)v[c];
}

}  // namespace

size_t measure_scratch_doubles(const MeasParams& p) {
  const size_t nb = p.nband > 0 ? p.nband : 1;
  const size_t ntr = (size_t)p.nrec * 3;
  return nb * ntr * 3 * (size_t)p.nstep + 2 * nb * ntr;
}

int check_measure_params(const sem_meas_cfg* c, int nrec, int nstep, double dt,
                         const double* windows_host, MeasParams* p) {
  if (!c) return report_error(SEM_ERR_ARG, "null measurement configuration");
  if (nrec < 1 || nstep < 2) return report_error(SEM_ERR_ARG, "need nrec >= 1 and nstep >= 2");
  if (c->nband < 0 || c->nband > SEM_MEAS_MAX_BANDS)
    return report_error(SEM_ERR_ARG, "nband must be 0..%d", SEM_MEAS_MAX_BANDS);
  if (c->obs_npts < 2 || !(c->obs_dt > 0.0))
    return report_error(SEM_ERR_ARG, "observed traces need obs_npts >= 2 and obs_dt > 0");
  if (!(c->pre_taper >= 0.0 && c->pre_taper <= 1.0) || !(c->win_taper >= 0.0 && c->win_taper <= 1.0))
    return report_error(SEM_ERR_ARG, "taper percentages must be in [0, 1]");
  if (c->win_taper_type < 1 || c->win_taper_type > 4)
    return report_error(SEM_ERR_ARG, "taper type must be 1..4");
  if (c->passes != 1 && c->passes != 2) return report_error(SEM_ERR_ARG, "passes must be 1 or 2");
  *p = MeasParams{};
  p->nrec = nrec;
  p->nstep = nstep;
  p->obs_npts = c->obs_npts;
  p->nband = c->nband;
  p->passes = c->passes;
  p->dt = dt;
  p->t0 = c->t0;
  p->obs_tbeg = c->obs_tbeg;
  p->obs_dt = c->obs_dt;
  p->pre_taper = c->pre_taper;
  p->win_taper = c->win_taper;
  p->win_taper_type = c->win_taper_type;
  p->weight = c->weight;
  p->rotate = c->rotate ? 1 : 0;
  p->adj_norm = c->adj_norm ? 1 : 0;
  for (int b = 0; b < c->nband; ++b) {
    if (!(c->short_p[b] > 0.0) || !(c->long_p[b] > c->short_p[b]))
      return report_error(SEM_ERR_ARG, "band %d: need 0 < short_p < long_p", b);
    int rc = design_bandpass(c->order, 1.0 / c->long_p[b], 1.0 / c->short_p[b], dt, &p->band[b]);
    if (rc) return rc;
  }
  if (windows_host) {
    const int nb = c->nband > 0 ? c->nband : 1;
    for (int b = 0; b < nb; ++b)
      for (int tr = 0; tr < nrec * 3; ++tr) {
        const double* w = windows_host + ((size_t)b * nrec * 3 + tr) * 2;
        const int wb = (int)((w[0] + c->t0) / dt), we = (int)((w[1] + c->t0) / dt);
        if (!(w[0] + c->t0 >= 0.0) || we - wb < 1 || we > nstep)
          return report_error(SEM_ERR_ARG,
                              "window [%g, %g] s of band %d trace %d is empty or outside the "
                              "record",
                              w[0], w[1], b, tr);
      }
  }
  return SEM_OK;
}

int launch_measure_waveform(const MeasParams& p, const float* seis, const double* obs,
                            const double* win, const double* baz, double* scratch, float* adj,
                            double* mis, cudaStream_t st) {
  const int nb = p.nband > 0 ? p.nband : 1;
  const int nthr = nb * p.nrec * 3;
  double* amax = scratch + (size_t)nthr * 3 * p.nstep;
  k_meas_trace<<<(nthr + 63) / 64, 64, 0, st>>>(p, seis, obs, win, baz, scratch, amax, mis);
  const size_t nq = (size_t)p.nrec * p.nstep;
  k_meas_combine<<<(unsigned)((nq + 255) / 256), 256, 0, st>>>(p, scratch, amax, baz, adj);
  return 2;
}

}  // namespace sem

using namespace sem;

// Device-buffer form: every array is device memory the caller owns.
extern "C" int sem_measure_waveform_dev(const float* seis_dev, int nrec, int nstep, double dt,
                                        const sem_meas_cfg* cfg, const double* obs_dev,
                                        const double* windows_dev, const double* baz_dev,
                                        float* adj_dev, double* misfit_trace_dev, void* stream) {
  if (!seis_dev || !obs_dev || !windows_dev || !adj_dev || !misfit_trace_dev)
    return report_error(SEM_ERR_ARG, "null device buffer");
  if (cfg && cfg->rotate && !baz_dev) return report_error(SEM_ERR_ARG, "rotate needs baz");
  if (!(dt > 0.0)) return report_error(SEM_ERR_ARG, "dt must be > 0");
  MeasParams p;
  int rc = check_measure_params(cfg, nrec, nstep, dt, nullptr, &p);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  double* scratch = nullptr;
  cudaError_t e = cudaMallocAsync((void**)&scratch, measure_scratch_doubles(p) * sizeof(double), st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return report_error(SEM_ERR_NOMEM, "measurement scratch: %s", cudaGetErrorString(e));
  }
  launch_measure_waveform(p, seis_dev, obs_dev, windows_dev, baz_dev, scratch, adj_dev,
                          misfit_trace_dev, st);
  e = cudaGetLastError();
  cudaFreeAsync(scratch, st);
  if (e != cudaSuccess)
    return report_error(SEM_ERR_CUDA, "measurement launch failed: %s", cudaGetErrorString(e));
  return SEM_OK;
}
