"""ctypes front end of the CPU oracle (test infrastructure only).

Loaded only by the tests, the smoke check and the CPU-baseline leg of the
benchmark, as the checker the CUDA solver is compared against.  See
``sem_oracle.cpp`` for the formulation and its parity status (unpinned
against the reference solver, which is absent from the reference tree;
pinned by physics known-answer tests instead).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libsem_oracle.so")
_lib = None


class OracleMesh(C.Structure):
    _fields_ = [
        ("nspec", C.c_int), ("nglob", C.c_int),
        ("ibool", C.POINTER(C.c_int)),
        ("x", C.POINTER(C.c_float)), ("y", C.POINTER(C.c_float)),
        ("z", C.POINTER(C.c_float)),
        ("xix", C.c_double), ("jac", C.c_double),
        ("kappa", C.POINTER(C.c_float)), ("mu", C.POINTER(C.c_float)),
        ("rho", C.POINTER(C.c_float)), ("rmass", C.POINTER(C.c_float)),
        ("rho_vp", C.POINTER(C.c_float)), ("rho_vs", C.POINTER(C.c_float)),
        ("nf", C.c_int),
        ("f_ispec", C.POINTER(C.c_int)), ("f_ijk", C.POINTER(C.c_int)),
        ("f_jw", C.POINTER(C.c_float)), ("f_n", C.POINTER(C.c_float)),
        ("irreg", C.POINTER(C.c_int)), ("geo", C.POINTER(C.c_float)),
    ]


class OracleSource(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double),
                ("mt", C.c_double * 6), ("f0", C.c_double),
                ("tshift", C.c_double)]


def build():
    """Compile the oracle with its Makefile (g++, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.oracle_create.restype = C.c_void_p
        L.oracle_create.argtypes = [C.POINTER(OracleMesh), C.c_int, C.c_int]
        L.oracle_destroy.argtypes = [C.c_void_p]
        L.oracle_set_flush_subnormals.argtypes = [C.c_void_p, C.c_int]
        L.oracle_forward.argtypes = [
            C.c_void_p, C.c_double, C.c_int, C.POINTER(OracleSource), C.c_int,
            C.c_void_p, C.c_void_p, C.c_int]
        L.oracle_adjoint.argtypes = [C.c_void_p, C.c_int, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p]
        L.oracle_get_hessian.argtypes = [C.c_void_p, C.c_void_p]
        L.oracle_set_injection.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int,
                                           C.c_void_p, C.c_void_p]
        L.oracle_energy.restype = C.c_double
        L.oracle_energy.argtypes = [C.c_void_p]
        L.oracle_get_field.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.oracle_forward_energy.argtypes = [
            C.c_void_p, C.c_double, C.c_int, C.POINTER(OracleSource), C.c_int,
            C.c_void_p]
        L.oracle_source_element.argtypes = [C.c_void_p, C.c_double,
                                            C.c_double, C.c_double, C.c_void_p]
        L.oracle_smooth_pde.argtypes = [
            C.POINTER(OracleMesh), C.c_int, C.c_int, C.c_void_p, C.c_void_p,
            C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
            C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def _ptr(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


class Oracle:
    """One mesh + model on the CPU, FP32 (``precision=4``) or FP64 (8)."""

    def __init__(self, db, precision=8, nthreads=None, stacey=True, flush_subnormals=False):
        """``flush_subnormals``: run with FP32 subnormals flushed to zero
        (x86 FTZ/DAZ), which only changes values below 1.2e-38 and avoids
        the cores' slow path for them on large FP32 runs."""
        self.db = db
        self.precision = precision
        nthreads = nthreads or os.cpu_count() or 1
        # keep references so the buffers outlive the C structure
        self._keep = dict(
            ibool=np.ascontiguousarray(db.ibool.reshape(-1), np.int32),
            x=np.ascontiguousarray(db.xstore, np.float32),
            y=np.ascontiguousarray(db.ystore, np.float32),
            z=np.ascontiguousarray(db.zstore, np.float32),
            kappa=np.ascontiguousarray(db.kappa.reshape(-1), np.float32),
            mu=np.ascontiguousarray(db.mu.reshape(-1), np.float32),
            rho=np.ascontiguousarray(db.rho.reshape(-1), np.float32),
            rmass=np.ascontiguousarray(db.rmass, np.float32),
            rho_vp=np.ascontiguousarray(db.rho_vp.reshape(-1), np.float32),
            rho_vs=np.ascontiguousarray(db.rho_vs.reshape(-1), np.float32),
            f_ispec=np.ascontiguousarray(db.abs_ispec, np.int32),
            f_ijk=np.ascontiguousarray(db.abs_ijk.reshape(-1), np.int32),
            f_jw=np.ascontiguousarray(db.abs_jw.reshape(-1), np.float32),
            f_n=np.ascontiguousarray(db.abs_normal.reshape(-1), np.float32),
        )
        irr = getattr(db, "irregular", None)
        if irr is not None and (irr >= 0).any():
            self._keep["irreg"] = np.ascontiguousarray(irr, np.int32)
            self._keep["geo"] = np.ascontiguousarray(db.geo.reshape(-1), np.float32)
        k = self._keep
        f, i = C.c_float, C.c_int
        self._mesh = OracleMesh(
            db.nspec, db.nglob, _ptr(k["ibool"], i), _ptr(k["x"], f),
            _ptr(k["y"], f), _ptr(k["z"], f), db.xix_regular,
            db.jacobian_regular, _ptr(k["kappa"], f), _ptr(k["mu"], f),
            _ptr(k["rho"], f), _ptr(k["rmass"], f), _ptr(k["rho_vp"], f),
            _ptr(k["rho_vs"], f), db.nfaces if stacey else 0,
            _ptr(k["f_ispec"], i), _ptr(k["f_ijk"], i), _ptr(k["f_jw"], f),
            _ptr(k["f_n"], f),
            _ptr(k["irreg"], i) if "irreg" in k else None,
            _ptr(k["geo"], f) if "geo" in k else None)
        self._h = lib().oracle_create(C.byref(self._mesh), precision, nthreads)
        if not self._h:
            raise RuntimeError("oracle_create failed")
        if flush_subnormals:
            lib().oracle_set_flush_subnormals(self._h, 1)
        self.nstep = 0
        self.nrec = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().oracle_destroy(h)
            self._h = None

    @staticmethod
    def source(x, y, z, mt, f0, tshift=0.0):
        return OracleSource(x, y, z, (C.c_double * 6)(*[float(m) for m in mt]),
                            f0, tshift)

    def forward(self, dt, nstep, src, rec_xyz, save_forward=False):
        """Forward run; returns seismograms [nrec, 3, nstep] (x=E, y=N, z=Up)."""
        rec = np.ascontiguousarray(rec_xyz, np.float64).reshape(-1, 3)
        seis = np.zeros((rec.shape[0], 3, nstep), np.float64)
        rc = lib().oracle_forward(self._h, dt, nstep, C.byref(src),
                                  rec.shape[0], rec.ctypes.data,
                                  seis.ctypes.data, int(bool(save_forward)))
        if rc:
            raise RuntimeError(f"oracle_forward failed ({rc})")
        self.nstep = nstep
        self.dt = dt
        return seis

    def adjoint(self, rec_xyz, adj, want_backward_seis=False,
                want_adjoint_seis=False):
        """Adjoint + backward run after ``forward(save_forward=True)``.

        ``adj`` is [nrec, 3, nstep] in forward time order.  Returns the six
        kernels [6, nspec, 5, 5, 5] (rho, mu, kappa, rhop, beta, alpha) and
        optionally the backward-field seismograms (forward time order)."""
        rec = np.ascontiguousarray(rec_xyz, np.float64).reshape(-1, 3)
        adj = np.ascontiguousarray(adj, np.float64)
        assert adj.shape == (rec.shape[0], 3, self.nstep)
        db = self.db
        kern = np.zeros((6, db.nspec, 5, 5, 5), np.float64)
        bseis = (np.zeros((rec.shape[0], 3, self.nstep))
                 if want_backward_seis else None)
        aseis = (np.zeros((rec.shape[0], 3, self.nstep))
                 if want_adjoint_seis else None)
        rc = lib().oracle_adjoint(
            self._h, rec.shape[0], rec.ctypes.data, adj.ctypes.data,
            kern.ctypes.data, None if bseis is None else bseis.ctypes.data,
            None if aseis is None else aseis.ctypes.data)
        if rc:
            raise RuntimeError(f"oracle_adjoint failed ({rc})")
        out = [kern]
        if want_backward_seis:
            out.append(bseis)
        if want_adjoint_seis:
            out.append(aseis)
        return out[0] if len(out) == 1 else tuple(out)

    def set_injection(self, veloc, tract, np_resamp=1, k0=0):
        """FK injection on the absorbing faces for the next forward runs:
        ``[nt, nf*25, 3]`` incident velocity and traction (sigma . n,
        outward normal), sample ``k`` at time ``(k + k0) * np_resamp * dt``;
        ``veloc=None`` removes it."""
        if veloc is None:
            lib().oracle_set_injection(self._h, 0, 1, 0, None, None)
            return
        v = np.ascontiguousarray(veloc, np.float64)
        t = np.ascontiguousarray(tract, np.float64)
        assert v.shape == t.shape and v.shape[1:] == (self.db.nfaces * 25, 3)
        if lib().oracle_set_injection(self._h, v.shape[0], int(np_resamp), int(k0),
                                      v.ctypes.data, t.ctypes.data):
            raise RuntimeError("oracle_set_injection failed")

    def hessian(self):
        """hess_kernel [nspec, 5, 5, 5] of the last ``adjoint`` run: twice
        the sum over steps of DT * (adjoint accel . backward accel)."""
        out = np.zeros((self.db.nspec, 5, 5, 5), np.float64)
        if lib().oracle_get_hessian(self._h, out.ctypes.data):
            raise RuntimeError("no adjoint run")
        return out

    def field(self, which):
        n = self.db.nglob * 3
        out = np.zeros(n, np.float64)
        lib().oracle_get_field(self._h, which, out.ctypes.data)
        return out.reshape(-1, 3)

    def energy(self):
        return lib().oracle_energy(self._h)

    def forward_energy(self, dt, nstep, src, every):
        e = np.zeros(nstep // every, np.float64)
        lib().oracle_forward_energy(self._h, dt, nstep, C.byref(src), every,
                                    e.ctypes.data)
        return e

    def locate(self, x, y, z):
        xi = np.zeros(3, np.float64)
        e = lib().oracle_source_element(self._h, x, y, z, xi.ctypes.data)
        return e, xi

    def smooth_pde(self, dat, sigma_h, sigma_v, distance_min, is_sph=False,
                   mapping=0, nstep=0, is_cpml=None):
        """PDE smoothing of element fields ``dat`` [nfield, nspec, 5, 5, 5]
        (or one field [nspec, 5, 5, 5]) in this oracle's precision, as the
        CPU branch of ``smooth_sem_pde`` (src/postproc/smooth.f90:7-437).
        ``mapping`` 0: the cube's diagonal mapping; 1: the reference's
        regular branch as written (all nine mapping terms xix_regular).
        Returns (smoothed fields, step count, (cv, ch))."""
        d = np.ascontiguousarray(dat, np.float32)
        one = d.ndim == 4
        d = d.reshape(-1, self.db.nspec * 125)
        out = np.zeros(d.shape, np.float64)
        cpml = (None if is_cpml is None
                else np.ascontiguousarray(is_cpml, np.int32))
        cvch = np.zeros(2, np.float64)
        n = lib().oracle_smooth_pde(
            C.byref(self._mesh), self.precision, d.shape[0], d.ctypes.data,
            None if cpml is None else cpml.ctypes.data, float(sigma_h),
            float(sigma_v), float(distance_min), int(bool(is_sph)), int(mapping),
            int(nstep), out.ctypes.data, cvch.ctypes.data)
        if n < 0:
            raise RuntimeError("oracle_smooth_pde: bad arguments")
        out = out.reshape((-1, self.db.nspec, 5, 5, 5))
        return (out[0] if one else out), n, (cvch[0], cvch[1])


# -- FP64 measurement restatement (L2 waveform misfit) ----------------------

def simpson(y, dx):
    """Composite Simpson rule as ``src/shared/utils.f90:1635-1663``: for an
    even sample count the last interval is added by the trapezoid rule.

    The even branch is reproduced as written there: its loop adds
    ``2 y(n-1)`` on top of the ``y(n-1)`` already in the initial sum, so the
    second-to-last sample carries weight 3 (not the textbook 1)."""
    y = np.asarray(y, np.float64)
    n = y.shape[-1]
    if n < 2:
        return np.zeros(y.shape[:-1])
    if n % 2 == 0:
        s = y[..., 0] + y[..., n - 2]
        s = s + 4.0 * y[..., 1:n - 2:2].sum(-1) + 2.0 * y[..., 2:n - 1:2].sum(-1)
        return dx / 3.0 * s + 0.5 * dx * (y[..., n - 2] + y[..., n - 1])
    s = y[..., 0] + y[..., n - 1]
    s = s + 4.0 * y[..., 1:n - 1:2].sum(-1) + 2.0 * y[..., 2:n - 2:2].sum(-1)
    return dx / 3.0 * s


def taper_window(npts, pct, itype=1):
    """Taper weights of ``src/shared/signal.f90:419-491`` (types 1 hann,
    2 hamming, 3 cos, 4 cos^10)."""
    w = np.ones(npts, np.float64)
    if pct in (0.0, 1.0):
        frac = int(npts * pct / 2.0)
    else:
        frac = int(npts * pct / 2.0 + 0.5)
    if frac <= 0:
        return w
    i = np.arange(frac, dtype=np.float64)
    den = 2 * frac - 1

    def f(x):
        if itype == 1:
            return 0.5 - 0.5 * np.cos(2.0 * np.pi * x / den)
        if itype == 2:
            return 0.54 - 0.46 * np.cos(2.0 * np.pi * x / den)
        if itype == 3:
            return np.cos(np.pi * x / den - np.pi / 2.0)
        if itype == 4:
            return 1.0 - np.cos(np.pi * x / den) ** 10
        raise ValueError(itype)

    w[:frac] = f(i)
    w[npts - frac:] = f(frac + i)
    return w


def l2_adjoint_source(syn, obs, dt, taper_pct=0.05, itype=1):
    """L2 waveform misfit and adjoint source over the full record, as
    ``src/preproc/adjoint_sources/waveform_misfit.f90:15-64``: taper s and
    d, misfit 0.5 * simpson((s-d)^2), adjoint source taper(s - d)."""
    syn = np.asarray(syn, np.float64)
    obs = np.asarray(obs, np.float64)
    w = taper_window(syn.shape[-1], taper_pct, itype)
    s = syn * w
    d = obs * w
    r = s - d
    misfit = 0.5 * simpson(r * r, dt)
    return misfit, r * w


# -- FP64 measurement pipeline: LEQData%measure_adj for IMEAS_WAVEFORM -------
#
# src/preproc/leq_data.f90:48-188 per receiver, component and band:
#   obs: interpolate_func_dp onto the synthetic axis (signal.f90:85-125),
#        detrend (signal.f90:382-406), demean (:408-417), Hann taper
#        taper_per (config.f90:69), bandpass_dp (signal.f90:7-36)
#   syn: rotated to Z,R,T (syn_data.f90:64-66, common.f90:136-152), Hann
#        taper, bandpass_dp
#   WaveformMisfit over the window (waveform_misfit.f90:15-64), filter_adj
#   (adjoint_source.f90:92-114), times src_weight
# then rotate_adj_src (noise_data.f90:213-252): sum (or normalised sum) over
# bands and rotation Z,R,T -> Z,N,E (common.f90:272-291).
# bandpass_dp runs SAC's xapiir (xapiir_sub.f90) in FP32; this restatement
# designs and applies the same Butterworth band-pass in FP64.

def butterworth_bandpass_sos(order, flo, fhi, dt):
    """Second-order sections [nsect, 5] = (b0, b1, b2, a1, a2), a0 = 1, of
    the Butterworth band-pass that xapiir designs (DESIGN, BUROOTS, WARP,
    LPTBP, BILIN2: xapiir_sub.f90:237-304,334-368,712-726,855-961,
    1270-1305): analog prototype poles on the unit circle, tangent-warped
    band edges, low-pass to band-pass transform, gain 1 at the geometric
    centre of the band, bilinear transform."""
    poles, kinds = [], []
    half = order // 2
    if 2 * half < order:
        poles.append(complex(-1.0, 0.0))
        kinds.append("SP")
    for k in range(1, half + 1):
        ang = np.pi * (0.5 + (2 * k - 1) / (2.0 * order))
        poles.append(complex(np.cos(ang), np.sin(ang)))
        kinds.append("CP")
    flw = np.tan(np.pi * flo * dt) / (2.0 * np.pi)
    fhw = np.tan(np.pi * fhi * dt) / (2.0 * np.pi)
    A = (2.0 * np.pi) ** 2 * flw * fhw
    B = 2.0 * np.pi * (fhw - flw)
    sn, sd = [], []
    for p, kind in zip(poles, kinds):
        if kind == "CP":
            c = np.sqrt(complex((B * p) ** 2 - 4.0 * A))
            for q in (0.5 * (B * p + c), 0.5 * (B * p - c)):
                sn.append([0.0, B, 0.0])
                sd.append([abs(q) ** 2, -2.0 * q.real, 1.0])
        else:
            sn.append([0.0, B, 0.0])
            sd.append([A, -B * p.real, 1.0])
    s = complex(0.0, np.sqrt(A))
    h = complex(1.0, 0.0)
    for n_, d_ in zip(sn, sd):
        h *= ((n_[2] * s + n_[1]) * s + n_[0]) / ((d_[2] * s + d_[1]) * s + d_[0])
    scale = 1.0 / abs(h)
    sn[0] = [v * scale for v in sn[0]]
    out = []
    for n_, d_ in zip(sn, sd):
        a0, a1, a2 = d_
        sc = a2 + a1 + a0
        b0, b1, b2 = n_
        out.append([(b2 + b1 + b0) / sc, 2.0 * (b0 - b2) / sc, (b2 - b1 + b0) / sc,
                    2.0 * (a0 - a2) / sc, (a2 - a1 + a0) / sc])
    return np.array(out, np.float64)


def iir_apply(x, sos, passes=2):
    """xapiir's APPLY (xapiir_sub.f90:118-200): the sections in turn over
    the whole trace, then (passes = 2) again over the reversed trace."""
    from scipy.signal import sosfilt
    sc = np.concatenate([sos[:, :3], np.ones((len(sos), 1)), sos[:, 3:]], axis=1)
    y = sosfilt(sc, np.asarray(x, np.float64), axis=-1)
    if passes == 2:
        y = sosfilt(sc, y[..., ::-1], axis=-1)[..., ::-1]
    return np.ascontiguousarray(y)


def interpolate_onto(data, t1, dt1, t2, dt2, npt2):
    """interpolate_func_dp (signal.f90:85-125): linear interpolation of a
    trace starting at t1 with step dt1 onto npt2 samples from t2 with step
    dt2; samples not strictly inside the data span are 0."""
    data = np.asarray(data, np.float64)
    npt1 = data.shape[-1]
    time = t2 + np.arange(npt2) * dt2
    inside = (time > t1) & (time < t1 + (npt1 - 1) * dt1)
    ii = np.floor((time - t1) / dt1).astype(np.int64)
    ii = np.clip(ii, 0, npt1 - 2)
    tt = time - (ii * dt1 + t1)
    out = (data[..., ii + 1] - data[..., ii]) * tt / dt1 + data[..., ii]
    return np.where(inside, out, 0.0)


def detrend(x):
    """signal.f90:382-406 as written: least-squares slope, removed about the
    1-based mean index (n+1)/2 from the 0-based index i-1."""
    x = np.asarray(x, np.float64)
    n = x.shape[-1]
    ds1 = x.sum(-1)
    ds2 = np.cumsum(x, axis=-1).sum(-1)
    davei = 0.5 * (n + 1.0)
    davex = ds1 / n
    dslope = -12.0 * (ds2 - davei * ds1) / (n * (n * n - 1.0))
    i = np.arange(n, dtype=np.float64)
    return x - davex[..., None] - dslope[..., None] * (i - davei)


def demean(x):
    x = np.asarray(x, np.float64)
    return x - x.sum(-1, keepdims=True) / x.shape[-1]


def measure_waveform(syn, obs, dt, t0, obs_tbeg, obs_dt, bands, windows,
                     order=2, passes=2, pre_taper=0.1, win_taper=0.05,
                     win_type=1, weight=1.0, baz=None, adj_norm=False):
    """FP64 restatement of LEQData%measure_adj (IMEAS_WAVEFORM), one
    window per trace and band.

    syn [nrec, 3, nstep] in x=E, y=N, z=Z; obs [nrec, 3, obs_npts] in Z,R,T
    when ``baz`` (degrees, per receiver) is given, else in x, y, z;
    ``bands`` [(short_p, long_p), ...] or [] for no band-pass; windows
    [nband, nrec, 3, 2] start/end in origin time (s).  Returns
    (misfit per band, adjoint source [nrec, 3, nstep] in x, y, z, per-trace
    misfits [nband, nrec, 3])."""
    syn = np.asarray(syn, np.float64)
    nrec, _, nstep = syn.shape
    if baz is not None:
        b = np.deg2rad(np.asarray(baz, np.float64))[:, None]
        e, nn, z = syn[:, 0], syn[:, 1], syn[:, 2]
        syn = np.stack([z, -e * np.sin(b) - nn * np.cos(b),
                        -e * np.cos(b) + nn * np.sin(b)], axis=1)
    d0 = interpolate_onto(obs, obs_tbeg, obs_dt, -t0, dt, nstep)
    d0 = demean(detrend(d0))
    wpre = taper_window(nstep, pre_taper, 1)
    d0 = d0 * wpre
    s0 = syn * wpre
    nb_ = max(1, len(bands))
    adjs = np.zeros((nb_, nrec, 3, nstep))
    mis = np.zeros((nb_, nrec, 3))
    for ib in range(nb_):
        if bands:
            sos = butterworth_bandpass_sos(order, 1.0 / bands[ib][1], 1.0 / bands[ib][0], dt)
            d = iir_apply(d0, sos, passes)
            s = iir_apply(s0, sos, passes)
        else:
            sos, d, s = None, d0, s0
        for r in range(nrec):
            for c in range(3):
                w0, w1 = windows[ib][r][c]
                nb = int((w0 + t0) / dt) + 1
                ne = int((w1 + t0) / dt)
                if ne - nb + 1 <= 0:
                    raise ValueError("empty window")
                tw = taper_window(ne - nb + 1, win_taper, win_type)
                sw = s[r, c, nb - 1:ne] * tw
                dw = d[r, c, nb - 1:ne] * tw
                res = sw - dw
                mis[ib, r, c] = 0.5 * simpson(res * res, dt) * weight
                a = np.zeros(nstep)
                a[nb - 1:ne] = res * tw
                if sos is not None:
                    a = iir_apply(a, sos, passes)
                out = np.zeros(nstep)
                out[nb - 1:ne] = a[nb - 1:ne] * tw
                adjs[ib, r, c] = out * weight
    if adj_norm and nb_ > 1:
        amax = np.abs(adjs).max(-1)                       # [band, rec, comp]
        mx = amax.max(0)                                  # [rec, comp]
        safe = np.where(amax > 0, amax, 1.0)
        comb = np.where((amax > 0)[..., None], adjs / safe[..., None] * mx[None, ..., None], 0.0).sum(0)
    else:
        comb = adjs.sum(0)
    if baz is not None:
        b = np.deg2rad(np.asarray(baz, np.float64))[:, None]
        z, rr, tt = comb[:, 0], comb[:, 1], comb[:, 2]
        comb = np.stack([-rr * np.sin(b) - tt * np.cos(b),
                         -rr * np.cos(b) + tt * np.sin(b), z], axis=1)
    return mis.sum((1, 2)), comb, mis


# --------------------------------------------------------------------------
# Kernel preconditioners (src/postproc/post_processing.f90:164-197,333-372;
# src/postproc/zprecond.f90:11-71), vectorised FP64 restatements.
# --------------------------------------------------------------------------

THRESHOLD_HESS = 1e-3   # src/shared/config.f90:42


def invert_hess(h):
    """``invert_hess`` (post_processing.f90:333-372): normalise by max|h|
    (all ones when it is below 1e-18), invert where |h| > THRESHOLD_HESS
    (1/THRESHOLD_HESS elsewhere), normalise by max|h| again."""
    h = np.asarray(h, np.float64)
    mx = np.abs(h).max()
    h = np.ones_like(h) if mx < 1e-18 else h / mx
    safe = np.where(np.abs(h) > THRESHOLD_HESS, h, 1.0)
    h = np.where(np.abs(h) > THRESHOLD_HESS, 1.0 / safe, 1.0 / THRESHOLD_HESS)
    return h / np.abs(h).max()


def hessian_precond(hess_sum, precond_type=1):
    """``apply_precond`` PRECOND_TYPE 0 (|sum hess|) or 1 (sum |hess| given)
    followed by ``invert_hess`` (post_processing.f90:171-185)."""
    h = np.asarray(hess_sum, np.float64)
    if precond_type == 0:
        h = np.abs(h)
    return invert_hess(h)


def depth_profile(zlev, precond_type):
    """``get_1d_precond`` (zprecond.f90:11-32): 1e-8 above the surface,
    z + 1e-8 below; 1/|z| (type 2) or 1/sqrt|z| (type 3)."""
    z = np.asarray(zlev, np.float64)
    zl = np.where(z > 0.0, 1e-8, z + 1e-8)
    return 1.0 / np.sqrt(zl * zl) if precond_type == 2 else 1.0 / np.sqrt(np.sqrt(zl * zl))


def interp1_clamped(x, v, xq):
    """``interp1`` (src/shared/utils.f90:889-910) on ascending levels:
    linear between the bracketing levels, the end value at and above the
    last level.  Below the first level the Fortran reads x(0); here the
    first value is taken."""
    return np.interp(np.asarray(xq, np.float64), np.asarray(x, np.float64),
                     np.asarray(v, np.float64))


def depth_precond(db, zlev, precond_type, nevents):
    """``zprecond_gll`` (zprecond.f90:34-71) on the mesh ``db``:
    [nspec, 5, 5, 5]."""
    prof = depth_profile(zlev, precond_type)
    z = np.asarray(db.zstore, np.float64)[np.asarray(db.ibool).reshape(db.nspec, 5, 5, 5)]
    h = interp1_clamped(zlev, prof, z) * nevents
    h = h / np.abs(h).max()
    h = 1.0 / h
    return h / np.abs(h).max()
