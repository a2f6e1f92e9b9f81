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
        L.oracle_forward.argtypes = [
            C.c_void_p, C.c_double, C.c_int, C.POINTER(OracleSource), C.c_int,
            C.c_void_p, C.c_void_p, C.c_int]
        L.oracle_adjoint.argtypes = [C.c_void_p, C.c_int, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p]
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

    def __init__(self, db, precision=8, nthreads=None, stacey=True):
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
        k = self._keep
        f, i = C.c_float, C.c_int
        self._mesh = OracleMesh(
            db.nspec, db.nglob, _ptr(k["ibool"], i), _ptr(k["x"], f),
            _ptr(k["y"], f), _ptr(k["z"], f), db.xix_regular,
            db.jacobian_regular, _ptr(k["kappa"], f), _ptr(k["mu"], f),
            _ptr(k["rho"], f), _ptr(k["rmass"], f), _ptr(k["rho_vp"], f),
            _ptr(k["rho_vs"], f), db.nfaces if stacey else 0,
            _ptr(k["f_ispec"], i), _ptr(k["f_ijk"], i), _ptr(k["f_jw"], f),
            _ptr(k["f_n"], f))
        self._h = lib().oracle_create(C.byref(self._mesh), precision, nthreads)
        if not self._h:
            raise RuntimeError("oracle_create failed")
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
