"""Kernel post-processing on the device: PDE smoothing and preconditioning.

- ``smooth_sem_pde`` mirrors the reference's ``smooth_sem_pde(dat_in,
  sigma_h, sigma_v, dat, is_sph)`` (src/postproc/smooth.f90:7-437), which
  ``PostFlow%pde_smooth`` and ``PostFlow%sum_precond`` call once per kernel
  or Hessian (src/postproc/post_processing.f90:222,270).  Here all fields of
  a call are smoothed on the GPU through ``sem_smooth_pde``, up to four at
  a time.
- ``hessian_precond``, ``depth_precond`` and ``apply_precond`` mirror
  ``PostFlow%apply_precond`` (post_processing.f90:164-197) with
  ``invert_hess`` (:333-372) and ``zprecond_gll``
  (src/postproc/zprecond.f90:34-71).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check

MAPPINGS = {"cube": _lib.SMOOTH_MAP_CUBE, "reference": _lib.SMOOTH_MAP_REFERENCE}


def smooth_sem_pde(mesh, dat_in, sigma_h, sigma_v, is_sph=False, *,
                   mapping="cube", distance_min=None, nstep=None,
                   is_cpml=None):
    """Smooth element fields on the device.

    ``dat_in``: one field ``[nspec, 5, 5, 5]`` (Fortran ``dat(5,5,5,nspec)``
    order) or several ``[nfield, nspec, 5, 5, 5]``.  ``mapping="cube"``
    uses the regular element's diagonal mapping; ``"reference"`` keeps the
    reference's regular branch as written (all nine mapping terms
    ``xix_regular``), which is unstable and only for parity checks.
    ``distance_min`` defaults to the mesh's minimum GLL point distance.

    Returns ``(dat, stats)``: the smoothed fields (same shape, FP32) and a
    dict with ``nstep``, ``cv``, ``ch``, ``distance_min``,
    ``fields_per_pass`` and ``step_ms`` (device time of the steps).
    """
    if mapping not in MAPPINGS:
        raise ValueError(f"mapping must be one of {sorted(MAPPINGS)}")
    d = np.ascontiguousarray(dat_in, np.float32)
    one = d.ndim == 4
    d = d.reshape(-1, mesh.nspec * 125)
    out = np.empty_like(d)
    cfg = _lib.SmoothCfg(float(sigma_h), float(sigma_v),
                         float(distance_min or 0.0), int(bool(is_sph)),
                         MAPPINGS[mapping], int(nstep or 0))
    cpml = (None if is_cpml is None
            else np.ascontiguousarray(is_cpml, np.int32))
    if cpml is not None and cpml.shape != (mesh.nspec,):
        raise ValueError("is_cpml must have one entry per element")
    st = _lib.SmoothStats()
    check(_lib.load().sem_smooth_pde(
        mesh.handle, C.byref(cfg), d.shape[0], d.ctypes.data,
        None if cpml is None else cpml.ctypes.data, out.ctypes.data,
        C.byref(st)))
    stats = {"nstep": st.nstep, "cv": st.cv, "ch": st.ch,
             "distance_min": st.distance_min,
             "fields_per_pass": st.fields_per_pass, "step_ms": st.step_ms}
    out = out.reshape((-1, mesh.nspec, 5, 5, 5))
    return (out[0] if one else out), stats


def hessian_precond(hess_sum, precond_type=1):
    """Preconditioner from the event-summed approximate Hessian.

    ``precond_type`` 1 (DEFAULT_PRECOND): ``hess_sum`` is the sum of |hess|
    over the events (``Simulation.sum_hessian(abs_each=True)``); 0: the plain
    sum, whose magnitude is taken.  The result is ``invert_hess`` of it:
    normalised by its maximum, inverted with THRESHOLD_HESS = 1e-3,
    normalised again.  Computed on the device; returns FP32 of the input's
    shape.
    """
    h = np.ascontiguousarray(hess_sum, np.float64)
    out = np.zeros(h.shape, np.float32)
    check(_lib.load().sem_hessian_precond(h.ctypes.data, h.size, int(precond_type),
                                          out.ctypes.data))
    return out


def depth_precond(mesh, zlev, precond_type, nevents):
    """Depth preconditioner ``zprecond_gll`` (PRECOND_TYPE 2: 1/|z|,
    3: 1/sqrt|z|) on the model grid's depth levels ``zlev`` (ascending),
    for ``nevents`` events.  Returns FP32 ``[nspec, 5, 5, 5]``."""
    z = np.ascontiguousarray(zlev, np.float64)
    out = np.zeros((mesh.nspec, 5, 5, 5), np.float32)
    check(_lib.load().sem_depth_precond(mesh._h, z.ctypes.data, z.size, int(precond_type),
                                        int(nevents), out.ctypes.data))
    return out


def apply_precond(kernels, precond):
    """``ker_data(:,:,:,:,iker) * total_hess`` for every kernel
    (post_processing.f90:193-195): ``kernels`` [..., nspec, 5, 5, 5]."""
    return np.asarray(kernels) * np.asarray(precond, np.float64)
