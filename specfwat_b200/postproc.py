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


KERNEL_ISO = ("alpha", "beta", "rhop")     # src/shared/config.f90:35
RHO_SCALING_FAC = 0.33                     # src/shared/config.f90:42
_SIX = ("rho", "mu", "kappa", "rhop", "beta", "alpha")


def gradient_on_grid(mesh, db, kernels6, x0, h, n, sigma_h, sigma_v, *, precond=None,
                     rho_scaling=False, taper=None, ngnod=8, smooth=None):
    """The post-processing of ``fwat_post_proc`` for an isotropic model
    (src/postproc/fwat_post_proc.f90:29-46), from the summed kernels to
    the gradient on the model grid:

    1. the ``KERNEL_ISO`` kernels alpha, beta, rhop of ``kernels6``
       [6, nspec, 5, 5, 5] (``Simulation.sum_kernels`` order);
    2. times ``precond`` [nspec, 5, 5, 5] when given (``apply_precond``);
    3. each smoothed on the device (``pde_smooth``: ``smooth_sem_pde``) and
       projected onto the grid ``x0 + i h``, i < n, on the device
       (``gll2grid``); with ``rho_scaling`` the rhop grid is the beta grid
       times 0.33 instead (USE_RHO_SCALING, post_processing.f90:262-264);
    4. times the boundary taper, on the device, when ``taper`` =
       (h_suppress, h_buffer, v_suppress, v_buffer) is given
       (``taper_kernel_grid``).

    Returns [3, nx, ny, nz] FP32 in KERNEL_ISO order.  ``smooth`` replaces
    the device smoother (a function of [nfield, nspec, 5, 5, 5] arrays)."""
    from .postgrid import gll2grid, taper_kernel_grid
    k6 = np.asarray(kernels6, np.float64)
    ker = np.stack([k6[_SIX.index(k)] for k in KERNEL_ISO])
    if precond is not None:
        ker = ker * np.asarray(precond, np.float64)
    nsm = 2 if rho_scaling else 3
    if smooth is None:
        def smooth(d):
            return smooth_sem_pde(mesh, d, sigma_h, sigma_v)[0]
    sm = np.asarray(smooth(ker[:nsm].astype(np.float32)), np.float64).reshape(
        (nsm,) + ker.shape[1:])
    grid = list(gll2grid(mesh, sm, x0, h, n, ngnod))
    if rho_scaling:
        grid.append(grid[1] * np.float32(RHO_SCALING_FAC))
    grid = np.stack(grid)
    if taper is not None:
        grid, _ = taper_kernel_grid(mesh, grid, x0, h, n, *taper)
    return grid


def hessian_on_grid(mesh, db, hess_sum, x0, h, n, sigma_h, sigma_v, precond_type=1, *,
                    zgrid=None, nevents=1, ngnod=8, smooth=None):
    """``PostFlow%sum_precond`` (src/postproc/post_processing.f90:199-230):
    the preconditioner on the model grid, normalised to a maximum of 1.

    - PRECOND_TYPE 0 and 1: ``invert_hess`` of the event-summed Hessian
      (``hessian_precond``), smoothed, projected onto the grid (all three
      on the device) and divided by its largest magnitude;
    - PRECOND_TYPE 2 and 3: ``zprecond_grid`` (on the device) on the
      grid's depth levels ``zgrid`` (defaults to ``x0[2] + k h[2]``) for
      ``nevents`` events.

    ``smooth`` replaces the device smoother."""
    from .postgrid import gll2grid, zprecond_grid
    if precond_type in (2, 3):
        z = (np.asarray(zgrid, np.float64) if zgrid is not None
             else x0[2] + np.arange(n[2]) * h[2])
        return zprecond_grid(z, n[0], n[1], precond_type, nevents)
    inv = hessian_precond(hess_sum, precond_type)
    if smooth is None:
        def smooth(d):
            return smooth_sem_pde(mesh, d, sigma_h, sigma_v)[0]
    sm = np.asarray(smooth(inv.reshape(db.nspec, 5, 5, 5)), np.float32)
    gm = gll2grid(mesh, sm, x0, h, n, ngnod).astype(np.float64)
    return (gm / np.abs(gm).max()).astype(np.float32)
