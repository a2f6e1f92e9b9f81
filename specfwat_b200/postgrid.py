"""Kernels on the model grid, on the device: GLL-to-grid projection, the
boundary taper and the depth preconditioner.

After smoothing, ``PostFlow%pde_smooth`` projects every kernel from the GLL
points onto the regular model grid (``gll2grid``,
src/grid/model_grid_data.f90:183-198, through ``Project_model_SEM2FD_grid``,
src/shared/projection_on_FD_grid_mod_fwat.f90:186-596), and
``PostFlow%taper_kernel_grid`` multiplies the grid kernels by a 3-D boundary
taper (src/postproc/post_processing.f90:283-325, ``taper_cls`` of
src/postproc/taper_3D_mod.f90).  ``sum_precond`` puts the depth
preconditioner on the same grid (``zprecond_grid``,
src/postproc/zprecond.f90:73-100).  The reference runs these on the host;
here they are ``sem_grid_project``, ``sem_grid_taper`` and
``sem_grid_zprecond`` of the C ABI.

Grid arrays are [nx, ny, nz] (z fastest), the C view of the reference's
Fortran (nz, ny, nx) model arrays.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check


def _desc(x0, h, n, ngnod=8):
    if len(x0) != 3 or len(h) != 3 or len(n) != 3:
        raise ValueError("x0, h and n take three values (x, y, z)")
    if ngnod not in (8, 27):
        raise ValueError("ngnod must be 8 or 27")
    return _lib.GridDesc((C.c_double * 3)(*map(float, x0)), (C.c_double * 3)(*map(float, h)),
                         (C.c_int * 3)(*map(int, n)), int(ngnod))


def gll2grid(mesh, gll, x0, h, n, ngnod=8):
    """Project element fields onto the grid ``x0[d] + i h[d]``, i < n[d].

    ``gll``: one field [nspec, 5, 5, 5] (Fortran ``dat(i,j,k,ispec)`` order,
    i fastest) or several [nfield, nspec, 5, 5, 5].  A grid point belongs to
    the first element whose candidate range holds it and takes that
    element's interpolant at the point's clamped reference coordinates;
    points no element takes are 0.  ``ngnod``: anchor nodes of the
    mesher's elements (8 or 27), used on irregular elements.  Returns
    [nx, ny, nz] (or [nfield, nx, ny, nz]) FP32."""
    desc = _desc(x0, h, n, ngnod)
    g = np.ascontiguousarray(gll, np.float32)
    one = g.ndim == 4
    g = g.reshape(-1, mesh.nspec * 125)
    shape = tuple(int(v) for v in n)
    out = np.empty((g.shape[0],) + shape, np.float32)
    check(_lib.load().sem_grid_project(mesh.handle, C.byref(desc), g.shape[0], g.ctypes.data,
                                       out.ctypes.data))
    return out[0] if one else out


def taper_kernel_grid(mesh, grid_kernels, x0, h, n, h_suppress, h_buffer, v_suppress,
                      v_buffer):
    """``PostFlow%taper_kernel_grid``: grid kernels [..., nx, ny, nz] times
    the mask of spacing (distance_min + distance_max) / 2 over the mesh's
    extent, interpolated at the grid points.  Returns (tapered FP32 grids,
    mask FP64 [nx, ny, nz])."""
    desc = _desc(x0, h, n)
    shape = tuple(int(v) for v in n)
    g = np.array(grid_kernels, np.float32, copy=True)
    if g.shape[-3:] != shape:
        raise ValueError(f"grid kernels must end in {shape}")
    lead = g.shape[:-3]
    g = np.ascontiguousarray(g.reshape((-1,) + shape))
    mask = np.empty(shape, np.float64)
    cfg = _lib.GridTaperCfg(float(h_suppress), float(h_buffer), float(v_suppress),
                            float(v_buffer))
    check(_lib.load().sem_grid_taper(mesh.handle, C.byref(desc), C.byref(cfg), g.shape[0],
                                     g.ctypes.data, mask.ctypes.data))
    return g.reshape(lead + shape), mask


def zprecond_grid(zgrid, nx, ny, precond_type, nevents):
    """``zprecond_grid``: the depth preconditioner on the grid levels
    ``zgrid`` [nz] (1e-8 above the surface, z + 1e-8 below; 1/|z| for type
    2, 1/sqrt|z| for type 3), repeated over x and y, times the event count,
    normalised, inverted and normalised.  [nx, ny, nz] FP32."""
    if precond_type not in (2, 3):
        raise ValueError("the depth forms are PRECOND_TYPE 2 and 3")
    z = np.ascontiguousarray(zgrid, np.float64).reshape(-1)
    desc = _desc((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (nx, ny, z.size))
    out = np.empty((int(nx), int(ny), z.size), np.float32)
    check(_lib.load().sem_grid_zprecond(C.byref(desc), z.ctypes.data, int(precond_type),
                                        int(nevents), out.ctypes.data))
    return out
