"""External tomography model on arbitrary grid axes, sampled at GLL points.

Restates what the reference's mesher does for an external model
(``model_external_values``, src/patch/model_external_values.f90:206-273):
the model is vp, vs, rho on a regular-topology grid with its own 1-D axes
x(nx), y(ny), z(nz) (ascending, any spacing; read from
``tomography_model.h5`` datasets /x, /y, /z, /vp, /vs, /rho at :178-190).
A GLL point inside the grid's box on all three axes takes the trilinear
interpolant (``interp3``, src/shared/utils.f90:1089-1159, cell located by
``locate_bissection``, :1490-1525); a point outside on any axis takes the
value of the nearest of the 8 nodes around it whose value is not zero
(``interp3_nearest_simple``, :1276-1325, with ``get_nearest_bound_idx``,
:1262-1274), chosen for each field on its own.

Arrays are indexed [ix, iy, iz] as the reference holds them after its
``transpose_3`` of the HDF5 datasets (a file written from numpy with
shape (nx, ny, nz)).  The reference computes in CUSTOM_REAL (FP32); here
the interpolation is FP64 and the result FP32.
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class ExternalModel:
    x: np.ndarray    # [nx] ascending
    y: np.ndarray    # [ny]
    z: np.ndarray    # [nz] (z up; depths are negative)
    vp: np.ndarray   # [nx, ny, nz]
    vs: np.ndarray
    rho: np.ndarray

    def __post_init__(self):
        for a in ("x", "y", "z"):
            v = np.asarray(getattr(self, a), np.float64)
            if v.ndim != 1 or v.size < 2 or np.any(np.diff(v) <= 0):
                raise ValueError(f"axis {a} must be strictly ascending with >= 2 nodes")
            setattr(self, a, v)
        shape = (self.x.size, self.y.size, self.z.size)
        for f in ("vp", "vs", "rho"):
            v = np.asarray(getattr(self, f), np.float64)
            if v.shape != shape:
                raise ValueError(f"{f} has shape {v.shape}, expected {shape}")
            setattr(self, f, v)


def read_tomography_h5(path: str) -> ExternalModel:
    """Read ``tomography_model.h5`` (datasets /x, /y, /z, /vp, /vs, /rho, the
    3-D ones written with shape (nx, ny, nz)).  Needs h5py."""
    try:
        import h5py
    except ImportError as e:  # pragma: no cover - depends on the host
        raise ImportError("reading tomography_model.h5 needs h5py; pass the arrays to "
                          "ExternalModel instead") from e
    with h5py.File(path, "r") as f:
        return ExternalModel(*(np.asarray(f[k]) for k in ("x", "y", "z", "vp", "vs", "rho")))


def _cell(ax, q):
    """0-based lower node of the interpolation cell (locate_bissection, then
    kx = min(max(ind, 1), n - 1) in 1-based terms) and whether q lies in
    [ax[0], ax[-1]]."""
    n = ax.size
    inside = (q >= ax[0]) & (q <= ax[-1])
    jl = np.searchsorted(ax, q, side="right")          # 1-based index of last node <= q
    ind = np.where(q == ax[0], 1, np.where(q == ax[-1], n - 1, jl))
    k = np.clip(ind, 1, n - 1) - 1
    # outside: get_nearest_bound_idx, 1 below the axis and n - 1 above
    k = np.where(inside, k, np.where(q < ax[0], 0, n - 2))
    return k, inside


def _trilinear(m, field, kx, ky, kz, xq, yq, zq):
    x, y, z = m.x, m.y, m.z
    xix1, yiy1, ziz1 = xq - x[kx], yq - y[ky], zq - z[kz]
    xix2, yiy2, ziz2 = xq - x[kx + 1], yq - y[ky + 1], zq - z[kz + 1]
    x1x2, y1y2, z1z2 = 1.0 / (x[kx] - x[kx + 1]), 1.0 / (y[ky] - y[ky + 1]), 1.0 / (z[kz] - z[kz + 1])
    x2x1, y2y1, z2z1 = -x1x2, -y1y2, -z1z2
    v = field
    out = xix2 * yiy2 * ziz2 * x1x2 * y1y2 * z1z2 * v[kx, ky, kz]
    out += xix2 * yiy2 * ziz1 * x1x2 * y1y2 * z2z1 * v[kx, ky, kz + 1]
    out += xix2 * yiy1 * ziz2 * x1x2 * y2y1 * z1z2 * v[kx, ky + 1, kz]
    out += xix2 * yiy1 * ziz1 * x1x2 * y2y1 * z2z1 * v[kx, ky + 1, kz + 1]
    out += xix1 * yiy2 * ziz2 * x2x1 * y1y2 * z1z2 * v[kx + 1, ky, kz]
    out += xix1 * yiy2 * ziz1 * x2x1 * y1y2 * z2z1 * v[kx + 1, ky, kz + 1]
    out += xix1 * yiy1 * ziz2 * x2x1 * y2y1 * z1z2 * v[kx + 1, ky + 1, kz]
    out += xix1 * yiy1 * ziz1 * x2x1 * y2y1 * z2z1 * v[kx + 1, ky + 1, kz + 1]
    return out


def _nearest_nonzero(m, field, kx, ky, kz, xq, yq, zq):
    """Value at the nearest of the 8 nodes (kx..kx+1, ky..ky+1, kz..kz+1)
    whose value is not zero; ties go to the first in the reference's loop
    order (x outer, z inner).  All eight zero: 0."""
    best = np.full(xq.shape, np.inf)
    val = np.zeros(xq.shape)
    for di in (0, 1):
        for dj in (0, 1):
            for dk in (0, 1):
                i, j, k = kx + di, ky + dj, kz + dk
                d = np.sqrt((xq - m.x[i]) ** 2 + (yq - m.y[j]) ** 2 + (zq - m.z[k]) ** 2)
                v = field[i, j, k]
                take = (d < best) & (v != 0.0)
                best = np.where(take, d, best)
                val = np.where(take, v, val)
    return val


def external_model_values(m: ExternalModel, xq, yq, zq):
    """(vp, vs, rho) FP32 at the points (xq, yq, zq) (any shape)."""
    xq = np.asarray(xq, np.float64)
    yq = np.asarray(yq, np.float64)
    zq = np.asarray(zq, np.float64)
    kx, ix = _cell(m.x, xq)
    ky, iy = _cell(m.y, yq)
    kz, iz = _cell(m.z, zq)
    inside = ix & iy & iz
    out = []
    for f in (m.vp, m.vs, m.rho):
        tri = _trilinear(m, f, kx, ky, kz, xq, yq, zq)
        near = _nearest_nonzero(m, f, kx, ky, kz, xq, yq, zq)
        out.append(np.where(inside, tri, near).astype(np.float32))
    return tuple(out)


def apply_external_model(db, m: ExternalModel):
    """The database with vp, vs, rho taken from the external model at every
    element GLL point (the mesher's model_external_values call per point)."""
    ib = db.ibool
    vp, vs, rho = external_model_values(m, db.xstore[ib], db.ystore[ib], db.zstore[ib])
    return db.with_model(vp.astype(np.float64), vs.astype(np.float64), rho.astype(np.float64))
