"""CPU restatement of the kernels-on-the-model-grid steps (test
infrastructure only): the checker ``sem_grid_project``, ``sem_grid_taper``
and ``sem_grid_zprecond`` are compared against.  Loaded only by the tests;
pinned to line-by-line transcriptions of the reference's loops in
``tests/golden/fortran_literal.py``.

After smoothing, ``PostFlow%pde_smooth`` projects every kernel from the GLL
points onto the regular model grid (``gll2grid``,
src/grid/model_grid_data.f90:183-198), and ``PostFlow%taper_kernel_grid``
multiplies the grid kernels by a 3-D boundary taper
(src/postproc/post_processing.f90:283-325, ``taper3d``,
src/postproc/taper_3D_mod.f90).  Both run on the host in the reference.

- ``gll2grid`` restates ``compute_interpolation_coeff_FD_SEM`` and
  ``Project_model_SEM2FD_grid`` (src/shared/projection_on_FD_grid_mod_fwat.f90:
  186-596) for one slice: elements in order; each element's grid
  candidates from its GLL bounding box, index ranges truncated as the
  Fortran integer assignment does; the candidate's reference coordinates
  from ``locate_point_in_element`` (:935-1125), whose Newton iterations
  clamp them to [-1, 1], so the 1.05 acceptance always holds and a
  candidate is taken by the first element whose range holds it (a point
  just outside an element takes the value on the element's face); its
  value is the element's 5x5x5 Lagrange interpolant there.  Points no
  element takes stay 0.  The locator starts from the nearest of the 27
  interior GLL nodes and takes ``NUM_ITER = 4`` Newton steps on the
  element's NGNOD anchor nodes (8: GLL corners; 27: corners, edge, face
  and centre nodes); on regular (affine) elements it is exact and the
  linear formula is used directly.
- ``Taper3D`` restates ``taper_cls``: a separable mask on a grid of
  spacing ``hx, hy, hz`` over the mesh's extent, zero for ``taph1`` from
  each side and the bottom, a half cosine over the next ``taph2``, one
  inside (no taper at the surface); ``interp`` is the trilinear ``interp3``
  (src/shared/utils.f90:1089-1159), zero outside the box.
- ``mesh_distances`` restates SPECFEM's ``check_mesh_distances`` (absent):
  the smallest and largest distance between neighbouring GLL points along
  the element directions; ``taper_kernel_grid`` spaces its mask by their
  mean.
- ``zprecond_grid`` is the depth preconditioner on the grid
  (src/postproc/zprecond.f90:73-100), as ``sum_precond`` uses it.
"""
from __future__ import annotations

import numpy as np

XG = np.array([-1.0, -np.sqrt(3.0 / 7.0), 0.0, np.sqrt(3.0 / 7.0), 1.0])


def lagrange5(x):
    """GLL Lagrange polynomials h_0..h_4 at the points x: [len(x), 5]."""
    x = np.asarray(x, np.float64)[:, None]
    h = np.ones((x.shape[0], 5))
    for i in range(5):
        for m in range(5):
            if m != i:
                h[:, i] *= (x[:, 0] - XG[m]) / (XG[i] - XG[m])
    return h


def _element_boxes(db):
    ib = np.asarray(db.ibool).reshape(db.nspec, 125)
    xyz = [np.asarray(a, np.float64)[ib] for a in (db.xstore, db.ystore, db.zstore)]
    return [(a.min(axis=1), a.max(axis=1)) for a in xyz]


NUM_ITER = 4


def _shape(u, m):
    """1-D Lagrange shape functions on m = 2 ([-1, 1]) or 3 ([-1, 0, 1])
    nodes at u [n]: values and derivatives [n, m]."""
    u = np.asarray(u, np.float64)
    if m == 2:
        return np.stack([0.5 * (1 - u), 0.5 * (1 + u)], 1), \
            np.stack([np.full_like(u, -0.5), np.full_like(u, 0.5)], 1)
    return np.stack([0.5 * u * (u - 1), 1 - u * u, 0.5 * u * (u + 1)], 1), \
        np.stack([u - 0.5, -2 * u, u + 0.5], 1)


def locate_in_element(nodes, targets, ngnod=8, niter=NUM_ITER):
    """``locate_point_in_element`` (projection_on_FD_grid_mod_fwat.f90:
    935-1125) for one element: ``nodes`` [5, 5, 5, 3] GLL point coordinates
    ([k][j][i]), ``targets`` [n, 3]; returns (xi, eta, gamma) [n, 3] after
    the initial guess at the nearest interior GLL node and ``niter`` Newton
    steps on the anchor-node mapping, each clamped to [-1, 1]."""
    t = np.asarray(targets, np.float64).reshape(-1, 3)
    inner = nodes[1:4, 1:4, 1:4].reshape(-1, 3)                    # k, j, i order
    best = np.argmin(((t[:, None, :] - inner[None]) ** 2).sum(-1), axis=1)
    k, j, i = np.unravel_index(best, (3, 3, 3))
    ref = np.stack([XG[i + 1], XG[j + 1], XG[k + 1]], 1)
    sel = [0, 4] if ngnod == 8 else [0, 2, 4]
    m = len(sel)
    anc = nodes[np.ix_(sel, sel, sel)]                              # [c][b][a][3]
    for _ in range(niter):
        (la, da), (lb, db_), (lc, dc) = (_shape(ref[:, q], m) for q in range(3))
        x = np.einsum("na,nb,nc,cbad->nd", la, lb, lc, anc)
        jac = np.stack([np.einsum("na,nb,nc,cbad->nd", da, lb, lc, anc),
                        np.einsum("na,nb,nc,cbad->nd", la, db_, lc, anc),
                        np.einsum("na,nb,nc,cbad->nd", la, lb, dc, anc)], axis=2)
        ref = np.clip(ref + np.linalg.solve(jac, (t - x)[..., None])[..., 0], -1.0, 1.0)
    return ref


def gll2grid(db, gll, x0, h, n, ngnod=8):
    """Project element values ``gll`` [nspec, 5, 5, 5] (Fortran dat(i,j,k,
    ispec) order, i fastest: [ispec][k][j][i]) onto the grid
    ``x0[d] + i h[d]``, i < n[d]; returns [nx, ny, nz] FP32.  ``ngnod``:
    anchor nodes of the mesher's elements (8 or 27), used on irregular
    elements."""
    if ngnod not in (8, 27):
        raise ValueError("ngnod must be 8 or 27")
    g = np.asarray(gll, np.float64).reshape(db.nspec, 5, 5, 5)
    irr = getattr(db, "irregular", None)
    irregular = (np.zeros(db.nspec, bool) if getattr(db, "geo", None) is None or irr is None
                 else np.asarray(irr) >= 0)
    ib5 = np.asarray(db.ibool).reshape(db.nspec, 5, 5, 5)
    xyz = np.stack([np.asarray(a, np.float64) for a in (db.xstore, db.ystore, db.zstore)], 1)
    x0 = np.asarray(x0, np.float64)
    h = np.asarray(h, np.float64)
    n = np.asarray(n, np.int64)
    boxes = _element_boxes(db)
    found = np.zeros(tuple(n), bool)
    out = np.zeros(tuple(n), np.float64)
    for e in range(db.nspec):
        rng, ref = [], []
        for d in range(3):
            lo, hi = boxes[d][0][e], boxes[d][1][e]
            # Fortran: kmin = 1 + (zmin - oz) / hz, truncated toward zero
            i0 = int(1 + (lo - x0[d]) / h[d]) - 1
            i1 = int(1 + (hi - x0[d]) / h[d]) - 1
            idx = np.arange(max(i0, 0), min(i1, n[d] - 1) + 1)
            if idx.size == 0:
                break
            c = x0[d] + idx * h[d]
            rng.append(idx)
            # the locator's Newton steps clamp to the element
            ref.append(np.clip(2.0 * (c - lo) / (hi - lo) - 1.0, -1.0, 1.0))
        if len(rng) < 3:
            continue
        ix, iy, iz = rng
        sub = np.ix_(ix, iy, iz)
        take = ~found[sub]
        if not take.any():
            continue
        if not irregular[e]:
            # affine element: the clamped linear coordinates are what the
            # locator's Newton steps reach; the 1.05 test always holds
            hx, hy, hz = (lagrange5(r) for r in ref)
            # sum_k sum_j sum_i hx_i hy_j hz_k g[e, k, j, i]
            val = np.einsum("ai,bj,ck,kji->abc", hx, hy, hz, g[e])
        else:
            gx, gy, gz = (x0[d] + rng[d] * h[d] for d in range(3))
            P = np.stack(np.meshgrid(gx, gy, gz, indexing="ij"), -1).reshape(-1, 3)
            r = locate_in_element(xyz[ib5[e]], P, ngnod)
            w = np.einsum("ni,nj,nk->nkji", lagrange5(r[:, 0]), lagrange5(r[:, 1]),
                          lagrange5(r[:, 2]))
            val = np.einsum("nkji,kji->n", w, g[e]).reshape(take.shape)
        blk = out[sub]
        blk[take] = val[take]
        out[sub] = blk
        fb = found[sub]
        fb[take] = True
        found[sub] = fb
    return out.astype(np.float32)


def coswin(n, opt):
    """``coswin`` (taper_3D_mod.f90): the rising (opt 1) or falling half of
    a 2n+1-point Hann window, without its centre."""
    nn = 2 * n + 1
    if n <= 0:
        return np.zeros(0)
    i = np.arange(nn)
    win = 0.5 - 0.5 * np.cos(2.0 * 3.1415926535 * i / (nn - 1))
    return win[:n] if opt == 1 else win[n + 1:]


def create_taper(taph1, taph2, tapz1, tapz2, hx, hy, hz, nx, ny, nz):
    """``create_taper`` (taper_3D_mod.f90): [nx, ny, nz] mask."""
    def side(n, h, t1, t2, both):
        w = np.zeros(n)
        nh1, nh2 = int(np.floor(t1 / h)), int(np.floor(t2 / h))
        a, b = nh1, nh1 + nh2                       # 0-based x1 - 1, x2 - 1
        w[a:b] = coswin(nh2, 1)
        if both:
            c, d = n - nh1 - nh2, n - nh1           # 0-based x3, x4 (exclusive)
            w[c:d] = coswin(nh2, 0)
            w[b:c] = 1.0
        else:
            w[b:] = 1.0
        return w
    xt = side(nx, hx, taph1, taph2, True)
    yt = side(ny, hy, taph1, taph2, True)
    zt = side(nz, hz, tapz1, tapz2, False)
    return xt[:, None, None] * yt[None, :, None] * zt[None, None, :]


class Taper3D:
    """``taper_cls``: the mask on its own grid and its interpolant."""

    def __init__(self, xmin, xmax, ymin, ymax, zmin, zmax, hx, hy, hz,
                 taph1, taph2, tapz1, tapz2):
        nx = int(np.floor((xmax - xmin) / hx + 1))
        ny = int(np.floor((ymax - ymin) / hy + 1))
        nz = int(np.floor((zmax - zmin) / hz + 1))
        self.x = xmin + np.arange(nx) * hx
        self.y = ymin + np.arange(ny) * hy
        self.z = zmin + np.arange(nz) * hz
        self.taper = create_taper(taph1, taph2, tapz1, tapz2, hx, hy, hz, nx, ny, nz)

    def interp(self, x, y, z):
        """Trilinear value at the points (x, y, z) (arrays of one shape);
        0 outside the mask's box."""
        x, y, z = (np.asarray(a, np.float64) for a in (x, y, z))
        inside = ((x >= self.x[0]) & (x <= self.x[-1]) & (y >= self.y[0]) & (y <= self.y[-1])
                  & (z >= self.z[0]) & (z <= self.z[-1]))
        out = np.zeros(np.broadcast(x, y, z).shape)

        def cell(c, v):
            # locate_bissection with the bracket clamped to [0, n-2]
            k = np.clip(np.searchsorted(c, v, side="right") - 1, 0, c.size - 2)
            return k, (v - c[k]) / (c[k + 1] - c[k])
        kx, fx = cell(self.x, x)
        ky, fy = cell(self.y, y)
        kz, fz = cell(self.z, z)
        t = self.taper
        val = 0.0
        for a, wa in ((0, 1 - fx), (1, fx)):
            for b, wb in ((0, 1 - fy), (1, fy)):
                for c, wc in ((0, 1 - fz), (1, fz)):
                    val = val + wa * wb * wc * t[kx + a, ky + b, kz + c]
        out[inside] = np.broadcast_to(val, out.shape)[inside]
        return out


def mesh_distances(db):
    """Smallest and largest distance between neighbouring GLL points along
    the element directions (SPECFEM's ``check_mesh_distances``, absent)."""
    ib = np.asarray(db.ibool).reshape(db.nspec, 5, 5, 5)
    p = np.stack([np.asarray(a, np.float64)[ib] for a in (db.xstore, db.ystore, db.zstore)],
                 axis=-1)                           # [e, k, j, i, 3]
    d = [np.linalg.norm(np.diff(p, axis=ax), axis=-1) for ax in (1, 2, 3)]
    return float(min(x.min() for x in d)), float(max(x.max() for x in d))


def taper_kernel_grid(db, grid_kernels, x0, h, n, h_suppress, h_buffer, v_suppress,
                      v_buffer):
    """``PostFlow%taper_kernel_grid``: grid kernels [..., nx, ny, nz] times
    the mask of spacing (distance_min + distance_max) / 2 over the mesh's
    extent, interpolated at the grid points."""
    dmin, dmax = mesh_distances(db)
    dh = 0.5 * (dmax + dmin)
    ext = [(float(np.min(a)), float(np.max(a))) for a in (db.xstore, db.ystore, db.zstore)]
    tap = Taper3D(ext[0][0], ext[0][1], ext[1][0], ext[1][1], ext[2][0], ext[2][1],
                  dh, dh, dh, h_suppress, h_buffer, v_suppress, v_buffer)
    gx, gy, gz = (np.asarray(x0[d], np.float64) + np.arange(n[d]) * h[d] for d in range(3))
    X, Y, Z = np.meshgrid(gx, gy, gz, indexing="ij")
    mask = tap.interp(X, Y, Z)
    return np.asarray(grid_kernels) * mask, mask


def zprecond_grid(zgrid, nx, ny, precond_type, nevents):
    """``zprecond_grid`` (src/postproc/zprecond.f90:73-100): the depth
    preconditioner on the model grid, [nx, ny, nz] FP32.  The 1-D profile
    of ``get_1d_precond`` (:11-32) on the levels ``zgrid`` (1e-8 above the
    surface, z + 1e-8 below; 1/|z| for type 2, 1/sqrt|z| for type 3),
    repeated over x and y, times the event count, normalised, inverted and
    normalised."""
    if precond_type not in (2, 3):
        raise ValueError("the depth forms are PRECOND_TYPE 2 and 3")
    z = np.asarray(zgrid, np.float64)
    zl = np.where(z > 0.0, 1e-8, z + 1e-8)
    zl = 1.0 / np.sqrt(zl * zl) if precond_type == 2 else 1.0 / np.sqrt(np.sqrt(zl * zl))
    h = np.broadcast_to(zl, (nx, ny, z.size)) * float(nevents)
    h = h / np.abs(h).max()
    h = 1.0 / h
    return (h / np.abs(h).max()).astype(np.float32)
