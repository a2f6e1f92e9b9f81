"""Regular-box mesh databases and seeded models for the elastic SEM solver.

This module produces, in memory, the arrays that the reference solver reads
from ``proc*_external_mesh.bin`` (layout in
``src/specfem_interface/read_mesh_databases.f90:158-193,455-486,766-804``):
``ibool``, GLL coordinates, ``kappastore``/``mustore``/``rhostore``, the
assembled mass ``rmass``, ``rho_vp``/``rho_vs`` and the Stacey absorbing
faces (``abs_boundary_ispec``, ``_ijk``, ``_jacobian2Dw``, ``_normal``).
The reference builds these with its own mesher
(``src/mesh_database_api/create_regions_mesh_fwat.f90:28-330``); that mesher
is not reproduced here.  Instead this module writes a structured box of
cubic elements (every element "regular": one ``xix_regular`` and one
``jacobian_regular`` for the whole mesh, ``read_mesh_databases.f90:168-170``)
and assigns a seeded model to its GLL points the way
``src/patch/model_external_values.f90:249-259`` does: trilinear
interpolation of a regular-grid model onto GLL points.

Array conventions (C order, 0-based indices):

* ``ibool[nspec, 5, 5, 5]`` is indexed ``[ispec, k, j, i]`` so that ``i`` is
  fastest in memory, which is the memory order of the Fortran
  ``ibool(i, j, k, ispec)``.
* ``abs_ijk[nf, 25, 3]`` holds ``(i, j, k)`` per face point (Fortran
  ``abs_boundary_ijk(3, 25, nf)``), ``abs_normal[nf, 25, 3]`` likewise.
* Coordinates are metres; ``z`` runs from ``-depth`` (bottom) to 0 (free
  surface on top).  Stacey faces cover the other five sides.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np

NGLL = 5


def gll_points_weights(n: int = NGLL):
    """GLL nodes and weights on [-1, 1] for ``n`` points (degree ``n-1``).

    Nodes are the end points plus the roots of P'_{n-1}, found by Newton
    iteration on the Legendre recurrence; weights are 2 / (N (N+1) P_N(x)^2)
    with N = n-1 (standard Gauss-Lobatto-Legendre quadrature).
    """
    N = n - 1
    x = -np.cos(np.pi * np.arange(n) / N)  # Chebyshev-Gauss-Lobatto start
    for _ in range(100):
        # P_N and P_{N-1} by recurrence
        p_prev = np.ones_like(x)
        p = x.copy()
        for k in range(2, N + 1):
            p_prev, p = p, ((2 * k - 1) * x * p - (k - 1) * p_prev) / k
        # Newton on (1-x^2) P'_N = N (P_{N-1} - x P_N): use the classic
        # Lobatto update x_new = x - (x P_N - P_{N-1}) / (n P_N)
        dx = (x * p - p_prev) / (n * p)
        x_new = x - dx
        if np.max(np.abs(x_new - x)) < 1e-16:
            x = x_new
            break
        x = x_new
    x[0], x[-1] = -1.0, 1.0
    p_prev = np.ones_like(x)
    p = x.copy()
    for k in range(2, N + 1):
        p_prev, p = p, ((2 * k - 1) * x * p - (k - 1) * p_prev) / k
    w = 2.0 / (N * (N + 1) * p * p)
    return x, w


@dataclasses.dataclass
class BoxSpec:
    """A box of ``nex x ney x nez`` cubic elements of edge ``h`` metres."""

    nex: int
    ney: int
    nez: int
    h: float = 4000.0
    x0: float = 0.0
    y0: float = 0.0

    @property
    def lx(self):
        return self.nex * self.h

    @property
    def ly(self):
        return self.ney * self.h

    @property
    def lz(self):
        return self.nez * self.h


@dataclasses.dataclass
class Database:
    """One mesh slice: the arrays a solver needs to run (see module doc)."""

    box: BoxSpec
    nspec: int
    nglob: int
    ibool: np.ndarray          # int32 [nspec,5,5,5]
    xstore: np.ndarray         # float32 [nglob]
    ystore: np.ndarray
    zstore: np.ndarray
    xix_regular: float
    jacobian_regular: float
    kappa: np.ndarray          # float32 [nspec,5,5,5]
    mu: np.ndarray
    rho: np.ndarray
    rmass: np.ndarray          # float32 [nglob]
    rho_vp: np.ndarray         # float32 [nspec,5,5,5]
    rho_vs: np.ndarray
    abs_ispec: np.ndarray      # int32 [nf]
    abs_ijk: np.ndarray        # int32 [nf,25,3]
    abs_jw: np.ndarray         # float32 [nf,25]
    abs_normal: np.ndarray     # float32 [nf,25,3]
    vp: Optional[np.ndarray] = None   # float32 [nspec,5,5,5] (diagnostics)
    vs: Optional[np.ndarray] = None
    # irregular elements (deformed meshes): irregular[e] = -1 for a regular
    # element, else its row in geo; geo [nirreg,5,5,5,10] holds xix, xiy,
    # xiz, etax, etay, etaz, gammax, gammay, gammaz, jacobian per point
    # (Fortran xixstore(i,j,k,ispec_irreg) ... jacobianstore)
    irregular: Optional[np.ndarray] = None
    geo: Optional[np.ndarray] = None

    @property
    def nspec_irregular(self):
        return 0 if self.geo is None else int(self.geo.shape[0])

    @property
    def nfaces(self):
        return int(self.abs_ispec.shape[0])

    def with_model(self, vp, vs, rho) -> "Database":
        """Return a copy whose material arrays come from (vp, vs, rho)."""
        kappa, mu, rho32, rho_vp, rho_vs, rmass = _materials(
            self, vp, vs, rho)
        return dataclasses.replace(
            self, kappa=kappa, mu=mu, rho=rho32, rho_vp=rho_vp,
            rho_vs=rho_vs, rmass=rmass,
            vp=vp.astype(np.float32), vs=vs.astype(np.float32))


def _materials(db: Database, vp, vs, rho):
    vp = np.asarray(vp, np.float64)
    vs = np.asarray(vs, np.float64)
    rho = np.asarray(rho, np.float64)
    mu = rho * vs * vs
    kappa = rho * vp * vp - 4.0 / 3.0 * mu
    _, w = gll_points_weights()
    www = (w[None, :, None, None] * w[None, None, :, None]
           * w[None, None, None, :])  # [1,k,j,i]
    jac = np.full(rho.shape, db.jacobian_regular, np.float64)
    if db.irregular is not None:
        sel = db.irregular >= 0
        jac[sel] = db.geo[db.irregular[sel], ..., 9]
    mass_el = rho * www * jac
    rmass = np.zeros(db.nglob, np.float64)
    np.add.at(rmass, db.ibool.reshape(-1), mass_el.reshape(-1))
    f = np.float32
    return (kappa.astype(f), mu.astype(f), rho.astype(f),
            (rho * vp).astype(f), (rho * vs).astype(f), rmass.astype(f))


def hill_topography(box: BoxSpec, height: float, width: float):
    """A Gaussian hill of ``height`` metres and 1/e half-width ``width``
    centred on the box, as a function z_surface(x, y)."""
    cx, cy = box.x0 + 0.5 * box.lx, box.y0 + 0.5 * box.ly

    def f(x, y):
        return height * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / width ** 2)
    return f


def gll_derivative_matrix():
    """D[i][l] = l_l'(xi_i) for the GLL nodes (FP64)."""
    x, _ = gll_points_weights()
    n = len(x)
    D = np.zeros((n, n))
    for i in range(n):
        for l in range(n):
            s = 0.0
            for m in range(n):
                if m == l:
                    continue
                prod = 1.0 / (x[l] - x[m])
                for q in range(n):
                    if q not in (l, m):
                        prod *= (x[i] - x[q]) / (x[l] - x[q])
                s += prod
            D[i, l] = s
    return D


def _geometry(ibool, xs, ys, zs):
    """Mapping derivatives of every element from its GLL coordinates:
    returns dX [nspec,5,5,5,3(a),3(d)] = dx_a/dxi_d (k, j, i order)."""
    D = gll_derivative_matrix()
    X = np.stack([xs[ibool], ys[ibool], zs[ibool]], axis=-1)   # [e,k,j,i,a]
    dxi = np.einsum("il,ekjla->ekjia", D, X)
    deta = np.einsum("jl,eklia->ekjia", D, X)
    dgam = np.einsum("kl,eljia->ekjia", D, X)
    return np.stack([dxi, deta, dgam], axis=-1)


def interior_warp(box: BoxSpec, amp: float):
    """Smooth displacement of the mesh interior that vanishes on the box
    faces: (dx, dy, dz) = amp * s(x) s(y) s(z) * (1, -1, 1) with
    s(q) = sin(pi (q - q0) / L)."""
    def f(x, y, z):
        s = (np.sin(np.pi * (x - box.x0) / box.lx) * np.sin(np.pi * (y - box.y0) / box.ly)
             * np.sin(np.pi * (z + box.lz) / box.lz))
        return amp * s, -amp * s, amp * s
    return f


def make_box(box: BoxSpec, absorb_top: bool = False, topo=None, warp=None) -> Database:
    """Structured mesh, global numbering and Stacey faces of a box.

    Global points form a ``(4 nex + 1) x (4 ney + 1) x (4 nez + 1)`` grid
    numbered x-fastest; elements are numbered x-fastest too, bottom layer
    first.  ``absorb_top`` also makes the top face absorbing (a full-space
    test box).  ``topo(x, y)`` stretches the columns so the free surface
    follows it (bottom fixed); ``warp(x, y, z)`` displaces every point.
    Either makes elements irregular: their mapping derivatives and Jacobian
    are computed from the GLL coordinates and stored per point in ``geo``,
    and the Stacey faces get per-point normals and jacobian2Dw.  The model
    arrays are left at zero: call :func:`homogeneous` or :func:`with_model`
    next.
    """
    nex, ney, nez, h = box.nex, box.ney, box.nez, box.h
    nxg, nyg, nzg = 4 * nex + 1, 4 * ney + 1, 4 * nez + 1
    nspec = nex * ney * nez
    nglob = nxg * nyg * nzg
    xi, w = gll_points_weights()

    ex, ey, ez = np.meshgrid(np.arange(nex), np.arange(ney), np.arange(nez),
                             indexing="ij")
    # element order: ex fastest, then ey, then ez
    ex = ex.transpose(2, 1, 0).reshape(-1)
    ey = ey.transpose(2, 1, 0).reshape(-1)
    ez = ez.transpose(2, 1, 0).reshape(-1)
    ii = np.arange(NGLL)
    gi = 4 * ex[:, None, None, None] + ii[None, None, None, :]
    gj = 4 * ey[:, None, None, None] + ii[None, None, :, None]
    gk = 4 * ez[:, None, None, None] + ii[None, :, None, None]
    ibool = (gi + nxg * (gj + nyg * gk)).astype(np.int32)

    # 1-D coordinates of the global GLL grid lines
    def lines(n_el, origin):
        c = np.empty(4 * n_el + 1, np.float64)
        for e in range(n_el):
            c[4 * e:4 * e + 5] = origin + e * h + (xi + 1.0) * 0.5 * h
        return c

    xl = lines(nex, box.x0)
    yl = lines(ney, box.y0)
    zl = lines(nez, -box.lz)
    gx = np.arange(nglob) % nxg
    gy = (np.arange(nglob) // nxg) % nyg
    gz = np.arange(nglob) // (nxg * nyg)
    xg64, yg64, zg64 = xl[gx], yl[gy], zl[gz]
    if topo is not None:
        # columns stretched so the top follows topo(x, y), bottom fixed
        zg64 = zg64 + topo(xg64, yg64) * (zg64 + box.lz) / box.lz
    if warp is not None:
        dxw, dyw, dzw = warp(xg64, yg64, zg64)
        xg64, yg64, zg64 = xg64 + dxw, yg64 + dyw, zg64 + dzw
    xstore = xg64.astype(np.float32)
    ystore = yg64.astype(np.float32)
    zstore = zg64.astype(np.float32)
    irregular = geo = None
    dX = None
    if topo is not None or warp is not None:
        dX = _geometry(ibool, xg64, yg64, zg64)                  # [e,k,j,i,3,3]
        jac = np.linalg.det(dX)
        inv = np.linalg.inv(dX)                                   # [.., d, a] = dxi_d/dx_a
        reg = np.zeros_like(dX)
        for a in range(3):
            reg[..., a, a] = 0.5 * h
        dev = np.abs(dX - reg).reshape(nspec, -1).max(axis=1)
        irr = dev > 1e-9 * h
        irregular = np.full(nspec, -1, np.int32)
        irregular[irr] = np.arange(int(irr.sum()), dtype=np.int32)
        g = np.concatenate([inv.reshape(inv.shape[:4] + (9,)), jac[..., None]], axis=-1)
        geo = g[irr].astype(np.float32)

    # Stacey faces: xmin, xmax, ymin, ymax, zmin (top is a free surface)
    a = np.arange(NGLL)
    A, B = np.meshgrid(a, a, indexing="xy")  # A fastest
    A = A.reshape(-1)
    B = B.reshape(-1)
    jw2 = (w[A] * w[B] * (0.5 * h) ** 2).astype(np.float32)
    faces_ispec, faces_ijk, faces_n = [], [], []

    faces_jw = []

    def add(sel, ijk, normal):
        els = np.nonzero(sel)[0]
        for e in els:
            faces_ispec.append(e)
            faces_ijk.append(ijk)
            if dX is None:
                faces_n.append(np.broadcast_to(np.asarray(normal, np.float64), (25, 3)))
                faces_jw.append(jw2.astype(np.float64))
                continue
            # deformed face: n = t1 x t2 of the two in-face mapping
            # derivatives, oriented outward; jacobian2D = |n|
            ii_, jj_, kk_ = ijk[:, 0], ijk[:, 1], ijk[:, 2]
            J = dX[e, kk_, jj_, ii_]                      # [25, a, d]
            fixed = [d for d in range(3) if np.all(ijk[:, d] == ijk[0, d])][0]
            d1, d2 = [d for d in range(3) if d != fixed]
            nv = np.cross(J[:, :, d1], J[:, :, d2])
            nv *= np.sign((nv * np.asarray(normal)).sum(axis=1))[:, None]
            nn = np.linalg.norm(nv, axis=1)
            faces_n.append(nv / nn[:, None])
            faces_jw.append(nn * w[ijk[:, d1]] * w[ijk[:, d2]])

    z4 = np.full(25, 4)
    z0 = np.zeros(25, np.int64)
    add(ex == 0, np.stack([z0, A, B], 1), (-1.0, 0.0, 0.0))
    add(ex == nex - 1, np.stack([z4, A, B], 1), (1.0, 0.0, 0.0))
    add(ey == 0, np.stack([A, z0, B], 1), (0.0, -1.0, 0.0))
    add(ey == ney - 1, np.stack([A, z4, B], 1), (0.0, 1.0, 0.0))
    add(ez == 0, np.stack([A, B, z0], 1), (0.0, 0.0, -1.0))
    if absorb_top:
        add(ez == nez - 1, np.stack([A, B, z4], 1), (0.0, 0.0, 1.0))
    nf = len(faces_ispec)
    abs_ispec = np.asarray(faces_ispec, np.int32)
    abs_ijk = np.asarray(faces_ijk, np.int32).reshape(nf, 25, 3)
    abs_normal = np.asarray(faces_n, np.float32).reshape(nf, 25, 3)
    abs_jw = np.asarray(faces_jw, np.float32).reshape(nf, 25)

    z = np.zeros((nspec, NGLL, NGLL, NGLL), np.float32)
    return Database(
        box=box, nspec=nspec, nglob=nglob,
        ibool=ibool.reshape(nspec, NGLL, NGLL, NGLL),
        xstore=xstore, ystore=ystore, zstore=zstore,
        xix_regular=float(2.0 / h), jacobian_regular=float((0.5 * h) ** 3),
        kappa=z, mu=z, rho=z, rmass=np.zeros(nglob, np.float32),
        rho_vp=z, rho_vs=z, abs_ispec=abs_ispec, abs_ijk=abs_ijk,
        abs_jw=abs_jw, abs_normal=abs_normal, irregular=irregular, geo=geo)


def gll_xyz(db: Database):
    """Per element-point coordinates [nspec,5,5,5] (float64)."""
    ib = db.ibool
    return (db.xstore[ib].astype(np.float64), db.ystore[ib].astype(np.float64),
            db.zstore[ib].astype(np.float64))


def gaussian_random_field(box: BoxSpec, corr_len: float, seed: int,
                          spacing: float = 1000.0):
    """Unit-variance Gaussian random field on a regular grid over the box.

    White noise is filtered in the wavenumber domain by the square root of
    the spectrum of the Gaussian covariance ``exp(-r^2 / corr_len^2)`` on a
    grid padded by ``4 corr_len`` per side (so the periodic FFT does not wrap
    correlations across the box), then cut to the box and normalised.
    Returns ``(grid, origin, spacing)`` with grid indexed [ix, iy, iz].
    """
    pad = 4.0 * corr_len
    n = [int(math.ceil((L + 2 * pad) / spacing)) + 1
         for L in (box.lx, box.ly, box.lz)]
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal(n)
    k = [2 * np.pi * np.fft.fftfreq(m, d=spacing) for m in n[:2]]
    kz = 2 * np.pi * np.fft.rfftfreq(n[2], d=spacing)
    K2 = (k[0][:, None, None] ** 2 + k[1][None, :, None] ** 2
          + kz[None, None, :] ** 2)
    filt = np.exp(-K2 * corr_len * corr_len / 8.0)
    field = np.fft.irfftn(np.fft.rfftn(noise) * filt, s=n, axes=(0, 1, 2))
    i0 = int(round(pad / spacing))
    nb = [int(math.ceil(L / spacing)) + 1 for L in (box.lx, box.ly, box.lz)]
    g = field[i0:i0 + nb[0], i0:i0 + nb[1], i0:i0 + nb[2]]
    g = (g - g.mean()) / g.std()
    origin = (box.x0, box.y0, -box.lz)
    return g, origin, spacing


def trilinear(grid, origin, spacing, x, y, z):
    """Trilinear interpolation of ``grid[ix,iy,iz]`` at points (x, y, z),
    with the nearest grid value outside the grid (the rule of
    ``model_external_values.f90:249-259``)."""
    out_shape = np.shape(x)
    p = [(np.asarray(c, np.float64).reshape(-1) - o) / spacing
         for c, o in zip((x, y, z), origin)]
    idx, frac = [], []
    for d in range(3):
        n = grid.shape[d]
        q = np.clip(p[d], 0.0, n - 1.0)
        i = np.minimum(np.floor(q).astype(np.int64), n - 2)
        idx.append(i)
        frac.append(q - i)
    i, j, k = idx
    fx, fy, fz = frac
    val = np.zeros_like(fx)
    for di in (0, 1):
        wx = fx if di else 1.0 - fx
        for dj in (0, 1):
            wy = fy if dj else 1.0 - fy
            for dk in (0, 1):
                wz = fz if dk else 1.0 - fz
                val += wx * wy * wz * grid[i + di, j + dj, k + dk]
    return val.reshape(out_shape)


def random_field_at_gll(db: Database, corr_len=8000.0, seed=1234,
                        spacing=1000.0):
    """Seeded unit-variance field ``g`` at every element GLL point."""
    g, origin, ds = gaussian_random_field(db.box, corr_len, seed, spacing)
    gglob = trilinear(g, origin, ds, db.xstore, db.ystore, db.zstore)
    return gglob[db.ibool]


def background_model(db: Database, seed=1234, perturb=0.05,
                     vp0=6000.0, vs0=3464.0, rho0=2700.0):
    """vp, vs, rho = (6000, 3464, 2700) x (1 + perturb * g)."""
    g = random_field_at_gll(db, seed=seed) if perturb else 0.0
    s = 1.0 + perturb * g
    shape = db.ibool.shape
    return (np.broadcast_to(vp0 * s, shape), np.broadcast_to(vs0 * s, shape),
            np.broadcast_to(rho0 * s, shape))


LAYERS = ((0.0, 20000.0, 5800.0, 3350.0, 2600.0),
          (20000.0, 36000.0, 6500.0, 3750.0, 2900.0),
          (36000.0, 1e30, 8000.0, 4500.0, 3300.0))


def layered_model(db: Database, seed=1234, perturb=0.03):
    """Three layers (0-20 km, 20-36 km, below 36 km depth; interfaces on
    element boundaries, layer picked per element by its centroid depth)
    times (1 + perturb * g)."""
    x, y, z = gll_xyz(db)
    depth_c = -z.mean(axis=(1, 2, 3))
    vp = np.empty(db.ibool.shape)
    vs = np.empty_like(vp)
    rho = np.empty_like(vp)
    for top, bot, a, b, r in LAYERS:
        sel = (depth_c >= top) & (depth_c < bot)
        vp[sel], vs[sel], rho[sel] = a, b, r
    if perturb:
        s = 1.0 + perturb * random_field_at_gll(db, seed=seed)
        vp, vs, rho = vp * s, vs * s, rho * s
    return vp, vs, rho


def gaussian_vs_anomaly(db: Database, vs, amp=0.10, radius=15000.0,
                        depth=30000.0):
    """vs x (1 + amp exp(-r^2/radius^2)), centred mid-box at ``depth``."""
    x, y, z = gll_xyz(db)
    cx = db.box.x0 + 0.5 * db.box.lx
    cy = db.box.y0 + 0.5 * db.box.ly
    r2 = (x - cx) ** 2 + (y - cy) ** 2 + (z + depth) ** 2
    return vs * (1.0 + amp * np.exp(-r2 / (radius * radius)))


def as_irregular(db: Database) -> Database:
    """The same regular mesh with every element flagged irregular and its
    constant mapping stored per point: runs the general-element path on a
    mesh whose answer the regular path gives."""
    geo = np.zeros((db.nspec, NGLL, NGLL, NGLL, 10), np.float32)
    for d in range(3):
        geo[..., 4 * d] = db.xix_regular
    geo[..., 9] = db.jacobian_regular
    return dataclasses.replace(db, irregular=np.arange(db.nspec, dtype=np.int32), geo=geo)


def surface_receivers(box: BoxSpec, n: int, frac=(0.2, 0.8)):
    """``n x n`` receivers on the free surface (z = 0) spanning the central
    part of the box.  Returns float64 [n*n, 3]."""
    t = np.linspace(frac[0], frac[1], n)
    xs = box.x0 + t * box.lx
    ys = box.y0 + t * box.ly
    X, Y = np.meshgrid(xs, ys, indexing="xy")
    return np.stack([X.reshape(-1), Y.reshape(-1),
                     np.zeros(n * n)], 1).astype(np.float64)


# -- the standard workloads -------------------------------------------------

def config_box(name: str) -> BoxSpec:
    """Mesh of a named workload: ``small`` (10x10x10 el over 40 km),
    ``medium`` (40x40x20 el over 160x160x80 km), ``large`` (96x96x48 el over
    384x384x192 km).  All elements are 4 km cubes."""
    return {"small": BoxSpec(10, 10, 10), "medium": BoxSpec(40, 40, 20),
            "large": BoxSpec(96, 96, 48)}[name]


def build(name: str, seed: int = 1234, anomaly: bool = False) -> Database:
    """Mesh + model of a named workload (``tiny`` = 3x3x3 el test box)."""
    if name == "tiny":
        box = BoxSpec(3, 3, 3)
    elif name == "mini":
        box = BoxSpec(6, 6, 4)
    else:
        box = config_box(name)
    db = make_box(box)
    if name == "large":
        vp, vs, rho = layered_model(db, seed=seed)
    else:
        vp, vs, rho = background_model(db, seed=seed)
    if anomaly:
        vs = gaussian_vs_anomaly(db, vs)
    return db.with_model(vp, vs, rho)


def homogeneous(db: Database, vp=6000.0, vs=3464.0, rho=2700.0) -> Database:
    shape = db.ibool.shape
    return db.with_model(np.full(shape, vp), np.full(shape, vs),
                         np.full(shape, rho))


def random_moment_tensor(rng, m0=1.0e16):
    """Random CMT-convention (Mrr, Mtt, Mpp, Mrt, Mrp, Mtp) of Euclidean
    norm ``m0`` (N m)."""
    m = rng.standard_normal(6)
    return m0 * m / np.linalg.norm(m)
