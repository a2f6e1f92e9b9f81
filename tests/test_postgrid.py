"""Kernels on the model grid: the CPU restatement ``oracle.postgrid``
that the device's ``sem_grid_*`` entry points are checked against
(``tests/test_gpu_grid.py``), pinned here to the reference's loops.

- ``gll2grid`` equals a line-by-line transcription of the reference's
  projection loop (first element wins, locator coordinates clamped to the
  element, truncated index ranges; tests/golden/fortran_literal.py) on a
  grid that is not aligned with the elements, including points outside
  the mesh;
- it reproduces a field that is a polynomial of degree <= 4 per element
  exactly at any grid point;
- ``create_taper`` and the trilinear ``Taper3D.interp`` equal FP32
  transcriptions of taper_3D_mod.f90 and utils.f90's ``interp3``;
- ``mesh_distances`` on a cube of edge h gives the GLL spacings, so the
  taper grid's spacing is h / 4, and ``taper_kernel_grid`` leaves the
  interior alone, zeroes the suppressed border and keeps the surface.
"""
import os
import sys

import numpy as np
import pytest

from specfwat_b200 import database as D
from oracle.postgrid import (Taper3D, create_taper, gll2grid, mesh_distances,
                             taper_kernel_grid)

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import fortran_literal as F  # noqa: E402


def small_box():
    return D.make_box(D.BoxSpec(3, 2, 2, h=2000.0))


def test_gll2grid_matches_literal_loop():
    db = small_box()
    rng = np.random.default_rng(3)
    data = rng.standard_normal((db.nspec, 5, 5, 5))       # discontinuous across elements
    x0, h, n = (-700.0, -300.0, -4200.0), (550.0, 610.0, 470.0), (13, 8, 10)
    ours = gll2grid(db, data, x0, h, n)
    lit = F.project_sem2fd((db.ibool.reshape(-1) + 1).tolist(), db.xstore, db.ystore,
                           db.zstore, db.nspec, data.reshape(-1), *x0, *h, *n)
    lit = np.asarray(lit, np.float64)
    assert np.abs(ours - lit).max() <= 1e-6 * np.abs(lit).max()
    # x = -700 and z = +30 are no element's candidates and stay zero;
    # x = -150 is a candidate of the first elements through the truncated
    # index range and takes their value on the face x = 0
    assert np.all(ours[0] == 0.0) and np.all(ours[:, :, -1] == 0.0)
    assert np.all(ours[1:, :, :-1] != 0.0)


def test_gll2grid_clamps_to_the_element_face():
    """x = -40 m lies outside the first elements; it is their candidate and
    takes their value on the face x = 0, since the locator clamps xi to -1."""
    db = small_box()
    rng = np.random.default_rng(4)
    data = rng.standard_normal((db.nspec, 5, 5, 5))
    x0, h, n = (-40.0, 35.0, -3980.0), (550.0, 610.0, 470.0), (12, 7, 9)
    ours = gll2grid(db, data, x0, h, n)
    lit = np.asarray(F.project_sem2fd((db.ibool.reshape(-1) + 1).tolist(), db.xstore,
                                      db.ystore, db.zstore, db.nspec, data.reshape(-1),
                                      *x0, *h, *n), np.float64)
    assert np.abs(ours - lit).max() <= 1e-6 * np.abs(lit).max()
    face = gll2grid(db, data, (0.0, 35.0, -3980.0), (550.0, 610.0, 470.0), (1, 7, 9))
    assert np.array_equal(ours[0], face[0])


def test_gll2grid_is_exact_for_element_polynomials():
    db = small_box()
    ib = db.ibool.reshape(-1)
    x, y, z = (np.asarray(a, np.float64)[ib] for a in (db.xstore, db.ystore, db.zstore))
    f = lambda x, y, z: 1e-8 * x * x - 3e-9 * y * z + 1e-16 * z ** 4 + 2e-4 * x  # noqa: E731
    data = f(x, y, z).reshape(db.nspec, 5, 5, 5)
    x0, h, n = (100.0, 150.0, -3900.0), (700.0, 450.0, 380.0), (8, 8, 10)
    grid = gll2grid(db, data, x0, h, n)
    gx, gy, gz = (x0[d] + np.arange(n[d]) * h[d] for d in range(3))
    X, Y, Z = np.meshgrid(gx, gy, gz, indexing="ij")
    ref = f(X, Y, Z)
    assert np.abs(grid - ref).max() <= 1e-5 * np.abs(ref).max()


def test_gll2grid_topography_matches_literal_locator():
    """All elements irregular: every candidate is located by the Newton
    iteration on the 8 anchor nodes, as in the transcription."""
    box = D.BoxSpec(3, 2, 2, h=2000.0)
    db = D.make_box(box, topo=D.hill_topography(box, 1200.0, 2500.0))
    assert db.nspec_irregular == db.nspec
    rng = np.random.default_rng(6)
    data = rng.standard_normal((db.nspec, 5, 5, 5))
    x0, h, n = (-300.0, 120.0, -4100.0), (610.0, 560.0, 700.0), (11, 8, 9)
    ours = gll2grid(db, data, x0, h, n)
    lit = np.asarray(F.project_sem2fd_located(
        (db.ibool.reshape(-1) + 1).tolist(), db.xstore, db.ystore, db.zstore, db.nspec,
        data.reshape(-1), *x0, *h, *n), np.float64)
    assert np.abs(ours - lit).max() <= 1e-5 * np.abs(lit).max()
    assert np.count_nonzero(ours) > 0.5 * ours.size


def test_gll2grid_newton_path_equals_linear_path():
    """A regular box flagged irregular takes the Newton locator, which must
    land where the linear formula does."""
    db = small_box()
    rng = np.random.default_rng(7)
    data = rng.standard_normal((db.nspec, 5, 5, 5))
    x0, h, n = (-700.0, -300.0, -4200.0), (550.0, 610.0, 470.0), (13, 8, 10)
    a = gll2grid(db, data, x0, h, n)
    b = gll2grid(D.as_irregular(db), data, x0, h, n)
    assert np.abs(a - b).max() <= 1e-5 * np.abs(a).max()


def test_gll2grid_linear_field_on_topography():
    """A linear field on a topography mesh.  Most grid points come back to
    the interpolation accuracy; a few do not, by the reference's rule: on a
    deformed mesh element bounding boxes overlap, and the first element
    whose box holds a point takes it at the clamped (face) coordinate even
    when the point lies in the next element."""
    box = D.BoxSpec(4, 4, 3, h=2000.0)
    db = D.make_box(box, topo=D.hill_topography(box, 800.0, 3000.0))
    ib = db.ibool.reshape(-1)
    f = lambda x, y, z: 1.0 + 2e-5 * x - 3e-5 * y + 4e-5 * z  # noqa: E731
    data = f(*(np.asarray(a, np.float64)[ib] for a in (db.xstore, db.ystore, db.zstore)))
    x0, h, n = (500.0, 500.0, -5500.0), (700.0, 700.0, 600.0), (10, 10, 9)
    grid = gll2grid(db, data.reshape(db.nspec, 5, 5, 5), x0, h, n, ngnod=27)
    gx, gy, gz = (x0[d] + np.arange(n[d]) * h[d] for d in range(3))
    X, Y, Z = np.meshgrid(gx, gy, gz, indexing="ij")
    ref = f(X, Y, Z)
    err = np.abs(grid - ref)
    assert np.median(err) < 1e-4 and np.percentile(err, 95) < 1e-3 and err.max() < 5e-3
    with pytest.raises(ValueError, match="ngnod"):
        gll2grid(db, data.reshape(db.nspec, 5, 5, 5), x0, h, n, ngnod=20)


@pytest.mark.parametrize("args", [(3000.0, 5000.0, 2000.0, 4000.0, 500.0, 500.0, 400.0, 41, 37, 30),
                                  (0.0, 2000.0, 0.0, 1500.0, 800.0, 700.0, 300.0, 20, 19, 17)])
def test_create_taper_matches_literal(args):
    ours = create_taper(*args)
    lit = F.create_taper(*args)
    assert np.abs(ours - lit).max() < 2e-6


def test_taper_interp_matches_literal():
    tap = Taper3D(0.0, 16000.0, 0.0, 12000.0, -8000.0, 0.0, 1000.0, 1000.0, 1000.0,
                  2000.0, 3000.0, 1000.0, 2000.0)
    rng = np.random.default_rng(5)
    pts = np.stack([rng.uniform(-500, 16500, 200), rng.uniform(-500, 12500, 200),
                    rng.uniform(-8500, 500, 200)], axis=1)
    pts[:4] = [[0.0, 0.0, -8000.0], [16000.0, 12000.0, 0.0], [8000.0, 6000.0, -4000.0],
               [16000.0, 3000.0, -2000.0]]
    ours = tap.interp(pts[:, 0], pts[:, 1], pts[:, 2])
    t = tap.taper.tolist()
    for p, v in zip(pts, ours):
        inside = (0 <= p[0] <= 16000) and (0 <= p[1] <= 12000) and (-8000 <= p[2] <= 0)
        lit = F.interp3(tap.x, tap.y, tap.z, t, *p) if inside else 0.0
        assert v == pytest.approx(lit, abs=1e-9), p


def test_mesh_distances_and_taper_kernel_grid():
    box = D.BoxSpec(8, 8, 4, h=2000.0)
    db = D.make_box(box)
    dmin, dmax = mesh_distances(db)
    assert dmin == pytest.approx(1000.0 * (1 - np.sqrt(3 / 7)), rel=1e-6)
    assert dmax == pytest.approx(1000.0 * np.sqrt(3 / 7), rel=1e-6)
    assert 0.5 * (dmin + dmax) == pytest.approx(500.0)
    n = (33, 33, 17)
    ker = np.ones((2,) + n)
    out, mask = taper_kernel_grid(db, ker, (0.0, 0.0, -8000.0), (500.0, 500.0, 500.0), n,
                                  1000.0, 2000.0, 1000.0, 2000.0)
    assert out.shape == ker.shape and np.array_equal(out[0], mask)
    assert np.all(mask[16, 16, 8:] == 1.0)          # interior and the surface column
    assert np.all(mask[0] == 0.0) and np.all(mask[:, :, 0] == 0.0)
    assert mask[16, 16, -1] == 1.0                  # no taper at the free surface
    assert 0.0 < mask[3, 16, 16] < 1.0              # the cosine ramp


@pytest.mark.parametrize("ptype", [2, 3])
def test_zprecond_grid_matches_literal(ptype):
    from oracle.postgrid import zprecond_grid
    zg = np.linspace(-30000.0, 2000.0, 17)
    ours = zprecond_grid(zg, 4, 3, ptype, 6)
    zl = np.array(F.get_1d_precond(zg, ptype), np.float32)
    h = np.broadcast_to(zl, (4, 3, zg.size)).astype(np.float32) * np.float32(6)
    h = h / np.abs(h).max()
    h = np.float32(1.0) / h
    lit = h / np.abs(h).max()
    assert ours.shape == (4, 3, 17)
    assert np.abs(ours - lit).max() <= 2e-6
    # deeper levels get the larger preconditioner
    assert np.all(np.diff(ours[0, 0][zg < 0]) < 0)
    with pytest.raises(ValueError):
        zprecond_grid(zg, 2, 2, 1, 1)
