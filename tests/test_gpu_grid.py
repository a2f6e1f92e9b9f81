"""Kernels on the model grid on the device (``sem_grid_project``,
``sem_grid_taper``, ``sem_grid_zprecond``) against the CPU restatement
``oracle.postgrid``, which ``tests/test_postgrid.py`` pins to the
reference's loops.

- The projection keeps the reference's ownership rule: a grid point is the
  first element's whose candidate range holds it. A grid aligned with the
  element faces and element fields that jump across the faces make every
  shared point depend on that rule. So do points just outside the mesh,
  which take the face value of the first element that lists them.
- Irregular elements go through the locator's Newton steps on 8 and 27
  anchor nodes.
- Both sides compute in FP64 and round to FP32; they agree to a few FP32
  ulps of the field's largest value.
"""
import numpy as np
import pytest

from oracle import postgrid as O
from specfwat_b200 import _lib
from specfwat_b200 import database as D
from specfwat_b200 import postgrid as P
from specfwat_b200 import solver as S

pytestmark = pytest.mark.gpu


def close(dev, ref, tol=1e-6):
    ref = np.asarray(ref, np.float64)
    return np.abs(np.asarray(dev, np.float64) - ref).max() <= tol * np.abs(ref).max()


def modelled(db):
    return db.with_model(*D.background_model(db, seed=30))


def small_box():
    return modelled(D.make_box(D.BoxSpec(3, 2, 2, h=2000.0)))


GRIDS = [((-700.0, -300.0, -4200.0), (550.0, 610.0, 470.0), (13, 8, 10)),   # unaligned, outside
         ((0.0, 0.0, -4000.0), (500.0, 500.0, 500.0), (13, 9, 9)),          # on the faces
         ((-40.0, 35.0, -3980.0), (550.0, 610.0, 470.0), (12, 7, 9))]       # just outside x = 0


@pytest.mark.parametrize("grid", GRIDS)
def test_project_matches_oracle(gpu, grid):
    db = small_box()
    rng = np.random.default_rng(31)
    data = rng.standard_normal((3, db.nspec, 5, 5, 5)).astype(np.float32)
    x0, h, n = grid
    mesh = S.Mesh(db)
    dev = P.gll2grid(mesh, data, x0, h, n)
    one = P.gll2grid(mesh, data[1], x0, h, n)
    mesh.close()
    assert dev.shape == (3,) + n and dev.dtype == np.float32
    assert np.array_equal(one, dev[1])
    for f in range(3):
        ref = O.gll2grid(db, data[f].astype(np.float64), x0, h, n)
        assert np.array_equal(dev[f] == 0.0, ref == 0.0)       # the same points taken
        assert close(dev[f], ref), f


@pytest.mark.parametrize("ngnod", [8, 27])
def test_project_topography_matches_oracle(gpu, ngnod):
    box = D.BoxSpec(3, 2, 2, h=2000.0)
    db = modelled(D.make_box(box, topo=D.hill_topography(box, 1200.0, 2500.0)))
    assert db.nspec_irregular == db.nspec
    rng = np.random.default_rng(32)
    data = rng.standard_normal((db.nspec, 5, 5, 5)).astype(np.float32)
    x0, h, n = (-300.0, 120.0, -4100.0), (610.0, 560.0, 700.0), (11, 8, 9)
    mesh = S.Mesh(db)
    dev = P.gll2grid(mesh, data, x0, h, n, ngnod=ngnod)
    mesh.close()
    ref = O.gll2grid(db, data.astype(np.float64), x0, h, n, ngnod=ngnod)
    assert np.array_equal(dev == 0.0, ref == 0.0)
    assert close(dev, ref, 1e-5)
    assert np.count_nonzero(dev) > 0.5 * dev.size


def test_project_newton_on_a_regular_box_equals_linear(gpu):
    db = small_box()
    rng = np.random.default_rng(33)
    data = rng.standard_normal((db.nspec, 5, 5, 5)).astype(np.float32)
    x0, h, n = GRIDS[0]
    m1, m2 = S.Mesh(db), S.Mesh(D.as_irregular(db))
    a = P.gll2grid(m1, data, x0, h, n)
    b = P.gll2grid(m2, data, x0, h, n)
    m1.close()
    m2.close()
    assert close(b, a, 1e-5)


def test_project_medium_mesh(gpu):
    """The bench's medium mesh on a 2 km grid that overhangs it: 2.1M GLL
    points, 32,000 elements."""
    db = D.build("medium")
    rng = np.random.default_rng(34)
    data = rng.standard_normal((db.nspec, 5, 5, 5)).astype(np.float32)
    x0, h, n = (-1000.0, -1000.0, -81000.0), (2000.0, 2000.0, 2000.0), (82, 82, 42)
    mesh = S.Mesh(db)
    dev = P.gll2grid(mesh, data, x0, h, n)
    mesh.close()
    ref = O.gll2grid(db, data.astype(np.float64), x0, h, n)
    assert np.array_equal(dev == 0.0, ref == 0.0)
    assert close(dev, ref)


def test_taper_matches_oracle(gpu):
    db = modelled(D.make_box(D.BoxSpec(8, 8, 4, h=2000.0)))
    n = (33, 33, 17)
    x0, h = (0.0, 0.0, -8000.0), (500.0, 500.0, 500.0)
    rng = np.random.default_rng(35)
    ker = rng.standard_normal((2,) + n).astype(np.float32)
    mesh = S.Mesh(db)
    out, mask = P.taper_kernel_grid(mesh, ker, x0, h, n, 1000.0, 2000.0, 1000.0, 2000.0)
    # the same on a grid that overhangs the mesh (0 outside the mask's box)
    x1, n1 = (-1250.0, -750.0, -9100.0), (38, 36, 22)
    _, mask1 = P.taper_kernel_grid(mesh, np.ones((1,) + n1), x1, h, n1, 1500.0, 2500.0,
                                   500.0, 1500.0)
    with pytest.raises(_lib.SemError, match="taper"):
        P.taper_kernel_grid(mesh, ker, x0, h, n, 6000.0, 4000.0, 1000.0, 2000.0)
    mesh.close()
    ref_out, ref_mask = O.taper_kernel_grid(db, ker.astype(np.float64), x0, h, n,
                                            1000.0, 2000.0, 1000.0, 2000.0)
    assert np.abs(mask - ref_mask).max() <= 1e-12
    assert close(out, ref_out, 1e-6)
    _, ref1 = O.taper_kernel_grid(db, np.ones((1,) + n1), x1, h, n1, 1500.0, 2500.0,
                                  500.0, 1500.0)
    assert np.abs(mask1 - ref1).max() <= 1e-12
    assert mask1[0].max() == 0.0 and 0.0 < mask1.max() <= 1.0


@pytest.mark.parametrize("ptype", [2, 3])
def test_zprecond_matches_oracle(gpu, ptype):
    zg = np.linspace(-30000.0, 2000.0, 17)
    dev = P.zprecond_grid(zg, 4, 3, ptype, 6)
    ref = O.zprecond_grid(zg, 4, 3, ptype, 6)
    assert dev.shape == ref.shape == (4, 3, 17)
    assert np.abs(dev - ref).max() <= 1e-7
    with pytest.raises(ValueError):
        P.zprecond_grid(zg, 2, 2, 1, 1)


def test_gradient_on_grid_chain(gpu):
    """The order of fwat_post_proc: precondition, smooth, project, scale
    rhop from beta, taper (the smoother replaced by a stand-in), against the
    oracle's projection and taper."""
    from specfwat_b200.postproc import RHO_SCALING_FAC, gradient_on_grid
    db = modelled(D.make_box(D.BoxSpec(4, 4, 2, h=2000.0)))
    rng = np.random.default_rng(8)
    k6 = rng.standard_normal((6, db.nspec, 5, 5, 5))
    pre = rng.uniform(0.5, 1.5, (db.nspec, 5, 5, 5))
    x0, h, n = (0.0, 0.0, -4000.0), (500.0, 500.0, 500.0), (17, 17, 9)
    calls = []

    def half(d):                      # stand-in smoother: records and halves
        calls.append(d.shape)
        return 0.5 * d

    mesh = S.Mesh(db)
    g = gradient_on_grid(mesh, db, k6, x0, h, n, 1.0, 1.0, precond=pre, smooth=half)
    assert calls == [(3, db.nspec, 5, 5, 5)]
    for i, k in enumerate((5, 4, 3)):                 # alpha, beta, rhop
        sm = (0.5 * (k6[k] * pre).astype(np.float32)).astype(np.float64)
        ref = O.gll2grid(db, sm, x0, h, n)
        assert np.allclose(g[i], ref, rtol=1e-5, atol=1e-6)
    calls.clear()
    tap = (500.0, 1000.0, 500.0, 1000.0)
    g2 = gradient_on_grid(mesh, db, k6, x0, h, n, 1.0, 1.0, rho_scaling=True, taper=tap,
                          smooth=half)
    mesh.close()
    assert calls == [(2, db.nspec, 5, 5, 5)]
    beta = O.gll2grid(db, (0.5 * k6[4].astype(np.float32)).astype(np.float64), x0, h, n)
    _, mask = O.taper_kernel_grid(db, np.ones((1,) + n), x0, h, n, *tap)
    assert np.allclose(g2[1], beta * mask, rtol=1e-5, atol=1e-6)
    assert np.allclose(g2[2], beta * np.float32(RHO_SCALING_FAC) * mask, rtol=1e-5, atol=1e-6)


def test_argument_errors(gpu):
    db = small_box()
    mesh = S.Mesh(db)
    data = np.zeros((db.nspec, 5, 5, 5), np.float32)
    with pytest.raises(ValueError, match="ngnod"):
        P.gll2grid(mesh, data, (0, 0, 0), (1, 1, 1), (2, 2, 2), ngnod=20)
    with pytest.raises(_lib.SemError):
        P.gll2grid(mesh, data, (0, 0, 0), (0.0, 1, 1), (2, 2, 2))
    with pytest.raises(_lib.SemError):
        P.gll2grid(mesh, data, (0, 0, 0), (1, 1, 1), (0, 2, 2))
    mesh.close()
