"""PDE kernel smoothing on the device against the CPU oracle.

``sem_smooth_pde`` (through ``specfwat_b200.postproc.smooth_sem_pde``) is
compared with ``oracle_smooth_pde`` (FP32 and FP64) on the same fields:
- one, three (one padded pass of 4) and six fields (two passes);
- the cube mapping over the full computed step count;
- the reference's regular branch over a few steps (it diverges later);
- the spherical branch on a box away from the origin;
- CPML elements held at zero.
At the bench's mesh size the size-independent properties are checked: a
constant stays constant and the lumped-volume integral is conserved.
The device result differs from the FP32 oracle only by the order of the
atomic sums; the tolerance is relative L2 1e-5.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from specfwat_b200 import database as D
from specfwat_b200 import solver as S
from specfwat_b200.postproc import smooth_sem_pde

pytestmark = pytest.mark.gpu

WG = np.array([0.1, 49 / 90, 32 / 45, 49 / 90, 0.1])
WK = WG[:, None, None] * WG[None, :, None] * WG[None, None, :]


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def box_db(*args, **kw):
    db = D.make_box(D.BoxSpec(*args, **kw))
    return db.with_model(*D.background_model(db, seed=21))


def fields(db, n, seed=11):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, db.nspec, 5, 5, 5)).astype(np.float32)


@pytest.mark.parametrize("nfield", [1, 3, 6])
def test_cube_mapping_matches_oracle(gpu, nfield):
    db = box_db(5, 4, 3)
    mesh = S.Mesh(db)
    dat = fields(db, nfield)
    out, st = smooth_sem_pde(mesh, dat, 7000.0, 3500.0)
    o32 = Oracle(db, precision=4)
    o64 = Oracle(db, precision=8)
    r32, n, (cv, ch) = o32.smooth_pde(dat, 7000.0, 3500.0, st["distance_min"])
    r64, _, _ = o64.smooth_pde(dat, 7000.0, 3500.0, st["distance_min"])
    assert st["nstep"] == n and st["cv"] == pytest.approx(cv) and st["ch"] == pytest.approx(ch)
    assert st["fields_per_pass"] == (1 if nfield == 1 else 4)
    assert rel(out, r32) < 1e-5, rel(out, r32)
    assert rel(out, r64) < 1e-4, rel(out, r64)
    mesh.close()


def test_reference_branch_and_cpml_match_oracle(gpu):
    db = box_db(4, 4, 3)
    mesh = S.Mesh(db)
    dat = fields(db, 2, seed=2)
    cpml = np.zeros(db.nspec, np.int32)
    cpml[:5] = 1
    out, st = smooth_sem_pde(mesh, dat, 6000.0, 3000.0, mapping="reference",
                             nstep=4, is_cpml=cpml)
    ref, n, _ = Oracle(db, precision=4).smooth_pde(
        dat, 6000.0, 3000.0, st["distance_min"], mapping=1, nstep=4, is_cpml=cpml)
    assert n == st["nstep"] == 4
    assert rel(out, ref) < 1e-5, rel(out, ref)
    g = db.ibool.reshape(db.nspec, -1)
    held = np.unique(g[:5])
    flat = out.reshape(2, -1)
    assert np.all(flat[:, np.isin(g.reshape(-1), held)] == 0.0)
    mesh.close()


def test_spherical_branch_matches_oracle(gpu):
    db = box_db(4, 3, 3, x0=3.0e5, y0=2.0e5)
    mesh = S.Mesh(db)
    dat = fields(db, 1, seed=7)[0]
    out, st = smooth_sem_pde(mesh, dat, 6000.0, 9000.0, is_sph=True)
    ref, n, _ = Oracle(db, precision=4).smooth_pde(
        dat, 6000.0, 9000.0, st["distance_min"], is_sph=True)
    assert n == st["nstep"]
    assert rel(out, ref) < 1e-5, rel(out, ref)
    mesh.close()


def test_medium_mesh_properties(gpu):
    db = D.build("medium")
    mesh = S.Mesh(db)
    dat = fields(db, 4, seed=5)
    dat[3] = 1.75
    one, _ = smooth_sem_pde(mesh, dat, 10000.0, 5000.0, nstep=1)
    out, st = smooth_sem_pde(mesh, dat, 10000.0, 5000.0)
    assert st["nstep"] > 100
    for f in range(3):
        a, b = float((one[f] * WK).sum()), float((out[f] * WK).sum())
        scale = float(np.abs(one[f] * WK).sum())
        assert abs(a - b) < 1e-4 * scale, (f, a, b)
        assert out[f].std() < 0.2 * one[f].std()
    assert np.abs(out[3] - 1.75).max() < 1e-4
    mesh.close()


def test_bad_arguments(gpu):
    db = box_db(2, 2, 2)
    mesh = S.Mesh(db)
    dat = fields(db, 1)[0]
    with pytest.raises(ValueError):
        smooth_sem_pde(mesh, dat, 1.0, 1.0, mapping="other")
    with pytest.raises(Exception, match="origin"):
        smooth_sem_pde(mesh, dat, 6000.0, 3000.0, is_sph=True)   # box corner at 0
    with pytest.raises(Exception, match="sigma"):
        smooth_sem_pde(mesh, dat, -1.0, 3000.0)
    mesh.close()


def test_gradient_on_grid_with_the_device_smoother(gpu):
    """The post-processing chain through the device smoother: each kernel's
    grid equals the oracle-smoothed kernel projected the same way."""
    from oracle.postgrid import gll2grid
    from specfwat_b200.postproc import gradient_on_grid
    db = box_db(5, 4, 3)
    mesh = S.Mesh(db)
    k6 = fields(db, 6, seed=9).astype(np.float64)
    x0, h, n = (0.0, 0.0, -12000.0), (1000.0, 1000.0, 1000.0), (21, 17, 13)
    grid = gradient_on_grid(mesh, db, k6, x0, h, n, 7000.0, 3500.0)
    dmin = (1.0 - np.sqrt(3.0 / 7.0)) / db.xix_regular
    ref, _, _ = Oracle(db, precision=4).smooth_pde(k6[[5, 4, 3]].astype(np.float32),
                                                    7000.0, 3500.0, dmin)
    for i in range(3):
        g_ref = gll2grid(db, ref[i], x0, h, n)
        assert rel(grid[i], g_ref) < 1e-4, i
    mesh.close()


def test_hessian_on_grid(gpu):
    """sum_precond on the device: invert, smooth, project, normalise; and the
    depth forms on the grid."""
    from oracle import oracle as O
    from oracle.postgrid import gll2grid, zprecond_grid
    from specfwat_b200.postproc import hessian_on_grid
    db = box_db(5, 4, 3)
    mesh = S.Mesh(db)
    hs = np.abs(fields(db, 1, seed=12)[0].astype(np.float64)) + 0.1
    x0, h, n = (0.0, 0.0, -12000.0), (1000.0, 1000.0, 1000.0), (21, 17, 13)
    g = hessian_on_grid(mesh, db, hs, x0, h, n, 7000.0, 3500.0, 1)
    inv = O.hessian_precond(hs, 1).astype(np.float32)
    dmin = (1.0 - np.sqrt(3.0 / 7.0)) / db.xix_regular
    ref, _, _ = Oracle(db, precision=4).smooth_pde(inv, 7000.0, 3500.0, dmin)
    gr = gll2grid(db, ref, x0, h, n).astype(np.float64)
    gr /= np.abs(gr).max()
    assert np.abs(g).max() == pytest.approx(1.0)
    assert rel(g, gr) < 1e-4
    z = hessian_on_grid(mesh, db, None, x0, h, n, 0.0, 0.0, 2, nevents=4)
    zref = zprecond_grid(x0[2] + np.arange(n[2]) * h[2], n[0], n[1], 2, 4)
    assert z.shape == zref.shape and np.abs(z - zref).max() <= 1e-7
    mesh.close()


@pytest.mark.parametrize("kind", ["topography", "warp", "mixed"])
def test_irregular_elements_match_oracle(gpu, kind):
    """Irregular elements (per-point mapping terms and Jacobian in the
    fluxes and the lumped volume): a topography mesh and an interior warp
    (every element irregular), and a regular box with half of its elements
    flagged irregular (both branches in one mesh).  The step count comes
    from the mesh's smallest GLL point distance."""
    import dataclasses
    box = D.BoxSpec(5, 4, 3)
    if kind == "topography":
        db = D.make_box(box, topo=D.hill_topography(box, 2000.0, 6000.0))
    elif kind == "warp":
        db = D.make_box(box, warp=D.interior_warp(box, 500.0))
    else:
        db = D.make_box(box)
        full = D.as_irregular(db)
        irr = np.full(db.nspec, -1, np.int32)
        pick = np.arange(1, db.nspec, 2)
        irr[pick] = np.arange(pick.size)
        db = dataclasses.replace(db, irregular=irr, geo=full.geo[pick].copy())
    db = db.with_model(*D.background_model(db, seed=21))
    mesh = S.Mesh(db)
    dat = fields(db, 3, seed=17)
    out, st = smooth_sem_pde(mesh, dat, 7000.0, 3500.0)
    mesh.close()
    r32, n, _ = Oracle(db, precision=4).smooth_pde(dat, 7000.0, 3500.0, st["distance_min"])
    r64, _, _ = Oracle(db, precision=8).smooth_pde(dat, 7000.0, 3500.0, st["distance_min"])
    assert st["nstep"] == n
    if kind == "mixed":
        assert st["distance_min"] == pytest.approx((1 - np.sqrt(3 / 7)) * 2000.0, rel=1e-6)
    assert rel(out, r32) < 1e-5, rel(out, r32)
    assert rel(out, r64) < 1e-4, rel(out, r64)
