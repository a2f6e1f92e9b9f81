"""Invariants of the regular-box database generator."""
import numpy as np
import pytest

from specfwat_b200 import database as D


def test_gll_nodes_weights():
    x, w = D.gll_points_weights()
    s = np.sqrt(3.0 / 7.0)
    assert np.allclose(x, [-1, -s, 0, s, 1], atol=1e-15)
    assert np.allclose(w, [0.1, 49 / 90, 32 / 45, 49 / 90, 0.1], atol=1e-15)
    assert abs(w.sum() - 2.0) < 1e-14


def test_small_box_counts_and_mass():
    db = D.build("small")
    assert db.nspec == 1000 and db.nglob == 41 ** 3
    assert db.nfaces == 5 * 100
    # total mass = integral of rho over the box
    vol_rho = (db.rho.astype(np.float64) * 0 + 1)  # unit weights check below
    total = float(db.rmass.astype(np.float64).sum())
    x, w = D.gll_points_weights()
    www = w[:, None, None] * w[None, :, None] * w[None, None, :]
    expect = float((db.rho.astype(np.float64) * www[None]).sum()
                   * db.jacobian_regular)
    assert abs(total - expect) / expect < 1e-6
    assert vol_rho.shape == db.rho.shape


def test_ibool_covers_every_point_and_shares_faces():
    db = D.make_box(D.BoxSpec(3, 2, 2))
    ib = db.ibool.reshape(-1)
    assert ib.min() == 0 and ib.max() == db.nglob - 1
    assert len(np.unique(ib)) == db.nglob
    # element 0's +x face equals element 1's -x face
    assert np.array_equal(db.ibool[0, :, :, 4], db.ibool[1, :, :, 0])
    # coordinates at GLL points of element 0 span one element
    h = db.box.h
    assert np.isclose(db.xstore[db.ibool[0]].max() - db.xstore[db.ibool[0]].min(), h)


def test_faces_are_on_the_boundary_with_outward_normals():
    db = D.make_box(D.BoxSpec(3, 3, 2))
    for f in range(db.nfaces):
        e = db.abs_ispec[f]
        n = db.abs_normal[f, 0]
        for p in range(25):
            i, j, k = db.abs_ijk[f, p]
            g = db.ibool[e, k, j, i]
            xyz = np.array([db.xstore[g], db.ystore[g], db.zstore[g]])
            lo = np.array([0.0, 0.0, -db.box.lz])
            hi = np.array([db.box.lx, db.box.ly, 0.0])
            ax = int(np.argmax(np.abs(n)))
            assert np.isclose(xyz[ax], hi[ax] if n[ax] > 0 else lo[ax])
    assert not np.any(db.abs_normal[:, :, 2] > 0)  # top is a free surface


def test_random_field_is_seeded_and_normalised():
    box = D.BoxSpec(4, 4, 4)
    g1, _, _ = D.gaussian_random_field(box, 8000.0, seed=5)
    g2, _, _ = D.gaussian_random_field(box, 8000.0, seed=5)
    g3, _, _ = D.gaussian_random_field(box, 8000.0, seed=6)
    assert np.array_equal(g1, g2) and not np.array_equal(g1, g3)
    assert abs(g1.mean()) < 1e-12 and abs(g1.std() - 1.0) < 1e-12


def test_layered_model_interfaces_on_element_boundaries():
    db = D.make_box(D.BoxSpec(2, 2, 12))
    vp, vs, rho = D.layered_model(db, perturb=0.0)
    depth_c = -db.zstore[db.ibool].mean(axis=(1, 2, 3))
    assert np.all(vp[depth_c < 20000] == 5800)
    assert np.all(vp[depth_c > 36000] == 8000)
    assert np.all(np.ptp(vp.reshape(db.nspec, -1), axis=1) == 0)


@pytest.mark.parametrize("name", ["tiny", "small"])
def test_material_consistency(name):
    db = D.build(name)
    mu = db.rho.astype(np.float64) * db.vs.astype(np.float64) ** 2
    assert np.allclose(db.mu, mu, rtol=1e-5)
    assert np.all(db.kappa > 0) and np.all(db.rmass > 0)
