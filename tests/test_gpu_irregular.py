"""Irregular (deformed) elements on the device against the CPU oracle.

A mesh with topography (every element irregular: per-point mapping
derivatives and Jacobian, read_mesh_databases.f90:168-181) runs the
thread-per-point element kernel (one event) or the register-prefetch
kernels (batches) with the general mapping.  Checked here:
- seismograms within relative L2 1e-4 of the FP32 and FP64 oracle runs;
- event kernels within 1e-3;
- several events batched equal each event alone;
- a regular mesh sent through the general path equals the regular path;
- regular-only kernel variants are refused on such a mesh.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle, l2_adjoint_source
from specfwat_b200 import _lib
from specfwat_b200 import database as D
from specfwat_b200 import solver as S

pytestmark = pytest.mark.gpu

SEIS_TOL = 1e-4
KERN_TOL = 1e-3


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def topo_case():
    box = D.BoxSpec(8, 8, 6)
    topo = D.hill_topography(box, 2500.0, 8000.0)
    db = D.make_box(box, topo=topo)
    vp, vs, rho = D.background_model(db, seed=7)
    db = db.with_model(vp, vs, rho)
    vs_obs = D.gaussian_vs_anomaly(db, vs, radius=6000.0, depth=12000.0)
    db_obs = db.with_model(vp, vs_obs, rho)
    rec = D.surface_receivers(box, 4)
    rec[:, 2] = topo(rec[:, 0], rec[:, 1])
    mt = D.random_moment_tensor(np.random.default_rng(5))
    src_xyz = (16000., 16000., -14000.)
    nstep, dt = 500, 0.02
    obs = Oracle(db_obs, precision=8).forward(dt, nstep, Oracle.source(*src_xyz, mt, 1.0), rec)
    return db, rec, mt, src_xyz, nstep, dt, obs


@pytest.mark.parametrize("variant", [0, 1])
def test_topography_forward_matches_oracle(gpu, topo_case, variant):
    db, rec, mt, sxyz, nstep, dt, _ = topo_case
    assert db.nspec_irregular == db.nspec
    mesh = S.Mesh(db)
    sim = S.Simulation(mesh, nstep, dt, nev=1, max_receivers=len(rec), kernel_variant=variant)
    sim.set_sources([S.make_source(*sxyz, mt, 1.0)])
    sim.set_receivers(rec)
    sim.iterate_time(1)
    g = sim.seismograms(0)
    src = Oracle.source(*sxyz, mt, 1.0)
    o32 = Oracle(db, precision=4).forward(dt, nstep, src, rec)
    o64 = Oracle(db, precision=8).forward(dt, nstep, src, rec)
    assert np.abs(g).max() > 1e-4
    assert rel_l2(g, o32) < SEIS_TOL
    assert rel_l2(g, o64) < SEIS_TOL
    sim.close()
    mesh.close()


@pytest.mark.parametrize("nev", [1, 3])
def test_topography_adjoint_kernels_match_oracle(gpu, topo_case, nev):
    """nev 1: the thread-per-point kernel; nev 3 (the same event in every
    lane): the batched register-prefetch kernels with the general mapping."""
    db, rec, mt, sxyz, nstep, dt, obs = topo_case
    mesh = S.Mesh(db)
    sim = S.Simulation(mesh, nstep, dt, nev=nev, max_receivers=len(rec))
    sim.set_sources([S.make_source(*sxyz, mt, 1.0)] * nev)
    sim.set_receivers(rec)
    sim.iterate_time(1, save_forward=True)
    syn = sim.seismograms(nev - 1)
    for e in range(nev - 1):
        sim.measure_l2(e, obs, 0.05, 1)
    misfit = sim.measure_l2(nev - 1, obs, 0.05, 1)
    sim.iterate_time(3)
    assert sim.kernel_variants() == ((11, 11) if nev > 1 else (1, 1))
    kg = sim.save_adjoint_kernels(nev - 1)
    src = Oracle.source(*sxyz, mt, 1.0)
    res = {}
    for prec in (4, 8):
        o = Oracle(db, precision=prec)
        osyn = o.forward(dt, nstep, src, rec, save_forward=True)
        om, oadj = l2_adjoint_source(osyn, obs, dt, 0.05, 1)
        res[prec] = (osyn, om.sum(), o.adjoint(rec, oadj))
    assert rel_l2(syn, res[4][0]) < SEIS_TOL
    assert abs(misfit - res[8][1]) / res[8][1] < 1e-3
    for q in range(3):
        assert rel_l2(kg[q], res[4][2][q]) < KERN_TOL, q
        assert rel_l2(kg[q], res[8][2][q]) < KERN_TOL, q
    sim.close()
    mesh.close()


def test_topography_batched_equals_alone(gpu, topo_case):
    db, rec, mt, _, nstep, dt, _ = topo_case
    rng = np.random.default_rng(9)
    srcs = [S.make_source(rng.uniform(8e3, 24e3), rng.uniform(8e3, 24e3),
                          -rng.uniform(6e3, 16e3), D.random_moment_tensor(rng), 1.0)
            for _ in range(3)]
    mesh = S.Mesh(db)
    sim = S.Simulation(mesh, 300, dt, nev=3, max_receivers=len(rec))
    sim.set_sources(srcs)
    sim.set_receivers(rec)
    sim.iterate_time(1)
    batch = [sim.seismograms(e) for e in range(3)]
    sim.close()
    for e in range(3):
        one = S.Simulation(mesh, 300, dt, nev=1, max_receivers=len(rec))
        one.set_sources([srcs[e]])
        one.set_receivers(rec)
        one.iterate_time(1)
        assert rel_l2(batch[e], one.seismograms(0)) < 1e-5
        one.close()
    mesh.close()


def test_general_path_on_regular_mesh_equals_regular_path(gpu):
    box = D.BoxSpec(5, 5, 4)
    db = D.make_box(box)
    db = db.with_model(*D.background_model(db, seed=21))
    rec = D.surface_receivers(box, 3)
    mt = D.random_moment_tensor(np.random.default_rng(2))
    out = []
    for d in (db, D.as_irregular(db)):
        mesh = S.Mesh(d)
        sim = S.Simulation(mesh, 200, 0.02, nev=1, max_receivers=len(rec), kernel_variant=1)
        sim.set_sources([S.make_source(9000., 11000., -7000., mt, 1.0)])
        sim.set_receivers(rec)
        sim.iterate_time(1)
        out.append(sim.seismograms(0))
        sim.close()
        mesh.close()
    assert rel_l2(out[1], out[0]) < 1e-5


def test_regular_only_variants_refused(gpu, topo_case):
    db, rec, *_ = topo_case
    mesh = S.Mesh(db)
    with pytest.raises(_lib.SemError, match="regular elements"):
        S.Simulation(mesh, 100, 0.02, nev=8, max_receivers=len(rec), kernel_variant=5)
    mesh.close()
