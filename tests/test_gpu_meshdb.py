"""A database read from ``proc*_external_mesh.bin`` runs on the device as
the database it was written from (read_mesh_databases.f90:158-1146 order):
seismograms within 1e-6 and kernels within 1e-5 (two runs, each with its
own autotuning and atomic order), regular and topography meshes."""
import dataclasses

import numpy as np
import pytest

from specfwat_b200 import database as D
from specfwat_b200 import solver as S
from specfwat_b200.meshdb import read_external_mesh, to_database, write_external_mesh

pytestmark = pytest.mark.gpu


def run(db, rec, src):
    mesh = S.Mesh(db)
    sim = S.Simulation(mesh, 300, 0.02, nev=2, max_receivers=len(rec))
    sim.set_sources([src, src])
    sim.set_receivers(rec)
    sim.iterate_time(1, save_forward=True)
    seis = sim.seismograms(1)
    for e in range(2):
        sim.set_adjoint_sources(e, seis.astype(np.float64))
    sim.iterate_time(3)
    k = sim.sum_kernels()
    sim.close()
    mesh.close()
    return seis, k


@pytest.mark.parametrize("topo", [False, True])
def test_read_database_runs_like_the_original(gpu, tmp_path, topo):
    box = D.BoxSpec(6, 5, 4)
    db = D.make_box(box, topo=D.hill_topography(box, 2000.0, 7000.0) if topo else None)
    db = db.with_model(*D.background_model(db, seed=9))
    db = dataclasses.replace(db, xix_regular=float(np.float32(db.xix_regular)),
                             jacobian_regular=float(np.float32(db.jacobian_regular)))
    path = tmp_path / "proc000000_external_mesh.bin"
    write_external_mesh(path, db, dt=0.02)
    back = to_database(read_external_mesh(path))
    rec = D.surface_receivers(box, 3)
    rec[:, 2] = -200.0
    src = S.make_source(11e3, 9e3, -7e3, D.random_moment_tensor(np.random.default_rng(4)), 1.0)
    s0, k0 = run(db, rec, src)
    s1, k1 = run(back, rec, src)
    assert np.abs(s0).max() > 0
    assert np.linalg.norm(s1 - s0) <= 1e-6 * np.linalg.norm(s0)
    for q in range(3):
        assert np.linalg.norm(k1[q] - k0[q]) <= 1e-5 * np.linalg.norm(k0[q]), q
