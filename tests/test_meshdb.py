"""``proc*_external_mesh.bin`` reader (read_mesh_databases.f90:158-1146).

The records are read in the reference reader's order; a slice written in
that order (``write_external_mesh``) must come back field for field, for a
regular box and for a topography mesh whose elements are all irregular,
and run the same in the oracle.  Wrong Par_file switches shift the record
sequence and are caught by the reference's check words; broken record
markers are caught too.
"""
import dataclasses
import os

import numpy as np
import pytest

from oracle.oracle import Oracle
from specfwat_b200 import database as D
from specfwat_b200.meshdb import read_external_mesh, to_database, write_external_mesh

NTH = min(8, os.cpu_count() or 1)


def box_dbs():
    box = D.BoxSpec(4, 3, 3)
    reg = D.make_box(box)
    reg = reg.with_model(*D.background_model(reg, seed=5))
    topo = D.make_box(box, topo=D.hill_topography(box, 2000.0, 6000.0))
    topo = topo.with_model(*D.background_model(topo, seed=5))
    return box, {"regular": reg, "topography": topo}


FIELDS = ("ibool", "xstore", "ystore", "zstore", "kappa", "mu", "rho", "rmass", "rho_vp",
          "rho_vs", "abs_ispec", "abs_ijk", "abs_jw", "abs_normal")


@pytest.mark.parametrize("kind", ["regular", "topography"])
def test_round_trip(tmp_path, kind):
    box, dbs = box_dbs()
    db = dbs[kind]
    path = tmp_path / "proc000000_external_mesh.bin"
    write_external_mesh(path, db, dt=0.02)
    rec = read_external_mesh(path)
    assert rec["NSPEC_AB"] == db.nspec and rec["NGLOB_AB"] == db.nglob
    assert rec["nspec_inner_elastic"] == db.nspec and rec["num_phase_ispec_elastic"] == db.nspec
    # rmassx carries M + dt/2 C on the absorbing faces, M elsewhere
    assert np.all(rec["rmassx"] >= rec["rmass"]) and np.any(rec["rmassx"] > rec["rmass"])
    back = to_database(rec)
    for f in FIELDS:
        assert np.array_equal(np.asarray(getattr(back, f)), np.asarray(getattr(db, f))), f
    assert back.xix_regular == pytest.approx(db.xix_regular)
    assert back.nspec_irregular == db.nspec_irregular
    if kind == "topography":
        assert back.nspec_irregular == db.nspec
        assert np.array_equal(back.irregular, db.irregular)
        assert np.array_equal(back.geo, db.geo)
    rec_xyz = D.surface_receivers(box, 2)
    if kind == "topography":
        rec_xyz[:, 2] = -100.0
    mt = D.random_moment_tensor(np.random.default_rng(3))
    src = Oracle.source(7000.0, 6000.0, -5000.0, mt, 1.0)
    # the file holds CUSTOM_REAL (4-byte) scalars
    db32 = dataclasses.replace(db, xix_regular=float(np.float32(db.xix_regular)),
                               jacobian_regular=float(np.float32(db.jacobian_regular)))
    a = Oracle(db32, precision=8, nthreads=NTH).forward(0.02, 150, src, rec_xyz)
    b = Oracle(back, precision=8, nthreads=NTH).forward(0.02, 150, src, rec_xyz)
    assert np.array_equal(a, b)


def test_wrong_switches_and_broken_files(tmp_path):
    _, dbs = box_dbs()
    path = tmp_path / "m.bin"
    write_external_mesh(path, dbs["regular"])
    with pytest.raises(ValueError):
        read_external_mesh(path, ocean_load=True)     # an extra record expected
    with pytest.raises(ValueError):
        read_external_mesh(path, stacey=False)        # rmassx/y/z left unread
    raw = bytearray(path.read_bytes())
    raw[-3] ^= 0xFF                                   # the last record's end marker
    bad = tmp_path / "bad.bin"
    bad.write_bytes(bytes(raw))
    with pytest.raises(ValueError, match="record markers"):
        read_external_mesh(bad)
    short = tmp_path / "short.bin"
    short.write_bytes(path.read_bytes()[:1000])
    with pytest.raises(ValueError):
        read_external_mesh(short)
