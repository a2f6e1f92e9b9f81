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


def test_optional_record_groups(tmp_path):
    """Ocean load, C-PML, element face lists, MPI interfaces and anisotropy
    records, each read under the reference's switch; the solver's
    conversion refuses the C-PML and anisotropic slices."""
    _, dbs = box_dbs()
    db = dbs["regular"]
    ne = db.nspec * 125
    rng = np.random.default_rng(1)
    ocean = rng.random(db.nglob).astype(np.float32)
    ncp = 5
    cpml = {"NSPEC_CPML": ncp, "CPML_width_x": 4000.0, "CPML_width_y": 4000.0,
            "CPML_width_z": 2000.0, "min_distance_between_CPML_parameter": 100.0,
            "CPML_regions": np.arange(1, ncp + 1), "CPML_to_spec": np.arange(ncp),
            "is_CPML": np.arange(db.nspec) < ncp,
            "points_interface_PML_elastic": np.arange(7)}
    for k in ("d_store_x", "d_store_y", "d_store_z", "k_store_x", "k_store_y", "k_store_z",
              "alpha_store_x", "alpha_store_y", "alpha_store_z"):
        cpml[k] = rng.random(ncp * 125).astype(np.float32)
    interfaces = ([1, 2], [3, 2], np.array([[0, 1, 2], [5, 6, 0]]))
    aniso = {k: rng.random(ne).astype(np.float32) for k in
             ("c11", "c12", "c13", "c14", "c15", "c16", "c22", "c23", "c24", "c25", "c26",
              "c33", "c34", "c35", "c36", "c44", "c45", "c46", "c55", "c56", "c66")}
    ibelm = {"ibelm_xmin": [0, 3], "ibelm_top": [7, 8, 9]}
    path = tmp_path / "m.bin"
    write_external_mesh(path, db, ocean_load=ocean, cpml=cpml, interfaces=interfaces,
                        anisotropy=aniso, ibelm=ibelm)
    rec = read_external_mesh(path, ocean_load=True, pml=True, anisotropy=True)
    assert np.array_equal(rec["rmass_ocean_load"], ocean)
    assert rec["NSPEC_CPML"] == ncp and rec["CPML_width_z"] == 2000.0
    assert np.array_equal(rec["CPML_to_spec"], np.arange(1, ncp + 1))
    assert np.array_equal(rec["is_CPML"], cpml["is_CPML"])
    assert np.array_equal(rec["alpha_store_y"], cpml["alpha_store_y"])
    assert np.array_equal(rec["points_interface_PML_elastic"], np.arange(1, 8))
    assert "rmassx" not in rec                       # no Stacey mass under C-PML
    assert rec["nspec2D_xmin"] == 2 and rec["NSPEC2D_TOP"] == 3
    assert np.array_equal(rec["ibelm_top"], [8, 9, 10]) and "ibelm_ymin" not in rec
    assert rec["num_interfaces_ext_mesh"] == 2 and rec["max_nibool_interfaces_ext_mesh"] == 3
    assert np.array_equal(rec["ibool_interfaces_ext_mesh"], [1, 2, 3, 6, 7, 1])
    assert np.array_equal(rec["c46store"], aniso["c46"])
    assert rec["num_phase_ispec_elastic"] == db.nspec
    with pytest.raises(ValueError, match="C-PML"):
        to_database(rec)
    # the same file read with a switch off stops at a check word
    for kw in ({"ocean_load": False, "pml": True, "anisotropy": True},
               {"ocean_load": True, "pml": False, "anisotropy": True}):
        with pytest.raises(ValueError):
            read_external_mesh(path, **kw)
    # past the last check word: the record sizes catch the ANISOTROPY switch
    with pytest.raises(ValueError, match="ANISOTROPY"):
        read_external_mesh(path, ocean_load=True, pml=True, anisotropy=False)
    plain = tmp_path / "plain.bin"
    write_external_mesh(plain, db)
    with pytest.raises(ValueError, match="ANISOTROPY"):
        read_external_mesh(plain, anisotropy=True)
