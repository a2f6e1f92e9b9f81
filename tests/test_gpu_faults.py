"""Faults injected on the host come back as status codes, and the device
stays usable after each.

- The mesh upload refuses a corrupt ibool, a non-finite or negative
  material, a zero density and a non-positive mass point (SEM_ERR_ARG).
- A run larger than the device is refused with SEM_ERR_NOMEM when its
  wavefields are allocated, and what was allocated is released.
- Malformed requests are refused before any launch (SEM_ERR_ARG):
  - an event index past the batch;
  - more receivers than the run holds;
  - a serving lane past the run's lanes;
  - a record longer than the run's;
  - a source position that is not finite.

No fault reaches the GPU: a host check catches each one before anything
is launched. After every refusal a valid run on a new mesh steps and
returns finite seismograms.
"""
import ctypes as C
import dataclasses

import numpy as np
import pytest

from specfwat_b200 import _lib
from specfwat_b200 import database as D
from specfwat_b200 import solver as S

pytestmark = pytest.mark.gpu


def box():
    db = D.make_box(D.BoxSpec(4, 4, 3))
    return db.with_model(*D.background_model(db, seed=3))


def still_usable():
    db = box()
    mesh = S.Mesh(db)
    rec = D.surface_receivers(db.box, 2)
    sim = S.Simulation(mesh, 40, 0.02, max_receivers=len(rec))
    mt = D.random_moment_tensor(np.random.default_rng(1))
    sim.set_sources([S.make_source(8000.0, 8000.0, -6000.0, mt, 1.0)])
    sim.set_receivers(rec)
    sim.iterate_time(1)
    s = sim.seismograms(0)
    sim.close()
    mesh.close()
    assert np.all(np.isfinite(s))


def _with(db, name, index, value):
    a = np.array(getattr(db, name), copy=True)
    a.reshape(-1)[index] = value
    return dataclasses.replace(db, **{name: a})


@pytest.mark.parametrize("name,index,value,msg", [
    ("ibool", 77, None, "ibool"),                 # a point index past nglob
    ("ibool", 12, -1, "ibool"),
    ("kappa", 5, np.nan, "material"),
    ("mu", 9, -1.0, "material"),
    ("rho", 300, 0.0, "material"),
    ("rmass", 40, 0.0, "mass"),
    ("rmass", 41, np.inf, "mass"),
])
def test_mesh_faults_are_refused(gpu, name, index, value, msg):
    db = box()
    bad = _with(db, name, index, db.nglob if value is None else value)
    with pytest.raises(_lib.SemError) as ei:
        S.Mesh(bad)
    assert ei.value.code == -1 and msg in str(ei.value), str(ei.value)
    still_usable()


def test_run_larger_than_the_device_is_refused(gpu):
    import torch
    db = D.build("medium")
    mesh = S.Mesh(db)
    nev = 4096       # the run's limit; its three forward fields alone take 309 GB
    cfg = _lib.RunCfg(nev, 4000, 0.02, _lib.SEM_STORE_FP16, 1, 50, 4, 0, 0)
    need = _lib.load().sem_run_bytes(mesh.handle, C.byref(cfg))
    _, total = torch.cuda.mem_get_info()
    assert need > total
    with pytest.raises(_lib.SemError) as ei:
        S.Simulation(mesh, 4000, 0.02, nev=nev, store="fp16", use_graph=True, max_receivers=4)
    assert ei.value.code == -3, str(ei.value)
    mesh.close()
    still_usable()


def test_malformed_requests_are_refused(gpu):
    db = box()
    mesh = S.Mesh(db)
    rec = D.surface_receivers(db.box, 2)
    sim = S.Simulation(mesh, 30, 0.02, nev=2, max_receivers=len(rec))
    mt = D.random_moment_tensor(np.random.default_rng(2))
    src = S.make_source(8000.0, 8000.0, -6000.0, mt, 1.0)
    sim.set_sources([src, src])
    with pytest.raises(_lib.SemError) as ei:
        sim.set_receivers(rec, 2)                         # event past the batch
    assert ei.value.code == -1
    with pytest.raises(_lib.SemError) as ei:
        sim.set_receivers(np.zeros((len(rec) + 1, 3)))     # more than max_receivers
    assert ei.value.code == -1
    sim.set_receivers(rec)
    sim.iterate_time(1)
    out = np.zeros((len(rec), 3, 30), np.float32)
    assert _lib.load().sem_get_seismograms(sim._h, 2, out.ctypes.data) == -1
    assert b"out of range" in _lib.load().sem_last_error()
    sim.close()
    lanes = S.Simulation(mesh, 30, 0.02, nev=8, store="fp16", max_receivers=len(rec))
    nan_src = S.make_source(np.nan, 8000.0, -6000.0, mt, 1.0)
    for lane, s, nstep in ((8, src, 30),                  # lane past the run's lanes
                           (0, src, 31),                  # record past the run's nstep
                           (0, nan_src, 30)):             # source position not finite
        with pytest.raises(_lib.SemError) as ei:
            lanes.lane_start_forward(lane, s, rec, nstep, False)
        assert ei.value.code == -1, (lane, nstep, str(ei.value))
    lanes.close()
    mesh.close()
    still_usable()
