"""FK injection on the device (``sem_set_injection``).

The Stacey kernel absorbs the velocity relative to the injected incident
field and adds its traction; the boundary store keeps that term for the
backward reconstruction.  Checked against the exact half-space plane wave
(``specfwat_b200.injection``) and the oracle:
- one event, P and SV incidence: receivers within relative L2 1e-3 of the
  exact field and 1e-4 of the FP32 and FP64 oracle;
- a batch mixing injected P (every step), injected SV (every 4th sample,
  cubic interpolation) and a point source, with CUDA graphs and the FP16
  store: every lane equals its own one-event run within 1e-5;
- the adjoint run after an injected forward: kernels within 1e-3 of the
  FP32 and FP64 oracle (the backward field replays the injected boundary
  term);
- a two-layer box driven by the layered field (``LayeredPlaneWave``):
  receivers within 2e-3 of that field and 1e-4 of the FP64 oracle;
- argument errors and an event with neither source nor injection.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle, l2_adjoint_source
from specfwat_b200 import _lib
from specfwat_b200 import database as D
from specfwat_b200 import solver as S
from specfwat_b200.injection import HalfspacePlaneWave, injection_arrays

pytestmark = pytest.mark.gpu

VP, VS, RHO = 6000.0, 3464.0, 2700.0
DT, NSTEP = 0.02, 800
ZERO_MT = np.zeros(6)
SRC_XYZ = (10e3, 10e3, -6e3)


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def case():
    box = D.BoxSpec(10, 10, 6, h=2000.0)
    db = D.homogeneous(D.make_box(box), VP, VS, RHO)
    rec = np.concatenate([D.surface_receivers(box, 4),
                          [[7e3, 9e3, -5e3], [13e3, 11e3, -9e3]]])
    waves = {k: HalfspacePlaneWave(VP, VS, RHO, th, 30.0, k, f0=0.2, t0=5.0,
                                   x0=(10e3, 10e3, -12e3))
             for k, th in (("P", 20.0), ("SV", 15.0))}
    return box, db, rec, waves


def device(db, rec, lanes, use_graph=False, store="fp32", adjoint_obs=None):
    """lanes: list of ("inject", v, t, np, k0) or ("source", src)."""
    mesh = S.Mesh(db)
    sim = S.Simulation(mesh, NSTEP, DT, nev=len(lanes), max_receivers=len(rec),
                       use_graph=use_graph, graph_steps=40, store=store)
    srcs = []
    for e, ln in enumerate(lanes):
        if ln[0] == "inject":
            sim.set_injection(e, *ln[1:])
            srcs.append(S.make_source(*SRC_XYZ, ZERO_MT, 1.0))
        else:
            srcs.append(ln[1])
    sim.set_sources(srcs)
    sim.set_receivers(rec)
    sim.iterate_time(1, save_forward=adjoint_obs is not None)
    seis = [sim.seismograms(e) for e in range(len(lanes))]
    kern = None
    if adjoint_obs is not None:
        for e in range(len(lanes)):
            sim.measure_l2(e, adjoint_obs[e], 0.05, 1)
        sim.iterate_time(3)
        kern = [sim.save_adjoint_kernels(e) for e in range(len(lanes))]
    sim.close()
    mesh.close()
    return seis, kern


def oracle_run(db, rec, v, t, prec, npr=1, k0=0, obs=None):
    o = Oracle(db, precision=prec)
    o.set_injection(v, t, npr, k0)
    syn = o.forward(DT, NSTEP, Oracle.source(*SRC_XYZ, ZERO_MT, 1.0), rec,
                    save_forward=obs is not None)
    if obs is None:
        return syn, None
    _, adj = l2_adjoint_source(syn, obs, DT, 0.05, 1)
    return syn, o.adjoint(rec, adj)


@pytest.mark.parametrize("kind", ["P", "SV"])
def test_device_reproduces_the_plane_wave(gpu, case, kind):
    box, db, rec, waves = case
    w = waves[kind]
    v, t = injection_arrays(db, w, NSTEP, DT)
    (seis,), _ = device(db, rec, [("inject", v, t, 1, 0)])
    ana = np.transpose(w.displacement(rec, np.arange(NSTEP) * DT), (1, 2, 0))
    assert rel(seis, ana) < 1e-3
    for prec in (4, 8):
        o, _ = oracle_run(db, rec, v, t, prec)
        assert rel(seis, o) < 1e-4, prec


def test_batched_lanes_equal_alone(gpu, case):
    box, db, rec, waves = case
    vp_, tp_ = injection_arrays(db, waves["P"], NSTEP, DT)
    vs_, ts_ = injection_arrays(db, waves["SV"], NSTEP // 4 + 10, DT, 4, -4)
    src = S.make_source(8e3, 12e3, -7e3, D.random_moment_tensor(np.random.default_rng(2)), 1.0)
    lanes = [("inject", vp_, tp_, 1, 0), ("source", src), ("inject", vs_, ts_, 4, -4)]
    batch, _ = device(db, rec, lanes, use_graph=True, store="fp16")
    for e, ln in enumerate(lanes):
        (one,), _ = device(db, rec, [ln])
        assert np.abs(one).max() > 0
        assert rel(batch[e], one) < 1e-5, e


def test_adjoint_after_injection_matches_oracle(gpu, case):
    box, db, rec, waves = case
    arrays = [injection_arrays(db, waves[k], NSTEP, DT) for k in ("P", "SV")]
    t = np.arange(NSTEP) * DT
    # "observed": the exact field, 20% weaker
    obs = [0.8 * np.transpose(waves[k].displacement(rec, t), (1, 2, 0)) for k in ("P", "SV")]
    _, kern = device(db, rec, [("inject", v, tr, 1, 0) for v, tr in arrays], adjoint_obs=obs)
    for e, (v, tr) in enumerate(arrays):
        for prec in (4, 8):
            _, ko = oracle_run(db, rec, v, tr, prec, obs=obs[e])
            for q in range(3):
                assert rel(kern[e][q], ko[q]) < 1e-3, (e, prec, q)


def test_injection_errors(gpu, case):
    box, db, rec, waves = case
    mesh = S.Mesh(db)
    sim = S.Simulation(mesh, NSTEP, DT, nev=2, max_receivers=len(rec))
    v, t = injection_arrays(db, waves["P"], 10, DT)
    with pytest.raises(_lib.SemError):
        sim.set_injection(0, v, t, 0, 0)          # np_resamp < 1
    bad = v.copy()
    bad[3, 5, 1] = np.nan
    with pytest.raises(_lib.SemError, match="non-finite"):
        sim.set_injection(0, bad, t)
    sim.set_injection(0, v, t)
    sim.set_receivers(rec)
    with pytest.raises(_lib.SemError, match="no source, injection"):
        sim.iterate_time(1)                       # event 1 has neither
    sim.close()
    mesh.close()


def test_layered_box_reproduces_the_layered_field(gpu):
    from specfwat_b200.injection import LayeredPlaneWave
    layers = ([4500.0, VP], [2600.0, VS], [2400.0, RHO], [4000.0])
    box = D.BoxSpec(10, 10, 6, h=2000.0)
    db = D.make_box(box)
    zc = db.zstore[db.ibool].reshape(db.nspec, 125).mean(axis=1)
    top = (zc > -4000.0)[:, None, None, None]
    ones = np.ones(db.ibool.shape)
    db = db.with_model(*[np.where(top, q[0], q[1]) * ones for q in layers[:3]])
    rec = np.concatenate([D.surface_receivers(box, 4), [[7e3, 9e3, -2e3], [13e3, 11e3, -9e3]]])
    L = LayeredPlaneWave(*layers, 15.0, 30.0, "SV", f0=0.2, t0=5.0, x0=(10e3, 10e3, -12e3))
    v, t = injection_arrays(db, L, NSTEP, DT)
    (seis,), _ = device(db, rec, [("inject", v, t, 1, 0)])
    ana = np.transpose(L.displacement(rec, np.arange(NSTEP) * DT), (1, 2, 0))
    assert rel(seis, ana) < 2e-3
    o, _ = oracle_run(db, rec, v, t, 8)
    assert rel(seis, o) < 1e-4


def test_injection_set_after_a_captured_forward_graph(gpu, case):
    """A forward step graph captured without an injection is dropped when
    one is set, so the next forward run injects."""
    box, db, rec, waves = case
    w = waves["P"]
    v, t = injection_arrays(db, w, NSTEP, DT)
    mesh = S.Mesh(db)
    sim = S.Simulation(mesh, NSTEP, DT, nev=1, max_receivers=len(rec), use_graph=True,
                       graph_steps=40)
    sim.set_sources([S.make_source(*SRC_XYZ, ZERO_MT, 1.0)])
    sim.set_receivers(rec)
    sim.iterate_time(1)
    assert np.abs(sim.seismograms(0)).max() == 0.0
    sim.set_injection(0, v, t)
    sim.iterate_time(1)
    seis = sim.seismograms(0)
    sim.set_injection(0, None, None)
    sim.iterate_time(1)
    after = sim.seismograms(0)
    sim.close()
    mesh.close()
    ana = np.transpose(w.displacement(rec, np.arange(NSTEP) * DT), (1, 2, 0))
    assert rel(seis, ana) < 1e-3
    assert np.abs(after).max() == 0.0
