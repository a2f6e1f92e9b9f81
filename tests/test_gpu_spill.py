"""Boundary store held partly in pinned host memory (sem_set_store_spill).

The spilled store must give the same run as the resident one: every record
that the adjoint run replays is the one the forward run wrote, whether it
stayed in its device slot or went to the host and back.  Two runs differ
only by the order of the element kernels' atomic scatter-adds (about 1e-6
relative between two identical forward runs); a record replayed from the
wrong chunk breaks the backward reconstruction by orders of magnitude
more.  Checked for FP16
and FP32 stores, with and without graphs, a record length that is not a
multiple of the chunk, two and three device slots, on a small box with two
8-lane groups and on the medium mesh with the bench's element kernels.
"""
import numpy as np
import pytest

from specfwat_b200 import database as D
from specfwat_b200 import solver as S

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def _slot_bytes(db, nev, store, chunk=50):
    elem = 2 if store == "fp16" else 4
    b = nev * chunk * db.nfaces * 75 * elem
    return b + (nev * chunk * db.nfaces * 4 if store == "fp16" else 0)


def _run(mesh, db, rec, srcs, obs, nstep, store, graph, spill=0, variant=0):
    nev = len(srcs)
    sim = S.Simulation(mesh, nstep, 0.02, nev=nev, store=store, use_graph=graph,
                       graph_steps=50, max_receivers=len(rec), kernel_variant=variant)
    if spill:
        sim.set_store_spill(spill)
    sim.set_sources(srcs)
    sim.set_receivers(rec)
    sim.iterate_time(1, save_forward=True)
    seis = [sim.seismograms(e) for e in range(nev)]
    for e in range(nev):
        sim.measure_l2(e, obs[e])
    sim.iterate_time(3)
    kern = [sim.save_adjoint_kernels(e) for e in range(nev)]
    info = sim.store_info()
    sim.close()
    return seis, kern, info


def _events(db, nev, seed):
    rng = np.random.default_rng(seed)
    box = db.box
    return [S.make_source(rng.uniform(0.3, 0.7) * box.lx, rng.uniform(0.3, 0.7) * box.ly,
                          -rng.uniform(0.2, 0.5) * box.lz, D.random_moment_tensor(rng),
                          rng.uniform(0.8, 1.2)) for _ in range(nev)]


@pytest.mark.parametrize("store,graph,nstep,slots", [("fp16", True, 430, 2),
                                                     ("fp16", False, 430, 3),
                                                     ("fp32", True, 400, 2)])
def test_spilled_store_equals_resident(gpu, store, graph, nstep, slots):
    db = D.build("mini")
    rec = D.surface_receivers(db.box, 3)
    nev = 9
    srcs = _events(db, nev, 11)
    rng = np.random.default_rng(12)
    obs = [1e-5 * rng.standard_normal((len(rec), 3, nstep)) for _ in range(nev)]
    mesh = S.Mesh(db)
    s0, k0, i0 = _run(mesh, db, rec, srcs, obs, nstep, store, graph)
    assert i0["device_slots"] == 0
    budget = slots * _slot_bytes(db, nev, store) + 4096
    s1, k1, i1 = _run(mesh, db, rec, srcs, obs, nstep, store, graph, spill=budget)
    mesh.close()
    chunks = (nstep + 49) // 50
    assert (i1["chunk_steps"], i1["device_slots"], i1["chunks"]) == (50, slots, chunks)
    assert i1["host_bytes"] == (chunks - slots) * _slot_bytes(db, nev, store)
    for e in range(nev):
        assert rel(s1[e], s0[e]) < 1e-5
        for q in range(6):
            assert rel(k1[e][q], k0[e][q]) < 1e-4, (e, q, rel(k1[e][q], k0[e][q]))


def test_spilled_store_equals_resident_medium(gpu):
    db = D.build("medium")
    rec = D.surface_receivers(db.box, 10)
    nev, nstep = 8, 330
    rng = np.random.default_rng(21)
    box = db.box
    # shallow sources under the receivers: the record holds the arrivals,
    # and the adjoint sources are the synthetics themselves (obs = 0)
    srcs = [S.make_source(rng.uniform(0.3, 0.7) * box.lx, rng.uniform(0.3, 0.7) * box.ly,
                          -rng.uniform(6e3, 12e3), D.random_moment_tensor(rng), 1.0)
            for _ in range(nev)]
    obs = [np.zeros((len(rec), 3, nstep)) for _ in range(nev)]
    mesh = S.Mesh(db)
    s0, k0, _ = _run(mesh, db, rec, srcs, obs, nstep, "fp16", True, variant=11)
    budget = 2 * _slot_bytes(db, nev, "fp16") + 4096
    s1, k1, i1 = _run(mesh, db, rec, srcs, obs, nstep, "fp16", True, spill=budget, variant=11)
    mesh.close()
    assert (i1["device_slots"], i1["chunks"]) == (2, 7)
    for e in (0, 5, 7):
        assert rel(s1[e], s0[e]) < 1e-5
        for q in range(3):
            assert rel(k1[e][q], k0[e][q]) < 1e-4, (e, q, rel(k1[e][q], k0[e][q]))


def test_spill_budget_too_small_is_refused(gpu):
    db = D.build("mini")
    rec = D.surface_receivers(db.box, 3)
    mesh = S.Mesh(db)
    sim = S.Simulation(mesh, 300, 0.02, nev=2, store="fp16", use_graph=True,
                       max_receivers=len(rec))
    sim.set_store_spill(_slot_bytes(db, 2, "fp16"))   # one slot
    sim.set_sources(_events(db, 2, 3))
    sim.set_receivers(rec)
    with pytest.raises(S._lib.SemError) as ei:
        sim.iterate_time(1, save_forward=True)
    assert ei.value.code == -3 and "at least 2" in str(ei.value)
    # a budget that holds the whole store keeps it resident
    sim.set_store_spill(1 << 40)
    sim.iterate_time(1, save_forward=True)
    assert sim.store_info()["device_slots"] == 0
    sim.close()
    mesh.close()


def test_sm_share_keeps_results(gpu):
    """A run whose persistent element kernels are capped to a few SMs and
    whose stream has the highest priority (sem_set_sm_share) computes the
    same seismograms and kernels."""
    db = D.build("mini")
    rec = D.surface_receivers(db.box, 3)
    nev, nstep = 9, 200
    srcs = _events(db, nev, 51)
    rng = np.random.default_rng(52)
    obs = [1e-5 * rng.standard_normal((len(rec), 3, nstep)) for _ in range(nev)]
    mesh = S.Mesh(db)
    s0, k0, _ = _run(mesh, db, rec, srcs, obs, nstep, "fp16", True, variant=11)
    sim = S.Simulation(mesh, nstep, 0.02, nev=nev, store="fp16", use_graph=True,
                       graph_steps=50, max_receivers=len(rec), kernel_variant=11)
    sim.set_sm_share(16, True)
    sim.set_sources(srcs)
    sim.set_receivers(rec)
    sim.iterate_time(1, save_forward=True)
    s1 = [sim.seismograms(e) for e in range(nev)]
    for e in range(nev):
        sim.measure_l2(e, obs[e])
    sim.iterate_time(3)
    k1 = [sim.save_adjoint_kernels(e) for e in range(nev)]
    sim.set_sm_share(0, False)
    sim.close()
    mesh.close()
    for e in range(nev):
        assert rel(s1[e], s0[e]) < 1e-5
        for q in range(3):
            assert rel(k1[e][q], k0[e][q]) < 1e-4
