"""Serving: continuous batching gives each request the result it gets alone.

Requests of different kinds (forward-only, forward+adjoint), record lengths
and meshes arrive at different times into fewer lanes than requests, so
lanes are reused while others run; every result is compared with the same
request run alone on the plain one-event path.
"""
import numpy as np
import pytest

from specfwat_b200 import database as D
from specfwat_b200 import solver as S
from specfwat_b200.serving import MeshServer, Request, Server, latency_stats

pytestmark = pytest.mark.gpu

SEIS_TOL = 1e-4
KERN_TOL = 1e-3


def rel(a, b, floor=0.0):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b)
                 / max(np.linalg.norm(b), floor))


def _requests(rng, name, db, n, kinds, nsteps, t0):
    box = db.box
    rec = D.surface_receivers(box, 3)
    out = []
    for k in range(n):
        src = S.make_source(rng.uniform(0.3, 0.7) * box.lx, rng.uniform(0.3, 0.7) * box.ly,
                            -rng.uniform(0.2, 0.5) * box.lz,
                            D.random_moment_tensor(rng), rng.uniform(0.8, 1.2))
        kind = kinds[k % len(kinds)]
        ns = nsteps[k % len(nsteps)]
        obs = None
        if kind == "fwdadj":
            obs = 0.01 * rng.standard_normal((len(rec), 3, ns)) * 1e-4
        out.append(Request(rid=len(out), mesh=name, kind=kind, nstep=ns, source=src,
                           receivers=rec, obs=obs, arrival=t0 + 0.03 * k,
                           want_kernels=kind == "fwdadj"))
    return out


def _alone(db, req, dt):
    mesh = S.Mesh(db)
    sim = S.Simulation(mesh, req.nstep, dt, max_receivers=len(req.receivers))
    sim.set_sources([req.source])
    sim.set_receivers(req.receivers)
    sim.iterate_time(1, save_forward=req.kind == "fwdadj")
    seis = sim.seismograms(0)
    out = dict(seis=seis)
    if req.kind == "fwdadj":
        out["misfit"] = sim.measure_l2(0, req.obs)
        sim.iterate_time(3)
        out["kernels"] = sim.save_adjoint_kernels(0)
    sim.close()
    mesh.close()
    return out


def test_results_same_alone_and_in_the_mix(gpu):
    rng = np.random.default_rng(77)
    dbs = {"small": D.build("small"), "mini": D.build("mini")}
    dt = 0.02
    reqs = (_requests(rng, "small", dbs["small"], 6, ["fwdadj", "fwd"], [300, 420, 240], 0.0)
            + _requests(rng, "mini", dbs["mini"], 5, ["fwd", "fwdadj"], [260, 380], 0.01))
    servers = {name: MeshServer(name, db, slots=3, nstep_max=450, dt=dt, store="fp32",
                                graph_steps=20, max_receivers=16)
               for name, db in dbs.items()}
    done = Server(servers, quantum=40).run(reqs, timeout=600)
    assert len(done) == len(reqs)
    st = latency_stats(done)
    assert st["p99_s"] >= st["p50_s"] > 0
    for r in reqs:
        a = _alone(dbs[r.mesh], r, dt)
        floor = 0.01 * np.linalg.norm(a["seis"]) + 1e-30
        assert rel(r.seismograms, a["seis"], floor) < SEIS_TOL, r.rid
        if r.kind == "fwdadj":
            assert abs(r.misfit - a["misfit"]) <= 1e-4 * abs(a["misfit"]), r.rid
            for q in range(3):
                assert rel(r.kernels[q], a["kernels"][q]) < KERN_TOL, (r.rid, q)
    for srv in servers.values():
        assert srv.store_in_use == 0
        srv.close()


def test_group_policy_same_results(gpu):
    rng = np.random.default_rng(31)
    db = D.build("small")
    dt = 0.02
    reqs = _requests(rng, "small", db, 10, ["fwdadj"], [260], 0.0)
    srv = MeshServer("small", db, slots=16, nstep_max=260, dt=dt, store="fp16",
                     graph_steps=20, max_receivers=16, policy="group", max_wait=0.05)
    done = Server({"small": srv}, quantum=60).run(reqs, timeout=600)
    assert len(done) == len(reqs)
    for r in reqs[:3]:
        a = _alone(db, r, dt)
        floor = 0.01 * np.linalg.norm(a["seis"]) + 1e-30
        assert rel(r.seismograms, a["seis"], floor) < SEIS_TOL
        for q in range(3):
            assert rel(r.kernels[q], a["kernels"][q]) < 5e-3   # FP16 store
    srv.close()


def test_store_budget_limits_admission(gpu):
    rng = np.random.default_rng(5)
    db = D.build("mini")
    srv = MeshServer("mini", db, slots=4, nstep_max=300, dt=0.02, store="fp16",
                     graph_steps=20, max_receivers=16)
    one = srv.sim.lane_store_bytes(300)
    srv.store_budget = int(1.5 * one)      # room for one forward+adjoint store
    reqs = _requests(rng, "mini", db, 3, ["fwdadj"], [300], 0.0)
    for r in reqs:
        srv.queue.append(r)
    assert srv.try_admit(0.0) == 1
    assert srv.store_in_use == one
    done = Server({"mini": srv}, quantum=50).run([], timeout=60)
    assert done == []
    srv.close()


def test_solo_routing_same_results(gpu):
    """A request that finds its mesh's batched server nearly empty and the
    one-lane server free runs on the one-lane server (the plain one-event
    kernels); the rest queue for the batched server.  A burst of five (one
    solo, four batched) and two late arrivals; every result equals the
    request run alone."""
    rng = np.random.default_rng(12)
    db = D.build("mini")
    dt = 0.02
    reqs = _requests(rng, "mini", db, 7, ["fwdadj", "fwd"], [240, 300], 0.0)
    for k, r in enumerate(reqs):
        r.arrival = 0.0 if k < 5 else 0.5   # a burst, then two late ones
    batched = MeshServer("mini", db, slots=8, nstep_max=300, dt=dt, store="fp32",
                         graph_steps=20, max_receivers=16)
    solo = MeshServer("mini", db, slots=1, nstep_max=300, dt=dt, store="fp32",
                      graph_steps=20, max_receivers=16)
    srv = Server({"mini": batched}, quantum=40, solo={"mini": solo}, solo_below=2)
    done = srv.run(reqs, timeout=600)
    assert len(done) == len(reqs)
    for r in reqs:
        a = _alone(db, r, dt)
        floor = 0.01 * np.linalg.norm(a["seis"]) + 1e-30
        assert rel(r.seismograms, a["seis"], floor) < SEIS_TOL, r.rid
        if r.kind == "fwdadj":
            assert abs(r.misfit - a["misfit"]) <= 1e-4 * abs(a["misfit"]), r.rid
            for q in range(3):
                assert rel(r.kernels[q], a["kernels"][q]) < KERN_TOL, (r.rid, q)
    assert {r.server for r in reqs} == {"solo", "batched"}
    assert solo.store_in_use == 0 and batched.store_in_use == 0
    solo.close()
    batched.close()


def test_async_lane_primitives_match_blocking(gpu):
    """The non-blocking lane calls a pipelined scheduler uses give what the
    blocking ones give: sem_lane_finish_async + sem_lane_ready returns the
    same seismograms as sem_lane_finish, sem_lane_misfit the misfit that
    sem_lane_start_adjoint returns, and the kernels summed through the
    asynchronous finish equal the blocking finish's; completion marks
    finish in order with positive device time between them."""
    import torch
    rng = np.random.default_rng(31)
    db = D.build("mini")
    reqs = _requests(rng, "mini", db, 2, ["fwdadj"], [240], 0.0)
    out = {}
    for mode in ("blocking", "async"):
        mesh = S.Mesh(db)
        sim = S.Simulation(mesh, 240, 0.02, nev=8, store="fp16", use_graph=True,
                           max_receivers=len(reqs[0].receivers))
        ksum = torch.zeros((6, db.nspec * 125), dtype=torch.float64, device="cuda")
        for lane, r in enumerate(reqs):
            sim.lane_start_forward(lane, r.source, r.receivers, r.nstep, save_forward=True)
        marks = []
        while sim.lane_status(0)[1] < 240:
            marks.append(sim.mark())
            sim.advance(60)
        marks.append(sim.mark())
        seis, mis = [], []
        for lane, r in enumerate(reqs):
            s = torch.empty(len(r.receivers) * 3 * 240, dtype=torch.float32).pin_memory().numpy()
            if mode == "blocking":
                sim.lane_finish(lane, seis_out=s)
                mis.append(sim.lane_start_adjoint(lane, r.obs))
            else:
                sim.lane_finish_async(lane, seis_out=s)
                sim.lane_start_adjoint(lane, r.obs, want_misfit=False)
                m = torch.empty(1, dtype=torch.float64).pin_memory().numpy()
                sim.lane_misfit(lane, m)
                assert sim.lane_ready(lane, wait=True)
                mis.append(float(m[0]))
            seis.append(s.copy())
        assert sim.mark_done(marks[-1], wait=True)
        assert all(sim.mark_done(t) for t in marks)
        assert sim.mark_elapsed(marks[0], marks[-1]) > 0.0
        while sim.lane_status(0)[1] < 240:
            sim.advance(60)
        for lane in range(len(reqs)):
            if mode == "blocking":
                sim.lane_finish(lane, ksum_dev_ptr=ksum.data_ptr())
            else:
                sim.lane_finish_async(lane, ksum_dev_ptr=ksum.data_ptr())
                assert sim.lane_ready(lane, wait=True)
        torch.cuda.synchronize()
        out[mode] = (seis, mis, ksum.cpu().numpy())
        sim.close()
        mesh.close()
    for a, b in zip(out["blocking"][0], out["async"][0]):
        assert rel(b, a) < 1e-5
    # the two runs differ only by the order of atomic adds (~1e-6)
    for a, b in zip(out["blocking"][1], out["async"][1]):
        assert abs(a - b) <= 1e-5 * abs(a)
    for q in range(3):
        assert rel(out["async"][2][q], out["blocking"][2][q]) < 1e-5


def test_lane_move_keeps_results(gpu):
    """sem_lane_move in the middle of a forward and of an adjoint run: the
    moved request (to a lane of another 8-lane group) ends with the
    seismograms, misfit and kernels it has without the moves."""
    rng = np.random.default_rng(41)
    db = D.build("mini")
    r = _requests(rng, "mini", db, 1, ["fwdadj"], [260], 0.0)[0]
    out = {}
    for moved in (False, True):
        mesh = S.Mesh(db)
        sim = S.Simulation(mesh, 260, 0.02, nev=16, store="fp16", use_graph=True,
                           max_receivers=len(r.receivers))
        lane = 9
        sim.lane_start_forward(lane, r.source, r.receivers, 260, save_forward=True)
        sim.advance(110)
        if moved:
            sim.lane_move(lane, 2)
            lane = 2
        while sim.lane_status(lane)[1] < 260:
            sim.advance(50)
        seis = np.zeros((len(r.receivers), 3, 260), np.float32)
        sim.lane_finish(lane, seis_out=seis)
        mis = sim.lane_start_adjoint(lane, r.obs)
        sim.advance(70)
        if moved:
            sim.lane_move(lane, 15)
            lane = 15
        while sim.lane_status(lane)[1] < 260:
            sim.advance(50)
        kern = np.zeros((6, db.nspec, 5, 5, 5))
        sim.lane_finish(lane, kernels_out=kern)
        out[moved] = (seis, mis, kern)
        sim.close()
        mesh.close()
    assert rel(out[True][0], out[False][0]) < 1e-5
    assert abs(out[True][1] - out[False][1]) <= 1e-5 * abs(out[False][1])
    for q in range(6):
        assert rel(out[True][2][q], out[False][2][q]) < 1e-4, q
