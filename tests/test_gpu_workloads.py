"""The standard workloads at their real sizes (B200).

* small box (10x10x10 el, 41^3 points), full NSTEP 2000 forward against the
  FP32 and FP64 oracle;
* medium box (40x40x20 el, 2.1M points): the batched path the bench times
  (8 events, variant 11, FP16 store, graphs) and the plain path, forward +
  adjoint past the first arrivals, against the FP32 and FP64 oracle;
* large box (96x96x48 el, 28.6M points, layered model): 4 events batched
  vs each event alone, FP16 store, and the HBM sizing of 8 events;
* failure detection: a time step far above the stability limit is
  reported as SEM_ERR_NUMERIC by the device non-finite check, the context
  stays usable; the periodic check stops a run (or a serving lane) at the
  check after its field goes non-finite and reports the step.
"""
import os

import numpy as np
import pytest

from specfwat_b200 import database as D
from specfwat_b200 import solver as S
from oracle.oracle import Oracle, l2_adjoint_source

pytestmark = pytest.mark.gpu
NTH = os.cpu_count() or 1


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def test_small_full_record_matches_oracle(gpu):
    db = D.build("small")
    rec = D.surface_receivers(db.box, 5)
    mt = D.random_moment_tensor(np.random.default_rng(1234))
    nstep, dt = 2000, 0.02
    mesh = S.Mesh(db)
    sim = S.Simulation(mesh, nstep, dt, max_receivers=len(rec), use_graph=True)
    sim.set_sources([S.make_source(20000., 20000., -10000., mt, 1.0)])
    sim.set_receivers(rec)
    sim.iterate_time(1)
    g = sim.seismograms(0)
    src = Oracle.source(20000., 20000., -10000., mt, 1.0)
    o32 = Oracle(db, precision=4, nthreads=NTH).forward(dt, nstep, src, rec)
    o64 = Oracle(db, precision=8, nthreads=NTH).forward(dt, nstep, src, rec)
    assert rel(g, o32) < 1e-4
    assert rel(g, o64) < 1e-4


def _medium_events(db, nev, seed):
    """Seeded events as the medium workload draws them, moved under the
    receiver grid and to 8-20 km depth so that P and S cross the receivers
    within the record."""
    rng = np.random.default_rng(seed)
    box = db.box
    out = []
    for _ in range(nev):
        x = rng.uniform(0.3, 0.7) * box.lx
        y = rng.uniform(0.3, 0.7) * box.ly
        z = -rng.uniform(8000.0, 20000.0)
        out.append((x, y, z, D.random_moment_tensor(rng), rng.uniform(0.5, 1.0)))
    return out


def test_medium_batched_path_matches_oracle_past_arrivals(gpu):
    """The bench's own path on the bench's mesh and model: 8 events in one
    batch with the register-prefetch element kernels (variant 11), the FP16
    per-face-scaled boundary store and 50-step CUDA graphs, beside the plain
    one-event path.  600 steps (12 s) so that P and S cross the receivers.
    Observed data comes from the FP64 oracle on the +10% vs anomaly model,
    and each path measures its own L2 adjoint sources from it.  Two distinct
    lanes are compared with the FP32 and the FP64 oracle: seismograms within
    relative L2 1e-4 and the six kernels within 1e-3.  (The FP32 oracle
    flushes subnormals below 1.2e-38 to zero for speed; the FP64 oracle is
    exact IEEE arithmetic.)"""
    db = D.build("medium")
    vp, vs, rho = D.background_model(db, seed=1234)
    db_obs = db.with_model(vp, D.gaussian_vs_anomaly(db, vs), rho)
    rec = D.surface_receivers(db.box, 10)
    nev, nstep, dt = 8, 600, 0.02
    ev = _medium_events(db, nev, 2024)
    checked = (1, 6)
    osrc = [Oracle.source(x, y, z, mt, f0) for (x, y, z, mt, f0) in ev]
    srcs = [S.make_source(x, y, z, mt, f0) for (x, y, z, mt, f0) in ev]

    # observed data: FP64 oracle on the anomaly model for the checked lanes,
    # the device (same model) for the others
    mesh_obs = S.Mesh(db_obs)
    so = S.Simulation(mesh_obs, nstep, dt, nev=nev, use_graph=True, max_receivers=len(rec))
    so.set_sources(srcs)
    so.set_receivers(rec)
    so.iterate_time(1)
    obs = [so.seismograms(e).astype(np.float64) for e in range(nev)]
    so.close()
    mesh_obs.close()
    o_obs = Oracle(db_obs, precision=8, nthreads=NTH)
    for e in checked:
        obs[e] = o_obs.forward(dt, nstep, osrc[e], rec)
    del o_obs

    mesh = S.Mesh(db)
    b = S.Simulation(mesh, nstep, dt, nev=nev, store="fp16", use_graph=True, graph_steps=50,
                     max_receivers=len(rec), kernel_variant=11)
    b.set_sources(srcs)
    b.set_receivers(rec)
    b.iterate_time(1, save_forward=True)
    for e in range(nev):
        b.measure_l2(e, obs[e])
    b.iterate_time(3)
    got = {("batched", e): (b.seismograms(e), b.save_adjoint_kernels(e)) for e in checked}
    b.close()
    for e in checked:
        p = S.Simulation(mesh, nstep, dt, nev=1, store="fp32", max_receivers=len(rec))
        p.set_sources([srcs[e]])
        p.set_receivers(rec)
        p.iterate_time(1, save_forward=True)
        p.measure_l2(0, obs[e])
        p.iterate_time(3)
        got[("plain", e)] = (p.seismograms(0), p.save_adjoint_kernels(0))
        p.close()
    mesh.close()

    report = []
    for e in checked:
        for prec in (4, 8):
            o = Oracle(db, precision=prec, nthreads=NTH, flush_subnormals=prec == 4)
            osyn = o.forward(dt, nstep, osrc[e], rec, save_forward=True)
            _, adj = l2_adjoint_source(osyn, obs[e], dt)
            ok = o.adjoint(rec, adj)
            del o
            # the record holds the arrivals: most of its energy is past
            # the first 150 samples
            assert np.linalg.norm(osyn[..., 150:]) > 0.5 * np.linalg.norm(osyn)
            for path in ("batched", "plain"):
                syn, kg = got[(path, e)]
                es = rel(syn, osyn)
                ek = max(rel(kg[q], ok[q]) for q in range(6))
                report.append(f"lane {e} {path} vs FP{8 * prec}: seismograms {es:.2e}, "
                              f"kernels {ek:.2e}")
                assert es < 1e-4, report[-1]
                assert ek < 1e-3, report[-1]
    print("\n".join(report))


def test_large_mesh_batched_equals_alone_and_fits(gpu):
    db = D.build("large")
    assert db.nglob == 385 * 385 * 193
    rec = D.surface_receivers(db.box, 10)
    rng = np.random.default_rng(3)
    box = db.box
    # shallow, high-frequency sources under the receiver grid so that the
    # record (6 s) holds the direct waves rather than sub-rounding noise
    srcs = [S.make_source(rng.uniform(0.4, 0.6) * box.lx, rng.uniform(0.4, 0.6) * box.ly,
                          -rng.uniform(6e3, 12e3), D.random_moment_tensor(rng),
                          rng.uniform(1.2, 1.5)) for _ in range(4)]
    nstep, dt = 400, 0.015
    mesh = S.Mesh(db)
    # 8 events with NSTEP 6000 and an FP16 store: the run's device bytes
    big = S._lib.RunCfg(8, 6000, dt, S._lib.SEM_STORE_FP16, 1, 50, len(rec), 0, 0)
    need = S._lib.load().sem_run_bytes(mesh.handle, big)
    assert need > 150e9
    b = S.Simulation(mesh, nstep, dt, nev=4, store="fp16", use_graph=True,
                     max_receivers=len(rec))
    b.set_sources(srcs)
    b.set_receivers(rec)
    b.iterate_time(1, save_forward=True)
    for e in range(4):
        b.measure_l2(e, np.zeros((len(rec), 3, nstep)))
    b.iterate_time(3)
    kb = b.save_adjoint_kernels(2)
    sb = b.seismograms(2)
    b.close()
    p = S.Simulation(mesh, nstep, dt, nev=1, store="fp16", max_receivers=len(rec))
    p.set_sources([srcs[2]])
    p.set_receivers(rec)
    p.iterate_time(1, save_forward=True)
    p.measure_l2(0, np.zeros((len(rec), 3, nstep)))
    p.iterate_time(3)
    assert rel(sb, p.seismograms(0)) < 1e-4
    kp = p.save_adjoint_kernels(0)
    for q in range(3):
        assert rel(kb[q], kp[q]) < 1e-3
    p.close()
    mesh.close()


def test_unstable_time_step_is_reported_not_faulted(gpu):
    db = D.build("tiny")
    rec = D.surface_receivers(db.box, 2)
    mt = D.random_moment_tensor(np.random.default_rng(1))
    mesh = S.Mesh(db)
    # dt 40x above the CFL limit: the explicit scheme blows up
    sim = S.Simulation(mesh, 400, 0.8, max_receivers=len(rec), check_every=1)
    sim.set_sources([S.make_source(6000., 6000., -6000., mt, 0.2)])
    sim.set_receivers(rec)
    with pytest.raises(S._lib.SemError) as ei:
        sim.iterate_time(1)
    assert ei.value.code == -6
    sim.close()
    # the context is still usable afterwards
    ok = S.Simulation(mesh, 50, 0.02, max_receivers=len(rec), check_every=1)
    ok.set_sources([S.make_source(6000., 6000., -6000., mt, 1.0)])
    ok.set_receivers(rec)
    ok.iterate_time(1)
    assert np.isfinite(ok.seismograms(0)).all()
    ok.close()
    mesh.close()


def _halt_step(msg):
    import re
    m = re.search(r"at step (-?\d+)", msg)
    assert m, msg
    return int(m.group(1))


@pytest.mark.parametrize("graph", [False, True])
def test_blowup_reported_before_nstep(gpu, graph):
    """check_every scans the wavefield every K steps inside the loop; an
    event that goes non-finite is stopped at that check and reported with
    the step, well before NSTEP."""
    db = D.build("tiny")
    rec = D.surface_receivers(db.box, 2)
    mt = D.random_moment_tensor(np.random.default_rng(1))
    mesh = S.Mesh(db)
    nstep = 2000
    sim = S.Simulation(mesh, nstep, 0.8, max_receivers=len(rec), check_every=20,
                       use_graph=graph, graph_steps=10)
    sim.set_sources([S.make_source(6000., 6000., -6000., mt, 0.2)])
    sim.set_receivers(rec)
    with pytest.raises(S._lib.SemError) as ei:
        sim.iterate_time(1, save_forward=True)
    assert ei.value.code == -6
    at = _halt_step(str(ei.value))
    assert 0 < at < nstep // 4 and at % 20 == 0, at
    # the failed forward cannot feed an adjoint run
    with pytest.raises(S._lib.SemError) as ei:
        sim.iterate_time(3)
    assert ei.value.code == -4
    sim.close()
    mesh.close()


def test_adjoint_overflow_reported_for_its_event_only(gpu):
    """In SIM 3 the adjoint field is scanned too: one event of a batch whose
    adjoint source overflows the field is flagged, the other is not."""
    db = D.build("tiny")
    rec = D.surface_receivers(db.box, 2)
    rng = np.random.default_rng(5)
    mesh = S.Mesh(db)
    nstep = 300
    sim = S.Simulation(mesh, nstep, 0.02, nev=2, max_receivers=len(rec), check_every=50,
                       use_graph=True, graph_steps=25, store="fp16")
    sim.set_sources([S.make_source(6000. + 1000 * e, 6000., -6000., D.random_moment_tensor(rng),
                                   1.0) for e in range(2)])
    sim.set_receivers(rec)
    sim.iterate_time(1, save_forward=True)
    syn = [sim.seismograms(e).astype(np.float64) for e in range(2)]
    sim.set_adjoint_sources(0, syn[0])
    sim.set_adjoint_sources(1, np.full_like(syn[1], 3.0e38))
    with pytest.raises(S._lib.SemError) as ei:
        sim.iterate_time(3)
    msg = str(ei.value)
    assert ei.value.code == -6 and "event 1 (1 of 2 events)" in msg, msg
    assert 0 < _halt_step(msg) < nstep
    sim.close()
    mesh.close()


def test_serving_lane_stopped_by_check_others_complete(gpu):
    """Lane-driven runs check their lanes too: a lane whose adjoint field
    overflows is reported by sem_lane_status and released by
    sem_lane_finish without results, while a lane running beside it
    completes with the kernels it has when run alone."""
    db = D.build("tiny")
    rec = D.surface_receivers(db.box, 2)
    rng = np.random.default_rng(9)
    srcs = [S.make_source(6000. + 1500 * e, 7000., -5000., D.random_moment_tensor(rng), 1.0)
            for e in range(2)]
    nstep = 240
    mesh = S.Mesh(db)
    # the good request alone
    alone = S.Simulation(mesh, nstep, 0.02, nev=8, max_receivers=len(rec), check_every=30,
                         use_graph=True, store="fp16")
    alone.lane_start_forward(0, srcs[0], rec, nstep, save_forward=True)
    while alone.lane_status(0)[1] < nstep:
        alone.advance(40)
    seis0 = np.zeros((len(rec), 3, nstep), np.float32)
    alone.lane_finish(0, seis_out=seis0)
    obs0 = 0.5 * seis0.astype(np.float64)
    alone.lane_start_adjoint(0, obs0)
    while alone.lane_status(0)[1] < nstep:
        alone.advance(40)
    k_alone = np.zeros((6, db.nspec, 5, 5, 5))
    alone.lane_finish(0, kernels_out=k_alone)
    alone.close()

    sim = S.Simulation(mesh, nstep, 0.02, nev=8, max_receivers=len(rec), check_every=30,
                       use_graph=True, store="fp16")
    for lane in range(2):
        sim.lane_start_forward(lane, srcs[lane], rec, nstep, save_forward=True)
    while sim.lane_status(0)[1] < nstep:
        sim.advance(40)
    for lane in range(2):
        seis = np.zeros((len(rec), 3, nstep), np.float32)
        sim.lane_finish(lane, seis_out=seis)
    sim.lane_start_adjoint(0, obs0)
    sim.lane_start_adjoint(1, np.full((len(rec), 3, nstep), 3.0e38))
    done = {}
    for _ in range(100):
        sim.advance(40)
        for lane in range(2):
            if lane in done:
                continue
            ph, st, ns = sim.lane_status(lane)
            if st >= ns:
                done[lane] = sim.lane_errors.get(lane, "")
        if len(done) == 2:
            break
    assert "non-finite" in done[1], done
    assert done[0] == "", done
    with pytest.raises(S._lib.SemError) as ei:
        sim.lane_finish(1)
    assert ei.value.code == -6
    k = np.zeros((6, db.nspec, 5, 5, 5))
    sim.lane_finish(0, kernels_out=k)
    for q in range(3):
        assert rel(k[q], k_alone[q]) < 1e-5
    # the released lane takes the next request
    sim.lane_start_forward(1, srcs[1], rec, 60, save_forward=False)
    while sim.lane_status(1)[1] < 60:
        sim.advance(30)
    seis = np.zeros((len(rec), 3, 60), np.float32)
    sim.lane_finish(1, seis_out=seis)
    assert np.isfinite(seis).all() and np.abs(seis).max() > 0
    sim.close()
    mesh.close()


def test_fp32_fma_peak_probe(gpu):
    """The FP32 roofline denominator: B200 has 148 SMs x 128 FP32 lanes, so
    the probe must land below 2 x 148 x 128 x 2.1 GHz (80 TFLOP/s) and well
    above a tenth of it."""
    import ctypes as C
    from specfwat_b200 import _lib
    t, ms = C.c_double(0.0), C.c_double(0.0)
    _lib.check(_lib.load().sem_fp32_fma_peak(C.byref(t), C.byref(ms)))
    assert 8.0 < t.value < 80.0, t.value
    assert ms.value > 0.0
