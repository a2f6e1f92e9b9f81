"""Parity of the CUDA solver (through the C ABI) with the CPU oracle.

Tolerances: seismograms within relative L2 1e-4 of the FP32 oracle run,
event kernels within relative L2 1e-3; errors against the FP64 oracle run
are asserted at the same bounds.  Runs need a B200.
"""
import numpy as np
import pytest

from specfwat_b200 import database as D
from specfwat_b200 import solver as S
from oracle.oracle import Oracle, l2_adjoint_source

pytestmark = pytest.mark.gpu

SEIS_TOL = 1e-4
KERN_TOL = 1e-3


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def small():
    db = D.build("small")
    rec = D.surface_receivers(db.box, 5)
    mt = D.random_moment_tensor(np.random.default_rng(1234))
    return db, rec, mt


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 13])
def test_forward_plain_matches_oracle(gpu, small, variant):
    db, rec, mt = small
    nstep, dt = 400, 0.02
    mesh = S.Mesh(db)
    sim = S.Simulation(mesh, nstep, dt, nev=1, max_receivers=len(rec),
                       kernel_variant=variant)
    sim.set_sources([S.make_source(20000., 20000., -10000., mt, 1.0)])
    sim.set_receivers(rec)
    sim.iterate_time(1)
    g = sim.seismograms(0)
    src = Oracle.source(20000., 20000., -10000., mt, 1.0)
    o32 = Oracle(db, precision=4).forward(dt, nstep, src, rec)
    o64 = Oracle(db, precision=8).forward(dt, nstep, src, rec)
    assert np.abs(g).max() > 1e-4
    assert rel_l2(g, o32) < SEIS_TOL
    assert rel_l2(g, o64) < SEIS_TOL


def test_forward_one_based_indices(gpu, small):
    db, rec, mt = small
    nstep, dt = 100, 0.02
    out = []
    for base in (0, 1):
        mesh = S.Mesh(db, index_base=base)
        sim = S.Simulation(mesh, nstep, dt, max_receivers=len(rec))
        sim.set_sources([S.make_source(20000., 20000., -10000., mt, 1.0)])
        sim.set_receivers(rec)
        sim.iterate_time(1)
        out.append(sim.seismograms(0))
        sim.close()
        mesh.close()
    assert rel_l2(out[1], out[0]) < 1e-5


@pytest.fixture(scope="module")
def mini_adjoint():
    """Forward on the background model, 'observed' data on the model with
    a vs anomaly (oracle FP64), L2 adjoint sources, kernels."""
    box = D.BoxSpec(8, 8, 6)
    db = D.make_box(box)
    vp, vs, rho = D.background_model(db, seed=7)
    db = db.with_model(vp, vs, rho)
    vs_obs = D.gaussian_vs_anomaly(db, vs, radius=6000.0, depth=12000.0)
    db_obs = db.with_model(vp, vs_obs, rho)
    rec = D.surface_receivers(box, 4)
    mt = D.random_moment_tensor(np.random.default_rng(5))
    src_xyz = (16000., 16000., -14000.)
    nstep, dt = 500, 0.02
    src = Oracle.source(*src_xyz, mt, 1.0)
    obs = Oracle(db_obs, precision=8).forward(dt, nstep, src, rec)
    return db, rec, mt, src_xyz, nstep, dt, obs


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 13])
def test_adjoint_kernels_match_oracle(gpu, mini_adjoint, variant):
    db, rec, mt, sxyz, nstep, dt, obs = mini_adjoint
    mesh = S.Mesh(db)
    sim = S.Simulation(mesh, nstep, dt, max_receivers=len(rec),
                       kernel_variant=variant)
    sim.set_sources([S.make_source(*sxyz, mt, 1.0)])
    sim.set_receivers(rec)
    sim.iterate_time(1, save_forward=True)
    syn = sim.seismograms(0)
    misfit = sim.measure_l2(0, obs, 0.05, 1)
    sim.iterate_time(3)
    kg = sim.save_adjoint_kernels(0)

    src = Oracle.source(*sxyz, mt, 1.0)
    res = {}
    for prec in (4, 8):
        o = Oracle(db, precision=prec)
        osyn = o.forward(dt, nstep, src, rec, save_forward=True)
        om, oadj = l2_adjoint_source(osyn, obs, dt, 0.05, 1)
        res[prec] = (osyn, om.sum(), o.adjoint(rec, oadj))
    assert rel_l2(syn, res[4][0]) < SEIS_TOL
    assert abs(misfit - res[8][1]) / res[8][1] < 1e-3
    for q, name in enumerate(S.KERNEL_NAMES[:3]):
        e32 = rel_l2(kg[q], res[4][2][q])
        e64 = rel_l2(kg[q], res[8][2][q])
        assert e32 < KERN_TOL, (name, e32)
        assert e64 < KERN_TOL, (name, e64)


@pytest.mark.parametrize("variant,nev", [(1, 5), (2, 3), (2, 11), (3, 3), (3, 11),
                                         (4, 3), (4, 6), (5, 3), (5, 11), (6, 13),
                                         (11, 5), (11, 19), (11, 7), (12, 5), (12, 19), (13, 3),
                                         (0, 7)])
def test_batched_equals_plain(gpu, small, variant, nev):
    db, rec, _ = small
    nstep, dt = 300, 0.02
    rng = np.random.default_rng(99)
    srcs = [S.make_source(rng.uniform(8e3, 32e3), rng.uniform(8e3, 32e3),
                          -rng.uniform(5e3, 15e3), D.random_moment_tensor(rng),
                          rng.uniform(0.8, 1.5)) for _ in range(nev)]
    mesh = S.Mesh(db)
    b = S.Simulation(mesh, nstep, dt, nev=nev, max_receivers=len(rec),
                     kernel_variant=variant)
    b.set_sources(srcs)
    b.set_receivers(rec)
    b.iterate_time(1)
    plain = []
    for e in range(nev):
        p = S.Simulation(mesh, nstep, dt, nev=1, max_receivers=len(rec),
                         kernel_variant=variant)
        p.set_sources([srcs[e]])
        p.set_receivers(rec)
        p.iterate_time(1)
        plain.append(p.seismograms(0))
        p.close()
    # same arithmetic per lane; only the order of the atomic scatter-adds
    # differs.  Norms are floored at 1% of the largest event so that
    # pre-arrival samples below the FP32 rounding floor do not dominate.
    floor = 0.01 * max(np.linalg.norm(x) for x in plain)
    for e in range(nev):
        d = np.linalg.norm(b.seismograms(e).astype(np.float64) - plain[e])
        assert d / max(np.linalg.norm(plain[e]), floor) < 1e-4, e


def test_graph_equals_stepwise(gpu, small):
    db, rec, mt = small
    nstep, dt = 130, 0.02   # not a multiple of graph_steps
    mesh = S.Mesh(db)
    out = []
    for g in (False, True):
        sim = S.Simulation(mesh, nstep, dt, use_graph=g, graph_steps=50,
                           max_receivers=len(rec))
        sim.set_sources([S.make_source(20000., 20000., -10000., mt, 1.0)])
        sim.set_receivers(rec)
        sim.iterate_time(1)
        out.append(sim.seismograms(0))
        sim.close()
    assert rel_l2(out[1], out[0]) < 1e-5


@pytest.mark.parametrize("nev,variant", [(2, 0), (9, 0), (9, 5), (12, 6), (9, 7), (12, 8),
                                         (9, 9), (12, 10), (9, 11), (16, 11), (12, 12),
                                         (9, 14), (16, 14), (9, 15), (16, 15)])
def test_batched_adjoint_fp16_store(gpu, mini_adjoint, nev, variant):
    db, rec, mt, sxyz, nstep, dt, obs = mini_adjoint
    mesh = S.Mesh(db)
    kern = {}
    for store in ("fp32", "fp16"):
        sim = S.Simulation(mesh, nstep, dt, nev=nev, store=store, use_graph=True,
                           max_receivers=len(rec), kernel_variant=variant)
        sim.set_sources([S.make_source(*sxyz, mt, 1.0)] * nev)
        sim.set_receivers(rec)
        sim.iterate_time(1, save_forward=True)
        for e in range(nev):
            sim.measure_l2(e, obs)
        sim.iterate_time(3)
        kern[store] = sim.sum_kernels()
        k0 = sim.save_adjoint_kernels(0)
        k1 = sim.save_adjoint_kernels(nev - 1)
        assert rel_l2(k0[:3], k1[:3]) < 1e-5
        assert rel_l2(kern[store][:3], nev * k0[:3]) < 1e-5
        sim.close()
    for q in range(3):
        assert rel_l2(kern["fp16"][q], kern["fp32"][q]) < 5e-3


def test_fp64_kernel_sum_over_distinct_events_matches_oracle(gpu):
    """sem_sum_kernels over a batch of distinct events (own source, own
    observed data) against the sum of the FP64 oracle's per-event kernels,
    and against the FP64 sum of the device's own per-event kernels."""
    db = D.build("mini")
    rec = D.surface_receivers(db.box, 3)
    rng = np.random.default_rng(77)
    nev, nstep, dt = 3, 300, 0.02
    box = db.box
    ev = [(rng.uniform(0.3, 0.7) * box.lx, rng.uniform(0.3, 0.7) * box.ly,
           -rng.uniform(0.2, 0.6) * box.lz, D.random_moment_tensor(rng),
           rng.uniform(0.8, 1.3)) for _ in range(nev)]
    obs = [1e-5 * rng.standard_normal((len(rec), 3, nstep)) for _ in range(nev)]
    mesh = S.Mesh(db)
    b = S.Simulation(mesh, nstep, dt, nev=nev, store="fp16", use_graph=True,
                     max_receivers=len(rec), kernel_variant=11)
    b.set_sources([S.make_source(*e) for e in ev])
    b.set_receivers(rec)
    b.iterate_time(1, save_forward=True)
    for e in range(nev):
        b.measure_l2(e, obs[e])
    b.iterate_time(3)
    ksum = b.sum_kernels()
    kev = [b.save_adjoint_kernels(e) for e in range(nev)]
    b.close()
    mesh.close()
    osum = np.zeros_like(ksum)
    for e in range(nev):
        o = Oracle(db, precision=8)
        osyn = o.forward(dt, nstep, Oracle.source(*ev[e]), rec, save_forward=True)
        _, adj = l2_adjoint_source(osyn, obs[e], dt)
        osum += o.adjoint(rec, adj)
    dev_sum = np.sum(kev, axis=0)
    for q in range(6):
        assert rel_l2(ksum[q], osum[q]) < KERN_TOL, (q, rel_l2(ksum[q], osum[q]))
        assert rel_l2(ksum[q], dev_sum[q]) < 1e-12, q
    # distinct events: the sum is not a multiple of any one event's kernel
    c = np.vdot(ksum[1], kev[0][1]) / np.vdot(kev[0][1], kev[0][1])
    assert rel_l2(c * kev[0][1], ksum[1]) > 0.05


def test_state_errors(gpu, small):
    db, rec, mt = small
    mesh = S.Mesh(db)
    sim = S.Simulation(mesh, 10, 0.02, max_receivers=len(rec))
    with pytest.raises(S._lib.SemError) as ei:
        sim.iterate_time(1)
    assert ei.value.code == -4
    sim.set_sources([S.make_source(20000., 20000., -10000., mt, 1.0)])
    sim.set_receivers(rec)
    with pytest.raises(S._lib.SemError) as ei:
        sim.iterate_time(3)
    assert ei.value.code == -4
    with pytest.raises(S._lib.SemError) as ei:
        sim.set_receivers(np.zeros((len(rec) + 1, 3)))
    assert ei.value.code == -1


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15])
def test_batched_adjoint_distinct_events_equal_alone(gpu, variant):
    """Each lane has its own source and observed data: the batched adjoint
    must give every event the kernels it gets alone."""
    db = D.build("mini")
    rec = D.surface_receivers(db.box, 3)
    rng = np.random.default_rng(40 + variant)
    nev, nstep, dt = 5, 260, 0.02
    box = db.box
    srcs = [S.make_source(rng.uniform(0.3, 0.7) * box.lx, rng.uniform(0.3, 0.7) * box.ly,
                          -rng.uniform(0.2, 0.6) * box.lz, D.random_moment_tensor(rng),
                          rng.uniform(0.8, 1.3)) for _ in range(nev)]
    obs = [1e-5 * rng.standard_normal((len(rec), 3, nstep)) for _ in range(nev)]
    mesh = S.Mesh(db)
    b = S.Simulation(mesh, nstep, dt, nev=nev, max_receivers=len(rec),
                     kernel_variant=variant)
    b.set_sources(srcs)
    b.set_receivers(rec)
    b.iterate_time(1, save_forward=True)
    for e in range(nev):
        b.measure_l2(e, obs[e])
    b.iterate_time(3)
    kb = [b.save_adjoint_kernels(e) for e in range(nev)]
    b.close()
    for e in range(nev):
        p = S.Simulation(mesh, nstep, dt, nev=1, max_receivers=len(rec), kernel_variant=2)
        p.set_sources([srcs[e]])
        p.set_receivers(rec)
        p.iterate_time(1, save_forward=True)
        p.measure_l2(0, obs[e])
        p.iterate_time(3)
        kp = p.save_adjoint_kernels(0)
        p.close()
        for q in range(3):
            assert rel_l2(kb[e][q], kp[q]) < 1e-3, (e, q, rel_l2(kb[e][q], kp[q]))
