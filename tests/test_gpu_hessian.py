"""Approximate Hessian kernel and preconditioners on the device.

- ``hess_kernel`` (``sem_set_approximate_hessian`` + ``sem_save_hessian_kernel``)
  against the FP32 and FP64 oracle, one event and a batch of three distinct
  events, within relative L2 1e-3 (the kernels' tolerance);
- ``sem_sum_hessian`` (sum of |hess| or of hess) against the per-event
  kernels summed on the host;
- the other kernels unchanged by the extra accumulator (within the 1e-5
  that two runs with their own autotuning and atomic order reach);
- linearity in the adjoint source at the bench mesh size;
- ``sem_hessian_precond`` (PRECOND_TYPE 0 and 1) and ``sem_depth_precond``
  (2 and 3) against ``oracle.oracle`` within 1e-6 (FP32 output of FP64
  arithmetic);
- a Hessian read without the switch on is refused.
"""
import numpy as np
import pytest

from oracle import oracle as O
from oracle.oracle import Oracle, l2_adjoint_source
from specfwat_b200 import _lib
from specfwat_b200 import database as D
from specfwat_b200 import solver as S
from specfwat_b200.postproc import apply_precond, depth_precond, hessian_precond

pytestmark = pytest.mark.gpu

KERN_TOL = 1e-3
NSTEP, DT = 400, 0.02


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def box_case():
    box = D.BoxSpec(6, 6, 5)
    db = D.make_box(box)
    db = db.with_model(*D.background_model(db, seed=8))
    vp, vs, rho = D.background_model(db, seed=8)
    db_obs = db.with_model(vp, D.gaussian_vs_anomaly(db, vs, radius=5000.0, depth=9000.0), rho)
    rec = D.surface_receivers(box, 3)
    rng = np.random.default_rng(4)
    srcs = [(rng.uniform(7e3, 17e3), rng.uniform(7e3, 17e3), -rng.uniform(5e3, 12e3),
             D.random_moment_tensor(rng), rng.uniform(0.8, 1.2)) for _ in range(3)]
    obs = [Oracle(db_obs, precision=8).forward(DT, NSTEP, Oracle.source(*s), rec) for s in srcs]
    return db, rec, srcs, obs


def device_run(db, rec, srcs, obs, hess=True):
    mesh = S.Mesh(db)
    sim = S.Simulation(mesh, NSTEP, DT, nev=len(srcs), max_receivers=len(rec))
    sim.set_sources([S.make_source(*s) for s in srcs])
    sim.set_receivers(rec)
    sim.iterate_time(1, save_forward=True)
    for e in range(len(srcs)):
        sim.measure_l2(e, obs[e], 0.05, 1)
    if hess:
        sim.set_approximate_hessian(True)
    sim.iterate_time(3)
    return mesh, sim


def oracle_hessians(db, rec, s, obs, prec):
    o = Oracle(db, precision=prec)
    syn = o.forward(DT, NSTEP, Oracle.source(*s), rec, save_forward=True)
    _, adj = l2_adjoint_source(syn, obs, DT, 0.05, 1)
    o.adjoint(rec, adj)
    return o.hessian()


@pytest.mark.parametrize("nev", [1, 3])
def test_hessian_kernel_matches_oracle(gpu, box_case, nev):
    db, rec, srcs, obs = box_case
    mesh, sim = device_run(db, rec, srcs[:nev], obs[:nev])
    hs = [sim.hessian_kernel(e) for e in range(nev)]
    for e in range(nev):
        h64 = oracle_hessians(db, rec, srcs[e], obs[e], 8)
        h32 = oracle_hessians(db, rec, srcs[e], obs[e], 4)
        assert np.abs(h64).max() > 0
        assert rel(hs[e], h64) < KERN_TOL, e
        assert rel(hs[e], h32) < KERN_TOL, e
    sa = sim.sum_hessian(abs_each=True)
    sp = sim.sum_hessian(abs_each=False)
    assert np.allclose(sa, np.abs(np.array(hs)).sum(0), rtol=1e-12, atol=0)
    assert np.allclose(sp, np.array(hs).sum(0), rtol=1e-12, atol=1e-30)
    k_on = sim.sum_kernels()
    sim.close()
    mesh.close()
    mesh, sim = device_run(db, rec, srcs[:nev], obs[:nev], hess=False)
    with pytest.raises(_lib.SemError, match="Hessian"):
        sim.hessian_kernel(0)
    k_off = sim.sum_kernels()
    for q in range(6):
        assert rel(k_on[q], k_off[q]) < 1e-5, q
    sim.close()
    mesh.close()


def test_hessian_linear_in_adjoint_source_medium_mesh(gpu):
    """Size-independent check at the bench's mesh: doubling the adjoint
    sources doubles hess (the backward field does not see them)."""
    db = D.build("medium")
    rec = D.surface_receivers(db.box, 10)
    box = db.box
    src = S.make_source(0.5 * box.lx, 0.4 * box.ly, -0.3 * box.lz,
                        D.random_moment_tensor(np.random.default_rng(3)), 1.0)
    nstep = 300
    mesh = S.Mesh(db)
    out = []
    for scale in (1.0, 2.0):
        sim = S.Simulation(mesh, nstep, DT, nev=2, max_receivers=len(rec))
        sim.set_sources([src, src])
        sim.set_receivers(rec)
        sim.iterate_time(1, save_forward=True)
        syn = sim.seismograms(0).astype(np.float64)
        for e in range(2):
            sim.set_adjoint_sources(e, scale * syn)
        sim.set_approximate_hessian(True)
        sim.iterate_time(3)
        out.append(sim.hessian_kernel(1))
        sim.close()
    mesh.close()
    assert np.abs(out[0]).max() > 0
    assert rel(out[1], 2.0 * out[0]) < 1e-5


@pytest.mark.parametrize("ptype", [0, 1])
def test_hessian_precond_matches_oracle(gpu, ptype):
    rng = np.random.default_rng(5 + ptype)
    h = rng.standard_normal((40, 5, 5, 5)) * np.exp(rng.uniform(-12, 0, (40, 5, 5, 5)))
    h[3] = 0.0
    if ptype == 1:
        h = np.abs(h)
    dev = hessian_precond(h, ptype)
    ref = O.hessian_precond(h, ptype)
    assert dev.dtype == np.float32 and dev.shape == h.shape
    assert np.abs(dev - ref).max() <= 1e-6 * np.abs(ref).max()
    assert np.all(hessian_precond(np.zeros(50), 1) == 1.0)
    kern = rng.standard_normal((6, 40, 5, 5, 5))
    assert np.allclose(apply_precond(kern, dev), kern * dev.astype(np.float64))


@pytest.mark.parametrize("ptype", [2, 3])
def test_depth_precond_matches_oracle(gpu, ptype):
    box = D.BoxSpec(5, 4, 4)
    db = D.homogeneous(D.make_box(box))
    mesh = S.Mesh(db)
    zlev = np.linspace(-box.lz, 0.0, 9)
    dev = depth_precond(mesh, zlev, ptype, 5)
    ref = O.depth_precond(db, zlev, ptype, 5)
    assert np.abs(dev - ref).max() <= 1e-6 * np.abs(ref).max()
    with pytest.raises(_lib.SemError, match="ascending"):
        depth_precond(mesh, zlev[::-1], ptype, 5)
    with pytest.raises(_lib.SemError, match="depth forms"):
        depth_precond(mesh, zlev, 1, 5)
    mesh.close()


def test_hessian_enabled_after_a_captured_adjoint_graph(gpu, box_case):
    """The adjoint step graph is captured by a first adjoint run without the
    Hessian; switching it on must take effect in the next adjoint run."""
    db, rec, srcs, obs = box_case
    mesh = S.Mesh(db)
    sim = S.Simulation(mesh, NSTEP, DT, nev=1, max_receivers=len(rec), use_graph=True,
                       graph_steps=40)
    sim.set_sources([S.make_source(*srcs[0])])
    sim.set_receivers(rec)
    for hess in (False, True):
        sim.iterate_time(1, save_forward=True)
        sim.measure_l2(0, obs[0], 0.05, 1)
        sim.set_approximate_hessian(hess)
        sim.iterate_time(3)
    h = sim.hessian_kernel(0)
    sim.close()
    mesh.close()
    ref = oracle_hessians(db, rec, srcs[0], obs[0], 8)
    assert rel(h, ref) < KERN_TOL
