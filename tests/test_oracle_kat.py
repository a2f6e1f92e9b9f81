"""Known-answer tests that pin the CPU oracle to the physics.

The reference solver (SPECFEM3D, an empty submodule in the reference tree)
cannot be run here, so the oracle is pinned by properties the continuous
and discrete problems must have: energy conservation, exact time
reversibility of the backward reconstruction, the analytic full-space
moment-tensor Green's function, agreement of the adjoint kernels with
finite differences of the misfit, FP32/FP64 agreement, and source-receiver
reciprocity.
"""
import os

import numpy as np
import pytest

from specfwat_b200 import database as D
from oracle.oracle import Oracle, l2_adjoint_source

HERE = os.path.dirname(os.path.abspath(__file__))
NTH = min(8, os.cpu_count() or 1)


def ricker(t, f0):
    a = (np.pi * f0) ** 2
    return (1 - 2 * a * t * t) * np.exp(-a * t * t)


def ricker_dot(t, f0):
    a = (np.pi * f0) ** 2
    return (-6 * a * t + 4 * a * a * t ** 3) * np.exp(-a * t * t)


def cmt_to_xyz(mt):
    Mrr, Mtt, Mpp, Mrt, Mrp, Mtp = mt
    return np.array([[Mpp, -Mtp, Mrp], [-Mtp, Mtt, -Mrt], [Mrp, -Mrt, Mrr]])


def fullspace_mt(M, xs, xr, t, stf, stf_dot, alpha, beta, rho):
    """Displacement of a moment-tensor point source in a homogeneous full
    space (Aki & Richards, 2nd ed., eq. 4.29): near, intermediate and far
    field P and S terms, M(t) = M stf(t)."""
    d = np.asarray(xr, float) - np.asarray(xs, float)
    r = np.linalg.norm(d)
    g = d / r
    dl = np.eye(3)
    u = np.zeros((3, len(t)))
    # near-field integral I(t) = int_{r/a}^{r/b} tau stf(t - tau) dtau
    tau = np.linspace(r / alpha, r / beta, 2001)
    I = np.trapezoid(tau[None, :] * stf(t[:, None] - tau[None, :]), tau, axis=1)
    for n in range(3):
        for p in range(3):
            for q in range(3):
                Mpq = M[p, q]
                if Mpq == 0.0:
                    continue
                gn, gp, gq = g[n], g[p], g[q]
                N = 15 * gn * gp * gq - 3 * gn * dl[p, q] - 3 * gp * dl[n, q] - 3 * gq * dl[n, p]
                IP = 6 * gn * gp * gq - gn * dl[p, q] - gp * dl[n, q] - gq * dl[n, p]
                IS = -(6 * gn * gp * gq - gn * dl[p, q] - gp * dl[n, q] - 2 * gq * dl[n, p])
                FP = gn * gp * gq
                FS = -(gn * gp - dl[n, p]) * gq
                u[n] += Mpq * (N / r ** 4 * I
                               + IP / (alpha ** 2 * r ** 2) * stf(t - r / alpha)
                               + IS / (beta ** 2 * r ** 2) * stf(t - r / beta)
                               + FP / (alpha ** 3 * r) * stf_dot(t - r / alpha)
                               + FS / (beta ** 3 * r) * stf_dot(t - r / beta))
    return u / (4 * np.pi * rho)


@pytest.mark.slow
def test_fullspace_green_function():
    box = D.BoxSpec(16, 16, 16, h=2000.0)
    db = D.homogeneous(D.make_box(box, absorb_top=True))
    xs = (16000.0, 16000.0, -16000.0)
    xr = np.array([[20000.0, 19000.0, -14000.0]])
    mt = D.random_moment_tensor(np.random.default_rng(17), m0=1e16)
    f0, dt, nstep = 0.5, 0.01, 580
    seis = Oracle(db, precision=8, nthreads=NTH).forward(
        dt, nstep, Oracle.source(*xs, mt, f0), xr)[0]
    t = np.arange(nstep) * dt
    t0 = 1.2 / f0
    u = fullspace_mt(cmt_to_xyz(mt), xs, xr[0], t,
                     lambda tt: ricker(tt - t0, f0),
                     lambda tt: ricker_dot(tt - t0, f0), 6000.0, 3464.0, 2700.0)
    err = np.linalg.norm(seis - u) / np.linalg.norm(u)
    assert np.abs(u).max() > 0
    assert err < 0.03, err


def test_energy_conserved_without_absorbing_faces():
    db = D.build("tiny")
    mt = D.random_moment_tensor(np.random.default_rng(1))
    o = Oracle(db, precision=8, nthreads=NTH, stacey=False)
    e = o.forward_energy(0.02, 600, Oracle.source(6000., 6000., -6000., mt, 1.0), 50)
    tail = e[3:]  # after the source has stopped (Ricker ends near 2.4 s)
    assert np.ptp(tail) / tail.mean() < 1e-3


def test_energy_decays_with_stacey():
    db = D.build("small")
    mt = D.random_moment_tensor(np.random.default_rng(1))
    o = Oracle(db, precision=8, nthreads=NTH)
    e = o.forward_energy(0.02, 1000, Oracle.source(20000., 20000., -10000., mt, 1.0), 100)
    assert np.all(np.diff(e[2:]) < 0)
    assert e[-1] < 0.5 * e[2]


@pytest.mark.parametrize("prec,tol", [(8, 1e-11), (4, 1e-4)])
def test_backward_reconstruction_is_time_reversible(prec, tol):
    db = D.build("mini")
    rec = D.surface_receivers(db.box, 3)
    mt = D.random_moment_tensor(np.random.default_rng(2))
    o = Oracle(db, precision=prec, nthreads=NTH)
    syn = o.forward(0.02, 300, Oracle.source(12000., 12000., -8000., mt, 1.0), rec,
                    save_forward=True)
    _, bseis = o.adjoint(rec, np.zeros_like(syn), want_backward_seis=True)
    assert np.linalg.norm(bseis - syn) / np.linalg.norm(syn) < tol


def test_fp32_and_fp64_agree():
    db = D.build("small")
    rec = D.surface_receivers(db.box, 5)
    mt = D.random_moment_tensor(np.random.default_rng(1234))
    src = Oracle.source(20000., 20000., -10000., mt, 1.0)
    s4 = Oracle(db, precision=4, nthreads=NTH).forward(0.02, 500, src, rec)
    s8 = Oracle(db, precision=8, nthreads=NTH).forward(0.02, 500, src, rec)
    assert np.linalg.norm(s4 - s8) / np.linalg.norm(s8) < 1e-5


def test_kernels_match_finite_difference_of_misfit():
    """d chi ~ sum_e,ijk w w w J K_beta dln(vs) for a smooth vs perturbation
    away from the boundaries (FP64, central differences)."""
    box = D.BoxSpec(8, 8, 6)
    db0 = D.make_box(box)
    vp, vs, rho = D.background_model(db0, seed=3)
    db = db0.with_model(vp, vs, rho)
    rec = D.surface_receivers(box, 4)
    mt = D.random_moment_tensor(np.random.default_rng(8))
    src = Oracle.source(16000., 16000., -16000., mt, 1.0)
    dt, nstep = 0.02, 450
    obs = Oracle(db0.with_model(vp, D.gaussian_vs_anomaly(db0, vs, radius=5000.0,
                                                         depth=9000.0), rho),
                 precision=8, nthreads=NTH).forward(dt, nstep, src, rec)
    o = Oracle(db, precision=8, nthreads=NTH)
    syn = o.forward(dt, nstep, src, rec, save_forward=True)
    _, adj = l2_adjoint_source(syn, obs, dt)
    K = o.adjoint(rec, adj)
    x, y, z = D.gll_xyz(db)
    g = np.exp(-((x - 14000) ** 2 + (y - 17000) ** 2 + (z + 11000) ** 2) / 4000.0 ** 2)
    _, w = D.gll_points_weights()
    www = w[:, None, None] * w[None, :, None] * w[None, None, :]
    pred = float((K[4] * g * www[None]).sum() * db.jacobian_regular)
    h = 1e-3

    def chi(sign):
        dbp = db0.with_model(vp, vs * (1 + sign * h * g), rho)
        s = Oracle(dbp, precision=8, nthreads=NTH).forward(dt, nstep, src, rec)
        return l2_adjoint_source(s, obs, dt)[0].sum()

    fd = (chi(+1) - chi(-1)) / (2 * h)
    assert abs(pred) > 0
    assert abs(fd - pred) / abs(fd) < 0.02, (fd, pred)


def test_golden_forward_regression():
    gold = np.load(os.path.join(HERE, "golden", "oracle_small_fwd.npz"))
    box = D.BoxSpec(4, 4, 3)
    db = D.make_box(box)
    vp, vs, rho = D.background_model(db, seed=11)
    db = db.with_model(vp, vs, rho)
    seis = Oracle(db, precision=8, nthreads=1).forward(
        0.02, 200, Oracle.source(8000.0, 8000.0, -6000.0, gold["mt"], 1.0), gold["rec"])
    assert np.allclose(seis, gold["seis"], rtol=1e-12, atol=1e-20)


@pytest.mark.parametrize("topo", [False, True])
def test_source_receiver_reciprocity(topo):
    """A point force in direction i at x_a recorded in direction j at x_b
    equals a force in j at x_b recorded in i at x_a.  The adjoint run
    injects the force (an adjoint source at a receiver, with the same
    Lagrange weights that record it), and the discrete operator is
    symmetric: diagonal mass with the Stacey term folded in, symmetric
    stiffness (regular and general mapping alike) and symmetric Stacey
    damping.  So the two traces agree to round-off in FP64."""
    box = D.BoxSpec(5, 5, 4)
    db = D.make_box(box, topo=D.hill_topography(box, 2000.0, 6000.0) if topo else None)
    db = db.with_model(*D.background_model(db, seed=21))
    rec = np.array([[6300.0, 7100.0, -5200.0], [13700.0, 12900.0, -9800.0]])
    n, dt = 300, 0.02
    g = np.exp(-((np.arange(n) * dt - 1.5) / 0.4) ** 2)
    mt = D.random_moment_tensor(np.random.default_rng(2))

    def force_run(r, c):
        o = Oracle(db, precision=8, nthreads=NTH)
        o.forward(dt, n, Oracle.source(9000., 11000., -7000., mt, 1.0), rec, save_forward=True)
        adj = np.zeros((2, 3, n))
        adj[r, c] = g[::-1]              # injected in adjoint time order
        _, aseis = o.adjoint(rec, adj, want_adjoint_seis=True)
        return aseis

    at_a = [force_run(0, i) for i in range(3)]
    at_b = [force_run(1, j) for j in range(3)]
    for i in range(3):
        for j in range(3):
            ab, ba = at_a[i][1, j], at_b[j][0, i]
            assert np.abs(ab).max() > 0
            assert np.abs(ab - ba).max() <= 1e-12 * np.abs(ab).max(), (i, j)
