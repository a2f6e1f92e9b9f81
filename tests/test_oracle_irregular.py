"""Known-answer tests of the oracle's general (irregular) element path.

Deformed meshes carry per-point mapping derivatives and Jacobians
(xixstore .. jacobianstore, read_mesh_databases.f90:172-181).  The general
path is pinned by:
- the same regular mesh run through the general path (every element
  flagged irregular with its constant mapping) against the regular path;
- energy conservation with free boundaries on a topography mesh;
- exact time reversibility of the backward reconstruction with Stacey
  replay on a topography mesh;
- the analytic full-space moment-tensor Green's function on a mesh whose
  interior is warped (every element irregular).
"""
import os

import numpy as np
import pytest

from oracle.oracle import Oracle
from specfwat_b200 import database as D

from test_oracle_kat import cmt_to_xyz, fullspace_mt, ricker, ricker_dot

NTH = min(8, os.cpu_count() or 1)


@pytest.mark.parametrize("prec,tol", [(8, 2e-6), (4, 2e-6)])
def test_general_path_equals_regular_path(prec, tol):
    box = D.BoxSpec(5, 5, 4)
    db = D.make_box(box)
    db = db.with_model(*D.background_model(db, seed=21))
    rec = D.surface_receivers(box, 3)
    mt = D.random_moment_tensor(np.random.default_rng(2))
    src = Oracle.source(9000., 11000., -7000., mt, 1.0)
    s0 = Oracle(db, precision=prec, nthreads=NTH).forward(0.02, 200, src, rec)
    s1 = Oracle(D.as_irregular(db), precision=prec, nthreads=NTH).forward(0.02, 200, src, rec)
    assert np.linalg.norm(s1 - s0) / np.linalg.norm(s0) < tol


def test_topography_mesh_is_deformed_consistently():
    box = D.BoxSpec(5, 5, 4)
    topo = D.hill_topography(box, 2000.0, 6000.0)
    db = D.make_box(box, topo=topo)
    assert db.nspec_irregular == db.nspec
    jac = db.geo[..., 9]
    assert jac.min() > 0
    # volume: sum of jacobian * w w w equals the box volume under the hill
    _, w = D.gll_points_weights()
    www = w[:, None, None] * w[None, :, None] * w[None, None, :]
    vol = float((jac * www).sum())
    xs = np.linspace(0, box.lx, 801)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    exact = box.lx * box.ly * box.lz + np.trapezoid(np.trapezoid(topo(X, Y), xs), xs)
    assert vol == pytest.approx(exact, rel=1e-5)
    # Stacey faces on the sides are still flat and vertical
    assert np.allclose(np.abs(db.abs_normal).max(axis=2), 1.0, atol=1e-5)


def test_energy_conserved_on_topography_mesh():
    box = D.BoxSpec(5, 5, 4)
    db = D.homogeneous(D.make_box(box, topo=D.hill_topography(box, 2000.0, 6000.0)))
    mt = D.random_moment_tensor(np.random.default_rng(1))
    o = Oracle(db, precision=8, nthreads=NTH, stacey=False)
    e = o.forward_energy(0.02, 600, Oracle.source(10000., 10000., -6000., mt, 1.0), 50)
    tail = e[3:]
    assert np.ptp(tail) / tail.mean() < 1e-3


def test_backward_reconstruction_reversible_on_topography_mesh():
    box = D.BoxSpec(6, 6, 5)
    topo = D.hill_topography(box, 2000.0, 6000.0)
    db = D.make_box(box, topo=topo)
    db = db.with_model(*D.background_model(db, seed=3))
    rec = D.surface_receivers(box, 3)
    rec[:, 2] = topo(rec[:, 0], rec[:, 1])
    mt = D.random_moment_tensor(np.random.default_rng(2))
    o = Oracle(db, precision=8, nthreads=NTH)
    syn = o.forward(0.02, 300, Oracle.source(12000., 12000., -8000., mt, 1.0), rec,
                    save_forward=True)
    _, bseis = o.adjoint(rec, np.zeros_like(syn), want_backward_seis=True)
    assert np.linalg.norm(bseis - syn) / np.linalg.norm(syn) < 1e-11


@pytest.mark.slow
def test_fullspace_green_function_on_warped_mesh():
    box = D.BoxSpec(16, 16, 16, h=2000.0)
    db = D.homogeneous(D.make_box(box, absorb_top=True, warp=D.interior_warp(box, 500.0)))
    assert db.nspec_irregular == db.nspec
    xs = (16000.0, 16000.0, -16000.0)
    xr = np.array([[20000.0, 19000.0, -14000.0]])
    mt = D.random_moment_tensor(np.random.default_rng(17), m0=1e16)
    f0, dt, nstep = 0.5, 0.01, 580
    seis = Oracle(db, precision=8, nthreads=NTH).forward(
        dt, nstep, Oracle.source(*xs, mt, f0), xr)[0]
    t = np.arange(nstep) * dt
    t0 = 1.2 / f0
    u = fullspace_mt(cmt_to_xyz(mt), xs, xr[0], t, lambda tt: ricker(tt - t0, f0),
                     lambda tt: ricker_dot(tt - t0, f0), 6000.0, 3464.0, 2700.0)
    assert np.linalg.norm(seis - u) / np.linalg.norm(u) < 0.03
