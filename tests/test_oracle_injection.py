"""FK injection on the absorbing faces: the oracle against the exact solution.

The reference injects a plane wave through the Stacey faces
(COUPLE_WITH_INJECTION_TECHNIQUE, prepare_timerun_fwat.f90:104-117; the
incident field Veloc_FK / Tract_FK of src/shared/fk_coupling.f90:71-439):
the boundary term absorbs the velocity relative to the incident field and
adds its traction.  For a homogeneous half-space with a free surface the
incident field is known exactly (``specfwat_b200.injection``: incident plus
reflected P and SV), and with it injected the interior solution must be
that field.  Checked here:
- the closed-form field: zero traction on the free surface, velocity the
  time derivative of the displacement;
- the oracle's receivers (surface and interior) against it, P and SV
  incidence, within relative L2 1e-3 (2e-4 reached); a one-step time shift
  of the injected samples is 60x worse, so the check resolves one step;
- resampled injection (every 4th step, k0 = -4, cubic interpolation);
- exact backward reconstruction with the injection in the boundary store;
- the layered-model field (``LayeredPlaneWave``, FK3D's role): equal to
  the closed form for one layer and for identical layers (1e-12); zero
  free-surface traction and continuity across an interface with an
  evanescent P layer; injected on a two-layer box, the oracle's receivers
  match it within 2e-3 (4e-4 and 9e-4 reached).
"""
import os

import numpy as np
import pytest

from oracle.oracle import Oracle
from specfwat_b200 import database as D
from specfwat_b200.injection import HalfspacePlaneWave, injection_arrays

NTH = min(8, os.cpu_count() or 1)
VP, VS, RHO = 6000.0, 3464.0, 2700.0
DT, NSTEP = 0.02, 800
ZERO_MT = np.zeros(6)


def box_db():
    box = D.BoxSpec(10, 10, 6, h=2000.0)
    return box, D.homogeneous(D.make_box(box), VP, VS, RHO)


def receivers(box):
    return np.concatenate([D.surface_receivers(box, 4),
                           [[7e3, 9e3, -5e3], [13e3, 11e3, -9e3]]])


def wave(kind):
    theta = 20.0 if kind == "P" else 15.0
    return HalfspacePlaneWave(VP, VS, RHO, theta, 30.0, kind, f0=0.2, t0=5.0,
                              x0=(10e3, 10e3, -12e3))


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("kind", ["P", "SV"])
def test_closed_form_field(kind):
    w = wave(kind)
    xs = np.array([[3e3, 4e3, 0.0], [15e3, 2e3, 0.0], [9e3, 9e3, -4e3]])
    t = np.linspace(0.0, 20.0, 4001)
    up = np.array([[0.0, 0.0, 1.0]] * 3)
    side = np.array([[1.0, 0.0, 0.0]] * 3)
    tr = w.traction(xs[:2], up[:2], t)
    assert np.abs(tr).max() < 1e-12 * np.abs(w.traction(xs, side, t)).max()
    u = w.displacement(xs, t)
    v = w.velocity(xs, t)
    assert np.abs(u).max() > 0.5
    assert np.abs(v - np.gradient(u, t, axis=0)).max() < 1e-4 * np.abs(v).max()


def run(db, rec, v, t, npr=1, k0=0, save=False):
    o = Oracle(db, precision=8, nthreads=NTH)
    o.set_injection(v, t, npr, k0)
    seis = o.forward(DT, NSTEP, Oracle.source(10e3, 10e3, -6e3, ZERO_MT, 1.0), rec,
                     save_forward=save)
    return o, seis


@pytest.mark.parametrize("kind", ["P", "SV"])
def test_oracle_reproduces_the_plane_wave(kind):
    box, db = box_db()
    rec = receivers(box)
    w = wave(kind)
    ana = np.transpose(w.displacement(rec, np.arange(NSTEP) * DT), (1, 2, 0))
    v, t = injection_arrays(db, w, NSTEP, DT)
    _, seis = run(db, rec, v, t)
    assert rel(seis, ana) < 1e-3
    if kind == "P":
        vs, ts = injection_arrays(db, w, NSTEP, DT, 1, 1)   # one step late
        _, late = run(db, rec, vs, ts)
        assert rel(late, ana) > 20 * rel(seis, ana)
        nt = NSTEP // 4 + 10
        vr, tr = injection_arrays(db, w, nt, DT, 4, -4)
        _, res = run(db, rec, vr, tr, 4, -4)
        assert rel(res, ana) < 1e-3


def test_backward_reconstruction_with_injection():
    box, db = box_db()
    rec = receivers(box)
    v, t = injection_arrays(db, wave("P"), NSTEP, DT)
    o, seis = run(db, rec, v, t, save=True)
    _, bseis = o.adjoint(rec, np.zeros_like(seis), want_backward_seis=True)
    assert rel(bseis, seis) < 1e-10


# --------------------------------------------------------------------------
# layered incident field (FK3D's job): LayeredPlaneWave
# --------------------------------------------------------------------------

LAYERS = ([4500.0, VP], [2600.0, VS], [2400.0, RHO], [4000.0])


@pytest.mark.parametrize("kind", ["P", "SV"])
def test_layered_solver_reduces_to_the_halfspace(kind):
    from specfwat_b200.injection import LayeredPlaneWave
    xs = np.array([[3e3, 4e3, 0.0], [15e3, 2e3, -3e3], [9e3, 9e3, -11e3]])
    nrm = np.array([[1.0, 0, 0], [0, -1.0, 0], [0, 0, -1.0]])
    t = np.arange(800) * DT
    hs = wave(kind)
    th = 20.0 if kind == "P" else 15.0
    for lay in (([VP], [VS], [RHO], []),
                ([VP] * 3, [VS] * 3, [RHO] * 3, [2000.0, 5000.0])):
        L = LayeredPlaneWave(*lay, th, 30.0, kind, f0=0.2, t0=5.0, x0=(10e3, 10e3, -12e3))
        for a, b in ((hs.displacement(xs, t), L.displacement(xs, t)),
                     (hs.velocity(xs, t), L.velocity(xs, t)),
                     (hs.traction(xs, nrm, t), L.traction(xs, nrm, t))):
            assert np.abs(a - b).max() < 1e-12 * np.abs(a).max()


def test_layered_boundary_conditions_with_an_evanescent_layer():
    """A fast layer (vp 8000 over a 6000 half-space) at 55 degrees: P is
    evanescent in it.  Free-surface traction vanishes and displacement and
    vertical traction are continuous across the interface."""
    from specfwat_b200.injection import LayeredPlaneWave
    L = LayeredPlaneWave([8000.0, VP], [4600.0, VS], [3000.0, RHO], [3000.0], 55.0, 10.0, "P",
                         f0=0.2, t0=5.0, x0=(0.0, 0.0, -10e3))
    t = np.arange(1000) * DT
    up = np.array([[0.0, 0.0, 1.0]] * 2)
    top = np.array([[1e3, 2e3, 0.0], [5e3, -3e3, 0.0]])
    side = np.array([[1.0, 0.0, 0.0]] * 2)
    assert np.isfinite(L.displacement(top, t)).all()
    scale = np.abs(L.traction(top, side, t)).max()
    assert np.abs(L.traction(top, up, t)).max() < 1e-9 * scale
    eps = 1e-3
    above = np.array([[2e3, 1e3, -3000.0 + eps]])
    below = np.array([[2e3, 1e3, -3000.0 - eps]])
    ua, ub = L.displacement(above, t), L.displacement(below, t)
    assert np.abs(ua - ub).max() < 1e-6 * np.abs(ua).max()
    ta, tb = L.traction(above, up[:1], t), L.traction(below, up[:1], t)
    assert np.abs(ta - tb).max() < 1e-6 * np.abs(ta).max()


def layered_box():
    box = D.BoxSpec(10, 10, 6, h=2000.0)
    db = D.make_box(box)
    zc = db.zstore[db.ibool].reshape(db.nspec, 125).mean(axis=1)
    top = (zc > -LAYERS[3][0])[:, None, None, None]
    ones = np.ones(db.ibool.shape)
    db = db.with_model(*[np.where(top, q[0], q[1]) * ones for q in LAYERS[:3]])
    return box, db


@pytest.mark.parametrize("kind", ["P", "SV"])
def test_oracle_reproduces_the_layered_plane_wave(kind):
    """Layer boundary at an element boundary (4 km); the layered field
    injected on the faces must be the interior solution."""
    from specfwat_b200.injection import LayeredPlaneWave
    box, db = layered_box()
    rec = np.concatenate([D.surface_receivers(box, 4), [[7e3, 9e3, -2e3], [13e3, 11e3, -9e3]]])
    th = 20.0 if kind == "P" else 15.0
    L = LayeredPlaneWave(*LAYERS, th, 30.0, kind, f0=0.2, t0=5.0, x0=(10e3, 10e3, -12e3))
    nstep = 900
    v, t = injection_arrays(db, L, nstep, DT)
    o = Oracle(db, precision=8, nthreads=NTH)
    o.set_injection(v, t)
    seis = o.forward(DT, nstep, Oracle.source(10e3, 10e3, -6e3, ZERO_MT, 1.0), rec)
    ana = np.transpose(L.displacement(rec, np.arange(nstep) * DT), (1, 2, 0))
    assert rel(seis, ana) < 2e-3
