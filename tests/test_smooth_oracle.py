"""PDE kernel smoothing: the CPU oracle against the reference's loops.

``oracle_smooth_pde`` (oracle/sem_oracle.cpp) restates the CPU branch of
``smooth_sem_pde`` (src/postproc/smooth.f90:7-437).  It is pinned here
against a line-by-line FP32 transcription of that Fortran
(tests/golden/fortran_literal.py) on small boxes, and by the properties the
diffusion operator has: a constant field stays constant and the
volume-weighted integral is conserved.  The reference's regular-element
branch (all nine mapping terms xix_regular) is unstable; that is checked
too, since the device path reproduces it on request.
"""
import os
import sys

import numpy as np
import pytest

from oracle.oracle import Oracle
from specfwat_b200 import database as D

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import fortran_literal as F  # noqa: E402

DMIN = (1.0 - np.sqrt(3.0 / 7.0)) * 2000.0   # 4 km elements


def _field(db, seed=3):
    return np.random.default_rng(seed).standard_normal(
        (db.nspec, 5, 5, 5)).astype(np.float32)


@pytest.mark.parametrize("is_sph,cpml", [(False, False), (False, True), (True, False)])
def test_oracle_matches_literal_fortran(is_sph, cpml):
    box = D.BoxSpec(2, 2, 2, x0=2.0e5 if is_sph else 0.0, y0=1.0e5 if is_sph else 0.0)
    db = D.make_box(box)
    dat = _field(db)
    is_cpml = np.array([1, 0, 0, 0, 0, 0, 0, 0]) if cpml else None
    o = Oracle(db, precision=4, nthreads=1)
    out, n, _ = o.smooth_pde(dat, 6000.0, 3000.0, DMIN, is_sph=is_sph,
                             mapping=1, nstep=3, is_cpml=is_cpml)
    lit, n2 = F.smooth_sem_pde_cpu(
        dat.reshape(-1), (db.ibool.reshape(-1) + 1).tolist(), db.xstore,
        db.ystore, db.zstore, db.xix_regular, db.jacobian_regular, 6000.0,
        3000.0, DMIN, is_sph, is_cpml=is_cpml, nstep=3)
    lit = np.asarray(lit, np.float64).reshape(out.shape)
    assert n == n2 == 3
    assert np.abs(out - lit).max() <= 1e-6 * np.abs(lit).max()


def test_step_count_and_coefficients():
    db = D.make_box(D.BoxSpec(2, 2, 2))
    o = Oracle(db, precision=8, nthreads=1)
    _, n, (cv, ch) = o.smooth_pde(_field(db), 6000.0, 3000.0, DMIN, nstep=1)
    cmax = np.float32(np.float32(DMIN) ** 2 / np.float32(9.0))
    assert ch == pytest.approx(float(cmax), rel=1e-7)
    assert cv == pytest.approx(float(cmax) * 0.25, rel=1e-6)
    _, n, _ = o.smooth_pde(_field(db), 6000.0, 3000.0, DMIN)
    assert n == int(np.ceil(6000.0 ** 2 / (2.0 * float(cmax))))


WG = np.array([0.1, 49 / 90, 32 / 45, 49 / 90, 0.1])
WK = WG[:, None, None] * WG[None, :, None] * WG[None, None, :]   # [k][j][i]


def volume_integral(out):
    """sum over element points of w_i w_j w_k * value: the lumped-volume
    integral of the continuous field (up to the constant Jacobian)."""
    return float((out * WK).sum())


def test_cube_mapping_conserves_and_keeps_constants():
    db = D.make_box(D.BoxSpec(4, 4, 3))
    o = Oracle(db, precision=8, nthreads=2)
    dat = _field(db, 5)
    one, _, _ = o.smooth_pde(dat, 8000.0, 4000.0, DMIN, nstep=1)
    out, _, _ = o.smooth_pde(dat, 8000.0, 4000.0, DMIN, nstep=60)
    scale = float(np.abs(out * WK).sum())
    assert abs(volume_integral(out) - volume_integral(one)) <= 1e-10 * scale
    assert out.std() < 0.5 * one.std()          # it smooths
    const = np.full_like(dat, 2.5)
    c, _, _ = o.smooth_pde(const, 8000.0, 4000.0, DMIN, nstep=40)
    assert np.abs(c - 2.5).max() < 1e-12


def test_reference_regular_branch_diverges():
    db = D.make_box(D.BoxSpec(4, 4, 4))
    o = Oracle(db, precision=8, nthreads=2)
    dat = _field(db)
    out, _, _ = o.smooth_pde(dat, 6000.0, 3000.0, DMIN, mapping=1, nstep=40)
    assert not np.isfinite(out).all() or np.abs(out).max() > 1e6 * np.abs(dat).max()
    ok, _, _ = o.smooth_pde(dat, 6000.0, 3000.0, DMIN, mapping=0, nstep=40)
    assert np.abs(ok).max() < np.abs(dat).max()


def _literal_irregular(db, dat, sigma_h, sigma_v, dmin, is_sph, nstep):
    irr = np.asarray(db.irregular)
    stores = [db.geo[..., q].reshape(-1).astype(np.float32) for q in range(10)]
    lit, n2 = F.smooth_sem_pde_cpu(
        dat.reshape(-1), (db.ibool.reshape(-1) + 1).tolist(), db.xstore, db.ystore, db.zstore,
        db.xix_regular, db.jacobian_regular, sigma_h, sigma_v, dmin, is_sph, nstep=nstep,
        irregular_element_number=(irr + 1).tolist(), stores=stores)
    return np.asarray(lit, np.float64).reshape(dat.shape), n2


@pytest.mark.parametrize("is_sph", [False, True])
def test_oracle_matches_literal_fortran_irregular(is_sph):
    """Every element irregular (an interior warp of a 2x2x2 box): the mapping
    terms and Jacobian come from the per-point stores, in the fluxes and in
    the lumped volume, as in the Fortran's ispec_irreg branch."""
    box = D.BoxSpec(2, 2, 2, x0=2.0e5 if is_sph else 0.0, y0=1.0e5 if is_sph else 0.0)
    db = D.make_box(box, warp=D.interior_warp(box, 500.0))
    assert (np.asarray(db.irregular) >= 0).all()
    dat = _field(db, 7)
    o = Oracle(db, precision=4, nthreads=1)
    out, n, _ = o.smooth_pde(dat, 6000.0, 3000.0, DMIN, is_sph=is_sph, nstep=4)
    lit, n2 = _literal_irregular(db, dat, 6000.0, 3000.0, DMIN, is_sph, 4)
    assert n == n2 == 4
    assert np.abs(out - lit).max() <= 2e-6 * np.abs(lit).max()


def test_irregular_mesh_conserves_and_keeps_constants():
    """On a topography mesh (columns stretched under a hill, every element
    irregular), the volume integral with each point's own Jacobian is
    conserved and a constant stays constant."""
    box = D.BoxSpec(4, 4, 3)
    db = D.make_box(box, topo=D.hill_topography(box, 1500.0, 4000.0))
    irr = np.asarray(db.irregular)
    assert (irr >= 0).all()
    jac = np.broadcast_to(np.float64(db.jacobian_regular), (db.nspec, 5, 5, 5)).copy()
    for e in np.nonzero(irr >= 0)[0]:
        jac[e] = db.geo[irr[e], ..., 9]
    o = Oracle(db, precision=8, nthreads=2)
    dat = _field(db, 11)
    one, _, _ = o.smooth_pde(dat, 8000.0, 4000.0, DMIN, nstep=1)
    out, _, _ = o.smooth_pde(dat, 8000.0, 4000.0, DMIN, nstep=40)
    integ = lambda f: float((f * WK * jac).sum())  # noqa: E731
    scale = float(np.abs(out * WK * jac).sum())
    assert abs(integ(out) - integ(one)) <= 1e-10 * scale
    assert out.std() < 0.6 * one.std()
    c, _, _ = o.smooth_pde(np.full_like(dat, -1.5), 8000.0, 4000.0, DMIN, nstep=30)
    assert np.abs(c + 1.5).max() < 1e-12


def test_mixed_flags_equal_regular():
    """A regular box with half of its elements flagged irregular (their
    constant mapping stored per point): regular and irregular branches meet
    in one mesh and give the cube-mapping result."""
    import dataclasses
    db = D.make_box(D.BoxSpec(3, 3, 2))
    full = D.as_irregular(db)
    irr = np.full(db.nspec, -1, np.int32)
    pick = np.arange(0, db.nspec, 2)
    irr[pick] = np.arange(pick.size)
    mixed = dataclasses.replace(db, irregular=irr, geo=full.geo[pick].copy())
    dat = _field(db, 13)
    a, _, _ = Oracle(db, precision=8, nthreads=1).smooth_pde(dat, 6000.0, 3000.0, DMIN, nstep=20)
    b, _, _ = Oracle(mixed, precision=8, nthreads=1).smooth_pde(dat, 6000.0, 3000.0, DMIN,
                                                                nstep=20)
    assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max()
