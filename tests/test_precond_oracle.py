"""Kernel preconditioners: the oracle's restatements against the reference's loops.

``oracle.oracle.invert_hess`` / ``hessian_precond`` restate
``PostFlow%apply_precond`` and ``invert_hess``
(src/postproc/post_processing.f90:164-197,333-372), and ``depth_precond``
restates ``zprecond_gll`` (src/postproc/zprecond.f90:11-71) with
``interp1`` (src/shared/utils.f90:889-910).  They are pinned against
FP32 line-by-line transcriptions (tests/golden/fortran_literal.py) and by
the properties the operators have.
"""
import os
import sys

import numpy as np
import pytest

from oracle import oracle as O
from specfwat_b200 import database as D

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import fortran_literal as F  # noqa: E402


def hess_sample(n, seed):
    rng = np.random.default_rng(seed)
    h = rng.standard_normal(n) * np.exp(rng.uniform(-12, 0, n))   # spans the threshold
    h[::17] = 0.0
    return h


@pytest.mark.parametrize("seed", [1, 2])
def test_invert_hess_matches_literal(seed):
    h = np.abs(hess_sample(600, seed))
    lit = np.array(F.invert_hess(h), np.float64)
    ours = O.invert_hess(h)
    assert np.abs(ours - lit).max() <= 2e-6 * np.abs(lit).max()


def test_invert_hess_zero_and_threshold():
    assert np.all(O.invert_hess(np.zeros(10)) == 1.0)
    assert np.all(np.array(F.invert_hess(np.zeros(10))) == 1.0)
    h = np.array([1.0, 0.5, 1e-4, 0.0])
    out = O.invert_hess(h)
    # 1/h normalised by its maximum 1/THRESHOLD_HESS; the small entries
    # both take 1/THRESHOLD_HESS
    assert out == pytest.approx([1e-3, 2e-3, 1.0, 1.0])


def test_precond_types_0_and_1():
    rng = np.random.default_rng(3)
    per_event = rng.standard_normal((4, 300))
    t1 = O.hessian_precond(np.abs(per_event).sum(0), 1)
    t0 = O.hessian_precond(per_event.sum(0), 0)
    assert np.all(t1 > 0) and t1.max() == pytest.approx(1.0)
    assert np.all(t0 > 0) and t0.max() == pytest.approx(1.0)
    assert not np.allclose(t0, t1)
    # the larger the Hessian, the smaller the preconditioner
    h = np.abs(per_event).sum(0)
    order = np.argsort(h)
    assert np.all(np.diff(t1[order]) <= 1e-12)


def test_interp1_matches_literal():
    x = [-40e3, -25e3, -10e3, -2e3, 0.0]
    v = [1.0, 3.0, -2.0, 5.0, 7.0]
    for xq in [-40e3, -33e3, -25e3, -9e3, -2e3, -1.5e3, 0.0, 100.0]:
        assert O.interp1_clamped(x, v, xq) == pytest.approx(F.interp1_0(x, v, xq), rel=1e-12)
    assert F.interp1_0(x, v, -41e3) is None   # the Fortran reads x(0) there


@pytest.mark.parametrize("ptype", [2, 3])
def test_depth_precond_matches_literal(ptype):
    box = D.BoxSpec(2, 2, 2)
    db = D.make_box(box)
    zgrid = np.linspace(-box.lz - 1000.0, 0.0, 13)
    lit = np.array(F.zprecond_gll((db.ibool.reshape(-1) + 1).tolist(), db.zstore, zgrid,
                                  ptype, 7), np.float64)
    ours = O.depth_precond(db, zgrid, ptype, 7).reshape(-1)
    assert np.abs(ours - lit).max() <= 2e-6 * np.abs(lit).max()
    # deeper points get a larger preconditioner (1/|z| grows toward the surface
    # and is inverted)
    z = db.zstore[db.ibool.reshape(-1)]
    deep, shallow = ours[z < -0.75 * box.lz].mean(), ours[z > -0.25 * box.lz].mean()
    assert deep > shallow
