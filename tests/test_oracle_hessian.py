"""The oracle's approximate Hessian kernel (APPROXIMATE_HESS_KL).

hess = 2 sum_j DT (adjoint accel . backward accel) at every GLL point, the
``hess_kernel`` that PostFlow%sum_precond and apply_precond read
(src/postproc/post_processing.f90:164-230).  The solver that computes it in
the reference is absent, so it is pinned by properties:
- linear in the adjoint source (the backward field does not depend on it);
- FP32 and FP64 runs agree;
- it does not change the other kernels.
"""
import os

import numpy as np

from oracle.oracle import Oracle
from specfwat_b200 import database as D

NTH = min(8, os.cpu_count() or 1)


def case():
    box = D.BoxSpec(5, 5, 4)
    db = D.make_box(box)
    db = db.with_model(*D.background_model(db, seed=21))
    rec = D.surface_receivers(box, 3)
    mt = D.random_moment_tensor(np.random.default_rng(2))
    return db, rec, Oracle.source(9000., 11000., -7000., mt, 1.0)


def run(db, rec, src, prec, scale):
    o = Oracle(db, precision=prec, nthreads=NTH)
    syn = o.forward(0.02, 200, src, rec, save_forward=True)
    kern = o.adjoint(rec, scale * syn)
    return kern, o.hessian()


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_hessian_linear_in_adjoint_source_and_precisions_agree():
    db, rec, src = case()
    k1, h1 = run(db, rec, src, 8, 1.0)
    k3, h3 = run(db, rec, src, 8, 3.0)
    k32, h32 = run(db, rec, src, 4, 1.0)
    assert np.abs(h1).max() > 0
    assert rel(h3, 3.0 * h1) < 1e-12
    assert rel(k3, 3.0 * k1) < 1e-12
    assert rel(h32, h1) < 1e-4
    # the Hessian is an extra accumulator: the six kernels are unchanged
    o = Oracle(db, precision=8, nthreads=NTH)
    syn = o.forward(0.02, 200, src, rec, save_forward=True)
    assert rel(o.adjoint(rec, syn), k1) < 1e-14
