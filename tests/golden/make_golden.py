"""Generate the golden vectors in this directory.

* measure_golden.json: L2 misfits, adjoint sources, Simpson integrals and
  taper windows of fixed seeded series, from the line-by-line Fortran
  transcriptions in fortran_literal.py.
* oracle_small_fwd.npz: FP64 oracle seismograms of a 4x4x3-element box
  (regression pin of the CPU restatement; physics pins are in
  test_oracle_kat.py).

Run from the repository root: ``python tests/golden/make_golden.py``.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import fortran_literal as F  # noqa: E402


def measure_cases():
    rng = np.random.default_rng(2024)
    cases = []
    for n, pct, it in [(7, 0.3, 1), (8, 0.3, 1), (64, 0.05, 1), (65, 0.1, 2),
                       (100, 0.2, 3), (101, 0.25, 4), (2, 0.0, 1), (1, 0.1, 1),
                       (50, 1.0, 1)]:
        syn = rng.standard_normal(n).tolist()
        dat = (0.7 * np.asarray(syn) + 0.1 * rng.standard_normal(n)).tolist()
        dt = 0.02
        mis, adj = F.l2_adjoint_source(syn, dat, dt, pct, it)
        cases.append(dict(n=n, pct=pct, itype=it, dt=dt, syn=syn, dat=dat,
                          misfit=mis, adj=adj,
                          simpson=F.simpson(syn, dt),
                          taper=F.window_taper([1.0] * n, pct, it)))
    return cases


def oracle_case():
    from specfwat_b200 import database as D
    from oracle.oracle import Oracle
    box = D.BoxSpec(4, 4, 3)
    db = D.make_box(box)
    vp, vs, rho = D.background_model(db, seed=11)
    db = db.with_model(vp, vs, rho)
    rec = D.surface_receivers(box, 3)
    mt = D.random_moment_tensor(np.random.default_rng(3))
    src = Oracle.source(8000.0, 8000.0, -6000.0, mt, 1.0)
    seis = Oracle(db, precision=8, nthreads=1).forward(0.02, 200, src, rec)
    return dict(seis=seis, rec=rec, mt=mt)


if __name__ == "__main__":
    with open(os.path.join(HERE, "measure_golden.json"), "w") as f:
        json.dump(measure_cases(), f)
    oc = oracle_case()
    np.savez_compressed(os.path.join(HERE, "oracle_small_fwd.npz"), **oc)
    print("golden vectors written")
