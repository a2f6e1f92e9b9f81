"""FP64 L2 measurement restatement pinned to the reference's Fortran loops.

The golden vectors in tests/golden/measure_golden.json come from
line-by-line transcriptions of utils.f90:simpson, signal.f90:window_taper
and waveform_misfit.f90:calc_adjoint_source (tests/golden/fortran_literal.py).
"""
import json
import os
import sys

import numpy as np
import pytest

from oracle.oracle import l2_adjoint_source, simpson, taper_window

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import fortran_literal as F  # noqa: E402

CASES = json.load(open(os.path.join(HERE, "golden", "measure_golden.json")))


@pytest.mark.parametrize("case", CASES, ids=[f"n{c['n']}" for c in CASES])
def test_golden_l2(case):
    syn = np.array(case["syn"])
    dat = np.array(case["dat"])
    mis, adj = l2_adjoint_source(syn, dat, case["dt"], case["pct"], case["itype"])
    assert mis == pytest.approx(case["misfit"], rel=1e-13, abs=1e-300)
    assert np.allclose(adj, case["adj"], rtol=1e-13, atol=1e-15)
    assert simpson(syn, case["dt"]) == pytest.approx(case["simpson"], rel=1e-12,
                                                     abs=1e-15)
    assert np.allclose(taper_window(case["n"], case["pct"], case["itype"]),
                       case["taper"], rtol=1e-14, atol=1e-15)


def test_simpson_even_branch_quirk():
    """The even-count branch weights y(n-1) by 3 (its loop adds 2 y(n-1)
    on top of the initial y(n-1)); the restatement keeps it."""
    y = np.zeros(8)
    y[6] = 1.0  # y(n-1) in 1-based terms
    dx = 1.0
    expect = dx / 3.0 * (1.0 + 2.0) + 0.5 * dx
    assert F.simpson(list(y), dx) == pytest.approx(expect)
    assert simpson(y, dx) == pytest.approx(expect)


def test_simpson_exact_on_cubics_odd():
    x = np.linspace(0.0, 2.0, 41)
    y = 3 * x ** 3 - x + 1
    exact = 3 * 2 ** 4 / 4 - 2 + 2
    assert simpson(y, x[1] - x[0]) == pytest.approx(exact, rel=1e-13)


def test_vectorised_matches_literal_on_batches():
    rng = np.random.default_rng(9)
    syn = rng.standard_normal((4, 3, 37))
    dat = rng.standard_normal((4, 3, 37))
    mis, adj = l2_adjoint_source(syn, dat, 0.05, 0.15, 2)
    for r in range(4):
        for c in range(3):
            m, a = F.l2_adjoint_source(list(syn[r, c]), list(dat[r, c]), 0.05, 0.15, 2)
            assert mis[r, c] == pytest.approx(m, rel=1e-13)
            assert np.allclose(adj[r, c], a, rtol=1e-13, atol=1e-15)
