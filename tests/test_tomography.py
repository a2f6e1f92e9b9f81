"""External tomography model sampled at GLL points (specfwat_b200.tomography),
pinned to line-by-line transcriptions of model_external_values and its
interpolators (tests/golden/fortran_literal.py): trilinear inside the grid's
box with the bisection cell search, nearest non-zero node of the surrounding
8 outside it, per field."""
import numpy as np
import pytest

from specfwat_b200 import database as D
from specfwat_b200.tomography import ExternalModel, apply_external_model, external_model_values
from tests.golden import fortran_literal as F


def _model(rng, zeros=False):
    x = np.cumsum(rng.uniform(800.0, 3000.0, 7)) - 2000.0
    y = np.cumsum(rng.uniform(1000.0, 2500.0, 6)) - 1500.0
    z = -np.cumsum(rng.uniform(500.0, 4000.0, 5))[::-1] + 200.0
    shape = (x.size, y.size, z.size)
    vp = rng.uniform(5000.0, 8000.0, shape)
    vs = vp / rng.uniform(1.6, 1.9, shape)
    rho = rng.uniform(2400.0, 3400.0, shape)
    if zeros:
        # fluid-like nodes with vs = 0 on the faces: the nearest-node rule
        # must skip them for vs only
        vs[0, :, :2] = 0.0
        vs[-1, 1::2, :] = 0.0
        rho[:, 0, -1] = 0.0
    return ExternalModel(x, y, z, vp, vs, rho)


def _points(m, rng, n):
    lo = np.array([m.x[0], m.y[0], m.z[0]])
    hi = np.array([m.x[-1], m.y[-1], m.z[-1]])
    span = hi - lo
    pts = lo + rng.uniform(-0.2, 1.2, (n, 3)) * span
    # grid nodes, axis ends and points on the box faces exactly
    extra = [(m.x[0], m.y[2], m.z[1]), (m.x[-1], m.y[-1], m.z[-1]), (m.x[3], m.y[0], m.z[-1]),
             (m.x[2], m.y[3], m.z[2]), (m.x[-1] + 10.0, m.y[1], m.z[0]),
             (m.x[1], m.y[-1] + 5.0, m.z[0] - 7.0)]
    return np.vstack([pts, np.array(extra)])


@pytest.mark.parametrize("zeros", [False, True])
def test_external_model_matches_transcription(zeros):
    rng = np.random.default_rng(5 + zeros)
    m = _model(rng, zeros)
    pts = _points(m, rng, 400)
    vp, vs, rho = external_model_values(m, pts[:, 0], pts[:, 1], pts[:, 2])
    for k, (px, py, pz) in enumerate(pts):
        p, s, r = F.model_external_values(list(m.x), list(m.y), list(m.z), m.vp.tolist(),
                                          m.vs.tolist(), m.rho.tolist(), px, py, pz)
        inside = (m.x[0] <= px <= m.x[-1] and m.y[0] <= py <= m.y[-1]
                  and m.z[0] <= pz <= m.z[-1])
        for got, want in ((vp[k], p), (vs[k], s), (rho[k], r)):
            want = 0.0 if want is None else want
            if inside:
                assert got == pytest.approx(want, rel=2e-7, abs=1e-3), (k, got, want)
            else:
                assert got == np.float32(want), (k, got, want)   # a node value, exactly


def test_outside_points_take_node_values_and_inside_is_continuous():
    rng = np.random.default_rng(9)
    m = _model(rng)
    # far outside on every side: the corner nodes of the grid
    vp, _, _ = external_model_values(m, [m.x[0] - 1e5, m.x[-1] + 1e5],
                                     [m.y[0] - 1e5, m.y[-1] + 1e5],
                                     [m.z[0] - 1e5, m.z[-1] + 1e5])
    assert vp[0] == np.float32(m.vp[0, 0, 0]) and vp[1] == np.float32(m.vp[-1, -1, -1])
    # a linear field is reproduced inside
    lin = ExternalModel(m.x, m.y, m.z,
                        1.0 + m.x[:, None, None] + 2 * m.y[None, :, None] + 3 * m.z[None, None, :],
                        m.vs, m.rho)
    pts = _points(m, rng, 200)
    ins = ((pts[:, 0] >= m.x[0]) & (pts[:, 0] <= m.x[-1]) & (pts[:, 1] >= m.y[0])
           & (pts[:, 1] <= m.y[-1]) & (pts[:, 2] >= m.z[0]) & (pts[:, 2] <= m.z[-1]))
    vp, _, _ = external_model_values(lin, *pts[ins].T)
    want = 1.0 + pts[ins, 0] + 2 * pts[ins, 1] + 3 * pts[ins, 2]
    assert np.allclose(vp, want, rtol=1e-6)


def test_apply_to_database():
    db = D.make_box(D.BoxSpec(3, 3, 2))
    box = db.box
    rng = np.random.default_rng(2)
    # model grid covering the box except a margin, so edge points use the
    # nearest-node rule
    x = np.linspace(box.x0 + 1000.0, box.x0 + box.lx - 1000.0, 6)
    y = np.linspace(box.y0 + 500.0, box.y0 + box.ly - 500.0, 5)
    z = np.linspace(-box.lz + 800.0, -300.0, 4)
    shape = (6, 5, 4)
    m = ExternalModel(x, y, z, rng.uniform(5500, 6500, shape), rng.uniform(3200, 3700, shape),
                      rng.uniform(2600, 2800, shape))
    out = apply_external_model(db, m)
    ib = db.ibool
    vp, vs, rho = external_model_values(m, db.xstore[ib], db.ystore[ib], db.zstore[ib])
    assert np.allclose(out.vp, vp) and np.allclose(out.vs, vs)
    assert np.allclose(out.rho, rho)
    assert np.all(out.mu > 0) and np.all(out.kappa > 0)
