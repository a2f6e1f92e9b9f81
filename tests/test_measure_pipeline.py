"""The FP64 measurement pipeline of the oracle against the reference's loops.

``oracle.oracle.measure_waveform`` restates ``LEQData%measure_adj`` for the
waveform misfit (src/preproc/leq_data.f90:48-188) in FP64.  Its pieces are
pinned here:
- the Butterworth band-pass against a line-by-line transcription of SAC's
  xapiir (src/shared/xapiir_sub.f90), run in the reference's FP32 and, to
  check the transcription itself, in FP64; and against scipy's independent
  Butterworth design;
- detrend and interpolation against line-by-line transcriptions;
- the rotations against each other (R,T -> E,N inverts E,N -> R,T);
- one trace end to end against the reference's call sequence written out
  with the transcribed pieces.
"""
import inspect
import os
import sys

import numpy as np
import pytest

from oracle import oracle as O

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import fortran_literal as F  # noqa: E402

DT = 0.02


def _trace(n=1500, seed=0):
    rng = np.random.default_rng(seed)
    t = np.arange(n) * DT
    return (np.sin(2 * np.pi * 0.1 * t) + 0.3 * rng.standard_normal(n)
            + 0.5 * np.sin(2 * np.pi * 2.0 * t))


def _xapiir_fp64():
    src = inspect.getsource(F.xapiir_bu_bp)
    src = src.replace("f32, c64 = np.float32, np.complex64",
                      "f32, c64 = np.float64, np.complex128")
    src = src.replace("return np.array(x, np.float32)", "return np.array(x, np.float64)")
    ns = {}
    exec(src, ns)
    return ns["xapiir_bu_bp"]


@pytest.mark.parametrize("band", [(5.0, 50.0), (2.0, 20.0), (10.0, 100.0)])
@pytest.mark.parametrize("order", [2, 3])
def test_bandpass_matches_xapiir(band, order):
    x = _trace()
    sos = O.butterworth_bandpass_sos(order, 1 / band[1], 1 / band[0], DT)
    ours = O.iir_apply(x, sos, 2)
    # transcription run in FP64: only its 8-digit pi differs
    lit64 = _xapiir_fp64()(x, order, 1 / band[1], 1 / band[0], DT, 2)
    assert np.abs(lit64 - ours).max() < 1e-7 * np.abs(ours).max()
    # the reference's FP32 run: FP32 rounding near the low band edge
    lit32 = F.xapiir_bu_bp(x, order, 1 / band[1], 1 / band[0], DT, 2).astype(np.float64)
    assert np.abs(lit32 - ours).max() < 3e-3 * np.abs(ours).max()


def test_bandpass_design_matches_scipy():
    from scipy import signal
    for order in (1, 2, 4):
        sos = O.butterworth_bandpass_sos(order, 1 / 50.0, 1 / 5.0, DT)
        sc = np.concatenate([sos[:, :3], np.ones((len(sos), 1)), sos[:, 3:]], axis=1)
        ref = signal.butter(order, [1 / 50.0, 1 / 5.0], btype="bandpass", fs=1 / DT,
                            output="sos")
        w = np.linspace(0.001, 5.0, 800)
        _, h1 = signal.sosfreqz(sc, worN=w, fs=1 / DT)
        _, h2 = signal.sosfreqz(ref, worN=w, fs=1 / DT)
        assert np.abs(h1 - h2).max() < 1e-8


def test_detrend_and_interpolation_literal():
    x = _trace(997, 3)
    assert np.abs(np.array(F.detrend(list(x))) - O.detrend(x)).max() < 1e-12
    rng = np.random.default_rng(4)
    xo = rng.standard_normal(900)
    a = np.array(F.interpolate_func_dp(list(xo), -1.3, 0.05, 900, -1.2, 0.02, 2000))
    b = O.interpolate_onto(xo, -1.3, 0.05, -1.2, 0.02, 2000)
    assert np.abs(a - b).max() < 1e-13
    # identical axes: the first and last samples are not strictly inside
    c = O.interpolate_onto(xo, 0.0, 0.02, 0.0, 0.02, 900)
    assert c[0] == 0.0 and c[-1] == 0.0 and np.allclose(c[1:-1], xo[1:-1])


def test_rotation_round_trip():
    rng = np.random.default_rng(5)
    nrec, n = 4, 300
    adj_zrt = rng.standard_normal((nrec, 3, n))
    baz = rng.uniform(0, 360, nrec)
    b = np.deg2rad(baz)[:, None]
    z, r, t = adj_zrt[:, 0], adj_zrt[:, 1], adj_zrt[:, 2]
    e = -r * np.sin(b) - t * np.cos(b)
    nn = -r * np.cos(b) + t * np.sin(b)
    r2 = -e * np.sin(b) - nn * np.cos(b)
    t2 = -e * np.cos(b) + nn * np.sin(b)
    assert np.allclose(r2, r) and np.allclose(t2, t)


def test_one_trace_end_to_end():
    """measure_waveform on one vertical trace against the reference's call
    sequence (leq_data.f90:93-150, waveform_misfit.f90:15-64,
    adjoint_source.f90:92-114) with the transcribed pieces, band-pass in
    FP64."""
    n, t0 = 1200, 1.6
    rng = np.random.default_rng(7)
    syn = np.zeros((1, 3, n))
    syn[0, 2] = _trace(n, 8)
    obs = np.zeros((1, 3, 700))
    obs[0, 2] = rng.standard_normal(700)
    obs_tbeg, obs_dt = -2.0, 0.04
    band = (4.0, 40.0)
    win = np.zeros((1, 1, 3, 2))
    win[0, 0, :] = (3.0, 17.0)
    mis, adj, per = O.measure_waveform(syn, obs, DT, t0, obs_tbeg, obs_dt, [band], win,
                                       pre_taper=0.1, win_taper=0.05, weight=1.5)
    xap = _xapiir_fp64()
    d = F.interpolate_func_dp(list(obs[0, 2]), obs_tbeg, obs_dt, 700, -t0, DT, n)
    d = np.array(F.detrend(d))
    d = d - d.sum() / n
    d = np.array(F.window_taper(list(d), 0.1, 1))
    d = xap(d, 2, 1 / band[1], 1 / band[0], DT, 2)
    s = np.array(F.window_taper(list(syn[0, 2]), 0.1, 1))
    s = xap(s, 2, 1 / band[1], 1 / band[0], DT, 2)
    nb = int((3.0 + t0) / DT) + 1
    ne = int((17.0 + t0) / DT)
    sw = np.array(F.window_taper(list(s[nb - 1:ne]), 0.05, 1))
    dw = np.array(F.window_taper(list(d[nb - 1:ne]), 0.05, 1))
    m = 0.5 * F.simpson(list((sw - dw) ** 2), DT)
    a = np.zeros(n)
    a[nb - 1:ne] = F.window_taper(list(sw - dw), 0.05, 1)
    a = xap(a, 2, 1 / band[1], 1 / band[0], DT, 2)
    out = np.zeros(n)
    out[nb - 1:ne] = F.window_taper(list(a[nb - 1:ne]), 0.05, 1)
    assert per[0, 0, 2] == pytest.approx(1.5 * m, rel=1e-6)
    assert mis[0] == pytest.approx(1.5 * m, rel=1e-6)
    assert np.abs(adj[0, 2] - 1.5 * out).max() < 1e-6 * np.abs(out).max() * 1.5
    assert per[0, 0, 0] == 0.0 and np.all(adj[0, :2] == 0.0)
