"""Waveform measurement on the device against the FP64 oracle pipeline.

``sem_measure_waveform_dev`` and ``sem_measure_waveform`` (through
``specfwat_b200.measure`` and ``Simulation.measure_waveform``) are compared
with ``oracle.oracle.measure_waveform`` on the same traces:
- observed data on a different time axis (interpolation), two bands,
  back-azimuth rotation, plain and normalised band sums;
- no band-pass;
- the run form feeding the adjoint run: the kernels equal those from the
  oracle's adjoint source injected through ``sem_set_adjoint_sources``.
Both sides are FP64; the adjoint source leaves the device as FP32.
"""
import numpy as np
import pytest

from oracle import oracle as O
from specfwat_b200 import database as D
from specfwat_b200 import solver as S
from specfwat_b200.measure import MeasureConfig, groupvel_windows, measure_waveform_dev

pytestmark = pytest.mark.gpu

DT = 0.02


def _inputs(nrec=5, nstep=1500, obs_npts=900, seed=1):
    rng = np.random.default_rng(seed)
    t = np.arange(nstep) * DT
    syn = np.zeros((nrec, 3, nstep), np.float32)
    for r in range(nrec):
        for c in range(3):
            f = rng.uniform(0.05, 0.4)
            syn[r, c] = (np.sin(2 * np.pi * f * t + rng.uniform(0, 6))
                         * np.exp(-((t - rng.uniform(5, 20)) / 6.0) ** 2))
    obs = rng.standard_normal((nrec, 3, obs_npts)) * 0.3
    baz = rng.uniform(0, 360, nrec)
    dist = rng.uniform(20e3, 60e3, nrec)
    return syn, obs, baz, dist


@pytest.mark.parametrize("adj_norm", [False, True])
def test_device_matches_oracle_bands_rotation(gpu, adj_norm):
    import torch
    syn, obs, baz, dist = _inputs()
    nrec, _, nstep = syn.shape
    t0 = 1.5
    bands = [(3.0, 30.0), (6.0, 60.0)]
    win = np.stack([np.broadcast_to(
        groupvel_windows(dist, 2500.0, 4000.0, b[1], t0, nstep, DT)[:, None, :],
        (nrec, 3, 2)) for b in bands]).copy()
    cfg = MeasureConfig(t0=t0, bands=bands, obs_tbeg=-2.0, obs_dt=0.04, weight=0.7,
                        rotate=True, adj_norm=adj_norm)
    dev = torch.device("cuda", 0)
    adj, mis = measure_waveform_dev(
        torch.from_numpy(syn).to(dev), torch.from_numpy(obs).to(dev),
        torch.from_numpy(win).to(dev), cfg, DT, baz=torch.from_numpy(baz).to(dev))
    torch.cuda.synchronize()
    mref, aref, pref = O.measure_waveform(syn, obs, DT, t0, -2.0, 0.04, bands, win,
                                          weight=0.7, baz=baz, adj_norm=adj_norm)
    mis = mis.cpu().numpy()
    adj = adj.cpu().numpy().astype(np.float64)
    assert np.allclose(mis, pref, rtol=1e-8, atol=1e-14 * np.abs(pref).max())
    assert np.linalg.norm(adj - aref) / np.linalg.norm(aref) < 1e-6


def test_device_matches_oracle_without_band(gpu):
    import torch
    syn, obs, _, _ = _inputs(nrec=3, obs_npts=1500, seed=4)
    nrec, _, nstep = syn.shape
    win = np.zeros((1, nrec, 3, 2))
    win[..., 0], win[..., 1] = 2.0, 25.0
    cfg = MeasureConfig(t0=0.0, bands=[], win_taper=0.1, win_taper_type=2)
    dev = torch.device("cuda", 0)
    adj, mis = measure_waveform_dev(
        torch.from_numpy(syn).to(dev), torch.from_numpy(obs).to(dev),
        torch.from_numpy(win).to(dev), cfg, DT)
    torch.cuda.synchronize()
    mref, aref, pref = O.measure_waveform(syn, obs, DT, 0.0, 0.0, DT, [], win,
                                          win_taper=0.1, win_type=2)
    assert np.allclose(mis.cpu().numpy(), pref, rtol=1e-10)
    a = adj.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(a - aref) / np.linalg.norm(aref) < 1e-6


def test_bad_window_is_nan_on_device(gpu):
    import torch
    syn, obs, _, _ = _inputs(nrec=2, obs_npts=1500)
    nrec, _, nstep = syn.shape
    win = np.zeros((1, nrec, 3, 2))
    win[..., 0], win[..., 1] = 2.0, 25.0
    win[0, 1, 2] = (10.0, 9.0)               # empty
    win[0, 0, 1] = (5.0, nstep * DT + 3.0)   # past the record
    dev = torch.device("cuda", 0)
    adj, mis = measure_waveform_dev(
        torch.from_numpy(syn).to(dev), torch.from_numpy(obs).to(dev),
        torch.from_numpy(win).to(dev), MeasureConfig(), DT)
    torch.cuda.synchronize()
    m = mis.cpu().numpy()
    assert np.isnan(m[0, 1, 2]) and np.isnan(m[0, 0, 1])
    assert np.isfinite(m[0, 0, 0])
    assert np.all(adj.cpu().numpy()[1, 2] == 0.0)


def test_run_form_drives_the_adjoint_run(gpu):
    box = D.BoxSpec(5, 5, 4)
    db = D.make_box(box)
    db = db.with_model(*D.background_model(db, seed=21))
    rec = D.surface_receivers(box, 3)
    rng = np.random.default_rng(6)
    srcs = [S.make_source(rng.uniform(6e3, 14e3), rng.uniform(6e3, 14e3),
                          -rng.uniform(4e3, 10e3), D.random_moment_tensor(rng), 1.0)
            for _ in range(2)]
    nstep = 300
    mesh = S.Mesh(db)
    cfg = MeasureConfig(t0=1.2, bands=[(1.0, 6.0)], weight=1.0, rotate=True)
    nrec = len(rec)
    baz = rng.uniform(0, 360, nrec)
    win = np.zeros((1, nrec, 3, 2))
    win[..., 0], win[..., 1] = -1.0, (nstep - 3) * DT - 1.2
    results = []
    for path in ("device", "host"):
        sim = S.Simulation(mesh, nstep, DT, nev=2, max_receivers=nrec, kernel_variant=1)
        sim.set_sources(srcs)
        sim.set_receivers(rec)
        sim.iterate_time(1, save_forward=True)
        total = []
        for e in range(2):
            syn = sim.seismograms(e)
            z = syn[:, 2]
            b = np.deg2rad(baz)[:, None]
            r_ = -syn[:, 0] * np.sin(b) - syn[:, 1] * np.cos(b)
            t_ = -syn[:, 0] * np.cos(b) + syn[:, 1] * np.sin(b)
            obs = 0.8 * np.stack([z, r_, t_], axis=1).astype(np.float64)
            if path == "device":
                mb, _ = sim.measure_waveform(e, obs, win, cfg, baz=baz)
                total.append(mb[0])
            else:
                m, a, _ = O.measure_waveform(syn, obs, DT, 1.2, -1.2, DT, [(1.0, 6.0)],
                                             win, baz=baz)
                sim.set_adjoint_sources(e, a)
                total.append(m[0])
        sim.iterate_time(3)
        results.append((np.array(total), sim.sum_kernels()))
        sim.close()
    mesh.close()
    (m_dev, k_dev), (m_host, k_host) = results
    assert np.allclose(m_dev, m_host, rtol=1e-6)
    for q in range(3):
        err = np.linalg.norm(k_dev[q] - k_host[q]) / np.linalg.norm(k_host[q])
        assert err < 1e-5, (q, err)
