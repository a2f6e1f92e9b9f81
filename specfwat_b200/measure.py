"""Waveform measurement with the reference's pre-processing, on the device.

Mirrors ``LEQData%measure_adj`` for the waveform (L2) misfit
(src/preproc/leq_data.f90:48-188): per receiver, component and band the
observed trace is interpolated onto the synthetic axis, detrended, demeaned,
tapered and band-passed, the synthetic is rotated to Z,R,T, tapered and
band-passed, and the window's L2 misfit and adjoint source follow
``WaveformMisfit`` and ``filter_adj``.  The defaults are the reference's
constants (src/shared/config.f90:69-77: taper_per 0.1, IORD 2, PASSES 2).
Windows are given per trace; ``groupvel_windows`` and ``arrival_windows``
compute the two formula-based window types of leq_data.f90:121-135.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import check


@dataclass
class MeasureConfig:
    t0: float = 0.0                  # the synthetic record starts at -t0 (s)
    bands: list = field(default_factory=list)   # [(SHORT_P, LONG_P), ...]
    obs_tbeg: float | None = None    # observed start time; default -t0
    obs_dt: float | None = None      # observed interval; default the run's dt
    order: int = 2                   # IORD
    passes: int = 2                  # PASSES
    pre_taper: float = 0.1           # taper_per
    win_taper: float = 0.05          # taper_percentage
    win_taper_type: int = 1          # itaper_type
    weight: float = 1.0              # src_weight
    rotate: bool = False             # obs in Z,R,T; needs back-azimuths
    adj_norm: bool = False           # ADJ_SRC_NORM

    def to_c(self, dt, obs_npts):
        if len(self.bands) > _lib.MEAS_MAX_BANDS:
            raise ValueError(f"at most {_lib.MEAS_MAX_BANDS} bands")
        sp = (C.c_double * 4)(*[b[0] for b in self.bands] + [0.0] * (4 - len(self.bands)))
        lp = (C.c_double * 4)(*[b[1] for b in self.bands] + [0.0] * (4 - len(self.bands)))
        return _lib.MeasCfg(
            float(self.t0), float(-self.t0 if self.obs_tbeg is None else self.obs_tbeg),
            float(dt if self.obs_dt is None else self.obs_dt), int(obs_npts),
            len(self.bands), sp, lp, int(self.order), int(self.passes),
            float(self.pre_taper), float(self.win_taper), int(self.win_taper_type),
            float(self.weight), int(bool(self.rotate)), int(bool(self.adj_norm)))

    @property
    def nband_out(self):
        return max(1, len(self.bands))


def groupvel_windows(dist, vmin, vmax, long_p, t0, nstep, dt):
    """WIN_GROUPVEL_TYPE (leq_data.f90:121-128): [dist/vmax - T/2,
    dist/vmin + T/2], clamped to [-t0, (NSTEP-2) dt - t0]."""
    w0 = np.maximum(np.asarray(dist) / vmax - long_p / 2.0, -t0)
    w1 = np.minimum(np.asarray(dist) / vmin + long_p / 2.0, (nstep - 2) * dt - t0)
    return np.stack([w0, w1], axis=-1)


def arrival_windows(tp, time_win, t0, nstep, dt):
    """WIN_ARRIVAL_TYPE (leq_data.f90:129-135): [tp + TIME_WIN(1),
    tp + TIME_WIN(2)], clamped likewise."""
    tp = np.asarray(tp, np.float64)
    w0 = np.maximum(tp + time_win[0], -t0)
    w1 = np.minimum(tp + time_win[1], (nstep - 2) * dt - t0)
    return np.stack([w0, w1], axis=-1)


def measure_waveform_dev(seis, obs, windows, cfg: MeasureConfig, dt, baz=None,
                         stream=None):
    """Device-buffer form on torch CUDA tensors: seis [nrec, 3, nstep]
    float32, obs [nrec, 3, obs_npts] float64, windows [nband, nrec, 3, 2]
    float64, baz [nrec] float64.  Returns (adjoint source [nrec, 3, nstep]
    float32, per-trace misfits [nband, nrec, 3] float64), both on the
    device, queued on ``stream`` (torch's current stream by default)."""
    import torch
    nrec, _, nstep = seis.shape
    adj = torch.empty_like(seis)
    mis = torch.empty((cfg.nband_out, nrec, 3), dtype=torch.float64, device=seis.device)
    c = cfg.to_c(dt, obs.shape[-1])
    st = stream if stream is not None else torch.cuda.current_stream(seis.device)
    check(_lib.load().sem_measure_waveform_dev(
        C.c_void_p(seis.data_ptr()), nrec, nstep, float(dt), C.byref(c),
        C.c_void_p(obs.data_ptr()), C.c_void_p(windows.data_ptr()),
        C.c_void_p(baz.data_ptr()) if baz is not None else None,
        C.c_void_p(adj.data_ptr()), C.c_void_p(mis.data_ptr()),
        C.c_void_p(st.cuda_stream)))
    return adj, mis
