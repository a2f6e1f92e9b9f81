"""Host-side mirror of the reference's per-event driver over the C ABI.

The reference runs one event as (``src/preproc/prepare_fwd.f90:297-384``)::

    run_simulation(1)   InitSpecfem, setup_sources_receivers_fwat,
                        prepare_timerun_fwat, iterate_time, FinalizeSpecfem
    measure_adj         seismograms -> misfit + adjoint sources (SEM/*.adj)
    run_simulation(3)   same chain with SIMULATION_TYPE=3
    postproc_adjoint    save_adjoint_kernels

:class:`Mesh` is the resident database (``read_mesh_databases_fwat`` +
``prepare_GPU``); :class:`Simulation` is one run (``prepare_timerun_fwat``)
with methods named after the reference entry points; :class:`PrepareFWD`
strings them together per run mode (``src/shared/config.f90:52-56``).  All
arrays stay on the device between the forward and adjoint runs: the
boundary store and the final forward state (``absorb_field.bin`` and
``save_forward_arrays.bin`` in the reference) are never written out.
"""
from __future__ import annotations

import ctypes as C
from typing import Iterable, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import check

FORWARD_ONLY, FORWARD_MEASADJ, FORWARD_ADJOINT = 1, 2, 3   # config.f90:52-56
KERNEL_NAMES = ("rho", "mu", "kappa", "rhop", "beta", "alpha")


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


class Mesh:
    """A mesh database resident in device memory."""

    def __init__(self, db, index_base: int = 0):
        L = _lib.load()
        self.db = db
        k = dict(
            ibool=np.ascontiguousarray(db.ibool.reshape(-1) + index_base, np.int32),
            x=np.ascontiguousarray(db.xstore, np.float32),
            y=np.ascontiguousarray(db.ystore, np.float32),
            z=np.ascontiguousarray(db.zstore, np.float32),
            kappa=np.ascontiguousarray(db.kappa.reshape(-1), np.float32),
            mu=np.ascontiguousarray(db.mu.reshape(-1), np.float32),
            rho=np.ascontiguousarray(db.rho.reshape(-1), np.float32),
            rmass=np.ascontiguousarray(db.rmass, np.float32),
            rho_vp=np.ascontiguousarray(db.rho_vp.reshape(-1), np.float32),
            rho_vs=np.ascontiguousarray(db.rho_vs.reshape(-1), np.float32),
            f_ispec=np.ascontiguousarray(db.abs_ispec + index_base, np.int32),
            f_ijk=np.ascontiguousarray(db.abs_ijk.reshape(-1) + index_base, np.int32),
            f_jw=np.ascontiguousarray(db.abs_jw.reshape(-1), np.float32),
            f_n=np.ascontiguousarray(db.abs_normal.reshape(-1), np.float32),
        )
        f, i = C.c_float, C.c_int
        irr = getattr(db, "irregular", None)
        nirr = 0
        geo_p = [None] * 10
        irr_p = None
        if irr is not None and (irr >= 0).any():
            # irregular_element_number: 0 regular, k >= 1 row k-1 of the
            # xixstore .. jacobianstore arrays (each [nirr][125])
            k["irr"] = np.ascontiguousarray(np.where(irr >= 0, irr + 1, 0), np.int32)
            nirr = int(db.geo.shape[0])
            for q in range(10):
                k[f"geo{q}"] = np.ascontiguousarray(db.geo[..., q].reshape(nirr, -1), np.float32)
            geo_p = [_p(k[f"geo{q}"], f) for q in range(10)]
            irr_p = _p(k["irr"], i)
        desc = _lib.MeshDesc(
            db.nspec, db.nglob, index_base, _p(k["ibool"], i), _p(k["x"], f),
            _p(k["y"], f), _p(k["z"], f), db.xix_regular, db.jacobian_regular,
            irr_p, _p(k["kappa"], f), _p(k["mu"], f), _p(k["rho"], f),
            _p(k["rmass"], f), _p(k["rho_vp"], f), _p(k["rho_vs"], f),
            db.nfaces, _p(k["f_ispec"], i), _p(k["f_ijk"], i), _p(k["f_jw"], f),
            _p(k["f_n"], f), nirr, *geo_p)
        h = C.c_void_p()
        check(L.sem_prepare_mesh(C.byref(desc), C.byref(h)))
        self._h = h
        self.nspec, self.nglob, self.nfaces = db.nspec, db.nglob, db.nfaces

    @property
    def handle(self):
        return self._h

    def device_bytes(self) -> int:
        b = C.c_longlong()
        check(_lib.load().sem_mesh_info(self._h, None, None, None, C.byref(b)))
        return b.value

    def close(self):
        if getattr(self, "_h", None):
            check(_lib.load().sem_release_mesh(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_source(x, y, z, mt: Sequence[float], f0: float, tshift=0.0):
    """CMT-convention source: ``mt`` = (Mrr, Mtt, Mpp, Mrt, Mrp, Mtp)."""
    return _lib.Source(float(x), float(y), float(z), *[float(m) for m in mt],
                       float(f0), float(tshift))


class Simulation:
    """One run: ``nev`` events sharing a mesh, ``nstep`` steps of ``dt``.

    ``nev == 1`` is the plain one-event-per-launch path; ``nev > 1`` runs all
    events in the same kernels with lane-interleaved wavefields.
    """

    def __init__(self, mesh: Mesh, nstep: int, dt: float, nev: int = 1,
                 store: str = "fp32", use_graph: bool = False,
                 graph_steps: int = 50, max_receivers: int = 128,
                 check_every: int = 0, kernel_variant: int = 0):
        L = _lib.load()
        self.mesh = mesh
        self.nstep, self.dt, self.nev = nstep, dt, nev
        kind = {"fp32": _lib.SEM_STORE_FP32, "fp16": _lib.SEM_STORE_FP16}[store]
        self.cfg = _lib.RunCfg(nev, nstep, dt, kind, int(use_graph),
                               graph_steps, max_receivers, check_every,
                               kernel_variant)
        h = C.c_void_p()
        check(L.sem_prepare_timerun(mesh.handle, C.byref(self.cfg), C.byref(h)))
        self._h = h
        self.nrec = [0] * nev
        self.lane_errors = {}

    # setup_sources_receivers_fwat
    def set_sources(self, sources: Iterable):
        src = list(sources)
        arr = (_lib.Source * len(src))(*src)
        check(_lib.load().sem_set_sources(self._h, len(src), arr))

    def set_receivers(self, xyz, ev: int = -1):
        xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
        check(_lib.load().sem_set_receivers(self._h, ev, xyz.shape[0],
                                            xyz.ctypes.data))
        for e in (range(self.nev) if ev < 0 else [ev]):
            self.nrec[e] = xyz.shape[0]

    # iterate_time
    def iterate_time(self, sim_type: int = 1, save_forward: bool = False,
                     synchronize: bool = True):
        check(_lib.load().sem_iterate_time(self._h, sim_type, int(save_forward)))
        if synchronize:
            self.synchronize()

    def synchronize(self):
        check(_lib.load().sem_synchronize(self._h))

    def seismograms(self, ev: int = 0, out=None) -> np.ndarray:
        if out is None:
            out = np.zeros((self.nrec[ev], 3, self.nstep), np.float32)
        assert out.dtype == np.float32 and out.flags.c_contiguous
        assert out.size == self.nrec[ev] * 3 * self.nstep
        check(_lib.load().sem_get_seismograms(self._h, ev, out.ctypes.data))
        return out

    def set_adjoint_sources(self, ev: int, adj):
        adj = np.ascontiguousarray(adj, np.float64)
        assert adj.shape == (self.nrec[ev], 3, self.nstep)
        check(_lib.load().sem_set_adjoint_sources(self._h, ev, adj.ctypes.data))

    def measure_l2(self, ev: int, obs, taper_pct=0.05, taper_type=1) -> float:
        obs = np.ascontiguousarray(obs, np.float64)
        assert obs.shape == (self.nrec[ev], 3, self.nstep)
        m = C.c_double()
        check(_lib.load().sem_measure_l2(self._h, ev, obs.ctypes.data,
                                         float(taper_pct), int(taper_type),
                                         C.byref(m)))
        return m.value

    def measure_waveform(self, ev: int, obs, windows, cfg, baz=None):
        """Waveform measurement of event ``ev`` with the reference's
        pre-processing (see :mod:`specfwat_b200.measure`); the adjoint
        source stays on the device.  ``obs`` [nrec, 3, obs_npts], windows
        [nband, nrec, 3, 2] (origin time).  Returns (misfit per band,
        per-trace misfits [nband, nrec, 3])."""
        obs = np.ascontiguousarray(obs, np.float64)
        nr = self.nrec[ev]
        assert obs.ndim == 3 and obs.shape[:2] == (nr, 3)
        win = np.ascontiguousarray(windows, np.float64)
        assert win.shape == (cfg.nband_out, nr, 3, 2)
        b = None if baz is None else np.ascontiguousarray(baz, np.float64)
        mb = np.zeros(cfg.nband_out)
        mt = np.zeros((cfg.nband_out, nr, 3))
        c = cfg.to_c(self.dt, obs.shape[-1])
        check(_lib.load().sem_measure_waveform(
            self._h, ev, C.byref(c), obs.ctypes.data, win.ctypes.data,
            None if b is None else b.ctypes.data, mb.ctypes.data, mt.ctypes.data))
        return mb, mt

    def set_observed(self, ev: int, obs):
        """Keep observed data of ``ev`` in device memory for measure_l2."""
        obs = np.ascontiguousarray(obs, np.float64)
        assert obs.shape == (self.nrec[ev], 3, self.nstep)
        check(_lib.load().sem_set_observed(self._h, ev, obs.ctypes.data))

    def measure_l2_resident(self, ev: int, taper_pct=0.05, taper_type=1,
                            want_misfit=False):
        """L2 measurement against the device-resident observed data."""
        m = C.c_double()
        check(_lib.load().sem_measure_l2(
            self._h, ev, None, float(taper_pct), int(taper_type),
            C.byref(m) if want_misfit else None))
        return m.value if want_misfit else None

    def set_stream(self, stream_handle: int):
        """Queue the run's device work on a caller CUDA stream (handle as an
        integer, e.g. ``torch.cuda.current_stream().cuda_stream``)."""
        check(_lib.load().sem_set_stream(self._h, C.c_void_p(stream_handle)))

    def sum_kernels_device(self, dev_ptr: int):
        """FP64 cross-event kernel sum into device memory [6, nspec, 125]."""
        check(_lib.load().sem_sum_kernels_device(self._h, C.c_void_p(dev_ptr)))

    def time_kernels(self, sim_type: int, nsteps: int):
        """Average ms of (forces, stacey, points, update) over nsteps steps."""
        ms = (C.c_double * 4)()
        check(_lib.load().sem_time_kernels(self._h, sim_type, nsteps, ms))
        return list(ms)

    # save_adjoint_kernels
    def save_adjoint_kernels(self, ev: int = 0, out=None) -> np.ndarray:
        if out is None:
            out = np.zeros((6, self.mesh.nspec, 5, 5, 5), np.float64)
        assert out.dtype == np.float64 and out.flags.c_contiguous
        assert out.size == 6 * self.mesh.nspec * 125
        check(_lib.load().sem_save_adjoint_kernels(self._h, ev, out.ctypes.data))
        return out

    def sum_kernels(self, out=None) -> np.ndarray:
        if out is None:
            out = np.zeros((6, self.mesh.nspec, 5, 5, 5), np.float64)
        assert out.dtype == np.float64 and out.flags.c_contiguous
        assert out.size == 6 * self.mesh.nspec * 125
        check(_lib.load().sem_sum_kernels(self._h, out.ctypes.data))
        return out

    # FK injection on the absorbing faces
    def set_injection(self, ev: int, veloc, tract, np_resamp: int = 1, k0: int = 0):
        """Incident velocity and traction on the absorbing face points of
        event ``ev``: ``[nt, nf*25, 3]`` each (Veloc_FK / Tract_FK), sample
        ``k`` at time ``(k + k0) * np_resamp * dt``.  ``veloc=None`` removes
        the injection."""
        if veloc is None:
            check(_lib.load().sem_set_injection(self._h, ev, None, None, 0, 1, 0))
            return
        v = np.ascontiguousarray(veloc, np.float32)
        t = np.ascontiguousarray(tract, np.float32)
        assert v.shape == t.shape and v.ndim == 3 and v.shape[2] == 3
        check(_lib.load().sem_set_injection(self._h, ev, v.ctypes.data, t.ctypes.data,
                                            v.shape[0], int(np_resamp), int(k0)))

    # approximate Hessian (APPROXIMATE_HESS_KL; hess_kernel)
    def set_approximate_hessian(self, enable: bool = True):
        """Accumulate hess = 2 sum DT accel_adj . accel_bwd in the next
        adjoint runs (enable before ``iterate_time(3)``)."""
        check(_lib.load().sem_set_approximate_hessian(self._h, int(bool(enable))))

    def hessian_kernel(self, ev: int = 0) -> np.ndarray:
        """hess_kernel of event ``ev``: [nspec, 5, 5, 5] FP64."""
        out = np.zeros((self.mesh.nspec, 5, 5, 5), np.float64)
        check(_lib.load().sem_save_hessian_kernel(self._h, ev, out.ctypes.data))
        return out

    def sum_hessian(self, abs_each: bool = True) -> np.ndarray:
        """FP64 sum over the events of |hess| (``abs_each``) or hess."""
        out = np.zeros((self.mesh.nspec, 5, 5, 5), np.float64)
        check(_lib.load().sem_sum_hessian(self._h, int(bool(abs_each)), out.ctypes.data))
        return out

    # -- serving primitives (one event per lane, lanes advance together) --
    def mark(self) -> int:
        """Token of a completion mark after everything queued so far."""
        t = C.c_longlong()
        check(_lib.load().sem_mark(self._h, C.byref(t)))
        return t.value

    def mark_done(self, token: int, wait: bool = False) -> bool:
        rc = _lib.load().sem_mark_done(self._h, int(token), int(wait))
        if rc < 0:
            check(rc)
        return rc == 1

    def mark_elapsed(self, t0: int, t1: int) -> float:
        """Device ms between two marks (both among the last 16)."""
        ms = C.c_double()
        check(_lib.load().sem_mark_elapsed(self._h, int(t0), int(t1), C.byref(ms)))
        return ms.value

    def set_store_spill(self, device_bytes: int):
        """Hold the boundary store partly in pinned host memory: at most
        ``device_bytes`` of HBM for it (0: all resident; -1: what is free when
        the store is allocated, less the output buffers)."""
        check(_lib.load().sem_set_store_spill(self._h, int(device_bytes)))

    def store_info(self) -> dict:
        """Layout of the boundary store after the first saved forward run."""
        c, d, n = C.c_int(), C.c_int(), C.c_int()
        db, hb = C.c_longlong(), C.c_longlong()
        check(_lib.load().sem_store_info(self._h, C.byref(c), C.byref(d), C.byref(n),
                                         C.byref(db), C.byref(hb)))
        return {"chunk_steps": c.value, "device_slots": d.value, "chunks": n.value,
                "device_bytes": db.value, "host_bytes": hb.value}

    def lane_store_bytes(self, nstep: int) -> int:
        return int(_lib.load().sem_lane_store_bytes(self._h, nstep))

    def lane_start_forward(self, lane: int, source, receivers, nstep: int,
                           save_forward: bool):
        xyz = np.ascontiguousarray(receivers, np.float64).reshape(-1, 3)
        check(_lib.load().sem_lane_start_forward(
            self._h, lane, C.byref(source), xyz.shape[0], xyz.ctypes.data,
            int(nstep), int(save_forward)))
        self.nrec[lane] = xyz.shape[0]

    def lane_start_adjoint(self, lane: int, obs, taper_pct=0.05, taper_type=1,
                           want_misfit=True):
        obs = np.ascontiguousarray(obs, np.float64)
        m = C.c_double()
        check(_lib.load().sem_lane_start_adjoint(
            self._h, lane, obs.ctypes.data, float(taper_pct), int(taper_type),
            C.byref(m) if want_misfit else None))
        return m.value if want_misfit else None

    def lane_finish_async(self, lane: int, seis_out=None, kernels_out=None,
                          ksum_dev_ptr: int = 0):
        """Queue a lane's results (into page-locked arrays for no waiting);
        read them after ``lane_ready(lane)``."""
        self.lane_errors.pop(lane, None)
        check(_lib.load().sem_lane_finish_async(
            self._h, lane,
            None if seis_out is None else seis_out.ctypes.data,
            None if kernels_out is None else kernels_out.ctypes.data,
            C.c_void_p(ksum_dev_ptr) if ksum_dev_ptr else None))

    def set_sm_share(self, sm_limit: int = 0, high_priority: bool = False):
        """Cap the SMs this run's persistent element kernels fill, and set the
        priority of its own stream (runs of several meshes at once)."""
        check(_lib.load().sem_set_sm_share(self._h, int(sm_limit), int(high_priority)))

    def lane_move(self, src: int, dst: int):
        """Move the request on lane ``src`` to the free lane ``dst``."""
        check(_lib.load().sem_lane_move(self._h, int(src), int(dst)))
        self.nrec[dst] = self.nrec[src]
        err = self.lane_errors.pop(src, None)
        if err is not None:
            self.lane_errors[dst] = err

    def lane_ready(self, lane: int, wait: bool = False) -> bool:
        rc = _lib.load().sem_lane_ready(self._h, lane, int(wait))
        if rc < 0:
            check(rc)
        return rc == 1

    def lane_misfit(self, lane: int, out) -> None:
        """Queue the copy of the lane's FP64 misfit into out[0] (a one-element
        float64 array, page-locked for no waiting)."""
        assert out.dtype == np.float64 and out.size >= 1
        check(_lib.load().sem_lane_misfit(self._h, lane, out.ctypes.data))

    def advance(self, nsteps: int):
        check(_lib.load().sem_advance(self._h, int(nsteps)))

    def lane_status(self, lane: int):
        """(phase, steps done, nstep) of a lane.  A lane stopped by the
        stability check (``check_every``) reports its phase complete and its
        message is kept in ``lane_errors[lane]`` until ``lane_finish``."""
        ph, st, ns = C.c_int(), C.c_int(), C.c_int()
        L = _lib.load()
        rc = L.sem_lane_status(self._h, lane, C.byref(ph), C.byref(st), C.byref(ns))
        if rc == _lib.SEM_ERR_NUMERIC:
            self.lane_errors[lane] = L.sem_last_error().decode()
        else:
            check(rc)
        return ph.value, st.value, ns.value

    def lane_finish(self, lane: int, seis_out=None, kernels_out=None,
                    ksum_dev_ptr: int = 0):
        self.lane_errors.pop(lane, None)
        check(_lib.load().sem_lane_finish(
            self._h, lane,
            None if seis_out is None else seis_out.ctypes.data,
            None if kernels_out is None else kernels_out.ctypes.data,
            C.c_void_p(ksum_dev_ptr) if ksum_dev_ptr else None))

    def kernel_variants(self):
        """(forward, adjoint) element-kernel variants in use."""
        f, a = C.c_int(), C.c_int()
        check(_lib.load().sem_kernel_variants(self._h, C.byref(f), C.byref(a)))
        return f.value, a.value

    def loop_ms(self) -> float:
        ms = C.c_double()
        check(_lib.load().sem_last_loop_ms(self._h, C.byref(ms)))
        return ms.value

    def launch_count(self) -> int:
        n = C.c_longlong()
        check(_lib.load().sem_last_launch_count(self._h, C.byref(n)))
        return n.value

    def close(self):
        if getattr(self, "_h", None):
            check(_lib.load().sem_release_run(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PrepareFWD:
    """Per-event driver in the shape of the reference's ``PrepareFWD``
    (``src/preproc/prepare_fwd.f90:28-35,297-384``): forward run, L2
    measurement against observed data, adjoint run, kernels.

    All ``nev`` events of one call share the mesh and run together.
    """

    def __init__(self, mesh: Mesh, nstep: int, dt: float, nev: int = 1,
                 store: str = "fp32", use_graph: bool = False,
                 graph_steps: int = 50, max_receivers: int = 128,
                 taper_pct: float = 0.05, taper_type: int = 1):
        self.sim = Simulation(mesh, nstep, dt, nev=nev, store=store,
                              use_graph=use_graph, graph_steps=graph_steps,
                              max_receivers=max_receivers)
        self.taper_pct, self.taper_type = taper_pct, taper_type
        self.misfits = np.zeros(nev)

    def setup(self, sources, receivers):
        self.sim.set_sources(sources)
        if isinstance(receivers, (list, tuple)):
            for e, r in enumerate(receivers):
                self.sim.set_receivers(r, e)
        else:
            self.sim.set_receivers(receivers)

    def simulation(self, obs: Optional[Sequence[np.ndarray]] = None,
                   run_mode: int = FORWARD_ADJOINT):
        """Run one pass for all events.  ``obs[ev]`` are observed
        seismograms [nrec, 3, nstep] (needed for run modes >= 2)."""
        sim = self.sim
        sim.iterate_time(1, save_forward=run_mode == FORWARD_ADJOINT,
                         synchronize=False)
        if run_mode == FORWARD_ONLY:
            sim.synchronize()
            return
        for ev in range(sim.nev):
            self.misfits[ev] = sim.measure_l2(ev, obs[ev], self.taper_pct,
                                              self.taper_type)
        if run_mode == FORWARD_ADJOINT:
            sim.iterate_time(3, synchronize=True)

    def close(self):
        self.sim.close()
