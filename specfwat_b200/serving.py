"""Serving loop: continuous batching of simulation requests on resident meshes.

Requests (forward-only or forward+adjoint, each with its own source,
receivers and record length) arrive over time.  Every resident mesh keeps
one lane-batched run (``slots`` event lanes); a request is admitted into a
free lane as soon as one exists and its boundary store fits the HBM budget,
then advances together with whatever else is on that mesh in the same
kernels.  A forward+adjoint request switches its lane to the adjoint run
when its forward is done (FP64 L2 measurement on the device) and frees the
lane when its kernels are summed; the next queued request takes the lane
while the other lanes keep running.  Runs of different meshes sit on their
own CUDA streams, so their work overlaps on the GPU.

The reference has no serving layer: ``xfwat_fwd_measure_adj`` runs events
one after another in one process (``fwat_fwd_measure_adj.f90:43-51``).
"""
from __future__ import annotations

import dataclasses
import time
from collections import deque
from typing import Dict, List, Optional

import numpy as np

from . import solver as S

PH_IDLE, PH_FWD, PH_ADJ = 0, 1, 3


@dataclasses.dataclass
class Request:
    rid: int
    mesh: str
    kind: str                  # "fwd" or "fwdadj"
    nstep: int
    source: object             # solver.make_source(...)
    receivers: np.ndarray      # [nrec, 3]
    obs: Optional[np.ndarray] = None   # [nrec, 3, nstep] for "fwdadj"
    arrival: float = 0.0       # seconds after the start of the stream
    want_kernels: bool = False
    # results
    admitted: float = float("nan")
    server: str = ""                   # "solo" or "batched" (set on admission)
    done: float = float("nan")
    misfit: float = float("nan")
    seismograms: Optional[np.ndarray] = None
    kernels: Optional[np.ndarray] = None
    error: str = ""                    # set when the run was stopped (non-finite field)

    @property
    def latency(self):
        return self.done - self.arrival


@dataclasses.dataclass
class StepCosts:
    """Device seconds per step on one mesh, for routing: one event alone on
    the plain path, and one active 8-lane group of the batched run (a
    batched step costs about this times its active groups), forward and
    adjoint phase."""
    plain_fwd: float
    plain_adj: float
    group_fwd: float
    group_adj: float

    def plain(self, kind, nsteps_fwd, nsteps_adj=None):
        """Plain-path seconds of nsteps_fwd forward steps, plus (fwd+adj
        requests) nsteps_adj adjoint steps (default: as many)."""
        na = nsteps_fwd if nsteps_adj is None else nsteps_adj
        return nsteps_fwd * self.plain_fwd + (na * self.plain_adj if kind == "fwdadj" else 0.0)

    def group(self, kind, nsteps):
        """Batched seconds of a request in one active group."""
        return nsteps * (self.group_fwd + (self.group_adj if kind == "fwdadj" else 0.0))


class MeshServer:
    """One resident mesh and its lane-batched run."""

    def __init__(self, name, db, slots, nstep_max, dt, store="fp16",
                 graph_steps=50, max_receivers=128, store_budget=None,
                 ksum_dev_ptr=0, taper_pct=0.05, taper_type=1, policy="lane",
                 group=8, max_wait=1.5, check_every=0):
        mesh = S.Mesh(db)
        sim = S.Simulation(mesh, nstep_max, dt, nev=slots, store=store, use_graph=True,
                           graph_steps=graph_steps, max_receivers=max_receivers,
                           check_every=check_every)
        self._setup(name, mesh, sim, slots, nstep_max, db.nspec, store_budget, ksum_dev_ptr,
                    taper_pct, taper_type, policy, group, max_wait)

    @classmethod
    def with_sim(cls, name, sim, slots, nstep_max, nspec, store_budget=None, ksum_dev_ptr=0,
                 taper_pct=0.05, taper_type=1, policy="lane", group=8, max_wait=1.5):
        """A server around an existing run object (anything with the lane
        primitives of ``solver.Simulation``), set up by the same code as a
        server that makes its own mesh and run."""
        self = cls.__new__(cls)
        self._setup(name, None, sim, slots, nstep_max, nspec, store_budget, ksum_dev_ptr,
                    taper_pct, taper_type, policy, group, max_wait)
        return self

    def _setup(self, name, mesh, sim, slots, nstep_max, nspec, store_budget, ksum_dev_ptr,
               taper_pct, taper_type, policy, group, max_wait):
        self.name = name
        self.mesh = mesh
        self.sim = sim
        self.slots = slots
        self.nstep_max = nstep_max
        self.lanes: List[Optional[Request]] = [None] * slots
        self.queue: deque = deque()
        self.store_budget = store_budget
        self.store_in_use = 0
        self.lane_store = [0] * slots
        self.ksum_dev_ptr = ksum_dev_ptr
        self.taper = (taper_pct, taper_type)
        self.nspec = nspec
        self.phase = [PH_IDLE] * slots
        # "lane": a request takes any free lane at once.  "group": requests
        # enter an 8-lane group together once the group is free and either a
        # full group is queued or the oldest request has waited `max_wait`
        # seconds, so a group's lanes stay in the same phase and share the
        # cheaper one-field launches while forward.
        self.policy = policy
        self.group = group
        self.max_wait = max_wait

    # -- admission ----------------------------------------------------------
    def _admit_one(self, req, lane, now):
        need = self.sim.lane_store_bytes(req.nstep) if req.kind == "fwdadj" else 0
        self.sim.lane_start_forward(lane, req.source, req.receivers, req.nstep,
                                    save_forward=req.kind == "fwdadj")
        self.lanes[lane] = req
        self.phase[lane] = PH_FWD
        self.lane_store[lane] = need
        self.store_in_use += need
        req.admitted = now
        req.server = "solo" if self.slots == 1 else "batched"

    def _fits(self, req):
        need = self.sim.lane_store_bytes(req.nstep) if req.kind == "fwdadj" else 0
        return self.store_budget is None or not need or \
            self.store_in_use + need <= self.store_budget

    def try_admit(self, now):
        if self.policy == "group":
            return self._admit_groups(now)
        started = 0
        while self.queue:
            req = self.queue[0]
            free = [i for i, r in enumerate(self.lanes) if r is None]
            if not free:
                break
            need = self.sim.lane_store_bytes(req.nstep) if req.kind == "fwdadj" else 0
            if self.store_budget is not None and need and \
                    self.store_in_use + need > self.store_budget:
                break
            self.queue.popleft()
            # prefer a lane whose 8-lane group runs no adjoint field, so
            # forward lanes share the cheaper one-field launches; then the
            # fullest group, so that fewer groups are launched
            lane = min(free, key=lambda l: (self._adj_in_group(l), -self._busy_in_group(l), l))
            self.sim.lane_start_forward(lane, req.source, req.receivers, req.nstep,
                                        save_forward=req.kind == "fwdadj")
            self.lanes[lane] = req
            self.phase[lane] = PH_FWD
            self.lane_store[lane] = need
            self.store_in_use += need
            req.admitted = now
            req.server = "solo" if self.slots == 1 else "batched"
            started += 1
        return started

    def _admit_groups(self, now):
        started = 0
        g = self.group
        while self.queue:
            full = len(self.queue) >= g
            waited = now - self.queue[0].arrival >= self.max_wait
            if not (full or waited):
                break
            free = [k for k in range(self.slots // g)
                    if all(self.lanes[l] is None for l in range(k * g, (k + 1) * g))]
            if not free:
                break
            base = free[0] * g
            n = 0
            while self.queue and n < g and self._fits(self.queue[0]):
                self._admit_one(self.queue.popleft(), base + n, now)
                n += 1
            if n == 0:
                break
            started += n
        return started

    def _busy_in_group(self, lane):
        g = lane // 8
        return sum(1 for l in range(8 * g, min(8 * g + 8, self.slots))
                   if self.lanes[l] is not None)

    def active_groups(self):
        return len({l // 8 for l, r in enumerate(self.lanes) if r is not None})

    def groups_after_admit(self):
        """Active 8-lane groups once one more request is admitted (it goes
        to an active group when one has a free lane), or None when no lane
        is free."""
        free = [l for l, r in enumerate(self.lanes) if r is None]
        if not free:
            return None
        g = self.active_groups()
        return g if any(self._busy_in_group(l) for l in free) else g + 1

    def lane_free_times(self, costs: StepCosts):
        """Sorted seconds until each busy lane frees, at the current number
        of active groups (for the batched server)."""
        g = max(1, self.active_groups())
        out = []
        for lane, req in enumerate(self.lanes):
            if req is None:
                continue
            ph, st, ns = self.sim.lane_status(lane)
            left = max(0, ns - st)
            if ph == PH_FWD:
                t = left * costs.group_fwd + (req.nstep * costs.group_adj
                                              if req.kind == "fwdadj" else 0.0)
            else:
                t = left * costs.group_adj
            out.append(t * g)
        return sorted(out)

    def backlog(self, costs: StepCosts):
        """Plain-path seconds of the work queued and running here (for the
        one-lane server)."""
        t = sum(costs.plain(r.kind, r.nstep) for r in self.queue)
        for lane, req in enumerate(self.lanes):
            if req is None:
                continue
            ph, st, ns = self.sim.lane_status(lane)
            left = max(0, ns - st)
            if ph == PH_FWD:
                t += costs.plain(req.kind, left, req.nstep)
            elif ph == PH_ADJ:
                t += left * costs.plain_adj
        return t

    def _adj_in_group(self, lane):
        g = lane // 8
        return sum(1 for l in range(8 * g, min(8 * g + 8, self.slots))
                   if self.phase[l] == PH_ADJ)

    def busy(self):
        return any(r is not None for r in self.lanes)

    def advance(self, nsteps):
        if self.busy():
            self.sim.advance(nsteps)

    def remaining(self):
        """Fewest steps until some active lane completes its phase."""
        best = None
        for lane, req in enumerate(self.lanes):
            if req is None:
                continue
            ph, st, ns = self.sim.lane_status(lane)
            if ph != PH_IDLE and st < ns:
                best = ns - st if best is None else min(best, ns - st)
        return best

    # -- phase transitions ----------------------------------------------------
    def poll(self, clock):
        finished = []
        for lane, req in enumerate(self.lanes):
            if req is None:
                continue
            ph, st, ns = self.sim.lane_status(lane)
            if ph == PH_IDLE or st < ns:
                continue
            if lane in self.sim.lane_errors:
                # stopped by the stability check: released without results
                req.error = self.sim.lane_errors[lane]
                try:
                    self.sim.lane_finish(lane)
                except S._lib.SemError as e:
                    if e.code != S._lib.SEM_ERR_NUMERIC:
                        raise
                self._free(lane)
                req.done = clock()
                finished.append(req)
                continue
            if ph == PH_FWD and req.kind == "fwd":
                req.seismograms = np.zeros((len(req.receivers), 3, req.nstep), np.float32)
                self.sim.lane_finish(lane, seis_out=req.seismograms)
                self._free(lane)
                req.done = clock()
                finished.append(req)
            elif ph == PH_FWD:
                req.seismograms = np.zeros((len(req.receivers), 3, req.nstep), np.float32)
                self.sim.lane_finish(lane, seis_out=req.seismograms)
                req.misfit = self.sim.lane_start_adjoint(lane, req.obs, *self.taper)
                self.phase[lane] = PH_ADJ
            elif ph == PH_ADJ:
                if req.want_kernels:
                    req.kernels = np.zeros((6, self.nspec, 5, 5, 5), np.float64)
                self.sim.lane_finish(lane, kernels_out=req.kernels,
                                     ksum_dev_ptr=self.ksum_dev_ptr)
                self._free(lane)
                req.done = clock()
                finished.append(req)
        return finished

    def _free(self, lane):
        self.phase[lane] = PH_IDLE
        self.store_in_use -= self.lane_store[lane]
        self.lane_store[lane] = 0
        self.lanes[lane] = None

    def close(self):
        self.sim.close()
        if self.mesh is not None:
            self.mesh.close()


class Server:
    """Request loop over several mesh servers.

    ``run(requests)`` replays a stream: a request becomes visible at its
    ``arrival`` time (wall clock from the start of the call), is queued on
    its mesh, admitted when a lane and budget are free, and completes when
    its results are on the host (and its kernels summed).  ``quantum`` is
    the number of steps every busy mesh advances between scheduling
    decisions (shortened when a lane completes sooner)."""

    def __init__(self, servers: Dict[str, MeshServer], quantum=100,
                 solo: Optional[Dict[str, MeshServer]] = None, solo_below=4,
                 costs: Optional[Dict[str, StepCosts]] = None):
        self.servers = servers
        self.quantum = quantum
        # Optional one-lane server per mesh (the plain one-event kernels).
        # A lone request in an 8-lane group costs the whole group's
        # launches, about four times the one-event path.  Without step
        # costs: while the batched server of its mesh holds fewer than
        # `solo_below` requests (running or queued) and the solo server is
        # free, an arriving request takes the solo server.  With step costs
        # per mesh: the request goes where it is predicted to finish first,
        # the solo server's backlog plus its plain time against its batched
        # time at the group count its admission leaves (plus the wait for
        # a lane when none is free).  A short burst is then served mostly
        # one event at a time and a sustained load mostly batched.
        self.solo = solo or {}
        self.solo_below = solo_below
        self.costs = costs or {}

    def _route(self, req):
        batched = self.servers[req.mesh]
        solo = self.solo.get(req.mesh)
        if solo is None:
            return batched
        c = self.costs.get(req.mesh)
        if c is None:
            if not solo.busy() and not solo.queue:
                load = sum(1 for r in batched.lanes if r is not None) + len(batched.queue)
                if load < self.solo_below:
                    return solo
            return batched
        t_solo = solo.backlog(c) + c.plain(req.kind, req.nstep)
        g = batched.groups_after_admit()
        if g is not None and not batched.queue:
            t_batched = c.group(req.kind, req.nstep) * g
        else:
            # wait for a lane: the (queued + 1)-th lane to free
            free_at = batched.lane_free_times(c) or [0.0]
            wait = free_at[min(len(batched.queue), len(free_at) - 1)]
            t_batched = wait + c.group(req.kind, req.nstep) * max(1, batched.active_groups())
        return solo if t_solo <= t_batched else batched

    def _all(self):
        return list(self.servers.values()) + list(self.solo.values())

    def run(self, requests: List[Request], timeout=3600.0):
        pending = sorted(requests, key=lambda r: r.arrival)
        t0 = time.perf_counter()
        clock = lambda: time.perf_counter() - t0  # noqa: E731
        done: List[Request] = []
        i = 0
        while len(done) < len(requests):
            now = clock()
            if now > timeout:
                raise TimeoutError("serving stream did not finish")
            while i < len(pending) and pending[i].arrival <= now:
                self._route(pending[i]).queue.append(pending[i])
                i += 1
            for srv in self._all():
                srv.try_admit(now)
            busy = [s for s in self._all() if s.busy()]
            if not busy:
                if i < len(pending):
                    time.sleep(max(0.0, min(0.01, pending[i].arrival - clock())))
                continue
            for srv in busy:
                rem = srv.remaining()
                n = self.quantum if rem is None else max(1, min(self.quantum, rem))
                srv.advance(n)
            # one quantum in flight per mesh: new arrivals wait at most one
            # quantum before they can take a lane
            for srv in busy:
                srv.sim.synchronize()
            for srv in busy:
                done += srv.poll(clock)
        return done


def latency_stats(reqs: List[Request]):
    lat = np.array([r.latency for r in reqs])
    span = max(r.done for r in reqs) - min(r.arrival for r in reqs)
    return {"n": len(reqs), "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "span_s": float(span),
            "events_per_hour": len(reqs) / span * 3600.0}
