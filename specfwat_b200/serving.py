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


def _pinned(n, dtype):
    """A 1-D host array of n elements in page-locked memory (through torch,
    when a CUDA device is there), so that result copies queue without
    waiting; pageable numpy memory otherwise."""
    try:
        import torch
        if torch.cuda.is_available():
            t = torch.empty(n, dtype={np.dtype(np.float32): torch.float32,
                                      np.dtype(np.float64): torch.float64}[np.dtype(dtype)])
            t = t.pin_memory()
            a = t.numpy()
            return a, t
    except Exception:
        pass
    return np.empty(n, dtype), None


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
                 group=8, max_wait=1.5, check_every=0, sm_limit=0, high_priority=False):
        mesh = S.Mesh(db)
        sim = S.Simulation(mesh, nstep_max, dt, nev=slots, store=store, use_graph=True,
                           graph_steps=graph_steps, max_receivers=max_receivers,
                           check_every=check_every)
        if high_priority:
            sim.set_sm_share(0, True)
        self._setup(name, mesh, sim, slots, nstep_max, db.nspec, store_budget, ksum_dev_ptr,
                    taper_pct, taper_type, policy, group, max_wait)
        # SMs this mesh's persistent element kernels may fill while another
        # mesh has work (sem_set_sm_share; 0: no limit)
        self.sm_limit = sm_limit
        self.high_priority = high_priority

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
        # pipelined operation: quanta queued on the run and not yet retired,
        # (mark before, mark after, steps, forward groups, adjoint groups);
        # per lane the mark after which its current phase is complete;
        # results queued to page-locked buffers and not yet collected
        self.inflight: deque = deque()
        self.done_tok: List[Optional[int]] = [None] * slots
        self.pending: Dict[int, tuple] = {}
        self._bufs: Dict[tuple, tuple] = {}
        # device ms per step of one active 8-lane group (one lane on a
        # one-lane server), forward and adjoint, learned from the marks
        self.step_ms = {"fwd": None, "adj": None}
        self.quanta = 0
        self.sm_limit = 0
        self.high_priority = False
        self._limit_on = False

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
        return any(r is not None for r in self.lanes) or bool(self.pending)

    def running(self):
        """Lanes that still have steps to queue."""
        out = []
        for lane, req in enumerate(self.lanes):
            if req is None or self.done_tok[lane] is not None:
                continue
            ph, st, ns = self.sim.lane_status(lane)
            if ph != PH_IDLE and st < ns:
                out.append((lane, ph, ns - st))
        return out

    def _groups(self, run):
        g = self.group if self.slots > 1 else 1
        fwd, adj = set(), set()
        for lane, ph, _ in run:
            (adj if ph == PH_ADJ else fwd).add(lane // g)
        return len(fwd - adj), len(adj)

    def share_gpu(self, others_busy):
        """Apply this mesh's SM limit while another mesh has work queued,
        and lift it when none has."""
        on = bool(self.sm_limit) and others_busy
        if on != self._limit_on:
            self.sim.set_sm_share(self.sm_limit if on else 0, self.high_priority)
            self._limit_on = on

    def advance(self, nsteps):
        """Queue nsteps steps of every running lane, bracketed by two marks;
        lanes that complete their phase inside are tagged with the closing
        mark."""
        run = self.running()
        if not run:
            return
        nf, na = self._groups(run)
        t0 = self.sim.mark()
        self.sim.advance(nsteps)
        t1 = self.sim.mark()
        self.inflight.append((t0, t1, nsteps, nf, na))
        for lane, ph, left in run:
            if left <= nsteps:
                self.done_tok[lane] = t1

    def remaining(self):
        """Fewest steps until a running lane completes its phase."""
        run = self.running()
        return min(left for _, _, left in run) if run else None

    def retire(self):
        """Retire the queued quanta that have finished and learn the step
        cost from their device time; returns how many retired."""
        n = 0
        while self.inflight and self.sim.mark_done(self.inflight[0][1]):
            t0, t1, steps, nf, na = self.inflight.popleft()
            n += 1
            try:
                ms = self.sim.mark_elapsed(t0, t1) / steps
            except Exception:
                continue
            self._learn(ms, nf, na)
        return n

    def _learn(self, ms, nf, na, rate=0.3):
        """Step cost model ms = nf * c_fwd + na * c_adj, fitted online."""
        cf, ca = self.step_ms["fwd"], self.step_ms["adj"]
        if na == 0 and nf > 0:
            v = ms / nf
            self.step_ms["fwd"] = v if cf is None else (1 - rate) * cf + rate * v
        elif nf == 0 and na > 0:
            v = ms / na
            self.step_ms["adj"] = v if ca is None else (1 - rate) * ca + rate * v
        elif cf is not None:
            v = max(0.0, (ms - nf * cf) / na)
            self.step_ms["adj"] = v if ca is None else (1 - rate) * ca + rate * v
        self.quanta += 1

    def compact(self):
        """Pack running requests into fewer 8-lane groups (each active group
        costs a share of every step): while a group of one kind (forward
        only, or with adjoint lanes) can be emptied into the free lanes of
        other groups of that kind, its requests move there
        (``sem_lane_move``).  Requests about to switch phase or with results
        still to collect stay put.  Returns the number of moves."""
        g = self.group
        # the group policy keeps requests admitted together in one group
        if self.slots <= g or self.policy == "group":
            return 0
        moves = 0
        for kind in (PH_FWD, PH_ADJ):
            while True:
                groups = {}
                for lane, req in enumerate(self.lanes):
                    if req is None:
                        continue
                    groups.setdefault(lane // g, []).append(lane)
                of_kind = [k for k, ls in groups.items()
                           if (PH_ADJ in (self.phase[l] for l in ls)) == (kind == PH_ADJ)]
                if len(of_kind) < 2:
                    break
                src = min(of_kind, key=lambda k: (len(groups[k]), -k))
                movable = [l for l in groups[src]
                           if self.done_tok[l] is None and l not in self.pending]
                if len(movable) != len(groups[src]):
                    break
                targets = sorted((k for k in of_kind if k != src),
                                 key=lambda k: -len(groups[k]))
                free = [l for k in targets for l in range(k * g, (k + 1) * g)
                        if self.lanes[l] is None and l not in self.pending]
                if len(free) < len(movable):
                    break
                for src_l, dst_l in zip(movable, free):
                    self.sim.lane_move(src_l, dst_l)
                    self.lanes[dst_l], self.lanes[src_l] = self.lanes[src_l], None
                    self.phase[dst_l], self.phase[src_l] = self.phase[src_l], PH_IDLE
                    self.lane_store[dst_l], self.lane_store[src_l] = self.lane_store[src_l], 0
                    moves += 1
        self.moves = getattr(self, "moves", 0) + moves
        return moves

    def _buf(self, lane, key, n, dtype):
        b = self._bufs.get((lane, key))
        if b is None or b[0].size < n:
            b = _pinned(n, dtype)
            self._bufs[(lane, key)] = b
        return b[0][:n]

    def _collect(self, lane, clock):
        kind, req, *rest = self.pending.pop(lane)
        if kind in ("fwd", "seis"):
            req.seismograms = rest[0].reshape(len(req.receivers), 3, req.nstep).copy()
        if kind == "seis":
            return []
        if kind == "adj":
            req.misfit = float(rest[0][0])
            if rest[1] is not None:
                req.kernels = rest[1].reshape(6, self.nspec, 5, 5, 5).copy()
        req.done = clock()
        return [req]

    # -- phase transitions ----------------------------------------------------
    def poll(self, clock):
        """Collect results that have landed, then switch or release the
        lanes whose phase has completed on the device.  Nothing here waits
        for the queued work."""
        finished = []
        for lane in list(self.pending):
            if self.sim.lane_ready(lane):
                finished += self._collect(lane, clock)
        for lane, req in enumerate(self.lanes):
            tok = self.done_tok[lane]
            if req is None or tok is None or not self.sim.mark_done(tok):
                continue
            self.done_tok[lane] = None
            ph, st, ns = self.sim.lane_status(lane)
            if lane in self.pending:            # an earlier result of this lane first
                self.sim.lane_ready(lane, wait=True)
                finished += self._collect(lane, clock)
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
            nseis = len(req.receivers) * 3 * req.nstep
            if ph == PH_FWD:
                buf = self._buf(lane, "seis", nseis, np.float32)
                self.sim.lane_finish_async(lane, seis_out=buf)
                if req.kind == "fwd":
                    self.pending[lane] = ("fwd", req, buf)
                    self._free(lane)
                else:
                    self.pending[lane] = ("seis", req, buf)
                    self.sim.lane_start_adjoint(lane, req.obs, *self.taper, want_misfit=False)
                    self.phase[lane] = PH_ADJ
            elif ph == PH_ADJ:
                mis = self._buf(lane, "misfit", 1, np.float64)
                self.sim.lane_misfit(lane, mis)
                kern = (self._buf(lane, "kern", 6 * self.nspec * 125, np.float64)
                        if req.want_kernels else None)
                self.sim.lane_finish_async(lane, kernels_out=kern,
                                           ksum_dev_ptr=self.ksum_dev_ptr)
                self.pending[lane] = ("adj", req, mis, kern)
                self._free(lane)
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
                 costs: Optional[Dict[str, StepCosts]] = None, compaction=True):
        self.servers = servers
        self.quantum = quantum
        # pack requests into fewer 8-lane groups as others complete
        self.compaction = compaction
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

    def _online_costs(self, name):
        """Step costs of a mesh learned from its servers' marks, once both
        the batched and (if any) the one-lane server have been measured in
        both phases; None before."""
        b = self.servers[name].step_ms
        so = self.solo.get(name)
        if b["fwd"] is None or b["adj"] is None:
            return None
        if so is None:
            return None
        p = so.step_ms
        if p["fwd"] is None or p["adj"] is None:
            return None
        return StepCosts(p["fwd"] / 1e3, p["adj"] / 1e3, b["fwd"] / 1e3, b["adj"] / 1e3)

    def run(self, requests: List[Request], timeout=3600.0, depth=2):
        """Replay a request stream.  Every busy mesh keeps ``depth`` quanta
        queued on its own stream; the host services whichever mesh has a
        quantum finished (marks on the run's stream, no device-wide
        synchronisation), so the GPU always has the next quantum while
        lanes switch, results come back and requests are admitted.  Step
        costs for routing are learned online per mesh once measured."""
        pending = sorted(requests, key=lambda r: r.arrival)
        t0 = time.perf_counter()
        clock = lambda: time.perf_counter() - t0  # noqa: E731
        done: List[Request] = []
        i = 0
        while len(done) < len(requests):
            now = clock()
            if now > timeout:
                raise TimeoutError("serving stream did not finish")
            for name in self.servers:
                learned = self._online_costs(name)
                if learned is not None:
                    self.costs[name] = learned
            while i < len(pending) and pending[i].arrival <= now:
                self._route(pending[i]).queue.append(pending[i])
                i += 1
            for srv in self._all():
                srv.try_admit(now)
                if self.compaction:
                    srv.compact()
            busy = [srv for srv in self._all() if srv.running() or srv.inflight]
            for srv in self._all():
                srv.share_gpu(any(o is not srv and o.mesh is not srv.mesh and
                                  o.name != srv.name for o in busy))
                while len(srv.inflight) < depth:
                    rem = srv.remaining()
                    if rem is None:
                        break
                    srv.advance(max(1, min(self.quantum, rem)))
            progressed = False
            for srv in self._all():
                progressed |= srv.retire() > 0
                got = srv.poll(clock)
                progressed |= bool(got)
                done += got
            if not progressed:
                if not any(srv.inflight or srv.pending for srv in self._all()):
                    if i < len(pending):
                        time.sleep(max(0.0, min(0.01, pending[i].arrival - clock())))
                else:
                    time.sleep(0.0005)
        return done


def latency_stats(reqs: List[Request]):
    """Latency percentiles and throughput of a completed stream: over the
    whole span (first arrival to last completion, ramp-up and drain
    included) and in steady state (the completions between the 10th and
    the 90th percentile completion times, over that interval)."""
    lat = np.array([r.latency for r in reqs])
    span = max(r.done for r in reqs) - min(r.arrival for r in reqs)
    done = np.sort([r.done for r in reqs])
    out = {"n": len(reqs), "p50_s": float(np.percentile(lat, 50)),
           "p99_s": float(np.percentile(lat, 99)),
           "mean_s": float(lat.mean()), "span_s": float(span),
           "events_per_hour": len(reqs) / span * 3600.0}
    if len(done) >= 10:
        i0, i1 = int(0.1 * (len(done) - 1)), int(0.9 * (len(done) - 1))
        if done[i1] > done[i0]:
            out["steady_events_per_hour"] = float((i1 - i0) / (done[i1] - done[i0]) * 3600.0)
    return out
