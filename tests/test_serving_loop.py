"""The serving loop's scheduling on the host, with a stand-in run.

``Server.run`` and ``MeshServer`` drive a run through the lane primitives
(``lane_start_forward``, ``advance``, ``lane_status``, ``lane_finish``,
``lane_start_adjoint``).  Here the run is a stand-in that only counts
steps, so the scheduling logic runs without a device:
- every request of a mixed stream completes once, through the phases its
  kind asks for, and every lane and store byte is released;
- no lane is started while busy, and the boundary-store budget is never
  exceeded;
- the group policy admits whole 8-lane groups, lanes aligned to the group;
- routing with step costs sends a short burst partly to the one-lane
  server.
The device results of the same loop are checked in tests/test_serving.py.
"""
import numpy as np
import pytest

from specfwat_b200.serving import (PH_ADJ, PH_FWD, PH_IDLE, MeshServer, Request, Server,
                                   StepCosts)


class FakeSim:
    def __init__(self, slots):
        self.state = [[PH_IDLE, 0, 0, False] for _ in range(slots)]
        self.store = 0
        self.max_store = 0
        self.starts = []
        self.lane_errors = {}

    def lane_store_bytes(self, nstep):
        return nstep * 1000

    def lane_start_forward(self, lane, source, receivers, nstep, save_forward):
        assert self.state[lane][0] == PH_IDLE, f"lane {lane} started while busy"
        self.state[lane] = [PH_FWD, 0, nstep, save_forward]
        if save_forward:
            self.store += self.lane_store_bytes(nstep)
            self.max_store = max(self.max_store, self.store)
        self.starts.append(lane)

    def advance(self, n):
        for s in self.state:
            if s[0] != PH_IDLE and s[1] < s[2]:
                s[1] = min(s[2], s[1] + n)

    def lane_status(self, lane):
        ph, st, ns, _ = self.state[lane]
        return ph, st, ns

    def lane_finish(self, lane, seis_out=None, kernels_out=None, ksum_dev_ptr=0):
        ph, st, ns, save = self.state[lane]
        assert st == ns and ph != PH_IDLE
        if seis_out is not None:
            seis_out[...] = lane
        if ph == PH_FWD and save:
            return                       # store kept for the adjoint run
        if ph == PH_ADJ:
            self.store -= self.lane_store_bytes(ns)
        self.state[lane] = [PH_IDLE, 0, 0, False]

    def lane_start_adjoint(self, lane, obs, taper_pct=0.05, taper_type=1, want_misfit=True):
        ph, st, ns, save = self.state[lane]
        assert ph == PH_FWD and st == ns and save
        self.state[lane] = [PH_ADJ, 0, ns, save]
        return 1.0 + lane if want_misfit else None

    def lane_move(self, src, dst):
        assert self.state[dst][0] == PH_IDLE and self.state[src][0] != PH_IDLE
        self.state[dst], self.state[src] = self.state[src], [PH_IDLE, 0, 0, False]
        self.moves = getattr(self, "moves", 0) + 1

    # queued work completes at once in this stand-in
    def lane_finish_async(self, lane, seis_out=None, kernels_out=None, ksum_dev_ptr=0):
        self.lane_finish(lane, seis_out, kernels_out, ksum_dev_ptr)

    def lane_ready(self, lane, wait=False):
        return True

    def lane_misfit(self, lane, out):
        out[0] = 1.0 + lane

    def mark(self):
        self.marks = getattr(self, "marks", 0) + 1
        return self.marks

    def mark_done(self, token, wait=False):
        return True

    def mark_elapsed(self, t0, t1):
        return 1.0

    def synchronize(self):
        pass

    def close(self):
        pass


def mesh_server(name, slots, budget=None, policy="lane", max_wait=0.05):
    return MeshServer.with_sim(name, FakeSim(slots), slots, 10000, 1, store_budget=budget,
                               policy=policy, max_wait=max_wait)


def stream(n, mesh="m", seed=0, spread=0.02):
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(n):
        kind = "fwd" if rng.random() < 0.5 else "fwdadj"
        ns = int(rng.choice([100, 200, 300, 400]))
        reqs.append(Request(rid=k, mesh=mesh, kind=kind, nstep=ns, source=None,
                            receivers=np.zeros((2, 3)),
                            obs=np.zeros((2, 3, ns)) if kind == "fwdadj" else None,
                            arrival=float(rng.uniform(0, spread))))
    return reqs


def check_done(reqs, done, servers):
    assert sorted(r.rid for r in done) == sorted(r.rid for r in reqs)
    for r in done:
        assert r.done >= r.arrival and r.admitted >= r.arrival
        assert r.seismograms is not None and r.seismograms.shape == (2, 3, r.nstep)
        if r.kind == "fwdadj":
            assert r.misfit >= 1.0
        else:
            assert np.isnan(r.misfit)
    for s in servers:
        assert s.store_in_use == 0 and all(x is None for x in s.lanes)
        assert all(st[0] == PH_IDLE for st in s.sim.state) and s.sim.store == 0


def test_mixed_stream_completes_and_releases_everything():
    srv = mesh_server("m", 16)
    reqs = stream(40)
    done = Server({"m": srv}, quantum=50).run(reqs, timeout=60)
    check_done(reqs, done, [srv])


def test_store_budget_is_respected():
    budget = 900 * 1000                       # room for a few stores at a time
    srv = mesh_server("m", 16, budget=budget)
    reqs = stream(30, seed=1)
    done = Server({"m": srv}, quantum=50).run(reqs, timeout=60)
    check_done(reqs, done, [srv])
    assert 0 < srv.sim.max_store <= budget


def test_group_policy_admits_aligned_groups():
    srv = mesh_server("m", 16, policy="group", max_wait=0.05)
    reqs = stream(24, seed=2, spread=0.0)     # all at once: three full groups
    done = Server({"m": srv}, quantum=50).run(reqs, timeout=60)
    check_done(reqs, done, [srv])
    starts = srv.sim.starts
    # consecutive admissions fill a group from its first lane
    for i in range(0, len(starts), 8):
        grp = starts[i:i + 8]
        assert grp[0] % 8 == 0 and grp == list(range(grp[0], grp[0] + len(grp)))


def test_cost_routing_sends_part_of_a_burst_to_the_solo_server():
    batched, solo = mesh_server("m", 16), mesh_server("m", 1)
    costs = {"m": StepCosts(plain_fwd=1e-4, plain_adj=2e-4, group_fwd=3.5e-4, group_adj=8e-4)}
    reqs = stream(30, seed=3, spread=0.0)
    done = Server({"m": batched}, quantum=50, solo={"m": solo}, costs=costs).run(
        reqs, timeout=60)
    check_done(reqs, done, [batched, solo])
    kinds = {r.server for r in done}
    assert kinds == {"solo", "batched"}


def test_busy_lane_start_is_caught_by_the_stand_in():
    sim = FakeSim(2)
    sim.lane_start_forward(0, None, None, 10, False)
    with pytest.raises(AssertionError):
        sim.lane_start_forward(0, None, None, 10, False)


def test_compaction_packs_running_requests_into_fewer_groups():
    """Requests spread over three 8-lane groups by completions are packed
    into fewer groups of the same kind; requests about to switch phase stay
    where they are; the boundary-store accounting follows the requests."""
    srv = mesh_server("m", 24)
    reqs = stream(12, seed=3)
    for k, r in enumerate(reqs):
        r.kind, r.nstep = "fwd", 300
    # lanes 0-1 in group 0, 8-9 in group 1, 16-18 in group 2
    for lane, r in zip([0, 1, 8, 9, 16, 17, 18], reqs):
        srv._admit_one(r, lane, 0.0)
    assert srv.active_groups() == 3
    srv.done_tok[17] = 5          # about to switch: must not move
    moved = srv.compact()
    # the sparsest groups (0, then 1) empty into the fullest (2, which keeps
    # the pinned lane 17): seven requests in one group
    assert moved >= 2
    assert srv.active_groups() < 3
    assert srv.lanes[17] is reqs[5]
    busy = [l for l, r in enumerate(srv.lanes) if r is not None]
    assert len(busy) == 7
    assert sorted(id(srv.lanes[l]) for l in busy) == sorted(id(r) for r in reqs[:7])
    for l in busy:
        assert srv.sim.state[l][0] == PH_FWD


def test_mixed_stream_completes_with_compaction():
    srv = mesh_server("m", 24)
    reqs = stream(60, seed=7, spread=0.05)
    done = Server({"m": srv}, quantum=50).run(reqs, timeout=60)
    # every request completes once and every lane and store byte comes back,
    # whatever moves the wall-clock arrivals led to
    check_done(reqs, done, [srv])


def test_latency_stats_steady_rate():
    """Completions every 2 s after a 30 s ramp: the steady rate is 1800/h
    while the span rate includes the ramp."""
    from specfwat_b200.serving import latency_stats
    reqs = []
    for k in range(50):
        r = Request(rid=k, mesh="m", kind="fwd", nstep=100, source=None,
                    receivers=np.zeros((1, 3)), arrival=0.5 * k)
        r.done = 30.0 + 2.0 * k
        reqs.append(r)
    st = latency_stats(reqs)
    assert st["steady_events_per_hour"] == pytest.approx(1800.0)
    assert st["events_per_hour"] == pytest.approx(50 / 128.0 * 3600.0)
    assert st["p50_s"] > 0
