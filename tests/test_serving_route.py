"""Routing between the one-lane and the batched server, on the host.

``Server._route`` with step costs sends a request where it is predicted to
finish first: the one-lane server's backlog plus the request's plain time,
against its batched time at the group count its admission leaves (plus the
wait for a lane when none is free).  Lanes are packed into the fullest
group.  Checked with server objects whose run is a stand-in (lane status
only), so no device is needed.
"""

import numpy as np
import pytest

from specfwat_b200.serving import PH_ADJ, PH_FWD, PH_IDLE, MeshServer, Request, Server, StepCosts

C = StepCosts(plain_fwd=0.10e-3, plain_adj=0.20e-3, group_fwd=0.35e-3, group_adj=0.80e-3)


class FakeSim:
    def __init__(self, status):
        self.status = status        # lane -> (phase, step, nstep)
        self.lane_errors = {}

    def lane_status(self, lane):
        return self.status.get(lane, (PH_IDLE, 0, 0))


def server(slots, running=()):
    """running: (lane, kind, nstep, phase, step)."""
    status = {}
    s = MeshServer.with_sim("m", FakeSim(status), slots, 10000, 1)
    for lane, kind, ns, ph, st in running:
        s.lanes[lane] = Request(rid=lane, mesh="m", kind=kind, nstep=ns, source=None,
                                receivers=np.zeros((1, 3)))
        s.phase[lane] = ph
        status[lane] = (ph, st, ns)
    return s


def req(kind="fwdadj", ns=4000):
    return Request(rid=99, mesh="m", kind=kind, nstep=ns, source=None, receivers=np.zeros((1, 3)))


def route(batched, solo, r, costs=True):
    srv = Server({"m": batched}, solo={"m": solo}, costs={"m": C} if costs else None)
    return srv._route(r)


def test_costs_arithmetic():
    assert C.plain("fwd", 100) == pytest.approx(100 * C.plain_fwd)
    assert C.plain("fwdadj", 100) == pytest.approx(100 * (C.plain_fwd + C.plain_adj))
    assert C.plain("fwdadj", 40, 100) == pytest.approx(40 * C.plain_fwd + 100 * C.plain_adj)
    assert C.group("fwdadj", 10) == pytest.approx(10 * (C.group_fwd + C.group_adj))


def test_idle_servers_take_the_plain_path():
    # one active group would cost group time > plain time: solo wins
    assert route(server(32), server(1), req()) is not None
    b, s = server(32), server(1)
    assert route(b, s, req()) is s


def test_busy_solo_sends_work_to_the_batched_server():
    b = server(32)
    s = server(1, [(0, "fwdadj", 4000, PH_FWD, 0)])
    for _ in range(3):
        s.queue.append(req())
    # solo backlog 4 x 4000 x 0.3 ms = 4.8 s; batched alone 4.6 s
    assert route(b, s, req()) is b


def test_packing_keeps_the_group_count():
    b = server(32, [(0, "fwd", 2000, PH_FWD, 500)])
    assert b.groups_after_admit() == 1          # lane 1 is free in group 0
    full = server(8, [(l, "fwd", 2000, PH_FWD, 500) for l in range(8)])
    assert full.groups_after_admit() is None
    b2 = server(16, [(l, "fwd", 2000, PH_FWD, 500) for l in range(8)])
    assert b2.groups_after_admit() == 2         # group 0 is full


def test_full_batched_server_waits_for_a_lane():
    full = server(8, [(l, "fwd", 2000, PH_FWD, 1990) for l in range(8)])
    free_at = full.lane_free_times(C)
    assert len(free_at) == 8 and np.isclose(free_at[0], 10 * C.group_fwd)
    s = server(1, [(0, "fwdadj", 4000, PH_ADJ, 0)])   # solo busy for 0.8 s
    # batched: 10 steps' wait + 4000 fwd+adj group steps = 4.6 s; solo 0.8 + 1.2 s
    assert route(full, s, req()) is s


def test_without_costs_the_old_rule_holds():
    b, s = server(32), server(1)
    assert route(b, s, req(), costs=False) is s
    s_busy = server(1, [(0, "fwd", 100, PH_FWD, 0)])
    assert route(b, s_busy, req(), costs=False) is b


def test_lane_choice_prefers_the_fullest_forward_group():
    b = server(16, [(0, "fwd", 100, PH_FWD, 0), (8, "fwd", 100, PH_FWD, 0),
                    (9, "fwd", 100, PH_FWD, 0)])
    free = [l for l, r in enumerate(b.lanes) if r is None]
    lane = min(free, key=lambda l: (b._adj_in_group(l), -b._busy_in_group(l), l))
    assert lane // 8 == 1
