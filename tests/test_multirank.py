"""Multi-rank host logic on CPU: event sharding and the FP64 kernel-sum and
Hessian-sum all-reduces, run as two gloo ranks."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from specfwat_b200.shard import (derived_kernels, events_of, reduce_hessian_sum,
                                 reduce_kernel_sum, shard_events)


def test_shard_covers_all_events_once():
    for n in (0, 1, 7, 32, 33):
        for world in (1, 2, 3, 8):
            idx = [i for r in range(world) for i in shard_events(n, r, world)]
            assert idx == list(range(n))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _kernel_sum_for(events):
    """Stand-in for one rank's device kernel sum: CPU oracle kernels of its
    events on a tiny mesh (FP64)."""
    from specfwat_b200 import database as D
    from oracle.oracle import Oracle, l2_adjoint_source
    db = D.build("tiny")
    rec = D.surface_receivers(db.box, 2)
    total = np.zeros((6, db.nspec, 5, 5, 5))
    for (x, y, z, seed) in events:
        mt = D.random_moment_tensor(np.random.default_rng(seed))
        o = Oracle(db, precision=8, nthreads=1)
        src = Oracle.source(x, y, z, mt, 1.0)
        syn = o.forward(0.02, 120, src, rec, save_forward=True)
        _, adj = l2_adjoint_source(syn, 0.5 * syn, 0.02)
        total += o.adjoint(rec, adj)
    return total


def _rank_main(rank, world, port, events, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = events_of(events, rank, world)
        k = torch.from_numpy(_kernel_sum_for(mine).reshape(6, -1).copy())
        reduce_kernel_sum(k)
        if rank == 0:
            np.save(out, k.numpy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.slow
def test_two_ranks_sum_equals_single_rank(tmp_path):
    events = [(4000.0 + 800 * i, 5000.0, -4000.0 - 500 * i, 100 + i) for i in range(4)]
    out = str(tmp_path / "k.npy")
    mp.start_processes(_rank_main, args=(2, _free_port(), events, out), nprocs=2,
                       join=True, start_method="spawn")
    got = np.load(out)
    ref = _kernel_sum_for(events).reshape(6, -1)
    # every row of the reduced [6, ne] tensor (the layout the device sum
    # hands to the collective) is the sum over all events, derived rows too
    for q in range(6):
        assert np.abs(ref[q]).max() > 0
        assert np.allclose(got[q], ref[q], rtol=1e-12, atol=1e-12 * np.abs(ref[q]).max()), q
    from specfwat_b200 import database as D
    db = D.build("tiny")
    mu = db.mu.reshape(-1).astype(np.float64)
    kap = db.kappa.reshape(-1).astype(np.float64)
    d = derived_kernels(got[:3], mu, kap)
    for q in range(3):
        assert np.allclose(d[q], got[3 + q], rtol=1e-9, atol=1e-30)
    with pytest.raises(ValueError):
        reduce_kernel_sum(torch.zeros((3, 4), dtype=torch.float64))


def _hessian_sum_for(events, abs_each):
    """One rank's event-summed approximate Hessian from the CPU oracle."""
    from specfwat_b200 import database as D
    from oracle.oracle import Oracle, l2_adjoint_source
    db = D.build("tiny")
    rec = D.surface_receivers(db.box, 2)
    total = np.zeros((db.nspec, 5, 5, 5))
    for (x, y, z, seed) in events:
        mt = D.random_moment_tensor(np.random.default_rng(seed))
        o = Oracle(db, precision=8, nthreads=1)
        syn = o.forward(0.02, 120, Oracle.source(x, y, z, mt, 1.0), rec, save_forward=True)
        _, adj = l2_adjoint_source(syn, 0.5 * syn, 0.02)
        o.adjoint(rec, adj)
        h = o.hessian()
        total += np.abs(h) if abs_each else h
    return total


def _hess_rank_main(rank, world, port, events, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        h = torch.from_numpy(_hessian_sum_for(events_of(events, rank, world), True).copy())
        reduce_hessian_sum(h)
        if rank == 0:
            np.save(out, h.numpy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_hessian_sum_equals_single_rank(tmp_path):
    events = [(4000.0 + 800 * i, 5000.0, -4000.0 - 500 * i, 200 + i) for i in range(3)]
    out = str(tmp_path / "h.npy")
    mp.start_processes(_hess_rank_main, args=(2, _free_port(), events, out), nprocs=2,
                       join=True, start_method="spawn")
    two = np.load(out)
    one = _hessian_sum_for(events, True)
    assert np.abs(one).max() > 0
    assert np.allclose(two, one, rtol=1e-12, atol=0)
    with pytest.raises(TypeError):
        reduce_hessian_sum(torch.zeros(4, dtype=torch.float32))
