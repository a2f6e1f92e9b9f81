"""Event sharding over ranks and the one exchange step of the path.

Events are independent, so N GPUs run N disjoint event sets with no
data-path collective.  The only exchange is the cross-event kernel sum
(the reference's ``PostFlow%sum_kernel``, ``post_processing.f90:108-149``),
done here as one FP64 all-reduce of the six summed kernels per batch
(rho, mu, kappa and the derived rhop, beta, alpha).  The derived rows are
linear in the primary ones at fixed model, so the sum of the ranks' derived
rows equals the rows derived from the summed primary kernels.  With the
approximate Hessian on, its event sum is reduced the same way.
"""
from __future__ import annotations

from typing import Sequence


def shard_events(n_events: int, rank: int, world: int) -> range:
    """Contiguous block of global event indices owned by ``rank``."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n_events, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def reduce_kernel_sum(ksum, group=None):
    """Sum a rank's event-summed kernels over all ranks in place: a
    [6, ...] FP64 tensor with rows rho, mu, kappa, rhop, beta, alpha (the
    layout of ``sem_sum_kernels``).  All six rows are reduced, so every row
    of the result is the sum over every rank's events."""
    import torch.distributed as dist
    if ksum.dtype.itemsize != 8:
        raise TypeError("kernel sums are reduced in FP64")
    if ksum.shape[0] != 6:
        raise ValueError("kernel sums have six rows (rho, mu, kappa, rhop, beta, alpha)")
    dist.all_reduce(ksum, op=dist.ReduceOp.SUM, group=group)
    return ksum


def reduce_hessian_sum(hsum, group=None):
    """Sum a rank's event-summed Hessian (``Simulation.sum_hessian``; sum of
    |hess| for PRECOND_TYPE 1, of hess for type 0) over all ranks in place,
    in FP64, before the preconditioner is formed
    (``PostFlow%apply_precond``, post_processing.f90:171-185)."""
    import torch.distributed as dist
    if hsum.dtype.itemsize != 8:
        raise TypeError("Hessian sums are reduced in FP64")
    dist.all_reduce(hsum, op=dist.ReduceOp.SUM, group=group)
    return hsum


def derived_kernels(k3, mu, kappa):
    """rhop, beta, alpha from summed rho/mu/kappa kernels (Tromp, Tape &
    Liu 2005), given the model's mu and kappa at the same points."""
    rk, mk, kk = k3
    return (rk + kk + mk, 2.0 * (mk - 4.0 / 3.0 * mu / kappa * kk),
            2.0 * (1.0 + 4.0 / 3.0 * mu / kappa) * kk)


def events_of(all_events: Sequence, rank: int, world: int):
    r = shard_events(len(all_events), rank, world)
    return [all_events[i] for i in r]
