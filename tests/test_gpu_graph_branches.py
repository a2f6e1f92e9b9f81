"""Batched CUDA graphs with one branch per 8-lane group.

With graphs, a batch of more than 8 events captures each lane group's steps
as a branch of its own, with every per-lane array offset to the group's
block of the lane-group layout. The same batch launched step by step
runs on one stream over all lanes. The two must agree for every lane:
- a group handed the wrong block of the fields, the kernel or Hessian
  accumulators or the lane table breaks its lanes by far more than the
  order of the atomic scatter-adds does (about 1e-6 relative between two
  runs);
- a partly filled last group must not touch lanes past the batch, and a
  last group of one event still runs the batch's kernels (variants 2 and 3
  have separate one-event kernels for the one-event layout).

Distinct events per lane, so that lanes of different groups cannot stand in
for one another.
"""
import numpy as np
import pytest

from specfwat_b200 import database as D
from specfwat_b200 import solver as S

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def _batch(mesh, rec, srcs, obs, nstep, graph, variant):
    nev = len(srcs)
    sim = S.Simulation(mesh, nstep, 0.02, nev=nev, store="fp16", use_graph=graph,
                       graph_steps=50, max_receivers=len(rec), kernel_variant=variant)
    sim.set_sources(srcs)
    sim.set_receivers(rec)
    sim.iterate_time(1, save_forward=True)
    seis = [sim.seismograms(e) for e in range(nev)]
    for e in range(nev):
        sim.measure_l2(e, obs[e])
    sim.set_approximate_hessian()
    sim.iterate_time(3)
    kern = [sim.save_adjoint_kernels(e) for e in range(nev)]
    hess = [sim.hessian_kernel(e) for e in range(nev)]
    ksum = sim.sum_kernels()
    sim.close()
    return seis, kern, ksum, hess


@pytest.mark.parametrize("nev,variant", [(20, 11), (17, 5), (17, 3), (9, 2)])
def test_group_branches_match_step_launches(gpu, nev, variant):
    db = D.build("mini")
    rec = D.surface_receivers(db.box, 3)
    rng = np.random.default_rng(400 + nev)
    box = db.box
    srcs = [S.make_source(rng.uniform(0.3, 0.7) * box.lx, rng.uniform(0.3, 0.7) * box.ly,
                          -rng.uniform(0.2, 0.5) * box.lz, D.random_moment_tensor(rng),
                          rng.uniform(0.8, 1.2)) for _ in range(nev)]
    nstep = 260  # not a multiple of the 50-step graph
    obs = [1e-5 * rng.standard_normal((len(rec), 3, nstep)) for _ in range(nev)]
    mesh = S.Mesh(db)
    s0, k0, sum0, h0 = _batch(mesh, rec, srcs, obs, nstep, False, variant)
    s1, k1, sum1, h1 = _batch(mesh, rec, srcs, obs, nstep, True, variant)
    mesh.close()
    for e in range(nev):
        assert rel(s1[e], s0[e]) < 1e-5, (e, rel(s1[e], s0[e]))
        for q in range(6):
            assert rel(k1[e][q], k0[e][q]) < 1e-4, (e, q, rel(k1[e][q], k0[e][q]))
        assert rel(h1[e], h0[e]) < 1e-4, (e, rel(h1[e], h0[e]))
    for q in range(6):
        assert rel(sum1[q], sum0[q]) < 1e-4
    # the lanes are distinct events: no two of them carry the same kernel
    assert rel(k1[0][1], k1[nev - 1][1]) > 0.05
