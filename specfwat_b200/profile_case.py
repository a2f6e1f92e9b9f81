"""Short forward + adjoint run of the solver for profilers and kernel timing.

``python -m specfwat_b200.profile_case --mesh medium --nev 8 --nstep 40``
runs ``nstep`` forward steps (saving the boundary store), an L2
measurement against zero data and ``nstep`` adjoint steps, all launched
step by step (no CUDA graphs) so that every kernel launch is visible to a
profiler, then prints the per-kernel CUDA-event timings as one JSON line.

``--smooth NF`` instead smooths NF random element fields on the mesh
(sigma_h 10 km, sigma_v 5 km, or ``--smooth-steps`` steps) and prints the
smoother's statistics.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import database as D
from . import solver as S


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--mesh", default="medium")
    p.add_argument("--nev", type=int, default=1)
    p.add_argument("--nstep", type=int, default=40)
    p.add_argument("--variant", type=int, default=0)
    p.add_argument("--store", default="fp32")
    p.add_argument("--time-steps", type=int, default=0,
                   help="also time each kernel over this many extra steps")
    p.add_argument("--smooth", type=int, default=0,
                   help="smooth this many element fields instead")
    p.add_argument("--smooth-steps", type=int, default=0)
    p.add_argument("--topo", type=float, default=0.0,
                   help="hill topography height (m): every element irregular")
    a = p.parse_args(argv)
    if a.topo:
        box = D.config_box(a.mesh)
        db = D.make_box(box, topo=D.hill_topography(box, a.topo, 0.25 * box.lx))
        db = db.with_model(*D.background_model(db, seed=1234))
    else:
        db = D.build(a.mesh)
    if a.smooth:
        from .postproc import smooth_sem_pde
        mesh = S.Mesh(db)
        dat = np.random.default_rng(1).standard_normal(
            (a.smooth, db.nspec, 5, 5, 5)).astype(np.float32)
        _, st = smooth_sem_pde(mesh, dat, 10000.0, 5000.0,
                               nstep=a.smooth_steps or None)
        print(json.dumps({"mesh": a.mesh, "fields": a.smooth, **st}), flush=True)
        mesh.close()
        return
    rec = D.surface_receivers(db.box, 10)
    rng = np.random.default_rng(7)
    box = db.box
    srcs = [S.make_source(rng.uniform(0.2, 0.8) * box.lx,
                          rng.uniform(0.2, 0.8) * box.ly,
                          -rng.uniform(0.1, 0.5) * box.lz,
                          D.random_moment_tensor(rng), rng.uniform(0.5, 1.5))
            for _ in range(a.nev)]
    mesh = S.Mesh(db)
    sim = S.Simulation(mesh, a.nstep, 0.02, nev=a.nev, store=a.store,
                       max_receivers=len(rec), kernel_variant=a.variant)
    sim.set_sources(srcs)
    sim.set_receivers(rec)
    sim.iterate_time(1, save_forward=True)
    fwd_ms = sim.loop_ms()
    zero = np.zeros((len(rec), 3, a.nstep))
    for e in range(a.nev):
        sim.measure_l2(e, zero)
    sim.iterate_time(3)
    adj_ms = sim.loop_ms()
    out = {"mesh": a.mesh, "nev": a.nev, "nstep": a.nstep,
           "variant": a.variant, "variants_used": sim.kernel_variants(),
           "fwd_ms_per_step": fwd_ms / a.nstep,
           "adj_ms_per_step": adj_ms / a.nstep}
    if a.time_steps:
        names = ("forces", "stacey", "points", "update")
        out["kernel_ms_fwd"] = dict(zip(names, sim.time_kernels(1, a.time_steps)))
        out["kernel_ms_adj"] = dict(zip(names, sim.time_kernels(3, a.time_steps)))
    print(json.dumps(out), flush=True)
    sim.close()
    mesh.close()


if __name__ == "__main__":
    main()
