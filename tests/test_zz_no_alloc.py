"""The allocation-free L2 measurement entry point, through the C ABI.

sem_measure_l2_noalloc serves callers that cannot call cudaMalloc (code
inside another framework's memory pool or a fixed device-memory budget, or a
Fortran host that only passes buffers it already owns): it works on
caller-owned device buffers and keeps its working memory in one static
device array.  Here it is checked against sem_measure_l2 on the same
seismograms and observed data, for two calls in a row: the misfits must
agree to FP64 rounding and the adjoint sources must drive the adjoint run to
the same kernels.  This file is collected last so that a failure here comes
after every other test has run; it also passes on its own in a fresh
process.
"""
import ctypes as C

import numpy as np
import pytest

from specfwat_b200 import _lib
from specfwat_b200 import database as D
from specfwat_b200 import solver as S

pytestmark = pytest.mark.gpu


def _case():
    box = D.BoxSpec(5, 5, 4)
    db = D.make_box(box)
    vp, vs, rho = D.background_model(db, seed=21)
    db = db.with_model(vp, vs, rho)
    rec = D.surface_receivers(box, 3)
    rng = np.random.default_rng(4)
    srcs = [S.make_source(rng.uniform(6e3, 14e3), rng.uniform(6e3, 14e3),
                          -rng.uniform(4e3, 10e3), D.random_moment_tensor(rng),
                          1.0) for _ in range(2)]
    return db, rec, srcs


def _forward(mesh, rec, srcs, nstep, dt):
    sim = S.Simulation(mesh, nstep, dt, nev=len(srcs), max_receivers=len(rec),
                       kernel_variant=1)
    sim.set_sources(srcs)
    sim.set_receivers(rec)
    sim.iterate_time(1, save_forward=True)
    return sim


def test_noalloc_matches_measure_l2(gpu):
    import torch
    db, rec, srcs = _case()
    nstep, dt = 240, 0.02
    mesh = S.Mesh(db)

    # existing entry point
    a = _forward(mesh, rec, srcs, nstep, dt)
    syn = [a.seismograms(e).astype(np.float64) for e in range(2)]
    obs = [0.8 * s + 1e-4 * np.sin(np.arange(nstep) * 0.05)[None, None, :]
           for s in syn]
    ref_misfit = [a.measure_l2(e, obs[e], 0.05, 1) for e in range(2)]
    a.iterate_time(3)
    ref_k = a.sum_kernels()
    a.close()

    # allocation-free entry point on caller-owned device buffers holding the
    # same seismograms, two calls in a row with separate outputs
    b = _forward(mesh, rec, srcs, nstep, dt)
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    adj_dev, mis_dev, keep = [], [], []
    for e in range(2):
        seis = torch.from_numpy(syn[e].astype(np.float32)).to(dev)
        ob = torch.from_numpy(np.ascontiguousarray(obs[e])).to(dev)
        adj = torch.empty((len(rec), 3, nstep), dtype=torch.float32, device=dev)
        mis = torch.empty(1, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rc = lib.sem_measure_l2_noalloc(
            C.c_void_p(seis.data_ptr()), C.c_void_p(ob.data_ptr()), len(rec),
            nstep, dt, 0.05, 1, C.c_void_p(adj.data_ptr()),
            C.c_void_p(mis.data_ptr()), None)
        _lib.check(rc)
        adj_dev.append(adj)
        mis_dev.append(mis)
        keep += [seis, ob]
    torch.cuda.synchronize()
    # a third call, on the set-up device, must not change the device's free
    # memory: the entry point allocates nothing
    free0, _ = torch.cuda.mem_get_info(dev)
    rc = lib.sem_measure_l2_noalloc(
        C.c_void_p(keep[0].data_ptr()), C.c_void_p(keep[1].data_ptr()), len(rec),
        nstep, dt, 0.05, 1, C.c_void_p(adj_dev[0].data_ptr()),
        C.c_void_p(mis_dev[0].data_ptr()), None)
    _lib.check(rc)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0, (free0, free1)
    for e in range(2):
        m = float(mis_dev[e].cpu().item())
        assert abs(m - ref_misfit[e]) <= 1e-12 * abs(ref_misfit[e])
        b.set_adjoint_sources(e, adj_dev[e].cpu().numpy().astype(np.float64))
    b.iterate_time(3)
    k = b.sum_kernels()
    b.close()
    mesh.close()
    for q in range(3):
        err = np.linalg.norm(k[q] - ref_k[q]) / np.linalg.norm(ref_k[q])
        assert err < 1e-5, (q, err)


def test_noalloc_rejects_oversized(gpu):
    lib = _lib.load()
    one = C.c_void_p(1)
    rc = lib.sem_measure_l2_noalloc(one, one, _lib.L2_NOALLOC_MAX_RECEIVERS + 1,
                                    100, 0.02, 0.05, 1, one, one, None)
    assert rc == -1 and b"receivers" in lib.sem_last_error()
    rc = lib.sem_measure_l2_noalloc(one, one, 10, _lib.L2_NOALLOC_MAX_STEPS + 1,
                                    0.02, 0.05, 1, one, one, None)
    assert rc == -1 and b"samples" in lib.sem_last_error()
