"""The C++ host side (``specfwat_b200/host``: PrepareFWD over the C ABI).

- CPU: the test driver ``tests/host/run_case.cpp`` compiles and links
  against ``libspecfwat_host.so`` and the CUDA library, and a refused call
  (an empty database) reaches a C++ caller as ``SemError`` with the
  library's status.
- GPU: a FORWARD_ADJOINT pass of three distinct events on the mini box
  through the C++ driver gives the Python PrepareFWD's misfits,
  seismograms and kernels on the same inputs; so does a FORWARD_SAVE pass
  followed by ADJOINT_ONLY with the caller's adjoint sources, and the C++
  gradient_on_grid gives postproc.gradient_on_grid's grids. Both use the FP16 store and
  graphs; their autotuned kernels may differ, so they agree to the
  scatter-add order (about 1e-6). A refused call (an event past the batch)
  reaches the C++ caller as SemError with SEM_ERR_ARG.
"""
import os
import subprocess

import numpy as np
import pytest

from specfwat_b200 import build as B
from specfwat_b200 import database as D
from specfwat_b200 import solver as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "host", "run_case.cpp")


def compile_driver(out_dir, src=SRC, name="run_case"):
    if not os.path.exists(B.HOST_LIB):
        B.build_host()
    exe = os.path.join(out_dir, name)
    host_dir, lib_dir = os.path.dirname(B.HOST_LIB), B.HERE
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"),
           "-I", host_dir, "-I", os.path.join(ROOT, "tests", "host"), src, "-L", host_dir, "-l:libspecfwat_host.so", "-L", lib_dir,
           "-l:libsem_b200.so", f"-Wl,-rpath,{host_dir}:{lib_dir}", "-o", exe]
    subprocess.run(cmd, check=True)
    return exe


def test_driver_builds(tmp_path):
    exe = compile_driver(str(tmp_path))
    assert os.access(exe, os.X_OK)


def test_refused_call_is_a_sem_error(tmp_path):
    """No device needed: sem_prepare_mesh refuses an empty database before
    touching the GPU, and the C++ Mesh turns that into SemError(-1)."""
    exe = compile_driver(str(tmp_path), os.path.join(ROOT, "tests", "host", "refuse_mesh.cpp"),
                         "refuse_mesh")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    status, msg = r.stdout.split("\n", 1)
    assert int(status) == -1 and "nspec" in msg


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def _write_mesh(d, db):
    arrays = {
        "ibool.i32": (db.ibool, np.int32), "x.f32": (db.xstore, np.float32),
        "y.f32": (db.ystore, np.float32), "z.f32": (db.zstore, np.float32),
        "kappa.f32": (db.kappa, np.float32), "mu.f32": (db.mu, np.float32),
        "rho.f32": (db.rho, np.float32), "rho_vp.f32": (db.rho_vp, np.float32),
        "rho_vs.f32": (db.rho_vs, np.float32), "rmass.f32": (db.rmass, np.float32),
        "f_ispec.i32": (db.abs_ispec, np.int32), "f_ijk.i32": (db.abs_ijk, np.int32),
        "f_jw.f32": (db.abs_jw, np.float32), "f_n.f32": (db.abs_normal, np.float32),
    }
    for name, (a, dtype) in arrays.items():
        np.ascontiguousarray(a, dtype).tofile(os.path.join(d, name))


def _case(tmp_path, mode, seed):
    """A three-event case on the mini box written for the C++ driver."""
    d = str(tmp_path)
    db = D.build("mini")
    rec = D.surface_receivers(db.box, 3)
    nev, nstep, dt = 3, 300, 0.02
    rng = np.random.default_rng(seed)
    box = db.box
    ev = [(rng.uniform(0.3, 0.7) * box.lx, rng.uniform(0.3, 0.7) * box.ly,
           -rng.uniform(0.2, 0.5) * box.lz, D.random_moment_tensor(rng),
           rng.uniform(0.8, 1.2)) for _ in range(nev)]
    srcs = [S.make_source(*e) for e in ev]
    obs = 1e-5 * rng.standard_normal((nev, len(rec), 3, nstep))
    with open(os.path.join(d, "case.txt"), "w") as f:
        f.write(f"{db.nspec} {db.nglob} {db.nfaces} {nev} {len(rec)} {nstep} {dt!r} "
                f"{float(db.xix_regular)!r} {float(db.jacobian_regular)!r} {mode} 0.05\n")
    _write_mesh(d, db)
    arrays = {
        "sources.f64": (np.array([[s.x, s.y, s.z, s.Mrr, s.Mtt, s.Mpp, s.Mrt, s.Mrp, s.Mtp,
                                   s.f0, s.tshift] for s in srcs]), np.float64),
        "stations.f64": (rec, np.float64), "obs.f64": (obs, np.float64),
    }
    for name, (a, dtype) in arrays.items():
        np.ascontiguousarray(a, dtype).tofile(os.path.join(d, name))
    return d, db, rec, srcs, obs, nev, nstep, dt


def _results(d, db, nev, nrec, nstep):
    ne = db.nspec * 125
    mis = np.fromfile(os.path.join(d, "misfits.f64"))
    kern = np.fromfile(os.path.join(d, "kernels.f64")).reshape(nev, 6, ne)
    ksum = np.fromfile(os.path.join(d, "sum.f64")).reshape(6, ne)
    seis = np.fromfile(os.path.join(d, "seis.f32"), np.float32).reshape(nev, nrec, 3, nstep)
    status, obj = open(os.path.join(d, "errors.txt")).read().split()
    return mis, kern, ksum, seis, int(status), float(obj)


@pytest.mark.gpu
def test_cpp_prepare_fwd_matches_python(gpu, tmp_path):
    d, db, rec, srcs, obs, nev, nstep, dt = _case(tmp_path, 3, 90)
    exe = compile_driver(d)
    r = subprocess.run([exe, d], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    mis, kern, ksum, seis, status, obj = _results(d, db, nev, len(rec), nstep)
    assert status == -1
    assert obj == pytest.approx(mis.sum(), rel=1e-12)

    # the Python PrepareFWD on the same inputs
    ne = db.nspec * 125
    mesh = S.Mesh(db)
    p = S.PrepareFWD(mesh, nstep, dt, nev=nev, store="fp16", use_graph=True,
                     max_receivers=len(rec))
    p.setup(srcs, rec)
    p.simulation([obs[e] for e in range(nev)], run_mode=S.FORWARD_ADJOINT)
    py_seis = [p.sim.seismograms(e) for e in range(nev)]
    py_kern = [p.sim.save_adjoint_kernels(e).reshape(6, ne) for e in range(nev)]
    py_sum = p.sim.sum_kernels().reshape(6, ne)
    py_mis = p.misfits.copy()
    p.close()
    mesh.close()
    for e in range(nev):
        assert mis[e] == pytest.approx(py_mis[e], rel=1e-5)
        assert rel(seis[e], py_seis[e]) < 1e-5
        for q in range(6):
            assert rel(kern[e, q], py_kern[e][q]) < 1e-4, (e, q)
    for q in range(6):
        assert rel(ksum[q], py_sum[q]) < 1e-4


@pytest.mark.gpu
def test_cpp_save_then_adjoint_only(gpu, tmp_path):
    """FORWARD_SAVE, then ADJOINT_ONLY on the kept state with the caller's
    adjoint sources (synthetics - observed); an ADJOINT_ONLY pass before
    any saved forward is refused with SEM_ERR_STATE (checked in the
    driver)."""
    d, db, rec, srcs, obs, nev, nstep, dt = _case(tmp_path, 3, 91)
    exe = compile_driver(d)
    r = subprocess.run([exe, d, "save-adjoint"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    _, kern, ksum, seis, status, _ = _results(d, db, nev, len(rec), nstep)
    assert status == -1
    ne = db.nspec * 125
    mesh = S.Mesh(db)
    sim = S.Simulation(mesh, nstep, dt, nev=nev, store="fp16", use_graph=True,
                       max_receivers=len(rec))
    sim.set_sources(srcs)
    sim.set_receivers(rec)
    sim.iterate_time(1, save_forward=True)
    py_seis = [sim.seismograms(e) for e in range(nev)]
    for e in range(nev):
        sim.set_adjoint_sources(e, py_seis[e].astype(np.float64) - obs[e])
    sim.iterate_time(3)
    py_kern = [sim.save_adjoint_kernels(e).reshape(6, ne) for e in range(nev)]
    sim.close()
    mesh.close()
    for e in range(nev):
        assert rel(seis[e], py_seis[e]) < 1e-5
        for q in range(6):
            assert rel(kern[e, q], py_kern[e][q]) < 1e-4, (e, q)
    assert rel(ksum[1], np.sum([k[1] for k in py_kern], axis=0)) < 1e-4


@pytest.mark.gpu
def test_cpp_gradient_on_grid_matches_python(gpu, tmp_path):
    """The C++ gradient_on_grid (precondition, smooth, project, rhop from
    beta, taper) against postproc.gradient_on_grid on the same kernels: the
    same device calls in the same order, so they agree to the smoother's
    scatter-add order."""
    from specfwat_b200.postproc import gradient_on_grid
    d = str(tmp_path)
    db = D.build("mini")
    rng = np.random.default_rng(92)
    k6 = rng.standard_normal((6, db.nspec, 5, 5, 5))
    pre = rng.uniform(0.5, 1.5, (db.nspec, 5, 5, 5)).astype(np.float32)
    box = db.box
    x0, h, n = (0.0, 0.0, -box.lz), (1000.0, 1000.0, 1000.0), (
        int(box.lx // 1000) + 1, int(box.ly // 1000) + 1, int(box.lz // 1000) + 1)
    sig = (6000.0, 3000.0)
    tap = (1000.0, 2000.0, 1000.0, 2000.0)
    _write_mesh(d, db)
    k6.tofile(os.path.join(d, "kernels.f64"))
    pre.tofile(os.path.join(d, "precond.f32"))
    with open(os.path.join(d, "case.txt"), "w") as f:
        f.write(f"{db.nspec} {db.nglob} {db.nfaces} {float(db.xix_regular)!r} "
                f"{float(db.jacobian_regular)!r} {' '.join(map(repr, x0))} "
                f"{' '.join(map(repr, h))} {' '.join(map(str, n))} {sig[0]!r} {sig[1]!r} 1 1 "
                f"{' '.join(map(repr, tap))}\n")
    exe = compile_driver(d, os.path.join(ROOT, "tests", "host", "run_gradient.cpp"),
                         "run_gradient")
    r = subprocess.run([exe, d], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    grad = np.fromfile(os.path.join(d, "grad.f32"), np.float32).reshape((3,) + n)
    mesh = S.Mesh(db)
    ref = gradient_on_grid(mesh, db, k6, x0, h, n, *sig, precond=pre.astype(np.float64),
                           rho_scaling=True, taper=tap)
    mesh.close()
    assert np.count_nonzero(grad[1]) > 0.3 * grad[1].size
    for q in range(3):
        assert rel(grad[q], ref[q]) < 1e-5, q
