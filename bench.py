#!/usr/bin/env python
"""Benchmark: forward+adjoint events/hour of the elastic SEM hot path.

Workload (one "step" = one batch of events through the whole hot path):
the 40x40x20-element box (160x160x80 km, 2,099,601 GLL points, NGLL=5),
background model vp/vs/rho = 6000/3464/2700 x (1 + 0.05 g) with a seeded
8 km Gaussian random field g, "observed" data from the same model plus a
+10% Gaussian vs anomaly (radius 15 km, depth 30 km) computed once before
timing, 100 surface receivers (10x10), NSTEP 4000, dt 0.02 s.  Each event:
forward run saving the Stacey boundary store, FP64 L2 waveform misfit and
adjoint sources on the device, adjoint + backward run with rho/mu/kappa
kernel accumulation, FP64 cross-event kernel sum.  Events have seeded
random moment tensors, depths 5-40 km and Ricker f0 in 0.5-1.5 Hz.

Lines printed (rank 0, one JSON line):
  value   events/hour of the batched path (events of a batch share every
          launch; FP16 per-face-scaled boundary store; CUDA graphs), device
          resident inputs, CUDA-event timed, max over ranks
  e2e     the same through the public API from pinned host buffers: sources
          and receivers set from the host, observed data H2D, kernels and
          seismograms D2H inside the timed region
  plain   one event per launch (FP32 boundary store, step-by-step launches)
`--impl reference` times the CPU restatement of the path (OpenMP, all host
threads) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("fwd+adj events/hour batched+served vs plain per-event on 1 B200; "
          "p50/p99 latency")
WORKLOAD = ("medium box 40x40x20 el over 160x160x80 km (2,099,601 GLL pts), "
            "NSTEP 4000, dt 0.02 s, 100 surface receivers, fwd + L2 adjoint "
            "source + adjoint/backward with rho/mu/kappa kernels")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=2)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--events", type=int, default=32)
    p.add_argument("--nstep", type=int, default=4000)
    p.add_argument("--mesh", default="medium")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-smooth", action="store_true",
                   help="skip the kernel-smoothing leg")
    p.add_argument("--e2e-steps", type=int, default=1)
    p.add_argument("--store", default="fp16", choices=["fp16", "fp32"])
    p.add_argument("--served-requests", type=int, default=128)
    p.add_argument("--served-mixed", type=int, default=48,
                   help="requests of the mixed served stream (two meshes, forward "
                        "and forward+adjoint, record lengths NSTEP/4 .. NSTEP); 0 skips it")
    p.add_argument("--mixed-policy", default="lane", choices=["lane", "group"],
                   help="admission policy of the mixed stream's batched servers")
    p.add_argument("--accuracy-steps", type=int, default=600,
                   help="record length of the after-timing accuracy check against the "
                        "FP64 oracle (0 skips it)")
    p.add_argument("--serve-requests", type=int, default=200,
                   help="--workload serve: requests of the stream")
    p.add_argument("--workload", default="batched", choices=["batched", "large", "serve"],
                   help="batched: the headline line (medium mesh, --events per batch); "
                        "large: the 96x96x48-element layered box, 8 events, NSTEP 6000, "
                        "dt 0.015 s, FP16 store with the host-spill ring (its own line); "
                        "serve: a request stream over the small, medium and large meshes "
                        "(its own line)")
    p.add_argument("--served-load", type=float, default=1.25,
                   help="Poisson arrival rate as a fraction of batched capacity "
                        "(above 1: a saturated server, throughput-limited)")
    return p.parse_args()


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------

def make_workload(mesh_name, nev, seed):
    from specfwat_b200 import database as D
    db = D.build(mesh_name, seed=1234)
    vp, vs, rho = D.background_model(db, seed=1234)
    db_obs = db.with_model(vp, D.gaussian_vs_anomaly(db, vs), rho)
    rec = D.surface_receivers(db.box, 10)
    rng = np.random.default_rng(seed)
    box = db.box
    events = []
    for _ in range(nev):
        x = rng.uniform(0.15, 0.85) * box.lx
        y = rng.uniform(0.15, 0.85) * box.ly
        z = -rng.uniform(5000.0, 40000.0)
        events.append((x, y, z, D.random_moment_tensor(rng),
                       rng.uniform(0.5, 1.5)))
    return db, db_obs, rec, events


# ---------------------------------------------------------------------------
# clocks sampler
# ---------------------------------------------------------------------------

class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# reference arm / CPU baseline: CPU restatement of the path
# ---------------------------------------------------------------------------

def cpu_sample(db, db_obs, rec, ev, nstep_full, sample_steps, dt=0.02):
    """FP32 oracle (OpenMP, all host threads): sample_steps forward (saving
    the boundary store) + sample_steps adjoint/backward steps, extrapolated
    to nstep_full.  Returns (seconds per event, threads)."""
    from oracle.oracle import Oracle, l2_adjoint_source
    nth = os.cpu_count() or 1
    x, y, z, mt, f0 = ev
    o = Oracle(db, precision=4, nthreads=nth)
    src = Oracle.source(x, y, z, mt, f0)
    t0 = time.perf_counter()
    syn = o.forward(dt, sample_steps, src, rec, save_forward=True)
    _, adj = l2_adjoint_source(syn, np.zeros_like(syn), dt)
    o.adjoint(rec, adj)
    t = time.perf_counter() - t0
    return t * nstep_full / sample_steps, nth


def cpu_anchor():
    """One whole record timed on the CPU, not extrapolated: the small
    workload's forward run (10x10x10 elements, 68,921 points, NSTEP 2000,
    25 receivers) with the FP32 CPU restatement on all host threads."""
    from specfwat_b200 import database as D
    from oracle.oracle import Oracle
    db = D.build("small")
    rec = D.surface_receivers(db.box, 5)
    mt = D.random_moment_tensor(np.random.default_rng(1234))
    nth = os.cpu_count() or 1
    o = Oracle(db, precision=4, nthreads=nth)
    t0 = time.perf_counter()
    o.forward(0.02, 2000, Oracle.source(20000.0, 20000.0, -10000.0, mt, 1.0), rec)
    return {"workload": "small box 10x10x10 el, forward only, NSTEP 2000, 25 receivers, "
                        "FP32 CPU restatement", "seconds": time.perf_counter() - t0,
            "threads": nth, "extrapolated": False}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    db, db_obs, rec, events = make_workload(args.mesh, 1, 4321)
    sample = 40
    per_step = []
    for i in range(args.warmup + args.steps):
        s, nth = cpu_sample(db, db_obs, rec, events[0], args.nstep, sample)
        if i >= args.warmup:
            per_step.append(s)
    sec = float(np.mean(per_step))
    v = 3600.0 / sec
    cb = {"value": v, "unit": "events/hour", "cores": nth, "kind": "port",
          "sample": f"{sample} forward + {sample} adjoint/backward steps of one "
                    f"event, extrapolated to NSTEP {args.nstep}",
          "extrapolated": True, "anchor": cpu_anchor()}
    line = {"metric": METRIC, "value": v, "unit": "events/hour",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": sec * 1e3, "ms_per_step_extrapolated": True,
            "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "events_per_step": 1,
                       "reference_solver": "unavailable on this box (SPECFEM3D "
                       "submodule absent); the CPU restatement of the path is timed"},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "events/hour", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def algorithmic_bytes(nspec, nglob, nev, adjoint):
    """Per-launch algorithmic bytes of the element (forces) kernel: element
    data once (ibool, kappa, mu: 1,500 B per element), per event the
    displacement gather (12 B/point) and the acceleration read-modify-write
    (24 B/point); adjoint launches carry two fields and the mu/kappa kernel
    read-modify-write (16 B per element point)."""
    b = nspec * 1500 + nglob * nev * 36
    if adjoint:
        b += nglob * nev * 36 + nspec * 125 * nev * 16
    return b


def accuracy_block(args, S, mesh, db, rec, srcs, events, obs, E, dt, variants, stream):
    """Errors of the timed batched path against an FP64 oracle run, on a
    shortened record of the same mesh, model and events (lane 0), and the
    FP16-vs-FP32 store difference of the whole batch."""
    from oracle.oracle import Oracle, l2_adjoint_source
    NA = args.accuracy_steps
    # public variants 10, 11 and 12 share the adjoint kernel (register
    # prefetch, field pair): the forward pick then fixes both phases
    rp = (10, 11, 12)
    if variants[0] in rp and variants[1] in rp:
        kv = variants[0]
    else:
        kv = variants[0] if variants[0] == variants[1] else 0

    def run(store):
        sim = S.Simulation(mesh, NA, dt, nev=E, store=store, use_graph=True, graph_steps=50,
                           max_receivers=len(rec), kernel_variant=kv)
        sim.set_stream(stream.cuda_stream)
        sim.set_sources(srcs)
        sim.set_receivers(rec)
        sim.iterate_time(1, save_forward=True)
        seis = [sim.seismograms(e) for e in range(E)]
        for e in range(E):
            sim.measure_l2(e, obs[e][:, :, :NA])
        sim.iterate_time(3)
        k0 = sim.save_adjoint_kernels(0)
        ks = sim.sum_kernels()
        sim.close()
        return seis, k0, ks

    def rel(a, b):
        return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))

    s16, k16, ks16 = run("fp16")
    s32, k32, ks32 = run("fp32")
    t0 = time.perf_counter()
    o = Oracle(db, precision=8, nthreads=os.cpu_count() or 1)
    x, y, z, mt, f0 = events[0]
    osyn = o.forward(dt, NA, Oracle.source(x, y, z, mt, f0), rec, save_forward=True)
    _, adj = l2_adjoint_source(osyn, obs[0][:, :, :NA], dt)
    ok = o.adjoint(rec, adj)
    t_oracle = time.perf_counter() - t0
    names = ("rho", "mu", "kappa", "rhop", "beta", "alpha")
    return {
        "record_steps": NA, "lane": 0,
        "kernel_variant": kv if kv else "autotuned",
        "what": (f"the timed {E}-event batch (FP16 store, graphs) rerun on the first {NA} "
                 "steps after the timed region; lane 0 against an FP64 CPU oracle run of "
                 "the same event and observed data"),
        "seismogram_rel_l2_vs_fp64": rel(s16[0], osyn),
        "kernel_rel_l2_vs_fp64": {names[q]: rel(k16[q], ok[q]) for q in range(6)},
        "fp32_store_seismogram_rel_l2_vs_fp64": rel(s32[0], osyn),
        "fp32_store_kernel_rel_l2_vs_fp64": {names[q]: rel(k32[q], ok[q]) for q in range(3)},
        "fp16_vs_fp32_store_kernel_sum_rel_l2": {names[q]: rel(ks16[q], ks32[q])
                                                for q in range(6)},
        "tolerance": {"seismograms": 1e-4, "kernels": 1e-3},
        "oracle_seconds": t_oracle,
    }


def run_ours(args):
    import torch
    from specfwat_b200 import solver as S

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    with torch.cuda.stream(stream):
        return _run_ours(args, torch, S, dist, world, rank, local, dev, stream)


def _run_ours(args, torch, S, dist, world, rank, local, dev, stream):
    from specfwat_b200.shard import reduce_kernel_sum
    E, NS, dt = args.events, args.nstep, 0.02

    db, db_obs, rec, events = make_workload(args.mesh, E, 1000 + rank)
    srcs = [S.make_source(x, y, z, mt, f0) for (x, y, z, mt, f0) in events]

    # observed data (synthetic, before timing): batched forward on the
    # anomaly model
    def observed(sources):
        mesh_obs = S.Mesh(db_obs)
        out = []
        for c0 in range(0, len(sources), 32):
            chunk = sources[c0:c0 + 32]
            so = S.Simulation(mesh_obs, NS, dt, nev=len(chunk), use_graph=True,
                              max_receivers=len(rec))
            so.set_sources(chunk)
            so.set_receivers(rec)
            so.iterate_time(1)
            out += [so.seismograms(e).astype(np.float64) for e in range(len(chunk))]
            so.close()
        mesh_obs.close()
        return out

    obs = observed(srcs)

    mesh = S.Mesh(db)
    result = {}

    # ---- plain path: one event per launch --------------------------------
    if not args.no_plain:
        sp = S.Simulation(mesh, NS, dt, nev=1, store="fp32", use_graph=False,
                          max_receivers=len(rec))
        sp.set_stream(stream.cuda_stream)
        sp.set_sources([srcs[0]])
        sp.set_receivers(rec)
        sp.set_observed(0, obs[0])
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        for rep in range(2):   # first pass warms up
            torch.cuda.synchronize()
            t0.record(stream)
            sp.iterate_time(1, save_forward=True, synchronize=False)
            sp.measure_l2_resident(0)
            sp.iterate_time(3, synchronize=False)
            t1.record(stream)
            torch.cuda.synchronize()
        plain_ms = t0.elapsed_time(t1)
        pvar = sp.kernel_variants()
        fms = sp.time_kernels(1, 20)
        ams = sp.time_kernels(3, 20)
        sp.close()
        result["plain"] = {
            "events_per_hour": 3600e3 / plain_ms, "ms_per_event": plain_ms,
            "store": "fp32", "graphs": False,
            "kernel_variants": {"fwd": pvar[0], "adj": pvar[1]},
            "kernel_ms_fwd": dict(zip(("forces", "stacey", "points", "update"), fms)),
            "kernel_ms_adj": dict(zip(("forces", "stacey", "points", "update"), ams)),
        }

    # ---- batched path ------------------------------------------------------
    sb = S.Simulation(mesh, NS, dt, nev=E, store=args.store, use_graph=True,
                      graph_steps=50, max_receivers=len(rec))
    sb.set_stream(stream.cuda_stream)
    sb.set_sources(srcs)
    sb.set_receivers(rec)
    for e in range(E):
        sb.set_observed(e, obs[e])
    ne = db.nspec * 125
    ksum = torch.zeros((6, ne), dtype=torch.float64, device=dev)
    launches_per_step = [0]

    def step():
        n = 0
        sb.iterate_time(1, save_forward=True, synchronize=False)
        n += sb.launch_count()
        for e in range(E):
            sb.measure_l2_resident(e)
        n += E
        sb.iterate_time(3, synchronize=False)
        n += sb.launch_count()
        sb.sum_kernels_device(ksum.data_ptr())
        n += E
        if dist is not None:
            reduce_kernel_sum(ksum)
        launches_per_step[0] = n

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        step()
    t1.record(stream)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clk = clocks.stop()
    ms = t0.elapsed_time(t1)
    if dist is not None:
        tt = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    ms_per_step = ms / args.steps
    value = E * world * args.steps / (ms / 1e3) * 3600.0

    # kernel timing for the roofline (same run, further steps)
    variants = sb.kernel_variants()
    fms = sb.time_kernels(1, 20)
    ams = sb.time_kernels(3, 20)

    # ---- end to end through the public API from pinned host buffers -------
    pin_obs = [torch.from_numpy(o).pin_memory() for o in obs]
    pin_k = torch.empty((6, db.nspec, 5, 5, 5), dtype=torch.float64).pin_memory()
    pin_seis = torch.empty((E, len(rec), 3, NS), dtype=torch.float32).pin_memory()
    h2d = sum(o.numel() * 8 for o in pin_obs)
    d2h = pin_k.numel() * 8 + pin_seis.numel() * 4
    e2e_ms = []
    for _ in range(max(1, args.e2e_steps)):
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        sb.set_sources(srcs)
        sb.set_receivers(rec)
        sb.iterate_time(1, save_forward=True, synchronize=False)
        for e in range(E):
            sb.measure_l2(e, pin_obs[e].numpy())
        sb.iterate_time(3, synchronize=False)
        for e in range(E):
            sb.seismograms(e, out=pin_seis[e].numpy())
        kout = pin_k.numpy()
        sb.sum_kernels(out=kout)
        if dist is not None:
            kt = torch.from_numpy(kout.reshape(6, -1)).to(dev)
            reduce_kernel_sum(kt)
        torch.cuda.synchronize()
        e2e_ms.append((time.perf_counter() - w0) * 1e3)
    e2e = float(np.mean(e2e_ms))
    if dist is not None:
        tt = torch.tensor([e2e], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e = float(tt.item())
    sb.close()

    # ---- accuracy of the timed path against the FP64 oracle ----------------
    # The same E-event batch (same events, same element kernels, FP16 store,
    # graphs) on a record shortened to args.accuracy_steps, after the timed
    # region: lane 0 against the FP64 oracle (seismograms, six kernels), and
    # the FP16-store batch against the same batch with an FP32 store.
    accuracy = None
    if rank == 0 and args.accuracy_steps > 0:
        accuracy = accuracy_block(args, S, mesh, db, rec, srcs, events, obs, E, dt,
                                  variants, stream)

    # ---- kernel post-processing: PDE smoothing of the six summed kernels ---
    smooth = None
    if rank == 0 and not args.no_smooth:
        from specfwat_b200.postproc import smooth_sem_pde
        kf = pin_k.numpy().astype(np.float32)
        _, sst = smooth_sem_pde(mesh, kf, 10000.0, 5000.0)
        nfield = kf.shape[0]
        fpp = sst["fields_per_pass"]
        passes = -(-nfield // fpp)
        # per step and pass, each datum once: gather 4 B, scatter
        # read-modify-write 8 B, update reads dat and ddat and writes both
        # (16 B) per point and field; the volume (4 B/point) and ibool
        # (500 B/element) per pass
        sbytes = (28 * fpp + 4) * db.nglob + 500 * db.nspec
        smooth = {"fields": nfield, "sigma_h": 10000.0, "sigma_v": 5000.0,
                  "nstep": sst["nstep"], "fields_per_pass": fpp,
                  "device_ms": sst["step_ms"],
                  "us_per_field_step": sst["step_ms"] * 1e3 / (sst["nstep"] * nfield),
                  "achieved_gbs": sbytes * sst["nstep"] * passes
                                  / (sst["step_ms"] * 1e-3) / 1e9,
                  "algorithmic_bytes_per_step_pass": sbytes}

    # ---- served: continuous batching of a Poisson request stream ----------
    served = None
    if args.served_requests > 0:
        from specfwat_b200.serving import MeshServer, Request, Server, latency_stats
        NR = args.served_requests
        _, _, _, sev = make_workload(args.mesh, NR, 5000 + rank)
        ssrc = [S.make_source(x, y, z, mt, f0) for (x, y, z, mt, f0) in sev]
        sobs = observed(ssrc)
        cap = E / (ms_per_step / 1e3)            # batched capacity, events/s
        lam = args.served_load * cap
        arr = np.cumsum(np.random.default_rng(99 + rank).exponential(1.0 / lam, NR))
        arr -= arr[0]
        reqs = [Request(rid=i, mesh=args.mesh, kind="fwdadj", nstep=NS, source=ssrc[i],
                        receivers=rec, obs=sobs[i], arrival=float(arr[i]))
                for i in range(NR)]
        ksum_srv = torch.zeros((6, ne), dtype=torch.float64, device=dev)
        srv = MeshServer(args.mesh, db, slots=E, nstep_max=NS, dt=dt, store=args.store,
                         graph_steps=50, max_receivers=len(rec),
                         ksum_dev_ptr=ksum_srv.data_ptr(), policy="group",
                         max_wait=2.0)
        if dist is not None:
            dist.barrier()
        done = Server({args.mesh: srv}, quantum=100).run(reqs, timeout=3000)
        srv.close()
        st = latency_stats(done)
        served = {"requests": NR, "kind": "fwd+adj", "arrivals": "Poisson",
                  "arrival_rate_per_hour": lam * 3600.0, "slots": E,
                  "policy": "8-lane groups, admitted when full or after 2 s", **st}
        if "plain" in result:
            # the plain path serves one request at a time (FIFO) with its
            # measured per-event time, on the same arrival sequence
            svc = result["plain"]["ms_per_event"] / 1e3
            t_free, lat = 0.0, []
            for a in arr:
                start = max(a, t_free)
                t_free = start + svc
                lat.append(t_free - a)
            served["plain_fifo"] = {
                "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)),
                "events_per_hour": NR / (t_free - arr[0]) * 3600.0}

    # ---- served, mixed stream: two resident meshes, both request kinds and
    # four record lengths arriving as a Poisson stream --------------------
    served_mixed = None
    if args.served_mixed > 0 and world == 1:
        from specfwat_b200.serving import MeshServer, Request, Server, StepCosts, latency_stats
        NR = args.served_mixed
        rng = np.random.default_rng(4242)
        lengths = tuple(NS * q // 4 for q in (1, 2, 3, 4))   # 1000 .. 4000 at NSTEP 4000
        work = {}
        for name in ("small", args.mesh):
            wdb, wdb_obs, wrec, wev = make_workload(name, NR, 6000 + len(work))
            work[name] = (wdb, wdb_obs, wrec,
                          [S.make_source(x, y, z, mt, f0) for (x, y, z, mt, f0) in wev])
        picks = []
        for k in range(NR):
            name = ("small", args.mesh)[int(rng.integers(2))]
            kind = "fwd" if rng.random() < 0.6 else "fwdadj"
            picks.append((name, kind, int(rng.choice(lengths))))
        # observed data: one batched forward run of 4000 steps per mesh on
        # its anomaly model, cut to each request's record length
        obs_m = {}
        for name, (wdb, wdb_obs, wrec, wsrc) in work.items():
            ks = [k for k, p_ in enumerate(picks) if p_[0] == name and p_[1] == "fwdadj"]
            if not ks:
                continue
            mo = S.Mesh(wdb_obs)
            so = S.Simulation(mo, max(lengths), dt, nev=len(ks), use_graph=True,
                              max_receivers=len(wrec))
            so.set_sources([wsrc[k] for k in ks])
            so.set_receivers(wrec)
            so.iterate_time(1)
            for q, k in enumerate(ks):
                obs_m[k] = so.seismograms(q).astype(np.float64)
            so.close()
            mo.close()
        # device cost of each request from the batched run's per-event step
        # time, scaled by element count, record length and phase share
        per_ev_step = ms_per_step / (E * NS)
        fwd_share = sum(fms) / (sum(fms) + sum(ams))
        def cost(name, kind, ns):
            w = per_ev_step * ns * work[name][0].nspec / db.nspec
            return w * (1.0 if kind == "fwdadj" else fwd_share)
        costs = np.array([cost(*p_) for p_ in picks]) / 1e3          # seconds
        # Poisson rate: served_load times what one event at a time would
        # sustain at the batched per-event cost (requests/s)
        lam = args.served_load / costs.mean()
        arr = np.cumsum(np.random.default_rng(77).exponential(1.0 / lam, NR))
        arr -= arr[0]
        reqs = []
        for k, (name, kind, ns) in enumerate(picks):
            wdb, _, wrec, wsrc = work[name]
            reqs.append(Request(rid=k, mesh=name, kind=kind, nstep=ns, source=wsrc[k],
                                receivers=wrec,
                                obs=obs_m[k][:, :, :ns].copy() if kind == "fwdadj" else None,
                                arrival=float(arr[k])))
        servers = {name: MeshServer(name, work[name][0], slots=E, nstep_max=max(lengths),
                                    dt=dt, store=args.store, graph_steps=50,
                                    max_receivers=len(work[name][2]),
                                    policy=args.mixed_policy, max_wait=2.0)
                   for name in work}
        solo = {name: MeshServer(name, work[name][0], slots=1, nstep_max=max(lengths), dt=dt,
                                 store=args.store, graph_steps=50,
                                 max_receivers=len(work[name][2]))
                for name in work}
        # routing costs from this run's own timings: the batched step per
        # active 8-lane group and the plain one-event step, per phase,
        # scaled to each mesh by its element count
        step_costs = None
        if "plain" in result:
            pf = sum(result["plain"]["kernel_ms_fwd"].values()) / 1e3
            pa = sum(result["plain"]["kernel_ms_adj"].values()) / 1e3
            groups = max(1, E // 8)
            gf, ga = sum(fms) / 1e3 / groups, sum(ams) / 1e3 / groups
            step_costs = {}
            for name in work:
                w_ = work[name][0].nspec / db.nspec
                step_costs[name] = StepCosts(pf * w_, pa * w_, gf * w_, ga * w_)
        done = Server(servers, quantum=100, solo=solo, costs=step_costs).run(reqs, timeout=3000)
        for sv in list(servers.values()) + list(solo.values()):
            sv.close()
        st = latency_stats(done)
        served_mixed = {
            "solo_share": sum(r.server == "solo" for r in done) / len(done),
            "requests": NR, "meshes": list(work), "kinds": "60% fwd, 40% fwd+adj",
            "nstep": list(lengths), "arrivals": "Poisson",
            "arrival_rate_per_hour": lam * 3600.0,
            "policy": (("8-lane groups" if args.mixed_policy == "group" else
                        "any free lane in the fullest forward-only group")
                       + " per mesh; a one-lane server per mesh takes each request "
                       + ("predicted to finish there first (measured step costs)"
                          if step_costs else "while the batched one holds fewer than 4")),
            **st}
        if "plain" in result:
            # the plain path, one request at a time in arrival order, with
            # the plain medium fwd+adj time scaled by the same work ratios
            scale = result["plain"]["ms_per_event"] / 1e3 / cost(args.mesh, "fwdadj", NS) * 1e3
            t_free, lat = 0.0, []
            for a_, c_ in zip(arr, costs):
                start = max(a_, t_free)
                t_free = start + c_ * scale
                lat.append(t_free - a_)
            served_mixed["plain_fifo_estimate"] = {
                "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)),
                "events_per_hour": NR / (t_free - arr[0]) * 3600.0}

    nglob = db.nglob
    adj_bytes = algorithmic_bytes(db.nspec, nglob, E, True)
    fwd_bytes = algorithmic_bytes(db.nspec, nglob, E, False)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs")
    peak_src = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    achieved = adj_bytes / (ams[0] * 1e-3) / 1e9
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "roofline_traffic.json")) as f:
            tr = json.load(f)
        key = f"forces_adj_{args.mesh}_nev{E}"
        if key in tr:
            traffic = tr[key]["dram_bytes_per_launch"]
    except Exception:
        pass

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0

    cpu = None
    if world == 1 and not args.no_cpu:
        sec, nth = cpu_sample(db, db_obs, rec, events[0], NS, 20)
        cpu = {"value": 3600.0 / sec, "unit": "events/hour", "cores": nth,
               "kind": "port",
               "sample": f"20 forward + 20 adjoint/backward steps of one event "
                         f"(FP32 CPU restatement, OpenMP), extrapolated to NSTEP {NS}",
               "extrapolated": True, "anchor": cpu_anchor()}
        if smooth is not None:
            from oracle.oracle import Oracle
            o = Oracle(db, precision=4, nthreads=1)
            one = np.random.default_rng(3).standard_normal(
                (db.nspec, 5, 5, 5)).astype(np.float32)
            c0 = time.perf_counter()
            o.smooth_pde(one, 10000.0, 5000.0, 690.0, nstep=2)
            c1 = time.perf_counter()
            o.smooth_pde(one, 10000.0, 5000.0, 690.0, nstep=4)
            c2 = time.perf_counter()
            per = ((c2 - c1) - (c1 - c0)) / 2.0
            smooth["cpu_us_per_field_step"] = per * 1e6
            smooth["cpu_sample"] = ("FP32 CPU restatement of smooth.f90's loops, "
                                    "1 thread, steps 3-4 of one field")

    flops_evt_step = 29750 * db.nspec
    fp32_peak = None
    try:
        import ctypes as C
        from specfwat_b200 import _lib
        pk, pm = C.c_double(0.0), C.c_double(0.0)
        if _lib.load().sem_fp32_fma_peak(C.byref(pk), C.byref(pm)) == 0:
            fp32_peak = pk.value
    except Exception:
        fp32_peak = None
    fp32_adj = (2 * flops_evt_step + 2500 * db.nspec) * E / (ams[0] * 1e-3) / 1e12
    fp32_fwd = flops_evt_step * E / (fms[0] * 1e-3) / 1e12
    line = {
        "metric": METRIC, "value": value, "unit": "events/hour",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "events_per_step": E,
                   "path": f"batched: {E} events per launch, {args.store} "
                           "per-face-scaled boundary store, CUDA graphs of 50 steps",
                   "l2": "inputs larger than L2 (per event 151 MB of wavefields "
                         "+ 2.9 GB boundary store)",
                   "parallelism": f"events sharded over {world} GPU(s), FP64 "
                                  "kernel-sum all-reduce per step"},
        "batched": {"events_per_hour": value, "ms_per_event": ms_per_step / E,
                    "kernel_variants": {"fwd": variants[0], "adj": variants[1]},
                    "kernel_ms_fwd": dict(zip(("forces", "stacey", "points",
                                               "update"), fms)),
                    "kernel_ms_adj": dict(zip(("forces", "stacey", "points",
                                               "update"), ams))},
        "roofline": {"kernel": "k_forces (adjoint+backward, batched)",
                     "bound": "hbm", "achieved": achieved, "peak": hbm,
                     "unit": "GB/s", "frac": achieved / hbm,
                     "peak_source": peak_src, "traffic": traffic,
                     "algorithmic_bytes_per_launch": adj_bytes,
                     "fwd_achieved": fwd_bytes / (fms[0] * 1e-3) / 1e9,
                     "fp32": {"achieved_tflops_adj": fp32_adj,
                              "achieved_tflops_fwd": fp32_fwd,
                              "peak_tflops": fp32_peak,
                              "peak_source": "measured by sem_fp32_fma_peak "
                                             "(fmaf chains on every SM, best of 5)",
                              "frac_adj": fp32_adj / fp32_peak if fp32_peak else None,
                              "frac_fwd": fp32_fwd / fp32_peak if fp32_peak else None}},
        "e2e": {"value": E * world / (e2e / 1e3) * 3600.0, "unit": "events/hour",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e},
        "gpu_launches": launches_per_step[0] * args.steps,
        "clocks": clk,
    }
    if "plain" in result:
        line["plain"] = result["plain"]
    if served:
        line["served"] = served
    if smooth:
        line["smooth"] = smooth
    if served_mixed:
        line["served_mixed"] = served_mixed
    if cpu:
        line["cpu_baseline"] = cpu
    if accuracy:
        line["accuracy"] = accuracy
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def run_large(args):
    """The large workload: 96x96x48 elements over 384x384x192 km (28.6M GLL
    points), three layers with a 3% seeded perturbation, 8 events batched
    forward + adjoint, NSTEP 6000, dt 0.015 s, FP16 boundary store.  The
    store (8 x 24.9 GB) does not fit next to the wavefields in 180 GB, so
    its oldest chunks are spilled to pinned host memory during the forward
    run and fetched back during the adjoint run.  One warm-up batch of 100
    steps (autotuning, graph capture), then --steps full batches timed with
    CUDA events.  Observed data: the same events on the model with the +10%
    vs anomaly (radius 15 km, depth 30 km), made before timing."""
    import torch
    from specfwat_b200 import database as D
    from specfwat_b200 import solver as S
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    E, NS, dt = 8, args.nstep if args.nstep != 4000 else 6000, 0.015
    db = D.build("large", seed=1234)
    db_obs = db.with_model(db.vp, D.gaussian_vs_anomaly(db, db.vs), db.rho)
    rec = D.surface_receivers(db.box, 10)
    rng = np.random.default_rng(3003)
    box = db.box
    ev = [(rng.uniform(0.15, 0.85) * box.lx, rng.uniform(0.15, 0.85) * box.ly,
           -rng.uniform(5000.0, 40000.0), D.random_moment_tensor(rng), rng.uniform(0.5, 1.5))
          for _ in range(E)]
    srcs = [S.make_source(*e) for e in ev]
    mo = S.Mesh(db_obs)
    so = S.Simulation(mo, NS, dt, nev=E, use_graph=True, max_receivers=len(rec))
    so.set_sources(srcs)
    so.set_receivers(rec)
    so.iterate_time(1)
    obs = [so.seismograms(e).astype(np.float64) for e in range(E)]
    so.close()
    mo.close()
    mesh = S.Mesh(db)
    full_bytes = S._lib.load().sem_run_bytes(
        mesh.handle, S._lib.RunCfg(E, NS, dt, S._lib.SEM_STORE_FP16, 1, 50, len(rec), 0, 0))

    def batch(nstep):
        sim = S.Simulation(mesh, nstep, dt, nev=E, store="fp16", use_graph=True,
                           graph_steps=50, max_receivers=len(rec))
        sim.set_stream(stream.cuda_stream)
        sim.set_store_spill(-1)
        sim.set_sources(srcs)
        sim.set_receivers(rec)
        for e in range(E):
            sim.set_observed(e, obs[e][:, :, :nstep])
        return sim

    w = batch(100)
    w.iterate_time(1, save_forward=True)
    for e in range(E):
        w.measure_l2_resident(e)
    w.iterate_time(3)
    w.synchronize()
    variants = w.kernel_variants()
    w.close()
    ne = db.nspec * 125
    ksum = torch.zeros((6, ne), dtype=torch.float64, device=dev)
    sim = batch(NS)
    clocks = Clocks(0)
    ms = []
    launches = 0
    for _ in range(max(1, args.steps)):
        torch.cuda.synchronize()
        if not ms:
            clocks.start()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            t0.record(stream)
            sim.iterate_time(1, save_forward=True, synchronize=False)
            launches += sim.launch_count()
            for e in range(E):
                sim.measure_l2_resident(e)
            sim.iterate_time(3, synchronize=False)
            launches += sim.launch_count()
            sim.sum_kernels_device(ksum.data_ptr())
            t1.record(stream)
        torch.cuda.synchronize()
        ms.append(t0.elapsed_time(t1))
    clk = clocks.stop()
    info = sim.store_info()
    fms = sim.time_kernels(1, 10)
    ams = sim.time_kernels(3, 10)
    sim.close()
    print(f"large batch: ms {ms}, store {info}, fwd {fms}, adj {ams}", file=sys.stderr,
          flush=True)
    k = ksum.cpu().numpy()
    finite = bool(np.isfinite(k).all() and np.abs(k[:3]).max() > 0)
    mesh.close()
    ms_batch = float(np.mean(ms))
    adj_bytes = algorithmic_bytes(db.nspec, db.nglob, E, True)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs") or 6650.0
    achieved = adj_bytes / (ams[0] * 1e-3) / 1e9
    line = {
        "metric": "fwd+adj events/hour, large mesh batched", "value": E / (ms_batch / 1e3) * 3600.0,
        "unit": "events/hour", "n_gpus": 1, "steps": len(ms), "warmup": 1,
        "ms_per_step": ms_batch, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "large box 96x96x48 el over 384x384x192 km (28,607,425 GLL "
                               f"pts), 3 layers + 3 percent perturbation, NSTEP {NS}, dt "
                               "0.015 s, 100 receivers, fwd + L2 adjoint + adjoint/backward "
                               "with kernels",
                   "events_per_step": E, "store": "fp16 per-face scaled, host-spill ring",
                   "warmup": "one 100-step batch (autotune, graph capture)",
                   "l2": "inputs larger than L2"},
        "run_bytes_all_resident": int(full_bytes),
        "store": info,
        "kernel_variants": {"fwd": variants[0], "adj": variants[1]},
        "kernel_ms_fwd": dict(zip(("forces", "stacey", "points", "update"), fms)),
        "kernel_ms_adj": dict(zip(("forces", "stacey", "points", "update"), ams)),
        "roofline": {"kernel": "k_forces (adjoint+backward, batched)", "bound": "hbm",
                     "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": None,
                     "algorithmic_bytes_per_launch": adj_bytes},
        "kernel_sum_finite": finite,
        "gpu_launches": launches,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_serve(args):
    """Serving stream shaped as the workload list's: requests over the
    small, medium and large meshes (50/35/15 %), NSTEP uniform on
    1000-8000, 60 % forward-only and 40 % forward+adjoint, each with its own
    seeded source and 25 (small) or 100 receivers at random surface
    positions, arriving as a Poisson stream.  Each mesh stays resident with
    a lane-batched run (32, 32 and 8 lanes) and a one-lane run; requests go
    where they are predicted to finish first, are admitted by each mesh's
    boundary-store budget, and advance in pipelined quanta.  Reports
    events/hour over the stream's span and p50/p99 latency, beside the
    plain path (one request at a time, FIFO, each mesh's measured plain
    step costs) on the same arrivals."""
    import torch
    from specfwat_b200 import database as D
    from specfwat_b200 import solver as S
    from specfwat_b200.serving import MeshServer, Request, Server, StepCosts, latency_stats
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    torch.cuda.set_device(0)
    NR = args.serve_requests
    rng = np.random.default_rng(2026)
    # dt, lanes, receivers per side, store budget of the batched and of the
    # one-lane server: each budget holds the largest request's store (an
    # 8000-step large request needs 34 GB), and with the wavefields of all
    # six runs (about 33 GB) they stay well inside 180 GB
    spec = {"small": (0.02, 32, 5, 2e9, 1e9), "medium": (0.02, 32, 10, 20e9, 6.2e9),
            "large": (0.015, 8, 10, 70e9, 35e9)}
    dbs, obs_dbs = {}, {}
    for name in spec:
        db = D.build(name, seed=1234)
        dbs[name] = db
        obs_dbs[name] = db.with_model(db.vp, D.gaussian_vs_anomaly(db, db.vs), db.rho)
    reqs = []
    for k in range(NR):
        name = ("small", "medium", "large")[int(rng.choice(3, p=[0.5, 0.35, 0.15]))]
        kind = "fwd" if rng.random() < 0.6 else "fwdadj"
        ns = int(rng.integers(1000, 8001))
        box = dbs[name].box
        src = S.make_source(rng.uniform(0.15, 0.85) * box.lx, rng.uniform(0.15, 0.85) * box.ly,
                            -rng.uniform(0.1, 0.45) * box.lz, D.random_moment_tensor(rng),
                            rng.uniform(0.5, 1.5))
        nr = spec[name][2] ** 2
        rec = np.stack([box.x0 + rng.uniform(0.1, 0.9, nr) * box.lx,
                        box.y0 + rng.uniform(0.1, 0.9, nr) * box.ly, np.zeros(nr)], 1)
        reqs.append(Request(rid=k, mesh=name, kind=kind, nstep=ns, source=src, receivers=rec))
    # observed data of the forward+adjoint requests: batched forward runs on
    # each mesh's anomaly model, every event with its own receivers
    for name, (dt, lanes, nside, _, _) in spec.items():
        ks = [r for r in reqs if r.mesh == name and r.kind == "fwdadj"]
        if not ks:
            continue
        mo = S.Mesh(obs_dbs[name])
        for c0 in range(0, len(ks), 32 if name != "large" else 8):
            chunk = ks[c0:c0 + (32 if name != "large" else 8)]
            so = S.Simulation(mo, max(r.nstep for r in chunk), dt, nev=len(chunk),
                              use_graph=True, max_receivers=nside * nside)
            so.set_sources([r.source for r in chunk])
            for e, r in enumerate(chunk):
                so.set_receivers(r.receivers, ev=e)
            so.iterate_time(1)
            for e, r in enumerate(chunk):
                r.obs = so.seismograms(e)[:, :, :r.nstep].astype(np.float64).copy()
            so.close()
        mo.close()
    # per-mesh step costs: the plain one-event path and one active 8-lane
    # group of the batched path, forward and adjoint
    costs, plain_ms = {}, {}
    for name, (dt, lanes, nside, _, _) in spec.items():
        m = S.Mesh(dbs[name])
        rec = D.surface_receivers(dbs[name].box, nside)
        box = dbs[name].box
        src = S.make_source(0.5 * box.lx, 0.5 * box.ly, -0.2 * box.lz,
                            D.random_moment_tensor(rng), 1.0)
        per = {}
        for nev in (1, 8):
            sim = S.Simulation(m, 60, dt, nev=nev, store="fp16", max_receivers=len(rec))
            sim.set_sources([src] * nev)
            sim.set_receivers(rec)
            sim.iterate_time(1, save_forward=True)
            for e in range(nev):
                sim.measure_l2(e, np.zeros((len(rec), 3, 60)))
            sim.iterate_time(3)
            sim.time_kernels(1, 10)            # first launches load the kernels
            sim.time_kernels(3, 10)
            per[nev] = (sum(sim.time_kernels(1, 20)), sum(sim.time_kernels(3, 20)))
            sim.close()
        m.close()
        plain_ms[name] = per[1]
        costs[name] = StepCosts(per[1][0] / 1e3, per[1][1] / 1e3, per[8][0] / 1e3,
                                per[8][1] / 1e3)
    def plain_s(r):
        f, a = plain_ms[r.mesh]
        return r.nstep * (f + (a if r.kind == "fwdadj" else 0.0)) / 1e3
    work = np.array([plain_s(r) for r in reqs])
    # arrivals at the rate that keeps the plain path busy 2x over (a load the
    # batched servers absorb, a queue for the one-at-a-time path)
    lam = 2.0 / work.mean()
    arr = np.cumsum(np.random.default_rng(77).exponential(1.0 / lam, NR))
    arr -= arr[0]
    for r, a in zip(reqs, arr):
        r.arrival = float(a)
    # spatial sharing: the large and medium meshes' persistent element
    # kernels leave SMs free for the others, and the small and medium runs'
    # streams go first, so that short requests do not queue behind a large
    # mesh's kernels
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    share = {"small": (0, True), "medium": (sms - 12, True), "large": (sms - 24, False)}
    servers = {name: MeshServer(name, dbs[name], slots=spec[name][1], nstep_max=8000,
                                dt=spec[name][0], store="fp16", graph_steps=50,
                                max_receivers=spec[name][2] ** 2, store_budget=spec[name][3],
                                sm_limit=share[name][0], high_priority=share[name][1])
               for name in spec}
    solo = {name: MeshServer(name, dbs[name], slots=1, nstep_max=8000, dt=spec[name][0],
                             store="fp16", graph_steps=50, max_receivers=spec[name][2] ** 2,
                             store_budget=spec[name][4], sm_limit=share[name][0],
                             high_priority=share[name][1])
            for name in spec}
    clocks = Clocks(0)
    clocks.start()
    done = Server(servers, quantum=100, solo=solo, costs=costs).run(reqs, timeout=5400)
    clk = clocks.stop()
    for sv in list(servers.values()) + list(solo.values()):
        sv.close()
    st = latency_stats(done)
    t_free, lat = 0.0, []
    for r in sorted(reqs, key=lambda q: q.arrival):
        start = max(r.arrival, t_free)
        t_free = start + plain_s(r)
        lat.append(t_free - r.arrival)
    fifo = {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "events_per_hour": NR / (t_free - arr[0]) * 3600.0,
            "how": "each request's plain one-event time from the mesh's measured plain "
                   "step costs (FP16 store), served one at a time in arrival order"}
    by_mesh = {}
    for name in spec:
        rs = [r for r in done if r.mesh == name]
        if rs:
            lt = np.array([r.latency for r in rs])
            by_mesh[name] = {"n": len(rs), "p50_s": float(np.percentile(lt, 50)),
                             "p99_s": float(np.percentile(lt, 99)),
                             "solo_share": sum(r.server == "solo" for r in rs) / len(rs)}
    line = {
        "metric": "served fwd and fwd+adj requests/hour over three resident meshes; p50/p99 "
                  "latency", "value": st["events_per_hour"], "unit": "events/hour",
        "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
        "config": {"workload": f"{NR} Poisson requests over the small/medium/large meshes "
                               "(50/35/15 percent), NSTEP uniform 1000-8000, 60 percent "
                               "forward-only, own source and receivers per request",
                   "arrival_rate_per_hour": lam * 3600.0,
                   "lanes": {n: v[1] for n, v in spec.items()},
                   "store_budget_bytes": {n: {"batched": v[3], "one_lane": v[4]}
                                          for n, v in spec.items()}},
        "served": st, "plain_fifo": fifo, "by_mesh": by_mesh,
        "errors": sum(bool(r.error) for r in done),
        "sm_share": {n: {"sm_limit": v[0] or sms, "high_priority": v[1]} for n, v in share.items()},
        "lane_moves": sum(getattr(sv, "moves", 0) for sv in servers.values()),
        "step_costs_ms": {n: {"plain_fwd": c.plain_fwd * 1e3, "plain_adj": c.plain_adj * 1e3,
                              "group_fwd": c.group_fwd * 1e3, "group_adj": c.group_adj * 1e3}
                          for n, c in costs.items()},
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "large":
        return run_large(args)
    if args.workload == "serve":
        return run_serve(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
