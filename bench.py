"""Benchmark of the B200 SCALE-DG advection RHS (one JSON line on rank 0).

Headline workload (default): plain FP64 DG advection at 32^3 elements,
p = 7 (16,777,216 DOF), the OPT1-equivalent kernels in FMA form ("GPU"),
constant velocity (1, 0.5, 0.25), the seeded Gaussian + Fourier initial
condition, dt = 0.1 h / (p+1)^2.  A bench step is one SSP-RK3 time step
(three right-hand-side evaluations fused with their stage updates).
Metric: DOF-updates per second per RHS evaluation = Ne*Np*3*K / time.

  value  device-resident state, K steps timed with CUDA events on the
         library's stream (inputs of 537 MB > 126 MB L2, so no L2 flush).
  e2e    the same steps through the C ABI with host buffers: each step
         uploads the state q from pinned host memory, runs the step and
         reads q back into that memory, in one call (sdg_rk3_steps_host,
         which overlaps the copies with the stages chunk by chunk); the
         next step starts from the host copy.  e2e.three_calls: the same
         with sdg_set_field + sdg_rk3_steps + sdg_get_field per step.
  e2e_cal_tend  the drop-in advect3d_eq_cal_tend call (sdg_cal_tend):
         q,u,v,w(Np,NeA) in, dqdt(Np,Ne) out per RHS evaluation.
  roofline  the fused stage kernel: algorithmic bytes (40/48/48 B per DOF
         for stages 1/2/3) over its CUDA-event duration, against the
         measured HBM copy bandwidth.
  cpu_baseline  the CPU oracle (restated reference OPT1 path) on the host
         cores, a bounded sample of the same workload (rank 0, N = 1).

The default run also measures, in the same process and after the headline,
the other forms under keys of their own (each with its value, stage times,
roofline, clocks and, for the mixed form, its accuracy):
  mixed_32c_p7, mixed_16c_p15  the mixed-precision form (FP32 state and
         derivatives, FP64 RK accumulation), divergence-free velocity;
  batch_fp64, batch_mixed  the 96-instance batched ensemble (Ne per axis
         U{6..24}, p in {3,5,7,9}), CUDA-graph RK steps, autotuned tiles;
  served  a short Poisson request stream at ~80 % load (--form-requests
         requests; the served workload runs the long stream), against the
         same requests solved one at a time in plain FP64.
--forms none skips them.

Other workloads (--workload): fp64_8c_p3, mixed_32c_p7, mixed_16c_p15,
batch_fp64, batch_mixed, served, divlike_var5_32c_p7 (the five-field
derivative operator), pscan (one instance of ~16.8 M DOF per order
p = 1..15, FP64 and mixed, through the autotuned batch path) and
zslab_fp64_32c_p7 (the 32^3 p = 7 mesh split into z-slabs over the N ranks,
a halo exchange per stage; strong scaling).

--impl reference runs the reference's CPU path (the oracle restatement; the
Fortran reference cannot be compiled in this image) on all host threads, a
bounded number of RK3 steps of the same workload, and prints its own line.

Multi-GPU (torchrun, N > 1): independent replicas, one per GPU (the path
has no data exchange on one mesh per device), weak scaling, time = max over
ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "scale-dg-kernel-extraction_b200"))

from sdg_b200.workloads import (WORKLOADS, IC_SEED, batch_composition,  # noqa: E402
                                dt_for, fields_kwargs, served_stream)

METRIC = "DOF-updates/s per RHS eval"
FLAGS = {"GPU": 0, "OPT1": 1, "GENERAL": 1 | 2, "MIXED": 4}


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="fp64_32c_p7",
                    choices=sorted(WORKLOADS) + ["batch_fp64", "batch_mixed", "served",
                                                 "divlike_var5_32c_p7", "pscan",
                                                 "zslab_fp64_32c_p7"])
    ap.add_argument("--forms", default="all", choices=["all", "none"],
                    help="headline run: also measure the mixed, batched and served forms")
    ap.add_argument("--requests", type=int, default=2000,
                    help="served workload: number of requests in the stream")
    ap.add_argument("--form-requests", type=int, default=40,
                    help="the served form of the default run: requests in its stream")
    ap.add_argument("--seq-sample", type=int, default=100,
                    help="served workload: requests solved one at a time (plain FP64) "
                         "for comparison")
    ap.add_argument("--orders", default="1-15",
                    help="pscan: the orders to sweep, e.g. 1-15 or 8,9,11")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=8.0,
                    help="budget of the CPU-baseline sample")
    return ap.parse_args(argv)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Replicas:
    """One independent replica of the workload per rank (the path has no data
    exchange between meshes): a process group for the barrier around the
    timed region and the max over ranks of its duration, nothing on the data
    path.  `backend` is "nccl" on GPUs; the CPU tests drive it with "gloo"
    and device "cpu"."""

    def __init__(self, backend="nccl", device="cuda", timeout_s=120):
        self.rank, self.world, self.local = dist_env()
        self.device = device
        self.pg = None
        if self.world > 1:
            import torch.distributed as dist
            from datetime import timedelta
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
            self.pg = dist

    def barrier(self):
        if self.device == "cuda":
            import torch
            torch.cuda.synchronize()
        if self.pg:
            self.pg.barrier()

    def max(self, x):
        """Max of a float over ranks (every rank gets it)."""
        if not self.pg:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x):
        if not self.pg:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def rate(self, units, seconds):
        """Whole-job throughput: the units all ranks processed over the
        slowest rank's time."""
        return self.sum(units) / self.max(seconds)

    def close(self):
        if self.pg:
            self.pg.barrier()
            self.pg.destroy_process_group()
            self.pg = None


def measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(workload):
    """Per-launch DRAM bytes of the fused stage kernel from the committed ncu
    summary (profiles/<kernel>_<workload>.json), or None."""
    name = workload if workload.startswith("divlike") else f"tend_stage_{workload}"
    path = os.path.join(REPO, "profiles", f"{name}.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f).get("dram_bytes_per_launch")
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        time.sleep(0.25)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                mhz.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz)}


def gpu_index(local):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        try:
            return int(vis.split(",")[local])
        except (ValueError, IndexError):
            pass
    return local


def workload_config(name, world):
    """The config dict of a single-mesh workload (identical in both arms)."""
    NeX, NeY, NeZ, p, form, vel, nstep = WORKLOADS[name]
    return {"workload": name, "mesh": [NeX, NeY, NeZ], "p": p,
            "dof_per_gpu": NeX * NeY * NeZ * (p + 1) ** 3, "rhs_evals_per_step": 3,
            "dt": dt_for(max(NeX, NeY, NeZ), p),
            "velocity": vel if vel == "divfree" else list(vel), "ic_seed": IC_SEED,
            "l2": "inputs larger than L2 (no flush)",
            "parallelism": f"replicas{world}" if world > 1 else "single"}


def build_problem(name, sdg):
    NeX, NeY, NeZ, p, form, vel, nstep = WORKLOADS[name]
    ops = sdg.read_operators(p)
    mesh = sdg.mesh_setup(NeX, NeY, NeZ, p, ops.x1D)
    q, u, v, w = sdg.init_fields(mesh, **fields_kwargs(vel))
    return ops, mesh, FLAGS[form], (q, u, v, w), dt_for(max(NeX, NeY, NeZ), p)


def stage_bytes_per_dof(mixed):
    # Algorithmic bytes per DOF of stages 1..3: reads q (+ q0) + u, v, w,
    # writes q_new.  FP64: 8-byte everything; mixed: FP32 velocity and
    # stage intermediates, FP64 q0 and final q.
    if mixed:
        return [8 + 12 + 4, 4 + 12 + 8 + 4, 4 + 12 + 8 + 8]
    return [8 + 24 + 8, 8 + 24 + 8 + 8, 8 + 24 + 8 + 8]


def mixed_accuracy(sdg, ops, mesh, fields, dt, nstep):
    """Error of the mixed form after `nstep` RK3 steps against the FP64 form
    (fast FP64 GPU path, itself within 1e-12 of the oracle): relative L2,
    relative max-norm and the relative drift of the FP64 mass diagnostic."""
    q, u, v, w = fields
    lgl_w = sdg.lgl_weights(ops.x1D)
    jac = 1.0 / (8.0 * mesh.Ne)  # (dx dy dz) / 8 on the unit box
    res = {}
    for name, flags in (("f64", 0), ("mixed", sdg.FLAG_MIXED)):
        h = sdg.Handle(ops, mesh, flags)
        h.set_state(q, u, v, w)
        mass0, _ = h.diagnostics(lgl_w, jac)
        h.rk3_steps(dt, nstep)
        mass, l2 = h.diagnostics(lgl_w, jac)
        res[name] = (h.get_field(), mass0, mass)
        h.close()
    ref, mass0, mass_ref = res["f64"]
    got, _, mass_got = res["mixed"]
    d = got - ref
    return {"nstep": nstep, "against": "FP64 fast GPU path",
            "rel_l2": float(np.linalg.norm(d) / np.linalg.norm(ref)),
            "rel_maxnorm": float(np.abs(d).max() / np.abs(ref).max()),
            "mass_drift_mixed": float((mass_got - mass0) / abs(mass0)),
            "mass_drift_f64": float((mass_ref - mass0) / abs(mass0))}


def time_mesh(sdg, rep, name, steps, warmup, gidx):
    """Device-timed RK3 steps of a single-mesh workload and the per-stage
    kernel durations.  Returns the result dict and the live objects (handle,
    problem) for the end-to-end legs."""
    import torch
    ops, mesh, flags, fields, dt = build_problem(name, sdg)
    mixed = bool(flags & sdg.FLAG_MIXED)
    H = sdg.Handle(ops, mesh, flags)
    H.set_state(*fields)
    stream = torch.cuda.ExternalStream(H.stream())
    dof = mesh.Ne * mesh.Np
    H.rk3_steps(dt, warmup)
    H.synchronize()
    l0 = H.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(gidx) as clk:
        rep.barrier()
        ev0.record(stream)
        H.rk3_steps(dt, steps)
        ev1.record(stream)
        H.synchronize()
        rep.barrier()
    t = ev0.elapsed_time(ev1) * 1e-3
    launches = H.launch_count() - l0
    t_max = rep.max(t)
    value = rep.world * dof * 3 * steps / t_max
    # Per-stage kernel durations on the launching stream (roofline).
    reps = 30
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(reps)]
    for r in range(reps):
        evs[r][0].record(stream)
        for s in (1, 2, 3):
            H.rk3_stage(s, dt)
            evs[r][s].record(stream)
    H.synchronize()
    stage_ms = [statistics.median(evs[r][s - 1].elapsed_time(evs[r][s]) for r in range(reps))
                for s in (1, 2, 3)]
    bpd = stage_bytes_per_dof(mixed)
    achieved = sum(b * dof for b in bpd) / (sum(stage_ms) * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    res = {"value": value, "unit": METRIC, "ms_per_step": 1e3 * t_max / steps,
           "steps": steps, "warmup": warmup, "dtype": "f32+f64" if mixed else "f64",
           "config": workload_config(name, rep.world),
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                        "traffic": profiled_traffic(name),
                        "kernel": "tend_pipe_kernel (fused flux+volume+lift+RK stage)",
                        "stage_ms": stage_ms, "alg_bytes_per_dof": bpd},
           "clocks": clk.summary(), "gpu_launches": launches}
    return res, (H, ops, mesh, flags, fields, dt)


def cpu_baseline(workload, seconds):
    """The CPU oracle (restated reference OPT1 path) on all host threads:
    repeated tendency evaluations of the same workload for ~`seconds`."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import orc
    NeX, NeY, NeZ, p, form, vel, nstep = WORKLOADS[workload]
    ops = orc.read_operators(p)
    mesh = orc.mesh_setup(NeX, NeY, NeZ, p, ops.x1D)
    q, u, v, w = orc.init_fields(mesh, **fields_kwargs(vel))
    orc.cal_tend(orc.OPT1, q, u, v, w, ops, mesh)  # warm-up
    n, t0 = 0, time.perf_counter()
    while True:
        orc.cal_tend(orc.OPT1, q, u, v, w, ops, mesh)
        n += 1
        el = time.perf_counter() - t0
        if el > seconds or n >= 200:
            break
    dof = mesh.Ne * mesh.Np
    return {"value": dof * n / el, "unit": METRIC, "cores": orc.num_threads(), "kind": "port",
            "sample": f"{n} tendency evaluations (OPT1 order) of the {workload} "
                      f"workload, {el:.1f} s"}


def run_reference(args):
    """--impl reference: the reference's CPU path (oracle restatement) on all
    host threads, RK3 steps of the same workload; rank 0 only."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    if args.workload not in WORKLOADS:
        print(json.dumps({"impl": "reference", "unavailable":
                          f"the reference has no {args.workload} form (one mesh per "
                          "process, FP64 only)"}), flush=True)
        return
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import orc
    NeX, NeY, NeZ, p, form, vel, nstep = WORKLOADS[args.workload]
    ops = orc.read_operators(p)
    mesh = orc.mesh_setup(NeX, NeY, NeZ, p, ops.x1D)
    q, u, v, w = orc.init_fields(mesh, **fields_kwargs(vel))
    dt = dt_for(max(NeX, NeY, NeZ), p)
    # Bounded sample: at most ~90 s of timed CPU work.
    t0 = time.perf_counter()
    orc.run_rk3(orc.OPT1, q, u, v, w, ops, mesh, dt, max(1, min(args.warmup, 3)))
    t_step = (time.perf_counter() - t0) / max(1, min(args.warmup, 3))
    k = max(1, min(args.steps, int(90.0 / max(t_step, 1e-6))))
    _, times = orc.run_rk3(orc.OPT1, q, u, v, w, ops, mesh, dt, k)
    dof = mesh.Ne * mesh.Np
    val = dof * 3 * k / times[0]
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": METRIC,
        "n_gpus": args.gpus, "steps": k, "warmup": args.warmup,
        "ms_per_step": 1e3 * times[0] / k, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "evaltype": "OPT1 (CPU, OpenMP)",
        "config": workload_config(args.workload, args.gpus),
        "cpu_baseline": {"value": val, "unit": METRIC, "cores": orc.num_threads(),
                         "kind": "port",
                         "sample": f"{k} of {args.steps} requested SSP-RK3 steps of the "
                                   f"{args.workload} workload (restated reference OPT1 "
                                   "path; the Fortran reference cannot be compiled here)"},
        "e2e": {"value": val, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Batched ensemble and served stream
# ---------------------------------------------------------------------------
class BatchFields:
    """Host fields of the batched composition, generated once and shared by
    the FP64 and mixed batches."""

    def __init__(self, sdg):
        self.comp = batch_composition()
        self.ops = {p: sdg.read_operators(p) for p in sorted({c["p"] for c in self.comp})}
        self.fields = []
        for it in self.comp:
            vel = tuple(sdg.random_velocity(it["seed"]))
            self.fields.append(sdg.box_fields(it["ne"], it["ne"], it["ne"], it["p"],
                                              self.ops[it["p"]].x1D, ic_kind=1,
                                              seed=it["seed"], vel_kind=0, vel=vel))


def time_batch(sdg, rep, mixed, steps, warmup, gidx, bf):
    """K RK3 steps of the 96-instance ensemble (graph replays)."""
    b = sdg.Batch(sdg.FLAG_MIXED if mixed else 0)
    for it, f in zip(bf.comp, bf.fields):
        b.add(it["ne"], it["ne"], it["ne"], it["p"], bf.ops[it["p"]], *f, it["dt"])
    b.commit(autotune=True)
    b.run(warmup)
    info0 = b.info()
    with ClockSampler(gidx) as clk:
        rep.barrier()
        b.run(steps)
        rep.barrier()
    info = b.info()
    b.close()
    t = info["run_s"] - info0["run_s"]
    dof = info["dof"]
    value = rep.rate(dof * 3 * steps, t)
    t = rep.max(t)
    bpd = stage_bytes_per_dof(mixed)
    achieved = dof * sum(bpd) * steps / t / 1e9
    peak, peak_kind = measured_peaks()
    gdof = {}
    for it in bf.comp:
        gdof[it["p"]] = gdof.get(it["p"], 0) + it["ne"] ** 3 * (it["p"] + 1) ** 3
    names = {1: "block", 2: "pipe", 3: "block8", 4: "split"}
    groups = []
    for g in info["groups"]:
        ms = {"pipe": g["ms_pipe"], "block": g["ms_block"], "block8": g["ms_block8"],
              "split": g["ms_split"]}
        chosen = ms[names.get(g["variant"], "pipe")]
        gb = gdof[g["p"]] * bpd[1] / (chosen * 1e-3) / 1e9 if chosen > 0 else None
        groups.append({"p": g["p"], "dof": gdof[g["p"]], "tiles": g["tiles"],
                       "variant": names.get(g["variant"], str(g["variant"])),
                       "stage2_ms": {k: round(v, 4) for k, v in ms.items() if v > 0},
                       "stage2_frac": gb / peak if gb else None})
    return {"value": value, "unit": METRIC, "ms_per_step": 1e3 * t / steps, "steps": steps,
            "warmup": warmup, "dtype": "f32+f64" if mixed else "f64",
            "config": {"workload": "batch_mixed" if mixed else "batch_fp64",
                       "instances": len(bf.comp), "dof_total": dof,
                       "ne_per_axis": "U{6..24}", "p": [3, 5, 7, 9], "nstep": 100,
                       "l2": "inputs larger than L2 (no flush)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                         "kernel": "tend_pipe_kernel, batched tile tables",
                         "alg_bytes_per_dof": bpd, "groups": groups},
            "clocks": clk.summary(),
            "gpu_launches": 3 * len(info["groups"]) * steps}


def time_served(sdg, rep, nreq, seq_sample, gidx):
    """Poisson request stream at ~80 % load against the serving loop.  The
    arrival rate comes from one-at-a-time plain FP64 solves (each request
    alone on the GPU, CUDA-graph steps) of the first `seq_sample` requests.
    Each request's fields are generated ahead of its arrival by a producer
    thread (bounded look-ahead), and results are fetched as they complete,
    so the host holds only the requests in flight."""
    import queue
    reqs, rng = served_stream(nreq)
    ops = {p: sdg.read_operators(p) for p in range(3, 12)}

    def make_fields(r):
        vel = tuple(sdg.random_velocity(r["seed"]))
        return sdg.box_fields(r["ne"], r["ne"], r["ne"], r["p"], ops[r["p"]].x1D,
                              ic_kind=1, seed=r["seed"], vel_kind=0, vel=vel)

    def dof(r):
        return r["ne"] ** 3 * (r["p"] + 1) ** 3

    work = [dof(r) * 3 * r["nstep"] for r in reqs]
    # One at a time, plain FP64: each request alone in a one-instance batch.
    n_seq = min(len(reqs), seq_sample)
    t_seq, w_seq = 0.0, 0
    for r in reqs[:n_seq]:
        f = make_fields(r)
        b = sdg.Batch(0)
        b.add(r["ne"], r["ne"], r["ne"], r["p"], ops[r["p"]], *f, r["dt"])
        del f
        b.commit(autotune=False)
        b.run(1)
        i0 = b.info()["run_s"]
        b.run(r["nstep"])
        t_seq += b.info()["run_s"] - i0
        w_seq += dof(r) * 3 * r["nstep"]
        b.close()
    seq_rate = w_seq / t_seq
    lam = 0.8 * seq_rate / float(np.mean(work))   # requests per second at ~80 % load
    gaps = rng.exponential(1.0 / lam, size=len(reqs))

    ahead = queue.Queue(maxsize=24)

    def producer():
        for r in reqs:
            ahead.put((r, make_fields(r)))

    srv = sdg.Server()
    ids, late, tts, qwait = [], 0, [], []
    pending = {}
    lock = threading.Lock()
    stop = threading.Event()

    def collect(final=False):
        with lock:
            items = list(pending.items())
        for i, shape in items:
            st, qw, t = srv.poll(i)
            if st == sdg.SERVE_DONE:
                srv.result(i)
                with lock:
                    del pending[i]
                tts.append(t)
                qwait.append(qw)
            elif st == sdg.SERVE_FAILED:
                raise RuntimeError(f"served request {i} failed")

    def collector():
        while not stop.is_set():
            collect()
            time.sleep(0.005)

    threading.Thread(target=producer, daemon=True).start()
    with ClockSampler(gidx) as clk:
        rep.barrier()
        col = threading.Thread(target=collector, daemon=True)
        col.start()
        t_start = time.perf_counter()
        t_next = t_start
        for g in gaps:
            r, f = ahead.get()
            t_next += g
            d = t_next - time.perf_counter()
            if d > 0:
                time.sleep(d)
            elif d < -0.01:
                late += 1
            i = srv.submit(r["ne"], r["ne"], r["ne"], r["p"], ops[r["p"]], *f, r["dt"],
                           r["nstep"], mixed=r["mixed"])
            del f
            with lock:
                pending[i] = True
            ids.append(i)
        t_arrivals = time.perf_counter() - t_start
        srv.wait(0)
        makespan = time.perf_counter() - t_start
        stop.set()
        col.join()
    collect(final=True)
    st = srv.stats()
    srv.close()
    tts = np.array(tts)
    qwait = np.array(qwait)
    total = float(sum(work))
    value = rep.rate(total, makespan)
    makespan = rep.max(makespan)
    busy = rep.max(st["busy_s"])
    busy_rate = rep.sum(st["dof_steps"] * 3) / max(busy, 1e-9)
    bytes_step = sum(dof(r) * r["nstep"] * sum(stage_bytes_per_dof(r["mixed"])) for r in reqs)
    peak, peak_kind = measured_peaks()
    achieved = rep.sum(bytes_step) / max(busy, 1e-9) / 1e9
    seq_all = rep.sum(seq_rate)
    return {"value": value, "unit": METRIC, "ms_per_step": 1e3 * makespan / len(reqs),
            "steps": len(reqs), "warmup": 0, "dtype": "f32+f64",
            "config": {"workload": "served", "requests": len(reqs),
                       "arrival_rate_per_s": lam, "load": 0.8, "ne_per_axis": "U{8..32}",
                       "p": "U{3..11}", "nstep": "U{50..400}", "fp32_fraction":
                       float(np.mean([r["mixed"] for r in reqs]))},
            "served": {"p50_tts_s": rep.max(np.percentile(tts, 50)),
                       "p99_tts_s": rep.max(np.percentile(tts, 99)),
                       "mean_tts_s": float(tts.mean()),
                       "p50_queue_s": float(np.percentile(qwait, 50)),
                       "p99_queue_s": float(np.percentile(qwait, 99)),
                       "makespan_s": makespan, "arrivals_s": t_arrivals,
                       "late_arrivals": late, "device_busy_s": busy,
                       "throughput_busy": busy_rate,
                       "one_at_a_time_fp64": seq_all,
                       "busy_vs_one_at_a_time": busy_rate / seq_all,
                       "one_at_a_time_sample": n_seq,
                       "rk_steps_run": st["iterations"]},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                         "over": "device-busy time",
                         "kernel": "tend_pipe_kernel, batched tile tables"},
            "clocks": clk.summary()}


# ---------------------------------------------------------------------------
# Arms
# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    rep = Replicas("nccl", "cuda")
    import sdg_b200 as sdg
    gidx = gpu_index(local)

    head, (H, ops, mesh, flags, (q, u, v, w), dt) = time_mesh(
        sdg, rep, args.workload, args.steps, args.warmup, gidx)
    mixed = bool(flags & sdg.FLAG_MIXED)
    dof = mesh.Ne * mesh.Np

    # ---- e2e: RK3 steps through the C ABI with host buffers ----
    n_e2e = max(10, min(40, args.steps // 5))  # ~4 ms a call at the headline size
    NE = mesh.Np * mesh.Ne
    q_pin = torch.empty(NE, dtype=torch.float64, pin_memory=True)
    q_pin.numpy()[:] = q.reshape(-1, order="F")[:NE]
    qp = q_pin.numpy()
    H.rk3_steps_host(qp, dt, 1)  # first-use set-up (chunk tables, streams)
    qp[:] = q.reshape(-1, order="F")[:NE]
    rep.barrier()
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        H.rk3_steps_host(qp, dt, 1)
    t_e2e = rep.max(time.perf_counter() - t0)
    e2e = world * dof * 3 * n_e2e / t_e2e
    qp[:] = q.reshape(-1, order="F")[:NE]
    rep.barrier()
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        H.set_field(sdg.FIELD_Q, qp)
        H.rk3_steps(dt, 1)
        H.get_field(sdg.FIELD_Q, out=qp)
    t_e2e3 = rep.max(time.perf_counter() - t0)
    e2e3 = world * dof * 3 * n_e2e / t_e2e3

    # ---- e2e of the drop-in tendency call (FP64 handles only) ----
    e2e_ct = None
    if not mixed:
        NA = mesh.Np * mesh.NeA
        pins = [torch.empty(NA, dtype=torch.float64, pin_memory=True) for _ in range(5)]
        for pt, a in zip(pins, (q, u, v, w)):
            pt.numpy()[:] = a.reshape(-1, order="F")
        Hc = sdg.Handle(ops, mesh, flags)
        arrs = [pt.numpy().reshape(mesh.Np, mesh.NeA, order="F") for pt in pins]
        Hc.cal_tend(*arrs[:4], dqdt=arrs[4])
        n_ct = 5
        rep.barrier()
        t0 = time.perf_counter()
        for _ in range(n_ct):
            Hc.cal_tend(*arrs[:4], dqdt=arrs[4])
        t_ct = rep.max(time.perf_counter() - t0)
        e2e_ct = {"value": world * dof * n_ct / t_ct, "unit": METRIC,
                  "h2d_bytes_per_step": 4 * NA * 8, "d2h_bytes_per_step": NE * 8}
        Hc.close()
        del pins, arrs
    H.close()
    del q_pin

    accuracy = None
    if mixed:
        accuracy = mixed_accuracy(sdg, ops, mesh, (q, u, v, w), dt, 200)
    del q, u, v, w, mesh

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.workload, args.cpu_seconds)

    # ---- the other forms, same process (default run) ----
    forms = {}
    if args.forms == "all" and args.workload == "fp64_32c_p7":
        for name in ("mixed_32c_p7", "mixed_16c_p15"):
            r, (Hm, o, m, fl, fd, dtm) = time_mesh(sdg, rep, name, args.steps, args.warmup,
                                                   gidx)
            Hm.close()
            r["accuracy"] = mixed_accuracy(sdg, o, m, fd, dtm, WORKLOADS[name][6])
            r["vs_fp64_32c_p7"] = r["value"] / head["value"]
            forms[name] = r
            del Hm, o, m, fd
        bf = BatchFields(sdg)
        for mx in (False, True):
            forms["batch_mixed" if mx else "batch_fp64"] = time_batch(
                sdg, rep, mx, max(3, min(args.steps, 20)), max(3, args.warmup), gidx, bf)
        forms["batch_fp64"]["vs_fp64_32c_p7"] = forms["batch_fp64"]["value"] / head["value"]
        forms["batch_mixed"]["vs_fp64_32c_p7"] = forms["batch_mixed"]["value"] / head["value"]
        del bf
        forms["served"] = time_served(sdg, rep, args.form_requests, args.form_requests,
                                      gidx)

    if rank == 0:
        line = {
            "metric": METRIC, "value": head["value"], "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": head["dtype"], "data": "synthetic",
            "evaltype": {0: "GPU (fast FP64)", 1: "OPT1 (bit-exact)", 3: "GENERAL (bit-exact)",
                         4: "MIXED"}.get(flags, str(flags)),
            "config": head["config"],
            "roofline": head["roofline"],
            "e2e": {"value": e2e, "unit": METRIC,
                    "h2d_bytes_per_step": NE * 8, "d2h_bytes_per_step": NE * 8,
                    "api": "sdg_rk3_steps_host per step (pinned q in and out)",
                    "steps_timed": n_e2e,
                    "three_calls": {"value": e2e3, "unit": METRIC,
                                    "api": "sdg_set_field + sdg_rk3_steps + sdg_get_field"}},
            "e2e_cal_tend": e2e_ct,
            "accuracy": accuracy,
            "cpu_baseline": cpu,
            "clocks": head["clocks"],
            "gpu_launches": head["gpu_launches"],
        }
        line.update(forms)
        print(json.dumps(line), flush=True)
    rep.close()


def run_mesh_only(args):
    """A single-mesh workload other than the headline, without the forms."""
    args.forms = "none"
    run_ours(args)


def run_batch(args):
    """Batched ensemble: 96 instances, Ne/axis U{6..24}, p in {3,5,7,9},
    own seeded IC, constant velocity U[-1,1]^3; K RK3 steps of all of them."""
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    rep = Replicas("nccl", "cuda")
    import sdg_b200 as sdg
    mixed = args.workload == "batch_mixed"
    r = time_batch(sdg, rep, mixed, args.steps, args.warmup, gpu_index(local), BatchFields(sdg))
    torch.cuda.synchronize()
    rep.close()
    if rank != 0:
        return
    r["config"]["parallelism"] = f"replicas{world}" if world > 1 else "single"
    line = {"metric": METRIC, "n_gpus": world, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "data": "synthetic"}
    line.update(r)
    print(json.dumps(line), flush=True)


def run_served(args):
    """Served request stream: Poisson arrivals at ~80% load; Ne/axis
    U{8..32}, p U{3..11}, nstep U{50..400}, FP32/FP64 flag.  A one-at-a-time
    FP64 run of the first requests gives the comparison throughput.  With N
    ranks each GPU serves its own copy of the stream; the aggregate is all
    ranks' work over the slowest makespan and the percentiles are the worst
    rank's."""
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    rep = Replicas("nccl", "cuda")
    import sdg_b200 as sdg
    r = time_served(sdg, rep, args.requests, args.seq_sample, gpu_index(local))
    rep.close()
    if rank != 0:
        return
    r["config"]["parallelism"] = f"replicas{world}" if world > 1 else "single"
    line = {"metric": METRIC, "n_gpus": world, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "data": "synthetic"}
    line.update(r)
    print(json.dumps(line), flush=True)


def run_zslab(args):
    """zslab_fp64_32c_p7: the 32^3 p = 7 FP64 mesh split into z-slabs over
    the N ranks (strong scaling).  Each RK stage: the local update_halo of
    the stage input, the exchange of the boundary layers with the two
    neighbouring ranks (torch.distributed point-to-point; NCCL on GPUs) into
    the z halo slots, then the stage kernel, which reads every boundary face
    from the halo.  N = 1 runs the same path with the local periodic halo."""
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    rep = Replicas("nccl", "cuda")
    import sdg_b200 as sdg
    from sdg_b200.zslab import ZSlab
    NeX, NeY, NeZ, p = 32, 32, 32, 7
    ops = sdg.read_operators(p)
    sl = ZSlab(NeX, NeY, NeZ, p, ops.x1D, rank, world, sdg.mesh_setup)
    gpos = sdg.mesh_setup(NeX, NeY, NeZ, p, ops.x1D)
    fields = sdg.init_fields(gpos, **fields_kwargs((1.0, 0.5, 0.25)))
    del gpos
    H = sdg.Handle(ops, sl.mesh, sdg.FLAG_EXTERNAL_HALO)
    H.set_state(*(sl.local(f) for f in fields))
    del fields
    dt = dt_for(NeZ, p)
    hs = torch.cuda.ExternalStream(H.stream())
    dist = rep.pg

    def exchange(t):
        if dist is not None:
            sl.exchange(t, dist, lambda n: torch.empty(n, dtype=t.dtype, device=t.device))

    with torch.cuda.stream(hs):
        for which in (sdg.FIELD_U, sdg.FIELD_V, sdg.FIELD_W):
            exchange(H.resident_array(which))
    stage_in = [H.stage_input(s) for s in (1, 2, 3)]

    def step():
        with torch.cuda.stream(hs):
            for s in (1, 2, 3):
                H.update_halo_stage(s)
                exchange(stage_in[s - 1])
                H.rk3_stage(s, dt)

    for _ in range(args.warmup):
        step()
    H.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu_index(local)) as clk:
        rep.barrier()
        ev0.record(hs)
        for _ in range(args.steps):
            step()
        ev1.record(hs)
        H.synchronize()
        rep.barrier()
    t = rep.max(ev0.elapsed_time(ev1) * 1e-3)
    dof = NeX * NeY * NeZ * (p + 1) ** 3
    H.close()
    rep.close()
    if rank != 0:
        return
    print(json.dumps({
        "metric": METRIC, "value": dof * 3 * args.steps / t, "unit": METRIC, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "zslab_fp64_32c_p7", "mesh": [NeX, NeY, NeZ], "p": p,
                   "dof_total": dof, "slabs": world,
                   "exchange_bytes_per_stage_per_rank": 2 * NeX * NeY * (p + 1) ** 2 * 8,
                   "parallelism": f"zslab{world}"},
        "clocks": clk.summary(), "gpu_launches": 6 * args.steps}), flush=True)


def run_pscan(args):
    """Per-order map: for p = 1..15, one periodic box of ~16.8 M DOF, FP64 and
    mixed, autotuned through the batch path; K RK3 steps each.  frac uses the
    mean algorithmic bytes per stage (45.3 B/DOF FP64, 28 B/DOF mixed)."""
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    rep = Replicas("nccl", "cuda")
    import sdg_b200 as sdg
    peak, peak_kind = measured_peaks()
    names = {1: "Block", 2: "Pipe", 3: "BlockOcc", 4: "Split"}
    orders = []
    for part in args.orders.split(","):
        lo, _, hi = part.partition("-")
        orders += list(range(int(lo), int(hi or lo) + 1))
    rows = []
    for mixed in (False, True):
        for p in orders:
            nq = p + 1
            N = max(2, round((16.8e6 / nq ** 3) ** (1 / 3)))
            ops = sdg.read_operators(p)
            f = sdg.box_fields(N, N, N, p, ops.x1D, ic_kind=1, seed=7, vel_kind=0,
                               vel=(1.0, 0.5, 0.25))
            b = sdg.Batch(sdg.FLAG_MIXED if mixed else 0)
            b.add(N, N, N, p, ops, *f, dt_for(N, p))
            del f
            b.commit(autotune=True)
            b.run(max(3, args.warmup))
            i0 = b.info()
            b.run(args.steps)
            i1 = b.info()
            b.close()
            t = rep.max(i1["run_s"] - i0["run_s"])
            dof = i1["dof"]
            g = i1["groups"][0]
            bpd = sum(stage_bytes_per_dof(mixed)) / 3
            G = world * dof * 3 * args.steps / t
            rows.append({"p": p, "mixed": mixed, "mesh": N, "dof": dof,
                         "G_dof_updates_per_s": G / 1e9, "frac": G * bpd / 1e9 / peak,
                         "variant": names.get(g["variant"], g["variant"]),
                         "stage2_ms": {"pipe": g["ms_pipe"], "block": g["ms_block"],
                                       "block8": g["ms_block8"], "split": g["ms_split"]}})
    rep.close()
    if rank != 0:
        return
    print(json.dumps({"metric": f"{METRIC} per order", "unit": METRIC, "n_gpus": world,
                      "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                      "data": "synthetic", "peak": peak, "peak_source": f"{peak_kind} hbm_gbs",
                      "config": {"workload": "pscan", "dof_per_order": "~16.8 M",
                                 "velocity": [1.0, 0.5, 0.25]},
                      "per_order": rows}), flush=True)


def run_derivative(args):
    """divlike_var5_32c_p7: the five-field derivative operator
    (sdg_divlike_dev, element_operation_kernel_matvec_divlike_dirXYZ_var5_P<p>)
    on 32^3 elements at p = 7, FMA form, seeded random fields.  A step is one
    call: the x-, y- and z-derivatives of 5 x 16.8 M field values, read from
    three input arrays and written to three outputs (4.0 GB in all, no L2
    flush needed).  Metric: field values differentiated per second (each gets
    its three derivatives).  e2e: the same call with the inputs copied from
    pinned host memory and the outputs read back every step."""
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    rep = Replicas("nccl", "cuda")
    import sdg_b200 as sdg
    p, nvar, NeX = 7, 5, 32
    Ne = NeX ** 3
    ops = sdg.read_operators(p)
    Np = (p + 1) ** 3
    n = Ne * nvar * Np
    gen = torch.Generator(device="cuda").manual_seed(7 + rank)
    ins = [torch.randn(n, dtype=torch.float64, device="cuda", generator=gen) for _ in range(3)]
    outs = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(3)]
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream

    def call():
        sdg.divlike_dirXYZ_var_dev(ops.D1D, nvar, Ne, *ins, *outs, flags=0, stream=sp)

    for _ in range(args.warmup):
        call()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu_index(local)) as clk:
        rep.barrier()
        ev0.record(stream)
        for _ in range(args.steps):
            call()
        ev1.record(stream)
        torch.cuda.synchronize()
        rep.barrier()
    t = ev0.elapsed_time(ev1) * 1e-3
    t_max = rep.max(t)
    value = world * n * args.steps / t_max
    bytes_per_value = 6 * 8  # three inputs read, three outputs written
    achieved = n * bytes_per_value / (t / args.steps) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = profiled_traffic(args.workload)

    # e2e: host inputs in, host outputs back, every step
    n_e2e = max(3, min(10, args.steps // 20))
    h_in = [torch.empty(n, dtype=torch.float64, pin_memory=True) for _ in range(3)]
    h_out = [torch.empty(n, dtype=torch.float64, pin_memory=True) for _ in range(3)]
    for hi, di in zip(h_in, ins):
        hi.copy_(di)
    torch.cuda.synchronize()
    rep.barrier()
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        for hi, di in zip(h_in, ins):
            di.copy_(hi, non_blocking=True)
        call()
        for ho, do in zip(h_out, outs):
            ho.copy_(do, non_blocking=True)
        torch.cuda.synchronize()
    t_e2e = rep.max(time.perf_counter() - t0)
    e2e = world * n * n_e2e / t_e2e

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import orc
        ne_s = 2048  # sample: 1/16 of the elements
        m = ne_s * nvar * Np
        xs = [ins[k][:m].cpu().numpy() for k in range(3)]
        orc.divlike_fields(orc.OPT1, ops.D1D, nvar, ne_s, *xs)
        k, t0 = 0, time.perf_counter()
        while True:
            orc.divlike_fields(orc.OPT1, ops.D1D, nvar, ne_s, *xs)
            k += 1
            el = time.perf_counter() - t0
            if el > args.cpu_seconds or k >= 200:
                break
        cpu = {"value": m * k / el, "unit": "field values/s", "cores": orc.num_threads(),
               "kind": "port",
               "sample": f"{k} calls on {ne_s} of the {Ne} elements (OPT1 order), {el:.1f} s"}
    rep.close()
    if rank != 0:
        return
    line = {"metric": "field values differentiated/s (x, y, z derivatives each)",
            "value": value, "unit": "field values/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded normal fields)",
            "config": {"workload": args.workload, "mesh": [NeX, NeX, NeX], "p": p,
                       "fields_per_element": nvar, "values_per_gpu": n,
                       "l2": "inputs larger than L2 (no flush)",
                       "parallelism": f"replicas{world}" if world > 1 else "single"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                         "traffic": traffic, "kernel": "derivative_kernel (sdg_divlike_dev)",
                         "alg_bytes_per_value": bytes_per_value},
            "e2e": {"value": e2e, "unit": "field values/s", "h2d_bytes_per_step": 3 * n * 8,
                    "d2h_bytes_per_step": 3 * n * 8,
                    "api": "host-to-device copies + sdg_divlike_dev + device-to-host copies"},
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": args.steps}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload in ("batch_fp64", "batch_mixed"):
        run_batch(args)
    elif args.workload == "served":
        run_served(args)
    elif args.workload == "divlike_var5_32c_p7":
        run_derivative(args)
    elif args.workload == "pscan":
        run_pscan(args)
    elif args.workload == "zslab_fp64_32c_p7":
        run_zslab(args)
    elif args.workload != "fp64_32c_p7":
        run_mesh_only(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
