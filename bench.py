"""Benchmark of the B200 SCALE-DG advection RHS (one JSON line on rank 0).

Workload (default): plain FP64 DG advection at 32^3 elements, p = 7
(16,777,216 DOF), the OPT1-equivalent kernels in FMA form ("GPU"), constant
velocity (1, 0.5, 0.25), the seeded Gaussian + Fourier initial condition,
dt = 0.1 h / (p+1)^2.  A bench step is one SSP-RK3 time step (three
right-hand-side evaluations fused with their stage updates).  Metric:
DOF-updates per second per RHS evaluation = Ne*Np*3*K / time.

  value  device-resident state, K steps timed with CUDA events on the
         library's stream (inputs of 537 MB > 126 MB L2, so no L2 flush).
  e2e    the same steps through the C ABI with host buffers: each step
         uploads the state q from pinned host memory (sdg_set_field), runs
         the step (sdg_rk3_steps) and reads q back (sdg_get_field).
  e2e_cal_tend  the drop-in advect3d_eq_cal_tend call (sdg_cal_tend):
         q,u,v,w(Np,NeA) in, dqdt(Np,Ne) out per RHS evaluation.
  roofline  the fused stage kernel: algorithmic bytes (40/48/48 B per DOF
         for stages 1/2/3) over its CUDA-event duration, against the
         measured HBM copy bandwidth.
  cpu_baseline  the CPU oracle (restated reference OPT1 path) on the host
         cores, a bounded sample of the same workload (rank 0, N = 1).

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

WORKLOADS = {
    # name: (NeX, NeY, NeZ, p, flags-name, vel)
    "fp64_32c_p7": (32, 32, 32, 7, "GPU", (1.0, 0.5, 0.25)),
    "fp64_8c_p3": (8, 8, 8, 3, "GPU", (1.0, 0.5, 0.25)),
    "mixed_32c_p7": (32, 32, 32, 7, "MIXED", "divfree"),
    "mixed_16c_p15": (16, 16, 16, 15, "MIXED", "divfree"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="fp64_32c_p7",
                    choices=sorted(WORKLOADS) + ["batch_fp64", "batch_mixed", "served",
                                                 "divlike_var5_32c_p7"])
    ap.add_argument("--requests", type=int, default=200,
                    help="served workload: number of requests in the stream")
    ap.add_argument("--seq-sample", type=int, default=12,
                    help="served workload: requests solved one at a time for comparison")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="budget of the CPU-baseline sample")
    return ap.parse_args()


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


def build_problem(workload, sdg):
    NeX, NeY, NeZ, p, kind, vel = WORKLOADS[workload]
    flags = {"GPU": 0, "OPT1": sdg.FLAG_EXACT, "MIXED": sdg.FLAG_MIXED}[kind]
    ops = sdg.read_operators(p)
    mesh = sdg.mesh_setup(NeX, NeY, NeZ, p, ops.x1D)
    if vel == "divfree":
        q, u, v, w = sdg.init_fields(mesh, ic_kind=1, seed=2024, vel_kind=1)
    else:
        q, u, v, w = sdg.init_fields(mesh, ic_kind=1, seed=2024, vel_kind=0, vel=vel)
    h = 1.0 / max(NeX, NeY, NeZ)
    dt = 0.1 * h / (p + 1) ** 2
    return ops, mesh, flags, (q, u, v, w), dt


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


def cpu_baseline(workload, seconds):
    """The CPU oracle (restated reference OPT1 path) on all host threads:
    repeated tendency evaluations of the same workload for ~`seconds`."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import orc
    NeX, NeY, NeZ, p, kind, vel = WORKLOADS[workload]
    ops = orc.read_operators(p)
    mesh = orc.mesh_setup(NeX, NeY, NeZ, p, ops.x1D)
    if vel == "divfree":
        q, u, v, w = orc.init_fields(mesh, ic_kind=1, seed=2024, vel_kind=1)
    else:
        q, u, v, w = orc.init_fields(mesh, ic_kind=1, seed=2024, vel_kind=0, vel=vel)
    orc.cal_tend(orc.OPT1, q, u, v, w, ops, mesh)  # warm-up
    n, t0 = 0, time.perf_counter()
    while True:
        orc.cal_tend(orc.OPT1, q, u, v, w, ops, mesh)
        n += 1
        el = time.perf_counter() - t0
        if el > seconds or n >= 200:
            break
    dof = mesh.Ne * mesh.Np
    return {"value": dof * n / el, "unit": "DOF-updates/s per RHS eval",
            "cores": orc.num_threads(), "kind": "port",
            "sample": f"{n} tendency evaluations (OPT1 order) of the {workload} "
                      f"workload, {el:.1f} s"}


def run_reference(args):
    """--impl reference: the reference's CPU path (oracle restatement) on all
    host threads, RK3 steps of the same workload; rank 0 only."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import orc
    NeX, NeY, NeZ, p, kind, vel = WORKLOADS[args.workload]
    ops = orc.read_operators(p)
    mesh = orc.mesh_setup(NeX, NeY, NeZ, p, ops.x1D)
    if vel == "divfree":
        q, u, v, w = orc.init_fields(mesh, ic_kind=1, seed=2024, vel_kind=1)
    else:
        q, u, v, w = orc.init_fields(mesh, ic_kind=1, seed=2024, vel_kind=0, vel=vel)
    dt = 0.1 / max(NeX, NeY, NeZ) / (p + 1) ** 2
    # Bounded sample: at most ~90 s of timed CPU work.
    t0 = time.perf_counter()
    orc.run_rk3(orc.OPT1, q, u, v, w, ops, mesh, dt, max(1, min(args.warmup, 3)))
    t_step = (time.perf_counter() - t0) / max(1, min(args.warmup, 3))
    k = max(1, min(args.steps, int(90.0 / max(t_step, 1e-6))))
    _, times = orc.run_rk3(orc.OPT1, q, u, v, w, ops, mesh, dt, k)
    dof = mesh.Ne * mesh.Np
    val = dof * 3 * k / times[0]
    line = {
        "impl": "reference", "metric": "DOF-updates/s per RHS eval", "value": val,
        "unit": "DOF-updates/s per RHS eval", "n_gpus": args.gpus, "steps": k,
        "warmup": args.warmup, "ms_per_step": 1e3 * times[0] / k,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "mesh": [NeX, NeY, NeZ], "p": p,
                   "dof": dof, "evaltype": "OPT1", "nstep_timed": k},
        "cpu_baseline": {"value": val, "unit": "DOF-updates/s per RHS eval",
                         "cores": orc.num_threads(), "kind": "port",
                         "sample": f"{k} of {args.steps} requested SSP-RK3 steps of the "
                                   f"{args.workload} workload (restated reference OPT1 "
                                   "path; the Fortran reference cannot be compiled here)"},
        "e2e": {"value": val, "unit": "DOF-updates/s per RHS eval",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    rep = Replicas("nccl", "cuda")
    import sdg_b200 as sdg

    ops, mesh, flags, (q, u, v, w), dt = build_problem(args.workload, sdg)
    mixed = bool(flags & sdg.FLAG_MIXED)
    H = sdg.Handle(ops, mesh, flags)
    H.set_state(q, u, v, w)
    stream = torch.cuda.ExternalStream(H.stream())
    dof = mesh.Ne * mesh.Np

    barrier = rep.barrier
    max_over_ranks = rep.max

    # ---- warm-up ----
    H.rk3_steps(dt, args.warmup)
    H.synchronize()

    # ---- timed region: K RK3 steps, device-resident ----
    l0 = H.launch_count()
    gpu_idx = local
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        try:
            gpu_idx = int(vis.split(",")[local])
        except ValueError:
            pass
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu_idx) as clk:
        barrier()
        ev0.record(stream)
        H.rk3_steps(dt, args.steps)
        ev1.record(stream)
        H.synchronize()
        barrier()
    t = ev0.elapsed_time(ev1) * 1e-3
    launches = H.launch_count() - l0
    t_max = max_over_ranks(t)
    value = world * dof * 3 * args.steps / t_max

    # ---- per-stage kernel durations (roofline) ----
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
    alg_bytes = [b * dof for b in bpd]
    achieved = sum(alg_bytes) / (sum(stage_ms) * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = profiled_traffic(args.workload)

    # ---- e2e: RK3 steps through the C ABI with host buffers ----
    n_e2e = max(3, min(20, args.steps // 50))
    NE = mesh.Np * mesh.Ne
    q_pin = torch.empty(NE, dtype=torch.float64, pin_memory=True)
    q_pin.numpy()[:] = q.reshape(-1, order="F")[:NE]
    barrier()
    t0 = time.perf_counter()
    qp = q_pin.numpy()
    for _ in range(n_e2e):
        H.set_field(sdg.FIELD_Q, qp)
        H.rk3_steps(dt, 1)
        H.get_field(sdg.FIELD_Q, out=qp)
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    e2e = world * dof * 3 * n_e2e / t_e2e

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
        barrier()
        t0 = time.perf_counter()
        for _ in range(n_ct):
            Hc.cal_tend(*arrs[:4], dqdt=arrs[4])
        t_ct = max_over_ranks(time.perf_counter() - t0)
        e2e_ct = {"value": world * dof * n_ct / t_ct, "unit": "DOF-updates/s per RHS eval",
                  "h2d_bytes_per_step": 4 * NA * 8, "d2h_bytes_per_step": NE * 8}
        Hc.close()

    # ---- accuracy of the mixed form against FP64 after nstep steps ----
    accuracy = None
    if mixed:
        accuracy = mixed_accuracy(sdg, ops, mesh, (q, u, v, w), dt, 200)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.workload, args.cpu_seconds)

    if rank == 0:
        NeX, NeY, NeZ, p, kind, vel = WORKLOADS[args.workload]
        line = {
            "metric": "DOF-updates/s per RHS eval", "value": value,
            "unit": "DOF-updates/s per RHS eval", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if mixed else "f64", "data": "synthetic",
            "config": {"workload": args.workload, "mesh": [NeX, NeY, NeZ], "p": p,
                       "dof_per_gpu": dof, "evaltype": kind,
                       "rhs_evals_per_step": 3, "dt": dt,
                       "l2": "inputs larger than L2 (no flush)",
                       "parallelism": f"replicas{world}" if world > 1 else "single"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": f"{peak_kind} hbm_gbs",
                         "traffic": traffic,
                         "kernel": "tend_pipe_kernel (fused flux+volume+lift+RK stage)",
                         "stage_ms": stage_ms,
                         "alg_bytes_per_dof": bpd},
            "e2e": {"value": e2e, "unit": "DOF-updates/s per RHS eval",
                    "h2d_bytes_per_step": NE * 8, "d2h_bytes_per_step": NE * 8,
                    "api": "sdg_set_field + sdg_rk3_steps + sdg_get_field per step"},
            "e2e_cal_tend": e2e_ct,
            "accuracy": accuracy,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    H.close()
    rep.close()


def ensemble_instances(n, seed, ne_range, p_choices, rng_nstep=None):
    """Seeded instance list: cubic boxes Ne ~ U{ne_range}, p from p_choices,
    constant velocity U[-1,1]^3, dt = 0.1 h / (p+1)^2."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        ne = int(rng.integers(ne_range[0], ne_range[1] + 1))
        p = int(rng.choice(p_choices))
        nstep = int(rng.integers(rng_nstep[0], rng_nstep[1] + 1)) if rng_nstep else None
        out.append({"ne": ne, "p": p, "seed": 1000 + k, "nstep": nstep,
                    "dt": 0.1 / ne / (p + 1) ** 2})
    return out


def run_batch(args):
    """Batched ensemble: 96 instances, Ne/axis U{6..24}, p in {3,5,7,9},
    own seeded IC, constant velocity U[-1,1]^3; K RK3 steps of all of them."""
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    rep = Replicas("nccl", "cuda")
    import sdg_b200 as sdg
    mixed = args.workload == "batch_mixed"
    inst = ensemble_instances(96, 4, (6, 24), [3, 5, 7, 9])
    b = sdg.Batch(sdg.FLAG_MIXED if mixed else 0)
    ops = {p: sdg.read_operators(p) for p in (3, 5, 7, 9)}
    for it in inst:
        vel = tuple(sdg.random_velocity(it["seed"]))
        f = sdg.box_fields(it["ne"], it["ne"], it["ne"], it["p"], ops[it["p"]].x1D,
                           ic_kind=1, seed=it["seed"], vel_kind=0, vel=vel)
        b.add(it["ne"], it["ne"], it["ne"], it["p"], ops[it["p"]], *f, it["dt"])
    b.commit(autotune=True)
    b.run(args.warmup)
    info0 = b.info()
    with ClockSampler(local) as clk:
        rep.barrier()
        b.run(args.steps)
        rep.barrier()
    info = b.info()
    t = info["run_s"] - info0["run_s"]
    dof = info["dof"]
    value = rep.rate(dof * 3 * args.steps, t)
    t = rep.max(t)
    groups = [{k: (round(v, 4) if isinstance(v, float) else v) for k, v in g.items()}
              for g in info["groups"]]
    b.close()
    torch.cuda.synchronize()
    rep.close()
    if rank != 0:
        return
    line = {"metric": "DOF-updates/s per RHS eval", "value": value,
            "unit": "DOF-updates/s per RHS eval", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if mixed else "f64", "data": "synthetic",
            "config": {"workload": args.workload, "instances": len(inst), "dof_total": dof,
                       "ne_per_axis": "U{6..24}", "p": [3, 5, 7, 9],
                       "groups": groups,
                       "parallelism": f"replicas{world}" if world > 1 else "single"},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


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
    gpu_idx = local
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        try:
            gpu_idx = int(vis.split(",")[local])
        except ValueError:
            pass
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu_idx) as clk:
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


def run_served(args):
    """Served request stream: Poisson arrivals at ~80% load; Ne/axis
    U{8..32}, p U{3..11}, nstep U{50..400}, FP32/FP64 flag.  The stream is
    shortened to --requests requests (the full 2,000 take ~3 minutes of GPU
    time at this load); a one-at-a-time FP64 run of the first requests gives
    the comparison throughput.  With N ranks each GPU serves its own copy of
    the stream; the aggregate is all ranks' work over the slowest makespan
    and the percentiles are the worst rank's."""
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    rep = Replicas("nccl", "cuda")
    import sdg_b200 as sdg
    reqs = ensemble_instances(args.requests, 5, (8, 32), list(range(3, 12)), (50, 400))
    rng = np.random.default_rng(6)
    for r in reqs:
        r["mixed"] = bool(rng.integers(0, 2))
    ops = {p: sdg.read_operators(p) for p in range(3, 12)}
    fields = []
    for r in reqs:
        vel = tuple(sdg.random_velocity(r["seed"]))
        fields.append(sdg.box_fields(r["ne"], r["ne"], r["ne"], r["p"], ops[r["p"]].x1D,
                                     ic_kind=1, seed=r["seed"], vel_kind=0, vel=vel))
    work = [r["ne"] ** 3 * (r["p"] + 1) ** 3 * 3 * r["nstep"] for r in reqs]
    # Service-rate estimate from the one-at-a-time FP64 solves of a sample.
    n_seq = min(len(reqs), args.seq_sample)
    t_seq, w_seq = 0.0, 0
    for r, f in zip(reqs[:n_seq], fields[:n_seq]):
        m = sdg.mesh_setup(r["ne"], r["ne"], r["ne"], r["p"], ops[r["p"]].x1D)
        h = sdg.Handle(ops[r["p"]], m, 0)
        h.set_state(*f)
        h.synchronize()
        t0 = time.perf_counter()
        h.rk3_steps(r["dt"], r["nstep"])
        h.synchronize()
        t_seq += time.perf_counter() - t0
        w_seq += r["ne"] ** 3 * (r["p"] + 1) ** 3 * 3 * r["nstep"]
        h.close()
        del m
    seq_rate = w_seq / t_seq
    mean_work = float(np.mean(work))
    lam = 0.8 * seq_rate / mean_work           # requests per second at ~80% load
    gaps = rng.exponential(1.0 / lam, size=len(reqs))
    srv = sdg.Server()
    rep.barrier()
    t_start = time.perf_counter()
    ids = []
    for r, f, g in zip(reqs, fields, gaps):
        time.sleep(g)
        ids.append(srv.submit(r["ne"], r["ne"], r["ne"], r["p"], ops[r["p"]], *f,
                              r["dt"], r["nstep"], mixed=r["mixed"]))
    srv.wait(0)
    makespan = time.perf_counter() - t_start
    tts = np.array([srv.poll(i)[2] for i in ids])
    st = srv.stats()
    srv.close()
    total = float(sum(work))
    value = rep.rate(total, makespan)
    makespan = rep.max(makespan)
    p50 = rep.max(np.percentile(tts, 50))
    p99 = rep.max(np.percentile(tts, 99))
    busy = rep.max(st["busy_s"])
    busy_rate = rep.sum(st["dof_steps"] * 3) / max(busy, 1e-9)
    seq_rate = rep.sum(seq_rate)
    rep.close()
    if rank != 0:
        return
    line = {"metric": "DOF-updates/s per RHS eval", "value": value,
            "unit": "DOF-updates/s per RHS eval", "n_gpus": world, "steps": len(reqs),
            "warmup": 0, "ms_per_step": 1e3 * makespan / len(reqs),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "served", "requests": len(reqs),
                       "arrival_rate_per_s": lam, "load": 0.8,
                       "ne_per_axis": "U{8..32}", "p": "U{3..11}", "nstep": "U{50..400}",
                       "parallelism": f"replicas{world}" if world > 1 else "single"},
            "served": {"p50_tts_s": p50, "p99_tts_s": p99,
                       "mean_tts_s": float(tts.mean()), "makespan_s": makespan,
                       "device_busy_s": busy, "throughput_busy": busy_rate,
                       "one_at_a_time_fp64": seq_rate, "one_at_a_time_sample": n_seq}}
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
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
