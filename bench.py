"""Throughput benchmark of the fused LBM step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: D3Q19 float32, 512^3 nodes, all faces PERIODICAL, tau = 0.6
(mu = 1/30), Taylor-Green vortex initial field (u0 = 0.05, k = 2 pi / N) --
the 512^3 D3Q19 point of the throughput sweep.  Metric: million lattice
updates per second (MLUPS), whole job.  One step = one fused kernel launch
over the lattice (20.4 GB of populations per step, far above the 126 MB L2,
so no flush is needed between steps).

For N > 1 (torchrun) every rank advances its own independent lattice
(replicas: the path has no exchange step); time = max over ranks.

``--impl reference`` times the reference itself -- funlbm 1.2.0 installed
unmodified in baseline/_ref, ``LBMD3.run_step`` through its public API -- on
the host cores (torch threads = cpu_count, as funlbm's ``set_cpu`` sets them)
on a bounded sample of the same workload (128^3 nodes, smaller when the run
would not fit a few minutes), and adds the same reference path on the GPU
(its torch code with the flow on ``cuda``) at the full size as
``reference_gpu``; under torchrun only rank 0 runs it.  funlbm imports five
helper packages that are not installable here; the project-written
stand-ins in tests/golden/_stubs replace them (none of them is on the step
path).  Without baseline/_ref the arm falls back to the oracle (numpy
restatement, "port").
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# one hardware queue per stream of the serving pool (read when CUDA starts)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

Q = 19
TAU_MU = 1.0 / 30.0
U0 = 0.05
BYTES_PER_LU = {"fp32": 2 * Q * 4, "fp16s": 2 * Q * 2, "bf16s": 2 * Q * 2, "fp64": 2 * Q * 8}
REF_DIR = os.path.join(ROOT, "baseline", "_ref")
REF_STUBS = os.path.join(ROOT, "tests", "golden", "_stubs")
FACE_NAMES = ("input", "output", "back", "forward", "bottom", "top")


def metric_name(n, storage):
    return "MLUPS (D3Q19 %s fused step, %d^3 periodic Taylor-Green)" % (storage, n)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=512, help="nodes per axis")
    ap.add_argument("--storage", default="fp32", choices=["fp32", "fp16s", "bf16s"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp16s", action="store_true",
                    help="skip the fp16s sub-object of the fp32 headline line")
    ap.add_argument("--vs-fp64", action="store_true",
                    help="with --case: run the case in fp64, fp32, fp16s and bf16s storage and "
                         "report each one's error against the fp64 run")
    ap.add_argument("--spread", default=None, choices=["claims", "tiles"],
                    help="with --case: the spreading kernels (ibm.spread)")
    ap.add_argument("--case-steps", type=int, default=None,
                    help="steps of the --vs-fp64 runs (default: the case's stated horizon)")
    ap.add_argument("--ke-errors", action="store_true",
                    help="throughput sweep's accuracy: kinetic-energy decay of the periodic "
                         "Taylor-Green vortex, D3Q13/15/19/27 x sizes x fp32/fp16s vs fp64")
    ap.add_argument("--ke-sizes", type=int, nargs="+", default=[128, 256, 512])
    ap.add_argument("--cpu-size", type=int, default=64)
    ap.add_argument("--serve", action="store_true",
                    help="run the served-stream benchmark and print its own line")
    ap.add_argument("--serve-requests", type=int, default=32)
    ap.add_argument("--serve-steps", type=int, nargs=2, default=[500, 5000])
    ap.add_argument("--serve-budget", type=float, default=160e9)
    ap.add_argument("--serve-mode", default="streams", choices=["streams", "batched"])
    ap.add_argument("--serve-particles", type=int, default=1,
                    help="0: particle-free stream (for comparison)")
    ap.add_argument("--case", default=None, choices=["sphere", "ellipsoids"],
                    help="sphere: the single-sphere free-fall workload (161x65x65 D3Q19, "
                         "walls, r = 8, rou 1.5, gl 2e-5); ellipsoids: multi-ellipsoid "
                         "sedimentation (257x129x129 D3Q27, 32 ellipsoids 6/4/4, rou 1.2, "
                         "gl 1e-5); both through LBMD3, IBM included")
    ap.add_argument("--shape", default=None,
                    help="fixed launch shape 'nodes,threads' (e.g. 2,128 or -1,256) instead of "
                         "the autotuner")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing (timing only; the data path has no collective)
# ---------------------------------------------------------------------------
def dist_setup(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(world, value):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        rows = []
        with open(self.path) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        def num(v):
            try:
                return float(v)
            except ValueError:
                return None

        power = [num(r[3]) for r in rows]
        pmax = max([p for p in power if p is not None] + [0.0])
        # samples under load: power above 40 % of the peak seen in the window
        load = [r for r, p in zip(rows, power) if p is not None and p >= 0.4 * pmax] or rows
        sm = [num(r[1]) for r in load if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in load for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples_under_load": len(load), "power_w_max": pmax}


# ---------------------------------------------------------------------------
# the measured path
# ---------------------------------------------------------------------------
def taylor_green_soa(lat, torch):
    """f0 = feq(1, u_TG) (float32 SoA) computed on the device."""
    from funlbm_b200.flow import equilibrium_soa, make_param, taylor_green_velocity

    param = make_param(Q, lat.device)
    u = taylor_green_velocity(lat.shape, U0, lat.device)
    rho = torch.ones(lat.shape + (1,), device=lat.device)
    f0 = equilibrium_soa(param, u, rho)
    del u, rho
    return f0


def run_device(args, world, rank, local):
    import torch

    from funlbm_b200.lattice import Lattice, tau_float32

    n = args.size
    shape = (n, n, n)
    lat = Lattice(Q, shape, [11000] * 6, tau_float32(TAU_MU), storage=args.storage,
                  device="cuda:%d" % local)
    f0 = taylor_green_soa(lat, torch)
    lat.init(f0)
    del f0
    if args.shape:
        shape = tuple(int(v) for v in args.shape.split(","))
        lat.set_launch_shape(*shape)
    else:
        shape, _ = lat.tune()      # launch-shape autotuner (scratch proxy lattice)
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        lat.step(None)
    stream = torch.cuda.current_stream()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.5)   # let nvidia-smi start sampling before the timed region
    ev0.record(stream)
    for _ in range(args.steps):
        lat.step(None)
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    barrier(world)
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(world, ms)
    status = lat.read_status()
    lat.release()
    del lat
    torch.cuda.empty_cache()
    return ms_max, clocks, status, shape


def run_e2e(args, world, local):
    """Same workload through the public API (LBMD3 + Config), with the initial
    populations uploaded from pinned host memory, the device status word read
    back every step, and the final density / velocity fields downloaded --
    all inside the timed region."""
    import torch

    from funlbm_b200.lattice import Lattice, tau_float32
    from funlbm_b200.lbm import LBMD3, Config

    n = args.size
    dev = "cuda:%d" % local
    tmp = Lattice(Q, (n, n, n), [11000] * 6, tau_float32(TAU_MU), device=dev, allocate=False)
    f0_dev = taylor_green_soa(tmp, torch)
    f0_host = torch.empty(f0_dev.shape, dtype=torch.float32, pin_memory=True)
    f0_host.copy_(f0_dev)
    del f0_dev, tmp
    torch.cuda.empty_cache()
    cfg = Config().from_json({
        "device": dev, "max_step": 10 ** 9, "log_per_steps": 10 ** 9,
        "file": {"per_steps": 10 ** 9},
        "flow": {"size": [n - 1] * 3, "param_type": "D3Q19", "param": {"mu": TAU_MU},
                 "precision": {"storage": args.storage},
                 "boundary": {k: {"code": "PERIODICAL"} for k in
                              ("input", "output", "back", "forward", "bottom", "top")}},
    })
    lbm = LBMD3(config=cfg)
    status_host = torch.zeros(1, dtype=torch.int32, pin_memory=True)
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    lbm.flow.init()
    lbm.flow._f.copy_(f0_host.view(Q, -1), non_blocking=True)   # H2D of the initial field
    lbm.flow.update_u_rou()
    lbm.flow.cul_equ()
    lbm.particle_swarm.init()
    for _ in range(args.steps):
        lbm.run_step(step=lbm.step)
        status_host.copy_(lbm.flow.lattice.status, non_blocking=True)   # per-step D2H
        lbm.step += 1
    rho = lbm.flow.rou.to("cpu")
    u = lbm.flow.u.to("cpu")
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    sec = max_over_ranks(world, sec)
    h2d = f0_host.numel() * 4 / args.steps
    d2h = (rho.numel() + u.numel()) * 4 / args.steps + 4
    del lbm, rho, u, f0_host
    torch.cuda.empty_cache()
    return sec, h2d, d2h


def oracle_workload(n):
    """The oracle on an n^3 sample of the workload (periodic Taylor-Green)."""
    from oracle import lbm_oracle as O

    fl = O.OracleFlow(Q, (n - 1,) * 3, TAU_MU, {k: O.PERIODICAL for k in O.FACES})
    e, w, _ = O.velocity_set(Q)
    x = np.arange(n)[:, None, None] * (2 * np.pi / n)
    y = np.arange(n)[None, :, None] * (2 * np.pi / n)
    z = np.arange(n)[None, None, :] * (2 * np.pi / n)
    ux = U0 * np.sin(x) * np.cos(y) * np.cos(z)
    uy = -U0 * np.cos(x) * np.sin(y) * np.cos(z)
    u = np.stack(np.broadcast_arrays(ux, uy, 0 * ux), -1).astype(np.float32)
    eu = (u @ e.T.astype(np.float32)) * 3
    f0 = ((1 + eu + eu * eu / 2 - 1.5 * (u * u).sum(-1, keepdims=True)) * w).astype(np.float32)
    lbm = O.OracleLBM(fl)
    lbm.init(f0)
    return lbm


# ---------------------------------------------------------------------------
# the reference itself (funlbm 1.2.0 from baseline/_ref)
# ---------------------------------------------------------------------------
def reference_available():
    return os.path.isfile(os.path.join(REF_DIR, "funlbm", "__init__.py"))


def import_reference():
    """Put baseline/_ref (and the stand-ins of funlbm's five absent helper
    packages) on the path.  Importing funlbm.lbm runs its set_cpu(), which sets
    torch's intra-op threads to cpu_count."""
    for p in (REF_STUBS, REF_DIR):
        if p not in sys.path:
            sys.path.insert(0, p)
    import funlbm.lbm  # noqa: F401


def taylor_green_feq(n, param, device):
    """f = feq(rho = 1, u_TG) as float32 [n, n, n, Q] with the reference's
    equilibrium formula (flow/d3/base.py:152-158) and its own lattice
    constants (`param`: e, w, cs of a funlbm flow), built on `device`."""
    import torch

    e, w, cs = param.e.to(device), param.w.to(device), param.cs.to(device)
    k = 2 * np.pi / n
    ax = torch.arange(n, device=device, dtype=torch.float32) * k
    x, y, z = ax[:, None, None], ax[None, :, None], ax[None, None, :]
    u = torch.stack(torch.broadcast_tensors(U0 * torch.sin(x) * torch.cos(y) * torch.cos(z),
                                            -U0 * torch.cos(x) * torch.sin(y) * torch.cos(z),
                                            torch.zeros_like(x)), -1)
    tmp = (u @ e.t()) / cs ** 2
    u2 = torch.linalg.norm(u, dim=-1, keepdim=True) ** 2 / cs ** 2 / 2
    return (1 + tmp + tmp ** 2 / 2 - u2) * w


def reference_workload(n, device, workdir):
    """funlbm's own LBMD3 on an n^3 sample of the workload.  LBMBase takes its
    device from Worker's default ("cpu") whatever the config says
    (lbm/base.py:56-84, base/work.py:41-43), so the flow is created on
    `device` with funlbm's create_flow and handed to LBMD3 (flow=...), the
    reference's own injection point.  Initialisation as the reference's
    LBMD3._init, with f replaced by the Taylor-Green equilibrium after
    FlowD3.init."""
    import_reference()
    from funlbm.flow import create_flow
    from funlbm.lbm import LBMD3, Config

    cfg = Config().from_json({
        "dt": 1, "dx": 1, "max_step": 10 ** 9,
        "file": {"per_steps": 10 ** 9, "cache_dir": workdir},
        "flow": {"size": [n - 1] * 3, "param_type": "D3Q%d" % Q, "param": {"mu": TAU_MU},
                 "boundary": {k: {"code": "PERIODICAL"} for k in FACE_NAMES}}})
    flow = create_flow(cfg.flow_config, device=device)
    lbm = LBMD3(config=cfg, flow=flow)
    lbm.flow.init()
    lbm.flow.f = taylor_green_feq(n, lbm.flow.param, device)
    lbm.flow.update_u_rou()
    lbm.flow.cul_equ()
    lbm.particle_swarm.init()
    return lbm


def reference_cpu(args, budget_s, max_steps=None):
    """funlbm on the host cores: MLUPS on the largest sample (128^3 at most)
    whose warm-up + timed steps fit `budget_s`.  Returns (line fields)."""
    import torch

    steps = args.steps if max_steps is None else min(args.steps, max_steps)
    with tempfile.TemporaryDirectory() as tmp:
        cwd = os.getcwd()
        os.chdir(tmp)          # funlbm opens its logs relative to the cwd
        try:
            n = 128
            lbm = reference_workload(n, "cpu", tmp)
            t0 = time.perf_counter()
            lbm.run_step(step=lbm.step)
            t1 = time.perf_counter() - t0
            want = (steps + args.warmup) * t1
            if want > budget_s:
                n = max(32, int(n * (budget_s / want) ** (1 / 3)) // 16 * 16)
                del lbm
                lbm = reference_workload(n, "cpu", tmp)
                lbm.run_step(step=lbm.step)
            for _ in range(args.warmup):
                lbm.step += 1
                lbm.run_step(step=lbm.step)
            t0 = time.perf_counter()
            for _ in range(steps):
                lbm.step += 1
                lbm.run_step(step=lbm.step)
            el = time.perf_counter() - t0
        finally:
            os.chdir(cwd)
    cores = torch.get_num_threads()
    return {"value": n ** 3 * steps / el / 1e6, "unit": "MLUPS", "cores": cores,
            "kind": "reference", "n": n, "steps": steps, "seconds": el,
            "sample": "funlbm 1.2.0 LBMD3.run_step (torch CPU, %d threads = cpu_count %d), %d^3 "
                      "nodes of the periodic Taylor-Green workload, %d timed steps after %d "
                      "warm-up, %.1f s" % (cores, os.cpu_count() or 0, n, steps, args.warmup, el)}


def reference_gpu(args, max_steps=5):
    """The reference's torch path with its flow on the GPU: CUDA-event MLUPS
    at the workload's size (halved until its temporaries fit in memory)."""
    import torch

    if not torch.cuda.is_available():
        return None
    n = args.size
    with tempfile.TemporaryDirectory() as tmp:
        cwd = os.getcwd()
        os.chdir(tmp)
        try:
            while n >= 64:
                try:
                    lbm = reference_workload(n, "cuda", tmp)
                    for _ in range(max(1, min(args.warmup, 3))):
                        lbm.run_step(step=lbm.step)
                        lbm.step += 1
                    steps = min(args.steps, max_steps)
                    a = torch.cuda.Event(enable_timing=True)
                    b = torch.cuda.Event(enable_timing=True)
                    torch.cuda.synchronize()
                    a.record()
                    for _ in range(steps):
                        lbm.run_step(step=lbm.step)
                        lbm.step += 1
                    b.record()
                    torch.cuda.synchronize()
                    ms = a.elapsed_time(b)
                    peak = torch.cuda.max_memory_allocated() / 1e9
                    del lbm
                    torch.cuda.empty_cache()
                    return {"value": n ** 3 * steps / (ms / 1e3) / 1e6, "unit": "MLUPS",
                            "nodes_per_axis": n, "steps": steps, "ms_per_step": ms / steps,
                            "peak_device_gb": peak,
                            "path": "funlbm 1.2.0 LBMD3.run_step, flow created on cuda "
                                    "(torch ATen kernels), CUDA events"}
                except torch.cuda.OutOfMemoryError:
                    lbm = None
                    torch.cuda.empty_cache()
                    n //= 2
        finally:
            os.chdir(cwd)
    return None


def host_threads():
    try:
        from threadpoolctl import threadpool_info

        return max([i.get("num_threads", 1) for i in threadpool_info()] + [1])
    except Exception:
        return 1


def cpu_baseline(args, seconds=12.0):
    """The reference's CPU path (funlbm from baseline/_ref) on a bounded sample
    of the workload, about `seconds` of CPU work; without baseline/_ref the
    oracle (numpy restatement of the reference's step) on a cpu_size^3
    lattice, as many steps as fit in `seconds`."""
    if reference_available():
        res = reference_cpu(args, seconds, max_steps=10)
        for k in ("n", "steps", "seconds"):
            res.pop(k, None)
        return res
    n = args.cpu_size
    lbm = oracle_workload(n)
    lbm.run(1)
    steps = 0
    t0 = time.perf_counter()
    while True:
        lbm.run(1)
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds or steps >= args.steps:
            break
    cores = host_threads()
    return {"value": n ** 3 * steps / el / 1e6, "unit": "MLUPS", "cores": cores, "kind": "port",
            "sample": "oracle (numpy restatement of the reference step), %d^3 nodes, %d steps, "
                      "%.1f s; elementwise numpy single-threaded, BLAS on %d threads"
                      % (n, steps, el, cores)}


# ---------------------------------------------------------------------------
# served stream (continuous batching) vs the same requests one by one
# ---------------------------------------------------------------------------
def make_requests(n, seed=0, steps=(500, 5000)):
    """Seeded mixed stream: grid size per axis uniform in {32, 48, ..., 192}
    (the reference's size, so size + 1 nodes: rows of odd length),
    D3Q19 / D3Q27 50/50, fp32 / fp16s 50/50, random WALL / PERIODICAL faces,
    0-8 spheres or ellipsoids of radius 4-8, steps uniform in `steps`."""
    from funlbm_b200.serve import Request

    rng = np.random.default_rng(seed)
    sizes = np.arange(32, 193, 16)
    faces = ("input", "output", "back", "forward", "bottom", "top")
    out = []
    for _ in range(n):
        dims = [int(v) for v in rng.choice(sizes, 3)]
        q = 19 if rng.random() < 0.5 else 27
        storage = "fp32" if rng.random() < 0.5 else "fp16s"
        parts = []
        for _ in range(int(rng.integers(0, 9))):
            r = int(rng.integers(4, 9))
            lo, hi = r + 3, [d - r - 4 for d in dims]
            if min(hi) <= lo:
                continue
            center = [float(rng.uniform(lo, h)) for h in hi]
            if rng.random() < 0.5:
                parts.append({"type": "sphere", "r": r, "rou": 1.2, "coord": {"center": center}})
            else:
                rot = rng.uniform(-np.pi, np.pi, 3)
                parts.append({"a": r, "b": max(2, round(0.75 * r)), "c": max(2, round(0.75 * r)),
                              "rou": 1.2, "coord": {"center": center, "alpha": float(rot[0]),
                                                    "beta": float(rot[1]), "gamma": float(rot[2])}})
        cfg = {"device": "cuda", "log_per_steps": 10 ** 9, "file": {"per_steps": 10 ** 9},
               "flow": {"size": list(dims), "param_type": "D3Q%d" % q,
                        "param": {"mu": 0.05, "gl": 1e-5}, "precision": {"storage": storage},
                        "boundary": {k: {"code": str(rng.choice(["WALL", "PERIODICAL"]))}
                                     for k in faces}},
               "particles": parts}
        out.append(Request(cfg, int(rng.integers(steps[0], steps[1] + 1))))
    return out


def run_serve(args):
    """Served stream vs one-by-one: aggregate MLUPS with every request queued
    at t = 0, p50/p99 time-to-result with Poisson arrivals at 80 % of that
    capacity, and the same requests sequentially through LBMD3.run_step."""
    import copy

    import torch

    from funlbm_b200.lbm import LBMD3, Config
    from funlbm_b200.serve import LBMServer, Request

    base = make_requests(args.serve_requests, seed=5, steps=tuple(args.serve_steps))
    if not args.serve_particles:
        for r in base:
            r.config["particles"] = []
    work = sum(r.steps * np.prod([d + 1 for d in r.config["flow"]["size"]]) for r in base)

    # sequential: each request alone through the plain FP32 path
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for r in base:
        cfg = copy.deepcopy(r.config)
        cfg["flow"]["precision"]["storage"] = "fp32"
        lbm = LBMD3(config=Config().from_json(cfg))
        lbm.init()
        for _ in range(r.steps):
            lbm.run_step(step=lbm.step)
            lbm.step += 1
        lbm.flow.rou.sum().item()
        del lbm
    seq_s = time.perf_counter() - t0
    torch.cuda.empty_cache()

    # served, saturated (everything queued at t = 0)
    server = LBMServer(budget_bytes=args.serve_budget, chunk=32, mode=args.serve_mode)
    reqs = [Request(copy.deepcopy(r.config), r.steps) for r in base]
    server.prepare(reqs)          # launch-shape classes tuned before the timed region
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    server.run(reqs, realtime=False)
    sat_s = time.perf_counter() - t0
    stats_sat = dict(server.stats)
    del server
    torch.cuda.empty_cache()

    # served, Poisson arrivals at 80 % of the saturated capacity
    rate = 0.8 * len(base) / sat_s
    rng = np.random.default_rng(11)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, len(base)))
    server = LBMServer(budget_bytes=args.serve_budget, chunk=32, mode=args.serve_mode)
    reqs = [Request(copy.deepcopy(r.config), r.steps, arrival=float(a))
            for r, a in zip(base, arrivals)]
    server.prepare(reqs)
    t0 = time.perf_counter()
    server.run(reqs, realtime=True)
    poi_s = time.perf_counter() - t0
    lat = np.array([r.latency for r in reqs])
    return {
        "requests": len(base), "lattice_updates": float(work),
        "steps_range": list(args.serve_steps),
        "served_mlups": work / sat_s / 1e6, "sequential_mlups": work / seq_s / 1e6,
        "speedup_vs_sequential": seq_s / sat_s,
        "served_s": sat_s, "sequential_s": seq_s,
        "poisson": {"rate_per_s": rate, "makespan_s": poi_s, "p50_s": float(np.percentile(lat, 50)),
                    "p99_s": float(np.percentile(lat, 99)),
                    "aggregate_mlups": work / poi_s / 1e6},
        "budget_gb": args.serve_budget / 1e9, "mode": args.serve_mode,
        "stats_saturated": stats_sat,
        "note": "sequential = each request alone through LBMD3.run_step with FP32 storage "
                "(the plain path); served = each request in its own storage (fp32 / fp16s)",
    }


def sphere_config(storage="fp32"):
    """Single-sphere free-fall: size [160, 64, 64] (161 x 65 x 65 nodes, the
    gravity axis is x), all faces WALL, mu 1/15 (tau 0.7), one sphere r = 8 at
    (130, 32, 32) with density 1.5, gl = 2e-5."""
    faces = ("input", "output", "back", "forward", "bottom", "top")
    return {"device": "cuda", "log_per_steps": 10 ** 9, "file": {"per_steps": 10 ** 9},
            "flow": {"size": [160, 64, 64], "param_type": "D3Q19",
                     "param": {"mu": 0.0666667, "gl": 2e-5}, "precision": {"storage": storage},
                     "boundary": {k: {"code": "WALL"} for k in faces}},
            "particles": [{"type": "sphere", "r": 8, "rou": 1.5,
                           "coord": {"center": [130.0, 32.0, 32.0]}}]}


def ellipsoids_config(storage="fp32", seed=0):
    """Multi-ellipsoid sedimentation: size [256, 128, 128] (257 x 129 x 129
    nodes, gravity along x), all faces WALL, D3Q27, mu 0.05 (tau 0.65), 32
    ellipsoids with semi-axes 6, 4, 4 and density 1.2, gl = 1e-5.  Centres by
    seeded rejection sampling (bounding sphere 6 plus 2 lu clearance, no
    overlap); orientations uniform (a random unit quaternion by Shoemake's
    method, passed as its rotation vector alpha / beta / gamma)."""
    rng = np.random.default_rng(seed)
    size = (256, 128, 128)
    reach = 6.0 + 2.0
    centres = []
    while len(centres) < 32:
        c = [float(rng.uniform(reach + 2.0, s - reach - 2.0)) for s in size]
        if all(np.linalg.norm(np.subtract(c, d)) >= 2.0 * reach for d in centres):
            centres.append(c)
    parts = []
    for c in centres:
        u1, u2, u3 = rng.random(3)
        qv = np.array([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2),
                       np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                       np.sqrt(u1) * np.sin(2 * np.pi * u3)])
        qw = np.sqrt(u1) * np.cos(2 * np.pi * u3)
        norm = float(np.linalg.norm(qv))
        angle = 2.0 * np.arctan2(norm, qw)
        rv = qv * (angle / norm) if norm > 0 else np.zeros(3)
        parts.append({"type": "ellipsoid", "a": 6, "b": 4, "c": 4, "rou": 1.2,
                      "coord": {"center": c, "alpha": float(rv[0]), "beta": float(rv[1]),
                                "gamma": float(rv[2])}})
    faces = ("input", "output", "back", "forward", "bottom", "top")
    return {"device": "cuda", "log_per_steps": 10 ** 9, "file": {"per_steps": 10 ** 9},
            "flow": {"size": list(size), "param_type": "D3Q27",
                     "param": {"mu": 0.05, "gl": 1e-5}, "precision": {"storage": storage},
                     "boundary": {k: {"code": "WALL"} for k in faces}},
            "particles": parts}


def run_case_sphere(args):
    """Steps of the sphere free-fall through the public API (LBMD3.run_step:
    interpolation, wall spring, rigid update, spreading, the fused step and
    the marker update), timed with CUDA events on the launching stream; then
    the same number of steps through LBMD3.run_steps, which replays them from
    captured CUDA graphs."""
    import torch

    from funlbm_b200.lbm import LBMD3, Config

    if args.case == "ellipsoids":
        cfg, label = ellipsoids_config(args.storage), "D3Q27 %s multi-ellipsoid 257x129x129"
    else:
        cfg, label = sphere_config(args.storage), "D3Q19 %s sphere free-fall 161x65x65"
    if args.spread:
        cfg["ibm"] = {"spread": args.spread}
    lbm = LBMD3(config=Config().from_json(cfg))
    lbm.init()
    for _ in range(args.warmup):
        lbm.run_step(step=lbm.step)
        lbm.step += 1
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        lbm.run_step(step=lbm.step)
        lbm.step += 1
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    # the same steps through LBMD3.run_steps: plain steps replayed from
    # captured CUDA graphs between logging / checkpoint steps
    lbm.run_steps(args.warmup)
    torch.cuda.synchronize()
    e0.record()
    lbm.run_steps(args.steps)
    e1.record()
    torch.cuda.synchronize()
    ms_graphed = e0.elapsed_time(e1) / max(args.steps, 1)
    nodes = lbm.flow.n
    p = lbm.particle_swarm.particles[0]
    return {"metric": "MLUPS (%s, IBM + rigid update)" % (label % args.storage),
            "value": nodes / (ms / 1e3) / 1e6, "unit": "MLUPS", "higher_is_better": True,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "graphed": {"value": nodes / (ms_graphed / 1e3) / 1e6, "ms_per_step": ms_graphed,
                        "how": "LBMD3.run_steps (graph_steps = 32)"},
            "config": {"workload": args.case, "nodes": nodes,
                       "markers": int(lbm.particle_swarm.struct().n_markers)},
            "particle": {"cx": [float(v) for v in p.cx.tolist()],
                         "cu": [float(v) for v in p.cu.tolist()]},
            "status": int(lbm.check_status())}


def _fields64(lbm):
    """End-of-step rho, u and every particle's cx, cu as float64 host arrays."""
    ps = lbm.particle_swarm.particles
    return {"rho": lbm.flow.rou.double().cpu().numpy(), "u": lbm.flow.u.double().cpu().numpy(),
            "cx": np.stack([p.cx.double().cpu().numpy() for p in ps]) if ps else None,
            "cu": np.stack([p.cu.double().cpu().numpy() for p in ps]) if ps else None}


def run_case_precision(args):
    """The case (--case) at its stated horizon in FP64 storage and then in
    fp32, fp16s and bf16s storage from the same seeded configuration; each
    one's error against the FP64 run: rho relative, u normalised by max|u|,
    particle position and velocity in lattice units (max over particles and
    over the checkpoints every `every` steps)."""
    import torch

    from funlbm_b200.lbm import LBMD3, Config

    horizon = {"ellipsoids": 3000, "sphere": 5000}[args.case]
    steps = args.case_steps or horizon
    every = max(1, steps // 10)
    make = ellipsoids_config if args.case == "ellipsoids" else sphere_config

    def one(storage):
        lbm = LBMD3(config=Config().from_json(make(storage)))
        lbm.init()
        traj = []
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        done = 0
        while done < steps:
            k = min(every, steps - done)
            lbm.run_steps(k)
            done += k
            ps = lbm.particle_swarm.particles
            traj.append((np.stack([p.cx.double().cpu().numpy() for p in ps]),
                         np.stack([p.cu.double().cpu().numpy() for p in ps])))
        b.record()
        torch.cuda.synchronize()
        out = _fields64(lbm)
        out["traj"] = traj
        out["ms_per_step"] = a.elapsed_time(b) / steps
        out["status"] = int(lbm.check_status())
        out["markers"] = int(lbm.particle_swarm.struct().n_markers)
        out["nodes"] = lbm.flow.n
        del lbm
        torch.cuda.empty_cache()
        return out

    ref = one("fp64")
    res = {}
    for storage in ("fp32", "fp16s", "bf16s"):
        got = one(storage)
        umax = np.abs(ref["u"]).max()
        ex = max(np.abs(g[0] - r[0]).max() for g, r in zip(got["traj"], ref["traj"]))
        eu = max(np.abs(g[1] - r[1]).max() for g, r in zip(got["traj"], ref["traj"]))
        res[storage] = {
            "rho_rel_err": float(np.abs(got["rho"] - ref["rho"]).max() / np.abs(ref["rho"]).max()),
            "u_err_of_umax": float(np.abs(got["u"] - ref["u"]).max() / umax),
            "cx_err_lu": float(ex), "cu_err_lu": float(eu),
            "ms_per_step": got["ms_per_step"], "status": got["status"]}
    return {"metric": "error vs the FP64 run of the same seed (%s, %d steps)" % (args.case, steps),
            "case": args.case, "steps": steps, "checkpoints_every": every,
            "nodes": ref["nodes"], "markers": ref["markers"],
            "fp64": {"ms_per_step": ref["ms_per_step"], "status": ref["status"],
                     "max_abs_u": float(np.abs(ref["u"]).max())},
            "errors": res}


def run_ke_errors(args, steps=200, every=20):
    """Accuracy of the throughput sweep: the periodic Taylor-Green vortex
    (u0 = 0.05, tau 0.6) for each velocity set and size, stored in fp32 and
    fp16s, against FP64 storage of the same case: the largest relative
    difference of the kinetic energy 1/2 sum rho |u|^2 over the samples every
    `every` steps, and the final rho / u errors."""
    import torch

    from funlbm_b200.lbm import LBMD3, Config

    def one(q, n, storage):
        faces = ("input", "output", "back", "forward", "bottom", "top")
        cfg = {"device": "cuda", "log_per_steps": 10 ** 9, "file": {"per_steps": 10 ** 9},
               "flow": {"size": [n - 1] * 3, "param_type": "D3Q%d" % q,
                        "param": {"mu": TAU_MU}, "precision": {"storage": storage},
                        "init_field": {"type": "taylor_green", "u0": U0},
                        "boundary": {k: {"code": "PERIODICAL"} for k in faces}}}
        lbm = LBMD3(config=Config().from_json(cfg))
        lbm.init()
        ke = []
        for _ in range(steps // every):
            lbm.run_steps(every)
            u = lbm.flow.u.double()
            rho = lbm.flow.rou.double()
            ke.append(float(0.5 * (rho * (u * u).sum(-1, keepdim=True)).sum()))
        out = (np.array(ke), lbm.flow.rou.double().cpu().numpy(), lbm.flow.u.double().cpu().numpy())
        del lbm, u, rho
        torch.cuda.empty_cache()
        return out

    rows = []
    for n in args.ke_sizes:
        for q in (13, 15, 19, 27):
            try:
                ref = one(q, n, "fp64")
                for storage in ("fp32", "fp16s"):
                    ke, rho, u = one(q, n, storage)
                    rows.append({"q": q, "n": n, "storage": storage, "steps": steps,
                                 "ke_rel_err": float(np.abs(ke - ref[0]).max() / ref[0].min()),
                                 "ke_decay": float(1 - ref[0][-1] / ref[0][0]),
                                 "rho_rel_err": float(np.abs(rho - ref[1]).max()),
                                 "u_err_of_umax": float(np.abs(u - ref[2]).max()
                                                        / np.abs(ref[2]).max())})
                del ref
            except torch.cuda.OutOfMemoryError:
                torch.cuda.empty_cache()
                rows.append({"q": q, "n": n, "skipped": "device memory"})
    return {"metric": "kinetic-energy decay error vs FP64 (periodic Taylor-Green, tau 0.6)",
            "rows": rows}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(args):
    """DRAM bytes per lattice update of the step kernel from a committed ncu
    capture (profiles/traffic.json), scaled to this lattice; None if absent."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as fh:
            data = json.load(fh)
        key = "k_step_q%d_%s" % (Q, args.storage)
        return float(data[key]["bytes_per_node"]) * args.size ** 3
    except (OSError, KeyError, ValueError):
        return None


def main_reference(args, world, rank):
    """Reference arm: funlbm itself on the host cores (each step one run_step
    of a bounded sample of the workload), plus the same path on the GPU as
    reference_gpu; the oracle port when baseline/_ref is absent."""
    if rank != 0:
        return
    if reference_available():
        cpu = reference_cpu(args, budget_s=150.0)
        value, n = cpu.pop("value"), cpu.pop("n")
        steps, el = cpu.pop("steps"), cpu.pop("seconds")
        line = {
            "impl": "reference", "metric": metric_name(args.size, "fp32"), "value": value,
            "unit": "MLUPS", "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * el / max(steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (Taylor-Green vortex initial field, u0=0.05)",
            "config": {"workload": "D3Q19 fp32, all faces periodic, tau 0.6, Taylor-Green u0=0.05;"
                                   " CPU sample %d^3 of the %d^3 workload" % (n, args.size),
                       "sample_nodes": n ** 3},
            "cpu_baseline": dict(cpu, value=value, unit="MLUPS"),
            "e2e": {"value": value, "unit": "MLUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
        try:
            line["reference_gpu"] = reference_gpu(args)
        except Exception as exc:        # the CPU figure stands on its own
            line["reference_gpu"] = {"unavailable": "%s: %s" % (type(exc).__name__, exc)}
        print(json.dumps(line), flush=True)
        return
    n = args.cpu_size
    lbm = oracle_workload(n)
    for _ in range(args.warmup):
        lbm.run(1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        lbm.run(1)
    el = time.perf_counter() - t0
    value = n ** 3 * args.steps / el / 1e6
    cores = host_threads()
    line = {
        "impl": "reference", "metric": metric_name(args.size, "fp32"), "value": value,
        "unit": "MLUPS", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * el / max(args.steps, 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (Taylor-Green vortex initial field)",
        "config": {"workload": "D3Q19 periodic Taylor-Green, tau 0.6; CPU sample %d^3 of the %d^3 "
                               "workload" % (n, args.size), "sample_nodes": n ** 3},
        "cpu_baseline": {"value": value, "unit": "MLUPS", "cores": cores, "kind": "port",
                         "sample": "oracle numpy restatement of the reference step, %d^3 nodes, "
                                   "%d timed steps" % (n, args.steps)},
        "e2e": {"value": value, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        main_reference(args, world, rank)
        return 0
    import torch

    from funlbm_b200 import build

    build.build()
    world, rank, local = dist_setup(args)
    if args.ke_errors:
        if rank == 0:
            print(json.dumps(run_ke_errors(args)), flush=True)
        return 0
    if args.case is not None:
        if rank == 0:
            res = run_case_precision(args) if args.vs_fp64 else run_case_sphere(args)
            print(json.dumps(res), flush=True)
        return 0
    if args.serve:
        if rank == 0:
            res = run_serve(args)
            print(json.dumps({"metric": "served stream: aggregate MLUPS and p50/p99 time-to-result "
                                        "vs the same requests one by one", "value": res["served_mlups"],
                              "unit": "MLUPS", "higher_is_better": True, "serve": res}), flush=True)
        return 0
    n = args.size
    ms, clocks, status, launch = run_device(args, world, rank, local)
    ms_per_step = ms / args.steps
    nodes = n ** 3
    value = world * nodes * args.steps / (ms / 1e3) / 1e6
    peak, peak_kind = measured_peak()
    bytes_per_launch = BYTES_PER_LU[args.storage] * nodes
    achieved = bytes_per_launch / (ms_per_step / 1e3) / 1e9
    fp16s = None
    if args.storage == "fp32" and not args.no_fp16s:
        # the same workload in FP16 shifted storage (half the bytes per update)
        a16 = argparse.Namespace(**vars(args))
        a16.storage = "fp16s"
        ms16, clocks16, status16, launch16 = run_device(a16, world, rank, local)
        step16 = ms16 / args.steps
        b16 = BYTES_PER_LU["fp16s"] * nodes
        ach16 = b16 / (step16 / 1e3) / 1e9
        v16 = world * nodes * args.steps / (ms16 / 1e3) / 1e6
        fp16s = {"value": v16, "unit": "MLUPS", "ms_per_step": step16, "vs_fp32": v16 / value,
                 "launch_shape": {"nodes_per_thread": launch16[0],
                                  "threads_per_block": launch16[1]},
                 "roofline": {"bound": "hbm", "achieved": ach16, "peak": peak, "unit": "GB/s",
                              "frac": ach16 / peak, "peak_kind": peak_kind,
                              "algorithmic_bytes_per_launch": b16},
                 "clocks": clocks16, "device_status": status16}
    e2e = None
    if not args.no_e2e:
        sec, h2d, d2h = run_e2e(args, world, local)
        e2e = {"value": world * nodes * args.steps / sec / 1e6, "unit": "MLUPS",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "includes": "public API (LBMD3.run_step) incl. init from a pinned host field, "
                           "per-step status read-back, final rho/u download"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": metric_name(n, args.storage), "value": value, "unit": "MLUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if args.storage == "fp32" else args.storage,
        "data": "synthetic (Taylor-Green vortex initial field, u0=0.05)",
        "config": {"workload": "D3Q19 %s, %d^3 nodes, all faces periodic, tau 0.6, Taylor-Green "
                               "u0=0.05; replicas per GPU" % (args.storage, n),
                   "nodes_per_gpu": nodes, "parallelism": "replicas",
                   "launch_shape": {"nodes_per_thread": launch[0], "threads_per_block": launch[1],
                                    "chosen_by": "funlbm_b200.tune"},
                   "l2_flush": "not needed: %.1f GB of populations per step >> 126 MB L2"
                               % (2 * bytes_per_launch / 2 / 1e9)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": profiled_traffic(args),
                     "algorithmic_bytes_per_launch": bytes_per_launch},
        "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": args.steps, "clocks": clocks,
        "device_status": status,
    }
    if fp16s is not None:
        line["fp16s"] = fp16s
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
