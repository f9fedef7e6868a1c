"""Benchmark of the ABD implicit contact time step on B200.

Workload: the 1024-body pile (512 cubes + 512 level-3 icospheres on a fixed ground box,
V = 332,808, T = 661,516, E = 992,274), seeded synthetic scene.  A step is one implicit time
step (Newton with CCD-bounded line search).  W warm-up steps run first (they also advance
the pile into contact), then K steps are timed with CUDA events; L2 is flushed between
timed steps by writing a 256 MiB buffer.

Multi-GPU: the step does not shard (one coupled Newton solve per scene), so N ranks run N
independent replicas; value = N * K / max-over-ranks time.

--impl reference times the CPU FP64 oracle (the restatement of the reference's step; the
reference itself needs Warp and abdtk, absent here) on the host cores for the same scene.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ABD steps/s vs plain FP64 on same B200 at ≤1e-6 rel pos err; adjoint grads/s"
WORKLOAD = "pile_1024_bodies_512cubes_512icosphereL3_ground (config 2)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of oracle work for cpu_baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def make_scene():
    from abd_warp_b200 import scenes
    bodies, prm, _ = scenes.make_config(2)
    return bodies, prm


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        mx = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def cpu_baseline_sample(bodies, prm, state, budget):
    """Time the CPU FP64 oracle on the same scene from the given state, for about `budget`
    seconds of work (at least one step).  Returns (steps_per_s, steps, threads)."""
    import oracle
    from abd_warp_b200 import scenes
    o = oracle.Oracle(scenes.flatten_bodies(bodies), prm)
    o.set_state(state["A0"], state["p0"], state["Adot"], state["pdot"], state["dq"])
    threads = oracle.max_threads()
    t0 = time.perf_counter()
    n = 0
    while True:
        o.step()
        n += 1
        if time.perf_counter() - t0 >= budget:
            break
    dt = time.perf_counter() - t0
    return n / dt, n, threads


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle
    from abd_warp_b200 import scenes
    bodies, prm = make_scene()
    o = oracle.Oracle(scenes.flatten_bodies(bodies), prm)
    threads = oracle.max_threads()
    budget = 150.0
    t_start = time.perf_counter()
    for _ in range(args.warmup):
        o.step()
        if time.perf_counter() - t_start > budget / 2:
            break
    t0 = time.perf_counter()
    n = 0
    for _ in range(args.steps):
        o.step()
        n += 1
        if time.perf_counter() - t0 > budget / 2:
            break
    el = time.perf_counter() - t0
    v = n / el
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": world,
        "steps": n, "warmup": args.warmup, "ms_per_step": 1e3 * el / n, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "bodies": len(bodies), "precision": "fp64"},
        "cpu_baseline": {"value": v, "unit": "steps/s", "cores": threads, "kind": "port",
                         "sample": f"{n} oracle steps after {args.warmup} warm-up steps (time-capped)"},
        "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import numpy as np
    import torch
    import torch.distributed as dist
    from abd_warp_b200.params import PRECISION_MIXED
    from abd_warp_b200.simulator import AffineBodySimulator

    rank, world, local = dist_env()
    if world > 1:
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    bodies, prm = make_scene()
    if args.precision == "mixed":
        prm.precision = PRECISION_MIXED
    sim = AffineBodySimulator(bodies=bodies, params=prm, device=f"cuda:{local}")
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(max(args.warmup, 3)):
        sim.step()
    torch.cuda.synchronize(dev)
    # state at the start of the timed region (for the CPU baseline sample)
    s = sim.states
    start_state = {"A0": s.A0.cpu().numpy(), "p0": s.p0.cpu().numpy(), "Adot": s.Adot.cpu().numpy(),
                   "pdot": s.pdot.cpu().numpy(), "dq": sim.dq.cpu().numpy()}
    # ---- device-resident timing ----
    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    launches0 = sim.launch_count()
    total_ms = 0.0
    infos = []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        infos.append(sim.step())
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    launches = sim.launch_count() - launches0
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    value = world * args.steps / (max_ms / 1e3)
    # ---- end to end through the public API with host buffers ----
    pin = {k: getattr(s, k).cpu().pin_memory() for k in ("A0", "p0", "Adot", "pdot")}
    xv_host = torch.empty(sim.x_view.shape, dtype=torch.float64).pin_memory()
    h2d = sum(v.numel() * 8 for v in pin.values())
    d2h = xv_host.numel() * 8
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e2e_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k, v in pin.items():
            getattr(s, k).copy_(v, non_blocking=True)
        info = sim.step()
        xv_host.copy_(sim.x_view, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
        for k in pin:
            pin[k].copy_(getattr(s, k))
    te = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * args.steps / (float(te.item()) / 1e3)
    newton = [i["newton_iters"] for i in infos]
    lin = [i["linear_iters"] for i in infos]
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded procedural scene)",
        "config": {"workload": WORKLOAD, "bodies": len(bodies), "verts": int(sim.n_verts),
                   "precision": args.precision, "parallelism": f"replicas{world}",
                   "l2": "flushed between timed steps (256 MiB write)",
                   "newton_iters_per_step": float(np.mean(newton)),
                   "linear_iters_per_step": float(np.mean(lin)),
                   "ls_trials_per_step": float(np.mean([i["ls_trials"] for i in infos])),
                   "active_contacts_last": infos[-1]["n_active"]},
        "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if rank == 0 and not args.no_cpu_baseline:
        v, n, threads = cpu_baseline_sample(bodies, prm, start_state, args.cpu_budget)
        line["cpu_baseline"] = {"value": v, "unit": "steps/s", "cores": threads, "kind": "port",
                                "sample": f"{n} CPU-oracle steps from the state at the start of the timed region"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    sim.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
