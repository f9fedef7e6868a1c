"""Benchmark of the ABD implicit contact time step on B200.

Workload: the 1024-body pile (512 cubes + 512 level-3 icospheres dropped on a fixed ground
box; V = 332,808, T = 661,516, E = 992,274), a seeded synthetic scene, 300-step trajectory.
A step is one implicit time step (Newton with CCD-bounded backtracking line search).

Timed steps: the trajectory is covered in four stretches that start from the oracle's states
at steps 0, 75, 150 and 225 (tests/golden/c2_states.npz; the GPU reproduces them bit for
bit).  --steps K times K // 4 consecutive steps from each state (the remainder from the
first ones), so that a short run samples the free fall, the landing and the settled pile
alike; K = 300 (the default) is exactly the whole trajectory.  W untimed warm-up steps run
first.  Each step is timed with CUDA events on the simulator's stream, and L2 is flushed
before every step by writing a 256 MiB buffer.

value: steps/s on device-resident states.  e2e: the same steps through the public API with
host buffers: every step copies its inputs (A0, p0, Adot, pdot) in from pinned host memory,
and copies the new vertex positions and the new states back, inside the timed region.

roofline: the narrow-phase kernel of the CCD pass, which also collects the line-search
candidates (the largest share of the step).  The step runs as one CUDA graph whose Newton loop
is a device-side WHILE node, where events cannot be recorded, so every launch of the kernel
inside the timed region is timed by the GPU's global timer: the kernel records the start of
its first CTA and the end of its last, on the stream it runs on.  The data it moves
(algorithmic bytes) is counted by the kernel in a replay of the same (deterministic) steps,
which makes the same launches.

batched: scene-steps/s of 512 independent scenes of 2 to 48 bodies (the batched
configuration) stepped by one graph launch per step, beside the same scenes stepped one after
another.  --no-batched skips it.

adjoint: gradients/s of the differentiable configuration's loss (16 icospheres on the ground
box, 100 steps, checkpoints every 10) with respect to all initial states, through the
torch.autograd trajectory of abd_warp_b200/adjoint.py (forward, then the backward's segment
recomputation and one adjoint step per step), with the oracle's forward and dense adjoint of
the same gradient as its CPU baseline.  --no-adjoint skips it.

Multi-GPU: the step does not shard (one coupled Newton solve per scene), so N ranks run N
independent replicas; value = N * K / max-over-ranks time.

--impl reference times the CPU FP64 oracle (the restatement of the reference's step; the
reference itself needs Warp and abdtk, absent here) on all host cores, over the same
schedule of steps (a bounded number per state when the full schedule would take too long;
the line says which).  The GPU arm's cpu_baseline is the same measurement on a smaller
budget.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ABD steps/s vs plain FP64 on same B200 at \u22641e-6 rel pos err; adjoint grads/s"
WORKLOAD = "pile of 1024 bodies (512 cubes + 512 level-3 icospheres) on a ground box, 300-step trajectory"
# DRAM bytes (read + write) per launch of k_chunk_narrow<CCD_LS> over the algorithmic bytes of
# the same launches, measured by ncu over the 20-step schedule (5 steps from each stored state,
# 176 launches, cold cache): 10.170 MB against 13.742 MB.  Below 1: tree nodes that several
# queries visit hit in L2.
NARROW_DRAM_PER_ALG_BYTE = 0.740
STATES = os.path.join(ROOT, "tests", "golden", "c2_states.npz")
STARTS = (0, 75, 150, 225)  # trajectory steps of the stored states


def schedule(k):
    """Steps timed from each stored state: k // 4 each, the remainder from the first ones."""
    return [k // len(STARTS) + (1 if i < k % len(STARTS) else 0) for i in range(len(STARTS))]


def schedule_text(per_state):
    return ", ".join(f"{n} from step {s}" for s, n in zip(STARTS, per_state) if n)


def measured_hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64"],
                    help="FP64 only: FP32 Krylov solves inside FP64 refinement diverge on the contact systems")
    ap.add_argument("--newton-loop", default="device", choices=["device", "host"],
                    help="the step's Newton iterations as a device loop (one graph launch per step) or driven "
                         "from the host (two waits per iteration); the same results")
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of oracle work for cpu_baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint gradient throughput")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched scenes' throughput")
    ap.add_argument("--start-state", type=int, default=None,
                    help="time all K steps from the stored oracle state at this step of the trajectory (0, 75, "
                         "150 or 225; for profiling one stretch) instead of K / 4 from each")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def slowest_ms(ms: float, world: int, device) -> float:
    """The replicas' time for their timed steps: the maximum of each rank's device time (after
    a barrier, so that every rank has finished them); a single rank's own time."""
    if world <= 1:
        return float(ms)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.barrier()
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, steps: int, max_ms: float) -> float:
    """Steps per second of all replicas together: each rank ran `steps` steps in at most max_ms."""
    return world * steps / (max_ms / 1e3)


def make_scene():
    from abd_warp_b200 import scenes
    bodies, prm, _ = scenes.make_config(2)
    return bodies, prm


ADJ_BODY = 1


def adjoint_scene():
    """The differentiable configuration: 16 level-2 icospheres on the ground box, 100 steps,
    loss ||com_1(T) - target||^2; the barrier stiffness lowered to 1e3 and Newton run to
    g.g < 1e-22 (60 iterations at most) so that the steps converge and the derivative exists."""
    import numpy as np
    from abd_warp_b200 import scenes
    bodies, prm, steps = scenes.make_config(4)
    prm.kappa, prm.tol, prm.max_iter = 1e3, 1e-22, 60
    flat = scenes.flatten_bodies(bodies)
    target = np.asarray(flat["p"][ADJ_BODY]) + np.array([0.3, 0.0, -0.2])
    return bodies, prm, steps, flat, target


def batched_gpu(dev, n_scenes=512, steps=4, warmup=2):
    """Scene-steps/s of the batched configuration (512 independent scenes of 2 to 48 bodies
    over their own ground boxes): every scene stepped by one graph launch (abd_batch_step),
    against the same scenes stepped one abd_step after another; the first steps of their
    trajectory (warm-up steps first, then the timed ones, CUDA events around each)."""
    import torch
    from abd_warp_b200 import scenes
    from abd_warp_b200.batch import BatchSimulator
    sc, prm, _ = scenes.config3(n_scenes=n_scenes)
    stream = torch.cuda.current_stream(dev)
    out = {}
    for mode in ("batched", "sequential"):
        b = BatchSimulator(sc, prm, device=str(dev))
        try:
            fn = b.step if mode == "batched" else b.step_sequential
            for _ in range(warmup):
                fn()
            torch.cuda.synchronize(dev)
            ms = 0.0
            contacts = 0
            for _ in range(steps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                infos = fn()
                e1.record(stream)
                e1.synchronize()
                ms += e0.elapsed_time(e1)
                contacts += sum(i["n_active"] for i in infos)
            out[mode] = n_scenes * steps / (ms / 1e3)
            out["active_contacts_per_step"] = contacts / steps
        finally:
            b.close()
    bodies = sum(len(x) for x in sc)
    return {"value": out["batched"], "unit": "scene-steps/s", "sequential": out["sequential"],
            "speedup": out["batched"] / out["sequential"],
            "workload": f"{n_scenes} scenes of 2-48 bodies ({bodies} bodies) over their own ground boxes, "
                        f"steps {warmup + 1}-{warmup + steps} of their trajectories",
            "active_contacts_per_step": out["active_contacts_per_step"], "dtype": "f64"}


def adjoint_gpu(dev, reps=2):
    """Gradients/s of the loss with respect to all initial states (positions, A, velocities)
    through the 100-step trajectory: forward with checkpoints every 10 steps, then the backward
    (segment recomputation and one adjoint step per step); the mean of reps gradients after one
    untimed, CUDA events around each."""
    import torch
    from abd_warp_b200.adjoint import trajectory
    from abd_warp_b200.simulator import AffineBodySimulator
    bodies, prm, steps, _, target = adjoint_scene()
    sim = AffineBodySimulator(bodies=bodies, params=prm, device=str(dev))
    tgt = torch.as_tensor(target, device=dev)
    stream = torch.cuda.current_stream(dev)
    times = []
    try:
        for r in range(reps + 1):
            sim.reset()
            x = [getattr(sim.states, k).clone().requires_grad_(True) for k in ("A0", "p0", "Adot", "pdot")]
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out = trajectory(sim, *x, steps=steps, checkpoint=10)
            d = out[1][ADJ_BODY] - tgt
            (d * d).sum().backward()
            e1.record(stream)
            e1.synchronize()
            if r:
                times.append(e0.elapsed_time(e1) / 1e3)
    finally:
        sim.close()
    return 1.0 / (sum(times) / len(times)), steps


def adjoint_cpu():
    """The oracle's forward and adjoint (dense exact Hessians) of the same gradient, timed once."""
    import numpy as np

    import oracle
    from oracle import adjoint_ref as AJ
    bodies, prm, steps, flat, target = adjoint_scene()
    t0 = time.perf_counter()
    o = oracle.Oracle(flat, prm)
    states, _ = AJ.forward(o, steps)
    _, gp = AJ.com_loss(states, ADJ_BODY, target)
    qb = np.zeros((o.n, 12))
    qb[ADJ_BODY, :3] = gp
    AJ.backward(o, flat, prm, states, qb, model="reference")
    return 1.0 / (time.perf_counter() - t0), oracle.max_threads()


class ClockSampler:
    """SM clocks, power and throttle reasons of the GPU sampled every 20 ms during the timed
    region, in-process through NVML (the data nvidia-smi reports; a polling nvidia-smi
    process would compete with the step's host synchronisations)."""

    NAMES = {"hw_slowdown": "nvmlClocksThrottleReasonHwSlowdown",
             "hw_thermal_slowdown": "nvmlClocksThrottleReasonHwThermalSlowdown",
             "sw_thermal_slowdown": "nvmlClocksThrottleReasonSwThermalSlowdown",
             "sw_power_cap": "nvmlClocksThrottleReasonSwPowerCap"}

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.thread = None
        self.stop_flag = False
        self.err = None

    def _handle(self, nv):
        import torch
        try:
            pr = torch.cuda.get_device_properties(self.device)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.device.index or 0)

    def start(self):
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._handle(nv)
        except Exception as exc:  # no NVML: reported in the line
            self.err = f"nvml unavailable: {exc}"
            return
        masks = {k: getattr(nv, v, 0) for k, v in self.NAMES.items()}

        def run():
            while not self.stop_flag:
                try:
                    sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                    mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                    pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                    rs = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                    self.rows.append((sm, mx, pw, [k for k, m in masks.items() if rs & m]))
                except Exception as exc:
                    self.err = str(exc)
                time.sleep(0.02)

        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()

    def stop(self):
        if self.thread is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [self.err or "not sampled"]}
        self.stop_flag = True
        self.thread.join()
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = sorted(r[0] for r in self.rows)
        return {"sm_mhz": float(sm[len(sm) // 2]), "sm_max_mhz": float(max(r[1] for r in self.rows)),
                "reasons": sorted({x for r in self.rows for x in r[3]}), "samples": len(self.rows),
                "power_w_max": max(r[2] for r in self.rows), "source": "NVML, every 20 ms"}


def oracle_sample(per_state, budget):
    """Oracle steps/s over the benchmark's schedule: from each stored state, up to per_state[i]
    consecutive steps, stopping early at budget / 4 seconds per state (at least one step).
    Returns (steps_per_s, steps done per state, threads, description)."""
    import numpy as np

    import oracle
    from abd_warp_b200 import scenes
    bodies, prm = make_scene()
    o = oracle.Oracle(scenes.flatten_bodies(bodies), prm)
    threads = oracle.max_threads()
    z = np.load(STATES)
    total_s, done = 0.0, []
    for s, want in zip(STARTS, per_state):
        if want == 0:
            done.append(0)
            continue
        o.set_state(*(z[f"s{s}_{k}"] for k in ("A0", "p0", "Adot", "pdot", "dq")))
        t0 = time.perf_counter()
        n = 0
        while n < want:
            o.step()
            n += 1
            if time.perf_counter() - t0 >= budget / len(STARTS):
                break
        total_s += (time.perf_counter() - t0) * (want / n)  # scaled to the whole stretch
        done.append(n)
    want_total = sum(per_state)
    same = done == list(per_state)
    desc = (f"oracle steps {schedule_text(done)} of the trajectory"
            + ("" if same else f" (the first steps of each stretch of the schedule {schedule_text(per_state)}, "
                               "each stretch's time scaled to its length)"))
    return want_total / total_s, done, threads, desc


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    bodies, _ = make_scene()
    per_state = schedule(args.steps)
    # the same steps as the GPU arm, bounded to about 2 minutes of host work
    v, done, threads, desc = oracle_sample(per_state, budget=120.0)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded procedural scene)",
        "config": {"workload": WORKLOAD, "bodies": len(bodies), "precision": "fp64",
                   "timed_steps": schedule_text(per_state), "oracle_steps_run": schedule_text(done)},
        "cpu_baseline": {"value": v, "unit": "steps/s", "cores": threads, "kind": "port", "sample": desc},
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
    from abd_warp_b200.simulator import AffineBodySimulator

    rank, world, local = dist_env()
    if world > 1:
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    bodies, prm = make_scene()
    prm.newton_loop = 0 if args.newton_loop == "device" else 1
    sim = AffineBodySimulator(bodies=bodies, params=prm, device=f"cuda:{local}")
    s = sim.states
    stream = torch.cuda.current_stream(dev)
    names = ("A0", "p0", "Adot", "pdot")

    z = np.load(STATES)
    per_state = schedule(args.steps)
    if args.start_state is not None:  # profiling: all K steps from one stored state
        if args.start_state not in STARTS:
            raise SystemExit(f"--start-state must be one of {STARTS}")
        per_state = [args.steps if st == args.start_state else 0 for st in STARTS]
    starts = {st: {k: torch.as_tensor(z[f"s{st}_{k}"], device=dev) for k in (*names, "dq")} for st in STARTS}

    def start_at(st):  # the stored state at trajectory step st, with its dq warm start
        sim.reset()
        for k in names:
            getattr(s, k).copy_(starts[st][k])
        s.A.copy_(s.A0)
        s.p.copy_(s.p0)
        sim.dq = starts[st]["dq"]
        torch.cuda.synchronize(dev)

    def run_schedule(counts, step_fn, at_start=None):
        """counts[i] consecutive steps from each stored state; returns (total ms, infos)."""
        total, infos = 0.0, []
        for st, n in zip(STARTS, counts):
            if n == 0:
                continue
            start_at(st)
            if at_start:
                at_start()
            for _ in range(n):
                ms, info = step_fn()
                total += ms
                infos.append(info)
        return total, infos

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def device_step():
        flush.zero_()
        e0.record(stream)
        info = sim.step()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), info

    # warm-up: W steps spread over the stored states like the timed ones (untimed)
    run_schedule(schedule(max(args.warmup, 3)), device_step)
    # ---- device-resident timing of the K steps ----
    clocks = ClockSampler(dev)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    sim.profile(1)  # the CCD pass's narrow kernel times its launches (global timer)
    launches0 = sim.launch_count()
    total_ms, infos = run_schedule(per_state, device_step)
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    launches = sim.launch_count() - launches0
    k_ms, k_launches, _ = sim.profile_read()
    sim.profile(0)
    max_ms = slowest_ms(total_ms, world, dev)
    value = whole_job_rate(world, args.steps, max_ms)
    # ---- end to end through the public API with host buffers ----
    # the caller keeps its states in pinned host memory: each step copies them in, steps, and
    # copies the new states and the vertex positions out (its next step's inputs)
    host = {"in": {k: torch.empty(getattr(s, k).shape, dtype=torch.float64).pin_memory() for k in names},
            "out": {k: torch.empty(getattr(s, k).shape, dtype=torch.float64).pin_memory() for k in names}}
    xv_host = torch.empty(sim.x_view.shape, dtype=torch.float64).pin_memory()
    h2d = sum(v.numel() * 8 for v in host["in"].values())
    d2h = xv_host.numel() * 8 + sum(v.numel() * 8 for v in host["out"].values())

    def e2e_begin():  # the stretch's start state, held by the caller on the host
        for k in names:
            host["in"][k].copy_(getattr(s, k))

    def e2e_step():
        flush.zero_()
        e0.record(stream)
        for k, v in host["in"].items():
            getattr(s, k).copy_(v, non_blocking=True)
        sim.step()
        xv_host.copy_(sim.x_view, non_blocking=True)
        for k, v in host["out"].items():
            v.copy_(getattr(s, k), non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        host["in"], host["out"] = host["out"], host["in"]
        return e0.elapsed_time(e1), None

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e2e_ms, _ = run_schedule(per_state, e2e_step, e2e_begin)
    e2e_value = whole_job_rate(world, args.steps, slowest_ms(e2e_ms, world, dev))
    # the algorithmic bytes of the same launches: the steps are deterministic, so a replay with
    # the kernel counting what it reads has the same launches (not timed: counting slows it)
    sim.profile(2)
    run_schedule(per_state, lambda: (0.0, sim.step()))
    _, c_launches, c_bytes = sim.profile_read()
    sim.profile(0)
    peak, peak_kind = measured_hbm_peak()
    bytes_per_launch = c_bytes / max(c_launches, 1)
    us_per_launch = 1e3 * k_ms / max(k_launches, 1)
    achieved = bytes_per_launch / (us_per_launch * 1e-6) / 1e9 if k_ms > 0 else None
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded procedural scene)",
        "config": {"workload": WORKLOAD, "bodies": len(bodies), "verts": int(sim.n_verts),
                   "timed_steps": schedule_text(per_state),
                   "precision": args.precision, "parallelism": f"replicas{world}",
                   "newton_loop": args.newton_loop,
                   "l2": "flushed before every timed step (256 MiB write)",
                   "newton_iters_per_step": float(np.mean([i["newton_iters"] for i in infos])),
                   "linear_iters_per_step": float(np.mean([i["linear_iters"] for i in infos])),
                   "ls_trials_per_step": float(np.mean([i["ls_trials"] for i in infos])),
                   "active_contacts_max": int(max(i["n_active"] for i in infos))},
        "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "clocks": clk,
        "roofline": {"kernel": "k_chunk_narrow<CCD_LS> (narrow phase of the CCD pass, which also collects "
                               "the line-search candidates)", "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "traffic": bytes_per_launch * NARROW_DRAM_PER_ALG_BYTE,
                     "traffic_how": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch over the "
                                    "20-step schedule, as a ratio to the kernel's algorithmic bytes "
                                    f"({NARROW_DRAM_PER_ALG_BYTE}), times this run's algorithmic bytes",
                     "peak_kind": peak_kind, "timed_launches": k_launches, "counted_launches": c_launches,
                     "avg_launch_us": us_per_launch, "bytes_per_launch": bytes_per_launch},
    }
    # the FP64 ceiling of the contact and solver kernels: the measured DFMA rate (their own
    # multiplies and adds are separate instructions, so half of it bounds them)
    import ctypes
    from abd_warp_b200 import _lib
    fp64 = ctypes.c_double(0.0)
    if _lib.load().abd_fp64_peak(ctypes.byref(fp64)) == _lib.ABD_OK:
        line["fp64_peak"] = {"value": fp64.value, "unit": "TFLOP/s", "how": "chains of DFMA on every SM, CUDA events"}
    if not args.no_batched:
        line["batched"] = batched_gpu(dev)
    if not args.no_adjoint:
        g, asteps = adjoint_gpu(dev)
        line["adjoint"] = {"value": g, "unit": "grads/s",
                           "workload": f"16 icospheres on a ground box, {asteps} steps, checkpoints every 10, "
                                       "gradient of ||com_1(T) - target||^2 with respect to all initial states",
                           "dtype": "f64"}
        if rank == 0 and not args.no_cpu_baseline:
            cg, cth = adjoint_cpu()
            line["adjoint"]["cpu_baseline"] = {"value": cg, "unit": "grads/s", "cores": cth, "kind": "port",
                                               "sample": "one gradient: oracle forward + dense exact-Hessian adjoint"}
    if rank == 0 and not args.no_cpu_baseline:
        v, _, threads, desc = oracle_sample(per_state, args.cpu_budget)
        line["cpu_baseline"] = {"value": v, "unit": "steps/s", "cores": threads, "kind": "port", "sample": desc}
    if rank == 0:
        print(json.dumps(line), flush=True)
    sim.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
