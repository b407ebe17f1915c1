#!/usr/bin/env python
"""Benchmark: body-steps/s of the plain FP64 step() path on one B200.

Workload (default): the box pile -- a static ground box (50,1,50) plus 4,096
boxes with half extents U[0.25,0.75]^3, density 1, random orientations,
dropped from a 16^3 lattice (spacing 1.6, from y=2) onto the ground; open
boundary, friction 0.5, restitution 0.2, g=-9.81, dt=1/60, 300 steps.

A "step" is one World::step() of that world.  The timed run starts from the
initial state and advances K steps (K defaults to the workload's 300), so the
early free fall and the settled pile (one ~20k-contact island) are both in it.

  value  -- state resident in HBM; per-step CUDA events on the world's stream;
            a 256 MiB buffer is rewritten between steps (outside the events)
            so every step starts with a cold L2.
  e2e    -- the same metric through the C-ABI with host buffers: each step
            uploads x/q/v/w from the host, steps, and downloads x/q/v/w.

Multi-GPU: the plain single-world path does not shard; --gpus N runs N
independent replicas (one per rank) and reports the aggregate.

--impl reference times the reference implementation (the NativeEngine C++
sources compiled unmodified, oracle/_ref) on the host cores: one process per
core, each stepping its own copy of the workload for a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "body-steps/s on 1 B200: plain FP64 vs batched FP32 at ≤1e-5 rel pose error"
UNIT = "body-steps/s"
WORKLOAD = ("box_pile_4096: static ground box (50,1,50) + 4,096 boxes, half extents U[0.25,0.75]^3, "
            "density 1, random unit quaternions, 16^3 lattice spacing 1.6 from y=2; open boundary, "
            "mu=0.5, e=0.2, g=-9.81, dt=1/60, from the initial state (seed 2)")
L2_FLUSH_BYTES = 256 << 20


def _cfg_box_pile():
    from nativeengine_b200 import scenes
    return scenes.box_pile()


def _cfg_box_pile_8():
    from nativeengine_b200 import scenes
    return scenes.box_pile(8, 8, 8)


def _cfg_gas():
    from nativeengine_b200 import scenes
    return scenes.gas()


def _cfg_batch():
    from nativeengine_b200 import scenes
    params, bodies, begin, kinds = scenes.batch_mix()
    return params, bodies, begin


def _cfg_batch_256():
    from nativeengine_b200 import scenes
    params, bodies, begin, kinds = scenes.batch_mix(nworlds=256)
    return params, bodies, begin


def _cfg_granular():
    from nativeengine_b200 import scenes
    return scenes.granular_mix(n=65536, max_attempts=2000)


CONFIGS = {
    "box_pile": (_cfg_box_pile, WORKLOAD),
    "box_pile_8": (_cfg_box_pile_8, "box_pile_512: as box_pile_4096 on an 8^3 lattice (profiling case)"),
    "gas": (_cfg_gas, "gas_1000: periodic elastic gas, 1,000 spheres r=0.5 m=1, L=25, v~N(0,1), e=1, mu=0, "
                      "g=0, dt=1/60 (seed 1)"),
    "batch": (_cfg_batch, "batch_2048: 2,048 independent worlds, body counts log-uniform in [16, 2048] "
                          "(~879k bodies), each a box pile (as box_pile at its size) or a periodic sphere gas "
                          "(as gas_1000 at its size), chosen 50/50 from seed 4; all worlds in one launch "
                          "sequence"),
    "batch_256": (_cfg_batch_256, "batch_256: the first 256 worlds of the batch_2048 recipe (seed 4; profiling case)"),
    "granular": (_cfg_granular, "granular_65536: periodic mix of spheres/capsules/cylinders/12-point hulls "
                                "(types by index mod 4), exact-overlap random sequential placement at the "
                                "densest box that places all bodies (true-volume packing fraction ~0.19), "
                                "v~N(0,0.5), mu=0.3, e=0.5, g=0, dt=1/60 (seed 3)"),
    "adjoint": (None, "adjoint_512: 512 worlds of a ground plane + 64 boxes (half extent 0.5, density 1) on an "
                      "8x8 grid, spacing 1.5, at y=0.5; v0 horizontal N(0,2^2); per-world friction U[0.2,0.8], "
                      "restitution U[0,0.5]; g=-9.81, dt=1/60, open boundary; 120 steps, checkpoint every 10; "
                      "loss sum |x_T - t|^2, t ~ U[-5,5]^3 (seed 6)"),
}
ADJ_STEPS, ADJ_K = 120, 10
# Reference-CPU sample per config: physics steps timed on one host core.
CPU_SAMPLE_STEPS = {"box_pile": 3, "box_pile_8": 20, "gas": 2000, "granular": 2, "batch": 2, "batch_256": 2}
PROFILE_SUMMARY = os.path.join(ROOT, "profiles", "solve_shared_box_pile_512.md")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--config", choices=sorted(CONFIGS), default="box_pile",
                    help="workload (box_pile is the headline; the others are for profiling and extra lines)")
    ap.add_argument("--precision", choices=("f64", "f32"), default="f64",
                    help="f64: bit-exact with the reference; f32: the batched FP32 form")
    ap.add_argument("--autotune", action="store_true", help="tune the big-island solver shape before timing")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(contacts):
    """DRAM bytes of one solver launch: the per-contact traffic of the
    committed ncu capture (a smaller pile; line 'traffic_bytes_per_contact: N')
    scaled by the contacts of the measured step, else None."""
    if not os.path.exists(PROFILE_SUMMARY):
        return None
    with open(PROFILE_SUMMARY) as f:
        for line in f:
            if line.strip().startswith("traffic_bytes_per_contact:"):
                try:
                    return float(line.split(":", 1)[1].strip().split()[0]) * contacts
                except ValueError:
                    return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"ne_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
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
        self.f.close()
        sms, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sms.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for nm, val in zip(names, parts[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(nm)
        busy = [s for s in sms if mx and s > 0.5 * mx] or sms
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sms)}


def cpu_baseline_reference(config: str, params, bodies):
    """The reference step (oracle/_ref, one host core) on a bounded sample:
    the first few steps of the same workload."""
    from oracle import oracle as O
    if not O.ref_available():
        return None
    steps = CPU_SAMPLE_STEPS[config]
    ora = O.RefOracle(params, bodies.copy())
    t0 = time.perf_counter()
    ora.step_plain(steps)
    dt = time.perf_counter() - t0
    return {"value": bodies.n * steps / dt, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"first {steps} steps of {config} ({bodies.n} bodies) on one host core ({dt:.1f} s)"}


def cpu_baseline_batch(params, bodies, begin, worlds: int = 64):
    """The reference on the first `worlds` worlds of the batch (one host core,
    one World at a time, as the reference steps them), 2 steps each."""
    from nativeengine_b200.bodies import BodyArrays
    from oracle import oracle as O
    if not O.ref_available():
        return None
    steps = CPU_SAMPLE_STEPS["batch"]
    work, t = 0, 0.0
    for k in range(min(worlds, len(params))):
        b0, b1 = int(begin[k]), int(begin[k + 1])
        sub = BodyArrays.__new__(BodyArrays)
        for key, v in bodies.__dict__.items():
            if isinstance(v, np.ndarray) and v.shape[:1] == (bodies.n,):
                setattr(sub, key, np.ascontiguousarray(v[b0:b1]))
        sub.n = b1 - b0
        sub.verts, sub.n_verts = bodies.verts, bodies.n_verts
        sub.nocollide, sub.n_nocollide = bodies.nocollide, 0
        sub.nocollide_count = np.zeros(sub.n, np.uint32)
        sub._c = None
        ora = O.RefOracle(params[k], sub)
        t0 = time.perf_counter()
        ora.step_plain(steps)
        t += time.perf_counter() - t0
        work += sub.n * steps
    return {"value": work / t, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"first {min(worlds, len(params))} worlds of batch_2048, {steps} steps each, one host core "
                      f"({t:.1f} s)"}


def _ref_worker(args):
    steps, q = args
    sys.path.insert(0, ROOT)
    from nativeengine_b200 import scenes
    from oracle import oracle as O
    params, bodies = scenes.box_pile()
    ora = O.RefOracle(params, bodies)
    t0 = time.perf_counter()
    ora.step_plain(steps)
    q.put((bodies.n * steps, time.perf_counter() - t0))


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libneref.so was not built"}))
        return 0
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    cores = os.cpu_count() or 1
    # Each process steps its own copy; a box-pile step costs seconds on a CPU
    # core, so the sample is capped at 2 steps per process (~10 s).
    steps = max(1, min(args.steps, 2))
    q = ctx.Queue()
    procs = [ctx.Process(target=_ref_worker, args=((steps, q),)) for _ in range(cores)]
    t0 = time.perf_counter()
    for p in procs:
        p.start()
    res = [q.get() for _ in procs]
    for p in procs:
        p.join()
    wall = time.perf_counter() - t0
    work = sum(r[0] for r in res)
    tmax = max(r[1] for r in res)
    value = work / tmax
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": 0, "ms_per_step": tmax / steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "bodies": 4097, "parallelism": f"{cores} processes, one world each"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{steps} steps of box_pile_4096 per process, {cores} processes "
                                   f"(wall {wall:.1f} s)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def fp32_one_step_error(dev):
    """One step from one device checkpoint in FP64 and in FP32, per-body
    errors |x32-x64|/max(|x64|,1), |q32-q64|, |v32-v64|/max(|v64|,1),
    |w32-w64|/max(|w64|,1) (max and upper quantiles).  Beside them, the same
    statistics for FP64 against FP64 with the velocities perturbed by 1e-12
    relative: the step is discontinuous where the reference's own contact
    decisions flip (manifold reference face, slop cut, contact on/off), so
    that baseline bounds what any precision can reach at the max."""
    import numpy as np

    def stats(a, b):
        out = {}
        for k, floor in (("x", 1.0), ("v", 1.0), ("w", 1.0)):
            d = np.linalg.norm(b[k] - a[k], axis=1) / np.maximum(np.linalg.norm(a[k], axis=1), floor)
            out[k] = {"max": float(d.max()), "p999": float(np.quantile(d, 0.999)), "p99": float(np.quantile(d, 0.99))}
        out["q"] = {"max": float(np.linalg.norm(b["q"] - a["q"], axis=1).max())}
        return out

    with dev.checkpoint() as ck:
        s0 = dev.state()
        dev.set_precision("f64")
        dev.step(1)
        a = dev.state()
        dev.restore(ck)
        dev.upload_state(v=s0["v"] * (1.0 + 1e-12), w=s0["w"] * (1.0 + 1e-12))
        dev.step(1)
        c = dev.state()
        dev.restore(ck)
        dev.set_precision("f32")
        dev.step(1)
        b = dev.state()
        dev.restore(ck)
    return {"fp32_vs_fp64": stats(a, b), "fp64_vs_fp64_perturbed_1e-12": stats(a, c),
            "definition": "one step from the same checkpoint; x, v, w relative to max(|.|, 1); q absolute"}


def plain_per_world(params, bodies, begin, steps: int, sample: int = 64):
    """The plain FP64 path on the batch's worlds one at a time (one
    single-world handle each, as a user of the reference's World API steps
    them): device time of `steps` steps for a seeded sample of worlds,
    extrapolated to the whole batch by body count."""
    import numpy as np
    import torch
    from nativeengine_b200 import DeviceWorld
    from nativeengine_b200.shard import slice_bodies
    rng = np.random.default_rng(5)
    nw = len(begin) - 1
    pick = sorted(rng.choice(nw, size=min(sample, nw), replace=False).tolist())
    t_total, b_total = 0.0, 0
    for w in pick:
        part, _ = slice_bodies(bodies, begin, w, w + 1)
        dev = DeviceWorld(params[w], part, record=False)
        dev.step(2)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dev.step(steps)
        torch.cuda.synchronize()
        t_total += time.perf_counter() - t0
        b_total += part.n
        dev.close()
    rate = b_total * steps / t_total
    return {"value": rate, "unit": UNIT, "sample": f"{len(pick)} of {nw} worlds, {steps} steps each, "
            f"one single-world handle per world, FP64, wall clock around synchronised steps"}


def run_ours(args):
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from nativeengine_b200 import DeviceWorld

    make, workload = CONFIGS[args.config]
    made = make()
    params, bodies = made[0], made[1]
    begin = made[2] if len(made) > 2 else None
    n_total = bodies.n
    if begin is not None and world > 1:
        # Independent worlds: each rank steps its own contiguous share (by
        # body count) on its own GPU; nothing crosses ranks during a step.
        from nativeengine_b200.shard import partition_worlds, slice_bodies
        w0, w1 = partition_worlds(begin, world)[rank]
        bodies, begin = slice_bodies(bodies, begin, w0, w1)
        params = params[w0:w1]
    n = bodies.n
    if begin is None:
        dev = DeviceWorld(params, bodies.copy(), record=False, precision=args.precision)
    else:
        dev = DeviceWorld(params[0], None, record=False, precision=args.precision)
        dev.upload_batch(params, bodies.copy(), begin)
    stream = torch.cuda.ExternalStream(dev.stream_handle())
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device="cuda")

    # Warm-up: W steps from the initial state (grows the device buffers).
    dev.step(max(args.warmup, 0))
    shape = dev.autotune(steps=3) if args.autotune else dev.solver_shape()

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def timed_run(host_io: bool):
        if begin is None:
            dev.upload(bodies.copy())
        else:
            dev.upload_batch(params, bodies.copy(), begin)
        dev.reset_warm_cache()
        st = bodies.state()
        K = args.steps
        ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
        ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
        launches = 0
        contacts = 0
        barrier()
        with torch.cuda.stream(stream):
            for k in range(K):
                ev0[k].record(stream)
                if host_io:
                    dev.upload_state(st["x"], st["q"], st["v"], st["w"])
                dev.step(1)
                launches += dev.launch_count()
                if host_io:
                    st = dev.state(out=st)
                ev1[k].record(stream)
                contacts += dev.stats()["contacts"]   # host-side counters of the step just taken
                flush.zero_()
        barrier()
        ms = [a.elapsed_time(b) for a, b in zip(ev0, ev1)]
        return ms, launches, contacts

    sampler = ClockSampler(local)
    sampler.start()
    ms_dev, launches, contacts_timed = timed_run(host_io=False)
    clocks = sampler.stop()
    stats = dev.stats()
    ms_e2e, _, _ = timed_run(host_io=True)
    # Stage breakdown: a separate run of the same steps with CUDA events
    # between the stages (which steps kernel by kernel, outside the graph).
    if begin is None:
        dev.upload(bodies.copy())
    else:
        dev.upload_batch(params, bodies.copy(), begin)
    dev.reset_warm_cache()
    dev.profile(True)
    dev.step(args.steps)
    stages = dev.stage_times()
    dev.profile(False)
    fp32_err = fp32_one_step_error(dev) if args.precision == "f32" else None

    t_dev = sum(ms_dev) / 1e3
    t_e2e = sum(ms_e2e) / 1e3
    contacts_job = float(contacts_timed)
    if world > 1:
        t = torch.tensor([t_dev, t_e2e], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        t_dev, t_e2e = float(t[0]), float(t[1])
        c = torch.tensor([contacts_job], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(c, op=torch.distributed.ReduceOp.SUM)
        contacts_job = float(c[0])
    K = args.steps
    # Whole-job throughput: replicas each step the full workload; a sharded
    # batch steps each world once across all ranks.
    sharded = begin is not None and world > 1
    work = n_total if sharded else world * n
    value = work * K / t_dev
    e2e_value = work * K / t_e2e

    if rank == 0:
        peak, peak_kind = load_peaks()
        steps_timed = max(stages.get("steps", 0), 1)
        stage_ms = {k: v / steps_timed for k, v in stages.items() if k != "steps"}
        dom = max(stage_ms, key=stage_ms.get)
        # Algorithmic bytes of the solve per step (each operand read once,
        # each result written once, FP64): per contact the constraint record
        # (n, rA, rB, restBias, mu, Kn, nImp, body indices: 120 B) read and
        # its impulses + warm-cache value (24 B) written; per body the state
        # it touches (v, w, x, q, invI, invMass: 128 B) read and v, w, x
        # (72 B) written.
        C_last = stats["contacts"]
        solve_bytes = 144.0 * C_last + 200.0 * n
        solve_ms = stage_ms["solve"]
        achieved = solve_bytes / (solve_ms * 1e-3) / 1e9 if solve_ms > 0 else 0.0
        # Whole-step algorithmic traffic: 360 B/body + 16 B/candidate pair +
        # 272 B/contact.
        step_bytes = 360.0 * n + 16.0 * stats["pairs"] + 272.0 * C_last
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup,
            "ms_per_step": t_dev / K * 1e3, "higher_is_better": True,
            "scaling": "strong" if sharded else "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "f64" else "f32 (FP64 poses, wrap, warm impulses, EPA tests)",
            "data": "synthetic",
            "config": {"workload": workload, "bodies": n_total, "steps_per_run": K, "precision": args.precision,
                       "solver_shape": {"threads": shape[0], "ctas_per_sm": shape[1], "team_max": shape[2],
                                        "autotuned": bool(args.autotune)},
                       "parallelism": (f"dp{world}: worlds sharded by body count, no data-path collective"
                                       if sharded else ("replicas" if world > 1 else
                                                        ("batch of worlds" if begin is not None else "single world"))),
                       "l2": "256 MiB buffer rewritten between timed steps (outside the events)",
                       "step_launch": "CUDA graph of the whole step, replayed once per step; one read of the "
                                      "device control block per step",
                       "graph_steps": stats["graph_steps"]},
            "roofline": {"bound": "hbm", "kernel": "solve (k_island_solve + k_big_rec + k_island_solve_shared + k_island_solve_local)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind, "traffic": profile_traffic(C_last),
                         "note": "latency-bound: the exact Gauss-Seidel order is a dependency chain; "
                                 "algorithmic bytes = 144 B/contact + 200 B/body of the last step"},
            # x, q, v, w: 13 doubles per body each way (ne_world_upload_state / ne_world_download)
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 13 * 8 * work,
                    "d2h_bytes_per_step": 13 * 8 * work},
            "gpu_launches": launches,
            "clocks": clocks,
            "stage_ms_per_step": stage_ms,
            "dominant_stage": dom,
            "last_step": {"pairs": stats["pairs"], "contacts": C_last, "islands": stats["islands"],
                          "max_island": stats["max_island"], "retries": stats["retries"]},
            "step_roofline": {"algorithmic_bytes_last_step": step_bytes,
                              "achieved_gbs_mean": step_bytes / (t_dev / K) / 1e9},
            "contacts_per_s": {"value": contacts_job / t_dev,
                               "contacts_timed_steps": contacts_job,
                               "hbm_frac": (272.0 * contacts_job / t_dev / 1e9) / peak,
                               "note": "contact constraints resolved per second over the timed steps "
                                       "(272 algorithmic bytes each, against the HBM peak)"},
        }
        if fp32_err is not None:
            line["fp32_vs_fp64"] = fp32_err
        if begin is not None and world == 1 and not args.no_cpu_baseline:
            line["plain_path_per_world"] = plain_per_world(params, bodies, begin, steps=20)
        if world == 1 and not args.no_cpu_baseline:
            if begin is None:
                line["cpu_baseline"] = cpu_baseline_reference(args.config, params, bodies)
            else:
                line["cpu_baseline"] = cpu_baseline_batch(params, bodies, begin)
        print(json.dumps(line))
    dev.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def run_adjoint(args):
    """The adjoint workload: a timed forward of the batch (fast path), a timed
    stepBackward of the same trajectory, and a spot check of its gradients
    against central finite differences of the FP64 reference on host cores."""
    import torch
    from nativeengine_b200 import DeviceWorld, scenes
    from nativeengine_b200.shard import slice_bodies
    from oracle import oracle as O
    from nativeengine_b200 import _ffi
    import ctypes as C

    rank, world, local = dist_env()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    params, bodies, begin, targets = scenes.adjoint_batch(nworlds=512, grid=8, seed=6)
    n = bodies.n
    dev = DeviceWorld(params[0], None, record=False)
    dev.upload_batch(params, bodies.copy(), begin)
    dyn = bodies.inv_mass > 0
    # warm-up: one forward and one backward
    with dev.checkpoint() as ck:
        dev.step(ADJ_STEPS)
        xT = dev.state()["x"]
        dev.restore(ck)
        xbar = np.where(dyn[:, None], 2.0 * (xT - targets), 0.0)
        dev.step_backward(ADJ_STEPS, ADJ_K, xbar=xbar)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dev.step(ADJ_STEPS)
        torch.cuda.synchronize()
        t_fwd = time.perf_counter() - t0
        dev.restore(ck)
        t0 = time.perf_counter()
        g = dev.step_backward(ADJ_STEPS, ADJ_K, xbar=xbar)
        torch.cuda.synchronize()
        t_bwd = time.perf_counter() - t0
    dev.close()
    loss = float((((xT - targets)[dyn]) ** 2).sum())
    # Finite differences of the reference, a few parameters of a few worlds.
    ref_cls = O.RefOracle if O.ref_available() else O.PortOracle

    def wloss(p, b, tw):
        o = ref_cls(p, b)
        o.step(ADJ_STEPS)
        d = (o.state()["x"] - tw)[b.inv_mass > 0]
        return float((d * d).sum())

    def pcopy(p):
        q = _ffi.NeWorldParams()
        C.pointer(q)[0] = p
        return q
    worst, nchk, nkink = 0.0, 0, 0
    t_ref = time.perf_counter()
    for wi in (0, 255, 511):
        part, _ = slice_bodies(bodies, begin, wi, wi + 1)
        tw = targets[begin[wi]:begin[wi + 1]]
        b0 = int(begin[wi])
        items = []
        for li, ax in ((3, 0), (40, 2)):
            def pv(p, b, d, li=li, ax=ax):
                b.v[li, ax] += d
                return p, b
            items.append((g["v"][b0 + li, ax], pv))

        def pmu(p, b, d):
            q = pcopy(p)
            q.friction += d
            return q, b

        def pe(p, b, d):
            q = pcopy(p)
            q.restitution += d
            return q, b
        items += [(g["friction"][wi], pmu), (g["restitution"][wi], pe)]
        for adj, pert in items:
            # The loss is piecewise smooth (contacts appear, support corners
            # switch), so a fixed step can straddle a kink.  Walk h down and
            # take the first pair of consecutive steps whose differences agree
            # to 1e-5: the function is smooth at that scale.  The adjoint is
            # compared with that value only; no agreeing pair = a kink within
            # 1e-8 of the parameter (counted, not compared).
            fds = []
            for h in (1e-5, 1e-6, 1e-7, 1e-8):
                lp = wloss(*pert(params[wi], part.copy(), h), tw)
                lm = wloss(*pert(params[wi], part.copy(), -h), tw)
                fds.append((lp - lm) / (2 * h))
            ref_fd = None
            for a, b in zip(fds, fds[1:]):
                if abs(a - b) <= 1e-5 * max(abs(a), abs(b), 1e-3):
                    ref_fd = b
                    break
            if ref_fd is None:
                nkink += 1
                continue
            worst = max(worst, abs(adj - ref_fd) / max(abs(ref_fd), abs(adj), 1e-3))
            nchk += 1
    t_ref = time.perf_counter() - t_ref
    line = {
        "metric": "adjoint (stepBackward) throughput: body-steps/s differentiated", "value": n * ADJ_STEPS / t_bwd,
        "unit": "body-steps/s", "n_gpus": 1, "steps": ADJ_STEPS, "warmup": 1, "ms_per_step": t_bwd / ADJ_STEPS * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": CONFIGS["adjoint"][1], "bodies": n, "worlds": 512, "checkpoint_every": ADJ_K},
        "forward_ms": t_fwd * 1e3, "backward_ms": t_bwd * 1e3, "backward_over_forward": t_bwd / t_fwd,
        "loss": loss,
        "fd_check": {"max_rel_err": worst, "parameters_compared": nchk, "parameters_on_a_kink": nkink,
                     "tolerance": 1e-4,
                     "sample": "worlds 0, 255, 511: v0 of 2 boxes, friction, restitution; central differences of "
                               "the FP64 reference on the host at h = 1e-5 .. 1e-8, compared at the first pair of "
                               f"consecutive h that agree to 1e-5 ({t_ref:.1f} s)"},
        "timing": "wall clock around synchronised calls (the backward is one kernel launch plus scratch setup)",
    }
    print(json.dumps(line))
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.config == "adjoint":
        return run_adjoint(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
