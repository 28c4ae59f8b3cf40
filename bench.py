#!/usr/bin/env python
"""Benchmark: particle-updates/s of the MPH-WC explicit step, 3-D dam break.

Workload (default): 100x100x200 type-0 fluid block (2.0 M particles, l0 =
0.005 m, seeded +-0.01 l0 jitter) in the corner of a 300x100x240-cell box closed
by 3 layers of type-2 wall particles (0.78 M), gravity -9.81 z, rho 1000,
mu 1e-3, no surface tension, radii 1.7/3.5 l0, c = 20 m/s, dt 2e-5 s.
Synthetic data from the seeded generator (mphexplicit_b200/scenes.py); the
reference publishes no input set for it.

A "step" is one explicit step of the whole scene (the reference's loop body).
value = fluid particles x steps / seconds, summed over ranks (replicas: the
step does not shard, each rank runs its own scene on its own GPU).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--mode fp64|mixed|mixed_p64] [--only]
                  [--forms fp64,mixed,mixed_p64,learned,batch,two_fluid,output]
  python bench.py --impl reference ...   # the reference's own CPU step, all host threads

One JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-updates/s, 3D 2M-particle dam break: FP64 plain vs mixed/learned"
UNIT = "particle-updates/s"
# algorithmic HBM bytes per particle per launch, 3-D without surface tension:
# sweep A reads x, v, type (52 B) and writes PressureP (8 B); sweep B reads
# x, v, type, PressureP (60 B) and writes x, v (48 B)  -> 168 B per update.
ALGO_BYTES = {"sweep_a": 60.0, "sweep_b": 108.0, "mix_sweep_a": 60.0, "mix_sweep_b": 108.0, "move": 96.0,
              "mix_move": 96.0}


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


def max_over_ranks(x: float, world: int) -> float:
    """x of the slowest rank: an all-reduce MAX over the process group (on the
    GPU under NCCL, on the host under gloo)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(units_per_rank: int, steps: int, world: int, ms: float) -> float:
    """Whole-job throughput: the units every rank updated over the slowest
    rank's time (weak scaling: each rank runs its own replica)."""
    return units_per_rank * steps * world / (ms / 1e3)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_bf16_peak():
    """Dense BF16 peak (TFLOP/s) and where it comes from."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["bf16_tflops"]), "measured bf16 burst (MEASURED_PEAKS.json)"
    return 1590.0, "fallback (MEASURED_PEAKS.json absent)"


def _profile_value(kernel: str, key: str):
    tag = kernel + ("_fp32" if kernel == "mix_sweep_b" else "")  # one FP32 force sweep in both mixed forms
    p = os.path.join(ROOT, "profiles", "ncu_%s_dam_break_3d.md" % tag)
    if not os.path.exists(p):
        return None
    m = re.search(key + r":\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


def ncu_traffic(kernel: str, mode: str):
    """DRAM bytes per step of the `kernel` scope on the full-size dam break,
    from the committed ncu summary (profiles/), or None."""
    return _profile_value(kernel, "traffic_bytes_per_step_full_size")


def ncu_pipe(kernel: str):
    """The busiest execution pipe of `kernel` and its active fraction (ncu
    sm__pipe_*_cycles_active of the committed summary), or None."""
    f = _profile_value(kernel, "fp64_pipe_active_frac")
    return {"pipe": "fp64", "active_frac": f, "source": "ncu sm__pipe_fp64_cycles_active, profiles/"} if f else None


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons during a timed region: the
    recipe's `nvidia-smi -lms 200` line, started before the region (the
    region waits for its first sample) and stopped after one more sample, plus
    NVML read every 10 ms from a thread while the region runs (a region of a
    few tens of ms falls between two nvidia-smi samples).  Reading clocks
    changes nothing on the GPU."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")
        self.nvml = []  # (sm MHz, max sm MHz, reason names)
        self._stop = None
        self._thread = None

    def _rows(self):
        try:
            return [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            return []

    def _nvml_loop(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(self.idx)
            bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                    nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            while True:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.nvml.append((float(sm), float(mx), [self.NAMES[k] for k in range(4) if r & bits[k]]))
                if self._stop.wait(0.01):
                    break
            nv.nvmlShutdown()
        except Exception:
            pass

    def __enter__(self):
        import threading
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--id=%d" % self.idx, "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        t0 = time.time()
        while self.proc is not None and not self._rows() and time.time() - t0 < 10.0:
            time.sleep(0.05)
        self._stop = threading.Event()
        self._thread = threading.Thread(target=self._nvml_loop, daemon=True)
        self._thread.start()
        time.sleep(0.02)
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._thread.join(timeout=5)
        if self.proc:
            n0, t0 = len(self._rows()), time.time()
            while len(self._rows()) <= n0 and time.time() - t0 < 2.0:
                time.sleep(0.05)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = self._rows()
        sm = [float(r[1]) for r in rows if len(r) > 2 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) > 2 and r[2].strip().replace(".", "").isdigit()]
        reasons = {self.NAMES[k] for r in rows for k in range(4) if len(r) > 5 + k and "Active" in r[5 + k]
                   and "Not" not in r[5 + k]}
        for _, _, rs in self.nvml:
            reasons.update(rs)
        nv_sm = [x[0] for x in self.nvml]
        if not sm and not nv_sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        allsm = nv_sm if nv_sm else sm
        return {"sm_mhz": float(np.median(allsm)), "sm_max_mhz": max(mx + [x[1] for x in self.nvml]) if (mx or nv_sm)
                else None, "reasons": sorted(reasons), "samples": len(rows), "nvml_samples": len(nv_sm),
                "sm_mhz_nvidia_smi": float(np.median(sm)) if sm else None}


# edge-MLP flops per evaluated edge: 2 * (9*128 + 128*128 + 128*128 + 128*3)
MLP_FLOPS_PER_EDGE = 2.0 * (9 * 128 + 128 * 128 * 2 + 128 * 3)


def measure_learned(args, rank):
    """The learned form on the 1 M-fluid dam break (80x80x160 fluid in a
    240x80x192-cell box): training data from the FP64 step on 8 seeded
    jitters (2000 FP64 steps in all, spread over the first ~1100 steps of the
    flow by an untimed pre-roll in MPH_MODE_MIXED_P64), Adam training of
    the edge MLP on the tensor cores, then a timed run of `learned_steps`
    steps with the plain FP64 step as judge every 20 steps (fallback above a
    relative force error of 1e-2), and its velocity error against the FP64 run
    of the same steps."""
    import torch
    import mphexplicit_b200 as M
    from mphexplicit_b200 import learned as LR
    from mphexplicit_b200 import scenes

    fluid = tuple(int(v) for v in args.learned_fluid.split(","))
    box = (3 * fluid[0], fluid[1], (6 * fluid[2]) // 5)

    def scene(seed):
        return scenes.dam_break_3d(fluid=fluid, box=box, seed=seed)

    t0 = time.perf_counter()
    seeds = 8
    per = max(1, args.learn_steps // seeds)
    every = max(1, per // 10)
    samples = 1 << 16
    ds = LR.Dataset(seeds * (per // every + 1) * samples)
    for k in range(seeds):
        sc = scene(1000 + rank * 100 + k)
        start = (k * 1000) // seeds  # spread the seeds over the first 1000 steps
        if start > 0:
            pre = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=3, mode="mixed_p64")
            pre.step(start)
            st = pre.state()
            pre.close()
            order = np.argsort(st["particle_index"], kind="stable")
            x0, v0, t0_ = st["xyz"][order], st["vel"][order], st["type"][order]
        else:
            x0, v0, t0_ = sc.xyz, sc.vel, sc.type
        s = M.Solver(sc.params, sc.header, t0_, x0, v0, dim=3, mode="fp64")
        for q in range(0, per, every):
            s.collect_samples(ds, samples, seed=k * 100003 + q)
            s.step(min(every, per - q))
        s.close()
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    t0 = time.perf_counter()
    m = LR.Model(seed=rank)
    m.fit_scales(ds)
    # Adam in three phases of falling step size (2e-3, 6e-4, 2e-4)
    loss = None
    per_phase = max(1, args.learn_epochs // 3)
    for k, lr in enumerate((2e-3, 6e-4, 2e-4)):
        loss = m.train(ds, epochs=per_phase, batch=4096, lr=lr, seed=rank * 7 + k)
    t_train = time.perf_counter() - t0
    n_samples = len(ds)
    ds.close()

    sc = scene(rank)
    steps = args.learned_steps
    s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=3, mode="learned")
    s.set_learned(m, 20, 1e-2)
    s.step(3)  # warm-up (counted in the judge's statistics)
    s.synchronize()
    stream = torch.cuda.ExternalStream(s.stream_handle)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.profile(True)
    ev0.record(stream)
    s.step(steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    prof = s.profile_read()
    stats = s.learned_stats()
    got = s.state()
    s.close()
    ref = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=3, mode="fp64")
    ref.step(3 + steps)
    rst = ref.state()
    ref.close()
    o1, o2 = np.argsort(got["particle_index"]), np.argsort(rst["particle_index"])
    fl = rst["type"][o2] < 2
    err = float(np.linalg.norm(got["vel"][o1][fl] - rst["vel"][o2][fl]) / np.linalg.norm(rst["vel"][o2][fl]))
    m.close()
    out = {"workload": "dam_break_3d fluid %dx%dx%d in a %dx%dx%d-cell box: %d particles (%d fluid)"
                       % (*fluid, *box, sc.n, sc.n_fluid),
           "value": sc.n_fluid * steps / (ms / 1e3), "ms_per_step": ms / steps, "steps": steps,
           "rel_l2_vel_vs_fp64": err, "error_steps": 3 + steps,
           "judge_interval": 20, "tolerance": 1e-2,
           "fallback_rate": stats["plain_steps"] / max(1, stats["steps"]), "judge": stats,
           "kernels_ms_per_step": {k: v[1] / steps for k, v in prof.items()},
           "training": {"fp64_steps": seeds * per, "seeds": seeds, "samples": n_samples, "epochs": 3 * per_phase,
                        "learning_rates": [2e-3, 6e-4, 2e-4],
                        "final_loss": loss, "data_s": t_data, "train_s": t_train}}
    if "mlp_edges" in prof:
        nl, tot = prof["mlp_edges"]
        avg_s = tot / max(1, nl) / 1e3
        tflops = stats["edges"] * MLP_FLOPS_PER_EDGE / avg_s / 1e12
        peak, peak_kind = measured_bf16_peak()
        out["roofline"] = {"kernel": "mlp_edges", "bound": "tensor", "achieved": tflops, "peak": peak, "unit": "TFLOP/s",
                           "frac": tflops / peak, "edges_per_launch": stats["edges"],
                           "flops_per_edge": MLP_FLOPS_PER_EDGE, "avg_launch_ms": avg_s * 1e3,
                           "peak_source": peak_kind}
    return out


# algorithmic HBM bytes per particle of the batched 2-D sweeps with surface
# tension (FP64 state, 2-D): sweep A reads x, v, type (36 B) and writes
# PressureP, PressureA, GravityCenter (32 B); sweep B reads x, v, type and those
# (68 B) and writes v (16 B) and, through the next move, x (16 B)  -> 168 B.
BATCH_ALGO_BYTES = {"batch_sweep_a": 68.0, "batch_sweep_b": 100.0}


def measure_batch(args, rank):
    """The batched form on 256 uneven 2-D droplets (each w x h particles,
    w, h ~ U[20, 140], l0 = 1e-3 m, mu log-uniform in [1e-3, 1] Pa s, sigma
    uniform in [0.02, 0.08] N/m, dt = 5e-6 s): autotune, then `batch_steps`
    steps timed as CUDA-graph replays, a per-kernel pass, the velocity error
    of a sample of scenes against the FP64 form run alone, and the
    reference's own step on a sample of the scenes (one after the other)."""
    import torch
    import mphexplicit_b200 as M
    from mphexplicit_b200 import scenes
    scs = scenes.droplet_batch_2d(count=256, seed=rank)
    b = M.Batch(scs)
    trials = b.autotune(steps=32)
    info0 = b.info()
    steps = args.batch_steps
    b.step(max(args.warmup, 3) + 13)  # warm-up: at least one full graph replay
    b.synchronize()
    stream = torch.cuda.ExternalStream(b.stream_handle)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    info1 = b.info()
    ev0.record(stream)
    b.step(steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    info2 = b.info()
    b.profile(True)
    b.step(32)
    prof = b.profile_read()
    b.profile(False)
    done = info2["steps"] + 32
    xyz, vel = b.state()
    off = b.offsets
    b.close()
    # error of a sample of scenes against the FP64 form (bit-identical to the reference)
    errs = []
    for k in range(0, len(scs), max(1, len(scs) // args.batch_check)):
        sc = scs[k]
        s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=2, mode="fp64")
        s.step(done)
        st = s.state()
        s.close()
        order = np.argsort(st["particle_index"], kind="stable")
        rv = st["vel"][order]
        gv = vel[off[k]:off[k + 1]]
        errs.append(float(np.linalg.norm(gv - rv) / np.linalg.norm(rv)))
    nf = int(sum(sc.n_fluid for sc in scs))
    name, (nl, tot_ms) = max(prof.items(), key=lambda kv: kv[1][1])
    avg_s = tot_ms / nl / 1e3
    peak, peak_kind = measured_peaks()
    achieved = BATCH_ALGO_BYTES.get(name, 0.0) * nf / avg_s / 1e9
    out = {"workload": "256 uneven 2-D droplets (w, h ~ U[20,140] particles, l0=1e-3, mu log-U[1e-3,1], "
                       "sigma U[0.02,0.08], dt=5e-6): %d particles" % nf,
           "value": nf * steps / (ms / 1e3), "ms_per_step": ms / steps, "steps": steps,
           "graph_steps": info0["graph_steps"], "tile": list(info0["tile"]), "threads": info0["threads"],
           "items": info0["items"], "scene_rebuilds_in_timed_region": info2["scene_rebuilds"] - info1["scene_rebuilds"],
           "tile_splits": info2["tile_splits"], "autotune": trials,
           "rel_l2_vel_vs_fp64": {"max": max(errs), "median": float(np.median(errs)), "scenes": len(errs),
                                  "steps": done},
           "kernels_ms_per_step": {k: v[1] / 32 for k, v in prof.items()},
           "roofline": {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "peak_source": peak_kind,
                        "algorithmic_bytes_per_launch": BATCH_ALGO_BYTES.get(name, 0.0) * nf,
                        "avg_launch_ms": avg_s * 1e3}}
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import pyoracle as po
        threads = os.cpu_count() or 1
        tot_s, tot_upd, n_sc = 0.0, 0, 0
        with tempfile.TemporaryDirectory() as td:
            for k in range(0, len(scs), max(1, len(scs) // args.batch_cpu_scenes)):
                sc = scs[k]
                d, g = os.path.join(td, "s.data"), os.path.join(td, "s.grid")
                sc.write(d, g)
                if po.ref_available(2):
                    r = po.time_reference(d, g, 2, 0, args.batch_cpu_steps, threads, timeout=600)
                    kind = "reference"
                else:
                    os.environ["OMP_NUM_THREADS"] = str(threads)
                    r = po.time_oracle(sc, 0, args.batch_cpu_steps)
                    kind = "port"
                tot_s += r["seconds"]
                tot_upd += r["fluid"] * r["steps"]
                n_sc += 1
        out["cpu_baseline"] = {"value": tot_upd / tot_s, "unit": UNIT, "cores": threads, "kind": kind,
                               "sample": "%d of the 256 scenes, %d steps each, one after the other, %.1f s wall"
                                         % (n_sc, args.batch_cpu_steps, tot_s)}
    return out


def measure_droplet(args, rank):
    """Benchmark config 1: the 2-D square droplet (40x40 type-0 particles,
    l0 = 0.004 m, mu 0.1, sigma 0.07, sound speed 10 m/s, dt 1e-5 s, no walls or
    gravity), FP64, `droplet_steps` steps in one mph_step call: the default
    graph launches (the rebuild test on the device) and the host path (one
    flag read per step, mph_set_step_graphs(0)), both bit-identical, and the
    reference's own 2-D build on the same scene on all host threads and on
    one.  At this size the sweeps run one warp per particle."""
    import torch
    import mphexplicit_b200 as M
    from mphexplicit_b200 import scenes
    sc = scenes.droplet_2d(n=40, seed=rank)
    steps = args.droplet_steps
    out = {"workload": "droplet_2d 40x40 fluid, no walls, surface tension: %d particles" % sc.n, "steps": steps,
           "form": "fp64"}
    res = {}
    for graphs in (True, False):
        s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=2, mode="fp64")
        s.set_step_graphs(graphs)
        s.step(3)  # warm-up (the first several-step call captures the graphs)
        s.synchronize()
        stream = torch.cuda.ExternalStream(s.stream_handle)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ev0.record(stream)
        s.step(steps)
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = max(ev0.elapsed_time(ev1), (time.perf_counter() - t0) * 1e3)
        info = s.info()
        st = s.state()
        s.close()
        res[graphs] = {"ms": ms, "st": st, "rebuilds": info["rebuild_count"]}
        key = "graphs" if graphs else "host_path"
        out[key] = {"value": sc.n * steps / (ms / 1e3), "ms_per_step": ms / steps, "rebuilds": info["rebuild_count"]}
    out["bit_identical"] = all(np.array_equal(res[True]["st"][k], res[False]["st"][k]) for k in ("xyz", "vel"))
    out["graphs_speedup_vs_host_path"] = res[False]["ms"] / res[True]["ms"]
    out["value"] = out["graphs"]["value"]
    from oracle import ref_inputs as RI
    if rank == 0 and RI.ref_available(2) and not args.no_cpu_baseline:
        cores = RI.host_cores()
        with tempfile.TemporaryDirectory() as td:
            d, g, n = RI.droplet_files(td, seed=rank)
            ref = {}
            for th in sorted({cores["logical"], 1}):
                r = RI.time_reference(d, g, 2, 1, steps, th, timeout=1800)
                ref[th] = {"value": n * r["steps"] / r["seconds"], "seconds": r["seconds"], "steps": r["steps"],
                           "threads": th, "rebuilds": r["rebuilds"]}
        best = max(ref.values(), key=lambda x: x["value"])
        out["reference"] = {"kind": "reference (oracle/_ref/ref_mph2d, the reference's Mph_gcc2d flags)",
                            "by_threads": list(ref.values()), "value": best["value"], "threads": best["threads"],
                            "cores": cores}
        out["vs_reference"] = out["value"] / best["value"]
    return out


def measure_two_fluid(args, rank):
    """Benchmark config 3: the two-fluid column (200^3 fluid, l0 = 0.0025 m,
    lower half type 0 at rho 500, upper half type 1 at rho 1000, interface
    displaced by a seeded sum of 4 cosine modes of amplitude 2 l0, 2-layer
    type-2/3 walls, mu 0.01, sigma 0.05, dt 1e-5 s): both mixed forms timed over
    `two_fluid_steps` steps, each with its velocity error against the FP64 form
    over the same steps."""
    import torch
    import mphexplicit_b200 as M
    from mphexplicit_b200 import scenes
    n = args.two_fluid_n
    sc = scenes.two_fluid_column(n=n, seed=rank)
    out = {"workload": "two_fluid_column %d^3 fluid, 2 wall layers: %d particles (%d fluid)" % (n, sc.n, sc.n_fluid)}
    res = {}
    for mode in ("mixed", "mixed_p64", "fp64"):
        s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=3, mode=mode)
        s.step(3)
        s.synchronize()
        stream = torch.cuda.ExternalStream(s.stream_handle)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.profile(True)
        ev0.record(stream)
        s.step(args.two_fluid_steps)
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        prof = s.profile_read()
        info = s.info()
        st = s.state()
        s.close()
        order = np.argsort(st["particle_index"], kind="stable")
        res[mode] = {"ms": ms, "vel": st["vel"][order], "fluid": st["type"][order] < 2, "prof": prof,
                     "rebuilds": info["rebuild_count"]}
    steps = args.two_fluid_steps
    f = res["fp64"]
    fl = f["fluid"]
    out.update({"steps": steps, "error_steps": 3 + steps, "fp64_ms_per_step": f["ms"] / steps})
    for mode in ("mixed", "mixed_p64"):
        r = res[mode]
        out[mode] = {"value": sc.n_fluid * steps / (r["ms"] / 1e3), "ms_per_step": r["ms"] / steps,
                     "speedup_vs_fp64": f["ms"] / r["ms"], "rebuilds": r["rebuilds"],
                     "rel_l2_vel_vs_fp64": float(np.linalg.norm(r["vel"][fl] - f["vel"][fl]) /
                                                 np.linalg.norm(f["vel"][fl])),
                     "kernels_ms_per_step": {k: v[1] / steps for k, v in r["prof"].items()}}
    out["value"] = out["mixed"]["value"]
    out["fp64_value"] = sc.n_fluid * steps / (f["ms"] / 1e3)
    from oracle import ref_inputs as RI
    if rank == 0 and RI.ref_available(3) and not args.no_cpu_baseline and args.two_fluid_ref_seconds > 0:
        # the reference on the same column, a bounded sample (its start-up,
        # reading 8.5 M particles and the first lists, is not timed)
        cores = RI.host_cores()
        with tempfile.TemporaryDirectory() as td:
            d, g, nn, nf = RI.two_fluid_files(td, seed=rank, n=n)
            r = RI.time_reference(d, g, 3, 0, 1000, cores["logical"], max_seconds=args.two_fluid_ref_seconds,
                                  timeout=3600)
        ref_value = nf * r["steps"] / r["seconds"]
        out["reference"] = {"kind": "reference (oracle/_ref/ref_mph3d, the reference's Mph_gcc3d flags)",
                            "value": ref_value, "threads": cores["logical"], "steps": r["steps"],
                            "seconds": r["seconds"], "startup_seconds": r.get("startup_seconds"),
                            "sample": "%d timed step(s) of the full column on %d OpenMP threads"
                                      % (r["steps"], cores["logical"])}
        out["fp64_vs_reference"] = out["fp64_value"] / ref_value
        out["mixed_vs_reference"] = out["mixed"]["value"] / ref_value
    return out


def measure_output(args, sc, rank):
    """The output path (writeVtkFile / writeProfFile, main.cpp:672-834) on the
    benchmark scene after 20 MPH_MODE_MIXED_P64 steps: the device formatting
    time per document (CUDA events on the context's stream, 3 launches each),
    mph_write_vtk / mph_write_prof end to end (wall clock: format, copy out,
    fwrite into the page cache), the host printf writer on the same state
    (the reference's writer), whether the bytes agree, and the stepping time
    with a VTK written behind every `output_every` steps against none."""
    import tempfile
    import time
    import mphexplicit_b200 as M
    s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=3, mode="mixed_p64")
    s.step(20)
    s.synchronize()
    out = {"workload": scene_workload(sc), "particles": sc.n}
    with tempfile.TemporaryDirectory() as td:
        vtk, prof, host = (os.path.join(td, f) for f in ("d.vtk", "d.prof", "h.vtk"))
        s.write_vtk(vtk)  # warm-up: buffers, writer thread
        s.write_prof(prof)
        s.profile(True)
        tv, tp = [], []
        for _ in range(3):
            a = time.perf_counter()
            s.write_vtk(vtk)
            tv.append(time.perf_counter() - a)
            a = time.perf_counter()
            s.write_prof(prof)
            tp.append(time.perf_counter() - a)
        p = s.profile_read()
        s.profile(False)
        vtk_bytes, prof_bytes = os.path.getsize(vtk), os.path.getsize(prof)
        st = s.state()
        a = time.perf_counter()
        M.write_vtk_arrays(host, st)
        host_s = time.perf_counter() - a
        same = open(host, "rb").read() == open(vtk, "rb").read()
        ms_vtk = p["text_vtk"][1] / 3
        ms_prof = p["text_prof"][1] / 3
        # VTK record inputs: pos, vel, force (double4), type, NeighborCount (int),
        # DensityA, VolStrainP, VirialPressure (double) = 128 B per particle
        out.update({"vtk_bytes": vtk_bytes, "prof_bytes": prof_bytes,
                    "vtk_device_ms": ms_vtk, "prof_device_ms": ms_prof,
                    "vtk_device_gbs": (vtk_bytes + 128.0 * sc.n) / (ms_vtk / 1e3) / 1e9,
                    "write_vtk_s": min(tv), "write_prof_s": min(tp), "host_printf_vtk_s": host_s,
                    "write_vtk_speedup_vs_host": host_s / min(tv), "bytes_equal_host": same})
        every, files = args.output_every, args.output_files
        s.synchronize()
        a = time.perf_counter()
        s.step(every * files)
        s.synchronize()
        base = time.perf_counter() - a
        a = time.perf_counter()
        for k in range(files):
            s.step(every)
            s.write_vtk_async(os.path.join(td, "a%d.vtk" % (k % 2)))
        s.synchronize()
        stepped = time.perf_counter() - a
        s.output_wait()
        done = time.perf_counter() - a
        out.update({"output_every": every, "files": files, "steps_s_no_output": base,
                    "steps_s_with_output_behind": stepped, "all_files_written_s": done})
    s.close()
    return out


SCENES = {  # bench scene -> dam-break fluid block and box (cells); 3 wall layers, l0 = 0.005 m
    "dam": ((100, 100, 200), (300, 100, 240)),
    "dam_mid": ((80, 80, 160), (240, 80, 192)),   # the 1 M-fluid scaled dam break (benchmark config 5)
    "dam_small": ((40, 40, 80), (120, 40, 96)),
}


def make_scene(args, rank):
    from mphexplicit_b200 import scenes
    if args.scene not in SCENES:
        raise SystemExit("unknown scene " + args.scene)
    fluid, box = SCENES[args.scene]
    return scenes.dam_break_3d(fluid=fluid, box=box, seed=rank)


def workload_name(fluid, box, walls, l0, n, n_fluid) -> str:
    return ("dam_break_3d fluid %dx%dx%d in a %dx%dx%d-cell box, %d wall layers, l0=%g: %d particles (%d fluid)"
            % (*fluid, *box, walls, l0, n, n_fluid))


def scene_workload(sc) -> str:
    m = sc.meta
    return workload_name(m["fluid"], m["box"], m["walls"], m["l0"], sc.n, sc.n_fluid)


def bench_config(workload: str, mode: str) -> dict:
    """The `config` object, identical in the product's line and the reference
    arm's line for the same workload and arithmetic."""
    return {"workload": workload, "form": mode,
            "arithmetic": "fp64 (the reference's)" if mode == "fp64" else "fp32 pairs + fp64 integration",
            "l2": "inputs larger than L2 (particle state and neighbour lists, several GB)"}


def cpu_reference_sample(args, threads: int, steps: int, warmup: int, budget: float, rebuild_at: int):
    """The reference's own step (oracle/_ref/ref_mph3d, OpenMP) on the bench
    scene, written by oracle/ref_inputs (nothing of the product is loaded):
    `warmup` untimed steps, then up to `steps` timed steps (stopping after the
    step that crosses `budget` seconds), the `rebuild_at`-th of which rebuilds
    the cell and neighbour lists (the developed flow rebuilds about every 20
    steps; a dam break at rest does not for its first few hundred)."""
    from oracle import ref_inputs as RI
    fluid, box = SCENES[args.scene]
    with tempfile.TemporaryDirectory() as td:
        d, g, n, nf = RI.dam_break_files(td, seed=0, fluid=fluid, box=box)
        if not RI.ref_available(3):
            raise SystemExit("oracle/_ref/ref_mph3d is missing: build it with `make -C oracle ref REF=<reference>`")
        r = RI.time_reference(d, g, 3, warmup, steps, threads, max_seconds=budget, timeout=3600,
                              rebuild_at=rebuild_at)
    r["workload"] = workload_name(fluid, box, 3, 0.005, n, nf)
    r["value"] = r["fluid"] * r["steps"] / r["seconds"]
    return r


def cpu_baseline_entry(r, cores) -> dict:
    return {"value": r["value"], "unit": UNIT, "cores": r["threads"], "kind": "reference",
            "physical_cores": cores["physical"], "logical_cpus": cores["logical"], "cpu_model": cores["model"],
            "sample": "%d timed step(s) after %d warm-up step(s) of the full %d-particle scene (%d fluid), "
                      "%d neighbour rebuild(s) inside the window, %.1f s wall, %d OpenMP thread(s); "
                      "the reference's Mph_gcc3d flags (-O3 -fopenmp), compiled from its sources"
                      % (r["steps"], r["warmup"], r["particles"], r["fluid"], r["rebuilds"], r["seconds"],
                         r["threads"])}


def run_reference_arm(args, rank, world):
    """`--impl reference`: the reference's own CPU step on this line's workload,
    all host threads, exactly --steps timed steps after --warmup untimed ones,
    with one neighbour rebuild inside the window; then one step on one thread.
    Rank 0 alone runs it (the other ranks exit without work)."""
    if rank != 0:
        return
    from oracle import ref_inputs as RI
    cores = RI.host_cores()
    r = cpu_reference_sample(args, cores["logical"], args.steps, args.warmup, 1.0e30, args.steps // 2)
    base = cpu_baseline_entry(r, cores)
    if args.ref_single_steps > 0:
        r1 = cpu_reference_sample(args, 1, args.ref_single_steps, 0, 1.0e30, -1)
        base["single_thread"] = {"value": r1["value"], "unit": UNIT, "steps": r1["steps"],
                                 "seconds": r1["seconds"], "rebuilds": r1["rebuilds"]}
        base["thread_speedup"] = r["value"] / r1["value"]
    ms = r["seconds"] * 1e3 / r["steps"]
    line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": r["steps"], "warmup": r["warmup"], "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": bench_config(r["workload"], "fp64"), "parallelism": "host CPU (OpenMP)",
            "cpu_baseline": base,
            "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def measure_form(args, sc, mode, world, gpu_index, with_e2e):
    """Time one form of the step on the bench scene: device-resident timed
    region (CUDA events on the library stream), per-kernel events, clocks;
    optionally the end-to-end path with host buffers."""
    import torch
    import torch.distributed as dist
    import mphexplicit_b200 as M
    s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=sc.dim, mode=mode)
    if args.preroll > 0:  # untimed: start the timed window inside the developed flow
        s.step(args.preroll)
    warm = max(args.warmup, 3)
    s.step(warm)
    s.synchronize()
    stream = torch.cuda.ExternalStream(s.stream_handle)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    info0 = s.info()  # before the profiled window: it may compute output-only fields
    torch.cuda.synchronize()
    s.profile(True)
    l0 = s.launch_count()
    with ClockSampler(gpu_index) as clk:
        ev0.record(stream)
        s.step(args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = s.launch_count() - l0
    prof = s.profile_read()
    s.profile(False)
    info1 = s.info()
    ms = max_over_ranks(ms, world)
    st = s.state()  # after warm + steps, for the cross-form error
    order = np.argsort(st["particle_index"], kind="stable")
    vel = st["vel"][order]
    fluid = st["type"][order] < 2
    n_fluid, n_all = sc.n_fluid, sc.n
    out = {"mode": mode, "ms": ms, "value": job_value(n_fluid, args.steps, world, ms), "launches": launches,
           "prof": prof, "clocks": clk.summary(), "rebuilds": info1["rebuild_count"] - info0["rebuild_count"],
           "vel": vel, "fluid": fluid}
    # roofline of the dominant kernel: algorithmic bytes per particle the
    # kernel updates (FP64 state, neighbour re-reads on chip) over its time per
    # step (every launch of that kernel in the step counts)
    name, (nl, tot_ms) = max(prof.items(), key=lambda kv: kv[1][1])
    avg_s = tot_ms / args.steps / 1e3
    peak, peak_kind = measured_peaks()
    units = n_fluid if name in ("mix_sweep_b", "sweep_b") else n_all  # the force sweeps update the fluid
    algo = ALGO_BYTES.get(name, 0.0) * units
    achieved = algo / avg_s / 1e9
    out["roofline"] = {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                       "frac": achieved / peak, "traffic": ncu_traffic(name, mode) if args.scene == "dam" else None,
                       "compute_bound": ncu_pipe(name), "peak_source": peak_kind,
                       "algorithmic_bytes_per_step": algo, "particles_per_step": units,
                       "launches_per_step": nl / args.steps, "ms_per_step": avg_s * 1e3,
                       "kernels_ms_per_step": {k: v[1] / args.steps for k, v in prof.items()}}
    if with_e2e:
        ke = max(1, args.e2e_steps)
        hx = torch.empty((n_all, 3), dtype=torch.float64, pin_memory=True).numpy()
        hv = torch.empty((n_all, 3), dtype=torch.float64, pin_memory=True).numpy()
        s.get_xv(hx, hv)

        def one(overlapped):
            s.set_state(hx, hv)
            if overlapped:
                s.step_read_state(1, hx, hv)  # copies overlap the step's sweeps
            else:
                s.step(1)
                s.get_xv(hx, hv)

        def host_loop(overlapped):
            # every step: the state from pinned host buffers, one step, the
            # state back into them (the public calls a host-resident caller
            # makes); one untimed round first (its first call makes the copy
            # stream and buffer)
            one(overlapped)
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ev0.record(stream)
            for _ in range(ke):
                one(overlapped)
            ev1.record(stream)
            torch.cuda.synchronize()
            ms = max(ev0.elapsed_time(ev1), (time.perf_counter() - t0) * 1e3)
            return max_over_ranks(ms, world)

        serial_ms = host_loop(False)
        e2e_ms = host_loop(True)
        out["e2e"] = {"value": job_value(n_fluid, ke, world, e2e_ms), "unit": UNIT,
                      "h2d_bytes_per_step": int(hx.nbytes + hv.nbytes),
                      "d2h_bytes_per_step": int(hx.nbytes + hv.nbytes), "steps": ke, "mode": mode,
                      "api": "mph_set_state + mph_step_read_state",
                      "ms_per_step": e2e_ms / ke,
                      "step_then_read": {"api": "mph_set_state + mph_step + mph_get_state",
                                         "value": job_value(n_fluid, ke, world, serial_ms),
                                         "ms_per_step": serial_ms / ke}}
    s.close()
    return out


DEFAULT_FORMS = "fp64,mixed,mixed_p64,mixed_walk,learned,batch,two_fluid,droplet,output"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--mode", default="fp64", choices=["fp64", "mixed", "mixed_p64", "mixed_walk"],
                    help="headline form (default fp64: the reference's arithmetic, bit-exact); "
                         "all three are measured unless --only")
    ap.add_argument("--only", action="store_true", help="measure the headline form only")
    ap.add_argument("--scene", default="dam", choices=sorted(SCENES))
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--droplet-steps", type=int, default=1000, help="steps of the 2-D droplet (config 1)")
    ap.add_argument("--forms", default=None,
                    help="forms to measure (comma list; the headline --mode must be among them for a full line); "
                         "default: all of " + DEFAULT_FORMS + " on one GPU, the headline form alone on several "
                         "(the replicas' scaling line, the GPUs held for its timed steps only)")
    ap.add_argument("--learned-fluid", default="80,80,160", help="fluid block of the learned form's dam break")
    ap.add_argument("--learned-steps", type=int, default=1000)
    ap.add_argument("--learn-steps", type=int, default=2000, help="FP64 steps of training data")
    ap.add_argument("--learn-epochs", type=int, default=30)
    ap.add_argument("--batch-steps", type=int, default=2000)
    ap.add_argument("--output-every", type=int, default=100, help="steps between VTK files written behind the step")
    ap.add_argument("--output-files", type=int, default=5)
    ap.add_argument("--two-fluid-n", type=int, default=200, help="fluid particles per axis of the two-fluid column")
    ap.add_argument("--two-fluid-steps", type=int, default=500)
    ap.add_argument("--two-fluid-ref-seconds", type=float, default=20.0,
                    help="budget of the reference's timed sample on the two-fluid column (0: skip)")
    ap.add_argument("--batch-check", type=int, default=16, help="scenes checked against the FP64 form")
    ap.add_argument("--batch-cpu-scenes", type=int, default=16)
    ap.add_argument("--batch-cpu-steps", type=int, default=200)
    ap.add_argument("--preroll", type=int, default=500,
                    help="untimed steps before the warm-up, so the timed window sees the neighbour "
                         "rebuilds of the developed flow (a dam break at rest rebuilds rarely)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-seconds", type=float, default=30.0,
                    help="wall-clock bound of the cpu_baseline sample of the product's line")
    ap.add_argument("--ref-single-steps", type=int, default=1,
                    help="steps of the reference arm's one-thread figure (0: none)")
    args = ap.parse_args()
    rank, world, local = dist_env()

    import torch
    import torch.distributed as dist
    if world > 1:
        dist.init_process_group("nccl" if args.impl == "b200" else "gloo",
                                timeout=__import__("datetime").timedelta(seconds=600))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        if world > 1:
            dist.destroy_process_group()
        return

    torch.cuda.set_device(local)
    gpu_index = local
    cvd = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    if cvd and "," not in cvd and cvd.isdigit():
        gpu_index = int(cvd)
    sc = make_scene(args, rank)
    forms_arg = args.forms if args.forms is not None else (DEFAULT_FORMS if world == 1 else args.mode)
    wanted = [args.mode] if args.only else [f.strip() for f in forms_arg.split(",") if f.strip()]
    modes = [m for m in ("fp64", "mixed", "mixed_p64", "mixed_walk") if m in wanted]
    res = {m: measure_form(args, sc, m, world, gpu_index, with_e2e=(m == args.mode)) for m in modes}
    forms = {}
    for m, r in res.items():
        f = {"value": r["value"], "ms_per_step": r["ms"] / args.steps, "dominant_kernel": r["roofline"]["kernel"],
             "kernels_ms_per_step": r["roofline"]["kernels_ms_per_step"], "rebuilds_in_timed_region": r["rebuilds"],
             "roofline_frac": r["roofline"]["frac"]}
        if "fp64" in res and m != "fp64":
            ref = res["fp64"]
            fl = ref["fluid"]
            f["rel_l2_vel_vs_fp64"] = float(np.linalg.norm(r["vel"][fl] - ref["vel"][fl]) /
                                           np.linalg.norm(ref["vel"][fl]))
            f["error_steps"] = args.preroll + max(args.warmup, 3) + args.steps
            f["speedup_vs_fp64"] = ref["ms"] / r["ms"]
        forms[m] = f

    if "learned" in wanted:
        forms["learned"] = measure_learned(args, rank)
    if "batch" in wanted:
        forms["batch"] = measure_batch(args, rank)
    if "two_fluid" in wanted:
        forms["two_fluid"] = measure_two_fluid(args, rank)
    if "droplet" in wanted:
        forms["droplet"] = measure_droplet(args, rank)
    if "output" in wanted:
        forms["output"] = measure_output(args, sc, rank)
    if args.mode not in res:  # a run of the extra forms alone (profiling)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "unit": UNIT, "n_gpus": world, "forms": forms}), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return
    head = res[args.mode]

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import ref_inputs as RI
        cores = RI.host_cores()
        # bounded sample: the steps that fit in --ref-seconds, the first of them a neighbour rebuild
        base = cpu_baseline_entry(cpu_reference_sample(args, cores["logical"], 1000, 1, args.ref_seconds, 0), cores)

    if rank == 0:
        n_all = sc.n
        warm = max(args.warmup, 3)
        line = {"metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": warm, "ms_per_step": head["ms"] / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.mode == "fp64" else "f32+f64",
                "data": "synthetic (seeded generator)",
                "config": bench_config(scene_workload(sc), args.mode),
                "parallelism": "replicas (one scene per GPU)" if world > 1 else "single GPU",
                "timed_window": "steps %d-%d of the run (%d untimed steps, %d warm-up), %d neighbour rebuild(s)"
                                % (args.preroll + warm + 1, args.preroll + warm + args.steps, args.preroll, warm,
                                   head["rebuilds"]),
                "updates_all_particles_per_s": n_all * args.steps * world / (head["ms"] / 1e3),
                "forms": forms, "roofline": head["roofline"], "cpu_baseline": base, "e2e": head["e2e"],
                "gpu_launches": head["launches"], "clocks": head["clocks"]}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
