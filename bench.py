"""Benchmark: Brownian-dynamics particle-steps/s on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config 4] [--precision f32c|f64]

A "step" is one Brownian-dynamics step of the whole workload (all systems of
the batch): pair forces, external forces, the Euler-Maruyama update with
Philox noise and whatever neighbour bookkeeping the step needs.  With the
neighbour search the autotuner picks (rdgpu_autotune, outside the timed
region) that is either the cell walk (step kernel + counting sort) or the
pair list (step kernel + a check of the particles that moved more than about
skin/2 + a conditional re-sort and list build when that check finds a pair
missing from the list).  The default workload is the
batched ensemble (512 periodic systems, N log-uniform in [500, 20000],
2.45 M particles), the configuration the FP32-batched-vs-FP64 metric is
quoted on.

value: particle-steps/s with the state resident in HBM, device-timed with CUDA
       events on the engine's stream (max over ranks).  The per-step state
       (2.45 M x 64 B = 157 MB read+written) exceeds the 126 MB L2.
e2e:   the same metric through the C ABI with host buffers: every frame of
       100 steps uploads the particles from pinned host memory
       (rdgpu_set_particles, FP32 coordinates for the FP32C engine as the
       reference's float frames, FP64 for the FP64 engine), steps, and
       downloads them (rdgpu_get_particles),
       the per-frame traffic of the reference's JNI frame loop.
plain_f64: the metric's denominator, the plain FP64 single-system path:
       every system of the workload alone in its own FP64 handle.
--impl reference: the CPU path of the reference semantics (the C oracle port,
       all host threads, the reference's Java core cannot run here) on a
       bounded sample of the same workload.
Multi-GPU: replicas only (independent replicate ensembles, one per rank, no
data-path collective); value sums all ranks' particle-steps over the slowest
rank's time.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

ALG_BYTES = {"f32c": 64, "f64": 64}   # state read + written per particle-step


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=200)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", type=int, default=4)
    p.add_argument("--precision", default="f32c", choices=["f32c", "f64"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--neighbour", default="auto", choices=["auto", "cells", "list"])
    p.add_argument("--skin", type=float, default=0.0)

    return p.parse_args()


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_per_particle(prec, config, mode):
    """DRAM bytes per particle-step of the step kernel from the committed ncu
    summary (profiles/step_kernel_traffic.json), scaled to this launch."""
    path = os.path.join(ROOT, "profiles", "step_kernel_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d[f"{prec}_config{config}_{mode}"]["bytes_per_particle_step"]
    except Exception:
        return None


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([v.strip() for v in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = sorted(float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit())
        mx = max((float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = [names[k] for k in range(4) if any(s[2 + k].lower() == "active" for s in self.samples)]
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(self.samples)}


def dist_env():
    from readdygpu_b200 import replicas
    return replicas.env()


def workload(config, reference=False):
    """The benchmark input.  Building it maps no library of the engine
    (readdygpu_b200 loads libreaddy_b200.so on first use only); the reference
    arm takes config 3's insertion from the oracle, which gives the same
    coordinates as the engine package's generator."""
    from readdygpu_b200 import configs
    if config == 3 and reference:
        from oracle import oracle as O
        return configs.config3(rsa=O.rsa_spheres)
    return configs.CONFIGS[config]()


def bench_config(w, ws):
    """The `config` object of the JSON line, the same in both arms."""
    alg = 64 * w.n
    return {"workload": w.name, "particles": w.n, "systems": len(w.boxes) if w.boxes else 1,
            "parallelism": f"replicas{ws}",
            "l2": "inputs larger than L2 (state read+written per step exceeds 126 MB)" if alg > 126e6
            else "state fits in L2"}


def cpu_baseline(w, budget_s=12.0, threads=None):
    """The oracle (C port of the reference CPU semantics) on a bounded sample of
    the workload: its systems in order, a few steps each, repeated until about
    budget_s seconds of CPU work; OpenMP over all host threads, Philox noise,
    particle-steps/s."""
    from oracle import oracle as O
    threads = threads or O.max_threads()
    d0 = w.system.to_desc()
    if w.boxes is None:
        systems = [(d0, w.xyz, w.types)]
    else:
        systems = []
        for k, (lo, hi, per, sd) in enumerate(w.boxes):
            d = w.system.to_desc()
            for a in range(3):
                d.lo[a], d.hi[a], d.periodic[a] = lo[a], hi[a], per[a]
            a_, b_ = w.offsets[k], w.offsets[k + 1]
            systems.append((d, w.xyz[a_:b_], w.types[a_:b_]))
    done = 0
    visits = 0
    steps = 2
    rel = [O.to_rel_f64(d, xyz) for (d, xyz, ty) in systems]
    t0 = time.perf_counter()
    while True:
        for k, (d, xyz, ty) in enumerate(systems):
            rel[k], _ = O.run_steps(d, rel[k], ty, 7, visits * steps, steps, threads)
            done += len(ty) * steps
        visits += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    npart = sum(len(ty) for (_, _, ty) in systems)
    return {"value": done / dt, "unit": "particle-steps/s", "cores": threads, "kind": "port",
            "sample": f"all {len(systems)} systems ({npart} particles) x {visits * steps} steps, "
                      f"C oracle, {threads} OpenMP threads, {dt:.1f} s"}


def rdf_frames(eng, nbins=200, rmax=20.0, frames=5, every=100):
    """The RDF of config 3 (200 bins over 0-20 nm, one frame every 100 steps)
    through the C ABI: the particles sorted into the RDF's grid, histogram
    kernel, counts to the host; wall time of whole synchronous calls after one
    untimed frame."""
    eng.rdf(nbins, rmax)
    t0 = time.perf_counter()
    for _ in range(frames):
        eng.rdf(nbins, rmax)
    ms = (time.perf_counter() - t0) * 1e3 / frames
    return {"bins": nbins, "rmax_nm": rmax, "every_steps": every, "ms_per_frame": ms,
            "ms_per_step_amortized": ms / every,
            "note": "rdgpu_rdf: particles sorted into the RDF grid, rdf_rows_kernel, uint64 counts to the host"}


def host_cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def plain_f64(w, local, steps=200):
    """The plain FP64 single-system GPU path (the drop-in): every system of the
    batch alone in its own FP64 handle with default options (autotuned
    before timing), stepped `steps` steps after as many warm-up steps; the
    particle-steps/s of running them one after another, device-timed."""
    import numpy as np
    import torch
    import readdygpu_b200 as R
    picks = [None] if w.boxes is None else list(range(len(w.boxes)))
    ps, ms, npart = 0.0, 0.0, 0
    for k in picks:
        if k is None:
            eng = R.Engine(w.system, precision="f64", device=local, seed=3)
            xyz, ty, off = w.xyz, w.types, None
        else:
            eng = R.Engine(w.system, precision="f64", device=local, boxes=[w.boxes[k]])
            a_, b_ = int(w.offsets[k]), int(w.offsets[k + 1])
            xyz, ty, off = w.xyz[a_:b_], w.types[a_:b_], np.array([0, b_ - a_], np.int64)
        eng.set_particles(xyz, ty, offsets=off)
        eng.autotune()
        eng.step(steps)
        st = torch.cuda.ExternalStream(eng.stream, device=local)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        eng.step(steps)
        e1.record(st)
        e1.synchronize()
        ms += e0.elapsed_time(e1)
        ps += len(ty) * steps
        npart += len(ty)
        eng.close()
    return {"value": ps / (ms / 1e3), "unit": "particle-steps/s", "systems": len(picks), "particles": npart,
            "steps": steps,
            "sample": f"all {len(picks)} systems of the workload, each alone in an FP64 handle, {steps} timed "
                      f"steps each"}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    w = workload(args.config, reference=True)
    cb = cpu_baseline(w, budget_s=20.0)
    cb["cpu_model"] = host_cpu_model()
    line = {"impl": "reference", "metric": "particle-steps/s", "value": cb["value"], "unit": "particle-steps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(w, ws),
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "reference CPU semantics via the C oracle port; the reference's own Java core needs a JVM, "
                    "which this image lacks"}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import numpy as np
    import torch
    import readdygpu_b200 as R

    from readdygpu_b200 import replicas
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    replicas.init("nccl")
    w = workload(args.config)
    kw = {}
    if w.boxes is not None:
        # each rank owns its own replicate ensemble: shift the seeds
        kw["boxes"] = replicas.replica_boxes(w.boxes, rank)
    eng = R.Engine(w.system, precision=args.precision, device=local, seed=replicas.replica_seed(11, rank),
                   neighbour_mode=args.neighbour, skin=args.skin, **kw)
    eng.set_particles(w.xyz, w.types, offsets=w.offsets)
    stream = torch.cuda.ExternalStream(eng.stream, device=local)
    eng.autotune()          # outside the timed region
    eng.step(args.warmup)
    nb = eng.metrics()

    def barrier():
        replicas.barrier()

    # ---- device-timed, state resident in HBM ----------------------------
    l0 = eng.launch_count()
    barrier()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        ev0.record(stream)
        eng.step(args.steps)
        ev1.record(stream)
        ev1.synchronize()
    barrier()
    launches = eng.launch_count() - l0
    ms = ev0.elapsed_time(ev1)
    # the dominant kernel alone: CUDA events around each fused step-kernel launch
    kernel_ms, sort_ms = eng.step_profile(min(100, max(10, args.steps // 5)))
    ms_max = replicas.max_over_ranks(ms, f"cuda:{local}")
    n_all = w.n * ws
    value = replicas.job_rate(w.n, ws, args.steps, ms_max / 1e3)
    ms_step = ms_max / args.steps
    per_launch_s = kernel_ms / 1e3
    alg = ALG_BYTES[args.precision] * w.n
    peak, peak_kind = measured_peak_hbm()
    achieved = alg / per_launch_s / 1e9
    tpp = traffic_per_particle(args.precision, args.config, nb["neighbour_mode"])

    # ---- end to end through the C ABI with host buffers ------------------
    e2e = None
    if not args.no_e2e:
        frame = 100
        frames = max(1, min(20, args.steps // frame))
        # pinned host buffers, as a host application would keep them; FP32
        # coordinates for the FP32C engine (the reference moves float frames,
        # ReaDDyGPU.cpp:264-292), FP64 for the FP64 engine
        xdt = torch.float32 if args.precision == "f32c" else torch.float64
        xh = torch.empty((w.n, 3), dtype=xdt, pin_memory=True).numpy()
        th = torch.empty(w.n, dtype=torch.int32, pin_memory=True).numpy()
        eng.get_particles(xh, th)
        barrier()
        t0 = time.perf_counter()
        for _ in range(frames):
            eng.set_particles(xh, th, offsets=w.offsets)
            eng.step(frame)
            eng.get_particles(xh, th)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        dt = replicas.max_over_ranks(dt, f"cuda:{local}")
        xb = xh.itemsize
        h2d = w.n * (3 * xb + 4) + (len(w.offsets) * 8 if w.offsets is not None else 0)
        d2h = w.n * (3 * xb + 4)
        e2e = {"value": n_all * frame * frames / dt, "unit": "particle-steps/s",
               "h2d_bytes_per_step": h2d / frame, "d2h_bytes_per_step": d2h / frame,
               "frame_steps": frame, "frames": frames,
               "coords": "float32" if xb == 4 else "float64",
               "note": "per frame: pinned-host upload + re-binning, 100 steps, download"}

    cb = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(w)
        # the same oracle on one host thread, and the host CPU model
        cb["single_thread"] = cpu_baseline(w, budget_s=4.0, threads=1)["value"]
        cb["cpu_model"] = host_cpu_model()
    rdf = None
    if rank == 0 and args.config == 3:
        rdf = rdf_frames(eng)
    plain = None
    if rank == 0 and not args.no_plain:
        plain = plain_f64(w, local)
    if rank == 0:
        line = {"metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.precision == "f32c" else "f64",
                "data": "synthetic",
                "config": bench_config(w, ws), "precision": args.precision,
                "neighbour": {"mode": nb["neighbour_mode"], "skin_nm": nb["skin"], "requested": args.neighbour},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "peak_kind": peak_kind,
                             "traffic": (tpp * w.n if tpp else None),
                             "kernel": "list_step_kernel" if nb["neighbour_mode"] == "list" else "step_kernel",
                             "kernel_ms": kernel_ms, "sort_ms": sort_ms,
                             "alg_bytes_per_particle_step": ALG_BYTES[args.precision]},
                "e2e": e2e, "cpu_baseline": cb, "gpu_launches": launches, "clocks": clk.summary(),
                "plain_f64": plain, "vs_plain_f64": (value / ws / plain["value"]) if plain else None}
        if rdf:
            line["rdf"] = rdf
        print(json.dumps(line), flush=True)
    eng.close()
    replicas.finalize()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
