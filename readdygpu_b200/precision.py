"""Precision study: the FP32-compensated engine against the FP64 engine.

For a workload it reports

* force error: FP32C forces against FP64 forces on identical positions (the
  initial positions snapped to the FP32 grid of the box, which both engines
  then store exactly): ||dF|| / ||F|| and the worst particle relative to
  its |F|;
* trajectory deviation: both precisions stepped from those positions with the
  same Philox stream (keyed by seed, step and particle id): the largest and
  the RMS position difference at the end (minimum image);
* energy: the FP64-reduced potential energy of both runs at every frame, the
  largest relative difference, and each run's drift (least-squares slope per
  step);
* diffusion: D per species from the mean squared displacement of both runs at
  the end (MSD / 6 t), and their relative deviation.

The FP64 engine itself is held to the CPU oracle by the parity tests, so these
figures are the FP32C error against FP64.  Command line:

    python -m readdygpu_b200.precision --config 5 --particles 20000 --steps 2000
"""
import argparse
import json

import numpy as np

from .engine import Engine


def snap_to_f32(w):
    """Positions on the FP32 grid of each box: lo + float32(x - lo), wrapped
    into periodic boxes first.  Both precisions store these exactly."""
    x = np.array(w.xyz, dtype=np.float64, copy=True)
    if w.boxes is None:
        spans = [(0, len(x), w.system.lo, w.system.hi, w.system.periodic)]
    else:
        spans = [(int(w.offsets[k]), int(w.offsets[k + 1]), lo, hi, per) for k, (lo, hi, per, _) in enumerate(w.boxes)]
    for a_, b_, lo, hi, per in spans:
        lo = np.array(lo, dtype=np.float64)
        L = np.array(hi, dtype=np.float64) - lo
        rel = x[a_:b_] - lo
        for ax in range(3):
            if per[ax]:
                rel[:, ax] = np.mod(rel[:, ax], L[ax])
        rel = rel.astype(np.float32).astype(np.float64)
        for ax in range(3):
            if per[ax]:
                rel[:, ax] = np.where(rel[:, ax] >= np.float32(L[ax]), 0.0, rel[:, ax])
        x[a_:b_] = lo + rel
    return x


def _engine(w, prec, seed, **kw):
    if w.boxes is None:
        return Engine(w.system, precision=prec, seed=seed, **kw)
    return Engine(w.system, precision=prec, boxes=w.boxes, **kw)


def force_error(w, seed=1, **kw):
    x = snap_to_f32(w)
    out = {}
    F = {}
    for prec in ("f32c", "f64"):
        with _engine(w, prec, seed, **kw) as e:
            e.set_particles(x, w.types, offsets=w.offsets)
            F[prec], out[f"energy_{prec}"] = e.forces()
    d = F["f32c"] - F["f64"]
    nrm = np.linalg.norm(F["f64"])
    per = np.linalg.norm(d, axis=1)
    mag = np.linalg.norm(F["f64"], axis=1)
    out["force_rel_err"] = float(np.linalg.norm(d) / nrm) if nrm > 0 else 0.0
    out["force_max_abs_err"] = float(per.max()) if per.size else 0.0
    sel = mag > 1e-3 * (mag.max() if mag.size else 0.0)
    out["force_max_rel_err_per_particle"] = float((per[sel] / mag[sel]).max()) if sel.any() else 0.0
    out["energy_rel_err"] = float(abs(out["energy_f32c"] - out["energy_f64"]) / max(1e-300, abs(out["energy_f64"])))
    return out


def _min_image(d, w):
    if w.boxes is None:
        L = np.array(w.system.box_lengths())
        per = np.array(w.system.periodic, bool)
        d[:, per] -= L[per] * np.round(d[:, per] / L[per])
        return d
    for k, (lo, hi, p, _) in enumerate(w.boxes):
        a_, b_ = int(w.offsets[k]), int(w.offsets[k + 1])
        L = np.array(hi) - np.array(lo)
        per = np.array(p, bool)
        d[a_:b_][:, per] -= L[per] * np.round(d[a_:b_][:, per] / L[per])
    return d


def trajectory(w, steps, frames=10, seed=1, **kw):
    """Both precisions from the same positions and noise; energy and MSD at
    every frame, positions at the end."""
    x = snap_to_f32(w)
    every = max(1, steps // frames)
    rec = {}
    for prec in ("f32c", "f64"):
        with _engine(w, prec, seed, **kw) as e:
            e.set_particles(x, w.types, offsets=w.offsets)
            en, msd, t = [], [], []
            done = 0
            m = e.metrics()
            en.append(m["energy"]); msd.append(m["msd"]); t.append(0)
            while done < steps:
                n = min(every, steps - done)
                e.step(n)
                done += n
                m = e.metrics()
                en.append(m["energy"]); msd.append(m["msd"]); t.append(done)
            xe, _ = e.get_particles()
        rec[prec] = (np.array(en), np.array(msd), np.array(t), xe)
    en32, msd32, t, x32 = rec["f32c"]
    en64, msd64, _, x64 = rec["f64"]
    dx = _min_image(x32 - x64, w)
    dist = np.linalg.norm(dx, axis=1)
    dt = w.system.dt
    T = steps * dt
    D32 = msd32[-1] / (6.0 * T)
    D64 = msd64[-1] / (6.0 * T)
    denom = np.maximum(np.abs(en64), 1e-300)
    return {
        "steps": steps,
        "position_max_dev_nm": float(dist.max()) if dist.size else 0.0,
        "position_rms_dev_nm": float(np.sqrt(np.mean(dist ** 2))) if dist.size else 0.0,
        "energy_max_rel_dev": float(np.max(np.abs(en32 - en64) / denom)),
        "energy_drift_per_step_f32c": float(np.polyfit(t, en32, 1)[0]) if len(t) > 1 else 0.0,
        "energy_drift_per_step_f64": float(np.polyfit(t, en64, 1)[0]) if len(t) > 1 else 0.0,
        "D_f32c_nm2_per_s": [float(v) for v in D32],
        "D_f64_nm2_per_s": [float(v) for v in D64],
        "D_max_rel_dev": float(np.max(np.abs(D32 - D64) / np.maximum(np.abs(D64), 1e-300))),
    }


def study(config, particles=None, steps=1000, frames=10, seed=1, **kw):
    from . import configs
    if config == 4:
        w = configs.config4(n_systems=particles or 512)
    elif config == 5 and particles:
        # the shell keeps config 5's share of the particles (15,000 of 250,000)
        w = configs.config5(n=particles, n_shell=max(1, round(0.06 * particles)))
    elif particles:
        w = configs.CONFIGS[config](n=particles)
    else:
        w = configs.CONFIGS[config]()
    out = {"workload": w.name, "particles": int(len(w.types))}
    out.update(force_error(w, seed, **kw))
    if steps > 0:
        out.update(trajectory(w, steps, frames, seed, **kw))
    return out


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--config", type=int, default=5)
    p.add_argument("--particles", type=int, default=0, help="particles (config 4: systems); 0: the config's size")
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--frames", type=int, default=10)
    p.add_argument("--seed", type=int, default=1)
    a = p.parse_args()
    print(json.dumps(study(a.config, a.particles or None, a.steps, a.frames, a.seed)), flush=True)


if __name__ == "__main__":
    main()
