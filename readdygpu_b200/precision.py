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


def _block_mean(v, blocks=10):
    """Mean of a time series and its standard error from block averages."""
    v = np.asarray(v, dtype=np.float64)
    nb = max(2, min(blocks, len(v)))
    parts = np.array_split(v, nb)
    m = np.array([p.mean() for p in parts])
    return float(v.mean()), float(m.std(ddof=1) / np.sqrt(nb))


def long_run(w, steps, samples=100, seed=1, rdf_bins=150, rdf_rmax=15.0, equil=0.1, **kw):
    """The long-run precision study: the FP32C and the FP64 engine stepped side
    by side from the same positions with the same Philox keys, sampled every
    steps / samples steps.  At each sample:

    * potential energy of both runs;
    * MSD per species from the unwrapped displacement since the start
      (MsdComputer.java:114-213 takes the first-seen position as the origin),
      with its standard error over particles;
    * the force error of the FP32C engine against the FP64 engine on the FP32C
      run's current positions (snapped to the FP32 grid);
    * one RDF frame of each run (accumulated counts).

    Statistical comparison (the two runs share the noise, so their
    differences are far below these bounds while the trajectories stay close,
    and the bounds hold after they decorrelate):

    * energy: the means over the samples after the first `equil` fraction,
      |E32 - E64| <= 3 sqrt(se32^2 + se64^2) (block standard errors);
    * D = MSD / 6t per species at the first sample and at the end:
      |D32 - D64| <= 3 sqrt(se32^2 + se64^2) (standard errors over
      particles);
    * RDF: the per-frame counts of every bin, averaged in blocks of frames;
      chi2 / dof = mean over bins of (m32 - m64)^2 / (se32^2 + se64^2) (block
      standard errors, bins with counts) <= 1.5.  Under the hypothesis
      that both runs sample the same distribution, with 10 blocks, chi2 / dof
      is 1.29 on average (t statistics with 9 degrees of freedom) and 1.5 is
      more than 3 standard deviations above that for >= 100 bins; the
      largest |z| of a single bin is reported too.
    """
    x0 = snap_to_f32(w)
    every = max(1, steps // samples)
    S = w.system.n_types
    eng = {}
    for prec in ("f32c", "f64"):
        eng[prec] = _engine(w, prec, seed, **kw)
        eng[prec].set_particles(x0, w.types, offsets=w.offsets)
        eng[prec].autotune()
    probe = {prec: _engine(w, prec, seed) for prec in ("f32c", "f64")}
    rec = {p: {"t": [], "E": [], "msd": [], "msd_se": []} for p in eng}
    ferr = []
    done = 0
    rdf_frames = {p: [] for p in eng}
    try:
        while done < steps:
            n = min(every, steps - done)
            for prec, e in eng.items():
                e.step(n)
            done += n
            for prec, e in eng.items():
                m = e.metrics()
                xe, _ = e.get_particles()
                if w.boxes is not None or any(w.system.periodic):
                    # periodic axes: the engine's image-unwrapped MSD (no per-particle spread)
                    msd = np.array(m["msd"][:S])
                    se = np.zeros(S)
                else:
                    # an open box: positions are unwrapped as they are
                    d2 = ((xe - x0) ** 2).sum(axis=1)
                    msd = np.array([d2[w.types == t].mean() for t in range(S)])
                    se = np.array([d2[w.types == t].std(ddof=1) / np.sqrt(max(1, (w.types == t).sum()))
                                   for t in range(S)])
                r = rec[prec]
                r["t"].append(done); r["E"].append(m["energy"]); r["msd"].append(msd); r["msd_se"].append(se)
                c, _ = e.rdf(rdf_bins, rdf_rmax, accumulate=False)
                rdf_frames[prec].append(c.reshape(-1).astype(np.float64))
                if prec == "f32c":
                    xs = xe
            # force error on the FP32C run's current positions
            F = {}
            xsn = snap_to_f32(_with_xyz(w, xs))
            for prec, e in probe.items():
                e.set_particles(xsn, w.types, offsets=w.offsets)
                F[prec], _ = e.forces()
            nrm = np.linalg.norm(F["f64"])
            ferr.append(float(np.linalg.norm(F["f32c"] - F["f64"]) / nrm) if nrm > 0 else 0.0)
    finally:
        for e in list(eng.values()) + list(probe.values()):
            e.close()
    dt = w.system.dt
    out = {"steps": steps, "sample_every": every, "samples": len(ferr),
           "force_rel_err_max": max(ferr), "force_rel_err_mean": float(np.mean(ferr))}
    k0 = int(equil * len(ferr))
    E = {}
    for prec in eng:
        E[prec] = _block_mean(rec[prec]["E"][k0:])
        t = np.array(rec[prec]["t"], dtype=np.float64)
        out[f"energy_mean_{prec}"], out[f"energy_se_{prec}"] = E[prec]
        out[f"energy_drift_per_step_{prec}"] = float(np.polyfit(t[k0:], rec[prec]["E"][k0:], 1)[0])
    dE = abs(E["f32c"][0] - E["f64"][0])
    out["energy_abs_dev"] = dE
    out["energy_bound_3sigma"] = 3.0 * float(np.hypot(E["f32c"][1], E["f64"][1]))
    for tag, k in (("first", 0), ("end", len(ferr) - 1)):
        T = rec["f64"]["t"][k] * dt
        D = {p: np.array(rec[p]["msd"][k]) / (6.0 * T) for p in eng}
        se = {p: np.array(rec[p]["msd_se"][k]) / (6.0 * T) for p in eng}
        out[f"D_{tag}_f32c"] = [float(v) for v in D["f32c"]]
        out[f"D_{tag}_f64"] = [float(v) for v in D["f64"]]
        out[f"D_{tag}_abs_dev"] = [float(v) for v in np.abs(D["f32c"] - D["f64"])]
        out[f"D_{tag}_bound_3sigma"] = [float(v) for v in 3.0 * np.hypot(se["f32c"], se["f64"])]
        out[f"D_{tag}_rel_dev"] = [float(v) for v in np.abs(D["f32c"] - D["f64"]) / np.maximum(np.abs(D["f64"]), 1e-300)]
    out["rdf_bins"] = rdf_bins
    out["rdf_rmax_nm"] = rdf_rmax
    out["rdf_pairs_counted"] = float(np.sum(rdf_frames["f64"]))
    mb, sb = {}, {}
    for prec in eng:
        fr = np.array(rdf_frames[prec])
        nb = max(2, min(10, len(fr)))
        blocks = np.array([b.mean(axis=0) for b in np.array_split(fr, nb)])
        mb[prec] = fr.mean(axis=0)
        sb[prec] = blocks.std(axis=0, ddof=1) / np.sqrt(nb)
    var = sb["f32c"] ** 2 + sb["f64"] ** 2
    sel = var > 0
    z2 = (mb["f32c"][sel] - mb["f64"][sel]) ** 2 / var[sel]
    out["rdf_bins_compared"] = int(sel.sum())
    out["rdf_chi2_per_dof"] = float(z2.mean()) if z2.size else 0.0
    out["rdf_max_abs_z"] = float(np.sqrt(z2.max())) if z2.size else 0.0
    both_zero = (~sel) & (mb["f32c"] != mb["f64"])
    out["rdf_bins_differing_without_spread"] = int(both_zero.sum())
    return out


def _with_xyz(w, xyz):
    from .configs import Workload
    return Workload(w.name, w.system, xyz, w.types, w.steps, boxes=w.boxes, offsets=w.offsets)


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
    p.add_argument("--long", action="store_true",
                   help="the long-run study (long_run): both precisions side by side, --frames samples")
    a = p.parse_args()
    if a.long:
        from . import configs
        if a.config == 5 and a.particles:
            w = configs.config5(n=a.particles, n_shell=max(1, round(0.06 * a.particles)))
        elif a.particles:
            w = configs.CONFIGS[a.config](n=a.particles)
        else:
            w = configs.CONFIGS[a.config]()
        out = {"workload": w.name, "particles": int(len(w.types))}
        out.update(long_run(w, a.steps, a.frames, a.seed))
        print(json.dumps(out), flush=True)
        return
    print(json.dumps(study(a.config, a.particles or None, a.steps, a.frames, a.seed)), flush=True)


if __name__ == "__main__":
    main()
