#!/usr/bin/env python3
"""Long-run precision comparison: the same seeded channel advanced in FP64,
FP32 and FP16 storage, with time-averaged statistics compared against the
FP64 run (the FP64 kernel is bit-identical to the CPU oracle).

    python dns-solvers_b200/longrun.py --workload channel180 --spinup 20000 \
        --steps 50000 --sample 100 --out longrun.json

Turbulence is chaotic: two runs that start apart by a small amount drift
apart exponentially, and once decorrelated their window averages differ by
the sampling error of the window.  The control run "64p" (FP64 from the same
field with every population multiplied by 1 + amp * N(0, 1), amp =
--control-amp, seeded) measures that floor for an initial difference of the
size of FP32 rounding (amp 1e-7); an FP32/FP16 error at the level of the
control's is the flow's sensitivity, not a precision bias.

Averaged over the window (after --spinup steps), per run:
  * the per-step wall shear stress (wshearstr.c:125) -> u_tau = sqrt(tau_w/rho),
    Re_tau = u_tau h / nu (h = zdv/2, nu = (2/omega - 1)/6);
  * the flow rate (encalc.c:132) -> bulk velocity and skin friction
    C_f = 2 tau_w / (rho U_b^2);
  * the plane statistics (statistics.c) sampled every --sample steps and
    averaged on the device (dnslbm_stats_accumulate): mean u(z) and rms
    u'(z), v'(z), w'(z) profiles, rms pooled as the root of the mean square;
  * for textured walls, the mean streamwise velocity in the first fluid plane
    over slip and over no-slip wall cells at the end of the window.
Errors against FP64: max |profile - profile_64| / max |profile_64| and the
relative differences of Re_tau, C_f, U_b.

The window is cut into --blocks equal blocks whose averages are kept: the
spread of the block averages gives each quantity's standard error (batch
means), so a difference is stated with the sampling error it must beat --
"sigma" (the combined standard error of the two runs' averages) and
"z" = |difference| / sigma.  The profiles are also folded about the channel
centre (the two half-channels are statistically the same), which halves
their sampling variance; "*_fold_*" entries use the folded profiles.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import dnslbm  # noqa: E402
import inputs  # noqa: E402


def run_one(wl, s0, flags, prec, spinup, steps, sample, blocks=1, device=0):
    bc = dnslbm.BC_GENERAL if inputs.needs_general(wl) else dnslbm.BC_REFERENCE
    ch = dnslbm.Channel(wl.nx, wl.ny, wl.nz, wl.omega, gx=wl.gx, force_mode=dnslbm.CONST_G, precision=prec,
                        bc_mode=bc, device=device)
    ch.set_flags(flags)
    ch.autotune()
    ch.load_state(s0)
    t0 = time.perf_counter()
    left = spinup
    while left > 0:
        n = min(4000, left)
        ch.step(n)
        left -= n
    nu = (2.0 / wl.omega - 1.0) / 6.0
    h = wl.nz / 2.0
    per_block = steps // blocks
    bq = []  # per block: the scalars and profiles averaged over the block
    for _b in range(blocks):
        stress, flow, rho = [], [], []
        ch.stats_reset()
        done = 0
        while done < per_block:
            n = min(sample, per_block - done)
            first = ch.steps_done
            ch.step(n)
            lg = ch.logs(first, n)
            stress.append(lg[:, dnslbm.LOG_NAMES.index("stress")])
            flow.append(lg[:, dnslbm.LOG_NAMES.index("flowrate")])
            rho.append(lg[:, dnslbm.LOG_NAMES.index("rho")])
            done += n
            ch.stats_accumulate()
        st, _ = ch.stats_average()
        stress, flow, rho = np.concatenate(stress), np.concatenate(flow), np.concatenate(rho)
        tau_w = float(np.mean(stress))
        rho_m = float(np.mean(rho))
        utau = math.sqrt(abs(tau_w) / rho_m)
        ub = float(np.mean(flow)) / (wl.ny * wl.nz)
        bq.append({"tau_w": tau_w, "u_tau": utau, "re_tau": utau * h / nu, "u_bulk": ub,
                   "cf": 2 * tau_w / (rho_m * ub * ub), "mean_u": st[0, 1:-1], "u_rms": st[3, 1:-1],
                   "v_rms": st[4, 1:-1], "w_rms": st[5, 1:-1]})
    secs = time.perf_counter() - t0
    vel, _ = ch.moments()
    ch.close()
    out = summarize(bq, prec, secs)
    slip = flags[:, :, 0] == -2
    if slip.any():
        u1 = vel[:, :, 1, 0]
        out["slip_u_first_plane"] = float(u1[slip].mean())
        out["noslip_u_first_plane"] = float(u1[~slip].mean())
    return out


def summarize(bq, prec, secs):
    """Window averages, batch-means standard errors and folded profiles of
    a run's block averages bq (kept under "block_values" for --save)."""
    blocks = len(bq)
    out = {"precision": prec, "seconds": round(secs, 2), "blocks": blocks,
           "block_values": {k: np.array([b[k] for b in bq]) for k in bq[0]}}
    for k in bq[0]:
        vals = np.array([b[k] for b in bq])
        out[k] = vals.mean(axis=0) if vals.ndim > 1 else float(vals.mean())
        se = vals.std(axis=0, ddof=1) / math.sqrt(blocks) if blocks > 1 else np.zeros_like(vals[0])
        out[k + "_se"] = se if vals.ndim > 1 else float(se)
        if vals.ndim > 1:  # folded about the centre plane
            fv = 0.5 * (vals + vals[:, ::-1])
            out[k + "_fold"] = fv.mean(axis=0)
            out[k + "_fold_se"] = fv.std(axis=0, ddof=1) / math.sqrt(blocks) if blocks > 1 else np.zeros_like(fv[0])
    return out


def save_runs(path, runs):
    """The block averages of every finished run, to compare later runs
    against (--ref)."""
    arrs = {}
    for r in runs:
        if "block_values" not in r:
            continue
        for k, v in r["block_values"].items():
            arrs[f"{r['run']}__{k}"] = v
        arrs[f"{r['run']}__seconds"] = np.array(r["seconds"])
        for k in ("slip_u_first_plane", "noslip_u_first_plane"):
            if k in r:
                arrs[f"{r['run']}__{k}"] = np.array(r[k])
    np.savez(path, **arrs)


def load_runs(path):
    """Runs saved by save_runs, by label."""
    z = np.load(path)
    by = {}
    for name in z.files:
        label, key = name.split("__", 1)
        by.setdefault(label, {})[key] = z[name]
    out = {}
    for label, d in by.items():
        secs = float(d.pop("seconds"))
        extra = {k: float(d.pop(k)) for k in ("slip_u_first_plane", "noslip_u_first_plane") if k in d}
        nb = len(next(iter(d.values())))
        bq = [{k: (v[i] if v.ndim > 1 else float(v[i])) for k, v in d.items()} for i in range(nb)]
        prec = int(label[:2])
        r = summarize(bq, prec, secs)
        r.update(extra)
        r["run"] = label
        r["from"] = os.path.basename(path)
        out[label] = r
    return out


def compare(ref, o):
    def prof(k):
        scale = max(np.max(np.abs(ref[k])), 1e-300)
        d = np.abs(o[k] - ref[k])
        sig = np.sqrt(ref[k + "_se"] ** 2 + o[k + "_se"] ** 2)
        i = int(np.argmax(d))
        return float(d[i] / scale), float(np.max(sig) / scale), float(np.max(d / np.maximum(sig, 1e-300)))
    e = {}
    for k in ("mean_u", "u_rms", "v_rms", "w_rms"):
        for name in (k, k + "_fold"):
            rel, sig, z = prof(name)
            e[f"{name}_max_rel"] = rel
            e[f"{name}_sigma_rel"] = sig
            e[f"{name}_max_z"] = z
    # the folded mean-u profile over the half channel: RMS difference, RMS
    # sampling error, and the mean of (difference / sigma)^2 (about 1 when
    # the difference is sampling noise)
    h = len(ref["mean_u_fold"]) // 2
    scale = max(np.max(np.abs(ref["mean_u"])), 1e-300)
    d = (o["mean_u_fold"] - ref["mean_u_fold"])[:h]
    sig = np.sqrt(ref["mean_u_fold_se"] ** 2 + o["mean_u_fold_se"] ** 2)[:h]
    e["mean_u_fold_rms_rel"] = float(np.sqrt(np.mean(d ** 2)) / scale)
    e["mean_u_fold_rms_sigma_rel"] = float(np.sqrt(np.mean(sig ** 2)) / scale)
    e["mean_u_fold_mean_rel"] = float(np.mean(d) / scale)
    if np.all(sig > 0):
        e["mean_u_fold_chi2_per_plane"] = float(np.mean((d / sig) ** 2))
    for k in ("re_tau", "cf", "u_bulk", "tau_w"):
        e[f"{k}_rel"] = abs(o[k] - ref[k]) / abs(ref[k])
        sig = math.sqrt(ref[k + "_se"] ** 2 + o[k + "_se"] ** 2)
        e[f"{k}_sigma_rel"] = sig / abs(ref[k])
        e[f"{k}_z"] = abs(o[k] - ref[k]) / sig if sig > 0 else float("inf")
    if "slip_u_first_plane" in ref:
        e["slip_u_rel"] = abs(o["slip_u_first_plane"] - ref["slip_u_first_plane"]) / abs(ref["slip_u_first_plane"])
    return e


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="channel180")
    ap.add_argument("--spinup", type=int, default=0, help="steps before the averaging window")
    ap.add_argument("--steps", type=int, default=50000, help="steps in the averaging window")
    ap.add_argument("--sample", type=int, default=100)
    ap.add_argument("--blocks", type=int, default=10, help="window blocks for the standard errors")
    ap.add_argument("--precisions", default="64,64p,32,16",
                    help="64p: FP64 control from a perturbed field (64pA: perturbation amplitude A)")
    ap.add_argument("--control-amp", type=float, default=1e-7, help="relative perturbation of the 64p control")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=None)
    ap.add_argument("--save", default=None, help="write the runs' block averages (.npz) for a later --ref")
    ap.add_argument("--ref", default=None, help="runs saved by --save: a listed run found there is not run again")
    ap.add_argument("--runs-command", default=None, help="the command that made the runs of --ref (recorded)")
    a = ap.parse_args()
    saved = load_runs(a.ref) if a.ref else {}
    wl = inputs.workload(a.workload)
    flags = inputs.make_flags(wl)
    s0 = None  # made when a run is needed (the runs of --ref are not run again)
    runs = []
    for p in a.precisions.split(","):
        if p in saved:
            runs.append(saved[p])
            continue
        if s0 is None:
            s0 = inputs.make_state(wl, seed=a.seed)
            if inputs.needs_general(wl):
                s0 = inputs.rest_solids(s0, flags)
        init = s0
        if p.startswith("64p"):
            amp = float(p[3:]) if len(p) > 3 else a.control_amp
            rng = np.random.default_rng(a.seed + 1)
            init = s0 * (1.0 + amp * rng.standard_normal(s0.shape))
            if inputs.needs_general(wl):
                init = inputs.rest_solids(init, flags)
        try:
            r = run_one(wl, init, flags, int(p[:2]), a.spinup, a.steps, a.sample, a.blocks)
        except dnslbm.DnsLbmError as e:  # e.g. a NaN wall stress: reported, not fatal
            r = {"failed": str(e)}
        r["run"] = p
        runs.append(r)
    ref = runs[0]
    summary = {"workload": wl.name, "grid": f"{wl.nx}x{wl.nz + 2}x{wl.ny}", "texture": wl.texture,
               "command": "python " + " ".join(sys.argv), "spinup": a.spinup, "steps": a.steps, "sample_every": a.sample,
               "blocks": a.blocks, "seed": a.seed, "control_amp": a.control_amp, "runs": []}
    if a.runs_command:
        summary["runs_command"] = a.runs_command
    if inputs.needs_general(wl):
        summary["note"] = ("walls with riblets: the reference's wall-stress formula (a one-sided difference of "
                           "plane means at a flat wall) does not measure the riblet drag; compare u_bulk at "
                           "the common body force")
    if a.save:
        save_runs(a.save, runs)
    for r in runs:
        row = {k: v for k, v in r.items() if not isinstance(v, (np.ndarray, dict))}
        if r is not ref and "failed" not in r and "failed" not in ref:
            row["error_vs_fp64"] = compare(ref, r)
        summary["runs"].append(row)
    if "mean_u" in ref:
        summary["fp64_mean_u_profile"] = ref["mean_u"].tolist()
    txt = json.dumps(summary, indent=1)
    if a.out:
        with open(a.out, "w") as f:
            f.write(txt)
    print(txt)


if __name__ == "__main__":
    main()
