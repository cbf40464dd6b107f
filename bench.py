#!/usr/bin/env python3
"""Benchmark of the fused D3Q19 channel step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): the Re_tau ~ 180 smooth-wall channel, 628 x 202 x 314
(x streamwise x wall-normal incl. walls x spanwise; 39,438,400 fluid cells),
FP64, constant body force g = u_tau^2/h, from a seeded turbulent-like field.
A step is one fused launch (collide + stream + wall rules + periodic wrap +
the per-step encalc/wshearstr reductions) over the whole grid.  The state
(6.0 GB at FP64) is far larger than the 126 MB L2, so no flush is needed
between timed steps.

One JSON line (rank 0):
  value       MLUPS of the FP64 kernel, inputs resident in HBM, CUDA events
  roofline    dominant step kernel: algorithmic bytes (2 x 19 x 8 B per cell)
              / mean launch time, against the measured HBM copy bandwidth
  variants    the same workload with FP32 / FP16 deviation storage: MLUPS,
              roofline fraction and error against the FP64 run (which is
              bit-identical to the CPU oracle, see tests/test_gpu_parity.py)
  e2e         through the C ABI with host buffers: load the state from pinned
              host memory, K steps each reading its log record back, store the
              state back to pinned host memory; wall clock
  cpu_baseline the reference's own C step (oracle/_ref) on this host's cores
--gpus N > 1 runs N independent replicas (the step does not shard: one GPU
holds a whole channel); value sums them, time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics as stats_mod
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dns-solvers_b200"))
METRIC = "MLUPS & % HBM roofline: FP64 vs FP32/FP16-storage, at stated stats error"
FALLBACK_HBM_GBS = 6650.0
# steps each candidate launch shape is timed for: launch shapes within a
# percent of each other change places over 6 steps
TUNE_STEPS = 16


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="channel180")
    ap.add_argument("--precision", type=int, choices=[64, 32, 16], default=64,
                    help="storage precision of the headline run (profiling other kernels)")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the library's default launch shapes")
    ap.add_argument("--no-batched", action="store_true", help="skip the 24-channel batched FP32 measurement")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="target length of the CPU-baseline sample")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers
def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(kernel_key):
    """DRAM bytes per launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f).get(kernel_key)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi samples (200 ms) of SM clock and throttle reasons."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        time.sleep(0.3)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": stats_mod.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


class Dist:
    """Barrier and max-over-ranks for replicas launched by torchrun (gloo on
    CPU tensors: no collective touches the data path)."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.dist = dist

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, v):
        if self.world == 1:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_baseline(wl, seconds, steps=None, warmup=0):
    """The reference's own C step (oracle/_ref/dnsref) on this host, as
    independent single-rank processes on x-slabs of the workload; falls back
    to the C restatement (oracle/lbm_oracle.c) if the reference build is
    absent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    procs = max(1, min(os.cpu_count() or 1, 64))
    plane = wl.ny * wl.nz
    rate = 3.0e6  # cells/s per core for the full reference step, conservative
    if steps is None:
        slab = max(2, wl.nx // procs)
        steps = max(2, int(seconds * rate / (slab * plane)))
    else:
        slab = max(2, min(wl.nx // procs, int(seconds * rate / (steps * plane))))
    xonly = None
    if oracle.have_reference():
        mlups, secs, procs, slab = oracle.time_reference(wl.nx, wl.ny, wl.nz, steps, warmup=warmup, omega=wl.omega,
                                                         ubulk=wl.ubulk or 0.05, procs=procs, slab=slab)
        kind = "reference"
        try:  # xcomputations alone, a shorter sample of the same slabs
            xonly = round(oracle.time_reference(wl.nx, wl.ny, wl.nz, max(2, steps // 2), warmup=min(warmup, 1),
                                                omega=wl.omega, ubulk=wl.ubulk or 0.05, procs=procs, slab=slab,
                                                only_step=True)[0], 3)
        except Exception:  # reported as absent, never fatal
            xonly = None
    else:
        import numpy as np
        s = np.zeros((slab, wl.ny, wl.nz + 2, 19))
        s[:, :, 1:-1] = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
        fl = oracle.flags("smooth", slab, wl.ny, wl.nz)
        t0 = time.perf_counter()
        oracle.run(s, fl, wl.omega, gx=wl.gx, const_g=True, nsteps=steps)
        secs = time.perf_counter() - t0
        mlups = slab * plane * steps / secs / 1e6
        procs, kind = os.cpu_count() or 1, "port"
    return {"value": round(mlups, 3), "unit": "MLUPS", "cores": procs, "kind": kind,
            "xcomputations_only_mlups": xonly, "cpu_model": _cpu_model(),
            "sample": f"{procs} independent single-rank processes x {slab}x{wl.ny}x{wl.nz} x-slab of {wl.name}, "
                      f"{steps} timed full reference steps (encalc+wshearstr+xcomputations), rest start",
            "seconds": round(secs, 3)}


# ------------------------------------------------------------------ arms
def run_reference_arm(args):
    import inputs
    d = Dist()
    if d.rank != 0:
        d.close()
        return
    wl = inputs.workload(args.workload)
    cb = cpu_baseline(wl, seconds=45.0, steps=args.steps, warmup=min(args.warmup, 2))
    line = {"metric": METRIC, "value": cb["value"], "unit": "MLUPS", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wl.name, "grid": f"{wl.nx}x{wl.nz + 2}x{wl.ny}", "sample": cb["sample"]},
            "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    d.close()


def parity_fracs(bpc, cells, ms_even, ms_odd, n_even, n_odd, peak):
    """Roofline fraction of the even- and odd-parity step launches (mean
    launch time of each)."""
    def frac(ms, n):
        return round(bpc * cells / (ms / n / 1e3) / 1e9 / peak, 4) if n and ms > 0 else None
    return frac(ms_even, n_even), frac(ms_odd, n_odd)


def variant_summary(v):
    r, e = v["roofline"], v["error_vs_f64"]
    return {"value": v["value"], "unit": "MLUPS", "ms_per_step": v["ms_per_step"], "speedup_vs_f64": v["speedup_vs_f64"],
            "frac_even": r["frac_even"], "frac_odd": r["frac_odd"], "whole_step_frac": r["whole_step_frac"],
            "err_mean_u": float(f"{e['mean_u_profile_max_rel']:.3g}"),
            "err_u_rms": float(f"{e['u_rms_profile_max_rel']:.3g}"), "err_after_steps": e["after_steps"]}


def batched_summary(b):
    if "error" in b:
        return b
    return {"channels": b["channels"], "seed": b["seed"], "cells": b["cells"], "dtype": b["dtype"],
            "value": b["value"], "ms_per_step": b["ms_per_step"], "one_at_a_time": b["one_at_a_time"]["value"],
            "speedup_vs_one_at_a_time": b["speedup_vs_one_at_a_time"],
            "whole_step_frac": b["whole_step_frac_of_hbm"], "kernel": b["kernel_config"].split(":")[0],
            "one_launch_per_step": b["one_launch_per_step"]["value"]}


def batched_report(args, dev):
    """24 independent FP32 channels (half-heights 20/32/48/64, seeded walls
    and Re_tau in [120, 180]) advanced by one launch per step with the time
    loop replayed from a CUDA graph, against the same channels stepped one at
    a time, each alone on the GPU (both arms autotuned unless --no-autotune).
    Initial fields: one turbulent-like field per half-height, shared by the
    channels of that height, with solid cells set to rest."""
    import dnslbm
    import inputs
    chans = inputs.batch_channels(24, seed=0)
    fields = {}
    for w in chans:
        if w.nz not in fields:
            fields[w.nz] = inputs.turbulent_state(w.nx, w.ny, w.nz, w.ubulk, 0.1, w.nz)

    def mode(w):
        return dnslbm.BC_GENERAL if inputs.needs_general(w) else dnslbm.BC_REFERENCE

    flags = [inputs.make_flags(w) for w in chans]

    decks = [dnslbm.deck(w.nx, w.ny, w.nz, w.omega, ubulk=w.ubulk, gx=w.gx, precision=32, bc_mode=mode(w),
                         device=dev) for w in chans]
    cells = sum(w.cells for w in chans)
    warm = max(args.warmup, 3)

    def run_batch(launch_mode):
        old = os.environ.pop("DNSLBM_BATCH", None)
        if launch_mode:
            os.environ["DNSLBM_BATCH"] = "launch"
        try:
            with dnslbm.Batch(decks) as b:
                for c, fl in zip(b.channels, flags):
                    c.set_flags(fl)
                tune = None if args.no_autotune else b.autotune(8)
                for c, w, fl in zip(b.channels, chans, flags):
                    c.load_state(inputs.rest_solids(fields[w.nz], fl) if inputs.needs_general(w) else fields[w.nz])
                b.step_timed(warm)
                return b.step_timed(args.steps), b.kernel, b.channels[0].bytes_per_cell, tune
        finally:
            os.environ.pop("DNSLBM_BATCH", None)
            if old is not None:
                os.environ["DNSLBM_BATCH"] = old

    ms_b, kdesc, bpc, tune = run_batch(False)
    ms_l, kdesc_l, _, _ = run_batch(True)
    ms_alone = 0.0
    for w, fl in zip(chans, flags):
        with dnslbm.Channel(w.nx, w.ny, w.nz, w.omega, ubulk=w.ubulk, gx=w.gx, precision=32, bc_mode=mode(w),
                            device=dev) as c:
            c.set_flags(fl)
            if not args.no_autotune:
                c.autotune()
            c.load_state(inputs.rest_solids(fields[w.nz], fl) if inputs.needs_general(w) else fields[w.nz])
            c.step_timed(warm)
            ms_alone += c.step_timed(args.steps, per_launch=False)[0]
    peak, _ = hbm_peak()
    return {"workload": "24 channels, h in {20, 32, 48, 64}, (2 pi h) x (2h + 2) x (pi h), seeded walls "
                        "(smooth / longitudinal grooves / transverse grooves / triangular riblets), Re_tau in "
                        "[120, 180]",
            "channels": len(chans), "seed": 0, "cells": cells, "dtype": "f32", "steps": args.steps,
            "value": round(cells * args.steps / (ms_b / 1e3) / 1e6, 1), "unit": "MLUPS",
            "ms_per_step": round(ms_b / args.steps, 4),
            "one_at_a_time": {"value": round(cells * args.steps / (ms_alone / 1e3) / 1e6, 1), "unit": "MLUPS",
                              "ms_per_step": round(ms_alone / args.steps, 4)},
            "speedup_vs_one_at_a_time": round(ms_alone / ms_b, 3),
            "whole_step_frac_of_hbm": round(bpc * cells / (ms_b / args.steps / 1e3) / 1e9 / peak, 4),
            "kernel_config": kdesc, "autotune": tune,
            "one_launch_per_step": {"value": round(cells * args.steps / (ms_l / 1e3) / 1e6, 1), "unit": "MLUPS",
                                    "ms_per_step": round(ms_l / args.steps, 4), "kernel_config": kdesc_l}}


def run_ours(args):
    import numpy as np

    import dnslbm
    import inputs
    d = Dist()
    dev = d.local
    wl = inputs.workload(args.workload)
    cells = wl.cells
    flags = inputs.make_flags(wl)
    bc = dnslbm.BC_GENERAL if inputs.needs_general(wl) else dnslbm.BC_REFERENCE
    big = cells * 19 * 8 > 16e9  # FP64 host state above 16 GB: generated and loaded in x-slabs
    s0 = None
    if not big:
        s0 = inputs.make_state(wl, seed=0)
        if inputs.needs_general(wl):
            s0 = inputs.rest_solids(s0, flags)
    else:
        args.no_e2e = True  # the pinned host copies of a state this size are left out

    def load(c):
        if s0 is not None:
            c.load_state(s0)
        else:
            c.load_state_slabs(inputs.turbulent_slabs(wl.nx, wl.ny, wl.nz, wl.ubulk, 0.1, 0, slab=16,
                                                      flags=flags if inputs.needs_general(wl) else None))
    peak, peak_src = hbm_peak()

    ch = dnslbm.Channel(wl.nx, wl.ny, wl.nz, wl.omega, ubulk=wl.ubulk, gx=wl.gx, force_mode=dnslbm.CONST_G,
                        precision=args.precision, bc_mode=bc, device=dev)
    ch.set_flags(flags)
    tune = None if args.no_autotune else ch.autotune(TUNE_STEPS)
    load(ch)
    ch.step_timed(args.warmup)
    d.barrier()
    clk = ClockSampler(dev)
    clk.start()
    tot, _, _ = ch.step_timed(args.steps, per_launch=False)
    clk.stop()
    tmax = d.max(tot)
    # the device time of every launch comes from a second run of K steps with
    # an event pair around each launch; events between launches keep a launch
    # from overlapping the end of the one before, so that run is not `value`
    _, even, odd = ch.step_timed(args.steps)
    n_even = (args.steps + 1) // 2 if (args.warmup + args.steps) % 2 == 0 else args.steps // 2
    n_odd = args.steps - n_even
    value = d.world * cells * args.steps / (tmax / 1e3) / 1e6
    bpc = ch.bytes_per_cell
    # dominant kernel: the parity with the larger summed device time
    kdesc = ch.kernel
    kbase = kdesc.split(" ")[0]
    if odd >= even:
        kname, kms, kn = kbase + " (odd parity)", odd, n_odd
    else:
        kname, kms, kn = kbase + " (even parity)", even, n_even
    launch_s = kms / kn / 1e3
    achieved = bpc * cells / launch_s / 1e9
    traffic = ncu_traffic(f"{wl.name}:f{args.precision}")
    fe, fo = parity_fracs(bpc, cells, even, odd, n_even, n_odd, peak)
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": f"{peak_src} (MEASURED_PEAKS.json)",
            "kernel": kname, "kernel_config": kdesc, "autotune": tune, "launch_ms": round(launch_s * 1e3, 4),
            "launch_ms_from": "a second run of K steps with a CUDA event pair around every launch",
            "frac_even": fe, "frac_odd": fo,
            "whole_step_frac": round(bpc * cells / (tmax / args.steps / 1e3) / 1e9 / peak, 4),
            "algorithmic_bytes_per_launch": bpc * cells, "bytes_per_cell": bpc}

    variants = {}
    if not args.no_variants and args.precision == 64:
        ref_stats = ch.statistics()
        ref_vel, _ = ch.moments()
        done = ch.steps_done
        for prec in (32, 16):
            c2 = dnslbm.Channel(wl.nx, wl.ny, wl.nz, wl.omega, ubulk=wl.ubulk, gx=wl.gx,
                                force_mode=dnslbm.CONST_G, precision=prec, bc_mode=bc, device=dev)
            c2.set_flags(flags)
            tune2 = None if args.no_autotune else c2.autotune(TUNE_STEPS)
            load(c2)
            c2.step_timed(args.warmup)
            t2 = c2.step_timed(args.steps, per_launch=False)[0]
            _, e2, o2 = c2.step_timed(args.steps)
            assert c2.steps_done == done
            st = c2.statistics()
            vel, _ = c2.moments()
            b2 = c2.bytes_per_cell
            k2 = max(e2, o2) / (n_odd if o2 >= e2 else n_even) / 1e3
            ach2 = b2 * cells / k2 / 1e9
            fe2, fo2 = parity_fracs(b2, cells, e2, o2, n_even, n_odd, peak)
            um_ref, um = ref_stats[0, 1:-1], st[0, 1:-1]
            urms_ref, urms = ref_stats[3, 1:-1], st[3, 1:-1]
            variants[f"f{prec}"] = {
                "value": round(cells * args.steps / (t2 / 1e3) / 1e6, 1), "unit": "MLUPS",
                "ms_per_step": round(t2 / args.steps, 4), "speedup_vs_f64": round(tot / t2, 3),
                "roofline": {"bound": "hbm", "achieved": round(ach2, 1), "peak": peak, "unit": "GB/s",
                             "frac": round(ach2 / peak, 4), "frac_even": fe2, "frac_odd": fo2, "bytes_per_cell": b2,
                             "whole_step_frac": round(b2 * cells / (t2 / args.steps / 1e3) / 1e9 / peak, 4),
                             "traffic": ncu_traffic(f"{wl.name}:f{prec}"), "kernel_config": c2.kernel,
                             "autotune": tune2},
                "error_vs_f64": {
                    "after_steps": done,
                    "mean_u_profile_max_rel": float(np.max(np.abs(um - um_ref)) / np.max(np.abs(um_ref))),
                    "u_rms_profile_max_rel": float(np.max(np.abs(urms - urms_ref)) / np.max(np.abs(urms_ref))),
                    "cell_velocity_max_abs": float(np.max(np.abs(vel - ref_vel))),
                    "cell_velocity_max_abs_over_ubulk": float(np.max(np.abs(vel - ref_vel)) / wl.ubulk),
                },
            }
            c2.close()
        del ref_vel

    batched = None
    if not args.no_batched:
        try:
            batched = batched_report(args, dev)
        except Exception as e:  # reported, never fatal
            batched = {"error": str(e)[:300]}

    e2e = None
    if not args.no_e2e:
        state_bytes = s0.nbytes
        pin_in = dnslbm.PinnedArray(s0.shape)
        pin_in.array[...] = s0
        pin_out = dnslbm.PinnedArray(s0.shape)
        ch.sync()
        d.barrier()
        t0 = time.perf_counter()
        ch.load_state(pin_in.array)
        for s in range(args.steps):
            ch.step(1)
            ch.logs(s, 1)
        ch.store_state(pin_out.array)
        t1 = time.perf_counter()
        e2e_s = d.max(t1 - t0)
        e2e = {"value": round(d.world * cells * args.steps / e2e_s / 1e6, 1), "unit": "MLUPS",
               "h2d_bytes_per_step": int(state_bytes / args.steps),
               "d2h_bytes_per_step": int((state_bytes + 72 * args.steps) / args.steps),
               "seconds": round(e2e_s, 4),
               "what": "dnslbm_load_state from pinned host (lbf layout, FP64) + K x (dnslbm_step(1) + "
                       "dnslbm_logs of that step) + dnslbm_store_state to pinned host; wall clock"}
        pin_in.free()
        pin_out.free()

    cb = None
    if d.rank == 0 and not args.no_cpu:
        try:
            cb = cpu_baseline(wl, args.cpu_seconds)
        except Exception as e:  # reported, never fatal
            cb = {"value": None, "error": str(e)[:200]}

    if d.rank == 0:
        line = {"metric": METRIC, "value": round(value, 1), "unit": "MLUPS", "n_gpus": d.world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(tmax / args.steps, 4),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": f"f{args.precision}",
                "data": "synthetic (seeded turbulent-like field: laminar profile + divergence-free perturbation "
                        "of 10% of U_b)",
                "config": {"workload": wl.name, "grid": f"{wl.nx}x{wl.nz + 2}x{wl.ny}", "cells": cells,
                           "walls": wl.texture, "force": f"constant g={wl.gx:.3e}", "omega": wl.omega,
                           "parallelism": f"replicas x{d.world}" if d.world > 1 else "single GPU",
                           "l2": f"state {cells * 19 * args.precision / 8 / 1e9:.2f} GB vs 126 MB L2, no flush"},
                "variants": variants, "roofline": roof, "e2e": e2e, "cpu_baseline": cb,
                "gpu_launches": args.steps * (2 if "links_pass_kernel" in kdesc else 1), "clocks": clk.summary()}
        # short summaries last, so that a reader of the line's tail sees them
        if batched is not None:
            line["batched"] = batched_summary(batched)
        for k, v in variants.items():
            line[f"{k}_storage"] = variant_summary(v)
        print(json.dumps(line), flush=True)
    ch.close()
    d.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
