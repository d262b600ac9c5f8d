#!/usr/bin/env python
"""Benchmark of the Strang split-operator step on B200 (one JSON line on stdout).

Headline workload (--config c4, the default): a batched tunnelling sweep of 256
independent 3D instances, grid sizes drawn from {32,48,64,96,128,160}^3
(radix 2/3/5; 369 M grid points in all), box side 20 n/32, barrier of height
U[0.5,4] and thickness 2 at x = 0, Gaussian packet (sigma U[1,2.5], k0
U[1,4]) at x = -L/4, cos^(1/8) absorber on the outer 8%, dt = 0.005,
propagated as complex64 with FP64-built tables through the batched path (one
launch per axis pass and grid-size class, CUDA graphs, autotuned tiles).
Inputs are synthetic and seeded (no dataset exists for this path); the fields
(2.9 GB) are far larger than the 126 MB L2, so no flush is needed between steps.

A "step" is one Strang step of every instance (potential kick, 3D FFT, kinetic
phase, inverse 3D FFT, kick, absorber).  value = grid points x steps per
second for the whole job.  Beside it: the plain FP64 path (complex128, each
instance stepped alone) on the same mix, the complex64-vs-complex128 error
after the config's 1000 steps, the serving loop (Poisson arrivals of mixed
1D/2D/3D requests, p50/p99 latency) with the plain FP64 path on the same
request mix, the single-instance C1/C2/C3 numbers and, on the host cores, the
reference's FP64 CPU core -- whose runs are also the checker of the device
results on the named configurations ("parity").  Multi-GPU runs split one
workload of 256 x N instances over the N ranks (balanced by grid points, no
collective on the data path): weak scaling.

--impl reference times the reference's own FP64 CPU core (compiled from its
sources into oracle/_ref) on a bounded sample of the same workload with all
host threads; it maps none of this repository's device code.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from collections import Counter
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "grid-pt*steps/s (FP32-batched; plain FP64 beside it; serve p50/p99)"
UNIT = "grid-pt*steps/s"
# algorithmic bytes per grid point per Strang step: 2*d*2*E + E_tab
MODEL_BYTES = {("c128", 3): 208, ("c64", 3): 104, ("c128", 2): 144, ("c64", 2): 72, ("c128", 1): 80,
               ("c64", 1): 40}
# bytes a step of this implementation moves per grid point: four sweeps of psi + the
# table; the two-sweep step (x-y plane pass + z pass, planes up to 128^2) two sweeps + the table
ACTUAL_BYTES = {"c128": 144, "c64": 72}
TWO_SWEEP_BYTES = {"c128": 80, "c64": 40}


def two_sweep(plan: str) -> bool:
    return "two sweeps" in plan
ESIZE = {"c128": 16, "c64": 8}
L2_BYTES = 126 * 2 ** 20  # B200
STAND_IN = ("the reference core transforms powers of two only (core/src/fft.ixx:42-44): its arm times "
            "48/96/160 at the per-point rate it reaches on 64/128/256")


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=["c4", "c2", "c3", "c1"], default="c4")
    ap.add_argument("--instances", type=int, default=256, help="batched sweep size per GPU (c4)")
    ap.add_argument("--sizes", default="", help="c4: keep only these grid sizes (comma list), for profiling")
    ap.add_argument("--n", type=int, default=0, help="grid size override for c1/c2/c3")
    ap.add_argument("--precision", choices=["c64", "c128"], default=None,
                    help="c1/c2/c3 line precision (default: c128 for c1, the plain FP64 config; else c64)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg and its parity checks")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle parity checks of the CPU leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving run")
    ap.add_argument("--no-single", action="store_true", help="skip the single-instance C1/C2/C3 lines")
    ap.add_argument("--serve-requests", type=int, default=48)
    ap.add_argument("--accuracy-steps", type=int, default=-1,
                    help="steps of the c64-vs-c128 accuracy check (-1: the config's step count)")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--quick", action="store_true",
                    help="timed region and per-pass profile only (for profiler launch lists)")
    return ap.parse_args(argv)


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples (every `ms` milliseconds) during a timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int, ms: int = 50):
        self.gpu = gpu_index
        self.ms = ms
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", str(self.ms)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            time.sleep(0.15)  # the first sample lands before the timed work starts
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": mx or None, "reasons": sorted(reasons), "samples": len(sm)}


def rel_l2(a, b):
    import numpy as np
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


# ---------------------------------------------------------------------------
# C4: the batched sweep
# ---------------------------------------------------------------------------
def c4_all_specs(args, world: int):
    """The whole job's instances: 256 per GPU (seeded, one list for all ranks)."""
    from shoeridingerequationsolver_b200 import scenes
    if not args.sizes:
        return scenes.config_c4_specs(args.instances * world)
    keep = {int(x) for x in args.sizes.split(",")}
    return [s for s in scenes.config_c4_specs(256 * world) if s["n"] in keep][:args.instances * world]


def c4_config(specs, world: int, args) -> dict:
    """The workload description, printed identically by both arms."""
    from shoeridingerequationsolver_b200 import scenes
    return {"workload": f"c4_batched_tunnel_{len(specs)}" + (f"_sizes_{args.sizes}" if args.sizes else ""),
            "instances": len(specs), "sizes": {str(k): v for k, v in sorted(Counter(sp["n"] for sp in specs).items())},
            "grid_points": sum(sp["n"] ** 3 for sp in specs), "dt": 0.005,
            "absorber": "cos^(1/8) on the outer 8%, after every step",
            "l2": "inputs (2.9 GB per GPU) larger than L2, no flush",
            "parallelism": f"replicas x{world} (instances split by grid points)",
            "seed": scenes.SEED_BASE + 3, "reference_stand_in": STAND_IN}


def build_c4(ses, specs, prec="c64"):
    from shoeridingerequationsolver_b200 import scenes
    ops = []
    for sp in specs:
        w = scenes.build_c4_instance(sp)
        op = ses.SplitOperator3D(w.grid, w.V, w.dt, w.mass, precision=prec, psi0=w.psi0)
        op.set_absorber_separable(*w.mask)
        ops.append(op)
    return ops


def class_order(specs):
    seen = []
    for sp in specs:
        if sp["n"] not in seen:
            seen.append(sp["n"])
    return seen


def batch_roofline(prof, specs, peak, peak_kind, traffic_table):
    """Dominant launch of the batched step (class x pass) and its algorithmic bandwidth.

    Per-launch algorithmic bytes split the 2*d*2*E + E_tab model per pass and
    multiply by the class's grid points: x between steps 4E + E_tab, y forward
    2E, z fused (fwd, K/N, inv) 4E, y inverse 2E (E = 8, complex64).  The bytes
    the launch actually moves are 2E + E_tab (x) and 2E (the others)."""
    E = ESIZE["c64"]
    per_pt = [4 * E + E, 2 * E, 4 * E, 2 * E]
    moved = [2 * E + E, 2 * E, 2 * E, 2 * E]
    names = ["x_mid", "y_fwd", "z_fused", "y_inv"]
    counts = Counter(sp["n"] for sp in specs)
    best = None
    for n, p in zip(class_order(specs), prof):
        times = [p["x_mid"]] + p["mid"]
        for k in range(4):
            if times[k] > 0 and (best is None or times[k] > best[0]):
                best = (times[k], n, k)
    ms, n, k = best
    pts = counts[n] * n ** 3
    alg = per_pt[k] * pts
    achieved = alg / (ms * 1e-3) / 1e9
    act = moved[k] * pts / (ms * 1e-3) / 1e9
    key = f"c4:{n}:{names[k]}"
    return {"kernel": f"{names[k]} pass of the {n}^3 class ({counts[n]} instances, one launch)",
            "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "peak_kind": peak_kind,
            "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic_table.get(key),
            "algorithmic_bytes_per_launch": alg, "launch_ms": round(ms, 5),
            "moved_bytes_per_launch": moved[k] * pts, "moved_gbs": round(act, 1),
            "moved_frac": round(act / peak, 4)}


def time_handle(op, stream, K, absorb):
    e0, e1 = events()
    e0.record(stream)
    op.advance(K, absorb=absorb)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def fp64_plain(ses, shapes, stream, warm=3, min_ms=300.0):
    """The plain FP64 path: complex128, one handle per shape stepped alone (its own
    launches), time per step measured over >= min_ms of steps.  shapes: list of
    (key, Workload)."""
    per = {}
    for key, w in shapes:
        op = ses.SplitOperator3D(w.grid, w.V, w.dt, w.mass, precision="c128", psi0=w.psi0)
        absorb = w.mask is not None
        if absorb:
            op.set_absorber_separable(*w.mask)
        op.set_stream(stream.cuda_stream)
        if not NO_AUTOTUNE:
            op.autotune(save=False)
        op.prepare(absorb)
        op.advance(warm, absorb=absorb)
        op.sync(60000)
        K = 16
        ms = time_handle(op, stream, K, absorb)
        K = max(K, int(min_ms / max(ms / K, 1e-4)))
        ms = time_handle(op, stream, K, absorb)
        plan = op.plan_info()
        op.close()
        per[key] = {"ms_per_step": round(ms / K, 5), "steps_timed": K,
                    "step_form": "two sweeps" if two_sweep(plan) else "four axis passes"}
    return per


def fp64_plain_mix(ses, specs, stream):
    """The plain FP64 path on the batched sweep's mix: per-size time per step x instance count."""
    from shoeridingerequationsolver_b200 import scenes
    counts = Counter(sp["n"] for sp in specs)
    shapes = [(n, scenes.build_c4_instance(next(s for s in specs if s["n"] == n))) for n in sorted(counts)]
    per = fp64_plain(ses, shapes, stream)
    total_ms = sum(per[n]["ms_per_step"] * counts[n] for n in counts)
    npts = sum(sp["n"] ** 3 for sp in specs)
    return {"value": npts / (total_ms * 1e-3), "ms_per_step": total_ms, "dtype": "c128",
            "ms_per_step_by_size": {str(n): per[n]["ms_per_step"] for n in sorted(per)},
            "step_form_by_size": {str(n): per[n]["step_form"] for n in sorted(per)},
            "how": "each size alone (>= 0.3 s of timed steps after 3), times the instance count"}


def c4_accuracy(ses, specs, steps):
    """complex64 batched vs the plain complex128 path after `steps` steps, one instance per size."""
    from shoeridingerequationsolver_b200 import scenes
    sample = [next(s for s in specs if s["n"] == n) for n in sorted({s["n"] for s in specs})]
    ops64 = build_c4(ses, sample, "c64")
    with ses.Batch(ops64) as b:
        b.step(steps, absorb=True)
        obs64 = b.observe(1.0, math.inf)
        psi64 = [op.readback() for op in ops64]
    out = []
    for sp, op, p64, o64 in zip(sample, ops64, psi64, obs64):
        w = scenes.build_c4_instance(sp)
        ref = ses.SplitOperator3D(w.grid, w.V, w.dt, w.mass, precision="c128", psi0=w.psi0)
        ref.set_absorber_separable(*w.mask)
        o0 = ref.observe(1.0, math.inf)
        ref.advance(steps, absorb=True)
        o128 = ref.observe(1.0, math.inf)
        out.append({"n": sp["n"], "rel_l2": rel_l2(p64, ref.readback()),
                    "norm_diff": o64["norm"] - o128["norm"], "energy_diff": o64["energy"] - o128["energy"],
                    "energy_drift_c128": o128["energy"] - o0["energy"], "transmitted": o128["p_range"]})
        ref.close()
        op.close()
    return {"steps": steps, "max_rel_l2": max(r["rel_l2"] for r in out),
            "max_abs_norm_diff": max(abs(r["norm_diff"]) for r in out),
            "max_abs_energy_diff": max(abs(r["energy_diff"]) for r in out), "per_size": out,
            "reference": "plain complex128 GPU path; against the FP64 oracle itself see parity.c4"}


def c4_e2e(ses, b, ops, specs, segment=100):
    """One request through the public batch API with host buffers (ses_batch_run):
    upload every field (pinned complex128), `segment` steps, observables, read every
    field back -- queued per class stream, so transfers overlap other classes' steps."""
    import numpy as np
    import torch
    from shoeridingerequationsolver_b200 import scenes
    bufs = {}
    for sp in specs:  # one pinned input/output pair per size, reused by its members
        if sp["n"] not in bufs:
            w = scenes.build_c4_instance(sp)
            hin = torch.empty(2 * w.grid.size(), dtype=torch.float64, pin_memory=True)
            hin.numpy()[:] = w.psi0.view(np.float64)
            bufs[sp["n"]] = (hin, torch.empty_like(hin, pin_memory=True))
    npts = sum(sp["n"] ** 3 for sp in specs)
    pin = [bufs[sp["n"]][0].data_ptr() for sp in specs]
    pout = [bufs[sp["n"]][1].data_ptr() for sp in specs]
    t0 = time.perf_counter()
    b.run(segment, psi_in=pin, psi_out=pout, absorb=True, xlo=1.0, xhi=math.inf)
    dt = time.perf_counter() - t0
    return {"value": npts * segment / dt, "unit": UNIT,
            "h2d_bytes_per_step": 16 * npts / segment, "d2h_bytes_per_step": (16 * npts + 14 * 8 * len(ops)) / segment,
            "step": f"one request: upload all {len(ops)} fields (complex128, pinned), {segment} batched steps, "
                    f"observables of every field, read every field back", "wall_s": round(dt, 3)}


def reference_c4_rates(specs, warmup: int, steps: int, budget_s: float):
    """The reference core (oracle/_ref) on the host cores: SplitOperator3D::step (+ mask)
    threaded by ses.parallel, one instance per power-of-two stand-in size.  A sample
    step = one step of each sampled size; `warmup` untimed sample steps, then up to
    `steps` timed ones (fewer if the budget runs out).  Returns the per-size rates and
    the sample's own timing."""
    from oracle.oracle import Reference
    from oracle.parity import full_mask
    from shoeridingerequationsolver_b200 import scenes
    counts = Counter(sp["n"] for sp in specs)
    pow2 = lambda n: n & (n - 1) == 0
    stand_in = {n: (n if pow2(n) else 1 << n.bit_length()) for n in counts}
    ref = Reference(workers=os.cpu_count())
    sims = {}
    for m in sorted(set(stand_in.values())):
        sp = next((s for s in specs if s["n"] == m), None)
        sp = dict(sp) if sp else dict(next(iter(specs)), n=m, side=20.0 * m / 32.0)
        w = scenes.build_c4_instance(sp)
        s = ref.split3d(w.grid.box, w.grid.dims, w.V, w.dt, w.mass)
        s.set_psi(w.psi0)
        sims[m] = (s, full_mask(w.mask))
    for _ in range(max(0, warmup)):
        for s, msk in sims.values():
            s.step(1, msk)
    spent = {m: 0.0 for m in sims}
    done = 0
    t_all = time.perf_counter()
    while done < max(1, steps):
        for m, (s, msk) in sims.items():
            t0 = time.perf_counter()
            s.step(1, msk)
            spent[m] += time.perf_counter() - t0
        done += 1
        if time.perf_counter() - t_all > budget_s:
            break
    wall = time.perf_counter() - t_all
    for s, _ in sims.values():
        s.close()
    rate = {m: m ** 3 * done / spent[m] for m in sims}
    npts = sum(sp["n"] ** 3 for sp in specs)
    total_s = sum(counts[n] * n ** 3 / rate[stand_in[n]] for n in counts)
    return {"value": npts / total_s, "cores": ref.workers(), "steps_timed": done,
            "sample_ms_per_step": 1e3 * wall / done, "sample_points": sum(m ** 3 for m in sims),
            "per_size": {str(m): {"ms_per_step": round(1e3 * spent[m] / done, 3)} for m in sims},
            "stand_in": {str(n): stand_in[n] for n in sorted(stand_in)}}


def cpu_baseline_c4(specs, budget_s=20.0):
    """The reference core (oracle/_ref, all host threads) on a bounded sample of the
    sweep (one instance per power-of-two stand-in size, about budget_s seconds);
    the C restatement on one thread when the reference was not built."""
    from oracle.oracle import Oracle, Reference
    from oracle.parity import full_mask
    from shoeridingerequationsolver_b200 import scenes
    if Reference.available():
        r = reference_c4_rates(specs, 1, 20, budget_s)
        return {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": "reference",
                "sample": f"reference SplitOperator3D::step (+ mask) via ses.parallel, {r['steps_timed']} steps of "
                          f"one instance per size {sorted(int(k) for k in r['per_size'])} after 1 untimed; "
                          f"48/96/160 (which the reference rejects) charged at the per-point rate of 64/128/256; "
                          f"mix time = sum over sizes", "per_size": r["per_size"]}
    counts = Counter(sp["n"] for sp in specs)
    npts = sum(sp["n"] ** 3 for sp in specs)
    o = Oracle()
    total_s, per = 0.0, {}
    for n in sorted(counts):
        w = scenes.build_c4_instance(next(s for s in specs if s["n"] == n))
        t0 = time.perf_counter()
        o.step3d(w.grid.box, w.grid.dims, w.V, w.dt, w.psi0, 1, w.mass, full_mask(w.mask))
        dt = time.perf_counter() - t0
        per[str(n)] = {"ms_per_step": round(dt * 1e3, 3), "steps": 1}
        total_s += dt * counts[n]
    return {"value": npts / total_s, "unit": UNIT, "cores": int(os.environ.get("SESO_THREADS", os.cpu_count())),
            "kind": "port", "sample": "one Strang step per grid size, C restatement", "per_size": per}


# ---------------------------------------------------------------------------
# parity of the device path on the named configurations (the CPU leg's runs as checker)
# ---------------------------------------------------------------------------
def _summary(r):
    keep = ("precision", "steps", "checker", "checker_cpu_s", "rel_l2", "max_rel_l2", "norm_diff",
            "max_abs_norm_diff", "energy_diff", "max_abs_energy_diff", "norm_drift", "norm_drift_oracle",
            "energy_drift", "energy_drift_oracle")
    return {k: r[k] for k in keep}


def parity_runs(ses):
    """The device path against the FP64 oracle on every named configuration, sized
    so the CPU side stays near a minute: C1 full (2000 steps, observables every
    100); C2 at 256^3 for 20 steps (both precisions) and its 1000-step complex64
    run on 128^3 (same box); C3 at 512^3 for 5 steps and its 500-step run on
    512 x 64 x 64 (same spacing, packet at x = -5 so that part of it crosses) with
    the transmitted probability every 50 steps; the batched sweep's 32/48/64/128
    instances after the config's 1000 steps (complex64, batched)."""
    from oracle.oracle import Oracle, Reference
    from oracle.parity import Checker, full_mask, run_segments
    from shoeridingerequationsolver_b200 import scenes
    o = Oracle()
    out = {}
    w = scenes.config_c1()
    r = run_segments(ses, o, Reference, w, "c128", w.steps, w.observe_every)
    out["c1_harmonic_64"] = dict(_summary(r), observed_every=w.observe_every,
                                 energy_series=[(row["step"], row["energy"], row["energy_oracle"]) for row in r["series"]],
                                 norm_series=[(row["step"], row["norm"], row["norm_oracle"]) for row in r["series"]])
    w = scenes.config_c2(256)
    out["c2_coulomb_stark_256"] = {prec: _summary(run_segments(ses, o, Reference, w, prec, 20, 20))
                                   for prec in ("c64", "c128")}
    w = scenes.config_c2(128)
    out["c2_coulomb_stark_128"] = {"c64": _summary(run_segments(ses, o, Reference, w, "c64", 1000, 1000))}
    w = scenes.config_c3(512)
    out["c3_tunnel_512"] = {"c64": _summary(run_segments(ses, o, Reference, w, "c64", 5, 5, (1.0, math.inf)))}
    for x0 in (-5.0,):
        w = scenes.config_c3_strip(x0)
        r = run_segments(ses, o, Reference, w, "c64", w.steps, w.observe_every, (1.0, math.inf))
        out[w.name] = dict(_summary(r), transmitted_every_50=[(row["step"], row["p_range"], row["p_range_oracle"])
                                                              for row in r["series"]])
    # the batched sweep: one instance per size, complex64 batched, 1000 steps
    specs = scenes.config_c4_specs(256)
    rows = []
    for n in (32, 48, 64, 128):
        sp = next(s for s in specs if s["n"] == n)
        w = scenes.build_c4_instance(sp)
        op = ses.SplitOperator3D(w.grid, w.V, w.dt, w.mass, precision="c64", psi0=w.psi0)
        op.set_absorber_separable(*w.mask)
        with ses.Batch([op]) as b:
            b.step(w.steps, absorb=True)
            obs = b.observe(1.0, math.inf)[0]
        got = op.readback()
        op.close()
        chk = Checker(o, Reference, w)
        want = chk.step(w.steps)
        rows.append({"n": n, "steps": w.steps, "rel_l2": rel_l2(got, want), "norm_diff": obs["norm"] - chk.norm(),
                     "energy_diff": obs["energy"] - chk.energy(), "checker": chk.kind,
                     "checker_cpu_s": round(chk.cpu_s, 2)})
        chk.close()
    out["c4_batched_c64_vs_oracle"] = {"per_size": rows, "max_rel_l2": max(r["rel_l2"] for r in rows),
                                       "note": "96^3 and 160^3 (slow in the mixed-radix restatement) are "
                                               "checked against the complex128 GPU path in `accuracy`; 48^3, 96 x 96 "
                                               "and 64^3 against the oracle in tests/test_gpu_configs.py"}
    return out


# ---------------------------------------------------------------------------
# C5: serving
# ---------------------------------------------------------------------------
def serve_autotune(ses, specs):
    """The deployment's autotune cache for the request shapes of the mix: one
    complex64 batch per distinct shape, tuned and saved (SES_TUNE_CACHE), which the
    server's batch classes then read."""
    from shoeridingerequationsolver_b200 import scenes
    seen = {}
    for s in specs:
        key = (s["kind"], tuple(s["dims"]))
        if key not in seen:
            seen[key] = s
    tuned = []
    for key, s in seen.items():
        req = scenes.build_c5_request(s)
        op = ses.SplitOperator3D(req["grid"], req["V"], req["dt"], precision="c64", psi0=req["psi0"])
        op.set_absorber_separable(*req["mask"])
        with ses.Batch([op]) as b:
            tuned.append(f"{key[0]} {'x'.join(map(str, key[1]))}: {b.autotune(save=True)}")
        op.close()
    return tuned


def serve_closed_loop(ses, specs):
    """The closed-loop batch rate of the server on the mix: every request submitted
    at once; grid-pt*steps of all rounds / wall time (and the device-busy share)."""
    from shoeridingerequationsolver_b200 import scenes
    built = [scenes.build_c5_request(s) for s in specs]
    with ses.Server(budget_bytes=150 * 10**9, max_round_steps=100) as srv:
        t0 = time.perf_counter()
        for req in built:
            srv.submit(**req)
        srv.wait_idle(900000)
        wall = time.perf_counter() - t0
        st = srv.stats()
    return {"value": st["gridpt_steps"] / wall, "wall_s": round(wall, 3), "rounds": st["rounds"],
            "device_busy_frac": round(st["busy_ms"] / 1e3 / wall, 3)}


def serve_run(ses, nreq, seed=None):
    """Poisson arrivals of mixed 1D/2D/3D requests into the request server; lambda
    set so the offered load is ~0.9 of the server's closed-loop batch rate on the
    same mix (measured first, every request submitted at once)."""
    import numpy as np
    from shoeridingerequationsolver_b200 import scenes
    specs = scenes.config_c5_specs(nreq) if seed is None else scenes.config_c5_specs(nreq, seed=seed)
    mean_work = sum(s["points"] * s["steps"] for s in specs) / len(specs)
    tuned = serve_autotune(ses, specs)
    closed = serve_closed_loop(ses, specs)
    capacity_ptsteps = closed["value"]
    lam = 0.9 * capacity_ptsteps / mean_work
    rng = np.random.default_rng(scenes.SEED_BASE + 50)
    gaps = rng.exponential(1.0 / lam, len(specs))
    built = [scenes.build_c5_request(s) for s in specs]   # host arrays before the clock starts
    ids = []
    with ses.Server(budget_bytes=150 * 10**9, max_round_steps=100) as srv:
        t0 = time.perf_counter()
        t_next = t0
        for req, gap in zip(built, gaps):
            t_next += gap
            delay = t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            ids.append(srv.submit(**req))
        srv.wait_idle(900000)
        wall = time.perf_counter() - t0
        st = srv.stats()
        lats, fails, nrec = [], 0, 0
        for rid in ids:
            state, recs = srv.poll(rid)
            nrec += len(recs)
            if state == "done":
                lats.append(srv.result(rid, want_psi=False)[1])
            else:
                fails += 1
    lats.sort()
    kinds = Counter(s["kind"] for s in specs)
    return {"requests": len(specs), "mix": dict(kinds), "failed": fails, "lambda_per_s": round(lam, 3),
            "latency_p50_ms": round(float(np.percentile(lats, 50)), 2) if lats else None,
            "latency_p99_ms": round(float(np.percentile(lats, 99)), 2) if lats else None,
            "throughput": st["gridpt_steps"] / wall, "unit": UNIT, "wall_s": round(wall, 2),
            "rounds": st["rounds"], "records": nrec, "budget_bytes": 150 * 10**9,
            "device_busy_frac": round(st["busy_ms"] / 1e3 / wall, 3),
            "closed_loop": closed, "serve_over_closed_loop": round(st["gridpt_steps"] / wall / capacity_ptsteps, 3),
            "autotuned": tuned,
            "offered_load": "0.9 x the server's closed-loop batch rate on the same mix"}


def fp64_plain_c5(ses, nreq, stream):
    """The plain FP64 path on the serving stream's request mix: each distinct request
    shape alone as complex128 (its potential, absorber, dt), time per step x the
    steps of every request of that shape; grid-pt*steps of the mix / that time."""
    from shoeridingerequationsolver_b200 import scenes
    specs = scenes.config_c5_specs(nreq)
    shapes, work = [], Counter()
    for s in specs:
        key = f"{s['kind']}:{'x'.join(map(str, s['dims']))}"
        work[key] += s["steps"]
        if key not in [k for k, _ in shapes]:
            req = scenes.build_c5_request(s)
            shapes.append((key, scenes.Workload(key, req["grid"], req["V"], req["psi0"], req["dt"], req["nsteps"],
                                                mask=req["mask"])))
    per = fp64_plain(ses, shapes, stream)
    total_s = sum(per[k]["ms_per_step"] * 1e-3 * work[k] for k in work)
    ptsteps = sum(s["points"] * s["steps"] for s in specs)
    return {"value": ptsteps / total_s, "unit": UNIT, "dtype": "c128", "grid_pt_steps": ptsteps,
            "ms_per_step_by_shape": {k: per[k]["ms_per_step"] for k in sorted(per)},
            "step_form_by_shape": {k: per[k]["step_form"] for k in sorted(per)},
            "how": "each distinct request shape alone (>= 0.3 s of timed steps, the first request's potential "
                   "and dt), times its requests' step counts"}


# ---------------------------------------------------------------------------
# single instance (C1/C2/C3)
# ---------------------------------------------------------------------------
def single_workload(args):
    from shoeridingerequationsolver_b200 import scenes
    if args.config == "c1":
        return scenes.config_c1()
    if args.config == "c3":
        return scenes.config_c3(args.n or 512)
    return scenes.config_c2(args.n or 256)


def single_roofline(prof, npts, prec, peak, peak_kind, traffic_table, wname, plan=""):
    """Dominant pass of a 3D step: per-launch algorithmic bytes x -> 4E + E_tab,
    y forward 2E, last-axis fused 4E, y inverse 2E; moved bytes 2E (+ E_tab on x).
    Two-sweep step: the plane pass (profiled as the x pass) carries both y
    transforms, 8E + E_tab of model bytes, and moves 2E + E_tab."""
    E = ESIZE[prec]
    per_pt = {"x_mid": 4 * E + E, "y_fwd": 2 * E, "fused": 4 * E, "y_inv": 2 * E}
    moved = {"x_mid": 3 * E, "y_fwd": 2 * E, "fused": 2 * E, "y_inv": 2 * E}
    if two_sweep(plan):
        per_pt["x_mid"] = 8 * E + E
    kinds = {k: prof[k] for k in per_pt if prof.get(k, 0) > 0}
    dom = max(kinds, key=kinds.get)
    alg = per_pt[dom] * npts
    achieved = alg / (kinds[dom] * 1e-3) / 1e9
    act = moved[dom] * npts / (kinds[dom] * 1e-3) / 1e9
    return {"kernel": dom, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "traffic": traffic_table.get(f"{wname}:{prec}:{dom}"), "algorithmic_bytes_per_launch": alg,
            "launch_ms": round(kinds[dom], 5), "moved_gbs": round(act, 1), "moved_frac": round(act / peak, 4),
            "pass_ms": {k: round(v, 5) for k, v in kinds.items()},
            "step_form": "two sweeps" if two_sweep(plan) else "four axis passes"}


def single_precision(ses, w, prec, W, stream, clocks_gpu, min_ms=600.0, K=None):
    """One handle of workload w: W warm-up steps, then K steps timed with CUDA events
    (K None: chosen so the timed region lasts >= min_ms, for a clock record of its own)."""
    op = ses.SplitOperator3D(w.grid, w.V, w.dt, w.mass, precision=prec)
    absorb = w.mask is not None
    if absorb:
        op.set_absorber_separable(*w.mask)
    op.set_stream(stream.cuda_stream)
    plan = op.plan_info() if NO_AUTOTUNE else op.autotune(save=False)
    op.upload_state(w.psi0)
    op.prepare(absorb)
    op.advance(W, absorb=absorb)
    op.sync(60000)
    if K is None:
        est = time_handle(op, stream, 16, absorb) / 16
        K = max(16, int(min_ms / max(est, 1e-4)))
    with ClockSampler(clocks_gpu) as clk:
        ms = time_handle(op, stream, K, absorb)
    prof = op.profile_step(8, absorb=absorb)
    op.close()
    return {"ms": ms, "K": K, "profile": prof, "clocks": clk.summary(), "plan": plan}


def single_entry(w, prec, r, peak, peak_kind, traffic_table):
    npts = w.grid.size()
    v = npts * r["K"] / (r["ms"] * 1e-3)
    mb = MODEL_BYTES[(prec, 3)]
    moved = TWO_SWEEP_BYTES[prec] if two_sweep(r["plan"]) else ACTUAL_BYTES[prec]
    return {"precision": prec, "value": v, "ms_per_step": r["ms"] / r["K"], "steps_timed": r["K"],
            "step_model_gbs": round(mb * v / 1e9, 1), "step_frac": round(mb * v / 1e9 / peak, 4),
            "step_moved_bytes_per_pt": moved, "step_moved_frac": round(moved * v / 1e9 / peak, 4),
            "roofline": single_roofline(r["profile"], npts, prec, peak, peak_kind, traffic_table, w.name,
                                        r["plan"]),
            "clocks": r["clocks"], "plan": r["plan"]}


def single_line(ses, w, W, stream, peak, peak_kind, traffic_table, clocks_gpu):
    out = {"workload": w.name, "grid": list(w.grid.dims), "dt": w.dt}
    for prec in ("c64", "c128"):
        r = single_precision(ses, w, prec, W, stream, clocks_gpu)
        out[prec] = single_entry(w, prec, r, peak, peak_kind, traffic_table)
    return out


def c3_transmission(ses, w):
    """C3's own output: P(x >= 1) every 50 steps over the config's 500 steps (complex64)."""
    op = ses.SplitOperator3D(w.grid, w.V, w.dt, w.mass, precision="c64", psi0=w.psi0)
    op.set_absorber_separable(*w.mask)
    rows = []
    for s in range(w.observe_every, w.steps + 1, w.observe_every):
        op.advance(w.observe_every, absorb=True)
        o = op.observe(1.0, math.inf)
        rows.append((s, o["p_range"], o["norm"]))
    op.close()
    return rows


def other_configs(ses, W, stream, peak, peak_kind, traffic_table, clocks_gpu):
    """The remaining named single-instance configurations at 1 GPU: C1 (64^3 harmonic,
    plain FP64) and C3 (512^3 tunnelling, complex64, 1 GiB field)."""
    from shoeridingerequationsolver_b200 import scenes
    out = {}
    for w, prec in ((scenes.config_c1(), "c128"), (scenes.config_c3(512), "c64")):
        r = single_precision(ses, w, prec, W, stream, clocks_gpu)
        e = single_entry(w, prec, r, peak, peak_kind, traffic_table)
        e["note"] = ("64^3 complex128 fits in L2 (4 MiB): the model fraction can exceed 1"
                     if w.grid.size() < 2 ** 20 else "field and table far larger than L2")
        if w.name.startswith("c3"):
            e["transmitted_every_50"] = c3_transmission(ses, w)
        out[w.name] = e
    return out


# ---------------------------------------------------------------------------
def run_reference(args):
    """The reference's own FP64 CPU core (oracle/_ref) on a bounded sample of the
    workload, all host threads; no device code of this repository is mapped."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle.oracle import Reference
    from oracle.parity import full_mask
    world = args.gpus
    if not Reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libsesref.so was not built "
                                                              "(the reference tree was absent at build time)"}))
        return 0
    if args.config == "c4":
        specs = c4_all_specs(args, world)
        r = reference_c4_rates(specs, args.warmup, args.steps, budget_s=120.0)
        cfg = c4_config(specs, world, args)
        cb = {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": "reference",
              "sample": f"each step: one reference SplitOperator3D::step (+ mask) of one instance per size "
                        f"{sorted(int(k) for k in r['per_size'])} ({r['sample_points']} points); value = the "
                        f"whole mix at those per-size rates (48/96/160 at 64/128/256)",
              "per_size": r["per_size"]}
        steps_done, ms_step = r["steps_timed"], r["sample_ms_per_step"]
    else:
        w = single_workload(args)
        npts = w.grid.size()
        mask = full_mask(w.mask)
        ref = Reference(workers=os.cpu_count())
        s = ref.split3d(w.grid.box, w.grid.dims, w.V, w.dt, w.mass)
        s.set_psi(w.psi0)
        s.step(max(0, args.warmup), mask)
        t0 = time.perf_counter()
        steps_done = 0
        while steps_done < max(1, args.steps):
            s.step(1, mask)
            steps_done += 1
            if time.perf_counter() - t0 > 120.0:
                break
        dt = time.perf_counter() - t0
        s.close()
        ms_step = 1e3 * dt / steps_done
        cb = {"value": npts * steps_done / dt, "unit": UNIT, "cores": ref.workers(), "kind": "reference",
              "sample": f"{steps_done} reference SplitOperator3D::step (+ mask) of {w.name}"}
        cfg = {"workload": w.name, "grid": list(w.grid.dims), "parallelism": f"replicas x{world}",
               "l2": "inputs larger than L2, no flush"}
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": world, "impl": "reference",
            "steps": steps_done, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic", "config": cfg,
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    if "SES_TUNE_CACHE" not in os.environ:  # this run's own autotune cache
        import tempfile
        os.environ["SES_TUNE_CACHE"] = os.path.join(tempfile.mkdtemp(prefix="ses_tune_"), "autotune.txt")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local)
    import torch
    import shoeridingerequationsolver_b200 as ses
    from shoeridingerequationsolver_b200 import replicas
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        torch.cuda.set_device(0)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    if ses.device_count() < 1:
        raise RuntimeError("no CUDA device visible")
    peak, peak_kind = load_peaks()
    traffic_table = {}
    tp = ROOT / "profiles" / "traffic.json"
    if tp.exists():
        traffic_table = json.loads(tp.read_text())
    stream = torch.cuda.Stream()
    K, W = args.steps, args.warmup
    if W < 3:
        raise SystemExit("--warmup must be >= 3")
    clocks_gpu = local if world > 1 else 0

    if args.config != "c4":  # single-instance workloads
        w = single_workload(args)
        r = single_precision(ses, w, args.precision, W, stream, clocks_gpu, K=K)
        e = single_entry(w, args.precision, r, peak, peak_kind, traffic_table)
        ms = replicas.max_over_ranks(r["ms"], dist, device="cuda")
        out = {"metric": METRIC, "value": world * w.grid.size() * r["K"] / (ms * 1e-3), "unit": UNIT,
               "n_gpus": world, "steps": r["K"], "warmup": W, "ms_per_step": ms / r["K"], "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
               "config": {"workload": w.name, "grid": list(w.grid.dims), "parallelism": f"replicas x{world}",
                          "l2": ("inputs larger than L2, no flush" if w.grid.size() * ESIZE[args.precision] > L2_BYTES
                                 else "field smaller than L2 (the configuration's whole working set): no flush")},
               "clocks": e["clocks"], "roofline": e["roofline"], "single": e}
        if rank == 0:
            print(json.dumps(out), flush=True)
        if dist:
            dist.destroy_process_group()
        return 0

    # ---- C4 batched sweep (headline) ----
    all_specs = c4_all_specs(args, world)
    specs = replicas.route_balanced(all_specs, rank, world, lambda s: s["n"] ** 3) if world > 1 else all_specs
    npts = sum(sp["n"] ** 3 for sp in specs)
    t_build = time.perf_counter()
    ops = build_c4(ses, specs)
    b = ses.Batch(ops)
    b.set_stream(stream.cuda_stream)
    plan = b.info() if NO_AUTOTUNE else b.autotune(save=False)
    b.prepare(absorb=True)           # every class's step graph, recorded before warm-up and timing
    build_s = time.perf_counter() - t_build
    b.step(W, absorb=True)
    b.sync(120000)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = events()
    with ClockSampler(clocks_gpu, ms=100) as clk:
        e0.record(stream)
        b.step(K, absorb=True)
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    ms = replicas.max_over_ranks(e0.elapsed_time(e1), dist, device="cuda")
    total_pts = replicas.sum_over_ranks(npts, dist, device="cuda")
    value = total_pts * K / (ms * 1e-3)
    prof = b.profile(8, absorb=True)
    ncls = len(prof)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64", "data": "synthetic", "config": c4_config(all_specs, world, args),
        "clocks": clk.summary(),
        "gpu_launches": ncls * (4 * K + 1),
        "roofline": batch_roofline(prof, specs, peak, peak_kind, traffic_table),
        "step_model": {"bytes_per_pt": MODEL_BYTES[("c64", 3)],
                       "achieved_gbs": round(MODEL_BYTES[("c64", 3)] * value / world / 1e9, 1),
                       "frac": round(MODEL_BYTES[("c64", 3)] * value / world / 1e9 / peak, 4),
                       "actual_bytes_per_pt": ACTUAL_BYTES["c64"],
                       "moved_gbs": round(ACTUAL_BYTES["c64"] * value / world / 1e9, 1),
                       "moved_frac": round(ACTUAL_BYTES["c64"] * value / world / 1e9 / peak, 4),
                       "note": "4 sweeps per step (x with the potential, y fwd, z fused, y inv) move "
                               "72 B/pt against the 104 B/pt model"},
        "per_class_ms": {str(n): {"step": round(p["step"], 4), "x_mid": round(p["x_mid"], 4),
                                  "mid": [round(x, 4) for x in p["mid"]]}
                         for n, p in zip(class_order(specs), prof)},
        "plan": plan, "build_s": round(build_s, 1),
        "setup": "autotune + graph recording (ses_batch_prepare) before the warm-up steps",
    }
    if args.quick:
        args.no_cpu = args.no_serve = args.no_single = True
        args.accuracy_steps = 0
    if rank == 0:
        line["fp64_plain"] = fp64_plain_mix(ses, specs, stream)
        line["fp64_plain"]["fp32_batched_over_fp64_plain"] = round(value / world / line["fp64_plain"]["value"], 3)
        line["e2e"] = c4_e2e(ses, b, ops, specs)
        if world > 1:
            line["e2e"]["value"] *= world
            line["e2e"]["note"] = "rank 0 measured its share; shares are independent, scaled by world size"
    b.close()
    for op in ops:
        op.close()
    del ops
    if rank == 0:
        acc_steps = 1000 if args.accuracy_steps < 0 else args.accuracy_steps
        if acc_steps > 0:
            line["accuracy"] = c4_accuracy(ses, specs, acc_steps)
        if not args.no_serve:
            line["serve"] = serve_run(ses, args.serve_requests)
            line["serve"]["fp64_plain"] = fp64_plain_c5(ses, args.serve_requests, stream)
            line["serve"]["fp32_serve_over_fp64_plain"] = round(
                line["serve"]["throughput"] / line["serve"]["fp64_plain"]["value"], 3)
        if not args.no_single:
            from shoeridingerequationsolver_b200 import scenes
            line["single_c2"] = single_line(ses, scenes.config_c2(256), W, stream, peak, peak_kind,
                                            traffic_table, clocks_gpu)
            line["configs"] = other_configs(ses, W, stream, peak, peak_kind, traffic_table, clocks_gpu)
        if world == 1 and not args.no_cpu:
            line["cpu_baseline"] = cpu_baseline_c4(specs)
            if not args.no_parity:
                line["parity"] = parity_runs(ses)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


NO_AUTOTUNE = False


def main(argv=None):
    global NO_AUTOTUNE
    args = parse_args(argv)
    if args.precision is None:
        args.precision = "c128" if args.config == "c1" else "c64"
    NO_AUTOTUNE = args.no_autotune
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
