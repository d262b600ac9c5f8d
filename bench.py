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
1D/2D/3D requests, p50/p99 latency), the single-instance 256^3 numbers and the
reference's FP64 CPU core on the host cores.  Multi-GPU runs are independent
replicas (the instances are independent; no collective), weak scaling.

--impl reference times the reference's own FP64 CPU core (compiled from its
sources into oracle/_ref) on a bounded sample of the same workload with all
host threads.
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
ESIZE = {"c128": 16, "c64": 8}


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=["c4", "c2", "c3", "c1"], default="c4")
    ap.add_argument("--instances", type=int, default=256, help="batched sweep size (c4)")
    ap.add_argument("--sizes", default="", help="c4: keep only these grid sizes (comma list), for profiling")
    ap.add_argument("--n", type=int, default=0, help="grid size override for c1/c2/c3")
    ap.add_argument("--precision", choices=["c64", "c128"], default="c64")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving run")
    ap.add_argument("--no-single", action="store_true", help="skip the single-instance 256^3 line")
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
    """nvidia-smi samples (200 ms) during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
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


def full_mask(mask):
    import numpy as np
    mx, my, mz = mask
    return np.ascontiguousarray((mx[None, None, :] * my[None, :, None]) * mz[:, None, None]).reshape(-1)


# ---------------------------------------------------------------------------
# C4: the batched sweep
# ---------------------------------------------------------------------------
def c4_specs(args):
    from shoeridingerequationsolver_b200 import scenes
    if not args.sizes:
        return scenes.config_c4_specs(args.instances)
    keep = {int(x) for x in args.sizes.split(",")}
    return [s for s in scenes.config_c4_specs(256) if s["n"] in keep][:args.instances]


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
    2E, z fused (fwd, K/N, inv) 4E, y inverse 2E (E = 8, complex64)."""
    E = ESIZE["c64"]
    per_pt = [4 * E + E, 2 * E, 4 * E, 2 * E]
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
    key = f"c4:{n}:{names[k]}"
    return {"kernel": f"{names[k]} pass of the {n}^3 class ({counts[n]} instances, one launch)",
            "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "peak_kind": peak_kind,
            "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic_table.get(key),
            "algorithmic_bytes_per_launch": alg, "launch_ms": round(ms, 5)}


def fp64_plain_mix(ses, specs, stream, warm=9, K=40):
    """The plain FP64 path on the same mix: complex128, every instance alone
    (one handle, its own launches), per-size time per step x instance count."""
    from shoeridingerequationsolver_b200 import scenes
    counts = Counter(sp["n"] for sp in specs)
    per_size = {}
    total_ms = 0.0
    for n in sorted(counts):
        sp = next(s for s in specs if s["n"] == n)
        w = scenes.build_c4_instance(sp)
        op = ses.SplitOperator3D(w.grid, w.V, w.dt, w.mass, precision="c128", psi0=w.psi0)
        op.set_absorber_separable(*w.mask)
        op.set_stream(stream.cuda_stream)
        if not NO_AUTOTUNE:
            op.autotune(save=False)
        op.advance(warm, absorb=True)
        op.sync(60000)
        e0, e1 = events()
        e0.record(stream)
        op.advance(K, absorb=True)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / K
        op.close()
        per_size[n] = round(ms, 5)
        total_ms += ms * counts[n]
    npts = sum(sp["n"] ** 3 for sp in specs)
    return {"value": npts / (total_ms * 1e-3), "ms_per_step": total_ms, "dtype": "c128",
            "ms_per_step_by_size": per_size,
            "how": f"each size alone ({K} timed steps after {warm}), times the instance count"}


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
            "reference": "plain complex128 GPU path (itself within 1e-12 per step of the FP64 oracle)"}


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


def cpu_baseline_c4(specs, budget_s=15.0):
    """The reference core (oracle/_ref) on the host cores: SplitOperator3D::step
    threaded by ses.parallel, one instance per grid size, per-size time per step
    x instance count.  The reference transforms powers of two only (it throws
    for 48, 96, 160: core/src/fft.ixx:42-44), so those sizes are charged at the
    per-point rate the reference reaches on the next power of two (64, 128, 256)."""
    from oracle.oracle import Reference, Oracle
    from shoeridingerequationsolver_b200 import scenes
    counts = Counter(sp["n"] for sp in specs)
    npts = sum(sp["n"] ** 3 for sp in specs)
    pow2 = lambda n: n & (n - 1) == 0
    stand_in = {n: (n if pow2(n) else 1 << n.bit_length()) for n in counts}
    per = {}
    if Reference.available():
        ref = Reference(workers=os.cpu_count())
        rate = {}
        for m in sorted(set(stand_in.values())):
            sp = next((s for s in specs if s["n"] == m), None)
            sp = dict(sp) if sp else dict(next(iter(specs)), n=m, side=20.0 * m / 32.0)
            w = scenes.build_c4_instance(sp)
            s = ref.split3d(w.grid.box, w.grid.dims, w.V, w.dt, w.mass)
            s.set_psi(w.psi0)
            msk = full_mask(w.mask)
            t0 = time.perf_counter()
            s.step(1, msk)
            t1 = time.perf_counter() - t0
            k = max(1, min(20, int(budget_s / len(stand_in) / max(t1, 1e-6))))
            t0 = time.perf_counter()
            s.step(k, msk)
            dt = (time.perf_counter() - t0) / k
            s.close()
            rate[m] = m ** 3 / dt
            per[m] = {"ms_per_step": round(dt * 1e3, 3), "steps": k}
        total_s = sum(counts[n] * n ** 3 / rate[stand_in[n]] for n in counts)
        return {"value": npts / total_s, "unit": UNIT, "cores": ref.workers(), "kind": "reference",
                "sample": "reference SplitOperator3D::step via ses.parallel, one instance per power-of-two "
                          "size (k steps + mask after 1 untimed step); 48/96/160 (which the reference "
                          "rejects) charged at the per-point rate of 64/128/256; mix time = sum over sizes",
                "per_size": per}
    o = Oracle()
    total_s = 0.0
    for n in sorted(counts):
        sp = next(s for s in specs if s["n"] == n)
        w = scenes.build_c4_instance(sp)
        t0 = time.perf_counter()
        o.step3d(w.grid.box, w.grid.dims, w.V, w.dt, w.psi0, 1, w.mass, full_mask(w.mask))
        dt = time.perf_counter() - t0
        per[n] = {"ms_per_step": round(dt * 1e3, 3), "steps": 1}
        total_s += dt * counts[n]
    return {"value": npts / total_s, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "one Strang step per grid size, C restatement, single thread", "per_size": per}


# ---------------------------------------------------------------------------
# C5: serving
# ---------------------------------------------------------------------------
def serve_capacity(ses, ncal=16):
    """Closed-loop capacity of the server on this mix: a separate seeded draw of
    `ncal` requests submitted at once; grid-pt*steps of all rounds / wall time."""
    from shoeridingerequationsolver_b200 import scenes
    built = [scenes.build_c5_request(s) for s in scenes.config_c5_specs(ncal, seed=scenes.SEED_BASE + 40)]
    with ses.Server(budget_bytes=150 * 10**9, max_round_steps=100) as srv:
        t0 = time.perf_counter()
        for req in built:
            srv.submit(**req)
        srv.wait_idle(900000)
        wall = time.perf_counter() - t0
        st = srv.stats()
    return st["gridpt_steps"] / wall


def serve_run(ses, nreq, capacity_ptsteps=None, seed=None):
    """Poisson arrivals of mixed 1D/2D/3D requests into the request server; lambda
    set so the offered load is ~0.9 of the server's closed-loop capacity on the mix."""
    import numpy as np
    from shoeridingerequationsolver_b200 import scenes
    specs = scenes.config_c5_specs(nreq) if seed is None else scenes.config_c5_specs(nreq, seed=seed)
    mean_work = sum(s["points"] * s["steps"] for s in specs) / len(specs)
    if capacity_ptsteps is None:
        capacity_ptsteps = serve_capacity(ses)
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
            "capacity": capacity_ptsteps,
            "offered_load": "0.9 x the server's closed-loop capacity on a separate draw of the mix"}


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


def single_roofline(prof, npts, prec, peak, peak_kind, traffic_table, wname):
    """Dominant pass of a 3D step: per-launch algorithmic bytes x -> 4E + E_tab,
    y forward 2E, last-axis fused 4E, y inverse 2E."""
    E = ESIZE[prec]
    per_pt = {"x_mid": 4 * E + E, "y_fwd": 2 * E, "fused": 4 * E, "y_inv": 2 * E}
    kinds = {k: prof[k] for k in per_pt if prof.get(k, 0) > 0}
    dom = max(kinds, key=kinds.get)
    alg = per_pt[dom] * npts
    achieved = alg / (kinds[dom] * 1e-3) / 1e9
    return {"kernel": dom, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "traffic": traffic_table.get(f"{wname}:{prec}:{dom}"), "algorithmic_bytes_per_launch": alg,
            "launch_ms": round(kinds[dom], 5), "pass_ms": {k: round(v, 5) for k, v in kinds.items()}}


def single_precision(ses, w, prec, K, W, stream, clocks_gpu):
    op = ses.SplitOperator3D(w.grid, w.V, w.dt, w.mass, precision=prec)
    absorb = w.mask is not None
    if absorb:
        op.set_absorber_separable(*w.mask)
    op.set_stream(stream.cuda_stream)
    plan = op.plan_info() if NO_AUTOTUNE else op.autotune(save=False)
    op.upload_state(w.psi0)
    op.advance(max(W, 9), absorb=absorb)
    op.sync(60000)
    e0, e1 = events()
    with ClockSampler(clocks_gpu) as clk:
        e0.record(stream)
        op.advance(K, absorb=absorb)
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1)
    prof = op.profile_step(K, absorb=absorb)
    op.close()
    return {"ms": ms, "profile": prof, "clocks": clk.summary(), "plan": plan}


def single_line(ses, w, K, W, stream, peak, peak_kind, traffic_table, clocks_gpu):
    npts = w.grid.size()
    out = {"workload": w.name, "grid": list(w.grid.dims), "dt": w.dt}
    for prec in ("c64", "c128"):
        r = single_precision(ses, w, prec, K, W, stream, clocks_gpu)
        v = npts * K / (r["ms"] * 1e-3)
        mb = MODEL_BYTES[(prec, 3)]
        out[prec] = {"value": v, "ms_per_step": r["ms"] / K,
                     "step_model_gbs": round(mb * v / 1e9, 1), "step_frac": round(mb * v / 1e9 / peak, 4),
                     "roofline": single_roofline(r["profile"], npts, prec, peak, peak_kind, traffic_table, w.name),
                     "clocks": r["clocks"], "plan": r["plan"]}
    return out


def other_configs(ses, stream, peak, peak_kind, traffic_table, clocks_gpu):
    """The remaining named single-instance configurations at 1 GPU: C1 (64^3 harmonic,
    plain FP64) and C3 (512^3 tunnelling, complex64, 1 GiB field)."""
    from shoeridingerequationsolver_b200 import scenes
    out = {}
    for w, prec, K in ((scenes.config_c1(), "c128", 400), (scenes.config_c3(512), "c64", 50)):
        r = single_precision(ses, w, prec, K, 3, stream, clocks_gpu)
        npts = w.grid.size()
        v = npts * K / (r["ms"] * 1e-3)
        mb = MODEL_BYTES[(prec, 3)]
        out[w.name] = {"precision": prec, "value": v, "ms_per_step": r["ms"] / K, "steps_timed": K,
                       "step_model_frac": round(mb * v / 1e9 / peak, 4),
                       "roofline": single_roofline(r["profile"], npts, prec, peak, peak_kind, traffic_table, w.name),
                       "note": "64^3 complex128 fits in L2 (4 MiB): the model fraction can exceed 1" if npts < 2**20
                       else "field and table far larger than L2"}
    return out


# ---------------------------------------------------------------------------
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.config == "c4":
        from shoeridingerequationsolver_b200 import scenes
        specs = c4_specs(args)
        cb = cpu_baseline_c4(specs, budget_s=60.0)
        cfg = {"workload": f"c4_batched_tunnel_{args.instances}", "instances": args.instances,
               "sizes": sorted({s["n"] for s in specs}), "dt": 0.005, "precision": "c128 (FP64 CPU core)"}
        step_pts = sum(s["n"] ** 3 for s in specs)
    else:
        w = single_workload(args)
        from oracle.oracle import Reference, Oracle
        npts = w.grid.size()
        mask = full_mask(w.mask) if w.mask is not None else None
        if Reference.available():
            ref = Reference(workers=os.cpu_count())
            s = ref.split3d(w.grid.box, w.grid.dims, w.V, w.dt, w.mass)
            s.set_psi(w.psi0)
            t0 = time.perf_counter()
            s.step(max(1, args.warmup), mask)
            t_w = (time.perf_counter() - t0) / max(1, args.warmup)
            k = max(1, min(args.steps, int(150.0 / max(t_w, 1e-6))))
            t0 = time.perf_counter()
            s.step(k, mask)
            dt = time.perf_counter() - t0
            s.close()
            cb = {"value": npts * k / dt, "unit": UNIT, "cores": ref.workers(), "kind": "reference",
                  "sample": f"{k} Strang steps (+ mask) of {w.name}, reference SplitOperator3D::step"}
        else:
            o = Oracle()
            t0 = time.perf_counter()
            o.step3d(w.grid.box, w.grid.dims, w.V, w.dt, w.psi0, 1, w.mass, mask)
            dt = time.perf_counter() - t0
            cb = {"value": npts / dt, "unit": UNIT, "cores": 1, "kind": "port",
                  "sample": f"1 Strang step of {w.name}, C restatement"}
        cfg = {"workload": w.name, "grid": list(w.grid.dims), "dt": w.dt}
        step_pts = npts
    # one step of the whole workload at the sampled rate
    ms_step = 1e3 * step_pts / cb["value"] if cb["value"] > 0 else None
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus, "impl": "reference",
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic", "config": cfg,
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local)
    import torch
    import shoeridingerequationsolver_b200 as ses
    from shoeridingerequationsolver_b200 import scenes
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
    K, W = args.steps, max(args.warmup, 3)
    clocks_gpu = local if world > 1 else 0

    from shoeridingerequationsolver_b200 import replicas

    def max_over_ranks(ms):  # every rank runs its own replica of the workload (weak scaling)
        return replicas.max_over_ranks(ms, dist, device="cuda")

    if args.config != "c4":  # single-instance workloads
        w = single_workload(args)
        line = single_line(ses, w, K, W, stream, peak, peak_kind, traffic_table, clocks_gpu)
        prim = line[args.precision]
        out = {"metric": METRIC, "value": world * prim["value"], "unit": UNIT, "n_gpus": world, "steps": K,
               "warmup": W, "ms_per_step": prim["ms_per_step"], "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
               "config": {"workload": w.name, "grid": list(w.grid.dims), "parallelism": f"replicas x{world}",
                          "l2": "inputs larger than L2, no flush"},
               "clocks": prim["clocks"], "roofline": prim["roofline"], "single": line}
        if rank == 0:
            print(json.dumps(out), flush=True)
        if dist:
            dist.destroy_process_group()
        return 0

    # ---- C4 batched sweep (headline) ----
    specs = c4_specs(args)
    npts = sum(sp["n"] ** 3 for sp in specs)
    t_build = time.perf_counter()
    ops = build_c4(ses, specs)
    b = ses.Batch(ops)
    b.set_stream(stream.cuda_stream)
    plan = b.info() if NO_AUTOTUNE else b.autotune(save=False)
    build_s = time.perf_counter() - t_build
    b.step(max(W, 9), absorb=True)          # >= 9 so every class's step graph exists before timing
    b.sync(120000)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = events()
    with ClockSampler(clocks_gpu) as clk:
        e0.record(stream)
        b.step(K, absorb=True)
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1))
    value = world * npts * K / (ms * 1e-3)
    prof = b.profile(8, absorb=True)
    ncls = len(prof)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": max(W, 9),
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64", "data": "synthetic",
        "config": {"workload": f"c4_batched_tunnel_{len(specs)}" + (f"_sizes_{args.sizes}" if args.sizes else ""),
                   "instances": len(specs),
                   "sizes": dict(sorted(Counter(sp["n"] for sp in specs).items())), "grid_points": npts,
                   "dt": 0.005, "precision": "complex64 fields, FP64-built tables, FP64 reductions",
                   "absorber": "cos^(1/8) on the outer 8%, after every step",
                   "l2": "inputs (2.9 GB) larger than L2, no flush", "parallelism": f"replicas x{world}",
                   "seed": scenes.SEED_BASE + 3},
        "clocks": clk.summary(),
        "gpu_launches": K * 4 * ncls,
        "roofline": batch_roofline(prof, specs, peak, peak_kind, traffic_table),
        "step_model": {"bytes_per_pt": MODEL_BYTES[("c64", 3)],
                       "achieved_gbs": round(MODEL_BYTES[("c64", 3)] * value / world / 1e9, 1),
                       "frac": round(MODEL_BYTES[("c64", 3)] * value / world / 1e9 / peak, 4),
                       "actual_bytes_per_pt": 72,
                       "note": "4 sweeps per step (x with the potential, y fwd, z fused, y inv) move "
                               "72 B/pt against the 104 B/pt model"},
        "per_class_ms": {str(n): {"step": round(p["step"], 4), "x_mid": round(p["x_mid"], 4),
                                  "mid": [round(x, 4) for x in p["mid"]]}
                         for n, p in zip(class_order(specs), prof)},
        "plan": plan, "build_s": round(build_s, 1),
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
            line["e2e"]["note"] = "rank 0 measured; replicas are independent, scaled by world size"
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
        if not args.no_single:
            w = scenes.config_c2(256)
            line["single_c2"] = single_line(ses, w, 200, 3, stream, peak, peak_kind, traffic_table, clocks_gpu)
            line["configs"] = other_configs(ses, stream, peak, peak_kind, traffic_table, clocks_gpu)
        if world == 1 and not args.no_cpu:
            line["cpu_baseline"] = cpu_baseline_c4(specs)
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
    NO_AUTOTUNE = args.no_autotune
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
