#!/usr/bin/env python
"""Benchmark of the Strang split-operator step on B200 (one JSON line on stdout).

Workload (default): the 256^3 hydrogen-like configuration -- regularized
Coulomb Z=1 plus Stark term 0.01 z on [-40,40)^3, seeded superposition of four
Gaussians, cos^(1/8) absorber on the outer 10% of each axis, dt = 0.01 --
propagated with the complex64 path (FP64-built tables, FP64 diagonal math and
reductions) as the headline and the plain complex128 path beside it.  Inputs
are synthetic (no dataset exists for this path); psi (128/256 MiB) plus its
potential table exceed the 126 MB L2, so no flush is needed between steps.

A "step" is one Strang step of the 256^3 instance (potential kick, 3D FFT,
kinetic phase, inverse 3D FFT, kick, absorber).  value = grid points x steps
per second for the whole job (N GPUs each propagate their own replica: the
path does not shard a single grid without an all-to-all, so multi-GPU runs are
independent replicas, weak scaling).

--impl reference times the reference's own FP64 CPU core (compiled from its
sources into oracle/_ref) on the same workload with all host threads.
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
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "grid-pt*steps/s"
UNIT = "grid-pt*steps/s"
# algorithmic bytes per grid point per Strang step: 2*d*2*E + E_tab (d = 3)
BYTES_PER_PT = {"c128": 208, "c64": 104}
ESIZE = {"c128": 16, "c64": 8}


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=["c1", "c2", "c3"], default="c2")
    ap.add_argument("--n", type=int, default=0, help="override the grid size (parity/size sweeps)")
    ap.add_argument("--precision", choices=["c64", "c128"], default="c64")
    ap.add_argument("--no-secondary", action="store_true", help="skip the complex128 line")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--e2e-requests", type=int, default=5)
    ap.add_argument("--segment", type=int, default=100, help="steps per end-to-end request")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the cached / SES_XVAR, SES_SVAR tile variants instead of tuning")
    ap.add_argument("--quick", action="store_true",
                    help="timed region and per-pass profile only (for profiler launch lists)")
    ap.add_argument("--accuracy-steps", type=int, default=-1,
                    help="steps of the c64-vs-c128 accuracy check (-1: the config's step count)")
    return ap.parse_args(argv)


def workload(args):
    from shoeridingerequationsolver_b200 import scenes
    if args.config == "c1":
        return scenes.config_c1()
    if args.config == "c3":
        return scenes.config_c3(args.n or 512)
    return scenes.config_c2(args.n or 256)


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
        return {"sm_mhz": med, "sm_max_mhz": mx or None, "reasons": sorted(reasons),
                "samples": len(sm)}


def timed_batch(op, stream, K, absorb):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    op.advance(K, absorb=absorb)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def roofline_from_profile(prof, npts, prec, peak_gbs, peak_kind, traffic_table, wname):
    """Dominant kernel of a 3D step and its achieved algorithmic bandwidth.

    Per-launch algorithmic bytes split the 2*d*2*E + E_tab model per pass:
    x between steps = x inverse + x forward + table read (4E + E_tab), y forward
    2E, last-axis fused = z forward + z inverse (4E), y inverse 2E."""
    E = ESIZE[prec]
    per_pt = {"x_mid": 4 * E + E, "y_fwd": 2 * E, "fused": 4 * E, "y_inv": 2 * E}
    kinds = {k: prof[k] for k in per_pt if prof.get(k, 0) > 0}
    dom = max(kinds, key=kinds.get)
    alg = per_pt[dom] * npts
    achieved = alg / (kinds[dom] * 1e-3) / 1e9
    tr = traffic_table.get(f"{wname}:{prec}:{dom}")
    return {
        "kernel": dom,
        "bound": "hbm",
        "achieved": round(achieved, 1),
        "peak": peak_gbs,
        "peak_kind": peak_kind,
        "unit": "GB/s",
        "frac": round(achieved / peak_gbs, 4),
        "traffic": tr,
        "algorithmic_bytes_per_launch": alg,
        "launch_ms": round(kinds[dom], 5),
        "pass_ms": {k: round(v, 5) for k, v in kinds.items()},
    }


def rel_l2(a, b):
    import numpy as np
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def cpu_baseline(w, budget_s=15.0):
    """The reference core (oracle/_ref) on the host cores, bounded sample."""
    from oracle.oracle import Reference, Oracle
    import numpy as np
    mask = None
    if w.mask is not None:
        mx, my, mz = w.mask
        # full-N mask = (mx[i] * my[j]) * mz[k], the product order of absorbing_mask
        mask = np.ascontiguousarray((mx[None, None, :] * my[None, :, None]) * mz[:, None, None]).reshape(-1)
    npts = w.grid.size()
    if Reference.available():
        ref = Reference(workers=os.cpu_count())
        s = ref.split3d(w.grid.box, w.grid.dims, w.V, w.dt, w.mass)
        s.set_psi(w.psi0)
        t0 = time.perf_counter()
        s.step(1, mask)
        t1 = time.perf_counter() - t0
        n = max(1, min(50, int(budget_s / max(t1, 1e-6))))
        t0 = time.perf_counter()
        s.step(n, mask)
        dt = time.perf_counter() - t0
        s.close()
        return {"value": npts * n / dt, "unit": UNIT, "cores": ref.workers(), "kind": "reference",
                "sample": f"{n} Strang steps (+ mask) of the {w.name} grid, after 1 untimed step; "
                          f"reference SplitOperator3D::step via ses.parallel",
                "ms_per_step": dt / n * 1e3}
    o = Oracle()
    t0 = time.perf_counter()
    o.step3d(w.grid.box, w.grid.dims, w.V, w.dt, w.psi0, 1, w.mass, mask)
    dt = time.perf_counter() - t0
    return {"value": npts / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"1 Strang step (+ mask, including table build) of the {w.name} grid, "
                      f"C restatement, single thread", "ms_per_step": dt * 1e3}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    w = workload(args)
    base = {"metric": METRIC, "unit": UNIT, "n_gpus": args.gpus, "impl": "reference",
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic",
            "config": {"workload": w.name, "grid": list(w.grid.dims), "dt": w.dt,
                       "absorber": "cos^(1/8), separable"}}
    from oracle.oracle import Reference, Oracle
    import numpy as np
    mx, my, mz = w.mask if w.mask is not None else (None, None, None)
    mask = None if mx is None else np.ascontiguousarray(
        (mx[None, None, :] * my[None, :, None]) * mz[:, None, None]).reshape(-1)
    npts = w.grid.size()
    if Reference.available():
        ref = Reference(workers=os.cpu_count())
        s = ref.split3d(w.grid.box, w.grid.dims, w.V, w.dt, w.mass)
        s.set_psi(w.psi0)
        t0 = time.perf_counter()
        s.step(max(1, args.warmup), mask)
        t_w = (time.perf_counter() - t0) / max(1, args.warmup)
        k = args.steps
        cap = max(1, int(150.0 / max(t_w, 1e-6)))
        k_timed = min(k, cap)
        t0 = time.perf_counter()
        s.step(k_timed, mask)
        dt = time.perf_counter() - t0
        s.close()
        kind, cores = "reference", ref.workers()
        sample = (f"{k_timed} of the requested {k} Strang steps (+ mask) of {w.name}, reference "
                  f"SplitOperator3D::step through ses.parallel")
    else:
        o = Oracle()
        k_timed = 1
        t0 = time.perf_counter()
        o.step3d(w.grid.box, w.grid.dims, w.V, w.dt, w.psi0, 1, w.mass, mask)
        dt = time.perf_counter() - t0
        kind, cores = "port", 1
        sample = f"1 Strang step of {w.name}, C restatement (reference core not built)"
    value = npts * k_timed / dt
    line = dict(base, value=value, steps=args.steps, warmup=args.warmup,
                ms_per_step=dt / k_timed * 1e3,
                cpu_baseline={"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                              "sample": sample},
                e2e={"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
    print(json.dumps(line), flush=True)
    return 0


def measure_precision(ses, w, prec, K, W, stream, dist, world, clocks_gpu):
    import torch
    op = ses.SplitOperator3D(w.grid, w.V, w.dt, w.mass, precision=prec)
    absorb = w.mask is not None
    if absorb:
        op.set_absorber_separable(*w.mask)
    op.set_stream(stream.cuda_stream)
    # pick tile variants on the scratch field (untimed)
    plan = op.plan_info() if NO_AUTOTUNE else op.autotune(save=False)
    op.upload_state(w.psi0)
    warm = max(W, 9)  # >= 9 so the captured step graph exists before timing
    op.advance(warm, absorb=absorb)
    op.sync(60000)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(clocks_gpu) as clk:
        ms = timed_batch(op, stream, K, absorb)
    torch.cuda.synchronize()
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    prof = op.profile_step(K, absorb=absorb)
    op.close()
    return {"ms": ms, "profile": prof, "clocks": clk.summary(), "warmup": warm, "plan": plan}


def accuracy(ses, w, steps):
    """complex64 path vs complex128 path after `steps` Strang steps from the same psi0."""
    out = {}
    res = {}
    for prec in ("c128", "c64"):
        op = ses.SplitOperator3D(w.grid, w.V, w.dt, w.mass, precision=prec)
        if w.mask is not None:
            op.set_absorber_separable(*w.mask)
        op.upload_state(w.psi0)
        o0 = op.observe(*w.x_range)
        op.advance(steps, absorb=w.mask is not None)
        o1 = op.observe(*w.x_range)
        res[prec] = (op.readback(), o0, o1)
        op.close()
    psi128, a0, a1 = res["c128"]
    psi64, b0, b1 = res["c64"]
    out["steps"] = steps
    out["rel_l2_c64_vs_c128"] = rel_l2(psi64, psi128)
    out["norm_c128"] = a1["norm"]
    out["norm_c64"] = b1["norm"]
    out["norm_diff"] = b1["norm"] - a1["norm"]
    out["energy_c128"] = a1["energy"]
    out["energy_diff"] = b1["energy"] - a1["energy"]
    out["energy0"] = a0["energy"]
    return out


def e2e(ses, w, prec, stream, requests, segment):
    """Requests through the public API with host buffers: upload psi (pinned
    complex128), `segment` steps, norm/energy readout, psi readback."""
    import torch
    npts = w.grid.size()
    op = ses.SplitOperator3D(w.grid, w.V, w.dt, w.mass, precision=prec)
    absorb = w.mask is not None
    if absorb:
        op.set_absorber_separable(*w.mask)
    op.set_stream(stream.cuda_stream)
    h_in = torch.empty(2 * npts, dtype=torch.float64, pin_memory=True)
    h_out = torch.empty(2 * npts, dtype=torch.float64, pin_memory=True)
    import numpy as np
    h_in.numpy()[:] = w.psi0.view(np.float64)
    # warm: one request untimed
    op.write_ptr(h_in.data_ptr())
    op.advance(segment, absorb=absorb)
    op.observe(*w.x_range)
    op.read_ptr(h_out.data_ptr())
    t0 = time.perf_counter()
    for _ in range(requests):
        op.write_ptr(h_in.data_ptr())
        op.advance(segment, absorb=absorb)
        op.observe(*w.x_range)
        op.read_ptr(h_out.data_ptr())
    dt = time.perf_counter() - t0
    op.close()
    return {"value": npts * segment * requests / dt, "unit": UNIT,
            "h2d_bytes_per_step": 16 * npts, "d2h_bytes_per_step": 16 * npts + 14 * 8,
            "step": f"one request: upload psi (complex128, pinned), {segment} Strang steps, "
                    f"norm/energy/observables readout, psi readback",
            "requests": requests}


def run_ours(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local)
    import torch
    import shoeridingerequationsolver_b200 as ses
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        torch.cuda.set_device(0)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    if ses.device_count() < 1:
        raise RuntimeError("no CUDA device visible")
    w = workload(args)
    npts = w.grid.size()
    peak, peak_kind = load_peaks()
    traffic_table = {}
    tp = ROOT / "profiles" / "traffic.json"
    if tp.exists():
        traffic_table = json.loads(tp.read_text())
    stream = torch.cuda.Stream()
    K = args.steps
    prim = measure_precision(ses, w, args.precision, K, args.warmup, stream, dist, world,
                             local if world > 1 else 0)
    value = world * npts * K / (prim["ms"] * 1e-3)
    roof = roofline_from_profile(prim["profile"], npts, args.precision, peak, peak_kind,
                                 traffic_table, w.name)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": prim["warmup"], "ms_per_step": prim["ms"] / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
        "config": {"workload": w.name, "grid": list(w.grid.dims), "dt": w.dt,
                   "absorber": "cos^(1/8) separable" if w.mask is not None else None,
                   "precision": args.precision,
                   "tables": "FP64-built (potential table stored complex64 as cis-1 for c64)",
                   "l2": "inputs larger than L2 (psi + potential table > 126 MB), no flush",
                   "parallelism": f"replicas x{world}"},
        "clocks": prim["clocks"],
        "gpu_launches": prim["profile"]["launches"],
        "roofline": roof,
        "step_roofline": {"model_bytes_per_pt": BYTES_PER_PT[args.precision],
                          "achieved_gbs": round(BYTES_PER_PT[args.precision] * npts * K /
                                                (prim["ms"] * 1e-3) / 1e9, 1),
                          "peak": peak, "frac": None},
        "profiled_batch_ms": prim["profile"]["total_ms"],
        "plan": prim["plan"],
    }
    line["step_roofline"]["frac"] = round(line["step_roofline"]["achieved_gbs"] / peak, 4)
    if args.quick:
        args.no_secondary, args.no_cpu, args.accuracy_steps, args.e2e_requests = True, True, 0, 0
    if not args.no_secondary and args.precision == "c64":
        sec = measure_precision(ses, w, "c128", K, args.warmup, stream, dist, world,
                                local if world > 1 else 0)
        v128 = world * npts * K / (sec["ms"] * 1e-3)
        line["fp64_plain"] = {
            "value": v128, "ms_per_step": sec["ms"] / K, "dtype": "c128",
            "roofline": roofline_from_profile(sec["profile"], npts, "c128", peak, peak_kind,
                                              traffic_table, w.name),
            "step_achieved_gbs": round(208 * npts * K / (sec["ms"] * 1e-3) / 1e9, 1),
            "step_frac": round(208 * npts * K / (sec["ms"] * 1e-3) / 1e9 / peak, 4),
            "clocks": sec["clocks"],
            "plan": sec["plan"],
            "c64_over_c128": value / v128,
        }
    if rank == 0:
        acc_steps = w.steps if args.accuracy_steps < 0 else args.accuracy_steps
        if acc_steps > 0:
            line["accuracy"] = accuracy(ses, w, acc_steps)
        if args.e2e_requests > 0:
            line["e2e"] = e2e(ses, w, args.precision, stream, args.e2e_requests, args.segment)
        if world > 1 and "e2e" in line:
            line["e2e"]["value"] *= world
            line["e2e"]["note"] = "rank 0 measured; replicas are independent, scaled by world size"
        if world == 1 and not args.no_cpu:
            line["cpu_baseline"] = cpu_baseline(w)
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
