"""Config-level parity runs of the device path against the FP64 oracle (TEST
INFRASTRUCTURE: used by tests/ and by bench.py's CPU-baseline leg as the checker).

A ``Checker`` steps one scene on the CPU in segments.  On grids that are powers
of two on every axis it runs the reference's own core (oracle/_ref,
SplitOperator3D::step over ses.parallel, core/src/propagator.ixx:110-119, mask
multiplied after every step) when that library was built, else the C
restatement (bit-identical to the reference there); mixed-radix grids use the
restatement.  Observables are the restatement's serial FP64 sums
(core/src/field.ixx:68-74, observables.ixx:121-234).
"""

from __future__ import annotations

import math
import time

import numpy as np


def rel_l2(a, b) -> float:
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def full_mask(mask):
    """The separable absorber (mx, my, mz) as one N-array, x fastest."""
    if mask is None:
        return None
    mx, my, mz = mask
    return np.ascontiguousarray((mx[None, None, :] * my[None, :, None]) * mz[:, None, None]).reshape(-1)


def _pow2(n: int) -> bool:
    return n & (n - 1) == 0


class Checker:
    """FP64 CPU propagation of workload `w` (fields of scenes.Workload)."""

    def __init__(self, oracle, reference_cls, w, use_reference: bool = True):
        self.w = w
        self.box, self.dims = w.grid.box, w.grid.dims
        self.mask = full_mask(w.mask)
        self.oracle = oracle
        self.ref = None
        if use_reference and reference_cls is not None and reference_cls.available() and \
                all(_pow2(d) for d in self.dims):
            self.ref = reference_cls().split3d(self.box, self.dims, w.V, w.dt, w.mass)
            self.ref.set_psi(w.psi0)
        self.psi = np.array(w.psi0, dtype=np.complex128, copy=True)
        self.kind = "reference core (oracle/_ref)" if self.ref else "C restatement (oracle/libses_oracle.so)"
        self.cpu_s = 0.0

    def step(self, k: int):
        t0 = time.perf_counter()
        if self.ref:
            self.ref.step(k, self.mask)
            self.psi = self.ref.get_psi()
        else:
            self.psi = self.oracle.step3d(self.box, self.dims, self.w.V, self.w.dt, self.psi, k, self.w.mass,
                                          self.mask)
        self.cpu_s += time.perf_counter() - t0
        return self.psi

    def norm(self) -> float:
        return self.oracle.norm3d(self.box, self.dims, self.psi)

    def energy(self) -> float:
        return self.oracle.mean_energy3d(self.box, self.dims, self.psi, self.w.V, self.w.mass)

    def p_range(self, a: float, b: float) -> float:
        return self.oracle.prob_x_range3d(self.box, self.dims, self.psi, a, b)

    def close(self):
        if self.ref:
            self.ref.close()
            self.ref = None


def device_op(ses, w, prec: str):
    op = ses.SplitOperator3D(w.grid, w.V, w.dt, w.mass, precision=prec, psi0=w.psi0)
    if w.mask is not None:
        op.set_absorber_separable(*w.mask)
    return op


def run_segments(ses, oracle, reference_cls, w, prec: str, steps: int, every: int, xr=(-math.inf, math.inf)):
    """Step `w` on the device and on the checker in segments of `every` steps;
    per segment: relative L2 of psi, norm and energy (device and oracle), and the
    probability in the x-interval xr."""
    chk = Checker(oracle, reference_cls, w)
    op = device_op(ses, w, prec)
    absorb = w.mask is not None
    rows = []
    o0 = op.observe(*xr)
    n0_ref, e0_ref = chk.norm(), chk.energy()
    done = 0
    while done < steps:
        k = min(every, steps - done)
        op.advance(k, absorb=absorb)
        chk.step(k)
        done += k
        obs = op.observe(*xr)
        rows.append({"step": done, "rel_l2": rel_l2(op.readback(), chk.psi),
                     "norm": obs["norm"], "norm_oracle": chk.norm(),
                     "energy": obs["energy"], "energy_oracle": chk.energy(),
                     "p_range": obs["p_range"], "p_range_oracle": chk.p_range(*xr)})
    op.close()
    chk.close()
    last = rows[-1]
    return {"precision": prec, "steps": steps, "checker": chk.kind, "checker_cpu_s": round(chk.cpu_s, 2),
            "rel_l2": last["rel_l2"], "max_rel_l2": max(r["rel_l2"] for r in rows),
            "norm_diff": last["norm"] - last["norm_oracle"],
            "max_abs_norm_diff": max(abs(r["norm"] - r["norm_oracle"]) for r in rows),
            "energy_diff": last["energy"] - last["energy_oracle"],
            "max_abs_energy_diff": max(abs(r["energy"] - r["energy_oracle"]) for r in rows),
            "norm_drift": last["norm"] - o0["norm"], "norm_drift_oracle": last["norm_oracle"] - n0_ref,
            "energy_drift": last["energy"] - o0["energy"], "energy_drift_oracle": last["energy_oracle"] - e0_ref,
            "series": rows}
