"""The named configurations against the FP64 oracle, through the C ABI.

The checker (oracle/parity.py) is the reference's own core (oracle/_ref) on
power-of-two grids when it was built, else the C restatement; mixed-radix grids
use the restatement.

* C1 (64^3 harmonic, complex128): the full 2000 steps, psi, norm and energy
  every 100 steps (the config's observable cadence).
* C2 (256^3 regularized Coulomb + Stark, cos^(1/8) absorber): 10 steps at the
  full size in both precisions; the full 1000 steps of the same scene on a 128^3
  grid of the same box (spacing 0.625 instead of 0.3125).
* C3 (512^3 tunnelling, complex64): 5 steps at the full size; the full 500 steps
  on a 512 x 64 x 64 grid with the same spacing (transverse box [-7.5, 7.5)),
  transmitted probability P(x >= 1) every 50 steps, also with the packet moved
  to x = -5 so that part of it crosses the barrier within the run.
* C4 mixed radix: 1000 steps on 48^3, a 96 x 96 plane and 64^3 in both
  precisions.

Tolerances (relative L2 error ||gpu - oracle|| / ||oracle||): complex128 1e-12
per step, i.e. steps x 1e-12 after a run (measured values are far below);
complex64 1e-5 after <= 1000 steps, the north-star bar.  Norms: complex128
1e-11, complex64 1e-5 absolute; energies: complex128 1e-10, complex64 1e-4
relative.
"""

import math

import numpy as np
import pytest

from oracle.parity import Checker, device_op, rel_l2, run_segments
from shoeridingerequationsolver_b200 import scenes

pytestmark = pytest.mark.gpu


def ref_cls():
    from oracle.oracle import Reference
    return Reference


def test_c1_full_run_with_observables_every_100_steps(ses, oracle):
    w = scenes.config_c1()
    r = run_segments(ses, oracle, ref_cls(), w, "c128", w.steps, w.observe_every)
    assert len(r["series"]) == 20
    for row in r["series"]:
        assert row["rel_l2"] <= row["step"] * 1e-12, row
        assert abs(row["norm"] - row["norm_oracle"]) <= 1e-11, row
        assert abs(row["energy"] - row["energy_oracle"]) <= 1e-10, row
    assert r["max_rel_l2"] < 1e-11


@pytest.mark.parametrize("n,steps", [(256, 10), (128, 1000)])
def test_c2_coulomb_stark_both_precisions(ses, oracle, n, steps):
    w = scenes.config_c2(n)
    chk = Checker(oracle, ref_cls(), w)
    want = chk.step(steps)
    n_want, e_want = chk.norm(), chk.energy()
    chk.close()
    for prec in ("c128", "c64"):
        op = device_op(ses, w, prec)
        op.advance(steps, absorb=True)
        got = op.readback()
        obs = op.observe()
        op.close()
        err = rel_l2(got, want)
        if prec == "c128":
            assert err <= steps * 1e-12, (n, err)
            assert abs(obs["norm"] - n_want) <= 1e-11
            assert abs(obs["energy"] - e_want) <= 1e-10 * max(1.0, abs(e_want))
        else:
            assert err <= 1e-5, (n, err)
            assert abs(obs["norm"] - n_want) <= 1e-5
            assert abs(obs["energy"] - e_want) <= 1e-4 * max(1.0, abs(e_want))


def test_c3_full_size_first_steps(ses, oracle):
    w = scenes.config_c3(512)
    chk = Checker(oracle, ref_cls(), w)
    want = chk.step(5)
    p_want = chk.p_range(1.0, math.inf)
    chk.close()
    op = device_op(ses, w, "c64")
    op.advance(5, absorb=True)
    got = op.readback()
    obs = op.observe(1.0, math.inf)
    op.close()
    assert rel_l2(got, want) <= 1e-5
    assert abs(obs["p_range"] - p_want) <= 1e-6


@pytest.mark.parametrize("x0", [-20.0, -5.0])
def test_c3_strip_500_steps_transmitted_probability_every_50(ses, oracle, x0):
    w = scenes.config_c3_strip(x0)
    r = run_segments(ses, oracle, ref_cls(), w, "c64", w.steps, w.observe_every, (1.0, math.inf))
    assert len(r["series"]) == 10
    for row in r["series"]:
        assert abs(row["p_range"] - row["p_range_oracle"]) <= 1e-6 + 1e-5 * row["p_range_oracle"], row
        assert abs(row["norm"] - row["norm_oracle"]) <= 1e-5, row
    assert r["rel_l2"] <= 1e-5
    if x0 > -10.0:
        assert r["series"][-1]["p_range_oracle"] > 1e-3  # part of the packet crossed: the observable is exercised


@pytest.mark.parametrize("dims", [(48, 48, 48), (96, 96, 1), (64, 64, 64)])
def test_c4_sizes_1000_steps_both_precisions(ses, oracle, dims):
    n = dims[0]
    sp = next(s for s in scenes.config_c4_specs(256) if s["n"] == n)
    w = scenes.build_c4_instance(sp) if dims[2] > 1 else scenes.build_c4_plane(sp)
    chk = Checker(oracle, ref_cls(), w)
    want = chk.step(1000)
    n_want = chk.norm()
    chk.close()
    for prec, tol in (("c128", 1000 * 1e-12), ("c64", 1e-5)):
        op = device_op(ses, w, prec)
        op.advance(1000, absorb=True)
        got = op.readback()
        obs = op.observe()
        op.close()
        assert rel_l2(got, want) <= tol, (dims, prec, rel_l2(got, want))
        assert abs(obs["norm"] - n_want) <= (1e-11 if prec == "c128" else 1e-5), (dims, prec)
