"""Two-sweep 3D step (x-y plane pass + z pass) against the four-pass step and the oracle.

Grids with a plane pass (32^2 .. 128^2; one CTA per plane, or a cluster of 2
or 4 CTAs that split the plane's rows and columns and transpose through
distributed shared memory) run each step as one plane pass -- inverse y,
inverse x, potential (and absorber), forward x, forward y, per z-plane -- and
the z pass.  The plane pass runs the axis passes' plans, radix orders and diagonal
arithmetic in differently structured kernels, where the compiler's FMA
contraction may round the last bit differently: the two forms must agree to
1e-14 (complex128) / 2e-7 (complex64) relative L2 after first, interior (graph
body of 8 steps) and last steps, with a separable absorber, a full-array
absorber and none; each form matches the FP64 oracle; within the plane form a
run split into two calls gives the bits of one call.  SES_PLANE (read when a
handle is created) selects the form: 0 the four axis passes, k the plane pass
of k CTAs per plane.
"""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_C128_STEP = 1e-12
TOL_C64 = 1e-5
TOL_FORMS = {"c128": 1e-14, "c64": 2e-7}


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _grid(ses, box, n):
    return ses.Grid3D(*(ses.Grid1D(box[2 * a], box[2 * a + 1], n[a]) for a in range(3)))


def _scene(oracle, n):
    box = (-8.0, 8.0, -8.0, 8.0, -6.0, 6.0)
    V = oracle.harmonic3d(box, n, 0.8, (0.5, -0.25, 0.0))
    psi0 = oracle.gaussian3d(box, n, (1.0, -0.5, 0.3), (1.1, 1.0, 0.9), (0.7, -0.4, 0.3))
    return box, V, psi0


def _run(ses, box, n, V, psi0, prec, steps, plane, mask=None, sep=None):
    """plane: CTAs per plane of the plane pass (0: the four axis passes)."""
    old = os.environ.get("SES_PLANE")
    os.environ["SES_PLANE"] = str(int(plane))
    try:
        op = ses.SplitOperator3D(_grid(ses, box, n), V, 0.01, precision=prec)
    finally:
        if old is None:
            del os.environ["SES_PLANE"]
        else:
            os.environ["SES_PLANE"] = old
    info = op.plan_info()
    if sep is not None:
        op.set_absorber_separable(*sep)
    elif mask is not None:
        op.set_absorber(mask)
    op.upload_state(psi0)
    op.advance(steps, absorb=(mask is not None or sep is not None))
    out = op.readback()
    op.close()
    return out, info


CASES = [((32, 32, 16), "c128", 1), ((32, 32, 16), "c128", 2), ((32, 32, 16), "c64", 1), ((32, 32, 16), "c64", 2),
         ((48, 48, 12), "c128", 1), ((48, 48, 12), "c128", 2), ((48, 48, 12), "c64", 1), ((48, 48, 12), "c64", 2),
         ((64, 64, 64), "c128", 1), ((64, 64, 64), "c128", 2), ((64, 64, 64), "c128", 4),
         ((64, 64, 20), "c64", 1), ((64, 64, 20), "c64", 2), ((64, 64, 20), "c64", 4),
         ((96, 96, 8), "c64", 1), ((96, 96, 8), "c64", 2), ((96, 96, 8), "c64", 4), ((128, 128, 6), "c64", 1)]


@pytest.mark.parametrize("n,prec,cs", CASES, ids=[f"{c[0][0]}x{c[0][1]}x{c[0][2]}-{c[1]}-cs{c[2]}" for c in CASES])
def test_plane_step_matches_four_pass_step_and_oracle(ses, oracle, n, prec, cs):
    box, V, psi0 = _scene(oracle, n)
    for steps in (1, 11):  # one step (start + end), and start + 8-step graph body + 1 + end
        a, ia = _run(ses, box, n, V, psi0, prec, steps, plane=0)
        b, ib = _run(ses, box, n, V, psi0, prec, steps, plane=cs)
        assert f"plane pass on {cs} CTA" in ib and "four axis passes" in ia, (ia, ib)
        assert _rel(b, a) < TOL_FORMS[prec], (steps, _rel(b, a))
        ref = oracle.step3d(box, n, V, 0.01, psi0, steps)
        assert _rel(b, ref) < (steps * TOL_C128_STEP if prec == "c128" else TOL_C64), (steps, _rel(b, ref))


@pytest.mark.parametrize("prec,cs", [("c128", 1), ("c128", 2), ("c64", 1), ("c64", 4)])
def test_plane_step_with_absorbers_matches_four_pass_step_and_oracle(ses, oracle, prec, cs):
    n = (64, 64, 16)
    box, V, psi0 = _scene(oracle, n)
    mx, my, mz = (oracle.mask1d(box[2 * a], box[2 * a + 1], n[a], 1.5) for a in range(3))
    full = (mx[None, None, :] * my[None, :, None] * mz[:, None, None]).reshape(-1)
    steps = 10
    ref = oracle.step3d(box, n, V, 0.01, psi0, steps, mask=full)
    tol = steps * TOL_C128_STEP if prec == "c128" else TOL_C64
    a, _ = _run(ses, box, n, V, psi0, prec, steps, plane=0, sep=(mx, my, mz))
    b, _ = _run(ses, box, n, V, psi0, prec, steps, plane=cs, sep=(mx, my, mz))
    assert _rel(b, a) < TOL_FORMS[prec]
    assert _rel(b, ref) < tol
    rng = np.random.default_rng(5)  # non-separable: the full-array path
    full2 = full * (1.0 - 0.01 * rng.random(full.size))
    ref2 = oracle.step3d(box, n, V, 0.01, psi0, steps, mask=full2)
    a2, _ = _run(ses, box, n, V, psi0, prec, steps, plane=0, mask=full2)
    b2, _ = _run(ses, box, n, V, psi0, prec, steps, plane=cs, mask=full2)
    assert _rel(b2, a2) < TOL_FORMS[prec]
    assert _rel(b2, ref2) < tol


@pytest.mark.parametrize("cs", [1, 2, 4])
def test_plane_step_c1_against_oracle_and_split_runs(ses, oracle, cs):
    """64^3 complex128 (the C1 grid) in the two-sweep form: 40 steps against the
    oracle, and 17 + 23 steps in two calls give the bits of one 40-step call."""
    n = (64, 64, 64)
    box = (-10.0, 10.0) * 3
    V = oracle.harmonic3d(box, n, 1.0)
    psi0 = oracle.gaussian3d(box, n, (2.0, 0.0, 0.0), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0))
    ref = oracle.step3d(box, n, V, 0.005, psi0, 40)
    os.environ["SES_PLANE"] = str(cs)
    try:
        op = ses.SplitOperator3D(_grid(ses, box, n), V, 0.005, precision="c128")
        op2 = ses.SplitOperator3D(_grid(ses, box, n), V, 0.005, precision="c128")
    finally:
        del os.environ["SES_PLANE"]
    assert f"plane pass on {cs} CTA" in op.plan_info()
    op.upload_state(psi0)
    op.advance(40)
    one = op.readback()
    op2.upload_state(psi0)
    op2.advance(17)
    op2.advance(23)
    two = op2.readback()
    op.close()
    op2.close()
    assert np.linalg.norm(one - ref) / np.linalg.norm(ref) < 40 * TOL_C128_STEP
    assert np.array_equal(one, two)


def test_default_and_autotuned_step_form(ses, oracle):
    """Without SES_PLANE a 64^3 grid takes its default plane pass; autotune times
    the four-pass form and every plane variant and keeps one, reported by plan_info."""
    n = (64, 64, 64)
    box, V, psi0 = _scene(oracle, n)
    os.environ.pop("SES_PLANE", None)
    op = ses.SplitOperator3D(_grid(ses, box, n), V, 0.01, precision="c128", psi0=psi0)
    assert "plane pass on" in op.plan_info()
    info = op.autotune(save=False)
    assert "step: " in info
    op.advance(9)
    got = op.readback()
    op.close()
    ref = oracle.step3d(box, n, V, 0.01, psi0, 9)
    assert _rel(got, ref) < 9 * TOL_C128_STEP


@pytest.mark.parametrize("prec", ["c64", "c128"])
def test_batched_plane_step_matches_four_pass_batch_and_oracle(ses, oracle, monkeypatch, prec):
    """A batch of several shapes with separable absorbers (two members of one shape):
    the classes in the two-sweep form (SES_BATCH_PLANE=1, read when the batch's
    classes are built) against the same batch in four passes and the oracle."""
    shapes = [(32, 32, 16), (48, 48, 12), (64, 64, 20), (64, 64, 20), (96, 96, 8), (128, 128, 6)]
    if prec == "c128":  # complex128 plane passes: 32^2 .. 64^2
        shapes = [(32, 32, 16), (48, 48, 12), (64, 64, 20), (64, 64, 20)]
    outs = {}
    for form in ("0", "1"):
        monkeypatch.setenv("SES_BATCH_PLANE", form)
        ops, refs = [], []
        for i, n in enumerate(shapes):
            box, V, psi0 = _scene(oracle, n)
            psi0 = psi0 * np.exp(0.1j * i)
            mx, my, mz = (oracle.mask1d(box[2 * a], box[2 * a + 1], n[a], 1.5) for a in range(3))
            op = ses.SplitOperator3D(_grid(ses, box, n), V, 0.01, precision=prec, psi0=psi0)
            op.set_absorber_separable(mx, my, mz)
            ops.append(op)
            refs.append((box, n, V, psi0, (mx[None, None, :] * my[None, :, None] * mz[:, None, None]).reshape(-1)))
        with ses.Batch(ops) as b:
            info = b.info()
            b.step(11, absorb=True)
            b.sync()
            outs[form] = [op.readback() for op in ops]
        for op in ops:
            op.close()
        assert ("plane" in info) == (form == "1"), info
    for i, (box, n, V, psi0, full) in enumerate(refs):
        assert _rel(outs["1"][i], outs["0"][i]) < TOL_FORMS[prec], (n, _rel(outs["1"][i], outs["0"][i]))
        ref = oracle.step3d(box, n, V, 0.01, psi0, 11, mask=full)
        tol = 11 * TOL_C128_STEP if prec == "c128" else TOL_C64
        assert _rel(outs["1"][i], ref) < tol, (n, _rel(outs["1"][i], ref))
