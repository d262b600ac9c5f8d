"""Batched propagation (ses_batch_*): many fields of mixed shapes advanced by one
launch per axis pass and shape class.

Every member must end where the same handle stepped alone ends: the batched
kernels run the same line-FFT bodies over per-instance arguments, so a member's
arithmetic does not depend on who else is in the batch.  They are separate
kernels from the single-handle ones, so the compiler may contract a different
multiply-add here and there: results agree to rounding (relative L2 below
TOL), not bit for bit.
"""

import math

import numpy as np
import pytest

from shoeridingerequationsolver_b200 import scenes

TOL = {"c128": 1e-14, "c64": 5e-7}


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def make_member(ses, shape, box, prec, seed, dt=0.01, absorber=True):
    rng = np.random.default_rng(seed)
    axes = [ses.Grid1D(-box[a], box[a], shape[a]) for a in range(3)]
    g = ses.Grid3D(*axes)
    V = scenes.harmonic(g, float(rng.uniform(0.5, 1.5)), tuple(rng.uniform(-0.5, 0.5, 3)))
    c = [float(rng.uniform(-0.3, 0.3)) * box[a] if shape[a] > 1 else 0.0 for a in range(3)]
    psi = scenes.gaussian(g, c, [max(0.12 * box[a], 0.3) for a in range(3)],
                          [float(rng.uniform(-1, 1)) if shape[a] > 1 else 0.0 for a in range(3)])
    op = ses.SplitOperator3D(g, V, dt, precision=prec)
    op.upload_state(psi)
    if absorber:
        op.set_absorber_separable(*scenes.mask_profiles(g, 0.1))
    return op, psi


SHAPES = [(16, 16, 16), (32, 32, 32), (48, 48, 48), (32, 16, 48), (96, 96, 1), (128, 1, 1),
          (64, 64, 64)]


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["c128", "c64"])
@pytest.mark.parametrize("nsteps", [1, 3, 11])
def test_batch_members_match_alone(ses, prec, nsteps):
    box = (8.0, 7.0, 6.0)
    members, alone = [], []
    for i, shape in enumerate(SHAPES + SHAPES[:3]):   # repeated shapes share a class
        op, psi = make_member(ses, shape, box, prec, seed=100 + i)
        ref, _ = make_member(ses, shape, box, prec, seed=100 + i)
        members.append(op)
        alone.append(ref)
    with ses.Batch(members) as b:
        assert b.counts() == (len(members), len(SHAPES))
        b.step(nsteps, absorb=True)
        b.sync()
        for op, ref, shape in zip(members, alone, SHAPES + SHAPES[:3]):
            ref.advance(nsteps, absorb=True)
            got, want = op.readback(), ref.readback()
            assert np.all(np.isfinite(got))
            assert rel(got, want) <= TOL[prec], shape
    for op in members + alone:
        op.close()


@pytest.mark.gpu
def test_batch_member_vs_oracle_mixed_radix(ses, oracle):
    """A 48^3 and a 96x96 member of a batch against the FP64 oracle step."""
    box = (6.0, 6.0, 6.0)
    ops = []
    for i, shape in enumerate([(48, 48, 48), (96, 96, 1)]):
        op, psi = make_member(ses, shape, box, "c128", seed=7 + i, absorber=False)
        rng = np.random.default_rng(7 + i)   # the potential make_member drew
        V = scenes.harmonic(op.grid, float(rng.uniform(0.5, 1.5)), tuple(rng.uniform(-0.5, 0.5, 3)))
        ops.append((op, psi, V))
    with ses.Batch([o for o, _, _ in ops]) as b:
        b.step(5)
        b.sync()
        for op, psi, V in ops:
            g = op.grid
            want = oracle.step3d(g.box, g.dims, V, 0.01, psi, 5)
            assert rel(op.readback(), want) <= 5e-12, g.dims
    for op, _, _ in ops:
        op.close()


@pytest.mark.gpu
def test_batch_membership_changes(ses):
    """Remove, re-add and destroy members between steps; the rest keep stepping
    exactly as alone; observe returns one record per member in add order."""
    box = (8.0, 8.0, 8.0)
    ops = [make_member(ses, s, box, "c64", seed=40 + i)[0] for i, s in enumerate(SHAPES[:4])]
    refs = [make_member(ses, s, box, "c64", seed=40 + i)[0] for i, s in enumerate(SHAPES[:4])]
    b = ses.Batch(ops)
    b.step(4, absorb=True)
    for r in refs:
        r.advance(4, absorb=True)
    b.remove(ops[1])
    with pytest.raises(Exception):
        b.remove(ops[1])                       # not a member any more
    ops[1].advance(2, absorb=True)             # steps alone on its own stream again
    refs[1].advance(2, absorb=True)
    ops[2].close()                             # destroying a member removes it first
    b.step(3, absorb=True)
    for i in (0, 3):
        refs[i].advance(3, absorb=True)
    obs = b.observe()
    assert len(obs) == 2
    for rec, i in zip(obs, (0, 3)):
        assert math.isclose(rec["norm"], refs[i].observe()["norm"], rel_tol=1e-6)
        assert rel(ops[i].readback(), refs[i].readback()) <= TOL["c64"]
    assert rel(ops[1].readback(), refs[1].readback()) <= TOL["c64"]
    b.add(ops[1])
    with pytest.raises(Exception):
        b.add(ops[1])                          # already a member
    b.close()
    for i in (0, 1, 3):
        ops[i].close()
    for r in refs:
        r.close()


@pytest.mark.gpu
def test_batch_profile_reports_every_class(ses):
    box = (8.0, 8.0, 8.0)
    ops = [make_member(ses, s, box, "c64", seed=60 + i)[0] for i, s in enumerate(SHAPES[:3])]
    with ses.Batch(ops) as b:
        prof = b.profile(4, absorb=True)
        assert len(prof) == 3
        for p in prof:
            assert p["step"] > 0 and p["x_mid"] > 0
        for op in ops:
            o = op.observe()
            assert 0.5 < o["norm"] <= 1.0 + 1e-6
    for op in ops:
        op.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["c64", "c128"])
def test_batch_run_equals_separate_calls(ses, prec):
    """ses_batch_run (uploads, steps, observables and readbacks queued per class
    stream) gives the bits of write_psi + ses_batch_step + observe + read_psi on
    twin members; members without an input keep their field, members without an
    output are not read back."""
    box = (8.0, 7.0, 6.0)
    shapes = [(64, 64, 64), (48, 48, 48), (96, 96, 1), (32, 16, 48), (64, 64, 64), (128, 1, 1)]
    run_ops, sep_ops, inputs = [], [], []
    for i, shape in enumerate(shapes):
        a, _ = make_member(ses, shape, box, prec, seed=300 + i)
        b, _ = make_member(ses, shape, box, prec, seed=300 + i)
        rng = np.random.default_rng(900 + i)
        g = a.grid
        c = [float(rng.uniform(-0.2, 0.2)) * box[k] if shape[k] > 1 else 0.0 for k in range(3)]
        psi = scenes.gaussian(g, c, [max(0.15 * box[k], 0.3) for k in range(3)],
                              [float(rng.uniform(-1, 1)) if shape[k] > 1 else 0.0 for k in range(3)])
        run_ops.append(a)
        sep_ops.append(b)
        inputs.append(None if i == 2 else np.ascontiguousarray(psi))
    # a 65536-point line: long lines step member by member on the batch stream
    g1 = ses.line_grid(ses.Grid1D(-200.0, 200.0, 65536))
    V1 = scenes.harmonic(g1, 0.05)
    p1 = scenes.gaussian(g1, (3.0, 0.0, 0.0), (1.0, 1.0, 1.0), (0.5, 0.0, 0.0))
    for ops in (run_ops, sep_ops):
        op = ses.SplitOperator3D(g1, V1, 0.005, precision=prec, psi0=p1)
        op.set_absorber_separable(scenes.mask_profiles(g1, 0.1)[0], np.ones(1), np.ones(1))
        ops.append(op)
    shapes.append((65536, 1, 1))
    inputs.append(np.ascontiguousarray(p1 * np.exp(0.3j)))
    outputs = [None if i == 3 else np.full(op.grid.size(), np.nan, complex) for i, op in enumerate(run_ops)]
    with ses.Batch(run_ops) as br, ses.Batch(sep_ops) as bs:
        obs_run = br.run(7, psi_in=inputs, psi_out=outputs, absorb=True, xlo=0.0, xhi=math.inf)
        for op, x in zip(sep_ops, inputs):
            if x is not None:
                op.upload_state(x)
        bs.step(7, absorb=True)
        obs_sep = bs.observe(0.0, math.inf)
        for i, (a, b) in enumerate(zip(run_ops, sep_ops)):
            want = b.readback()
            if outputs[i] is not None:
                assert np.array_equal(outputs[i], want), shapes[i]
            assert np.array_equal(a.readback(), want), shapes[i]
            assert obs_run[i] == obs_sep[i], shapes[i]
        # a second round trip on the same buffers: steps only, no observables
        assert br.run(3, psi_out=outputs, absorb=True, observe=False) is None
        bs.step(3, absorb=True)
        for i, b in enumerate(sep_ops):
            if outputs[i] is not None:
                assert np.array_equal(outputs[i], b.readback()), shapes[i]
        with pytest.raises(ValueError):
            br.run(1, psi_in=inputs[:2])
    for op in run_ops + sep_ops:
        op.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["c64", "c128"])
def test_programmatic_launch_changes_no_bits(ses, prec, monkeypatch):
    """Passes launched with programmatic dependent launch (the default) wait for the
    previous kernel before touching any field, so the results equal those of plain
    launches bit for bit -- single handles and batches."""
    box = (8.0, 7.0, 6.0)
    shapes = [(64, 64, 64), (48, 48, 48), (96, 96, 1), (16, 16, 16)]
    runs = {}
    for pdl in ("0", "1"):
        monkeypatch.setenv("SES_PDL", pdl)   # read when a handle is created
        single = [make_member(ses, s, box, prec, seed=500 + i)[0] for i, s in enumerate(shapes)]
        batched = [make_member(ses, s, box, prec, seed=500 + i)[0] for i, s in enumerate(shapes)]
        for op in single:
            op.advance(13, absorb=True)
        with ses.Batch(batched) as b:
            b.step(13, absorb=True)
            b.sync()
            runs[pdl] = ([op.readback() for op in single], [op.readback() for op in batched])
        for op in single + batched:
            op.close()
    for kind in (0, 1):
        for a, b, s in zip(runs["0"][kind], runs["1"][kind], shapes):
            assert np.array_equal(a, b), (kind, s)
