"""Pipelined (TMA-fed, persistent) passes vs the register-path passes and the
oracle.  Both paths run the same FFT arithmetic; the FP64 diagonal multiplies
are compiled in differently structured code, so the compiler's FMA
contraction choices may differ in the last bit: the complex128 results must
agree to 1e-14 relative L2, the complex64 results (rounded to FP32 after the
FP64 diagonal math) to 2e-7.  SES_PIPELINED=0 at handle creation selects the
register path."""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# shapes chosen so each pipelined kernel runs: x (contiguous), y (3D TMA map),
# z (2D TMA map), and 512-long strided lines (two 256-row TMA boxes per tile)
SHAPES = [(64, 64, 64), (256, 256, 4), (8, 8, 256), (512, 16, 4), (4, 8, 512), (512, 512, 2),
          (256, 32, 256)]


def make(ses, dims, prec, pipelined, box, V, mask):
    os.environ["SES_PIPELINED"] = "1" if pipelined else "0"
    try:
        g = ses.Grid3D(*(ses.Grid1D(box[2 * a], box[2 * a + 1], dims[a]) for a in range(3)))
        op = ses.SplitOperator3D(g, V, 0.01, precision=prec)
    finally:
        os.environ.pop("SES_PIPELINED", None)
    op.set_absorber(mask)
    return op


@pytest.mark.parametrize("dims", SHAPES, ids=["x".join(map(str, d)) for d in SHAPES])
@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_pipelined_bitwise_equals_register_path(ses, oracle, dims, prec):
    box = (-12.0, 12.0, -10.0, 10.0, -8.0, 8.0)
    V = oracle.harmonic3d(box, dims, 0.7, (0.3, -0.2, 0.1))
    psi0 = oracle.gaussian3d(box, dims, (1.0, 0.5, -0.5), (1.5, 1.2, 1.1), (0.7, -0.4, 0.3))
    mask = oracle.mask3d(box, dims, 2.0, 1)
    outs = []
    for pipelined in (True, False):
        op = make(ses, dims, prec, pipelined, box, V, mask)
        op.upload_state(psi0)
        op.advance(11, absorb=True)
        outs.append(op.readback())
        o = op.observe()
        outs.append(np.array([o["norm"], o["energy"]]))
        op.close()
    tol = 1e-14 if prec == "c128" else 2e-7
    assert np.linalg.norm(outs[0] - outs[2]) / np.linalg.norm(outs[2]) < tol
    assert np.max(np.abs(outs[1] - outs[3]) / np.abs(outs[3])) < tol


@pytest.mark.parametrize("dims", [(256, 256, 4), (8, 8, 256), (4, 8, 512)])
def test_pipelined_matches_oracle(ses, oracle, dims):
    box = (-12.0, 12.0, -10.0, 10.0, -8.0, 8.0)
    V = oracle.harmonic3d(box, dims, 0.7)
    psi0 = oracle.gaussian3d(box, dims, (1.0, 0.5, -0.5), (1.5, 1.2, 1.1), (0.7, -0.4, 0.3))
    mask = oracle.mask3d(box, dims, 2.0, 1)
    ref = oracle.step3d(box, dims, V, 0.01, psi0, 3, mask=mask)
    for prec, tol in (("c128", 3e-12), ("c64", 1e-5)):
        op = make(ses, dims, prec, True, box, V, mask)
        op.upload_state(psi0)
        op.advance(3, absorb=True)
        out = op.readback()
        op.close()
        assert np.linalg.norm(out - ref) / np.linalg.norm(ref) < tol


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_autotune_keeps_results(ses, oracle, prec, tmp_path, monkeypatch):
    monkeypatch.setenv("SES_TUNE_CACHE", str(tmp_path / "tune.txt"))
    dims, box = (64, 64, 64), (-10.0, 10.0) * 3
    V = oracle.harmonic3d(box, dims, 1.0)
    psi0 = oracle.gaussian3d(box, dims, (2.0, 0.0, 0.0), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0))
    g = ses.Grid3D(*(ses.Grid1D(box[2 * a], box[2 * a + 1], dims[a]) for a in range(3)))
    op = ses.SplitOperator3D(g, V, 0.005, precision=prec)
    op.upload_state(psi0)
    info = op.autotune(save=True)
    assert info.startswith("x:64") and "z:64" in info
    assert (tmp_path / "tune.txt").read_text().count(":64:") >= 3
    op.advance(6)
    out = op.readback()
    op.close()
    ref = oracle.step3d(box, dims, V, 0.005, psi0, 6)
    tol = 6e-12 if prec == "c128" else 1e-5
    assert np.linalg.norm(out - ref) / np.linalg.norm(ref) < tol
    # a new handle of the same shape picks up the cached choice
    op2 = ses.SplitOperator3D(g, V, 0.005, precision=prec)
    assert op2.plan_info() == info
    op2.close()
