"""Dipole-driven steps (ses_gpu_step_driven) against the FP64 oracle's restatement
of the reference ses::driven_step (core/src/drive.ixx:50-65), which is pinned bit
for bit to the reference library (tests/test_oracle_pins.py)."""

import numpy as np
import pytest


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.gpu
@pytest.mark.parametrize("dims,prec,tol", [((32, 32, 32), "c128", 1e-11), ((48, 32, 16), "c128", 1e-11),
                                           ((64, 64, 1), "c128", 1e-11), ((32, 32, 32), "c64", 1e-5)])
def test_driven_steps_match_oracle(ses, oracle, dims, prec, tol):
    box = (-8.0, 8.0, -7.0, 7.0, -6.0, 6.0) if dims[2] > 1 else (-8.0, 8.0, -7.0, 7.0, 0.0, 1.0)
    V = oracle.harmonic3d(box, dims, 0.8)
    psi = oracle.gaussian3d(box, dims, (1.0, -0.5, 0.0), (1.2, 1.0, 1.1 if dims[2] > 1 else 1.0),
                            (0.4, 0.0, 0.0))
    g = ses.Grid3D(*[ses.Grid1D(box[2 * a], box[2 * a + 1], dims[a]) for a in range(3)])
    op = ses.SplitOperator3D(g, V, 0.02, precision=prec, psi0=psi)
    drive = ses.DipoleDrive((0.6, 0.8, 0.0), 0.5, 1.3)
    f = ses.Field3D(g, psi)
    ses.driven_step(f, op, drive, 0.1, 12)
    want = oracle.driven_step3d(box, dims, V, 0.02, psi, 12, drive.axis, 0.5, 1.3, 0.1)
    assert rel(f.data, want) <= tol
    # the drive moves the packet: different from the undriven step
    plain = oracle.step3d(box, dims, V, 0.02, psi, 12)
    assert rel(want, plain) > 1e-3
    op.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["c64", "c128"])
def test_snapshot_restore_and_density_slices(ses, oracle, prec):
    """Checkpoint mid-run, continue, restore into a fresh handle, continue again:
    the same bits; density slices equal |psi|^2 of the read-back field."""
    box, dims = (-8.0, 8.0, -7.0, 7.0, -6.0, 6.0), (32, 16, 24)
    V = oracle.harmonic3d(box, dims, 0.8)
    psi = oracle.gaussian3d(box, dims, (1.0, -0.5, 0.5), (1.2, 1.0, 1.1), (0.4, 0.2, 0.0))
    g = ses.Grid3D(*[ses.Grid1D(box[2 * a], box[2 * a + 1], dims[a]) for a in range(3)])
    a = ses.SplitOperator3D(g, V, 0.02, precision=prec, psi0=psi)
    a.advance(10)
    snap = a.snapshot(steps=10)
    esize = 8 if prec == "c64" else 16
    assert len(snap) == 128 + g.size() * esize and snap[:7] == b"SESPSI1"
    a.advance(15)
    b = ses.SplitOperator3D(g, V, 0.02, precision=prec)
    assert b.restore(snap) == 10
    b.advance(15)
    assert np.array_equal(a.readback(), b.readback())
    field = a.readback().reshape(dims[2], dims[1], dims[0])
    dens = np.abs(field) ** 2
    assert np.allclose(a.density_slice(2, 5), dens[5], rtol=1e-6, atol=1e-12)
    assert np.allclose(a.density_slice(0, 7), dens[:, :, 7], rtol=1e-6, atol=1e-12)
    assert np.allclose(a.density_slice(1, 3), dens[:, 3, :], rtol=1e-6, atol=1e-12)
    other = ses.SplitOperator3D(ses.Grid3D(g.x, g.y, ses.Grid1D(-6.0, 6.0, 16)), np.zeros(32 * 16 * 16), 0.02,
                                precision=prec)
    with pytest.raises(ValueError):
        other.restore(snap)
    for op in (a, b, other):
        op.close()
