"""1D lines above 4096 points (the serving mix's 65536-point requests).

Such a line runs as N1 x N2 (65536 = 256 x 256) in four steps: a strided pass
does the length-N2 transforms with the twiddles W_N^{n1 k2}, a contiguous pass
the length-N1 transforms with the kinetic phase of frequency k2 + N2 k1 in
between; a step is two sweeps.  Checked against the FP64 oracle's 1D step
(the reference SplitOperator1D algorithm, core/src/propagator.ixx:21-66).
"""

import numpy as np
import pytest

N, LO, HI = 65536, -200.0, 200.0


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def line(ses, oracle, prec, pot="morse", mask=False, dt=0.005):
    g1 = ses.Grid1D(LO, HI, N)
    g = ses.line_grid(g1)
    if pot == "morse":
        V = oracle.morse1d(LO, HI, N, 4.0, 0.5, 0.0)
        x0 = 0.0
    else:
        V = oracle.double_well1d(LO, HI, N, 3.0, 3.0)
        x0 = 3.0
    psi = oracle.gaussian1d(LO, HI, N, x0, 1.0, 0.5)
    op = ses.SplitOperator3D(g, V, dt, precision=prec, psi0=psi)
    m = None
    if mask:
        m = oracle.mask1d(LO, HI, N, 40.0, 1)
        op.set_absorber_separable(m, np.ones(1), np.ones(1))
    return op, V, psi, m


@pytest.mark.gpu
@pytest.mark.parametrize("pot", ["morse", "double_well"])
def test_long_line_c128_matches_oracle(ses, oracle, pot):
    op, V, psi, m = line(ses, oracle, "c128", pot, mask=True)
    assert "four-step" in op.plan_info()
    op.advance(5, absorb=True)
    want = oracle.step1d(LO, HI, N, V, 0.005, psi, 5, m)
    assert rel(op.readback(), want) <= 5e-12
    op.close()


@pytest.mark.gpu
def test_long_line_c64_after_many_steps(ses, oracle):
    # double well: bounded enough on [-200, 200) for <V> to be well conditioned
    # (the Morse potential reaches 1e87 at the left wall)
    op, V, psi, m = line(ses, oracle, "c64", "double_well", mask=True)
    op.advance(400, absorb=True)
    want = oracle.step1d(LO, HI, N, V, 0.005, psi, 400, m)
    got = op.readback()
    assert rel(got, want) <= 1e-5
    o = op.observe()
    # FP32 rounding in a packet that occupies a few hundred grid points (and a few
    # dozen wavenumbers) moves the norm by a few 1e-9 per step
    assert abs(o["norm"] - oracle.norm1d(LO, HI, N, want)) <= 1e-5
    # <V> weighs the FP32 rounding floor (|psi|^2 ~ 1e-15 everywhere) with V ~ 6e7 at
    # the walls: a few 1e-5 of the energy, which the complex64 storage cannot remove
    assert abs(o["energy"] - oracle.mean_energy1d(LO, HI, N, want, V)) <= 1e-4 * max(1.0, abs(o["energy"]))
    op.close()


@pytest.mark.gpu
def test_long_line_observables_and_tables(ses, oracle):
    op, V, psi, _ = line(ses, oracle, "c128", "double_well")
    o = op.observe()
    assert abs(o["norm"] - oracle.norm1d(LO, HI, N, psi)) <= 1e-12
    assert abs(o["energy"] - oracle.mean_energy1d(LO, HI, N, psi, V)) <= 1e-10 * max(1.0, abs(o["energy"]))
    hv, kin = op.half_potential_phase(), op.kinetic_phase()
    k = 2 * np.pi / (HI - LO) * np.fft.fftfreq(N, 1.0 / N)
    assert np.max(np.abs(kin - np.exp(-0.5j * k * k * 0.005))) < 1e-13
    assert np.max(np.abs(hv - np.exp(-0.5j * V * 0.005))) < 1e-13
    # the natural-order transform of the resident line (four-step passes plus a transpose)
    op.fft3()
    assert np.linalg.norm(op.readback() - oracle.fft1d(psi)) / np.linalg.norm(oracle.fft1d(psi)) < 1e-14 * 16
    op.fft3(inverse=True)
    assert np.linalg.norm(op.readback() - psi) / np.linalg.norm(psi) < 1e-14 * 16
    op.close()


@pytest.mark.gpu
def test_long_lines_in_a_batch_match_alone(ses, oracle):
    """Long lines form their own batch class (one launch per four-step pass for all
    of them); each member ends exactly where it ends stepped alone."""
    members, alone = [], []
    for pot in ("morse", "double_well", "morse"):
        a, V, psi, m = line(ses, oracle, "c64", pot, mask=True)
        b, _, _, _ = line(ses, oracle, "c64", pot, mask=True)
        members.append(a)
        alone.append(b)
    with ses.Batch(members) as bt:
        assert bt.counts() == (3, 1)
        bt.step(23, absorb=True)
        bt.sync()
        for a, b in zip(members, alone):
            b.advance(23, absorb=True)
            assert np.array_equal(a.readback(), b.readback())
    for op in members + alone:
        op.close()
