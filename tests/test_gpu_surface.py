"""The rest of the reference's call surface on the device, against the FP64 oracle:

* fft(std::vector<cd>&) / ifft for power-of-two lines above 4096 points
  (core/src/fft.ixx:75-98) -- four-step layout plus a transpose;
* Engine::norm_and_peak and Engine::scale (solver/src/vk_engine.ixx:1665-1692,
  2120-2133), the directors' drift renormalisation
  (scenario/src/base_director.ixx:340-352);
* WavepacketSimulation (core/src/simulation.ixx:22-88) with the reference's
  own test cases (tests/simulation_test.cpp: time, norm, MatchesManualPropagation,
  density).
"""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("n", [8192, 65536, 1 << 18])
def test_long_line_fft_natural_order(ses, oracle, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    for inverse in (False, True):
        want = oracle.fft1d(a, inverse=inverse)
        got = (ses.ifft if inverse else ses.fft)(a, precision="c128")
        assert rel_l2(got, want) < 1e-14 * math.log2(n), (n, inverse)
        got32 = (ses.ifft if inverse else ses.fft)(a, precision="c64")
        assert rel_l2(got32, want) < 1e-6, (n, inverse)
    # round trip and a plane-wave spike in the bin it names
    assert np.allclose(ses.ifft(ses.fft(a)), a, atol=1e-12)
    k0 = 12345 % n
    spike = ses.fft(np.exp(2j * np.pi * k0 * np.arange(n) / n))
    assert abs(spike[k0] - n) < 1e-8 * n
    assert np.max(np.abs(np.delete(spike, k0))) < 1e-8 * n


def test_long_line_fft_field1d_in_place(ses, oracle):
    g = ses.Grid1D(-200.0, 200.0, 65536)
    x = g.coords()
    f = ses.Field1D(g, np.exp(-x * x / 8.0) * np.exp(0.5j * x))
    want = oracle.fft1d(f.data)
    ses.fft(f)
    assert rel_l2(f.data, want) < 1e-13


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_norm_and_peak_and_scale(ses, oracle, prec):
    box, n = (-8.0, 8.0) * 3, (32, 48, 20)
    g = ses.Grid3D(*(ses.Grid1D(box[2 * a], box[2 * a + 1], n[a]) for a in range(3)))
    V = oracle.harmonic3d(box, n, 1.0)
    psi0 = oracle.gaussian3d(box, n, (1.0, -0.5, 0.0), (1.0, 1.5, 1.2), (0.5, 0.0, 0.3))
    op = ses.SplitOperator3D(g, V, 0.01, precision=prec, psi0=psi0)
    op.advance(7)
    psi = op.readback()
    nrm, peak = op.norm_and_peak()
    tol = 1e-13 if prec == "c128" else 1e-6
    assert abs(nrm - oracle.norm3d(box, n, psi)) <= tol
    assert abs(peak - float(np.max(np.abs(psi) ** 2))) <= tol * peak
    # the directors' drift renormalisation: scale by 1/sqrt(norm)
    op.scale(3.0)
    n3, p3 = op.norm_and_peak()
    assert abs(n3 - 9.0 * nrm) <= 9 * tol and abs(p3 - 9.0 * peak) <= 9 * tol * peak
    op.scale(1.0 / math.sqrt(n3))
    assert abs(op.norm_and_peak()[0] - 1.0) <= tol
    # deterministic: the same field gives the same bits
    assert op.norm_and_peak() == op.norm_and_peak()
    op.close()


def simulation_config(ses, oracle):
    box, n = (-8.0, 8.0) * 3, (16, 16, 16)
    g = ses.Grid3D(*(ses.Grid1D(-8.0, 8.0, 16) for _ in range(3)))
    return box, n, ses.WavepacketSimulation.Config(g, oracle.harmonic3d(box, n, 1.0), (2.0, 0.0, 0.0),
                                                   (1.0, 1.0, 1.0), (0.0, 0.5, 0.0), 0.02)


def test_wavepacket_simulation_matches_manual_propagation(ses, oracle):
    box, n, cfg = simulation_config(ses, oracle)
    sim = ses.WavepacketSimulation(cfg)
    assert sim.time() == 0.0
    manual = oracle.gaussian3d(box, n, cfg.r0, cfg.sigma, cfg.k0)
    assert np.max(np.abs(sim.psi().data - manual)) < 1e-15  # host builder == the reference builder
    sim.advance(3)
    sim.advance(2)
    assert sim.time() == pytest.approx(5 * 0.02, abs=1e-15)
    want = oracle.step3d(box, n, cfg.potential, cfg.dt, manual, 5)
    got = sim.psi().data
    # simulation_test.cpp MatchesManualPropagation: < 1e-14 between two CPU runs of the
    # same code; device vs oracle differ by FFT summation order
    assert max(np.max(np.abs(got.real - want.real)), np.max(np.abs(got.imag - want.imag))) < 1e-13
    assert np.array_equal(sim.density(), got.real * got.real + got.imag * got.imag)  # probability_density
    sim.close()


def test_wavepacket_simulation_norm_set_psi_and_relax(ses, oracle):
    box, n, cfg = simulation_config(ses, oracle)
    sim = ses.WavepacketSimulation(cfg)
    sim.advance(50)
    assert abs(oracle.norm3d(box, n, sim.psi().data) - 1.0) < 1e-12  # ConservesNormWhileAdvancing
    other = oracle.gaussian3d(box, n, (-1.0, 1.0, 0.0), (1.3, 1.0, 0.8), (0.2, 0.0, 0.0))
    sim.set_psi(ses.Field3D(cfg.grid, other))
    assert np.array_equal(sim.psi().data, other)
    sim.advance(4)
    want = oracle.step3d(box, n, cfg.potential, cfg.dt, other, 4)
    assert rel_l2(sim.psi().data, want) < 1e-12
    sim.relax(200, 0.01)
    assert abs(oracle.norm3d(box, n, sim.psi().data) - 1.0) < 1e-12
    # the oracle's 200 imaginary-time steps (renormalised every step) from the same field
    ref = oracle.relax3d(box, n, cfg.potential, 0.01, want, 200)
    assert rel_l2(sim.psi().data, ref) < 1e-10
    sim.close()
