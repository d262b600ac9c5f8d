"""Pin the oracle (oracle/ses_oracle.c) before trusting it.

1. Against golden vectors produced by the reference's own core
   (tests/golden/reference_core.npz, made by tests/golden/make_golden.py):
   power-of-two paths must match BIT FOR BIT (same steps, same rounding).
2. Against the reference's own known-answer tests, restated (tests/fft_test.cpp,
   fft3_test.cpp, spectral_test.cpp, potential_test.cpp, field3_test.cpp,
   propagator_test.cpp, harmonic_dynamics_test.cpp).
3. The mixed-radix extension (lengths with factors 3 and 5, which the
   reference rejects) against an O(n^2) long-double DFT.
4. Live against the reference library when it was built here.
"""

import math
from pathlib import Path

import numpy as np
import pytest

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "reference_core.npz")


def same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b))


# ------------------------------------------------------------ golden vectors (bitwise)

@pytest.mark.parametrize("n", [1, 8, 16, 1024])
def test_fft1d_golden_bitwise(oracle, n):
    s = GOLD[f"fft1d_{n}_in"]
    assert same(oracle.fft1d(s), GOLD[f"fft1d_{n}_out"])
    assert same(oracle.fft1d(s, inverse=True), GOLD[f"ifft1d_{n}_out"])


def test_fft3d_golden_bitwise(oracle):
    assert same(oracle.fft3d(GOLD["fft3d_8x16x4_planewave_in"], (8, 16, 4)),
                GOLD["fft3d_8x16x4_planewave_out"])
    assert same(oracle.fft3d(GOLD["fft3d_8x4x2_in"], (8, 4, 2)), GOLD["fft3d_8x4x2_out"])
    assert same(oracle.fft3d(GOLD["fft3d_8x4x2_in"], (8, 4, 2), inverse=True),
                GOLD["ifft3d_8x4x2_out"])


def test_tables_golden_bitwise(oracle):
    box, n = (0.0, 4.0, 0.0, 4.0, 0.0, 4.0), (4, 4, 4)
    V = oracle.harmonic3d(box, n, 2.0, (1.0, 2.0, 3.0))
    assert same(V, GOLD["tables_cube4_V"])
    for m in (1.0, 2.0):
        h, k = oracle.tables3d(box, n, V, 0.1, m)
        assert same(h, GOLD[f"tables_cube4_m{m:g}_half"])
        assert same(k, GOLD[f"tables_cube4_m{m:g}_kin"])


def test_step_golden_bitwise(oracle):
    box8, n8 = (-4.0, 4.0) * 3, (8, 8, 8)
    V = oracle.soft_coulomb3d(box8, n8, 1.0, 1.0)
    p0 = oracle.gaussian3d(box8, n8, (1.0, 0.0, 0.0), (1.2, 1.2, 1.2), (0.0, 0.5, 0.0))
    assert same(V, GOLD["step_8cube_V"]) and same(p0, GOLD["step_8cube_psi0"])
    assert same(oracle.step3d(box8, n8, V, 0.02, p0, 20), GOLD["step_8cube_psi20"])
    m = oracle.mask3d(box8, n8, 2.0, 0)
    assert same(m, GOLD["absorb_8cube_mask"])
    assert same(oracle.step3d(box8, n8, V, 0.02, p0, 5, mask=m), GOLD["absorb_8cube_psi5"])
    box16, n16 = (-8.0, 8.0) * 3, (16, 16, 16)
    V16 = oracle.harmonic3d(box16, n16, 1.0)
    p16 = oracle.gaussian3d(box16, n16, (2.0, 0.0, 0.0), (1.0, 1.0, 1.0), (0.0, 0.5, 0.0))
    assert same(V16, GOLD["step_16cube_V"]) and same(p16, GOLD["step_16cube_psi0"])
    out = oracle.step3d(box16, n16, V16, 0.02, p16, 5)
    assert same(out, GOLD["step_16cube_psi5"])
    assert oracle.norm3d(box16, n16, out) == GOLD["step_16cube_norm5"][0]
    assert oracle.mean_energy3d(box16, n16, out, V16) == GOLD["step_16cube_energy5"][0]


def test_line_and_relax_golden_bitwise(oracle):
    p0 = oracle.gaussian1d(-40.0, 40.0, 1024, -15.0, 1.0, 2.0)
    assert same(p0, GOLD["line_1024_psi0"])
    assert same(oracle.step1d(-40.0, 40.0, 1024, np.zeros(1024), 0.05, p0, 200),
                GOLD["line_1024_psi200"])
    box, n = (-4.0, 4.0) * 3, (16, 16, 16)
    V = oracle.harmonic3d(box, n, 2.0)
    p = oracle.gaussian3d(box, n, (0.5, -0.5, 0.3), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0))
    assert same(V, GOLD["relax_16cube_V"]) and same(p, GOLD["relax_16cube_psi0"])
    assert same(oracle.relax3d(box, n, V, 0.01, p, 50), GOLD["relax_16cube_psi50"])


def test_dipole_drive_golden_bitwise(oracle):
    box, n = (-6.0, 6.0, -5.0, 5.0, -4.0, 4.0), (16, 8, 8)
    V = oracle.harmonic3d(box, n, 1.0)
    p = oracle.gaussian3d(box, n, (0.5, 0.0, 0.0), (1.0, 1.0, 1.0), (0.3, 0.0, 0.0))
    got = oracle.driven_step3d(box, n, V, 0.05, p, 7, (0.6, 0.0, 0.8), 0.3, 1.1, 0.2)
    assert same(got, GOLD["drive_16x8x8_psi7"])


def test_builders_golden_bitwise(oracle):
    box16, n16 = (-8.0, 8.0) * 3, (16, 16, 16)
    assert same(oracle.regularized_coulomb3d(box16, n16, 1.0), GOLD["coulomb_16cube_h1"])
    assert same(oracle.barrier3d(box16, n16, 0.25, 0.0, 3.0), GOLD["barrier_16cube"])
    assert same(oracle.mask3d(box16, n16, 3.0, 0), GOLD["mask_16cube_w3"])
    assert same(oracle.mask1d(-8.0, 8.0, 16, 3.0, 0), GOLD["mask1d_16_w3"])
    assert same(oracle.double_well1d(-8.0, 8.0, 16, 0.1, 4.0), GOLD["double_well_16"])
    assert same(oracle.poschl_teller1d(-8.0, 8.0, 16, 0.375, 2.0), GOLD["poschl_teller_16"])
    assert same(oracle.morse1d(-8.0, 8.0, 16, 0.3, 0.5, -2.0), GOLD["morse_16"])
    assert same(oracle.wavenumbers(0.0, 8.0, 8), GOLD["wavenumbers_8"])


# ------------------------------------------------------------ reference known answers

def test_fft_known_answers(oracle):
    tol = 1e-12
    assert np.allclose(oracle.fft1d(np.array([3 - 4j])), [3 - 4j], atol=tol)
    assert np.allclose(oracle.fft1d(np.ones(8, complex)), [8] + [0] * 7, atol=tol)
    d = np.zeros(8, complex)
    d[0] = 1
    assert np.allclose(oracle.fft1d(d), np.ones(8), atol=tol)
    x = np.exp(2j * np.pi * 3 * np.arange(16) / 16)
    X = oracle.fft1d(x)
    assert abs(X[3] - 16) < tol and np.max(np.abs(np.delete(X, 3))) < tol
    c = oracle.fft1d(np.cos(2 * np.pi * 3 * np.arange(16) / 16).astype(complex))
    assert abs(c[3] - 8) < tol and abs(c[13] - 8) < tol
    s = GOLD["fft1d_16_in"]
    assert np.allclose(oracle.fft1d(oracle.fft1d(s), inverse=True), s, atol=tol)
    y = 0.5 * np.arange(8) - 1j
    s8 = GOLD["fft1d_8_in"]
    assert np.allclose(oracle.fft1d(2 * s8 + y), 2 * oracle.fft1d(s8) + oracle.fft1d(y), atol=tol)
    assert abs(np.sum(np.abs(s) ** 2) - np.sum(np.abs(oracle.fft1d(s)) ** 2) / 16) < 1e-10


def test_fft3_plane_wave_spike(oracle):
    out = GOLD["fft3d_8x16x4_planewave_out"]
    expect = np.zeros_like(out)
    expect[3 + 8 * (5 + 16 * 1)] = 512
    assert np.max(np.abs(out - expect)) < 1e-9
    assert np.max(np.abs(oracle.fft3d(GOLD["fft3d_8x16x4_planewave_in"], (8, 16, 4)) - expect)) < 1e-9


def test_wavenumbers_fftfreq(oracle):
    dk = 2 * math.pi / 8
    assert list(oracle.wavenumbers(0, 8, 8)) == [0, dk, 2 * dk, 3 * dk, -4 * dk, -3 * dk, -2 * dk, -dk]
    assert list(oracle.wavenumbers(-1, 1, 1)) == [0.0]


def test_mask_and_coulomb_known_values(oracle):
    ax = (-8.0, 8.0)
    box, n = ax * 3, (16, 16, 16)
    m = oracle.mask3d(box, n, 3.0, 0)
    flat = lambda i, j, k: i + 16 * (j + 16 * k)
    assert m[flat(8, 8, 8)] == 1.0
    assert abs(m[flat(0, 0, 0)]) < 1e-12
    s = math.sin(0.5 * 3.14159265358979323846 / 3.0)
    assert abs(m[flat(1, 8, 8)] - s * s) < 1e-12
    v = oracle.regularized_coulomb3d(box, n, 1.0)
    assert v[flat(8, 8, 8)] == -2.3800774
    assert v[flat(9, 8, 8)] == -1.0
    assert v[flat(9, 9, 9)] == -1.0 / math.sqrt(3.0)
    # collapsed axis has no walls
    assert list(oracle.mask1d(-1, 1, 1, 3.0, 0)) == [1.0]


def test_cos8_mask_profile(oracle):
    # m(d) = cos(pi/2 (1 - d/w))^(1/8) inside the layer, 1 beyond, 0 on the wall
    m = oracle.mask1d(-10.0, 10.0, 80, 2.0, 1)
    x = -10.0 + np.arange(80) * 0.25
    d = np.minimum(x + 10.0, 10.0 - x)
    expect = np.where(d >= 2.0, 1.0, np.cos(0.5 * np.pi * (1 - np.minimum(d, 2.0) / 2.0)) ** 0.125)
    assert m[0] == 0.0
    assert np.allclose(m[1:], expect[1:], rtol=1e-14, atol=1e-15)


def test_norm_includes_cell_volume(oracle):
    box, n = (0.0, 8.0, 0.0, 4.0, -1.0, 1.0), (16, 8, 4)
    assert oracle.norm3d(box, n, np.ones(512, complex)) == 64.0


def test_oracle_propagator_physics(oracle):
    # propagator_test.cpp:27-77 on the oracle
    p = GOLD["line_1024_psi200"]
    box = (-40.0, 40.0, 0, 1, 0, 1)
    assert abs(oracle.norm1d(-40.0, 40.0, 1024, p) - 1.0) < 1e-12
    assert abs(oracle.mean_position3d(box, (1024, 1, 1), p)[0] - 5.0) < 1e-6
    assert abs(oracle.sigma_position3d(box, (1024, 1, 1), p)[0] - math.sqrt(1 + 25)) < 1e-6
    assert abs(oracle.mean_momentum3d(box, (1024, 1, 1), p)[0] - 2.0) < 1e-8


# ------------------------------------------------------------ mixed radix extension

@pytest.mark.parametrize("n", [3, 5, 6, 12, 15, 20, 30, 48, 60, 96, 160, 240, 375])
def test_mixed_radix_vs_long_double_dft(oracle, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = oracle.dft_naive(a)
    assert np.linalg.norm(oracle.fft1d(a) - ref) / np.linalg.norm(ref) < 1e-15 * max(4, math.log2(n))
    refi = oracle.dft_naive(a, inverse=True)
    assert np.linalg.norm(oracle.fft1d(a, inverse=True) - refi) / np.linalg.norm(refi) < 1e-14


def test_mixed_radix_3d_consistent_with_lines(oracle):
    dims = (12, 5, 6)
    rng = np.random.default_rng(7)
    a = rng.standard_normal(360) + 1j * rng.standard_normal(360)
    ref = np.fft.fftn(a.reshape(dims[2], dims[1], dims[0])).reshape(-1)
    assert np.linalg.norm(oracle.fft3d(a, dims) - ref) / np.linalg.norm(ref) < 1e-14


def test_unsupported_length_rejected(oracle):
    with pytest.raises(ValueError):
        oracle.fft1d(np.ones(7, complex))


# ------------------------------------------------------------ live reference

@pytest.mark.parametrize("dims", [(8, 8, 8), (16, 4, 2), (32, 16, 8)])
def test_live_reference_step_bitwise(oracle, reference, dims):
    box = (-6.0, 6.0, -5.0, 5.0, -4.0, 4.0)
    V = reference.harmonic3d(box, dims, 1.3, (0.5, 0.0, -0.25))
    p = reference.gaussian3d(box, dims, (1.0, 0.5, 0.0), (1.1, 0.9, 1.3), (0.4, -0.2, 0.1))
    m = reference.absorbing_mask3d(box, dims, 1.5)
    for mass in (1.0, 0.38):
        assert same(oracle.step3d(box, dims, V, 0.01, p, 7, mass=mass, mask=m),
                    reference.step3d(box, dims, V, 0.01, p, 7, mass=mass, mask=m))


def test_live_reference_rejects_mixed_radix(reference):
    # the reference's FFT throws for 48 (fft.ixx:40-44): the oracle extension covers it
    with pytest.raises(ValueError):
        reference.fft1d(np.ones(48, complex))
