"""CUDA path vs the FP64 oracle, through the C ABI (libses_b200.so).

Mirrors the reference's own hot-path tests (tests/fft_test.cpp, fft3_test.cpp,
propagator_test.cpp, propagator_tables_test.cpp, dynamics3_test.cpp,
harmonic_dynamics_test.cpp) and its GPU oracle checks
(solver/src/vkcheck_main.cpp check_fft3 :1847-1948, check_engine_step
:2192-2248, check_engine_planar_mass :2325-2387, check_engine_absorber
:2446-2493).

Tolerances (relative L2 error ||gpu - oracle|| / ||oracle||):
  complex128 path: 1e-12 per Strang step (FFT summation order differs from the
                   oracle's radix-2 DIT, so results are not bit-exact)
  complex64 path:  FP32 FFT arithmetic, FP64-built tables: 1e-5 over <= 1000 steps
"""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_C128_STEP = 1e-12
TOL_C64 = 1e-5


def rel_l2(a, b):
    a = np.asarray(a).reshape(-1)
    b = np.asarray(b).reshape(-1)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def cube(lo, hi, n):
    return (lo, hi, lo, hi, lo, hi), (n, n, n)


def grid3(ses, box, n):
    return ses.Grid3D(ses.Grid1D(box[0], box[1], n[0]), ses.Grid1D(box[2], box[3], n[1]),
                      ses.Grid1D(box[4], box[5], n[2]))


def deterministic_signal(N):
    t = np.arange(N, dtype=np.float64)
    return (np.sin(1.3 * t) + 0.1 * t) + 1j * (np.cos(2.7 * t) - 0.05 * t)


# ---------------------------------------------------------------- fft surface

def test_fft3_plane_wave_spikes_at_its_bin(ses):
    # fft3_test.cpp:40-60: distinct axis sizes catch axis/stride mix-ups
    nx, ny, nz = 8, 16, 4
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    th = 2 * np.pi * (3.0 * i / nx + 5.0 * j / ny + 1.0 * k / nz)
    f = np.exp(1j * th).reshape(-1)
    for prec, tol in (("c128", 1e-9), ("c64", 1e-3)):
        out = ses.fft(f.reshape(nz, ny, nx), precision=prec).reshape(-1)
        expect = np.zeros_like(f)
        expect[3 + nx * (5 + ny * 1)] = 512.0
        assert np.max(np.abs(out - expect)) < tol


@pytest.mark.parametrize("dims", [(8, 4, 2), (16, 8, 4), (4, 8, 2), (64, 64, 64), (48, 12, 5),
                                  (1, 4, 1), (3, 5, 15), (256, 16, 8), (128, 1, 1), (2, 2, 2),
                                  (96, 20, 6), (512, 4, 2)])
def test_fft3_matches_oracle(ses, oracle, dims):
    rng = np.random.default_rng(sum(dims))
    N = dims[0] * dims[1] * dims[2]
    a = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    arr = a.reshape(dims[2], dims[1], dims[0])
    for inverse in (False, True):
        ref = oracle.fft3d(a, dims, inverse=inverse)
        got = (ses.ifft if inverse else ses.fft)(arr, precision="c128").reshape(-1)
        assert rel_l2(got, ref) < 1e-14 * max(1.0, math.log2(N))
        got32 = (ses.ifft if inverse else ses.fft)(arr, precision="c64").reshape(-1)
        assert rel_l2(got32, ref) < 1e-6


def test_fft_known_answers(ses):
    # fft_test.cpp:28-142 on the device path (lines as n x 1 x 1)
    a = np.zeros(8, complex)
    a[0] = 1
    assert np.allclose(ses.fft(a), np.ones(8), atol=1e-12)                 # delta -> flat
    assert np.allclose(ses.fft(np.ones(8, complex))[1:], 0, atol=1e-12)   # DC -> bin 0
    n, k0 = 16, 3
    x = np.exp(2j * np.pi * k0 * np.arange(n) / n)
    X = ses.fft(x)                                                          # kernel sign
    assert abs(X[k0] - 16) < 1e-12 and np.max(np.abs(np.delete(X, k0))) < 1e-12
    c = ses.fft(np.cos(2 * np.pi * k0 * np.arange(n) / n).astype(complex))
    assert abs(c[3] - 8) < 1e-12 and abs(c[13] - 8) < 1e-12
    s = deterministic_signal(16)
    assert np.allclose(ses.ifft(ses.fft(s)), s, atol=1e-12)                # inverse
    assert abs(np.sum(np.abs(s) ** 2) - np.sum(np.abs(ses.fft(s)) ** 2) / 16) < 1e-10  # Parseval
    assert np.allclose(ses.fft(np.array([3 - 4j])), [3 - 4j])              # size one


def test_fft_rejects_unsupported_length(ses):
    with pytest.raises(ValueError):
        ses.fft(np.ones(7, complex))
    with pytest.raises(ValueError):
        ses.fft(np.ones(7 * 1024, complex))  # above 4096 and not N1 x N2 with compiled factors


# ---------------------------------------------------------------- tables

def ulp_diff(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.abs(a - b) / np.spacing(np.maximum(np.abs(a), np.abs(b)))


def test_propagator_tables_match_formula(ses, oracle):
    # propagator_tables_test.cpp:28-65 (EXPECT_DOUBLE_EQ = 4 ulp)
    box, n = cube(0.0, 4.0, 4)
    V = oracle.harmonic3d(box, n, 2.0, (1.0, 2.0, 3.0))
    for mass in (1.0, 2.0, 0.38):
        op = ses.SplitOperator3D(grid3(ses, box, n), V, 0.1, mass)
        half, kin = oracle.tables3d(box, n, V, 0.1, mass)
        h = op.half_potential_phase()
        k = op.kinetic_phase()
        for got, ref in ((h, half), (k, kin)):
            assert np.all(ulp_diff(got.real, ref.real) <= 4)
            assert np.all(ulp_diff(got.imag, ref.imag) <= 4)
        assert op.dt() == 0.1
        op.close()


def test_tables_large_grid_match_oracle(ses, oracle):
    box, n = (-40, 40, -40, 40, -40, 40), (32, 32, 32)
    V = oracle.regularized_coulomb3d(box, n, 1.0)
    op = ses.SplitOperator3D(grid3(ses, box, n), V, 0.01)
    half, kin = oracle.tables3d(box, n, V, 0.01)
    assert np.max(np.abs(op.half_potential_phase() - half)) < 1e-15
    assert np.max(np.abs(op.kinetic_phase() - kin)) < 1e-15


# ---------------------------------------------------------------- Strang step

def run_gpu(ses, box, n, V, dt, psi0, nsteps, prec="c128", mass=1.0, mask=None, separable=None):
    op = ses.SplitOperator3D(grid3(ses, box, n), V, dt, mass, precision=prec)
    if separable is not None:
        op.set_absorber_separable(*separable)
    elif mask is not None:
        op.set_absorber(mask)
    op.upload_state(psi0)
    op.advance(nsteps, absorb=(mask is not None or separable is not None))
    out = op.readback()
    op.close()
    return out


STEP_CASES = [
    # name, box, n, potential builder, dt, packet (r0, sigma, k0), steps, mass
    ("vkcheck_8cube_soft_coulomb", cube(-4, 4, 8), lambda o, b, n: o.soft_coulomb3d(b, n, 1.0, 1.0),
     0.02, ((1, 0, 0), (1.2, 1.2, 1.2), (0, 0.5, 0)), 20, 1.0),
    ("simulation_16cube_harmonic", cube(-8, 8, 16), lambda o, b, n: o.harmonic3d(b, n, 1.0),
     0.02, ((2, 0, 0), (1, 1, 1), (0, 0.5, 0)), 5, 1.0),
    ("c1_64cube_harmonic", cube(-10, 10, 64), lambda o, b, n: o.harmonic3d(b, n, 1.0),
     0.005, ((2, 0, 0), (1, 1, 1), (0, 0, 0)), 20, 1.0),
    ("planar_64sq_harmonic_mass", ((-16, 16, -16, 16, 0, 2), (64, 64, 1)),
     lambda o, b, n: o.harmonic3d(b, n, 0.5), 0.01, ((3, 1, 0), (1.5, 1.5, 1.0), (2, 0, 0)), 12, 0.38),
    ("mixed_radix_48x24x20_coulomb", ((-12, 12, -6, 6, -5, 5), (48, 24, 20)),
     lambda o, b, n: o.regularized_coulomb3d(b, n, 1.0), 0.01, ((1, 0, 0), (1, 1, 1), (0, 0, 0.5)), 9,
     1.0),
    ("line_1024_free", ((-40, 40, 0, 1, 0, 1), (1024, 1, 1)), lambda o, b, n: np.zeros(1024),
     0.05, ((-15, 0, 0), (1, 1, 1), (2, 0, 0)), 30, 1.0),
    # the serving mix's large planes: 1024-point rows and 1024-point strided columns
    ("planar_1024sq_harmonic", ((-30, 30, -30, 30, 0, 1), (1024, 1024, 1)),
     lambda o, b, n: o.harmonic3d(b, n, 0.5), 0.005, ((2, -1, 0), (1.5, 1.5, 1.0), (2, 0, 0)), 4, 1.0),
]


@pytest.mark.parametrize("case", STEP_CASES, ids=[c[0] for c in STEP_CASES])
@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_step_matches_oracle(ses, oracle, case, prec):
    name, (box, n), vb, dt, (r0, sig, k0), nsteps, mass = case
    V = vb(oracle, box, n)
    psi0 = oracle.gaussian3d(box, n, r0, sig, k0)
    ref = oracle.step3d(box, n, V, dt, psi0, nsteps, mass=mass)
    got = run_gpu(ses, box, n, V, dt, psi0, nsteps, prec=prec, mass=mass)
    err = rel_l2(got, ref)
    if prec == "c128":
        assert err < TOL_C128_STEP * nsteps, err
    else:
        assert err < TOL_C64, err


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_absorber_matches_oracle(ses, oracle, prec):
    # vkcheck check_engine_absorber: 8^3, sin^2 mask width 2, 5 steps, mask after every step
    (box, n) = cube(-4, 4, 8)
    V = oracle.soft_coulomb3d(box, n, 1.0, 1.0)
    psi0 = oracle.gaussian3d(box, n, (1, 0, 0), (1.2, 1.2, 1.2), (0, 0.5, 0))
    mask = oracle.mask3d(box, n, 2.0, 0)
    ref = oracle.step3d(box, n, V, 0.02, psi0, 5, mask=mask)
    got = run_gpu(ses, box, n, V, 0.02, psi0, 5, prec=prec, mask=mask)    # detected separable
    tol = TOL_C128_STEP * 5 if prec == "c128" else TOL_C64
    assert rel_l2(got, ref) < tol
    # non-separable mask takes the full-array path
    rng = np.random.default_rng(3)
    mask2 = mask * (1.0 - 0.01 * rng.random(mask.size))
    ref2 = oracle.step3d(box, n, V, 0.02, psi0, 5, mask=mask2)
    got2 = run_gpu(ses, box, n, V, 0.02, psi0, 5, prec=prec, mask=mask2)
    assert rel_l2(got2, ref2) < tol


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_cos8_absorber_separable_profiles(ses, oracle, prec):
    box, n = (-10, 10, -10, 10, -10, 10), (32, 32, 32)
    V = oracle.harmonic3d(box, n, 0.3)
    psi0 = oracle.gaussian3d(box, n, (4, 0, 0), (1.5, 1.5, 1.5), (2, 0, 0))
    mx = oracle.mask1d(-10, 10, 32, 2.0, 1)
    mask = oracle.mask3d(box, n, 2.0, 1)
    ref = oracle.step3d(box, n, V, 0.01, psi0, 40, mask=mask)
    got = run_gpu(ses, box, n, V, 0.01, psi0, 40, prec=prec, separable=(mx, mx, mx))
    tol = TOL_C128_STEP * 40 if prec == "c128" else TOL_C64
    assert rel_l2(got, ref) < tol


def test_reference_step_semantics(ses, oracle):
    # SplitOperator3D::step(Field3D&, n) in place on a caller-owned field
    box, n = cube(-8, 8, 16)
    V = oracle.harmonic3d(box, n, 1.0)
    psi0 = oracle.gaussian3d(box, n, (2, 0, 0), (1, 1, 1), (0, 0.5, 0))
    g = grid3(ses, box, n)
    f = ses.Field3D(g, psi0)
    op = ses.SplitOperator3D(g, V, 0.02)
    op.step(f, 5)
    assert rel_l2(f.data, oracle.step3d(box, n, V, 0.02, psi0, 5)) < 5e-12
    op.step(f, 0)  # zero steps is the identity (propagator_test.cpp:44-51)
    assert rel_l2(f.data, oracle.step3d(box, n, V, 0.02, psi0, 5)) < 5e-12
    with pytest.raises(ValueError):
        op.advance(-1)


def test_batches_compose(ses, oracle):
    box, n = cube(-10, 10, 32)
    V = oracle.harmonic3d(box, n, 1.0)
    psi0 = oracle.gaussian3d(box, n, (2, 0, 0), (1, 1, 1), (0, 0, 0))
    op = ses.SplitOperator3D(grid3(ses, box, n), V, 0.005)
    op.upload_state(psi0)
    op.advance(3)
    op.advance(17)
    a = op.readback()
    op.upload_state(psi0)
    op.advance(20)
    b = op.readback()
    assert rel_l2(a, b) < 1e-13


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_bitwise_deterministic(ses, oracle, prec):
    box, n = cube(-10, 10, 64)
    V = oracle.harmonic3d(box, n, 1.0)
    psi0 = oracle.gaussian3d(box, n, (2, 0, 0), (1, 1, 1), (0, 0, 0))
    a = run_gpu(ses, box, n, V, 0.005, psi0, 12, prec=prec)
    b = run_gpu(ses, box, n, V, 0.005, psi0, 12, prec=prec)
    assert np.array_equal(a, b)


# ---------------------------------------------------------------- physics checks

def test_free_packet_1d_analytic(ses, oracle):
    # propagator_test.cpp:27-77: 1024 points on [-40, 40), dt 0.05, 200 steps
    xmin, xmax, N = -40.0, 40.0, 1024
    psi0 = oracle.gaussian1d(xmin, xmax, N, -15.0, 1.0, 2.0)
    g = ses.Grid1D(xmin, xmax, N)
    f = ses.Field1D(g, psi0)
    op = ses.SplitOperator1D(g, np.zeros(N), 0.05)
    op.step(f, 200)
    box = (xmin, xmax, 0, 1, 0, 1)
    t = 10.0
    assert abs(oracle.norm1d(xmin, xmax, N, f.data) - 1.0) < 1e-12
    pos = oracle.mean_position3d(box, (N, 1, 1), f.data)[0]
    assert abs(pos - (-15.0 + 2.0 * t)) < 1e-6
    sx = oracle.sigma_position3d(box, (N, 1, 1), f.data)[0]
    assert abs(sx - math.sqrt(1 + (t / 2) ** 2)) < 1e-6
    assert abs(oracle.mean_momentum3d(box, (N, 1, 1), f.data)[0] - 2.0) < 1e-8


def test_anisotropic_free_packet_3d(ses, oracle):
    # dynamics3_test.cpp:29-62: 64^3 on [-12,12), dt 1.0 (V = 0 is time exact), 2 steps
    box, n = cube(-12, 12, 64)
    r0, s0, k0 = (-3, 1, 0), (0.8, 1.0, 1.2), (1.5, 0, -1)
    psi0 = oracle.gaussian3d(box, n, r0, s0, k0)
    out = run_gpu(ses, box, n, np.zeros(64 ** 3), 1.0, psi0, 2)
    assert abs(oracle.norm3d(box, n, out) - 1.0) < 1e-12
    r = oracle.mean_position3d(box, n, out)
    s = oracle.sigma_position3d(box, n, out)
    p = oracle.mean_momentum3d(box, n, out)
    for a in range(3):
        assert abs(r[a] - (r0[a] + k0[a] * 2.0)) < 1e-6
        q = 2.0 / (2 * s0[a] ** 2)
        assert abs(s[a] - s0[a] * math.sqrt(1 + q * q)) < 1e-6
        assert abs(p[a] - k0[a]) < 1e-8


def test_strang_second_order_in_dt(ses, oracle):
    # harmonic_dynamics_test.cpp:76-92: halving dt drops the <x> error ~4x
    xmin, xmax, N = -16.0, 16.0, 512
    V = oracle.harmonic1d(xmin, xmax, N, 1.0)
    psi0 = oracle.gaussian1d(xmin, xmax, N, 2.0, 1 / math.sqrt(2), 0.0)
    g = ses.Grid1D(xmin, xmax, N)
    box = (xmin, xmax, 0, 1, 0, 1)

    def err(dt, steps):
        f = ses.Field1D(g, psi0)
        ses.SplitOperator1D(g, V, dt).step(f, steps)
        return abs(oracle.mean_position3d(box, (N, 1, 1), f.data)[0] - 2.0 * math.cos(1.0))

    ratio = err(0.1, 10) / err(0.05, 20)
    assert 3.4 < ratio < 4.6


# ---------------------------------------------------------------- observables

@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_observables_match_oracle(ses, oracle, prec):
    box, n = (-10, 10, -10, 10, -5, 5), (32, 24, 20)
    V = oracle.harmonic3d(box, n, 1.0)
    psi = oracle.gaussian3d(box, n, (2, -1, 0.5), (1.0, 1.3, 0.9), (0.5, -0.3, 0.2))
    op = ses.SplitOperator3D(grid3(ses, box, n), V, 0.005, 1.0, precision=prec)
    op.upload_state(psi)
    o = op.observe(0.5, 10.0)
    tol = 1e-12 if prec == "c128" else 1e-6
    assert abs(o["norm"] - oracle.norm3d(box, n, psi)) < tol
    assert abs(o["energy"] - oracle.mean_energy3d(box, n, psi, V)) < tol * 10
    assert abs(o["p_range"] - oracle.prob_x_range3d(box, n, psi, 0.5, 10.0)) < tol
    for a in range(3):
        assert abs(o["mean_pos"][a] - oracle.mean_position3d(box, n, psi)[a]) < tol * 10
        assert abs(o["sigma_pos"][a] - oracle.sigma_position3d(box, n, psi)[a]) < tol * 10
        assert abs(o["mean_mom"][a] - oracle.mean_momentum3d(box, n, psi)[a]) < tol * 10


def test_observables_line(ses, oracle):
    xmin, xmax, N = -20.0, 20.0, 512
    V = oracle.morse1d(xmin, xmax, N, 3.0, 0.5, 0.0)
    psi = oracle.gaussian1d(xmin, xmax, N, 0.5, 1.0, 0.5)
    op = ses.SplitOperator3D(ses.line_grid(ses.Grid1D(xmin, xmax, N)), V, 0.01)
    op.upload_state(psi)
    o = op.observe()
    assert abs(o["norm"] - oracle.norm1d(xmin, xmax, N, psi)) < 1e-12
    assert abs(o["energy"] - oracle.mean_energy1d(xmin, xmax, N, psi, V)) < 1e-11


def test_c1_energy_conservation_c128(ses, oracle):
    # C1 shape: 64^3 harmonic, dt 0.005; E0 = 3.875 exactly by the formula
    box, n = cube(-10, 10, 64)
    V = oracle.harmonic3d(box, n, 1.0)
    psi0 = oracle.gaussian3d(box, n, (2, 0, 0), (1, 1, 1), (0, 0, 0))
    op = ses.SplitOperator3D(grid3(ses, box, n), V, 0.005)
    op.upload_state(psi0)
    e0 = op.observe()["energy"]
    assert abs(e0 - 3.875) < 1e-9
    op.advance(200)
    o = op.observe()
    assert abs(o["norm"] - 1.0) < 1e-12
    assert abs(o["energy"] - e0) < 1e-4
