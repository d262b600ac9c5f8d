"""Host workload builders (shoeridingerequationsolver_b200/scenes.py) against the
oracle's restatement of the reference builders, and the benchmark inputs'
stated properties."""

import math

import numpy as np

from shoeridingerequationsolver_b200 import scenes
from shoeridingerequationsolver_b200.core import Grid1D, Grid3D


def test_builders_match_oracle(oracle):
    g = Grid3D(Grid1D(-8, 8, 16), Grid1D(-6, 6, 12), Grid1D(-5, 5, 10))
    box, n = g.box, g.dims
    assert np.allclose(scenes.harmonic(g, 1.3, (0.5, 0, -1)), oracle.harmonic3d(box, n, 1.3, (0.5, 0, -1)),
                       rtol=1e-15, atol=0)
    assert np.array_equal(scenes.regularized_coulomb(g, 1.0), oracle.regularized_coulomb3d(box, n, 1.0))
    assert np.array_equal(scenes.barrier(g, 0.25, 0.0, 3.0), oracle.barrier3d(box, n, 0.25, 0.0, 3.0))
    v = scenes.regularized_coulomb(g, 1.0)
    assert np.allclose(scenes.stark_fold(g, v, 0.01), oracle.stark_fold3d(box, n, 0.01, v), rtol=1e-15)
    assert np.array_equal(scenes.stadium(g, 2.0, 4.0, 50.0), oracle.stadium3d(box, n, 2.0, 4.0, 50.0))
    psi = scenes.gaussian(g, (1, -0.5, 0.2), (1.1, 0.9, 1.4), (0.5, 0.2, -0.3))
    ref = oracle.gaussian3d(box, n, (1, -0.5, 0.2), (1.1, 0.9, 1.4), (0.5, 0.2, -0.3))
    assert np.max(np.abs(psi - ref)) < 1e-14
    for prof, code in (("sin2", 0), ("cos8", 1)):
        mx = scenes.mask_profile(g.x, 3.0, prof)
        assert np.allclose(mx, oracle.mask1d(-8, 8, 16, 3.0, code), rtol=1e-14, atol=1e-15)
    g1 = Grid1D(-8, 8, 16)
    assert np.allclose(scenes.morse(g1, 0.3, 0.5, -2.0), oracle.morse1d(-8, 8, 16, 0.3, 0.5, -2.0))
    assert np.allclose(scenes.double_well(g1, 0.1, 4.0), oracle.double_well1d(-8, 8, 16, 0.1, 4.0))
    assert np.allclose(scenes.poschl_teller(g1, 0.375, 2.0), oracle.poschl_teller1d(-8, 8, 16, 0.375, 2.0))


def test_c1_initial_energy_is_3_875(oracle):
    w = scenes.config_c1()
    e = oracle.mean_energy3d(w.grid.box, w.grid.dims, w.psi0, w.V)
    assert abs(e - 3.875) < 1e-9


def test_c2_inputs_small_grid(oracle):
    w = scenes.config_c2(n=32)
    g = w.grid
    assert abs(oracle.norm3d(g.box, g.dims, w.psi0) - 1.0) < 1e-12
    # nucleus cell sits on grid point 16 (coord 0) and takes -Z * 2.3800774 / h (+ Stark 0)
    h = g.x.spacing()
    assert w.V[g.flat(16, 16, 16)] == -2.3800774 / h
    assert len(w.meta["packets"]) == 4
    for p in w.meta["packets"]:
        assert np.linalg.norm(p["centre"]) < 5 and 0.8 <= p["sigma"] <= 2.0
    mx = w.mask[0]
    assert mx[0] == 0.0 and mx[16] == 1.0 and np.all((mx >= 0) & (mx <= 1))
    # same seed -> same inputs
    w2 = scenes.config_c2(n=32)
    assert np.array_equal(w.psi0, w2.psi0)


def test_c3_inputs_small_grid(oracle):
    w = scenes.config_c3(n=32)
    g = w.grid
    assert 1.0 <= w.meta["barrier_height"] <= 5.0
    x = g.x.coords()
    row = w.V.reshape(g.shape)[0, 0, :]
    assert np.all(row[(x >= -1) & (x < 1)] == w.meta["barrier_height"])
    assert np.all(row[(x < -1) | (x >= 1)] == 0.0)
    assert abs(oracle.norm3d(g.box, g.dims, w.psi0) - 1.0) < 1e-12
    assert math.isclose(w.mask[0][1], scenes.mask_profile(g.x, 9.6)[1])
