"""Imaginary-time relaxation (ses_gpu_create_imag / ses_gpu_relax) against the
FP64 oracle's restatement of the reference ImaginaryTimePropagator3D
(core/src/imaginary_time.ixx:64-144), and the reference's own known answer:
the 3D harmonic trap relaxes to its ground state, E0 = 3/2 (dynamics3_test.cpp:64-87).
"""

import numpy as np
import pytest

from shoeridingerequationsolver_b200 import scenes


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def setup(ses, n=32, box=8.0):
    g = scenes.cube_grid(-box, box, n)
    V = scenes.harmonic(g, 1.0, (0.3, 0.0, -0.2))
    psi = scenes.gaussian(g, (1.0, -0.5, 0.5), (1.3, 0.9, 1.1), (0.0, 0.0, 0.0))
    return g, V, psi


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [("c128", 1e-12), ("c64", 1e-5)])
@pytest.mark.parametrize("every", [1, 7])
def test_relax_matches_oracle(ses, oracle, prec, tol, every):
    g, V, psi = setup(ses)
    op = ses.ImaginaryTimePropagator3D(g, V, 0.02, precision=prec, psi0=psi)
    op.relax_resident(40, renorm_every=every)
    want = oracle.relax3d(g.box, g.dims, V, 0.02, psi, 40)
    got = op.readback()
    assert rel(got, want) <= tol
    assert abs(op.observe()["norm"] - 1.0) <= (1e-12 if prec == "c128" else 1e-6)
    op.close()


@pytest.mark.gpu
def test_relax_reaches_harmonic_ground_state(ses):
    g, V, psi = setup(ses, n=48, box=9.0)
    f = ses.Field3D(g, psi)
    op = ses.ImaginaryTimePropagator3D(g, V, 0.01)
    e_est = op.relax(f, 1500, renorm_every=10)
    o = op.observe()
    assert abs(o["energy"] - 1.5) < 1e-3          # <H> of the relaxed state
    assert abs(e_est - 1.5) < 1e-3                # -ln(norm^2)/(2 r dtau)
    with pytest.raises(ValueError):
        op.half_potential_phase()
    op.close()
