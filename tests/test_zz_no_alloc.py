"""Allocation-free real-space observables (ses_observe_real_noalloc).

The entry point serves callers that cannot allocate device memory -- a host
framework whose caching allocator already owns the GPU (a library cudaMalloc
could fail), or a loop that must not pay cudaMalloc synchronisation.  It takes
the field, the potential and the 9-double output in the caller's device memory
and keeps its per-CTA partial sums in a fixed array inside the library.  These
tests call it through the C ABI twice in a row and compare with the FP64 oracle
on the same field (read back from the device) and with the handle-based
ses_gpu_observe, which reduces the same field with its own buffers; they cover a
3D grid, a 1024 x 1024 plane, a 65536-point line and a call without a potential.
"""

import ctypes as C

import numpy as np
import pytest

TOL = 1e-12  # the device reductions: the same values in FP64, only the blocked summation order differs


def tol_oracle(npts):
    """The oracle sums left to right (core/src/field.ixx:68-74), whose rounding grows
    with the point count (about sqrt(N) ulps): 1e-11 relative at 65536 points,
    scaled by sqrt(N / 65536) above."""
    return 1e-11 * max(1.0, (npts / 65536.0) ** 0.5)


def _grid(ses, box, n):
    return ses.Grid3D(*(ses.Grid1D(box[2 * a], box[2 * a + 1], n[a]) for a in range(3)))


CASES = {
    "3d": ((-10.0, 10.0, -8.0, 8.0, -6.0, 6.0), (64, 48, 40)),
    "plane": ((-30.0, 30.0, -30.0, 30.0, 0.0, 1.0), (1024, 1024, 1)),
    "line": ((-200.0, 200.0, 0.0, 1.0, 0.0, 1.0), (65536, 1, 1)),
}


def _field(oracle, box, n):
    V = oracle.harmonic3d(box, n, 0.9, (0.5, -0.25, 0.0))
    c = [1.5, -0.5 if n[1] > 1 else 0.0, 0.25 if n[2] > 1 else 0.0]
    s = [1.2, 1.0 if n[1] > 1 else 1.0, 0.9 if n[2] > 1 else 1.0]
    psi = oracle.gaussian3d(box, n, c, s, (0.6, 0.0, -0.4 if n[2] > 1 else 0.0))
    return V, psi


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["3d", "plane", "line"])
@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_noalloc_matches_oracle_and_observe_on_two_calls(ses, oracle, prec, case):
    import torch
    from shoeridingerequationsolver_b200 import _abi
    from shoeridingerequationsolver_b200.core import PRECISIONS

    box, n = CASES[case]
    V, psi = _field(oracle, box, n)
    op = ses.SplitOperator3D(_grid(ses, box, n), V, 0.01, precision=prec)
    op.upload_state(psi)
    op.advance(3)
    ref = op.observe(0.5, 7.0)
    field = op.readback()  # the field both reductions see (complex64 widened exactly)
    op.sync()
    psi_ptr, _ = op.psi_device()
    # the oracle's serial FP64 sums on the same field
    nrm = oracle.norm3d(box, n, field)
    want = np.array([nrm, np.nan, oracle.prob_x_range3d(box, n, field, 0.5, 7.0),
                     *oracle.mean_position3d(box, n, field), *oracle.sigma_position3d(box, n, field)])
    expect = np.array([ref["norm"], ref["energy_v"], ref["p_range"], *ref["mean_pos"], *ref["sigma_pos"]])

    V_dev = torch.from_numpy(V).to("cuda")        # caller-owned device buffers
    out = torch.full((9,), float("nan"), dtype=torch.float64, device="cuda")
    desc = _abi.grid_desc(_grid(ses, box, n))
    for call in range(2):                          # the shared scratch carries over between calls
        out.fill_(float("nan"))
        st = _abi.lib.ses_observe_real_noalloc(C.byref(desc), PRECISIONS[prec], C.c_void_p(psi_ptr),
                                              C.c_void_p(V_dev.data_ptr()), 0.5, 7.0,
                                              C.c_void_p(out.data_ptr()), None)
        assert st == _abi.SES_OK, _abi.last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got)), (call, got)
        assert np.allclose(got, expect, rtol=TOL, atol=TOL), (call, got, expect)
        # the oracle: norm, probability and moments; <V> against the FP64 sum of V |psi|^2 / sum |psi|^2
        idx = [0, 2, 3, 4, 5, 6, 7, 8]
        to = tol_oracle(n[0] * n[1] * n[2])
        assert np.allclose(got[idx], want[idx], rtol=to, atol=to), (call, got[idx], want[idx])
        w = field.real ** 2 + field.imag ** 2
        assert abs(got[1] - float(np.sum(V * w) / np.sum(w))) <= 1e-12 * max(1.0, abs(got[1]))
    # without a potential: <V> is 0, the other eight values are unchanged
    out.fill_(float("nan"))
    st = _abi.lib.ses_observe_real_noalloc(C.byref(desc), PRECISIONS[prec], C.c_void_p(psi_ptr), None, 0.5, 7.0,
                                          C.c_void_p(out.data_ptr()), None)
    assert st == _abi.SES_OK, _abi.last_error()
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert got[1] == 0.0
    assert np.allclose(np.delete(got, 1), np.delete(expect, 1), rtol=TOL, atol=TOL)
    op.close()


def test_noalloc_rejects_grids_beyond_its_scratch():
    import shoeridingerequationsolver_b200 as ses
    from shoeridingerequationsolver_b200 import _abi

    # 1024 x 1024 x 129 points needs more partial-sum rows than the fixed array holds
    desc = _abi.grid_desc(_grid(ses, (0.0, 1.0) * 3, (1024, 1024, 129)))
    st = _abi.lib.ses_observe_real_noalloc(C.byref(desc), _abi.SES_C64, C.c_void_p(16), None, 0.0, 1.0,
                                          C.c_void_p(16), None)
    assert st == _abi.SES_EINVAL
    assert "2^27" in _abi.last_error()
