"""Failure detection on the device without a GPU fault: a bounded wait that runs out.

The reference's engine marks itself device_lost when a fence wait exceeds 10 s
(solver/src/vk_compute.ixx:297-327) and its directors fall back to the CPU.
Here every wait inside a pipelined (TMA-fed) pass is bounded; when one runs out
the pass records an error word, drains its own copies (bounded) and returns, and
the host reports SES_ETIMEDOUT (TimeoutError).  The test makes the wait run out
through ses_gpu_set_wait_limit: every tile barrier expects 16 bytes more than its
copies deliver (no load or store changes), with a ~1 ms limit.  The context must
stay usable: the same handle, reset, and a re-created handle both step correctly.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIMIT_CYCLES = 2_000_000  # ~1 ms at the B200's SM clock


def scene(ses, oracle):
    box, n = (-8.0, 8.0) * 3, (64, 64, 64)
    g = ses.Grid3D(*(ses.Grid1D(-8.0, 8.0, 64) for _ in range(3)))
    V = oracle.harmonic3d(box, n, 1.0)
    psi0 = oracle.gaussian3d(box, n, (1.0, 0.0, 0.0), (1.0, 1.0, 1.0), (0.5, 0.0, 0.0))
    return box, n, g, V, psi0


def test_expired_wait_reports_timeout_and_context_survives(ses, oracle, tmp_path, monkeypatch):
    monkeypatch.setenv("SES_TUNE_CACHE", str(tmp_path / "empty_cache.txt"))  # default (pipelined) variants
    box, n, g, V, psi0 = scene(ses, oracle)
    want = oracle.step3d(box, n, V, 0.01, psi0, 6)
    op = ses.SplitOperator3D(g, V, 0.01, precision="c64", psi0=psi0)
    info = op.plan_info()
    assert "pipelined" in info, info
    op.set_wait_limit(LIMIT_CYCLES, 16)
    op.advance(6)
    with pytest.raises(TimeoutError):
        op.sync(30000)
    # the error word was consumed: a second wait on the same (now idle) handle is clean
    op.sync(30000)
    # normal limits again: the same handle steps correctly
    op.set_wait_limit(0, 0)
    op.upload_state(psi0)
    op.advance(6)
    op.sync(30000)
    err = np.linalg.norm(op.readback() - want) / np.linalg.norm(want)
    assert err < 1e-5
    op.close()
    # and so does a handle created after the failure
    op2 = ses.SplitOperator3D(g, V, 0.01, precision="c64", psi0=psi0)
    op2.advance(6)
    err2 = np.linalg.norm(op2.readback() - want) / np.linalg.norm(want)
    assert err2 < 1e-5
    op2.close()


def test_wait_limit_arguments_are_checked(ses, oracle):
    box, n, g, V, psi0 = scene(ses, oracle)
    op = ses.SplitOperator3D(g, V, 0.01, precision="c64", psi0=psi0)
    with pytest.raises(ValueError):
        op.set_wait_limit(-1, 0)
    with pytest.raises(ValueError):
        op.set_wait_limit(0, 1 << 20)
    op.close()
