"""Request server (ses_serve_*): continuous batching of solves.

The key property: a request's result does not depend on what else is being
served.  Members of a batch compute exactly what they compute alone, and the
one thing the mix changes -- where a request's rounds end, since other
requests' observation points end rounds too -- changes nothing either: the
kick between two steps is applied as the half kick that ends a batch followed
by the half kick that starts the next, and the batch-start FFT runs in the
radix order of the between-steps pass.  So a complex64 request served in a mix
returns the same bits as served alone, and both match the FP64 oracle within
the complex64 bar.
"""

import math

import numpy as np
import pytest

from shoeridingerequationsolver_b200 import scenes

TOL_ORACLE = 1e-5   # complex64 vs the FP64 oracle


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def spec(ses, dims, box, seed, nsteps, every, dt=0.005):
    rng = np.random.default_rng(seed)
    g = ses.Grid3D(*[ses.Grid1D(-box, box, n) for n in dims])
    V = scenes.harmonic(g, float(rng.uniform(0.5, 1.5)))
    c = [float(rng.uniform(-0.2, 0.2)) * box if n > 1 else 0.0 for n in dims]
    k = [float(rng.uniform(-1, 1)) if n > 1 else 0.0 for n in dims]
    psi = scenes.gaussian(g, c, [0.15 * box if n > 1 else 1.0 for n in dims], k)
    mask = scenes.mask_profiles(g, 0.1)
    return dict(grid=g, V=V, psi0=psi, dt=dt, nsteps=nsteps, observe_every=every, mask=mask,
                x_range=(0.0, math.inf))


def run_all(srv, specs):
    ids = [srv.submit(**s) for s in specs]
    srv.wait_idle(300000)
    out = []
    for rid in ids:
        state, recs = srv.poll(rid)
        assert state == "done", state
        psi, lat = srv.result(rid)
        out.append((psi, recs, lat))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("batch_plane", ["0", "1"])
def test_serve_alone_equals_mix_and_oracle(ses, oracle, monkeypatch, batch_plane):
    """batch_plane "1": the 3D classes step in the two-sweep form (batched plane
    pass + z pass), chosen by shape, so alone and in the mix alike."""
    monkeypatch.setenv("SES_BATCH_PLANE", batch_plane)
    a = spec(ses, (32, 32, 32), 8.0, 1, nsteps=250, every=100)
    others = [spec(ses, (48, 48, 48), 9.0, 2, nsteps=130, every=50),
              spec(ses, (64, 64, 1), 10.0, 3, nsteps=370, every=100),
              spec(ses, (256, 1, 1), 12.0, 4, nsteps=90, every=30),
              spec(ses, (32, 32, 32), 7.0, 5, nsteps=310, every=70)]
    with ses.Server(budget_bytes=8 * 2**30) as srv:
        (alone, recs_alone, _), = run_all(srv, [a])
    with ses.Server(budget_bytes=8 * 2**30) as srv:
        res = run_all(srv, others[:2] + [a] + others[2:])
        st = srv.stats()
    mix, recs_mix, _ = res[2]
    assert st["completed"] == 5 and st["failed"] == 0
    assert np.array_equal(mix, alone), rel(mix, alone)
    assert [r["step"] for r in recs_alone] == [100, 200, 250] == [r["step"] for r in recs_mix]
    assert recs_mix[-1]["final"] and not recs_mix[0]["final"]
    for ra, rm in zip(recs_alone, recs_mix):
        assert ra["norm"] == rm["norm"] and ra["energy"] == rm["energy"]
    # the FP64 oracle on the same request (mask after every step)
    g = a["grid"]
    mx, my, mz = a["mask"]
    full = ((mx[None, None, :] * my[None, :, None]) * mz[:, None, None]).reshape(-1)
    want = oracle.step3d(g.box, g.dims, a["V"], a["dt"], a["psi0"], a["nsteps"], 1.0, full)
    assert rel(mix, want) <= TOL_ORACLE
    # every request of the mix against its own oracle run
    for s, (psi, recs, _) in zip(others[:2] + [a] + others[2:], res):
        g = s["grid"]
        mx, my, mz = s["mask"]
        full = ((mx[None, None, :] * my[None, :, None]) * mz[:, None, None]).reshape(-1)
        want = oracle.step3d(g.box, g.dims, s["V"], s["dt"], s["psi0"], s["nsteps"], 1.0, full)
        assert rel(psi, want) <= TOL_ORACLE, g.dims
        assert recs[-1]["step"] == s["nsteps"]


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(48, 48, 48), (64, 64, 64), (96, 96, 1), (256, 1, 1), (65536, 1, 1)])
def test_step_calls_compose_exactly(ses, dims):
    """n steps in one call == the same n steps split over several calls (complex64)."""
    s = spec(ses, dims, 8.0, 30, nsteps=0, every=0)
    ops = []
    for _ in range(2):
        op = ses.SplitOperator3D(s["grid"], s["V"], s["dt"], precision="c64")
        op.set_absorber_separable(*s["mask"])
        op.upload_state(s["psi0"])
        ops.append(op)
    ops[0].advance(21, absorb=True)
    for k in (3, 1, 9, 8):
        ops[1].advance(k, absorb=True)
    a, b = ops[0].readback(), ops[1].readback()
    assert np.array_equal(a, b), rel(a, b)
    for op in ops:
        op.close()


@pytest.mark.gpu
def test_serve_admission_respects_budget(ses):
    specs = [spec(ses, (32, 32, 32), 8.0, 10 + i, nsteps=60, every=20) for i in range(3)]
    # one 32^3 complex64 request is estimated at 13 MiB: a 20 MiB budget admits one at a time
    with ses.Server(budget_bytes=20 * 2**20) as srv:
        res = run_all(srv, specs)
        st = srv.stats()
        assert st["completed"] == 3 and st["admitted"] == 3
        assert st["bytes_in_use"] == 0
    lats = [lat for _, _, lat in res]
    assert lats[0] < lats[1] < lats[2]
    with ses.Server(budget_bytes=2**20) as srv:
        with pytest.raises(MemoryError):
            srv.submit(**specs[0])


@pytest.mark.gpu
def test_serve_cancel_and_continue(ses):
    long_run = spec(ses, (64, 64, 64), 8.0, 20, nsteps=5000, every=100)
    short = spec(ses, (32, 32, 32), 8.0, 21, nsteps=40, every=0)
    with ses.Server(budget_bytes=4 * 2**30, max_round_steps=50) as srv:
        rid = srv.submit(**long_run)
        srv.cancel(rid)
        sid = srv.submit(**short)
        srv.wait_idle(120000)
        assert srv.poll(rid)[0] == "cancelled"
        state, recs = srv.poll(sid)
        assert state == "done" and len(recs) == 1 and recs[0]["final"] and recs[0]["step"] == 40
        with pytest.raises(Exception):
            srv.result(rid)
        psi, lat = srv.result(sid)
        assert np.all(np.isfinite(psi)) and lat > 0


@pytest.mark.gpu
def test_serve_mixed_precision_and_mass(ses):
    """A complex128 request with an effective mass, served next to complex64 ones
    that start and finish while it runs, ends where the same handle stepped alone
    ends (batched kernels vs single-field kernels: rounding-level agreement)."""
    heavy = spec(ses, (48, 48, 48), 8.0, 31, nsteps=240, every=60)
    heavy.update(precision="c128", mass=0.38)
    light = [spec(ses, (32, 32, 32), 7.0, 40 + i, nsteps=20 + 15 * i, every=0) for i in range(6)]
    with ses.Server(budget_bytes=8 * 2**30, max_round_steps=40) as srv:
        hid = srv.submit(**heavy)
        lids = [srv.submit(**s) for s in light]
        srv.wait_idle(300000)
        for rid in [hid] + lids:
            assert srv.poll(rid)[0] == "done"
        psi, _ = srv.result(hid)
        st = srv.stats()
        assert st["completed"] == 7 and st["failed"] == 0 and st["bytes_in_use"] == 0
    op = ses.SplitOperator3D(heavy["grid"], heavy["V"], heavy["dt"], 0.38, precision="c128", psi0=heavy["psi0"])
    op.set_absorber_separable(*heavy["mask"])
    op.advance(240, absorb=True)
    want = op.readback()
    op.close()
    assert rel(psi, want) <= 1e-13
