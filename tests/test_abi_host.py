"""Host-side checks that need no GPU: the C-ABI library loads and exports every
symbol include/ses_gpu.h declares, argument errors are reported without a
device, and the device index arithmetic (fast division, tile plans, shared
memory carve-up) stays in bounds for every grid the tests and bench use."""

import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "ses_gpu.h"


def header_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"SES_API\s+[\w\s\*]+?\b(ses_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = header_symbols()
    assert "ses_gpu_create" in syms and "ses_gpu_step" in syms and "ses_fft3_host" in syms
    assert len(syms) >= 20


def test_library_exports_every_header_symbol():
    from shoeridingerequationsolver_b200 import _abi
    lib = C.CDLL(str(_abi.LIB_PATH))
    for s in header_symbols():
        assert hasattr(lib, s), s
    out = subprocess.run(["nm", "-D", "--defined-only", str(_abi.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(header_symbols()) <= exported
    # nothing beyond the declared C ABI leaks out of the library
    assert {s for s in exported if s.startswith("ses_")} == set(header_symbols())


def test_abi_binding_covers_header():
    from shoeridingerequationsolver_b200 import _abi
    assert sorted(_abi.EXPORTS) == header_symbols()


def test_invalid_arguments_without_device():
    import shoeridingerequationsolver_b200 as s
    g = s.Grid3D(s.Grid1D(-1, 1, 7), s.Grid1D(-1, 1, 8), s.Grid1D(-1, 1, 8))
    with pytest.raises(ValueError, match="2\\^a 3\\^b 5\\^c"):
        s.SplitOperator3D(g, np.zeros(448), 0.1)
    g2 = s.Grid3D(s.Grid1D(-1, 1, 8), s.Grid1D(-1, 1, 8), s.Grid1D(-1, 1, 8))
    with pytest.raises(ValueError):
        s.SplitOperator3D(g2, np.zeros(10), 0.1)          # potential size mismatch
    with pytest.raises(ValueError):
        s.SplitOperator3D(g2, np.zeros(512), 0.1, precision="fp16")
    from shoeridingerequationsolver_b200 import _abi
    h = C.c_void_p()
    bad = _abi.GridDesc(_abi.Axis(1.0, 1.0, 8), _abi.Axis(0, 1, 8), _abi.Axis(0, 1, 8))
    v = np.zeros(512)
    st = _abi.lib.ses_gpu_create(C.byref(bad), 0, 0.1, 1.0, v.ctypes.data_as(C.POINTER(C.c_double)),
                                 None, C.byref(h))
    assert st == _abi.SES_EINVAL and "xmax > xmin" in _abi.last_error()
    assert _abi.lib.ses_gpu_step(None, 1, 0) == _abi.SES_EINVAL


def test_wavenumbers_and_grid_mirror(oracle):
    import shoeridingerequationsolver_b200 as s
    for (lo, hi, n) in [(0, 8, 8), (-1, 1, 1), (-13, -5, 8), (-40, 40, 256), (-10, 10, 48)]:
        assert np.array_equal(s.wavenumbers(s.Grid1D(lo, hi, n)), oracle.wavenumbers(lo, hi, n))
    g = s.Grid3D(s.Grid1D(0, 8, 16), s.Grid1D(0, 4, 8), s.Grid1D(-1, 1, 4))
    assert g.size() == 512 and g.flat(3, 2, 1) == 3 + 16 * (2 + 8 * 1)
    assert g.cell_volume() == 0.125


# ---------------------------------------------------------------------------
# Device index arithmetic, modelled on the CPU.  These restate the host plan
# (ses_gpu.cu plan_pass / factor_radices) and the kernels' index ranges.

def fastdiv(d):
    if d <= 1:
        return (d, 0, 0)
    l = 0
    while (1 << l) < d:
        l += 1
    p = 31 + l
    return (d, ((1 << p) + d - 1) // d, p - 32)


def fdiv(x, f):
    d, m, s = f
    return x if d <= 1 else ((x * m) >> 32) >> s


def test_fastdiv_exact_below_2_31():
    rng = np.random.default_rng(0)
    divisors = list(range(1, 4200)) + [n * n for n in (48, 96, 160, 256, 512, 1024)]
    for d in divisors:
        f = fastdiv(d)
        assert f[1] < 2 ** 32
        xs = list(range(0, 600)) + [int(v) for v in rng.integers(0, 2 ** 31, 200)] + [2 ** 31 - 1]
        for x in xs:
            assert fdiv(x, f) == x // d, (d, x)


EPT, MAXLOG = 8, 3


def radices(n):
    a = b = c = 0
    m = n
    while m % 2 == 0:
        m //= 2
        a += 1
    while m % 3 == 0:
        m //= 3
        b += 1
    while m % 5 == 0:
        m //= 5
        c += 1
    if m != 1:
        return None
    r = []
    if a:
        p = (a + MAXLOG - 1) // MAXLOG
        base, ex = a // p, a % p
        r += [1 << (base + (1 if i < ex else 0)) for i in range(p)]
    return r + [3] * b + [5] * c


def plan(n, es, strided, nlines):
    rad = radices(n)
    L = 256 // es if strided else 128 // es
    while L * n < 2048 and L < 256:
        L *= 2
    pitch = n if strided else (n + 1 if n % 2 == 0 else n)
    while L > 1 and L * pitch * es > 64 * 1024:
        L //= 2
    while L > 1 and L // 2 >= nlines:
        L //= 2

    def threads(L):
        t = 32
        for R in rad:
            t = max(t, -(-(L * n // R) // (EPT // R)))
        return -(-t // 32) * 32
    T = threads(L)
    while T > 512 and L > 1:
        L //= 2
        T = threads(L)
    smem = L * pitch * es
    if strided:
        smem = ((smem + 15) & ~15) + L * 40
    return L, T, pitch, smem, rad


GRIDS = [(8, 8, 8), (16, 8, 4), (8, 16, 4), (4, 4, 4), (64, 64, 64), (256, 256, 256),
         (512, 512, 512), (48, 48, 48), (96, 96, 96), (160, 160, 160), (32, 32, 32),
         (128, 128, 128), (512, 512, 1), (1024, 1024, 1), (4096, 1, 1), (1, 4, 1), (3, 5, 15),
         (2, 2, 2), (48, 24, 20), (96, 20, 6), (512, 4, 2), (1024, 1, 1)]


@pytest.mark.parametrize("dims", GRIDS)
@pytest.mark.parametrize("es", [8, 16])
def test_plans_stay_in_bounds(dims, es):
    nx, ny, nz = dims
    nlines = [ny * nz, nx * nz, nx * ny]
    N = nx * ny * nz
    for ax in range(3):
        n = dims[ax]
        L, T, pitch, smem, rad = plan(n, es, ax != 0, nlines[ax])
        assert T <= 512 and L >= 1 and (L & (L - 1)) == 0
        assert smem <= 200 * 1024
        for R in rad:                     # butterflies per thread within the register budget
            assert -(-(L * (n // R)) // T) <= EPT // R
        if ax == 0:
            assert (L - 1) * pitch + n - 1 < L * pitch
        else:
            assert (L - 1) + (n - 1) * L < L * n
            assert ((L * n * es + 15) & ~15) % 16 == 0
        # Stockham stage indices stay inside [0, n)
        Ns = 1
        for R in rad:
            for j in range(n // R):
                k = j % Ns
                assert (R - 1) * k * (n // (Ns * R)) < n            # twiddle index
                assert (j - k) * R + k + (R - 1) * Ns < n           # write index
                assert j + (R - 1) * (n // R) < n                   # read index
            Ns *= R
        # last line's last element addresses inside psi
        if ax == 0:
            assert (nlines[0] - 1) * nx + nx - 1 < N
        elif ax == 1:
            assert (nx - 1) + (nz - 1) * nx * ny + (ny - 1) * nx < N
        else:
            assert (nx * ny - 1) + (nz - 1) * nx * ny < N


# ---------------------------------------------------------------------------
# Compiled plans (ses_pass2.cuh): the register-resident FFT with thread
# q = j mod (N/E), exchanges through shared memory, per-stage twiddle tables
# laid out forward-then-reversed, and the reversed-order continuation used by
# fused passes -- modelled exactly and compared with numpy's FFT.

COMPILED_PLANS = [(16, 16, (16,)), (32, 8, (8, 4)), (48, 12, (4, 4, 3)), (48, 12, (12, 4)), (64, 8, (8, 8)),
                  (96, 24, (12, 8)),
                  (96, 12, (6, 4, 4)), (128, 16, (16, 8)), (160, 20, (10, 4, 4)), (160, 40, (20, 8)),
                  (256, 16, (16, 16)),
                  (512, 16, (8, 8, 8)), (512, 32, (16, 32)), (1024, 32, (16, 8, 8)),
                  (1024, 32, (32, 32))]


def xpad(N, E):
    """Contiguous-pass line padding (ses_pass2.cuh XPad): element pos at pos + PM (pos >> SH),
    line pitch N + PM (N >> SH) + LPAD."""
    sh = 3 if N in (160, 96, 64) else (2 if N in (48, 32) else 4)
    pm = 3 if N == 48 else 1
    lpad = 0 if (N, E) == (160, 40) else {160: 4, 96: 12, 32: 4}.get(N, 0)
    return sh, pm, lpad


def stage_table(N, rads):
    """Host table (ses_gpu.cu stage_twiddles): forward order then reversed order."""
    out = []
    for order in (rads, tuple(reversed(rads))):
        Ns = 1
        for R in order:
            for r in range(R):
                for k in range(Ns):
                    out.append(np.exp(-2j * np.pi * ((r * k * (N // (Ns * R))) % N) / N))
            Ns *= R
    return np.array(out)


def model_fft(x, N, E, rads, tab, toff):
    TL = N // E
    R0 = rads[0]
    v = [[x[q + TL * b + r * (N // R0)] for b in range(E // R0) for r in range(R0)] for q in range(TL)]
    Ns, off = 1, toff
    smem_max = -1
    for si, R in enumerate(rads):
        for q in range(TL):
            for b in range(E // R):
                k = (q + TL * b) % Ns
                for r in range(1, R):
                    if Ns > 1:
                        idx = off + r * Ns + k
                        assert idx < len(tab)
                        v[q][b * R + r] *= tab[idx]
                v[q][b * R:(b + 1) * R] = list(np.fft.fft(np.array(v[q][b * R:(b + 1) * R])))
        if si + 1 < len(rads):
            Rn = rads[si + 1]
            buf = np.full(N, np.nan, complex)
            for q in range(TL):
                for b in range(E // R):
                    j = q + TL * b
                    k = j % Ns
                    for r in range(R):
                        pos = (j - k) * R + k + r * Ns
                        assert 0 <= pos < N and np.isnan(buf[pos])  # each slot written once
                        sh, pm, _ = xpad(N, E)
                        smem_max = max(smem_max, pos + pm * (pos >> sh))
                        buf[pos] = v[q][b * R + r]
            v = [[buf[q + TL * b + r * (N // Rn)] for b in range(E // Rn) for r in range(Rn)]
                 for q in range(TL)]
        off += R * Ns
        Ns *= R
    RL = rads[-1]
    out = np.zeros(N, complex)
    for q in range(TL):
        for b in range(E // RL):
            for r in range(RL):
                out[q + TL * b + r * (N // RL)] = v[q][b * RL + r]
    sh, pm, lpad = xpad(N, E)
    assert smem_max < N + pm * (N >> sh) + lpad or len(rads) == 1
    return out


@pytest.mark.parametrize("plan", COMPILED_PLANS, ids=[str(p[0]) for p in COMPILED_PLANS])
def test_compiled_plan_index_model(plan):
    N, E, rads = plan
    assert np.prod(rads) == N and all(E % R == 0 for R in rads) and 32 % (N // E) == 0
    tab = stage_table(N, rads)
    fwd_entries = sum(R * int(np.prod(rads[:i])) for i, R in enumerate(rads))
    rng = np.random.default_rng(N)
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    y = model_fft(x, N, E, rads, tab, 0)
    assert np.allclose(y, np.fft.fft(x), rtol=0, atol=1e-10 * np.abs(y).max())
    # the reversed plan consumes the forward plan's register layout directly
    z = model_fft(y, N, E, tuple(reversed(rads)), tab, fwd_entries)
    assert np.allclose(z, np.fft.fft(np.fft.fft(x)), rtol=0, atol=1e-10 * np.abs(z).max())


def test_batch_arguments_without_device():
    from shoeridingerequationsolver_b200 import _abi
    assert _abi.lib.ses_batch_step(None, 1, 0) == _abi.SES_EINVAL
    assert _abi.lib.ses_batch_add(None, None) == _abi.SES_EINVAL
    assert _abi.lib.ses_batch_observe(None, 0.0, 1.0, None, 0) == _abi.SES_EINVAL
    b = C.c_void_p()
    st = _abi.lib.ses_batch_create(C.byref(b))
    if st == _abi.SES_OK:                      # a device is visible
        assert _abi.lib.ses_batch_step(b, -1, 0) == _abi.SES_EINVAL
        assert _abi.lib.ses_batch_step(b, 5, 0) == _abi.SES_OK    # empty batch: nothing to do
        assert _abi.lib.ses_batch_destroy(b) == _abi.SES_OK
    else:
        assert st == _abi.SES_EDEVICE and not b.value


def test_c4_specs_are_seeded_and_cover_every_size():
    from shoeridingerequationsolver_b200 import scenes
    a, b = scenes.config_c4_specs(), scenes.config_c4_specs()
    assert a == b and len(a) == 256
    assert {s["n"] for s in a} == set(scenes.C4_SIZES)
    for s in a:
        assert 0.5 <= s["barrier"] <= 4.0 and 1.0 <= s["k0"] <= 4.0 and 1.0 <= s["sigma"] <= 2.5
        assert abs(s["side"] / s["n"] - 0.625) < 1e-15
    w = scenes.build_c4_instance(a[0])
    assert w.grid.dims == (a[0]["n"],) * 3 and w.psi0.size == a[0]["n"] ** 3


def test_serve_arguments_without_device():
    from shoeridingerequationsolver_b200 import _abi
    rid = C.c_int64()
    assert _abi.lib.ses_serve_submit(None, None, C.byref(rid)) == _abi.SES_EINVAL
    assert _abi.lib.ses_serve_close(None) == _abi.SES_EINVAL
    s = C.c_void_p()
    assert _abi.lib.ses_serve_open(0, 0, C.byref(s)) == _abi.SES_EINVAL
    st = _abi.lib.ses_serve_open(1 << 30, 0, C.byref(s))
    if st == _abi.SES_OK:                      # a device is visible
        r = _abi.Request()
        assert _abi.lib.ses_serve_submit(s, C.byref(r), C.byref(rid)) == _abi.SES_EINVAL
        assert _abi.lib.ses_serve_close(s) == _abi.SES_OK
    else:
        assert st == _abi.SES_EDEVICE


def test_four_step_layout_of_long_lines():
    """Long 1D lines (ses_gpu.cu long1d, ses_pass2.cuh SM_TW_*): the stored
    layout, twiddle index and frequency map of the four-step transform, modelled
    with numpy on a 24 x 16 line and compared with the plain DFT."""
    n1, n2 = 24, 16
    N = n1 * n2
    rng = np.random.default_rng(3)
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    a = x.reshape(n2, n1)                               # a[n2, n1] = x[n1 + N1 n2]
    y = np.fft.fft(a, axis=0)                           # y pass: length-N2 transforms -> [k2, n1]
    f = np.arange(N).reshape(n2, n1)                    # flat index n1 + N1 k2 of each stored element
    tw = np.exp(-2j * np.pi * (((f % n1) * (f // n1)) % N) / N)
    z = np.fft.fft(y * tw, axis=1)                      # x pass: length-N1 transforms -> [k2, k1]
    k1, k2 = f % n1, f // n1
    X = np.fft.fft(x)
    assert np.allclose(z, X[k2 + n2 * k1], atol=1e-9)   # stored (k1, k2) is frequency k2 + N2 k1
    # inverse: conj trick with conj(W) before the y transforms, as the between-steps pass
    back = np.conj(np.fft.fft(np.conj(np.conj(np.fft.fft(np.conj(z), axis=1)) / n1 * np.conj(tw)), axis=0)) / n2
    assert np.allclose(back.reshape(-1), x, atol=1e-12)
