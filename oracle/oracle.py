"""ctypes bindings for the CPU oracle (TEST INFRASTRUCTURE).

Two libraries, both checkers and never part of the product path:

* ``oracle/libses_oracle.so`` -- the C restatement (``ses_oracle.c``) of the
  reference core's FP64 split-operator algorithm, with the mixed-radix and
  cos^(1/8)-mask extensions.  Always buildable (``make -C oracle``).
* ``oracle/_ref/libsesref.so`` -- the reference's own core compiled from its
  sources by ``oracle/build_ref.py``; optional (absent when the reference tree
  was not available at build time).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (cpu baseline and
reference arm) import this module.

Arrays: complex fields are numpy ``complex128`` (interleaved re/im in memory,
x-fastest flat layout, index ``i + nx*(j + ny*k)``); real fields ``float64``.
A grid is ``box = (xmin, xmax, ymin, ymax, zmin, zmax)`` with ``n = (nx, ny, nz)``.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "libses_oracle.so"
REF_SO = HERE / "_ref" / "libsesref.so"

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _box(box):
    return np.ascontiguousarray(box, dtype=np.float64)


def _n(n):
    return np.ascontiguousarray(n, dtype=np.int32)


def _nptr(n):
    return n.ctypes.data_as(_ip)


def _total(n):
    return int(n[0]) * int(n[1]) * int(n[2])


def build_oracle() -> Path:
    import subprocess
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return ORACLE_SO


class Oracle:
    """The C restatement (libses_oracle.so)."""

    def __init__(self, path: Path | str = ORACLE_SO):
        if not Path(path).exists():
            build_oracle()
        self.lib = L = C.CDLL(str(path))
        for name in ["seso_fft1d", "seso_ifft1d"]:
            getattr(L, name).argtypes = [_dp, C.c_size_t]
            getattr(L, name).restype = C.c_int
        for name in ["seso_fft3d", "seso_ifft3d"]:
            getattr(L, name).argtypes = [_dp, _ip]
            getattr(L, name).restype = C.c_int
        L.seso_dft_naive.argtypes = [_dp, _dp, C.c_size_t, C.c_int]
        L.seso_fft_twiddles.argtypes = [C.c_size_t, _dp]
        L.seso_wavenumbers.argtypes = [C.c_double, C.c_double, C.c_int, _dp]
        L.seso_tables3d.argtypes = [_dp, _ip, _dp, C.c_double, C.c_double, _dp, _dp]
        L.seso_step3d.argtypes = [_dp, _ip, _dp, C.c_double, C.c_double, _dp, _dp, C.c_int]
        L.seso_step3d.restype = C.c_int
        L.seso_step1d.argtypes = [C.c_double, C.c_double, C.c_int, _dp, C.c_double, _dp, _dp,
                                  C.c_int]
        L.seso_step1d.restype = C.c_int
        L.seso_relax3d.argtypes = [_dp, _ip, _dp, C.c_double, C.c_double, _dp, C.c_int]
        L.seso_relax3d.restype = C.c_int
        L.seso_driven_step3d.argtypes = [_dp, _ip, _dp, C.c_double, C.c_double, _dp, C.c_double, C.c_double,
                                         C.c_double, _dp, C.c_int]
        L.seso_driven_step3d.restype = C.c_int
        L.seso_harmonic3d.argtypes = [_dp, _ip, C.c_double, _dp, _dp]
        L.seso_soft_coulomb3d.argtypes = [_dp, _ip, C.c_double, C.c_double, _dp, _dp]
        L.seso_regularized_coulomb3d.argtypes = [_dp, _ip, C.c_double, _dp, _dp]
        L.seso_barrier3d.argtypes = [_dp, _ip, C.c_double, C.c_double, C.c_double, _dp]
        L.seso_stark_fold3d.argtypes = [_dp, _ip, C.c_double, _dp]
        L.seso_stadium3d.argtypes = [_dp, _ip, C.c_double, C.c_double, C.c_double, _dp]
        L.seso_harmonic1d.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double, C.c_double, _dp]
        L.seso_morse1d.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double, C.c_double,
                                   C.c_double, _dp]
        L.seso_double_well1d.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double, C.c_double,
                                         _dp]
        L.seso_poschl_teller1d.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double,
                                           C.c_double, C.c_double, _dp]
        L.seso_mask1d.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double, C.c_int, _dp]
        L.seso_mask3d.argtypes = [_dp, _ip, C.c_double, C.c_int, _dp]
        L.seso_gaussian3d.argtypes = [_dp, _ip, _dp, _dp, _dp, _dp]
        L.seso_gaussian1d.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double, C.c_double,
                                      C.c_double, _dp]
        for name in ["seso_norm3d"]:
            getattr(L, name).argtypes = [_dp, _ip, _dp]
            getattr(L, name).restype = C.c_double
        L.seso_norm1d.argtypes = [C.c_double, C.c_double, C.c_int, _dp]
        L.seso_norm1d.restype = C.c_double
        L.seso_mean_energy3d.argtypes = [_dp, _ip, _dp, _dp, C.c_double]
        L.seso_mean_energy3d.restype = C.c_double
        L.seso_mean_energy1d.argtypes = [C.c_double, C.c_double, C.c_int, _dp, _dp]
        L.seso_mean_energy1d.restype = C.c_double
        L.seso_prob_x_range3d.argtypes = [_dp, _ip, _dp, C.c_double, C.c_double]
        L.seso_prob_x_range3d.restype = C.c_double
        for name in ["seso_mean_position3d", "seso_sigma_position3d", "seso_mean_momentum3d"]:
            getattr(L, name).argtypes = [_dp, _ip, _dp, _dp]

    # ---- FFT ----
    def fft1d(self, a, inverse=False):
        a = np.array(a, dtype=np.complex128, copy=True)
        fn = self.lib.seso_ifft1d if inverse else self.lib.seso_fft1d
        if fn(a.ctypes.data_as(_dp), a.size) != 0:
            raise ValueError("unsupported FFT length")
        return a

    def fft3d(self, a, n, inverse=False):
        a = np.array(a, dtype=np.complex128, copy=True).reshape(-1)
        nn = _n(n)
        fn = self.lib.seso_ifft3d if inverse else self.lib.seso_fft3d
        if fn(a.ctypes.data_as(_dp), _nptr(nn)) != 0:
            raise ValueError("unsupported FFT length")
        return a

    def dft_naive(self, a, inverse=False):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        out = np.empty_like(a)
        self.lib.seso_dft_naive(a.ctypes.data_as(_dp), out.ctypes.data_as(_dp), a.size,
                                1 if inverse else 0)
        return out

    def twiddles(self, n):
        w = np.empty(n // 2, dtype=np.complex128)
        self.lib.seso_fft_twiddles(n, w.ctypes.data_as(_dp))
        return w

    def wavenumbers(self, xmin, xmax, n):
        k = np.empty(n)
        self.lib.seso_wavenumbers(xmin, xmax, n, _d(k))
        return k

    # ---- tables / steps ----
    def tables3d(self, box, n, V, dt, mass=1.0):
        b, nn = _box(box), _n(n)
        N = _total(nn)
        V = np.ascontiguousarray(V, dtype=np.float64)
        half = np.empty(N, dtype=np.complex128)
        kin = np.empty(N, dtype=np.complex128)
        self.lib.seso_tables3d(_d(b), _nptr(nn), _d(V), dt, mass, half.ctypes.data_as(_dp),
                               kin.ctypes.data_as(_dp))
        return half, kin

    def step3d(self, box, n, V, dt, psi, nsteps, mass=1.0, mask=None):
        b, nn = _box(box), _n(n)
        V = np.ascontiguousarray(V, dtype=np.float64)
        psi = np.array(psi, dtype=np.complex128, copy=True).reshape(-1)
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
        rc = self.lib.seso_step3d(_d(b), _nptr(nn), _d(V), dt, mass, _d(m),
                                  psi.ctypes.data_as(_dp), nsteps)
        if rc != 0:
            raise ValueError("unsupported grid")
        return psi

    def step1d(self, xmin, xmax, n, V, dt, psi, nsteps, mask=None):
        V = np.ascontiguousarray(V, dtype=np.float64)
        psi = np.array(psi, dtype=np.complex128, copy=True)
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
        if self.lib.seso_step1d(xmin, xmax, n, _d(V), dt, _d(m), psi.ctypes.data_as(_dp),
                                nsteps) != 0:
            raise ValueError("unsupported grid")
        return psi

    def driven_step3d(self, box, n, V, dt, psi, nsteps, axis, amplitude, omega, t0=0.0, mass=1.0):
        """drive.ixx:50-65: kick(t) . Strang step . kick(t + dt), no mask."""
        b, nn = _box(box), _n(n)
        V = np.ascontiguousarray(V, dtype=np.float64)
        psi = np.array(psi, dtype=np.complex128, copy=True).reshape(-1)
        ax = np.ascontiguousarray(axis, dtype=np.float64)
        if self.lib.seso_driven_step3d(_d(b), _nptr(nn), _d(V), dt, mass, _d(ax), amplitude, omega, t0,
                                       psi.ctypes.data_as(_dp), nsteps) != 0:
            raise ValueError("unsupported grid")
        return psi

    def relax3d(self, box, n, V, dtau, psi, nsteps, mass=1.0):
        b, nn = _box(box), _n(n)
        V = np.ascontiguousarray(V, dtype=np.float64)
        psi = np.array(psi, dtype=np.complex128, copy=True).reshape(-1)
        if self.lib.seso_relax3d(_d(b), _nptr(nn), _d(V), dtau, mass, psi.ctypes.data_as(_dp),
                                 nsteps) != 0:
            raise ValueError("unsupported grid")
        return psi

    # ---- builders ----
    def _grid_out(self, fn, box, n, *args):
        b, nn = _box(box), _n(n)
        out = np.empty(_total(nn))
        fn(_d(b), _nptr(nn), *args, _d(out))
        return out

    def harmonic3d(self, box, n, omega, c=(0.0, 0.0, 0.0)):
        return self._grid_out(self.lib.seso_harmonic3d, box, n, omega, _d(_box(c)))

    def soft_coulomb3d(self, box, n, Z, a, c=(0.0, 0.0, 0.0)):
        return self._grid_out(self.lib.seso_soft_coulomb3d, box, n, Z, a, _d(_box(c)))

    def regularized_coulomb3d(self, box, n, Z, c=(0.0, 0.0, 0.0)):
        return self._grid_out(self.lib.seso_regularized_coulomb3d, box, n, Z, _d(_box(c)))

    def barrier3d(self, box, n, v0, xlo, xhi):
        return self._grid_out(self.lib.seso_barrier3d, box, n, v0, xlo, xhi)

    def stadium3d(self, box, n, half_len, r, v_out):
        return self._grid_out(self.lib.seso_stadium3d, box, n, half_len, r, v_out)

    def stark_fold3d(self, box, n, e, V):
        V = np.array(V, dtype=np.float64, copy=True)
        b, nn = _box(box), _n(n)
        self.lib.seso_stark_fold3d(_d(b), _nptr(nn), e, _d(V))
        return V

    def mask3d(self, box, n, width, profile=1):
        return self._grid_out(self.lib.seso_mask3d, box, n, width, profile)

    def mask1d(self, xmin, xmax, n, width, profile=1):
        out = np.empty(n)
        self.lib.seso_mask1d(xmin, xmax, n, width, profile, _d(out))
        return out

    def harmonic1d(self, xmin, xmax, n, omega, x0=0.0):
        out = np.empty(n)
        self.lib.seso_harmonic1d(xmin, xmax, n, omega, x0, _d(out))
        return out

    def morse1d(self, xmin, xmax, n, d, alpha, x0):
        out = np.empty(n)
        self.lib.seso_morse1d(xmin, xmax, n, d, alpha, x0, _d(out))
        return out

    def double_well1d(self, xmin, xmax, n, vb, a):
        out = np.empty(n)
        self.lib.seso_double_well1d(xmin, xmax, n, vb, a, _d(out))
        return out

    def poschl_teller1d(self, xmin, xmax, n, v0, a, x0=0.0):
        out = np.empty(n)
        self.lib.seso_poschl_teller1d(xmin, xmax, n, v0, a, x0, _d(out))
        return out

    def gaussian3d(self, box, n, r0, sigma, k0):
        b, nn = _box(box), _n(n)
        out = np.empty(_total(nn), dtype=np.complex128)
        self.lib.seso_gaussian3d(_d(b), _nptr(nn), _d(_box(r0)), _d(_box(sigma)), _d(_box(k0)),
                                 out.ctypes.data_as(_dp))
        return out

    def gaussian1d(self, xmin, xmax, n, x0, sigma, k0):
        out = np.empty(n, dtype=np.complex128)
        self.lib.seso_gaussian1d(xmin, xmax, n, x0, sigma, k0, out.ctypes.data_as(_dp))
        return out

    # ---- observables ----
    def norm3d(self, box, n, psi):
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        return self.lib.seso_norm3d(_d(_box(box)), _nptr(_n(n)), psi.ctypes.data_as(_dp))

    def norm1d(self, xmin, xmax, n, psi):
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        return self.lib.seso_norm1d(xmin, xmax, n, psi.ctypes.data_as(_dp))

    def mean_energy3d(self, box, n, psi, V, mass=1.0):
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        V = np.ascontiguousarray(V, dtype=np.float64)
        return self.lib.seso_mean_energy3d(_d(_box(box)), _nptr(_n(n)), psi.ctypes.data_as(_dp),
                                           _d(V), mass)

    def mean_energy1d(self, xmin, xmax, n, psi, V):
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        V = np.ascontiguousarray(V, dtype=np.float64)
        return self.lib.seso_mean_energy1d(xmin, xmax, n, psi.ctypes.data_as(_dp), _d(V))

    def prob_x_range3d(self, box, n, psi, a, b):
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        return self.lib.seso_prob_x_range3d(_d(_box(box)), _nptr(_n(n)), psi.ctypes.data_as(_dp),
                                            a, b)

    def _vec3(self, fn, box, n, psi):
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        out = np.empty(3)
        fn(_d(_box(box)), _nptr(_n(n)), psi.ctypes.data_as(_dp), _d(out))
        return out

    def mean_position3d(self, box, n, psi):
        return self._vec3(self.lib.seso_mean_position3d, box, n, psi)

    def sigma_position3d(self, box, n, psi):
        return self._vec3(self.lib.seso_sigma_position3d, box, n, psi)

    def mean_momentum3d(self, box, n, psi):
        return self._vec3(self.lib.seso_mean_momentum3d, box, n, psi)


class Reference:
    """The reference's own core (oracle/_ref/libsesref.so), when it was built."""

    @staticmethod
    def available() -> bool:
        return REF_SO.exists()

    def __init__(self, path: Path | str = REF_SO, workers: int | None = None):
        if workers is not None:
            os.environ["SES_PARALLEL_WORKERS"] = str(workers)
        self.lib = L = C.CDLL(str(path))
        vp = C.c_void_p
        L.sesref_workers.restype = C.c_int
        L.sesref_fft1d.argtypes = [_dp, C.c_size_t, C.c_int]
        L.sesref_fft1d.restype = C.c_int
        L.sesref_fft3d.argtypes = [_dp, _ip, C.c_int]
        L.sesref_fft3d.restype = C.c_int
        L.sesref_fft_twiddles.argtypes = [C.c_size_t, _dp]
        L.sesref_wavenumbers.argtypes = [C.c_double, C.c_double, C.c_int, _dp]
        L.sesref_harmonic3d.argtypes = [_dp, _ip, C.c_double, _dp, _dp]
        L.sesref_soft_coulomb3d.argtypes = [_dp, _ip, C.c_double, C.c_double, _dp, _dp]
        L.sesref_regularized_coulomb3d.argtypes = [_dp, _ip, C.c_double, _dp, _dp]
        L.sesref_barrier3d.argtypes = [_dp, _ip, C.c_double, C.c_double, C.c_double, _dp]
        L.sesref_absorbing_mask3d.argtypes = [_dp, _ip, C.c_double, _dp]
        L.sesref_absorbing_mask1d.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double, _dp]
        L.sesref_harmonic1d.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double, C.c_double,
                                        _dp]
        L.sesref_morse1d.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double, C.c_double,
                                     C.c_double, _dp]
        L.sesref_double_well1d.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double,
                                           C.c_double, _dp]
        L.sesref_poschl_teller1d.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double,
                                             C.c_double, C.c_double, _dp]
        L.sesref_barrier1d.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double, C.c_double,
                                       C.c_double, _dp]
        L.sesref_gaussian3d.argtypes = [_dp, _ip, _dp, _dp, _dp, _dp]
        L.sesref_gaussian1d.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double, C.c_double,
                                        C.c_double, _dp]
        L.sesref_split3d_new.argtypes = [_dp, _ip, _dp, C.c_double, C.c_double]
        L.sesref_split3d_new.restype = vp
        L.sesref_split3d_free.argtypes = [vp]
        L.sesref_split3d_tables.argtypes = [vp, _dp, _dp]
        L.sesref_field3d_new.argtypes = [_dp, _ip]
        L.sesref_field3d_new.restype = vp
        L.sesref_field3d_free.argtypes = [vp]
        L.sesref_field3d_set.argtypes = [vp, _dp]
        L.sesref_field3d_get.argtypes = [vp, _dp]
        L.sesref_split3d_step.argtypes = [vp, vp, C.c_int, _dp]
        L.sesref_norm3d.argtypes = [vp]
        L.sesref_norm3d.restype = C.c_double
        L.sesref_mean_energy3d.argtypes = [vp, _dp, C.c_double]
        L.sesref_mean_energy3d.restype = C.c_double
        for name in ["sesref_mean_position3d", "sesref_sigma_position3d",
                     "sesref_mean_momentum3d"]:
            getattr(L, name).argtypes = [vp, _dp]
        L.sesref_split1d_new.argtypes = [C.c_double, C.c_double, C.c_int, _dp, C.c_double]
        L.sesref_split1d_new.restype = vp
        L.sesref_split1d_free.argtypes = [vp]
        L.sesref_split1d_step.argtypes = [vp, _dp, C.c_int, _dp]
        for name in ["sesref_norm1d", "sesref_mean_position1d", "sesref_sigma_x1d",
                     "sesref_mean_momentum1d"]:
            getattr(L, name).argtypes = [C.c_double, C.c_double, C.c_int, _dp]
            getattr(L, name).restype = C.c_double
        L.sesref_mean_energy1d.argtypes = [C.c_double, C.c_double, C.c_int, _dp, _dp]
        L.sesref_mean_energy1d.restype = C.c_double
        L.sesref_probability_in_range1d.argtypes = [C.c_double, C.c_double, C.c_int, _dp,
                                                    C.c_double, C.c_double]
        L.sesref_probability_in_range1d.restype = C.c_double
        L.sesref_relax3d.argtypes = [_dp, _ip, _dp, C.c_double, C.c_double, _dp, C.c_int]
        L.sesref_driven_step3d.argtypes = [C.c_void_p, C.c_void_p, _dp, C.c_double, C.c_double, C.c_double,
                                           C.c_int]

    def workers(self) -> int:
        return self.lib.sesref_workers()

    def fft1d(self, a, inverse=False):
        a = np.array(a, dtype=np.complex128, copy=True)
        if self.lib.sesref_fft1d(a.ctypes.data_as(_dp), a.size, 1 if inverse else 0) != 0:
            raise ValueError("reference fft rejected the length")
        return a

    def fft3d(self, a, n, inverse=False):
        a = np.array(a, dtype=np.complex128, copy=True).reshape(-1)
        if self.lib.sesref_fft3d(a.ctypes.data_as(_dp), _nptr(_n(n)), 1 if inverse else 0) != 0:
            raise ValueError("reference fft rejected the length")
        return a

    def twiddles(self, n):
        w = np.empty(n // 2, dtype=np.complex128)
        self.lib.sesref_fft_twiddles(n, w.ctypes.data_as(_dp))
        return w

    def wavenumbers(self, xmin, xmax, n):
        k = np.empty(n)
        self.lib.sesref_wavenumbers(xmin, xmax, n, _d(k))
        return k

    def _grid_out(self, fn, box, n, *args):
        b, nn = _box(box), _n(n)
        out = np.empty(_total(nn))
        fn(_d(b), _nptr(nn), *args, _d(out))
        return out

    def harmonic3d(self, box, n, omega, c=(0.0, 0.0, 0.0)):
        return self._grid_out(self.lib.sesref_harmonic3d, box, n, omega, _d(_box(c)))

    def soft_coulomb3d(self, box, n, Z, a, c=(0.0, 0.0, 0.0)):
        return self._grid_out(self.lib.sesref_soft_coulomb3d, box, n, Z, a, _d(_box(c)))

    def regularized_coulomb3d(self, box, n, Z, c=(0.0, 0.0, 0.0)):
        return self._grid_out(self.lib.sesref_regularized_coulomb3d, box, n, Z, _d(_box(c)))

    def barrier3d(self, box, n, v0, xlo, xhi):
        return self._grid_out(self.lib.sesref_barrier3d, box, n, v0, xlo, xhi)

    def absorbing_mask3d(self, box, n, width):
        return self._grid_out(self.lib.sesref_absorbing_mask3d, box, n, width)

    def absorbing_mask1d(self, xmin, xmax, n, width):
        out = np.empty(n)
        self.lib.sesref_absorbing_mask1d(xmin, xmax, n, width, _d(out))
        return out

    def harmonic1d(self, xmin, xmax, n, omega, x0=0.0):
        out = np.empty(n)
        self.lib.sesref_harmonic1d(xmin, xmax, n, omega, x0, _d(out))
        return out

    def morse1d(self, xmin, xmax, n, d, alpha, x0):
        out = np.empty(n)
        self.lib.sesref_morse1d(xmin, xmax, n, d, alpha, x0, _d(out))
        return out

    def double_well1d(self, xmin, xmax, n, vb, a):
        out = np.empty(n)
        self.lib.sesref_double_well1d(xmin, xmax, n, vb, a, _d(out))
        return out

    def poschl_teller1d(self, xmin, xmax, n, v0, a, x0=0.0):
        out = np.empty(n)
        self.lib.sesref_poschl_teller1d(xmin, xmax, n, v0, a, x0, _d(out))
        return out

    def gaussian3d(self, box, n, r0, sigma, k0):
        b, nn = _box(box), _n(n)
        out = np.empty(_total(nn), dtype=np.complex128)
        self.lib.sesref_gaussian3d(_d(b), _nptr(nn), _d(_box(r0)), _d(_box(sigma)),
                                   _d(_box(k0)), out.ctypes.data_as(_dp))
        return out

    def gaussian1d(self, xmin, xmax, n, x0, sigma, k0):
        out = np.empty(n, dtype=np.complex128)
        self.lib.sesref_gaussian1d(xmin, xmax, n, x0, sigma, k0, out.ctypes.data_as(_dp))
        return out

    def tables3d(self, box, n, V, dt, mass=1.0):
        b, nn = _box(box), _n(n)
        N = _total(nn)
        V = np.ascontiguousarray(V, dtype=np.float64)
        h = self.lib.sesref_split3d_new(_d(b), _nptr(nn), _d(V), dt, mass)
        half = np.empty(N, dtype=np.complex128)
        kin = np.empty(N, dtype=np.complex128)
        self.lib.sesref_split3d_tables(h, half.ctypes.data_as(_dp), kin.ctypes.data_as(_dp))
        self.lib.sesref_split3d_free(h)
        return half, kin

    def split3d(self, box, n, V, dt, mass=1.0):
        return RefSplit3D(self, box, n, V, dt, mass)

    def step3d(self, box, n, V, dt, psi, nsteps, mass=1.0, mask=None):
        s = self.split3d(box, n, V, dt, mass)
        try:
            s.set_psi(psi)
            s.step(nsteps, mask)
            return s.get_psi()
        finally:
            s.close()

    def step1d(self, xmin, xmax, n, V, dt, psi, nsteps, mask=None):
        V = np.ascontiguousarray(V, dtype=np.float64)
        psi = np.array(psi, dtype=np.complex128, copy=True)
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
        h = self.lib.sesref_split1d_new(xmin, xmax, n, _d(V), dt)
        self.lib.sesref_split1d_step(h, psi.ctypes.data_as(_dp), nsteps, _d(m))
        self.lib.sesref_split1d_free(h)
        return psi

    def relax3d(self, box, n, V, dtau, psi, nsteps, mass=1.0):
        psi = np.array(psi, dtype=np.complex128, copy=True).reshape(-1)
        V = np.ascontiguousarray(V, dtype=np.float64)
        self.lib.sesref_relax3d(_d(_box(box)), _nptr(_n(n)), _d(V), dtau, mass,
                                psi.ctypes.data_as(_dp), nsteps)
        return psi

    def norm1d(self, xmin, xmax, n, psi):
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        return self.lib.sesref_norm1d(xmin, xmax, n, psi.ctypes.data_as(_dp))

    def mean_energy1d(self, xmin, xmax, n, psi, V):
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        V = np.ascontiguousarray(V, dtype=np.float64)
        return self.lib.sesref_mean_energy1d(xmin, xmax, n, psi.ctypes.data_as(_dp), _d(V))

    def probability_in_range1d(self, xmin, xmax, n, psi, a, b):
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        return self.lib.sesref_probability_in_range1d(xmin, xmax, n, psi.ctypes.data_as(_dp), a, b)


class RefSplit3D:
    """Reference SplitOperator3D + a resident Field3D (for timing the CPU arm)."""

    def __init__(self, ref: Reference, box, n, V, dt, mass=1.0):
        self.ref = ref
        L = ref.lib
        self.n = _n(n)
        self.box = _box(box)
        V = np.ascontiguousarray(V, dtype=np.float64)
        self.h = L.sesref_split3d_new(_d(self.box), _nptr(self.n), _d(V), dt, mass)
        self.f = L.sesref_field3d_new(_d(self.box), _nptr(self.n))
        self.N = _total(self.n)

    def set_psi(self, psi):
        psi = np.ascontiguousarray(psi, dtype=np.complex128).reshape(-1)
        self.ref.lib.sesref_field3d_set(self.f, psi.ctypes.data_as(_dp))

    def get_psi(self):
        out = np.empty(self.N, dtype=np.complex128)
        self.ref.lib.sesref_field3d_get(self.f, out.ctypes.data_as(_dp))
        return out

    def step(self, nsteps, mask=None):
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
        self.ref.lib.sesref_split3d_step(self.h, self.f, nsteps, _d(m))

    def driven_step(self, nsteps, axis, amplitude, omega, t0=0.0):
        ax = np.ascontiguousarray(axis, dtype=np.float64)
        self.ref.lib.sesref_driven_step3d(self.h, self.f, _d(ax), amplitude, omega, t0, nsteps)

    def norm(self):
        return self.ref.lib.sesref_norm3d(self.f)

    def mean_energy(self, V, mass=1.0):
        V = np.ascontiguousarray(V, dtype=np.float64)
        return self.ref.lib.sesref_mean_energy3d(self.f, _d(V), mass)

    def close(self):
        if self.h:
            self.ref.lib.sesref_split3d_free(self.h)
            self.ref.lib.sesref_field3d_free(self.f)
            self.h = self.f = None
