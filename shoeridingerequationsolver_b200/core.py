"""Host-side mirror of the reference core's split-operator call surface.

Same names, argument meaning and error behaviour as the reference's C++
modules (parkyere/ShoeridingerEquationSolver core/src/), backed by the B200
library through its C ABI:

* ``Grid1D`` / ``Grid3D``          -- core/src/grid.ixx:10-30
* ``Field1D`` / ``Field3D``        -- core/src/field.ixx:11-66 (numpy complex128 data)
* ``wavenumbers``                  -- core/src/spectral.ixx:14-23
* ``fft`` / ``ifft``               -- core/src/fft.ixx:75-188
* ``SplitOperator3D``              -- core/src/propagator.ixx:68-134, plus the resident
                                      engine calls of solver/src/vk_engine.ixx
                                      (upload_state, step(n, absorb), set_absorber,
                                      readback, norm/energy readouts)
* ``SplitOperator1D``              -- core/src/propagator.ixx:21-66

Sizes that are not 2^a 3^b 5^c raise ``ValueError`` (the reference raises
std::invalid_argument for non-powers of two).
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import check, lib

_dp = C.POINTER(C.c_double)

PRECISIONS = {"c128": _abi.SES_C128, "c64": _abi.SES_C64}


@dataclass(frozen=True)
class Grid1D:
    xmin: float
    xmax: float
    n: int

    def size(self) -> int:
        return self.n

    def spacing(self) -> float:
        return (self.xmax - self.xmin) / self.n

    def coord(self, i: int) -> float:
        return self.xmin + i * self.spacing()

    def coords(self) -> np.ndarray:
        return self.xmin + np.arange(self.n) * self.spacing()


@dataclass(frozen=True)
class Grid3D:
    x: Grid1D
    y: Grid1D
    z: Grid1D

    def size(self) -> int:
        return self.x.n * self.y.n * self.z.n

    def flat(self, i: int, j: int, k: int) -> int:
        return i + self.x.n * (j + self.y.n * k)

    def cell_volume(self) -> float:
        return self.x.spacing() * self.y.spacing() * self.z.spacing()

    @property
    def shape(self) -> tuple[int, int, int]:
        """numpy C-order shape (nz, ny, nx) of the x-fastest flat layout."""
        return (self.z.n, self.y.n, self.x.n)

    @property
    def box(self) -> tuple[float, ...]:
        return (self.x.xmin, self.x.xmax, self.y.xmin, self.y.xmax, self.z.xmin, self.z.xmax)

    @property
    def dims(self) -> tuple[int, int, int]:
        return (self.x.n, self.y.n, self.z.n)


def line_grid(g: Grid1D) -> Grid3D:
    """A 1D grid as Grid3D (n x 1 x 1) with unit-length collapsed axes."""
    return Grid3D(g, Grid1D(0.0, 1.0, 1), Grid1D(0.0, 1.0, 1))


class Field3D:
    def __init__(self, grid: Grid3D, data=None):
        self.grid = grid
        if data is None:
            self.data = np.zeros(grid.size(), dtype=np.complex128)
        else:  # owns its values, like the reference's std::vector (field.ixx:52-66)
            self.data = np.array(data, dtype=np.complex128, copy=True).reshape(-1)
            if self.data.size != grid.size():
                raise ValueError("field size does not match the grid")

    def size(self) -> int:
        return self.grid.size()

    def __call__(self, i: int, j: int, k: int) -> complex:
        return self.data[self.grid.flat(i, j, k)]


class Field1D:
    def __init__(self, grid: Grid1D, data=None):
        self.grid = grid
        self.data = (np.zeros(grid.n, dtype=np.complex128) if data is None else
                     np.array(data, dtype=np.complex128, copy=True).reshape(-1))
        if self.data.size != grid.n:
            raise ValueError("field size does not match the grid")

    def size(self) -> int:
        return self.grid.n

    def __getitem__(self, i):
        return self.data[i]


def wavenumbers(g: Grid1D) -> np.ndarray:
    """fftfreq layout: k_j = (2 pi/L) * (j if 2j < n else j - n)."""
    dk = 2.0 * math.pi / (g.xmax - g.xmin)
    j = np.arange(g.n)
    return dk * np.where(2 * j < g.n, j, j - g.n).astype(np.float64)


def norm_sq(f) -> float:
    """sum |psi|^2 times the cell volume (field.ixx:30-36, 68-74)."""
    if isinstance(f, Field1D):
        return float(np.sum(np.abs(f.data) ** 2) * f.grid.spacing())
    return float(np.sum(np.abs(f.data) ** 2) * f.grid.cell_volume())


def _fft_host(data: np.ndarray, dims, inverse: bool, precision: str) -> None:
    n = (C.c_int32 * 3)(*dims)
    check(lib.ses_fft3_host(n, PRECISIONS[precision], data.ctypes.data_as(_dp), 1 if inverse else 0))


def _transform(x, inverse: bool, precision: str):
    if isinstance(x, Field3D):
        _fft_host(x.data, x.grid.dims, inverse, precision)
        return x
    if isinstance(x, Field1D):
        _fft_host(x.data, (x.grid.n, 1, 1), inverse, precision)
        return x
    a = np.ascontiguousarray(np.asarray(x, dtype=np.complex128))
    if a.ndim == 1:
        dims = (a.size, 1, 1)
    elif a.ndim == 3:
        dims = (a.shape[2], a.shape[1], a.shape[0])
    else:
        raise ValueError("expected a 1D line or a (nz, ny, nx) array")
    out = a.copy()
    _fft_host(out.reshape(-1), dims, inverse, precision)
    return out


def fft(x, precision: str = "c128"):
    """Forward unnormalised FFT (fft.ixx:14-18): Field3D/Field1D in place, arrays by copy."""
    return _transform(x, False, precision)


def ifft(x, precision: str = "c128"):
    """Inverse FFT with 1/N (fft.ixx:89-98, 177-188)."""
    return _transform(x, True, precision)


class SplitOperator3D:
    """Strang split-operator propagator on the B200 (propagator.ixx:68-134).

    ``step(psi, nsteps)`` keeps the reference's in-place semantics on a
    caller-owned Field3D (upload, nsteps Strang steps, readback).  The
    engine-style calls (``upload_state`` / ``advance`` / ``readback`` /
    ``observe``) keep psi resident in HBM between calls.
    """

    def __init__(self, grid: Grid3D, potential, dt: float, mass: float = 1.0,
                 precision: str = "c128", psi0=None):
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {list(PRECISIONS)}")
        self.grid = grid
        self.precision = precision
        self.mass = mass
        self._dt = float(dt)
        v = np.ascontiguousarray(np.asarray(potential, dtype=np.float64).reshape(-1))
        if v.size != grid.size():
            raise ValueError("potential size does not match the grid")
        p0 = None
        if psi0 is not None:
            p0 = np.ascontiguousarray(np.asarray(psi0, dtype=np.complex128).reshape(-1))
            if p0.size != grid.size():
                raise ValueError("psi0 size does not match the grid")
        h = C.c_void_p()
        desc = _abi.grid_desc(grid)
        check(lib.ses_gpu_create(C.byref(desc), PRECISIONS[precision], self._dt, float(mass),
                                 v.ctypes.data_as(_dp),
                                 p0.ctypes.data_as(_dp) if p0 is not None else None, C.byref(h)))
        self._h = h

    # ---- reference surface ----
    def dt(self) -> float:
        return self._dt

    def half_potential_phase(self) -> np.ndarray:
        out = np.empty(self.grid.size(), dtype=np.complex128)
        check(lib.ses_gpu_tables(self._h, out.ctypes.data_as(_dp), None))
        return out

    def kinetic_phase(self) -> np.ndarray:
        out = np.empty(self.grid.size(), dtype=np.complex128)
        check(lib.ses_gpu_tables(self._h, None, out.ctypes.data_as(_dp)))
        return out

    def step(self, psi: Field3D, nsteps: int = 1) -> None:
        if psi.data.size != self.grid.size():
            raise ValueError("field size does not match the propagator")
        self.upload_state(psi.data)
        self.advance(nsteps)
        self.readback(out=psi.data)

    # ---- resident engine surface ----
    @property
    def handle(self):
        return self._h

    def upload_state(self, psi) -> None:
        a = np.ascontiguousarray(np.asarray(psi, dtype=np.complex128).reshape(-1))
        if a.size != self.grid.size():
            raise ValueError("psi size does not match the grid")
        check(lib.ses_gpu_write_psi(self._h, a.ctypes.data))

    def write_ptr(self, host_ptr: int) -> None:
        """Upload from a raw host pointer to N interleaved complex128 values."""
        check(lib.ses_gpu_write_psi(self._h, C.c_void_p(host_ptr)))

    def read_ptr(self, host_ptr: int) -> None:
        check(lib.ses_gpu_read_psi(self._h, C.c_void_p(host_ptr)))

    def readback(self, out=None) -> np.ndarray:
        if out is None:
            out = np.empty(self.grid.size(), dtype=np.complex128)
        if not (out.flags.c_contiguous and out.dtype == np.complex128 and out.size == self.grid.size()):
            raise ValueError("readback target must be a contiguous complex128 array of N elements")
        check(lib.ses_gpu_read_psi(self._h, out.ctypes.data))
        return out

    def advance(self, nsteps: int, absorb: bool = False) -> None:
        check(lib.ses_gpu_step(self._h, int(nsteps), 1 if absorb else 0))

    def advance_driven(self, nsteps: int, axis, amplitude: float, omega: float, t0: float = 0.0,
                       absorb: bool = False) -> None:
        """Dipole-driven steps on the resident psi (drive.ixx:50-65): each step is
        kick(t) . step . kick(t + dt), kick phase amplitude cos(omega t) dt/2 (axis . r)."""
        ax = np.ascontiguousarray(np.asarray(axis, dtype=np.float64).reshape(3))
        check(lib.ses_gpu_step_driven(self._h, int(nsteps), 1 if absorb else 0, ax.ctypes.data_as(_dp),
                                      float(amplitude), float(omega), float(t0)))

    def snapshot(self, steps: int = 0) -> bytes:
        """psi snapshot: 128-byte header + psi in the handle's precision (no conversion)."""
        n = C.c_size_t()
        check(lib.ses_gpu_snapshot(self._h, int(steps), None, 0, C.byref(n)))
        buf = (C.c_char * n.value)()
        check(lib.ses_gpu_snapshot(self._h, int(steps), buf, n.value, C.byref(n)))
        return bytes(buf)

    def restore(self, snap: bytes) -> int:
        steps = C.c_int64()
        check(lib.ses_gpu_restore(self._h, snap, len(snap), C.byref(steps)))
        return steps.value

    def density_slice(self, axis: int, index: int) -> np.ndarray:
        dims = self.grid.dims
        shape = [dims[a] for a in range(3) if a != axis]
        out = np.empty(shape[0] * shape[1], dtype=np.float32)
        check(lib.ses_gpu_density_slice(self._h, int(axis), int(index), out.ctypes.data_as(C.POINTER(C.c_float))))
        return out.reshape(shape[1], shape[0])

    def set_absorber(self, mask) -> None:
        if mask is None:
            check(lib.ses_gpu_set_absorber(self._h, None))
            return
        m = np.ascontiguousarray(np.asarray(mask, dtype=np.float64).reshape(-1))
        if m.size != self.grid.size():
            raise ValueError("mask size does not match the grid")
        check(lib.ses_gpu_set_absorber(self._h, m.ctypes.data_as(_dp)))

    def set_absorber_separable(self, mx, my, mz) -> None:
        arrs = [np.ascontiguousarray(np.asarray(a, dtype=np.float64)) for a in (mx, my, mz)]
        for a, n in zip(arrs, self.grid.dims):
            if a.size != n:
                raise ValueError("mask profile size does not match its axis")
        check(lib.ses_gpu_set_absorber_separable(self._h, *[a.ctypes.data_as(_dp) for a in arrs]))

    def set_potential(self, potential) -> None:
        v = np.ascontiguousarray(np.asarray(potential, dtype=np.float64).reshape(-1))
        if v.size != self.grid.size():
            raise ValueError("potential size does not match the grid")
        check(lib.ses_gpu_set_potential(self._h, v.ctypes.data_as(_dp)))

    def fft3(self, inverse: bool = False) -> None:
        check(lib.ses_gpu_fft3(self._h, 1 if inverse else 0))

    def observe(self, xlo: float = -math.inf, xhi: float = math.inf) -> dict:
        o = _abi.Observables()
        check(lib.ses_gpu_observe(self._h, float(xlo), float(xhi), C.byref(o)))
        return o.as_dict()

    def sync(self, timeout_ms: int = 0) -> None:
        check(lib.ses_gpu_sync(self._h, int(timeout_ms)))

    def norm_and_peak(self) -> tuple[float, float]:
        """Engine::norm_and_peak (vk_engine.ixx:1665-1692): (sum |psi|^2 dV, max |psi|^2)."""
        nrm, peak = C.c_double(), C.c_double()
        check(lib.ses_gpu_norm_and_peak(self._h, C.byref(nrm), C.byref(peak)))
        return nrm.value, peak.value

    def scale(self, factor: float) -> None:
        """Engine::scale (vk_engine.ixx:2120-2133): psi <- factor * psi on the device."""
        check(lib.ses_gpu_scale(self._h, float(factor)))

    def prepare(self, absorb: bool = False) -> None:
        """Record the step graph now (not inside the first long advance)."""
        check(lib.ses_gpu_prepare(self._h, 1 if absorb else 0))

    def set_wait_limit(self, wait_cycles: int = 0, extra_tx_bytes: int = 0) -> None:
        """Failure-detection hook (ses_gpu_set_wait_limit): bound the pipelined passes'
        waits by wait_cycles SM cycles and, with extra_tx_bytes > 0, make every tile's
        wait run out; (0, 0) restores normal operation."""
        check(lib.ses_gpu_set_wait_limit(self._h, int(wait_cycles), int(extra_tx_bytes)))

    def set_stream(self, stream_ptr: int | None) -> None:
        check(lib.ses_gpu_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def psi_device(self) -> tuple[int, int]:
        p, b = C.c_void_p(), C.c_size_t()
        check(lib.ses_gpu_psi_device(self._h, C.byref(p), C.byref(b)))
        return p.value, b.value

    PASS_NAMES = ("x_mid", "y_fwd", "fused", "y_inv", "x_start", "x_end")

    def profile_step(self, nsteps: int, absorb: bool = False) -> dict:
        """Per-pass mean launch times (ms) of an nsteps batch (Engine::profile_step)."""
        out = (C.c_double * 8)()
        check(lib.ses_gpu_profile_step(self._h, int(nsteps), 1 if absorb else 0, out))
        d = {k: out[i] for i, k in enumerate(self.PASS_NAMES)}
        d["total_ms"] = out[6]
        d["launches"] = int(out[7])
        return d

    def autotune(self, save: bool = True) -> str:
        """Time the compiled tile variants of each axis pass and keep the fastest."""
        check(lib.ses_gpu_autotune(self._h, 1 if save else 0))
        return self.plan_info()

    def plan_info(self) -> str:
        buf = C.create_string_buffer(512)
        check(lib.ses_gpu_plan_info(self._h, buf, 512))
        return buf.value.decode()

    def footprint(self) -> int:
        b = C.c_size_t()
        check(lib.ses_gpu_footprint(self._h, C.byref(b)))
        return b.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            check(lib.ses_gpu_destroy(self._h))   # leaves its batch first
            self._h = None
            b = getattr(self, "_batch", None)
            if b is not None and self in b._members:
                b._members.remove(self)
            self._batch = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


@dataclass
class DipoleDrive:
    """Polarization axis (need not be unit: scales E0), amplitude E0, angular frequency (drive.ixx:19-23)."""
    axis: tuple
    amplitude: float
    omega: float


def driven_step(psi: Field3D, prop: "SplitOperator3D", d: DipoleDrive, t0: float, nsteps: int) -> None:
    """ses::driven_step (drive.ixx:50-65) on a caller-owned field: upload, nsteps driven steps, readback."""
    prop.upload_state(psi.data)
    prop.advance_driven(nsteps, d.axis, d.amplitude, d.omega, t0)
    prop.readback(out=psi.data)


class ImaginaryTimePropagator3D(SplitOperator3D):
    """Imaginary-time relaxation (core/src/imaginary_time.ixx:64-144) on the B200:
    the split-operator step with the real weights exp(-V dtau/2), exp(-k^2 dtau/(2m)),
    renormalised on the device.  ``relax(psi, nsteps)`` keeps the reference's in-place
    semantics on a Field3D; ``relax_resident`` works on the uploaded state and returns
    the energy estimate -ln(norm^2)/(2 r dtau)."""

    def __init__(self, grid: Grid3D, potential, dtau: float, mass: float = 1.0,
                 precision: str = "c128", psi0=None):
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {list(PRECISIONS)}")
        self.grid = grid
        self.precision = precision
        self.mass = mass
        self._dt = float(dtau)
        v = np.ascontiguousarray(np.asarray(potential, dtype=np.float64).reshape(-1))
        if v.size != grid.size():
            raise ValueError("potential size does not match the grid")
        p0 = None
        if psi0 is not None:
            p0 = np.ascontiguousarray(np.asarray(psi0, dtype=np.complex128).reshape(-1))
        h = C.c_void_p()
        desc = _abi.grid_desc(grid)
        check(lib.ses_gpu_create_imag(C.byref(desc), PRECISIONS[precision], self._dt, float(mass),
                                      v.ctypes.data_as(_dp), p0.ctypes.data_as(_dp) if p0 is not None else None,
                                      C.byref(h)))
        self._h = h

    def relax(self, psi: Field3D, nsteps: int, renorm_every: int = 1) -> float:
        if psi.data.size != self.grid.size():
            raise ValueError("field size does not match the propagator")
        self.upload_state(psi.data)
        e = self.relax_resident(nsteps, renorm_every)
        self.readback(out=psi.data)
        return e

    def relax_resident(self, nsteps: int, renorm_every: int = 1) -> float:
        e = C.c_double()
        check(lib.ses_gpu_relax(self._h, int(nsteps), int(renorm_every), C.byref(e)))
        return e.value


def gaussian_wavepacket(grid: Grid3D, r0, sigma, k0) -> Field3D:
    """gaussian_wavepacket(Grid3D, r0, sigma, k0) (core/src/wavepacket.ixx:29-49):
    per-axis envelope (2 pi s^2)^(-1/4) exp(-(u - u0)^2 / (4 s^2)) times
    e^{i k0 . r}, normalised to norm_sq = 1 on the grid."""
    def env(u, u0, s):
        return math.pow(2.0 * math.pi * s * s, -0.25) * np.exp(-(u - u0) * (u - u0) / (4.0 * s * s))
    x = grid.x.coords()[None, None, :]
    y = grid.y.coords()[None, :, None]
    z = grid.z.coords()[:, None, None]
    amp = env(x, r0[0], sigma[0]) * env(y, r0[1], sigma[1]) * env(z, r0[2], sigma[2])
    ph = k0[0] * x + k0[1] * y + k0[2] * z
    psi = (amp * np.cos(ph) + 1j * (amp * np.sin(ph))).reshape(-1)
    n2 = float(np.sum(psi.real * psi.real + psi.imag * psi.imag)) * grid.cell_volume()
    if n2 > 0.0:
        psi = psi / math.sqrt(n2)
    return Field3D(grid, psi)


@dataclass
class SimulationConfig:
    """WavepacketSimulation::Config (core/src/simulation.ixx:24-31)."""
    grid: Grid3D
    potential: np.ndarray
    r0: tuple
    sigma: tuple
    k0: tuple
    dt: float


class WavepacketSimulation:
    """WavepacketSimulation (core/src/simulation.ixx:22-88) on the B200.

    The config builds the propagator tables (on the device) and psi0 =
    gaussian_wavepacket(grid, r0, sigma, k0); psi stays resident in HBM.
    ``advance(n)`` steps it there; ``psi()`` / ``density()`` read it back when it
    changed; ``set_psi`` uploads a field (the reference's hook for injecting a
    GPU-evolved field); ``relax(n, dtau)`` runs imaginary time on it.  The POVM
    ``measure`` of the reference is not part of the step and is not provided."""

    Config = SimulationConfig

    def __init__(self, cfg: SimulationConfig, precision: str = "c128"):
        self._grid = cfg.grid
        self._dt = float(cfg.dt)
        self._precision = precision
        self._potential = np.ascontiguousarray(np.asarray(cfg.potential, dtype=np.float64).reshape(-1))
        self._prop = SplitOperator3D(cfg.grid, self._potential, cfg.dt, precision=precision)
        self._psi = gaussian_wavepacket(cfg.grid, cfg.r0, cfg.sigma, cfg.k0)
        self._prop.upload_state(self._psi.data)
        self._stale = False
        self._steps = 0
        self._relaxer = None
        self._relaxer_dtau = 0.0

    def advance(self, nsteps: int) -> None:
        self._prop.advance(int(nsteps))
        self._steps += int(nsteps)
        self._stale = True

    def relax(self, nsteps: int, dtau: float) -> None:
        if self._relaxer is None or self._relaxer_dtau != dtau:
            if self._relaxer is not None:
                self._relaxer.close()
            self._relaxer = ImaginaryTimePropagator3D(self._grid, self._potential, dtau,
                                                      precision=self._precision)
            self._relaxer_dtau = dtau
        f = self.psi()
        self._relaxer.relax(f, int(nsteps))
        self._prop.upload_state(f.data)

    def time(self) -> float:
        return self._steps * self._dt

    def dt(self) -> float:
        return self._dt

    def grid(self) -> Grid3D:
        return self._grid

    def potential(self) -> np.ndarray:
        return self._potential

    def propagator(self) -> SplitOperator3D:
        return self._prop

    def psi(self) -> Field3D:
        if self._stale:
            self._prop.readback(out=self._psi.data)
            self._stale = False
        return self._psi

    def set_psi(self, psi: Field3D) -> None:
        data = psi.data if isinstance(psi, Field3D) else np.asarray(psi)
        if data.size != self._grid.size():
            raise ValueError("field size does not match the grid")
        self._psi = Field3D(self._grid, data)
        self._prop.upload_state(self._psi.data)
        self._stale = False

    def density(self) -> np.ndarray:
        """probability_density (core/src/field.ixx:100-106): |psi|^2 per cell."""
        d = self.psi().data
        return d.real * d.real + d.imag * d.imag

    def close(self) -> None:
        self._prop.close()
        if self._relaxer is not None:
            self._relaxer.close()
            self._relaxer = None


class SplitOperator1D:
    """1D Strang propagator (propagator.ixx:21-66): the 3D engine on n x 1 x 1."""

    def __init__(self, grid: Grid1D, potential, dt: float, precision: str = "c128"):
        self.grid = grid
        self._op = SplitOperator3D(line_grid(grid), potential, dt, 1.0, precision)

    def dt(self) -> float:
        return self._op.dt()

    def step(self, psi: Field1D, nsteps: int = 1) -> None:
        if psi.data.size != self.grid.n:
            raise ValueError("field size does not match the propagator")
        self._op.upload_state(psi.data)
        self._op.advance(nsteps)
        self._op.readback(out=psi.data)

    @property
    def engine(self) -> SplitOperator3D:
        return self._op

    def close(self) -> None:
        self._op.close()


class Batch:
    """Many independent propagations advanced together (the reference batches
    sweeps on the CPU with parallel_for over instances, core/src/parallel.ixx:
    195-238).  Members are SplitOperator3D handles; members of one shape and
    precision share one launch per axis pass, classes of different shapes run
    concurrently."""

    def __init__(self, members=()):
        self._b = C.c_void_p()
        check(lib.ses_batch_create(C.byref(self._b)))
        self._members: list[SplitOperator3D] = []
        for m in members:
            self.add(m)

    def add(self, op: SplitOperator3D) -> None:
        check(lib.ses_batch_add(self._b, op.handle))
        self._members.append(op)
        op._batch = self

    def remove(self, op: SplitOperator3D) -> None:
        check(lib.ses_batch_remove(self._b, op.handle))
        self._members.remove(op)
        op._batch = None

    @property
    def members(self) -> list:
        return list(self._members)

    def step(self, nsteps: int, absorb: bool = False) -> None:
        check(lib.ses_batch_step(self._b, int(nsteps), 1 if absorb else 0))

    def prepare(self, absorb: bool = False) -> None:
        """Record every class's step graph now (ses_batch_prepare)."""
        check(lib.ses_batch_prepare(self._b, 1 if absorb else 0))

    def observe(self, xlo: float = -math.inf, xhi: float = math.inf) -> list[dict]:
        n = len(self._members)
        out = (_abi.Observables * max(n, 1))()
        check(lib.ses_batch_observe(self._b, float(xlo), float(xhi), out, n))
        return [out[i].as_dict() for i in range(n)]

    def sync(self, timeout_ms: int = 0) -> None:
        check(lib.ses_batch_sync(self._b, int(timeout_ms)))

    def run(self, nsteps: int, psi_in=None, psi_out=None, absorb: bool = False,
            xlo: float = -math.inf, xhi: float = math.inf, observe: bool = True,
            timeout_ms: int = 0):
        """One host round trip of every member (ses_batch_run): upload psi_in[i]
        (or skip where None), nsteps steps, observables, read back into psi_out[i].
        Entries are contiguous complex128 numpy arrays of the member's size or raw
        host addresses (ints) of such arrays; page-locked memory lets each class's
        transfers overlap the other classes' steps.  Returns the observables (a
        list of dicts, member order) or None."""
        n = len(self._members)

        def ptrs(seq, name):
            if seq is None:
                return None
            if len(seq) != n:
                raise ValueError(f"{name} needs one entry per member ({n})")
            arr = (C.POINTER(C.c_double) * max(n, 1))()
            for i, (x, op) in enumerate(zip(seq, self._members)):
                if x is None:
                    continue
                if isinstance(x, int):
                    addr = x
                else:
                    if not (isinstance(x, np.ndarray) and x.dtype == np.complex128 and x.flags.c_contiguous
                            and x.size == op.grid.size()):
                        raise ValueError(f"{name}[{i}] must be a contiguous complex128 array of the member's size")
                    if name == "psi_out" and not x.flags.writeable:
                        raise ValueError("psi_out arrays must be writeable")
                    addr = x.ctypes.data
                arr[i] = C.cast(C.c_void_p(addr), C.POINTER(C.c_double))
            return arr

        pin, pout = ptrs(psi_in, "psi_in"), ptrs(psi_out, "psi_out")
        out = (_abi.Observables * max(n, 1))() if observe else None
        check(lib.ses_batch_run(self._b, pin, int(nsteps), 1 if absorb else 0, float(xlo), float(xhi),
                                out, pout, n, int(timeout_ms)))
        return [out[i].as_dict() for i in range(n)] if observe else None

    def set_stream(self, stream_ptr: int | None) -> None:
        check(lib.ses_batch_set_stream(self._b, C.c_void_p(stream_ptr or 0)))

    def counts(self) -> tuple[int, int]:
        m, c = C.c_int(0), C.c_int(0)
        check(lib.ses_batch_members(self._b, C.byref(m), C.byref(c)))
        return m.value, c.value

    def profile(self, nsteps: int, absorb: bool = False) -> list[dict]:
        """Per class: mean ms per launch of each pass of an interior step."""
        _, ncls = self.counts()
        out = (C.c_double * (5 * max(ncls, 1)))()
        check(lib.ses_batch_profile(self._b, int(nsteps), 1 if absorb else 0, out, 5 * ncls))
        return [{"x_mid": out[5 * i], "mid": [out[5 * i + 1], out[5 * i + 2], out[5 * i + 3]],
                 "step": out[5 * i + 4]} for i in range(ncls)]

    def autotune(self, save: bool = True) -> str:
        """Pick the fastest kernel variant of every class pass (timed on scratch fields)."""
        check(lib.ses_batch_autotune(self._b, 1 if save else 0))
        return self.info()

    def info(self) -> str:
        buf = C.create_string_buffer(4096)
        check(lib.ses_batch_info(self._b, buf, 4096))
        return buf.value.decode()

    def close(self) -> None:
        if getattr(self, "_b", None):
            check(lib.ses_batch_destroy(self._b))
            self._b = None
            for op in self._members:
                op._batch = None
            self._members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
