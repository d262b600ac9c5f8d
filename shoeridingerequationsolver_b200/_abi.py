"""ctypes binding of the C ABI in include/ses_gpu.h (libses_b200.so).

The library is built in-tree (``python shoeridingerequationsolver_b200/build.py``)
and mapped on the first call that needs it (creating a handle, a batch, a
server, an FFT, a device count): importing the package to build host arrays
(``scenes``) does not map it.  There is no fallback: if the shared library is
missing or fails to load, that first call raises ``ImportError``.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libses_b200.so"

SES_OK, SES_EINVAL, SES_ENOMEM, SES_ETIMEDOUT, SES_EDEVICE, SES_EBUSY, SES_ENOTFOUND = range(7)
SES_C128, SES_C64 = 0, 1

# every symbol include/ses_gpu.h declares
EXPORTS = [
    "ses_version", "ses_last_error", "ses_device_count",
    "ses_gpu_create", "ses_gpu_destroy", "ses_gpu_set_potential", "ses_gpu_set_absorber",
    "ses_gpu_set_absorber_separable", "ses_gpu_step", "ses_gpu_fft3", "ses_gpu_tables",
    "ses_gpu_dt", "ses_gpu_observe", "ses_gpu_read_psi", "ses_gpu_write_psi", "ses_gpu_sync",
    "ses_gpu_set_stream", "ses_gpu_psi_device", "ses_gpu_footprint", "ses_fft3_host",
    "ses_gpu_profile_step", "ses_gpu_autotune", "ses_gpu_plan_info", "ses_observe_real_noalloc",
    "ses_batch_create", "ses_batch_destroy", "ses_batch_add", "ses_batch_remove", "ses_batch_step",
    "ses_batch_observe", "ses_batch_sync", "ses_batch_set_stream", "ses_batch_members",
    "ses_batch_profile", "ses_batch_autotune", "ses_batch_info",
    "ses_serve_open", "ses_serve_submit", "ses_serve_poll", "ses_serve_result", "ses_serve_cancel",
    "ses_serve_wait_idle", "ses_serve_stats", "ses_serve_close", "ses_gpu_create_imag", "ses_gpu_relax",
    "ses_gpu_step_driven", "ses_gpu_snapshot", "ses_gpu_restore", "ses_gpu_density_slice",
    "ses_batch_observe_some", "ses_batch_run", "ses_gpu_norm_and_peak", "ses_gpu_scale", "ses_gpu_prepare",
    "ses_batch_prepare", "ses_gpu_set_wait_limit", "ses_gpu_observe_async",
]


class Axis(C.Structure):
    _fields_ = [("xmin", C.c_double), ("xmax", C.c_double), ("n", C.c_int32)]


class GridDesc(C.Structure):
    _fields_ = [("x", Axis), ("y", Axis), ("z", Axis)]


class Observables(C.Structure):
    _fields_ = [("norm", C.c_double), ("energy", C.c_double), ("energy_v", C.c_double),
                ("energy_t", C.c_double), ("p_range", C.c_double),
                ("mean_pos", C.c_double * 3), ("sigma_pos", C.c_double * 3),
                ("mean_mom", C.c_double * 3)]

    def as_dict(self) -> dict:
        return {
            "norm": self.norm, "energy": self.energy, "energy_v": self.energy_v,
            "energy_t": self.energy_t, "p_range": self.p_range,
            "mean_pos": list(self.mean_pos), "sigma_pos": list(self.sigma_pos),
            "mean_mom": list(self.mean_mom),
        }


class Request(C.Structure):
    _fields_ = [("grid", GridDesc), ("prec", C.c_int), ("dt", C.c_double), ("mass", C.c_double),
                ("V", C.c_void_p), ("psi0", C.c_void_p), ("mask_x", C.c_void_p), ("mask_y", C.c_void_p),
                ("mask_z", C.c_void_p), ("nsteps", C.c_int32), ("observe_every", C.c_int32),
                ("xlo", C.c_double), ("xhi", C.c_double)]


class Record(C.Structure):
    _fields_ = [("id", C.c_int64), ("step", C.c_int32), ("final_record", C.c_int32), ("t_ms", C.c_double),
                ("obs", Observables)]


class ServeStats(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("submitted", "admitted", "completed", "cancelled", "failed",
                                          "queued", "running", "rounds")] + \
               [("bytes_in_use", C.c_size_t), ("budget", C.c_size_t), ("gridpt_steps", C.c_double),
                ("busy_ms", C.c_double), ("wall_ms", C.c_double), ("latency_p50_ms", C.c_double),
                ("latency_p99_ms", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_CANCELLED, REQ_FAILED = range(5)


class SesError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"ses status {status}: {msg}")
        self.status = status


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is not built; run python shoeridingerequationsolver_b200/build.py")
    lib = C.CDLL(str(LIB_PATH))
    dp, vp, hp = C.POINTER(C.c_double), C.c_void_p, C.c_void_p
    st = C.c_int
    sig = {
        "ses_version": ([], C.c_char_p),
        "ses_last_error": ([], C.c_char_p),
        "ses_device_count": ([C.POINTER(C.c_int)], st),
        "ses_gpu_create": ([C.POINTER(GridDesc), C.c_int, C.c_double, C.c_double, dp, dp,
                            C.POINTER(hp)], st),
        "ses_gpu_destroy": ([hp], st),
        "ses_gpu_create_imag": ([C.POINTER(GridDesc), C.c_int, C.c_double, C.c_double, dp, dp,
                                 C.POINTER(hp)], st),
        "ses_gpu_relax": ([hp, C.c_int, C.c_int, dp], st),
        "ses_gpu_step_driven": ([hp, C.c_int, C.c_int, dp, C.c_double, C.c_double, C.c_double], st),
        "ses_gpu_snapshot": ([hp, C.c_int64, vp, C.c_size_t, C.POINTER(C.c_size_t)], st),
        "ses_gpu_restore": ([hp, vp, C.c_size_t, C.POINTER(C.c_int64)], st),
        "ses_gpu_density_slice": ([hp, C.c_int, C.c_int, C.POINTER(C.c_float)], st),
        "ses_gpu_set_potential": ([hp, dp], st),
        "ses_gpu_set_absorber": ([hp, dp], st),
        "ses_gpu_set_absorber_separable": ([hp, dp, dp, dp], st),
        "ses_gpu_step": ([hp, C.c_int, C.c_int], st),
        "ses_gpu_fft3": ([hp, C.c_int], st),
        "ses_gpu_tables": ([hp, dp, dp], st),
        "ses_gpu_dt": ([hp, dp], st),
        "ses_gpu_observe": ([hp, C.c_double, C.c_double, C.POINTER(Observables)], st),
        "ses_gpu_read_psi": ([hp, vp], st),
        "ses_gpu_write_psi": ([hp, vp], st),
        "ses_gpu_sync": ([hp, C.c_int], st),
        "ses_gpu_set_stream": ([hp, vp], st),
        "ses_gpu_psi_device": ([hp, C.POINTER(vp), C.POINTER(C.c_size_t)], st),
        "ses_gpu_footprint": ([hp, C.POINTER(C.c_size_t)], st),
        "ses_gpu_norm_and_peak": ([hp, dp, dp], st),
        "ses_gpu_scale": ([hp, C.c_double], st),
        "ses_gpu_prepare": ([hp, C.c_int], st),
        "ses_batch_prepare": ([vp, C.c_int], st),
        "ses_gpu_set_wait_limit": ([hp, C.c_int64, C.c_uint32], st),
        "ses_gpu_observe_async": ([hp, C.c_double, C.c_double, C.POINTER(Observables)], st),
        "ses_fft3_host": ([C.POINTER(C.c_int32), C.c_int, dp, C.c_int], st),
        "ses_gpu_profile_step": ([hp, C.c_int, C.c_int, dp], st),
        "ses_gpu_autotune": ([hp, C.c_int], st),
        "ses_gpu_plan_info": ([hp, C.c_char_p, C.c_size_t], st),
        "ses_observe_real_noalloc": ([C.POINTER(GridDesc), C.c_int, vp, vp, C.c_double, C.c_double, vp,
                                      vp], st),
        "ses_batch_create": ([C.POINTER(vp)], st),
        "ses_batch_destroy": ([vp], st),
        "ses_batch_add": ([vp, hp], st),
        "ses_batch_remove": ([vp, hp], st),
        "ses_batch_step": ([vp, C.c_int, C.c_int], st),
        "ses_batch_observe": ([vp, C.c_double, C.c_double, C.POINTER(Observables), C.c_int], st),
        "ses_batch_sync": ([vp, C.c_int], st),
        "ses_batch_observe_some": ([vp, C.POINTER(hp), C.c_int, dp, dp, C.POINTER(Observables)], st),
        "ses_batch_run": ([vp, C.POINTER(dp), C.c_int, C.c_int, C.c_double, C.c_double, C.POINTER(Observables),
                           C.POINTER(dp), C.c_int, C.c_int], st),
        "ses_batch_set_stream": ([vp, vp], st),
        "ses_batch_members": ([vp, C.POINTER(C.c_int), C.POINTER(C.c_int)], st),
        "ses_batch_profile": ([vp, C.c_int, C.c_int, dp, C.c_int], st),
        "ses_batch_autotune": ([vp, C.c_int], st),
        "ses_batch_info": ([vp, C.c_char_p, C.c_size_t], st),
        "ses_serve_open": ([C.c_size_t, C.c_int, C.POINTER(vp)], st),
        "ses_serve_submit": ([vp, C.POINTER(Request), C.POINTER(C.c_int64)], st),
        "ses_serve_poll": ([vp, C.c_int64, C.POINTER(Record), C.c_int, C.POINTER(C.c_int),
                            C.POINTER(C.c_int)], st),
        "ses_serve_result": ([vp, C.c_int64, vp, dp], st),
        "ses_serve_cancel": ([vp, C.c_int64], st),
        "ses_serve_wait_idle": ([vp, C.c_int], st),
        "ses_serve_stats": ([vp, C.POINTER(ServeStats)], st),
        "ses_serve_close": ([vp], st),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


class _LazyLib:
    """Stands for the CDLL of libses_b200.so and maps it on first attribute use."""

    _cdll: C.CDLL | None = None

    def __getattr__(self, name):
        if _LazyLib._cdll is None:
            _LazyLib._cdll = _load()
        return getattr(_LazyLib._cdll, name)

    @staticmethod
    def loaded() -> bool:
        return _LazyLib._cdll is not None


lib = _LazyLib()


def ensure_loaded() -> None:
    """Map the library now (raises ImportError when it is not built)."""
    lib.ses_version  # noqa: B018  (attribute access maps the library)


def last_error() -> str:
    return lib.ses_last_error().decode()


def check(status: int) -> None:
    """Map a ses_status to the reference's error behaviour: invalid sizes raise
    ValueError (std::invalid_argument in core/src/fft.ixx:42-44), exhausted
    memory MemoryError, an expired bounded wait TimeoutError, device errors
    SesError."""
    if status == SES_OK:
        return
    msg = last_error()
    if status == SES_EINVAL:
        raise ValueError(msg)
    if status == SES_ENOMEM:
        raise MemoryError(msg)
    if status == SES_ETIMEDOUT:
        raise TimeoutError(msg)
    raise SesError(status, msg)


def grid_desc(grid) -> GridDesc:
    return GridDesc(Axis(grid.x.xmin, grid.x.xmax, grid.x.n), Axis(grid.y.xmin, grid.y.xmax, grid.y.n),
                    Axis(grid.z.xmin, grid.z.xmax, grid.z.n))


def device_count() -> int:
    c = C.c_int(0)
    st = lib.ses_device_count(C.byref(c))
    return c.value if st == SES_OK else 0
