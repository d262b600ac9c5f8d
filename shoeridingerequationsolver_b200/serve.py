"""Request server (ses_serve_* in include/ses_gpu.h): continuous batching of
independent solves on one GPU.

Requests carry their grid, potential, initial packet, dt, step count,
observation cadence and optional separable absorber.  The server admits them
against a device-memory budget, keeps each field resident as a member of one
batch, and advances all running requests together in rounds that end at the
next observation point or completion of any of them, so requests join and
leave between rounds.  Observations stream back as records.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _abi
from ._abi import check, lib
from .core import PRECISIONS, Grid3D

STATE_NAMES = {_abi.REQ_QUEUED: "queued", _abi.REQ_RUNNING: "running", _abi.REQ_DONE: "done",
               _abi.REQ_CANCELLED: "cancelled", _abi.REQ_FAILED: "failed"}


class Server:
    def __init__(self, budget_bytes: int = 150 * 10**9, max_round_steps: int = 100):
        self._s = C.c_void_p()
        check(lib.ses_serve_open(C.c_size_t(int(budget_bytes)), int(max_round_steps), C.byref(self._s)))
        self._dims: dict[int, int] = {}

    def submit(self, grid: Grid3D, V, psi0, dt: float, nsteps: int, observe_every: int = 100,
               mask=None, precision: str = "c64", mass: float = 1.0,
               x_range=(-math.inf, math.inf)) -> int:
        v = np.ascontiguousarray(np.asarray(V, dtype=np.float64).reshape(-1))
        p = np.ascontiguousarray(np.asarray(psi0, dtype=np.complex128).reshape(-1))
        if v.size != grid.size() or p.size != grid.size():
            raise ValueError("V and psi0 must have one value per grid point")
        masks = [None, None, None]
        if mask is not None:
            masks = [np.ascontiguousarray(np.asarray(m, dtype=np.float64)) for m in mask]
            for m, n in zip(masks, grid.dims):
                if m.size != n:
                    raise ValueError("absorber profile length does not match its axis")
        r = _abi.Request()
        r.grid = _abi.grid_desc(grid)
        r.prec = PRECISIONS[precision]
        r.dt, r.mass = float(dt), float(mass)
        r.V, r.psi0 = v.ctypes.data, p.ctypes.data
        r.mask_x, r.mask_y, r.mask_z = [m.ctypes.data if m is not None else None for m in masks]
        r.nsteps, r.observe_every = int(nsteps), int(observe_every)
        r.xlo, r.xhi = float(x_range[0]), float(x_range[1])
        rid = C.c_int64()
        check(lib.ses_serve_submit(self._s, C.byref(r), C.byref(rid)))   # arrays copied here
        self._dims[rid.value] = grid.size()
        return rid.value

    def poll(self, rid: int) -> tuple[str, list[dict]]:
        """(state, records not returned before)."""
        out = []
        state = C.c_int()
        buf = (_abi.Record * 64)()
        while True:
            n = C.c_int()
            check(lib.ses_serve_poll(self._s, int(rid), buf, 64, C.byref(n), C.byref(state)))
            for i in range(n.value):
                rec = buf[i]
                out.append({"id": rec.id, "step": rec.step, "final": bool(rec.final_record),
                            "t_ms": rec.t_ms, **rec.obs.as_dict()})
            if n.value < 64:
                return STATE_NAMES[state.value], out

    def result(self, rid: int, want_psi: bool = True) -> tuple[np.ndarray | None, float]:
        lat = C.c_double()
        psi = np.empty(self._dims[rid], dtype=np.complex128) if want_psi else None
        check(lib.ses_serve_result(self._s, int(rid), psi.ctypes.data if want_psi else None, C.byref(lat)))
        return psi, lat.value

    def cancel(self, rid: int) -> None:
        check(lib.ses_serve_cancel(self._s, int(rid)))

    def wait_idle(self, timeout_ms: int = 0) -> None:
        check(lib.ses_serve_wait_idle(self._s, int(timeout_ms)))

    def stats(self) -> dict:
        st = _abi.ServeStats()
        check(lib.ses_serve_stats(self._s, C.byref(st)))
        return st.as_dict()

    def close(self) -> None:
        if getattr(self, "_s", None):
            check(lib.ses_serve_close(self._s))
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
