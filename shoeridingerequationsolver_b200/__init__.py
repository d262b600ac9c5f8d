"""B200-native Strang split-operator TDSE step (drop-in for the reference core's
propagator / propagator-tables / fft3 surface).  The compute path is the
sm_100a library libses_b200.so behind the C ABI in include/ses_gpu.h."""

from .core import (Batch, DipoleDrive, Field1D, ImaginaryTimePropagator3D, driven_step, Field3D, Grid1D, Grid3D,
                   SplitOperator1D, SplitOperator3D, WavepacketSimulation, fft, gaussian_wavepacket, ifft, line_grid,
                   norm_sq, wavenumbers)
from ._abi import device_count, last_error, LIB_PATH
from .serve import Server

__all__ = ["Batch", "DipoleDrive", "driven_step", "Field1D", "ImaginaryTimePropagator3D", "Field3D", "Grid1D", "Grid3D", "SplitOperator1D", "SplitOperator3D", "fft",
           "ifft", "line_grid", "norm_sq", "wavenumbers", "WavepacketSimulation", "gaussian_wavepacket", "device_count", "last_error", "LIB_PATH", "Server"]
