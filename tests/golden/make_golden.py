"""Generate tests/golden/*.npz from the reference's own FP64 core.

Runs the reference (parkyere/ShoeridingerEquationSolver core/src, compiled by
oracle/build_ref.py into oracle/_ref/libsesref.so) on the inputs of its own
hot-path tests and GPU oracle checks, and stores inputs and outputs as small
fixtures so parity can be checked where the reference tree is absent.

Usage: python oracle/build_ref.py && python tests/golden/make_golden.py
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle.oracle import Reference  # noqa: E402


def deterministic_signal(n):
    x = np.arange(n, dtype=np.float64)
    return (np.sin(1.3 * x) + 0.1 * x) + 1j * (np.cos(2.7 * x) - 0.05 * x)


def main() -> int:
    if not Reference.available():
        print("reference core not built: run python oracle/build_ref.py first")
        return 1
    ref = Reference()
    out = {}

    # fft_test.cpp signals; fft3_test.cpp plane wave and signal
    for n in (1, 8, 16, 1024):
        s = deterministic_signal(n)
        out[f"fft1d_{n}_in"] = s
        out[f"fft1d_{n}_out"] = ref.fft1d(s)
        out[f"ifft1d_{n}_out"] = ref.fft1d(s, inverse=True)
    nx, ny, nz = 8, 16, 4
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    pw = np.exp(2j * np.pi * (3.0 * i / nx + 5.0 * j / ny + 1.0 * k / nz)).reshape(-1)
    out["fft3d_8x16x4_planewave_in"] = pw
    out["fft3d_8x16x4_planewave_out"] = ref.fft3d(pw, (nx, ny, nz))
    t = np.arange(64, dtype=np.float64)
    sig = (np.sin(1.3 * t) + 0.1 * t) + 1j * np.cos(2.7 * t)
    out["fft3d_8x4x2_in"] = sig
    out["fft3d_8x4x2_out"] = ref.fft3d(sig, (8, 4, 2))
    out["ifft3d_8x4x2_out"] = ref.fft3d(sig, (8, 4, 2), inverse=True)

    # propagator_tables_test.cpp: cube4 harmonic(2, {1,2,3}), dt 0.1; mass 2.0
    box4, n4 = (0.0, 4.0, 0.0, 4.0, 0.0, 4.0), (4, 4, 4)
    v4 = ref.harmonic3d(box4, n4, 2.0, (1.0, 2.0, 3.0))
    out["tables_cube4_V"] = v4
    for m in (1.0, 2.0):
        h, kk = ref.tables3d(box4, n4, v4, 0.1, m)
        out[f"tables_cube4_m{m:g}_half"] = h
        out[f"tables_cube4_m{m:g}_kin"] = kk

    # vkcheck check_engine_step: 8^3 soft Coulomb, dt 0.02, 20 steps
    box8, n8 = (-4.0, 4.0) * 3, (8, 8, 8)
    v8 = ref.soft_coulomb3d(box8, n8, 1.0, 1.0)
    p8 = ref.gaussian3d(box8, n8, (1.0, 0.0, 0.0), (1.2, 1.2, 1.2), (0.0, 0.5, 0.0))
    out["step_8cube_V"], out["step_8cube_psi0"] = v8, p8
    out["step_8cube_psi20"] = ref.step3d(box8, n8, v8, 0.02, p8, 20)
    # vkcheck check_engine_absorber: same + sin^2 mask width 2, 5 steps
    m8 = ref.absorbing_mask3d(box8, n8, 2.0)
    out["absorb_8cube_mask"] = m8
    out["absorb_8cube_psi5"] = ref.step3d(box8, n8, v8, 0.02, p8, 5, mask=m8)

    # simulation_test.cpp demo config: 16^3 harmonic, dt 0.02, 5 steps
    box16, n16 = (-8.0, 8.0) * 3, (16, 16, 16)
    v16 = ref.harmonic3d(box16, n16, 1.0)
    p16 = ref.gaussian3d(box16, n16, (2.0, 0.0, 0.0), (1.0, 1.0, 1.0), (0.0, 0.5, 0.0))
    out["step_16cube_V"], out["step_16cube_psi0"] = v16, p16
    s = ref.split3d(box16, n16, v16, 0.02)
    s.set_psi(p16)
    s.step(5)
    out["step_16cube_psi5"] = s.get_psi()
    out["step_16cube_norm5"] = np.array([s.norm()])
    out["step_16cube_energy5"] = np.array([s.mean_energy(v16)])
    s.close()

    # potential_test.cpp grids
    out["coulomb_16cube_h1"] = ref.regularized_coulomb3d(box16, n16, 1.0)
    out["barrier_16cube"] = ref.barrier3d(box16, n16, 0.25, 0.0, 3.0)
    out["mask_16cube_w3"] = ref.absorbing_mask3d(box16, n16, 3.0)
    out["mask1d_16_w3"] = ref.absorbing_mask1d(-8.0, 8.0, 16, 3.0)
    out["double_well_16"] = ref.double_well1d(-8.0, 8.0, 16, 0.1, 4.0)
    out["poschl_teller_16"] = ref.poschl_teller1d(-8.0, 8.0, 16, 0.375, 2.0)
    out["morse_16"] = ref.morse1d(-8.0, 8.0, 16, 0.3, 0.5, -2.0)
    out["wavenumbers_8"] = ref.wavenumbers(0.0, 8.0, 8)

    # propagator_test.cpp free packet: 1024 points, dt 0.05, 200 steps
    p1 = ref.gaussian1d(-40.0, 40.0, 1024, -15.0, 1.0, 2.0)
    out["line_1024_psi0"] = p1
    out["line_1024_psi200"] = ref.step1d(-40.0, 40.0, 1024, np.zeros(1024), 0.05, p1, 200)

    # imaginary time (dynamics3_test.cpp:64-87 shape, shortened): 16^3 harmonic w=2
    boxi, ni = (-4.0, 4.0) * 3, (16, 16, 16)
    vi = ref.harmonic3d(boxi, ni, 2.0)
    pi0 = ref.gaussian3d(boxi, ni, (0.5, -0.5, 0.3), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0))
    out["relax_16cube_V"], out["relax_16cube_psi0"] = vi, pi0
    out["relax_16cube_psi50"] = ref.relax3d(boxi, ni, vi, 0.01, pi0, 50)

    # dipole drive (drive.ixx:25-65): kick(t) . step . kick(t + dt), 16 x 8 x 8 harmonic
    boxd, nd = (-6.0, 6.0, -5.0, 5.0, -4.0, 4.0), (16, 8, 8)
    vd = ref.harmonic3d(boxd, nd, 1.0)
    pd = ref.gaussian3d(boxd, nd, (0.5, 0.0, 0.0), (1.0, 1.0, 1.0), (0.3, 0.0, 0.0))
    sd = ref.split3d(boxd, nd, vd, 0.05)
    sd.set_psi(pd)
    sd.driven_step(7, (0.6, 0.0, 0.8), 0.3, 1.1, 0.2)
    out["drive_16x8x8_psi7"] = sd.get_psi()
    sd.close()

    np.savez_compressed(HERE / "reference_core.npz", **out)
    size = (HERE / "reference_core.npz").stat().st_size
    print(f"wrote {len(out)} arrays, {size / 1024:.0f} KiB")
    return 0


if __name__ == "__main__":
    sys.exit(main())
