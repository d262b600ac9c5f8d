"""Host-side builders of potentials, absorbers and initial packets (FP64, numpy).

Vectorised restatements of the reference builders (core/src/potential.ixx,
core/src/wavepacket.ixx) plus the inputs of the benchmarked workloads.  They
produce the arrays handed to SplitOperator3D; the propagation itself runs on
the device.  Layout: flat x-fastest, index i + nx*(j + ny*k).

Absorber profile (new; the reference has only a sin^2 ramp,
potential.ixx:192-233): within `width` of a wall, at wall distance d,
    m(d) = cos(pi/2 * (1 - d/width))^(1/8)   (evaluated as sin(pi d/(2 width))^(1/8),
                                              which is exactly 0 on the wall)
and 1 further in; 3D masks are products of the per-axis profiles.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .core import Grid1D, Grid3D

K_COULOMB_CELL_AVERAGE = 2.3800774  # potential.ixx:99-100
SEED_BASE = 0x5E5B200


def _axes(g: Grid3D):
    return (g.x.coords()[None, None, :], g.y.coords()[None, :, None], g.z.coords()[:, None, None])


def harmonic(g: Grid3D, omega: float, c=(0.0, 0.0, 0.0)) -> np.ndarray:
    """0.5 w^2 |r - c|^2 (potential.ixx:35-49)."""
    x, y, z = _axes(g)
    dx, dy, dz = x - c[0], y - c[1], z - c[2]
    return (0.5 * omega * omega * (dx * dx + dy * dy + dz * dz)).reshape(-1)


def regularized_coulomb(g: Grid3D, Z: float, c=(0.0, 0.0, 0.0)) -> np.ndarray:
    """Bare -Z/r, nucleus cell -Z * 2.3800774 / h (potential.ixx:134-151)."""
    h = g.x.spacing()
    x, y, z = _axes(g)
    dx, dy, dz = x - c[0], y - c[1], z - c[2]
    r = np.sqrt(dx * dx + dy * dy + dz * dz)
    with np.errstate(divide="ignore"):
        v = np.where(r < 1e-6 * h, -Z * K_COULOMB_CELL_AVERAGE / h, -Z / r)
    return v.reshape(-1)


def stark_fold(g: Grid3D, v: np.ndarray, e_field: float) -> np.ndarray:
    """V += E z (hydrogen_director.ixx:1359-1370)."""
    z = g.z.coords()[:, None, None]
    return (v.reshape(g.shape) + e_field * z).reshape(-1)


def barrier(g: Grid3D, v0: float, x_lo: float, x_hi: float) -> np.ndarray:
    """v0 on the slab x in [x_lo, x_hi) (potential.ixx:114-129)."""
    x = g.x.coords()
    row = np.where((x >= x_lo) & (x < x_hi), v0, 0.0)
    return np.broadcast_to(row[None, None, :], g.shape).reshape(-1).copy()


def stadium(g: Grid3D, half_len: float, r: float, v_out: float) -> np.ndarray:
    """v_out where the stadium SDF > 0 in the x-y plane (billiard2d_director.ixx:26-29)."""
    x = g.x.coords()[None, None, :]
    y = g.y.coords()[None, :, None]
    cx = np.clip(x, -half_len, half_len)
    sdf = np.hypot(x - cx, y) - r
    v = np.where(sdf > 0.0, v_out, 0.0)
    return np.broadcast_to(v, g.shape).reshape(-1).copy()


def morse(g: Grid1D, d: float, alpha: float, x0: float) -> np.ndarray:
    q = 1.0 - np.exp(-alpha * (g.coords() - x0))
    return d * q * q


def double_well(g: Grid1D, vb: float, a: float) -> np.ndarray:
    s = g.coords() / a
    q = s * s - 1.0
    return vb * q * q


def poschl_teller(g: Grid1D, v0: float, a: float, x0: float = 0.0) -> np.ndarray:
    c = np.cosh((g.coords() - x0) / a)
    return -v0 / (c * c)


def mask_profile(g: Grid1D, width: float, profile: str = "cos8") -> np.ndarray:
    """Per-axis absorber: 'sin2' is the reference ramp, 'cos8' the cos^(1/8) ramp."""
    if g.n == 1:
        return np.ones(1)
    x = g.coords()
    d = np.minimum(x - g.xmin, g.xmax - x)
    s = np.sin(0.5 * 3.14159265358979323846 * np.minimum(d, width) / width)
    m = s * s if profile == "sin2" else np.power(s, 0.125)
    return np.where(d >= width, 1.0, m)


def mask_profiles(g: Grid3D, frac: float, profile: str = "cos8"):
    """Absorber on the outer `frac` of each axis: width = frac * axis length."""
    return tuple(mask_profile(a, frac * (a.xmax - a.xmin), profile) for a in (g.x, g.y, g.z))


def gaussian(g: Grid3D, r0, sigma, k0) -> np.ndarray:
    """Separable Gaussian packet times e^{i k0.r}, normalised on the grid (wavepacket.ixx:29-49)."""
    def env(u, u0, s):
        return math.pow(2.0 * math.pi * s * s, -0.25) * np.exp(-(u - u0) * (u - u0) / (4.0 * s * s))
    x, y, z = _axes(g)
    amp = env(x, r0[0], sigma[0]) * env(y, r0[1], sigma[1]) * env(z, r0[2], sigma[2])
    ph = k0[0] * x + k0[1] * y + k0[2] * z
    psi = (amp * np.exp(1j * ph)).reshape(-1)
    return normalized(g, psi)


def normalized(g: Grid3D, psi: np.ndarray) -> np.ndarray:
    n2 = float(np.vdot(psi, psi).real) * g.cell_volume()
    return psi / math.sqrt(n2) if n2 > 0 else psi


def gaussian_superposition(g: Grid3D, rng: np.random.Generator, m: int = 4, radius: float = 5.0,
                           sigma_range=(0.8, 2.0)) -> tuple[np.ndarray, list]:
    """Normalised sum of m isotropic Gaussians: centres uniform in |c| < radius
    (rejection), widths U[sigma_range], phases U[0, 2 pi), zero momentum."""
    psi = np.zeros(g.size(), dtype=np.complex128)
    parts = []
    for _ in range(m):
        while True:
            c = rng.uniform(-radius, radius, 3)
            if np.dot(c, c) < radius * radius:
                break
        s = float(rng.uniform(*sigma_range))
        phi = float(rng.uniform(0.0, 2.0 * math.pi))
        psi += np.exp(1j * phi) * gaussian(g, c, (s, s, s), (0.0, 0.0, 0.0))
        parts.append({"centre": c.tolist(), "sigma": s, "phase": phi})
    return normalized(g, psi), parts


def cube_grid(lo: float, hi: float, n: int) -> Grid3D:
    a = Grid1D(lo, hi, n)
    return Grid3D(a, a, a)


@dataclass
class Workload:
    name: str
    grid: Grid3D
    V: np.ndarray
    psi0: np.ndarray
    dt: float
    steps: int
    mask: tuple | None = None
    mass: float = 1.0
    observe_every: int = 100
    x_range: tuple = (-math.inf, math.inf)
    meta: dict = field(default_factory=dict)


def config_c1() -> Workload:
    """Plain FP64 single instance: 64^3 harmonic trap on [-10,10)^3, packet at (2,0,0), dt 0.005."""
    g = cube_grid(-10.0, 10.0, 64)
    return Workload("c1_harmonic_64", g, harmonic(g, 1.0), gaussian(g, (2, 0, 0), (1, 1, 1), (0, 0, 0)),
                    0.005, 2000, observe_every=100)


def config_c2(n: int = 256) -> Workload:
    """Regularized Coulomb Z=1 + Stark 0.01 z on [-40,40)^3, seeded 4-Gaussian superposition,
    cos^(1/8) absorber on the outer 10% of each axis, dt 0.01, 1000 steps."""
    g = cube_grid(-40.0, 40.0, n)
    rng = np.random.default_rng(SEED_BASE + 1)
    V = stark_fold(g, regularized_coulomb(g, 1.0), 0.01)
    psi0, parts = gaussian_superposition(g, rng)
    return Workload(f"c2_coulomb_stark_{n}", g, V, psi0, 0.01, 1000, mask=mask_profiles(g, 0.10),
                    observe_every=100, meta={"seed": SEED_BASE + 1, "packets": parts})


def config_c3(n: int = 512) -> Workload:
    """3D tunnelling on [-60,60)^3: barrier of thickness 2 at x=0 with height U[1,5]
    (seeded), packet sigma 3 at x=-20 with k0 = (3,0,0), cos^(1/8) absorber on the
    outer 8%, dt 0.002, 500 steps, transmitted P(x >= 1) every 50 steps."""
    g = cube_grid(-60.0, 60.0, n)
    v0 = config_c3_meta()
    return Workload(f"c3_tunnel_{n}", g, barrier(g, v0, -1.0, 1.0),
                    gaussian(g, (-20.0, 0.0, 0.0), (3.0, 3.0, 3.0), (3.0, 0.0, 0.0)), 0.002, 500,
                    mask=mask_profiles(g, 0.08), observe_every=50, x_range=(1.0, math.inf),
                    meta={"seed": SEED_BASE + 2, "barrier_height": v0})


def config_c3_strip(x0: float = -20.0) -> Workload:
    """C3's scene on a 512 x 64 x 64 grid of the same spacing (transverse box
    [-7.5, 7.5)): same barrier, packet (centred at x0), absorber, dt and step
    count -- the reduced size on which the full 500-step run is checked."""
    full_h = config_c3_meta()
    gx = Grid1D(-60.0, 60.0, 512)
    gt = Grid1D(-7.5, 7.5, 64)
    g = Grid3D(gx, gt, gt)
    psi0 = gaussian(g, (x0, 0.0, 0.0), (3.0, 3.0, 3.0), (3.0, 0.0, 0.0))
    return Workload(f"c3_strip_512x64x64_x0_{x0:g}", g, barrier(g, full_h, -1.0, 1.0), psi0, 0.002, 500,
                    mask=mask_profiles(g, 0.08), observe_every=50, x_range=(1.0, math.inf),
                    meta={"seed": SEED_BASE + 2, "barrier_height": full_h, "x0": x0})


def config_c3_meta() -> float:
    """C3's seeded barrier height U[1, 5]."""
    return float(np.random.default_rng(SEED_BASE + 2).uniform(1.0, 5.0))


C4_SIZES = (32, 48, 64, 96, 128, 160)


def config_c4_specs(count: int = 256, sizes=C4_SIZES, seed: int = SEED_BASE + 3) -> list[dict]:
    """Batched tunnelling sweep: `count` independent 3D instances, n uniform over
    `sizes`, box side 20 n/32 centred on 0 (spacing 0.625 at every n), barrier of
    thickness 2 at x = 0 with height U[0.5, 4], packet sigma U[1, 2.5] (isotropic)
    at x = -L/4 with k0 = (U[1, 4], 0, 0), cos^(1/8) absorber on the outer 8%,
    complex64 with FP64-built tables, dt 0.005, 1000 steps.  Drawn in this order
    per instance: n, height, k0, sigma."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(sizes[int(rng.integers(0, len(sizes)))])
        v0 = float(rng.uniform(0.5, 4.0))
        k0 = float(rng.uniform(1.0, 4.0))
        sigma = float(rng.uniform(1.0, 2.5))
        out.append({"index": i, "n": n, "side": 20.0 * n / 32.0, "barrier": v0, "k0": k0,
                    "sigma": sigma, "dt": 0.005, "steps": 1000, "mask_frac": 0.08})
    return out


def build_c4_instance(spec: dict) -> Workload:
    half = 0.5 * spec["side"]
    g = cube_grid(-half, half, spec["n"])
    s = spec["sigma"]
    psi0 = gaussian(g, (-0.5 * half, 0.0, 0.0), (s, s, s), (spec["k0"], 0.0, 0.0))
    return Workload(f"c4_tunnel_{spec['n']}_{spec['index']}", g, barrier(g, spec["barrier"], -1.0, 1.0),
                    psi0, spec["dt"], spec["steps"], mask=mask_profiles(g, spec["mask_frac"]),
                    observe_every=100, x_range=(1.0, math.inf), meta=dict(spec))


def build_c4_plane(spec: dict) -> Workload:
    """The scene of a batched-sweep instance on one z-plane (n x n x 1)."""
    half = 0.5 * spec["side"]
    a = Grid1D(-half, half, spec["n"])
    g = Grid3D(a, a, Grid1D(0.0, 1.0, 1))
    s = spec["sigma"]
    psi0 = gaussian(g, (-0.5 * half, 0.0, 0.0), (s, s, s), (spec["k0"], 0.0, 0.0))
    mx, my, _ = mask_profiles(g, spec["mask_frac"])
    return Workload(f"c4_plane_{spec['n']}_{spec['index']}", g, barrier(g, spec["barrier"], -1.0, 1.0), psi0,
                    spec["dt"], spec["steps"], mask=(mx, my, np.ones(1)), observe_every=100,
                    x_range=(1.0, math.inf), meta=dict(spec))


def config_c5_specs(count: int = 48, seed: int = SEED_BASE + 4) -> list[dict]:
    """Serving stream: `count` requests, 40% 1D / 30% 2D / 30% 3D, steps log-uniform in
    [100, 5000], dt U[0.002, 0.01], complex64, observables every 100 steps, cos^(1/8)
    absorber on the outer 10% of each transformed axis.
      1D: 65536 points on [-200, 200): Morse (depth U[0.5,10], alpha 0.5, x0 0), double well
          (barrier U[0.5,10], a 3) or Poschl-Teller (depth U[0.5,10], a 1); packet sigma 1
          at the well minimum, k0 = 0.5.
      2D: 512^2 or 1024^2 on [-30, 30)^2: harmonic dot (omega U[0.2,1]) or stadium (R 13,
          half-length 6.5, V = 50 outside); packet sigma 1.5 at the origin, k0 = (2, 0).
      3D: n in {64, 128, 256}: harmonic (omega U[0.5,2], box [-10,10)) or regularized
          Coulomb Z = 1 (box [-40,40)); packet sigma 1 at (1, 0, 0) (harmonic) or sigma 1.5
          at (2, 0, 0) (Coulomb), at rest.
    Drawn per request in this order: kind, variant, size, strength, steps, dt."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        u = float(rng.uniform())
        kind = "1d" if u < 0.4 else ("2d" if u < 0.7 else "3d")
        variant = int(rng.integers(0, 3 if kind == "1d" else 2))
        size = int(rng.integers(0, 2 if kind == "2d" else 3))
        strength = float(rng.uniform())
        steps = int(round(math.exp(rng.uniform(math.log(100.0), math.log(5000.0)))))
        dt = float(rng.uniform(0.002, 0.01))
        if kind == "1d":
            pot = ("morse", "double_well", "poschl_teller")[variant]
            dims, val = (65536, 1, 1), 0.5 + 9.5 * strength
        elif kind == "2d":
            pot = ("harmonic", "stadium")[variant]
            n = (512, 1024)[size]
            dims, val = (n, n, 1), 0.2 + 0.8 * strength
        else:
            pot = ("harmonic", "coulomb")[variant]
            n = (64, 128, 256)[size]
            dims, val = (n, n, n), 0.5 + 1.5 * strength
        out.append({"index": i, "kind": kind, "potential": pot, "dims": dims, "strength": val,
                    "steps": steps, "dt": dt, "points": dims[0] * dims[1] * dims[2]})
    return out


def build_c5_request(spec: dict) -> dict:
    """Keyword arguments of Server.submit for one serving request."""
    from .core import line_grid
    kind, pot, v = spec["kind"], spec["potential"], spec["strength"]
    if kind == "1d":
        g1 = Grid1D(-200.0, 200.0, spec["dims"][0])
        if pot == "morse":
            V, x0 = morse(g1, v, 0.5, 0.0), 0.0
        elif pot == "double_well":
            V, x0 = double_well(g1, v, 3.0), 3.0
        else:
            V, x0 = poschl_teller(g1, v, 1.0), 0.0
        g = line_grid(g1)
        psi = gaussian(g, (x0, 0.0, 0.0), (1.0, 1.0, 1.0), (0.5, 0.0, 0.0))
    elif kind == "2d":
        n = spec["dims"][0]
        a = Grid1D(-30.0, 30.0, n)
        g = Grid3D(a, a, Grid1D(0.0, 2.0, 1))
        V = harmonic(g, v) if pot == "harmonic" else stadium(g, 6.5, 13.0, 50.0)
        psi = gaussian(g, (0.0, 0.0, 0.0), (1.5, 1.5, 1.0), (2.0, 0.0, 0.0))
    else:
        n = spec["dims"][0]
        if pot == "harmonic":
            g = cube_grid(-10.0, 10.0, n)
            V = harmonic(g, v)
            psi = gaussian(g, (1.0, 0.0, 0.0), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0))
        else:
            g = cube_grid(-40.0, 40.0, n)
            V = regularized_coulomb(g, 1.0)
            psi = gaussian(g, (2.0, 0.0, 0.0), (1.5, 1.5, 1.5), (0.0, 0.0, 0.0))
    mask = tuple(np.ones(1) if ax.n == 1 else mask_profile(ax, 0.1 * (ax.xmax - ax.xmin))
                 for ax in (g.x, g.y, g.z))
    return dict(grid=g, V=V, psi0=psi, dt=spec["dt"], nsteps=spec["steps"], observe_every=100, mask=mask,
                precision="c64", x_range=(0.0, math.inf))
