"""Seeded synthetic disk-galaxy generator (stars + dark matter).

The reference ships only ``data/nbody/ini/start_S0.txt`` (262 144 stars); its
``start_DM0.txt`` is missing, so the initial conditions of every workload are
generated here from a seed:

* stars: exponential disk, surface density ~ exp(-R/h) truncated at R_max,
  vertical sech^2(z/z0) profile, azimuthal velocity equal to the circular
  velocity of the spherically enclosed particle mass plus an isotropic Gaussian
  dispersion of ``sigma_frac * v_c`` per component;
* dark matter: Plummer sphere of scale ``a`` truncated at ``r_max``, velocities
  drawn from the (untruncated) Plummer distribution function by the
  Aarseth-Henon-Wielen (1974) rejection method.

Units are the reference's (G = 1).  The output is in the galaxy frame; the
centre offset, bulk velocity and tilt are applied by the loader exactly as the
reference does it (``nbody/src/nbody.cu:1342-1360``), so the same arrays can be
written through the reference's ``start_S{k}.txt`` / ``start_DM{k}.txt`` text
format and read back by both the oracle and the GPU driver.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

STAR_MASS_DEFAULT = 1.0
DM_MASS_DEFAULT = 6.699356


@dataclasses.dataclass
class Galaxy:
    """One galaxy in its own frame.  Arrays are float64, shape (n, 3)."""

    star_pos: np.ndarray
    star_vel: np.ndarray
    dm_pos: np.ndarray
    dm_vel: np.ndarray
    m_stars: float
    m_dm: float
    eps_stars: float
    eps_dm: float

    @property
    def n_stars(self) -> int:
        return int(self.star_pos.shape[0])

    @property
    def n_dm(self) -> int:
        return int(self.dm_pos.shape[0])

    @property
    def n(self) -> int:
        return self.n_stars + self.n_dm

    def arrays(self):
        """(pos, vel, mass, eps) with stars first, then DM (reference layout)."""
        pos = np.concatenate([self.star_pos, self.dm_pos]).astype(np.float64)
        vel = np.concatenate([self.star_vel, self.dm_vel]).astype(np.float64)
        mass = np.empty(self.n, np.float64)
        eps = np.empty(self.n, np.float64)
        if self.n_stars:
            mass[: self.n_stars] = self.m_stars / self.n_stars
            eps[: self.n_stars] = self.eps_stars
        if self.n_dm:
            mass[self.n_stars:] = self.m_dm / self.n_dm
            eps[self.n_stars:] = self.eps_dm
        return pos, vel, mass, eps


def _exp_disk_radius(u: np.ndarray, h: float) -> np.ndarray:
    """Invert M(<R)/M_inf = 1 - (1 + R/h) exp(-R/h) by vectorised bisection."""
    lo = np.zeros_like(u)
    hi = np.full_like(u, 60.0 * h)
    for _ in range(64):
        mid = 0.5 * (lo + hi)
        x = mid / h
        f = 1.0 - (1.0 + x) * np.exp(-x)
        below = f < u
        lo = np.where(below, mid, lo)
        hi = np.where(below, hi, mid)
    return 0.5 * (lo + hi)


def _isotropic(rng: np.random.Generator, n: int) -> np.ndarray:
    cos_t = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * math.pi, n)
    sin_t = np.sqrt(np.maximum(0.0, 1.0 - cos_t * cos_t))
    return np.stack([sin_t * np.cos(phi), sin_t * np.sin(phi), cos_t], axis=1)


def _plummer_q(rng: np.random.Generator, n: int) -> np.ndarray:
    """Sample q = v/v_esc from g(q) ~ q^2 (1 - q^2)^(7/2) on [0, 1]."""
    out = np.empty(n)
    filled = 0
    while filled < n:
        m = max(1024, 3 * (n - filled))
        x = rng.uniform(0.0, 1.0, m)
        y = rng.uniform(0.0, 0.1, m)
        ok = x[y < x * x * (1.0 - x * x) ** 3.5]
        take = min(ok.size, n - filled)
        out[filled:filled + take] = ok[:take]
        filled += take
    return out


def make_galaxy(
    n_stars: int,
    n_dm: int,
    seed: int,
    m_stars: float = STAR_MASS_DEFAULT,
    m_dm: float = DM_MASS_DEFAULT,
    eps_stars: float = 0.004,
    eps_dm: float = 0.004,
    disk_h: float = 0.2,
    disk_rmax: float = 1.0,
    disk_z0: float = 0.02,
    plummer_a: float = 0.3333,
    plummer_rmax: float = 2.0,
    sigma_frac: float = 0.1,
) -> Galaxy:
    """Generate one galaxy from ``seed`` (numpy PCG64 stream, fixed draw order)."""
    rng = np.random.default_rng(seed)

    # --- dark matter: truncated Plummer sphere -------------------------------
    a = plummer_a
    frac_max = plummer_rmax ** 3 / (plummer_rmax ** 2 + a * a) ** 1.5
    u = rng.uniform(0.0, frac_max, n_dm)
    u = np.maximum(u, 1e-300)
    r_dm = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
    dm_pos = _isotropic(rng, n_dm) * r_dm[:, None]
    q = _plummer_q(rng, n_dm)
    # Escape speed of the (untruncated) Plummer potential of mass m_dm.
    v_esc = np.sqrt(2.0 * m_dm) * (r_dm * r_dm + a * a) ** (-0.25)
    dm_vel = _isotropic(rng, n_dm) * (q * v_esc)[:, None]

    # --- stars: exponential disk with sech^2 vertical profile -----------------
    h = disk_h
    f_max = 1.0 - (1.0 + disk_rmax / h) * math.exp(-disk_rmax / h)
    u = rng.uniform(0.0, f_max, n_stars)
    R = _exp_disk_radius(u, h)
    phi = rng.uniform(0.0, 2.0 * math.pi, n_stars)
    uz = rng.uniform(1e-12, 1.0 - 1e-12, n_stars)
    z = disk_z0 * np.arctanh(2.0 * uz - 1.0)
    cphi, sphi = np.cos(phi), np.sin(phi)
    star_pos = np.stack([R * cphi, R * sphi, z], axis=1)

    # Circular velocity from the spherically enclosed particle mass.
    r_s = np.sqrt(R * R + z * z)
    radii = np.concatenate([r_s, r_dm])
    masses = np.concatenate([
        np.full(n_stars, m_stars / max(n_stars, 1)),
        np.full(n_dm, m_dm / max(n_dm, 1)),
    ])
    order = np.argsort(radii, kind="stable")
    m_enc_sorted = np.cumsum(masses[order])
    m_enc = np.empty_like(m_enc_sorted)
    m_enc[order] = m_enc_sorted
    m_enc_s = m_enc[:n_stars]
    vc = np.sqrt(np.where(r_s > 0.0, m_enc_s / np.maximum(r_s, 1e-300), 0.0))
    disp = rng.normal(0.0, 1.0, (n_stars, 3)) * (sigma_frac * vc)[:, None]
    star_vel = np.stack([-vc * sphi, vc * cphi, np.zeros(n_stars)], axis=1) + disp

    return Galaxy(star_pos, star_vel, dm_pos, dm_vel,
                  m_stars if n_stars else 0.0, m_dm if n_dm else 0.0,
                  eps_stars, eps_dm)


def place(pos: np.ndarray, vel: np.ndarray, alpha_deg: float,
          centre=(0.0, 0.0, 0.0), bulk=(0.0, 0.0, 0.0)):
    """Apply the reference's tilt + shift to galaxy-frame arrays.

    Follows ``nbody/src/nbody.cu:1342-1360`` literally, including its use of
    the already-updated x when computing z (so for alpha != 0 the "rotation"
    is a shear); this defines the reference's initial conditions.
    """
    # The reference's DEG2RAD uses PI = 3.14159265358979 (common.cuh:7,10).
    rad = (3.14159265358979 / 180.0) * alpha_deg
    c = math.cos(rad)
    s = math.sin(rad)
    p = pos.copy()
    v = vel.copy()
    p[:, 0] = centre[0] + pos[:, 0] * c + pos[:, 2] * s
    p[:, 1] = pos[:, 1] + centre[1]
    p[:, 2] = centre[2] + pos[:, 2] * c - p[:, 0] * s
    v[:, 0] = bulk[0] + vel[:, 0] * c + vel[:, 2] * s
    v[:, 1] = vel[:, 1] + bulk[1]
    v[:, 2] = bulk[2] + vel[:, 2] * c - v[:, 0] * s
    return p, v


def assemble(galaxies, placements):
    """Reference memory layout of several galaxies (nbody/src/nbody.cu:1318-1417):
    the stars of every galaxy first, then the dark matter of every galaxy,
    each placed by ``place`` (tilt alpha_deg, centre, bulk velocity).
    Returns (pos, vel, mass, eps2)."""
    parts = {"s": [], "d": []}
    for g, (alpha, centre, bulk) in zip(galaxies, placements):
        if g.n_stars:
            p, v = place(g.star_pos, g.star_vel, alpha, centre, bulk)
            parts["s"].append((p, v, g.m_stars / g.n_stars, g.eps_stars, g.n_stars))
        if g.n_dm:
            p, v = place(g.dm_pos, g.dm_vel, alpha, centre, bulk)
            parts["d"].append((p, v, g.m_dm / g.n_dm, g.eps_dm, g.n_dm))
    seq = parts["s"] + parts["d"]
    pos = np.concatenate([s[0] for s in seq])
    vel = np.concatenate([s[1] for s in seq])
    mass = np.concatenate([np.full(s[4], s[2]) for s in seq])
    eps2 = np.concatenate([np.full(s[4], s[3] * s[3]) for s in seq])
    return pos, vel, mass, eps2


def two_galaxy_encounter(n_stars: int = 131072, n_dm: int = 262144, seed: int = 3000):
    """Two generator galaxies centred at (+-1.5, 0, 0) with bulk velocities
    (-+0.3, +-0.1, 0); the second is tilted by 30 degrees."""
    g1 = make_galaxy(n_stars, n_dm, seed)
    g2 = make_galaxy(n_stars, n_dm, seed + 1)
    return assemble([g1, g2], [(0.0, (1.5, 0.0, 0.0), (-0.3, 0.1, 0.0)),
                               (30.0, (-1.5, 0.0, 0.0), (0.3, -0.1, 0.0))])


def round_to(n: int, m: int = 1024) -> int:
    return max(m, int(round(n / m)) * m)


def ensemble_sizes(count: int, seed: int, lo: int = 4096, hi: int = 131072,
                   multiple: int = 1024):
    """Log-uniform total particle counts in [lo, hi], rounded to ``multiple``.

    Each total is split about 1:2 between stars and DM, with the star count a
    multiple of 512 (so both parts stay multiples of 512)."""
    rng = np.random.default_rng(seed)
    tot = np.exp(rng.uniform(math.log(lo), math.log(hi), count))
    out = []
    for t in tot:
        n = round_to(float(t), multiple)
        ns = max(512, int(round(n / 3 / 512)) * 512)
        nd = n - ns
        out.append((ns, nd))
    return out
