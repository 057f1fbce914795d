"""Seeded synthetic inputs with the shapes of the path's five workloads.

Every generator is deterministic for its seed (numpy PCG64) and returns a
``(desc, frame)`` pair: ``desc`` is a dict of :func:`atomiverse_b200.make_desc`
keywords, ``frame`` a dict of float64 / int64 numpy arrays in the reference's
metal units (A, eV, fs, amu, e).

Reduced Lennard-Jones workloads map onto metal units with eps = 1 eV,
sigma = 1 A, m = 1 amu, so tau = sqrt(m sigma^2 / eps) = sqrt(103.6427) fs
= 10.1805 fs and T* = 1 corresponds to eps / k_B = 11604.5 K.
"""
from __future__ import annotations

import math

import numpy as np

KB = 8.617333262e-5          # eV/K   (units.h:138)
MVV2E = 103.6427             # amu A^2/fs^2 -> eV (units.h:166)
TAU_LJ_FS = math.sqrt(MVV2E)  # 10.1805 fs
KJMOL_PER_EV = 96.48533212


def recommend_alpha(cutoff: float, accuracy: float = 1e-5) -> float:
    """LAMMPS heuristic g_ewald = (1.35 - 0.15 ln(accuracy)) / cutoff
    (the reference's EwaldSum::recommend_alpha, ewald_sum.h:58-60)."""
    return (1.35 - 0.15 * math.log(accuracy)) / cutoff


def good_fft_size(n: int) -> int:
    """Smallest 2,3,5,7-smooth integer >= max(n, 4) (the reference's
    good_fft_size, pme_spline.h:99-111, restated)."""
    k = max(int(n), 4)
    while True:
        m = k
        for p in (2, 3, 5, 7):
            while m % p == 0:
                m //= p
        if m == 1:
            return k
        k += 1


def fcc_sites(ncell: int, a: float) -> np.ndarray:
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.arange(ncell)
    cells = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)
    pts = (cells[:, None, :] + base[None, :, :]).reshape(-1, 3) * a
    return pts


def maxwell_velocities(mass: np.ndarray, T: float, rng) -> np.ndarray:
    """Gaussian velocities at T [K], net momentum removed, rescaled so the
    kinetic temperature with 3N-3 degrees of freedom is exactly T."""
    n = len(mass)
    sd = np.sqrt(KB * T / (mass * MVV2E))
    v = rng.normal(size=(n, 3)) * sd[:, None]
    v -= (mass[:, None] * v).sum(0) / mass.sum()
    ke = 0.5 * MVV2E * (mass[:, None] * v * v).sum()
    ndof = max(3 * n - 3, 1)
    t_now = 2.0 * ke / (ndof * KB)
    if t_now > 0:
        v *= math.sqrt(T / t_now)
    return v


def _frame(pos, vel, mass, charge):
    n = len(mass)
    return {
        "x": np.ascontiguousarray(pos[:, 0]), "y": np.ascontiguousarray(pos[:, 1]),
        "z": np.ascontiguousarray(pos[:, 2]),
        "vx": np.ascontiguousarray(vel[:, 0]), "vy": np.ascontiguousarray(vel[:, 1]),
        "vz": np.ascontiguousarray(vel[:, 2]),
        "fx": np.zeros(n), "fy": np.zeros(n), "fz": np.zeros(n),
        "mass": np.ascontiguousarray(mass, dtype=np.float64),
        "charge": np.ascontiguousarray(charge, dtype=np.float64),
        "tag": np.arange(1, n + 1, dtype=np.int64),
    }


def lj_fcc(ncell: int = 10, rho: float = 0.8442, t_star: float = 1.44,
           seed: int = 2026, rc: float = 2.5, skin: float = 0.3,
           dt_tau: float = 0.005, precision: int = 0, n_keep: int | None = None,
           thermostat: int = 0, damp_tau: float = 1.0):
    """FCC Lennard-Jones fluid in reduced units (eps = sigma = m = 1).

    Plain LJ NVE: ncell=10 -> 4,000 atoms at rho* = 0.8442, T* = 1.44.
    Precision study: ncell=63 -> 1,000,188 atoms at T* = 0.72.
    ``n_keep`` keeps the first n sites of the lattice (ladder systems) with
    the box rescaled to keep rho*.
    """
    n_full = 4 * ncell ** 3
    n = n_full if n_keep is None else int(n_keep)
    L = (n / rho) ** (1.0 / 3.0)
    a = L / ncell
    pos = fcc_sites(ncell, a)[:n]
    rng = np.random.default_rng(seed)
    mass = np.ones(n)
    T = t_star / KB
    vel = maxwell_velocities(mass, T, rng)
    dt = dt_tau * TAU_LJ_FS
    desc = dict(n_atoms=n, box=(L, L, L), precision=precision, nl_cutoff=rc,
                nl_skin=skin, lj_enabled=1, lj_epsilon=1.0, lj_sigma=1.0,
                lj_cutoff=rc, dt=dt, thermostat=thermostat, temperature=T,
                damp=damp_tau * TAU_LJ_FS, seed=seed)
    return desc, _frame(pos, vel, mass, np.zeros(n))


def rocksalt_melt(ncell: int = 64, spacing: float = 2.82, jitter: float = 0.2,
                  seed: int = 2027, T: float = 1200.0, rc: float = 12.0,
                  skin: float = 1.0, grid=None, grid_spacing: float | None = None,
                  order: int = 4, precision: int = 0, tau: float = 100.0,
                  dt: float = 2.0):
    """Charged LJ melt with PME: ncell^3 ions of +-1 e on a rock-salt lattice
    (default 64^3 = 262,144 ions, spacing 2.82 A, box 180.48 A), positions
    jittered U(-jitter, jitter) per component, LJ sigma = 3.0 A and
    eps = 0.5 kJ/mol, masses 23.0 / 35.45 amu, real-space cutoff 12 A,
    alpha at Ewald tolerance 1e-5, PME order 4 on a 192^3 grid (or the
    spacing rule), Nose-Hoover at T (tau = 100 fs), dt = 2 fs."""
    n = ncell ** 3
    g = np.arange(ncell)
    ijk = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)
    L = ncell * spacing
    rng = np.random.default_rng(seed)
    pos = ijk * spacing + rng.uniform(-jitter, jitter, size=(n, 3))
    pos = np.mod(pos, L)
    even = (ijk.sum(1) % 2) == 0
    charge = np.where(even, 1.0, -1.0)
    mass = np.where(even, 23.0, 35.45)
    vel = maxwell_velocities(mass, T, rng)
    alpha = recommend_alpha(rc, 1e-5)
    desc = dict(n_atoms=n, box=(L, L, L), precision=precision, nl_cutoff=rc,
                nl_skin=skin, lj_enabled=1, lj_epsilon=0.5 / KJMOL_PER_EV,
                lj_sigma=3.0, lj_cutoff=rc, coul_enabled=1, coul_alpha=alpha,
                coul_cutoff=rc, pme_enabled=1, pme_alpha=alpha, pme_order=order,
                dt=dt, thermostat=1, temperature=T, tau=tau)
    if grid is not None:
        desc["pme_grid"] = tuple(grid)
    elif grid_spacing is not None:
        desc["pme_grid_spacing"] = grid_spacing
    else:
        K = good_fft_size(math.ceil(L / 0.94))
        desc["pme_grid"] = (K, K, K) if ncell != 64 else (192, 192, 192)
    return desc, _frame(pos, vel, mass, charge)


def ladder(n_systems: int = 512, seed: int = 2029, n_min: int = 256,
           n_max: int = 32768, t_lo: float = 0.70, t_hi: float = 1.50,
           precision: int = 1):
    """Replica ladder: atom counts log-uniform in [n_min, n_max], FCC-derived
    boxes at rho* = 0.8442, T* geometric from t_lo to t_hi, Langevin with
    damp = 1 tau, mixed precision."""
    rng = np.random.default_rng(seed)
    sizes = np.round(np.exp(rng.uniform(math.log(n_min), math.log(n_max), n_systems))).astype(int)
    out = []
    for k, nk in enumerate(sizes):
        c = math.ceil((nk / 4) ** (1.0 / 3.0))
        t = t_lo * (t_hi / t_lo) ** (k / max(n_systems - 1, 1))
        desc, frame = lj_fcc(ncell=c, t_star=t, seed=seed + 1 + k, n_keep=int(nk),
                             precision=precision, thermostat=2, damp_tau=1.0)
        out.append((desc, frame))
    return out


def request_specs(n_requests: int = 2000, rate: float = 200.0, seed: int = 2030,
                  n_min: int = 500, n_max: int = 200000, frac_lj: float = 0.6,
                  steps: int = 1000):
    """Poisson arrivals of MD segments as specs (no atoms generated yet):
    dicts with arrival time [s], kind ("lj" or "pme"), lattice size and
    seed.  60 % LJ fluids (4 c^3 atoms, as the 4,000-atom fluid rescaled)
    and 40 % rock-salt PME melts (n even, n^3 ions, grid spacing ~0.94 A),
    sizes log-uniform in [n_min, n_max]."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n_requests))
    sizes = np.exp(rng.uniform(math.log(n_min), math.log(n_max), n_requests))
    kinds = rng.uniform(size=n_requests) < frac_lj
    out = []
    for k in range(n_requests):
        if kinds[k]:
            c = max(4, round((sizes[k] / 4) ** (1 / 3)))
            out.append(dict(t=float(t[k]), kind="lj", cells=int(c), seed=seed + 1 + k,
                            n_atoms=4 * c ** 3, steps=steps))
        else:
            m = max(8, int(round(sizes[k] ** (1 / 3))))
            m += m % 2
            out.append(dict(t=float(t[k]), kind="pme", cells=int(m), seed=seed + 1 + k,
                            n_atoms=m ** 3, steps=steps))
    return out


def build_request(spec: dict, precision: int = 1):
    """(desc, frame) of one request spec from ``request_specs``."""
    if spec["kind"] == "lj":
        return lj_fcc(ncell=spec["cells"], seed=spec["seed"], precision=precision)
    m = spec["cells"]
    L = m * 2.82
    K = good_fft_size(math.ceil(L / 0.94))
    # small boxes: shrink the real-space cutoff so that 2 (rc + skin) < L
    rc = min(12.0, 0.5 * L - 1.0 - 0.05)
    return rocksalt_melt(ncell=m, seed=spec["seed"], grid=(K, K, K), precision=precision,
                         rc=rc)


def request_stream(n_requests: int = 2000, rate: float = 200.0, seed: int = 2030,
                   n_min: int = 500, n_max: int = 200000, frac_lj: float = 0.6,
                   precision: int = 1):
    """Materialised request stream: (arrival_time_s, desc, frame) per
    request (small streams only; large ones use request_specs and
    build_request on arrival)."""
    specs = request_specs(n_requests, rate, seed, n_min, n_max, frac_lj)
    return [(sp["t"], *build_request(sp, precision)) for sp in specs]
