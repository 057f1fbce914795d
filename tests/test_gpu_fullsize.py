"""Parity at the benchmark sizes, against the oracle (one force pass on all
host threads) and through properties that hold at any size:

- the 262,144-ion rock-salt melt (64^3 ions, 192^3 PME grid, rc 12 A,
  skin 1 A): FP64 and mixed forces, energies and the pair set (count and an
  order-free checksum of the unordered pairs) against the oracle;
  Newton's third law on the pair forces; invariance under a shift of every
  ion by whole PME grid cells; bit-for-bit repeatability of 100
  Nose-Hoover steps, and the total energy over 100 NVE steps;
- the 1,000,188-atom LJ crystal (63^3 FCC cells, rho* = 0.8442, T* = 0.72):
  FP64 and mixed forces and the pair set against the oracle.

Tolerances as in the small-case parity tests: RMS relative force error
<= 1e-6 (FP64 with PME; its 2^-40 e fixed-point grid) or 1e-10 (FP64 LJ),
<= 5e-6 mixed.
"""
import numpy as np
import pytest

from atomiverse_b200 import workloads as W
from conftest import oracle_system, rms_rel

pytestmark = pytest.mark.gpu

M1 = np.uint64(0x9E3779B97F4A7C15)
M2 = np.uint64(0xBF58476D1CE4E5B9)


def _f(fr):
    return np.stack([fr["fx"], fr["fy"], fr["fz"]], 1)


def _pair_checksum(pi, pj):
    """Count and wrap-around sum of a mixed hash of the unordered pairs: equal
    sets give equal sums whatever their order."""
    a = np.minimum(pi, pj).astype(np.uint64)
    b = np.maximum(pi, pj).astype(np.uint64)
    k = (a << np.uint64(32)) | b
    with np.errstate(over="ignore"):
        h = k * M1
        h ^= h >> np.uint64(31)
        h *= M2
        h ^= h >> np.uint64(29)
        return len(k), int(np.sum(h, dtype=np.uint64))


def _forces(atvb, ctx, desc, frame, precision, pairs=False):
    s = atvb.System(ctx, dict(desc, precision=precision, stress_required=1), frame)
    s.compute_forces()
    out, sc = s.download()
    cs = _pair_checksum(*s.pairs()) if pairs else None
    s.close()
    return out, sc, cs


def _oracle(orc, desc, frame):
    o = oracle_system(orc, desc, frame)
    cs = _pair_checksum(*o.pairs())          # builds the list
    o.compute_forces()
    return o.state(), o.scalars(), cs


@pytest.fixture(scope="module")
def melt():
    return W.rocksalt_melt()


def test_rocksalt_262k_against_oracle(atvb, ctx, orc, melt):
    desc, frame = melt
    assert desc["n_atoms"] == 262144 and tuple(desc["pme_grid"]) == (192, 192, 192)
    ref, rsc, rcs = _oracle(orc, desc, frame)
    fref = _f(ref)
    out, sc, cs = _forces(atvb, ctx, desc, frame, 0, pairs=True)
    assert cs == rcs
    assert rms_rel(_f(out), fref) < 1e-6
    assert sc["energy"] == pytest.approx(rsc["energy"], rel=1e-8)
    vir = rsc["virial"]
    assert np.allclose(sc["stress"], vir, rtol=1e-6, atol=1e-7 * np.abs(vir).max())
    out, sc, cs = _forces(atvb, ctx, desc, frame, 1, pairs=True)
    assert cs == rcs
    assert rms_rel(_f(out), fref) < 5e-6
    assert sc["energy"] == pytest.approx(rsc["energy"], rel=1e-6)


def test_rocksalt_262k_newton_third_law(atvb, ctx, melt):
    """Real-space Ewald + LJ only: every pair force appears twice with
    opposite signs, so the forces sum to rounding."""
    desc, frame = melt
    d = dict(desc, pme_enabled=0)
    out, _, _ = _forces(atvb, ctx, d, frame, 0)
    f = _f(out)
    assert np.abs(f.sum(0)).max() < 1e-12 * np.abs(f).sum()


def test_rocksalt_262k_grid_cell_shift(atvb, ctx, melt):
    """Moving every ion by whole PME grid cells moves the charge grid by
    whole points: forces and energy are unchanged up to rounding."""
    desc, frame = melt
    L = np.array(desc["box"], dtype=float)
    h = L / np.array(desc["pme_grid"], dtype=float)
    shift = np.array([1.0, 2.0, -3.0]) * h
    moved = dict(frame)
    for ax, k in enumerate("xyz"):
        moved[k] = np.mod(np.asarray(frame[k], dtype=float) + shift[ax], L[ax])
    a, sa, _ = _forces(atvb, ctx, desc, frame, 0)
    b, sb, _ = _forces(atvb, ctx, desc, moved, 0)
    assert rms_rel(_f(b), _f(a)) < 1e-10
    assert sb["energy"] == pytest.approx(sa["energy"], rel=1e-11)


def test_rocksalt_262k_repeatable_and_conserved(atvb, ctx, melt):
    """Two Nose-Hoover runs of 100 steps agree bit for bit (rebuilds
    included); in NVE the total energy stays within 1e-3 of the kinetic
    energy over the same 100 steps."""
    desc, frame = melt
    runs = []
    for d in (desc, desc, dict(desc, thermostat=0)):
        s = atvb.System(ctx, d, frame)
        s.compute_forces()
        c0 = s.scalars()["conserved"]
        s.step(100)
        out, sc = s.download()
        s.close()
        runs.append((out, sc, c0))
    (a, sa, _), (b, sb, _), (_, se, e0) = runs
    for k in ("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz"):
        assert np.array_equal(a[k], b[k]), k
    assert sa["energy"] == sb["energy"] and sa["rebuilds"] == sb["rebuilds"] > 0
    assert abs(se["conserved"] - e0) < 1e-3 * se["kinetic"]


def test_lj_million_against_oracle(atvb, ctx, orc):
    desc, frame = W.lj_fcc(ncell=63, t_star=0.72, seed=2028)
    assert desc["n_atoms"] == 1000188
    rng = np.random.default_rng(2028)
    L = desc["box"][0]
    for k in "xyz":       # off the lattice, where forces are not all zero
        frame[k] = np.mod(np.asarray(frame[k]) + rng.uniform(-0.05, 0.05, len(frame[k])), L)
    ref, rsc, rcs = _oracle(orc, desc, frame)
    fref = _f(ref)
    out, sc, cs = _forces(atvb, ctx, desc, frame, 0, pairs=True)
    assert cs == rcs
    assert rms_rel(_f(out), fref) < 1e-10
    assert sc["energy"] == pytest.approx(rsc["energy"], rel=1e-10)
    out, sc, cs = _forces(atvb, ctx, desc, frame, 1, pairs=True)
    assert cs == rcs
    assert rms_rel(_f(out), fref) < 5e-6
