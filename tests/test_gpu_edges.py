"""Edge cases of the device path, against the oracle or a known answer:

- two atoms at the LJ minimum 2^(1/6) sigma: zero force, energy -eps minus
  the shift (tests/cuda/potentials/test_pair_lj_tile_step0.cu:102-136);
- a lone atom: no neighbours, zero force and energy;
- a ragged 97-atom, low-density, non-cubic box with edges between 2 and 3
  (rc + skin) (two bins per axis, so the +1 and -1 neighbours alias): pair
  set and forces (an edge below 2 (rc + skin) is refused on the host);
- coordinates outside [0, L) and on the box faces: wrapped on upload
  (cpu/frame/pbc.h:48-50), so the forces are those of the wrapped frame;
- neutral ions beside charged ones with real-space Ewald and PME (real-space
  terms with q == 0 skipped, coul_long.cpp:146-222) and a net charge;
- an empty system is refused when it is created, and a system or batch with
  nothing uploaded refuses to step, each with an error the caller can read.
"""
import numpy as np
import pytest

from atomiverse_b200 import workloads as W
from conftest import oracle_system, rms_rel

pytestmark = pytest.mark.gpu


def _f(fr):
    return np.stack([fr["fx"], fr["fy"], fr["fz"]], 1)


def _pairs(pi, pj):
    a = np.minimum(pi, pj).astype(np.int64)
    b = np.maximum(pi, pj).astype(np.int64)
    return np.unique(a * (1 << 32) + b)


def _lj_desc(n, box, **kw):
    d = dict(n_atoms=n, box=box, nl_cutoff=2.5, nl_skin=0.3, lj_enabled=1,
             lj_epsilon=1.0, lj_sigma=1.0, lj_cutoff=2.5, dt=0.005, stress_required=1)
    d.update(kw)
    return d


@pytest.mark.parametrize("precision,tol,ftol", [(0, 1e-9, 1e-12), (1, 1e-6, 5e-5)])
def test_two_atoms_at_lj_minimum(atvb, ctx, precision, tol, ftol):
    """Energies are summed in 2^-32 eV fixed point (order-independent), so
    each per-atom term carries up to 1.2e-10 eV of rounding.  FP32 distances
    put the mixed build's r within ~1e-7 r of 2^(1/6); the force there is
    V''(r0) dr ~ 57 dr, hence its looser force bound."""
    r0 = 2.0 ** (1.0 / 6.0)
    desc = _lj_desc(2, (10.0, 10.0, 10.0), precision=precision)
    frame = dict(x=np.array([1.0, 1.0 + r0]), y=np.array([1.0, 1.0]),
                 z=np.array([1.0, 1.0]), mass=np.ones(2))
    s = atvb.System(ctx, desc, frame)
    s.compute_forces()
    out, sc = s.download()
    s.close()
    shift = 4.0 * (2.5 ** -12 - 2.5 ** -6)
    assert sc["energy"] == pytest.approx(-1.0 - shift, abs=tol)
    assert np.abs(_f(out)).max() < ftol


def test_lone_atom(atvb, ctx):
    desc = _lj_desc(1, (10.0, 10.0, 10.0))
    frame = dict(x=np.array([3.0]), y=np.array([4.0]), z=np.array([5.0]),
                 vx=np.array([0.01]), vy=np.zeros(1), vz=np.zeros(1), mass=np.ones(1))
    s = atvb.System(ctx, desc, frame)
    s.compute_forces()
    s.step(10)
    out, sc = s.download()
    s.close()
    assert sc["energy"] == 0.0
    assert np.abs(_f(out)).max() == 0.0
    assert out["x"][0] == pytest.approx(3.0 + 10 * 0.005 * 0.01, rel=1e-13)
    assert out["y"][0] == 4.0 and out["z"][0] == 5.0


def _ragged_97(seed=4):
    rng = np.random.default_rng(seed)
    a = 1.2
    nx, ny, nz = 5, 5, 6
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"),
                 -1).reshape(-1, 3).astype(float)
    keep = np.sort(rng.choice(len(g), 97, replace=False))
    pos = (g[keep] + 0.5 + rng.uniform(-0.12, 0.12, (97, 3))) * a
    box = (nx * a, ny * a, nz * a)
    frame = dict(x=np.mod(pos[:, 0], box[0]), y=np.mod(pos[:, 1], box[1]),
                 z=np.mod(pos[:, 2], box[2]), mass=np.ones(97))
    return _lj_desc(97, box), frame


@pytest.mark.parametrize("precision,tol", [(0, 1e-11), (1, 5e-6)])
def test_ragged_noncubic_aliased_box(atvb, ctx, orc, precision, tol):
    desc, frame = _ragged_97()
    rl = desc["nl_cutoff"] + desc["nl_skin"]
    assert 2 * rl < min(desc["box"]) < 3 * rl     # two bins per axis: +1 and -1 alias
    s = atvb.System(ctx, dict(desc, precision=precision), frame)
    s.compute_forces()
    out, sc = s.download()
    pi, pj = s.pairs()
    s.close()
    o = oracle_system(orc, desc, frame)
    o.build_list()
    oi, oj = o.pairs()
    assert np.array_equal(_pairs(pi, pj), _pairs(oi, oj))
    o.compute_forces()
    assert rms_rel(_f(out), _f(o.state())) < tol
    # energies sum in 2^-32 eV fixed point: ~1e-10 eV per atom
    assert sc["energy"] == pytest.approx(o.scalars()["energy"], rel=max(tol, 1e-10))


def test_coordinates_outside_the_box_are_wrapped(atvb, ctx):
    desc, frame = W.lj_fcc(ncell=8, seed=9)
    rng = np.random.default_rng(5)
    L = np.array(desc["box"], dtype=float)
    n = len(frame["x"])
    moved = {k: np.array(frame[k], dtype=float) for k in "xyz"}
    for ax, k in enumerate("xyz"):
        shift = rng.integers(-3, 4, n).astype(float)
        moved[k] = moved[k] + shift * L[ax]
    moved["x"][0] = 0.0
    moved["x"][1] = L[0]                 # on the far face: the same as 0
    moved["y"][2] = -0.0
    moved["z"][3] = -L[2]
    wrapped = {k: np.mod(moved[k], L[ax]) for ax, k in enumerate("xyz")}
    res = []
    for pos in (moved, wrapped):
        fr = dict(frame, **pos)
        s = atvb.System(ctx, dict(desc, stress_required=1), fr)
        s.compute_forces()
        out, sc = s.download()
        s.close()
        res.append((out, sc))
    (a, sa), (b, sb) = res
    for ax, k in enumerate("xyz"):
        # x - L floor(x / L), as pbc.h:48-50 writes it, may leave -ulp when
        # x / L rounds up to an integer
        assert np.all(a[k] >= -1e-13 * L[ax]) and np.all(a[k] < L[ax])
        d = a[k] - b[k]
        d -= L[ax] * np.rint(d / L[ax])
        assert np.abs(d).max() < 1e-12
    assert rms_rel(_f(a), _f(b)) < 1e-12
    assert sa["energy"] == pytest.approx(sb["energy"], rel=1e-12)


@pytest.mark.parametrize("precision,tol", [(0, 1e-6), (1, 5e-6)])
def test_neutral_ions_and_net_charge(atvb, ctx, orc, precision, tol):
    desc, frame = W.rocksalt_melt(ncell=10, seed=3, grid=(30, 30, 30), rc=12.0)
    q = np.array(frame["charge"], dtype=float)
    q[::5] = 0.0                          # neutral sites; the net charge is no longer 0
    q[1::7] *= 0.5
    assert abs(q.sum()) >= 1.0
    frame = dict(frame, charge=q)
    s = atvb.System(ctx, dict(desc, precision=precision, stress_required=1), frame)
    s.compute_forces()
    out, sc = s.download()
    s.close()
    o = oracle_system(orc, desc, frame)
    o.build_list()
    o.compute_forces()
    assert rms_rel(_f(out), _f(o.state())) < tol
    assert sc["energy"] == pytest.approx(o.scalars()["energy"], rel=tol)
    vir = o.scalars()["virial"]
    assert np.allclose(sc["stress"], vir, rtol=1e-5, atol=1e-6 * np.abs(vir).max())


def test_empty_and_unuploaded_systems_are_refused(atvb, ctx):
    with pytest.raises(atvb.AtvbError, match="n_atoms"):
        atvb.System(ctx, _lj_desc(0, (10.0, 10.0, 10.0)))
    s = atvb.System(ctx, _lj_desc(4, (10.0, 10.0, 10.0)))
    with pytest.raises(atvb.AtvbError, match="upload"):
        s.step(1)
    s.close()
    b = atvb.Batch(ctx, [(_lj_desc(4, (10.0, 10.0, 10.0)), None)])
    with pytest.raises(atvb.AtvbError, match="upload"):
        b.step(1)
    b.close()
