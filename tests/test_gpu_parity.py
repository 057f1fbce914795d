"""Parity of the CUDA path (through the C ABI) with the CPU FP64 oracle.

Tolerances (RMS relative force error over all atoms,
sqrt(sum |F - F_ref|^2) / sqrt(sum |F_ref|^2)):
  FP64 build  <= 1e-6 (observed ~1e-12 without PME; the 2^-40 e fixed-point
              PME grid keeps it near 1e-9 with PME)
  mixed build <= 5e-6
The pair set (unordered pairs within cutoff+skin) must be EQUAL.
"""
import numpy as np
import pytest

from atomiverse_b200 import workloads as W
from conftest import oracle_system, rms_rel

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-6
MIXED_TOL = 5e-6


def _pairs_set(pi, pj):
    a = np.minimum(pi, pj).astype(np.int64)
    b = np.maximum(pi, pj).astype(np.int64)
    return np.unique(a * (1 << 32) + b)


def _forces(frame):
    return np.stack([frame["fx"], frame["fy"], frame["fz"]], axis=1)


def _gpu_forces(atvb, ctx, desc, frame, precision=None):
    d = dict(desc)
    if precision is not None:
        d["precision"] = precision
    d.setdefault("stress_required", 1)
    sys = atvb.System(ctx, d, frame)
    sys.compute_forces()
    out, sc = sys.download()
    return sys, out, sc


def _oracle_forces(orc, desc, frame):
    s = oracle_system(orc, desc, frame)
    s.build_list()
    s.compute_forces()
    return s, s.state(), s.scalars()


def _small_rocksalt(ncell=16, seed=7, rc=12.0):
    L = ncell * 2.82
    K = max(8, round(L / 0.94))
    return W.rocksalt_melt(ncell=ncell, seed=seed, grid=(K, K, K), rc=rc)


def _jittered(desc_frame, amp=0.05, seed=1):
    """A perfect lattice has zero net force on every atom, which makes a
    relative force error meaningless; move every atom by U(-amp, amp)."""
    desc, frame = desc_frame
    rng = np.random.default_rng(seed)
    L = desc["box"][0]
    for k in ("x", "y", "z"):
        frame[k] = np.mod(frame[k] + rng.uniform(-amp, amp, len(frame[k])), L)
    return desc, frame


CASES = {
    "lj_fcc_4000": lambda: _jittered(W.lj_fcc(ncell=10)),
    "lj_small_aliased_256": lambda: _jittered(W.lj_fcc(ncell=4, n_keep=256, seed=11)),
    "rocksalt_4096": lambda: _small_rocksalt(16),
    "rocksalt_1000": lambda: _small_rocksalt(10, seed=3),
}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("precision", [0, 1])
def test_pair_set_equals_oracle(atvb, ctx, orc, case, precision):
    desc, frame = CASES[case]()
    d = dict(desc, precision=precision)
    sys = atvb.System(ctx, d, frame)
    gi, gj = sys.pairs()
    s = oracle_system(orc, desc, frame)
    oi, oj = s.pairs()
    g = _pairs_set(gi, gj)
    o = _pairs_set(oi, oj)
    assert len(gi) == len(g), "GPU list holds a duplicate pair"
    assert g.size == o.size
    assert np.array_equal(g, o)


@pytest.mark.parametrize("case", list(CASES))
def test_forces_fp64(atvb, ctx, orc, case):
    desc, frame = CASES[case]()
    _, out, sc = _gpu_forces(atvb, ctx, desc, frame, precision=0)
    _, ref, rsc = _oracle_forces(orc, desc, frame)
    err = rms_rel(_forces(out), _forces(ref))
    assert err <= FP64_TOL, err
    assert sc["energy"] == pytest.approx(rsc["energy"], rel=1e-9, abs=1e-7)
    assert np.allclose(sc["stress"], rsc["virial"], rtol=1e-8,
                       atol=1e-8 * np.abs(rsc["virial"]).max())


@pytest.mark.parametrize("case", list(CASES))
def test_forces_mixed(atvb, ctx, orc, case):
    desc, frame = CASES[case]()
    _, out, sc = _gpu_forces(atvb, ctx, desc, frame, precision=1)
    _, ref, rsc = _oracle_forces(orc, desc, frame)
    err = rms_rel(_forces(out), _forces(ref))
    assert err <= MIXED_TOL, err
    assert sc["energy"] == pytest.approx(rsc["energy"], rel=2e-5)


def test_madelung_nacl(atvb, ctx):
    """64-ion rock salt, d = 2.82 A, rc = 1.9 d, alpha = 3.5 / rc, spacing
    0.5, order 6 (tests/cuda/longrange/test_pme_coul.cu:46-69 of the
    reference, which accepts rel 3e-3)."""
    d, n = 2.82, 4
    g = np.arange(n)
    ijk = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pos = ijk * d
    q = np.where(ijk.sum(1) % 2 == 0, 1.0, -1.0)
    L = n * d
    rc = 1.9 * d
    alpha = 3.5 / rc
    desc = dict(n_atoms=64, box=(L, L, L), nl_cutoff=rc, nl_skin=0.2, coul_enabled=1,
                coul_alpha=alpha, coul_cutoff=rc, pme_enabled=1, pme_alpha=alpha,
                pme_grid_spacing=0.5, pme_order=6, dt=1.0)
    frame = {"x": pos[:, 0], "y": pos[:, 1], "z": pos[:, 2], "charge": q,
             "mass": np.ones(64)}
    sys = atvb.System(ctx, desc, frame)
    sys.compute_forces()
    e = sys.scalars()["energy"]
    e_exp = -0.5 * 64 * 1.747564594633182 * 14.399645 / d
    assert abs(e / e_exp - 1.0) < 5e-4


def _traj_compare(atvb, ctx, orc, desc, frame, steps, tol_x, setup=None, oracle_over=None):
    sys = atvb.System(ctx, desc, frame)
    if setup is not None:
        setup(sys)
    sys.compute_forces()
    sys.step(steps)
    out, sc = sys.download()
    s = oracle_system(orc, desc, frame, **(oracle_over or {}))
    s.build_list()
    s.compute_forces()
    s.run(steps)
    ref = s.state()
    rsc = s.scalars()
    L = np.array(desc["box"][:3]) if len(desc["box"]) == 3 else np.array(desc["box"][::4])
    for k, ax in zip("xyz", range(3)):
        d = out[k] - ref[k]
        d -= L[ax] * np.rint(d / L[ax])
        assert np.abs(d).max() < tol_x, (k, np.abs(d).max())
    v_err = rms_rel(np.stack([out["vx"], out["vy"], out["vz"]], 1),
                    np.stack([ref["vx"], ref["vy"], ref["vz"]], 1))
    assert v_err < 1e3 * tol_x, v_err
    assert sc["step"] == steps
    assert sc["rebuilds"] == rsc["rebuilds"]
    return sc, rsc


def test_trajectory_nve_lj_fp64(atvb, ctx, orc):
    desc, frame = W.lj_fcc(ncell=10)
    sc, rsc = _traj_compare(atvb, ctx, orc, desc, frame, 100, 1e-9)
    assert sc["energy"] == pytest.approx(rsc["energy"], rel=1e-9)
    assert sc["kinetic"] == pytest.approx(rsc["kinetic"], rel=1e-9)


def test_trajectory_nose_hoover_rocksalt_fp64(atvb, ctx, orc):
    desc, frame = _small_rocksalt(10, seed=5)
    sc, rsc = _traj_compare(atvb, ctx, orc, desc, frame, 30, 1e-8)
    assert sc["nh_xi"] == pytest.approx(rsc["xi"], rel=1e-6, abs=1e-12)
    assert sc["energy"] == pytest.approx(rsc["energy"], rel=1e-8)


def test_trajectory_langevin_fp64(atvb, ctx, orc):
    desc, frame = W.lj_fcc(ncell=5, thermostat=2, seed=9)
    _traj_compare(atvb, ctx, orc, desc, frame, 40, 1e-8)


def test_trajectory_langevin_ramp_fp64(atvb, ctx, orc):
    """FixLangevin(T, 3 T).set_run_span(5, 35) (fix_langevin.cpp:94-104):
    the setpoint ramps over steps 5-35 and holds after them; the trajectory
    follows the oracle's, which ramps the same way."""
    desc, frame = W.lj_fcc(ncell=5, thermostat=2, seed=9)
    T0 = desc["temperature"]
    ramp = dict(lang_T_stop=3.0 * T0, lang_nfirst=5, lang_nlast=35)
    _traj_compare(atvb, ctx, orc, desc, frame, 45, 1e-8,
                  setup=lambda s: s.set_langevin_ramp(3.0 * T0, 5, 35), oracle_over=ramp)


def test_langevin_ramp_heats(atvb, ctx):
    """A ramp T -> 3 T over 400 steps ends clearly hotter than the
    constant setpoint from the same state (damping time 0.1 tau)."""
    desc, frame = W.lj_fcc(ncell=6, thermostat=2, seed=4, damp_tau=0.1)
    T0 = desc["temperature"]
    kin = []
    for ramp in (False, True):
        s = atvb.System(ctx, desc, frame)
        if ramp:
            s.set_langevin_ramp(3.0 * T0, 0, 400)
        s.compute_forces()
        s.step(600)
        kin.append(s.scalars()["kinetic"])
        s.close()
    assert kin[1] > 2.0 * kin[0], kin
    with pytest.raises(atvb.AtvbError):
        d2, f2 = W.lj_fcc(ncell=4)                 # NVE: no Langevin to ramp
        atvb.System(ctx, d2, f2).set_langevin_ramp(2.0, 0, 10)


def test_bitwise_reproducible_mixed(atvb, ctx):
    desc, frame = _small_rocksalt(12, seed=2)
    runs = []
    for _ in range(2):
        sys = atvb.System(ctx, dict(desc, precision=1), frame)
        sys.compute_forces()
        sys.step(25)
        out, sc = sys.download()
        runs.append((out, sc))
    for k in ("x", "vx", "fx", "fy"):
        assert np.array_equal(runs[0][0][k], runs[1][0][k]), k
    assert runs[0][1]["energy"] == runs[1][1]["energy"]
