"""The CPU oracle pinned against the reference's known answers (CPU only).

Known-answer sources (reference tree paths):
  tests/cpu/longrange/test_pme_math.cpp:19-46    good_fft_size pins, B-spline
  tests/cpu/longrange/test_pme_coul.cpp:157-244  Madelung, PME vs Ewald, FD forces
  tests/cuda/potentials/test_pair_lj_tile_step0.cu:102-136  two-atom LJ
  tests/cpu/potentials/test_pair_virial.cpp:233-262         virial identity
  tests/cpu/dynamics/test_full_neighbor_list.cpp:107-151    brute-force pair set
  regressions/md/lj_argon/REFERENCE.md           NVE drift gates
plus golden vectors produced by the reference's own PME headers
(tests/golden/make_golden.py).
"""
import os

import numpy as np
import pytest

from atomiverse_b200 import workloads as W
from conftest import oracle_system, rms_rel

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "pme_reference.npz")
MADELUNG = 1.747564594633182
KE = 14.399645


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN)


def test_good_fft_size_pins(orc, gold):
    for n, k in [(1, 4), (2, 4), (3, 4), (4, 4), (11, 12), (13, 14), (15, 15),
                 (16, 16), (23, 24), (49, 49)]:
        assert orc.good_fft_size(n) == k
    for n, k in gold["good_fft_size"]:
        assert orc.good_fft_size(int(n)) == int(k)


def test_bspline_matches_reference_bitwise(orc, gold):
    for n in (4, 5, 6, 8):
        for k, fr in enumerate((0.0, 0.1, 0.33, 0.5, 0.999)):
            th, dth = orc.bspline(fr, n)
            assert np.array_equal(th, gold[f"bspline_{n}_theta"][k])
            assert np.array_equal(dth, gold[f"bspline_{n}_dtheta"][k])
            assert abs(th.sum() - 1.0) < 1e-12
    th, _ = orc.bspline(0.0, 4)
    assert np.allclose(th, [1 / 6, 4 / 6, 1 / 6, 0.0], atol=1e-14)


def test_spline_moduli_match_reference(orc, gold):
    for K, n in ((12, 4), (24, 6), (30, 4), (49, 5)):
        assert np.allclose(orc.spline_moduli(K, n), gold[f"moduli_{K}_{n}"], rtol=1e-14, atol=0)


def test_fft_matches_numpy(orc):
    rng = np.random.default_rng(0)
    for shape in [(12, 12, 12), (6, 10, 14), (7, 9, 15), (16, 8, 4)]:
        a = rng.normal(size=shape) + 1j * rng.normal(size=shape)
        assert np.allclose(orc.fft3d(a, -1), np.fft.fftn(a), rtol=0, atol=1e-10)
        assert np.allclose(orc.fft3d(a, +1), np.fft.ifftn(a) * a.size, rtol=0, atol=1e-10)


def test_pme_matches_reference_golden(orc, gold):
    e, f, w = orc.pme(*gold["fd_pos"].T, gold["fd_q"], (8.0, 8.0, 8.0), 0.45, (12, 12, 12), 6)
    assert e == pytest.approx(gold["fd_energy"][0], rel=1e-12, abs=1e-12)
    assert np.allclose(f, gold["fd_force"], rtol=0, atol=1e-12)
    assert np.allclose(w, gold["fd_virial"], rtol=1e-10, atol=1e-12)
    L = gold["salt_L"]
    e, f, w = orc.pme(*gold["salt_pos"].T, gold["salt_q"], L, 0.55, (10, 10, 18), 4)
    assert e == pytest.approx(gold["salt_energy"][0], rel=1e-12)
    assert np.allclose(f, gold["salt_force"], rtol=0, atol=1e-11)
    assert np.allclose(w, gold["salt_virial"], rtol=1e-10, atol=1e-10)


def _rocksalt(n=4, d=2.82):
    g = np.arange(n)
    ijk = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    return ijk * d, np.where(ijk.sum(1) % 2 == 0, 1.0, -1.0), n * d


def _coul_system(orc, pos, q, L, rc, alpha, K, order, skin=0.1):
    d = orc.make_desc(len(q), (L, L, L), nl_cutoff=rc, skin=skin, has_coul=1,
                      coul_alpha=alpha, coul_rc=rc, has_pme=1, pme_alpha=alpha,
                      pme_K=(K, K, K), pme_order=order)
    s = orc.OracleSystem(d)
    s.set_state(pos[:, 0], pos[:, 1], pos[:, 2], q=q)
    s.build_list()
    s.compute_forces()
    return s


def test_madelung_nacl(orc):
    pos, q, L = _rocksalt()
    rc = 1.9 * 2.82
    alpha = 3.5 / rc
    K = orc.good_fft_size(int(np.ceil(L / 0.5)))
    s = _coul_system(orc, pos, q, L, rc, alpha, K, 6, skin=0.2)
    e_exp = -0.5 * 64 * MADELUNG * KE / 2.82
    assert abs(s.scalars()["energy"] / e_exp - 1.0) < 5e-4


def test_pme_agrees_with_ewald(orc):
    pos, q, L = _rocksalt()
    rc = 1.9 * 2.82
    alpha = 3.5 / rc
    K = orc.good_fft_size(int(np.ceil(L / 0.5)))
    s = _coul_system(orc, pos, q, L, rc, alpha, K, 6, skin=0.2)
    sc = s.scalars()
    e_ew, f_ew, w_ew = orc.ewald_recip(pos[:, 0], pos[:, 1], pos[:, 2], q, (L, L, L), alpha, 1e-8)
    e_pme = sc["energy"] - sc["e_coul"]
    assert abs(e_pme / e_ew - 1.0) < 5e-4


def test_pme_finite_difference_forces(orc, gold):
    pos, q = gold["fd_pos"], gold["fd_q"]

    def energy(p):
        s = _coul_system(orc, p, q, 8.0, 3.9, 0.45, 12, 6, skin=0.05)
        return s.scalars()["energy"], s.state()

    _, st = energy(pos)
    F = np.stack([st["fx"], st["fy"], st["fz"]], 1)
    h = 1e-5
    for a in range(4):
        for ax in range(3):
            p = pos.copy()
            p[a, ax] += h
            ep, _ = energy(p)
            p[a, ax] -= 2 * h
            em, _ = energy(p)
            assert abs(F[a, ax] + (ep - em) / (2 * h)) < 2e-3


def _brute_pairs(x, y, z, L, rl):
    p = np.stack([x, y, z], 1)
    n = len(p)
    out = []
    for i in range(n):
        d = p[i] - p[i + 1:]
        for k in range(3):
            h = 0.5 * L[k]
            d[:, k] = np.where(d[:, k] > h, d[:, k] - L[k], np.where(d[:, k] < -h, d[:, k] + L[k], d[:, k]))
        r2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        js = np.nonzero(r2 < rl * rl)[0] + i + 1
        out.extend(i * (1 << 32) + js)
    return np.sort(np.array(out, dtype=np.int64))


@pytest.mark.parametrize("case", ["fcc_500", "aliased_256", "rocksalt_1000", "ragged_97"])
def test_pair_set_equals_brute_force(orc, case):
    if case == "fcc_500":
        desc, fr = W.lj_fcc(ncell=5)
    elif case == "aliased_256":
        desc, fr = W.lj_fcc(ncell=4, n_keep=256)
    elif case == "rocksalt_1000":
        desc, fr = W.rocksalt_melt(ncell=10, grid=(30, 30, 30))
    else:
        desc, fr = W.lj_fcc(ncell=3, n_keep=97, rho=0.5)
    rng = np.random.default_rng(3)
    L = desc["box"]
    for k in "xyz":
        fr[k] = np.mod(fr[k] + rng.uniform(-0.1, 0.1, len(fr[k])), L[0])
    s = oracle_system(orc, desc, fr)
    pi, pj = s.pairs()
    assert np.all(pj > pi)
    got = np.sort(pi.astype(np.int64) * (1 << 32) + pj)
    assert len(np.unique(got)) == len(got)
    rl = desc["nl_cutoff"] + desc["nl_skin"]
    ref = _brute_pairs(fr["x"], fr["y"], fr["z"], L, rl)
    assert np.array_equal(got, ref)


def test_lj_two_atoms_at_minimum(orc):
    r0 = 2 ** (1 / 6)
    d = orc.make_desc(2, (10.0, 10.0, 10.0), nl_cutoff=2.5, skin=0.3, has_lj=1,
                      lj_eps=1.0, lj_sigma=1.0, lj_rc=2.5)
    s = orc.OracleSystem(d)
    s.set_state(np.array([1.0, 1.0 + r0]), np.array([1.0, 1.0]), np.array([1.0, 1.0]))
    s.build_list()
    s.compute_forces()
    st = s.state()
    shift = 4.0 * (2.5 ** -12 - 2.5 ** -6)
    assert s.scalars()["energy"] == pytest.approx(-1.0 - shift, abs=1e-12)
    assert abs(st["fx"][0]) < 1e-12 and abs(st["fx"][1]) < 1e-12


def test_lj_virial_trace_identity(orc):
    """tr W = -3 V dE/dV under uniform scaling (test_pair_virial.cpp:255)."""
    desc, fr = W.lj_fcc(ncell=5, rho=0.8442)
    rng = np.random.default_rng(2)
    L = desc["box"][0]
    for k in "xyz":
        fr[k] = np.mod(fr[k] + rng.uniform(-0.05, 0.05, len(fr[k])), L)

    def energy(scale):
        d = dict(desc, box=(L * scale,) * 3, nl_skin=0.6)
        f2 = {k: fr[k] * scale for k in "xyz"}
        s = oracle_system(orc, d, f2)
        s.build_list()
        s.compute_forces()
        return s.scalars()

    sc = energy(1.0)
    h = 1e-6
    dEds = (energy(1 + h)["energy"] - energy(1 - h)["energy"]) / (2 * h)
    # V = (sL)^3 -> dE/dV = dE/ds / (3 V) at s = 1
    tr = sc["virial"][:3].sum()
    assert tr == pytest.approx(-dEds, rel=1e-6)


def test_nve_drift_gates(orc):
    """lj_argon gates: max|E-E0|/(N eps) <= 1e-2; second-half drift <= 4x first."""
    desc, fr = W.lj_fcc(ncell=5)
    s = oracle_system(orc, desc, fr)
    s.build_list()
    s.compute_forces()
    _, hist = s.run(400, history=True)
    etot = hist[:, 0] + hist[:, 1]
    n = desc["n_atoms"]
    dev = np.abs(etot - etot[0]).max() / n
    assert dev <= 1e-2
    half = len(etot) // 2
    d1 = abs(etot[half - 1] - etot[0])
    d2 = abs(etot[-1] - etot[half])
    assert d2 <= 4 * max(d1, 1e-6 * n)


def test_skin_gating(orc):
    desc, fr = W.lj_fcc(ncell=5)
    for k in ("vx", "vy", "vz"):
        fr[k] = np.zeros_like(fr[k])
    s = oracle_system(orc, desc, fr)
    s.build_list()
    assert s.run(20) == 0  # frozen lattice: no rebuilds
    desc2 = dict(desc)
    fr2 = dict(fr)
    fr2["vx"] = np.zeros_like(fr["vx"])
    fr2["vx"][0] = 0.2 / desc["dt"] / 2  # 0.2 sigma over two steps > skin/2
    s2 = oracle_system(orc, desc2, fr2)
    s2.build_list()
    assert s2.run(3) >= 1


def test_langevin_stream(orc):
    a = orc.gauss3(7, 3, 11)
    b = orc.gauss3(7, 3, 11)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, orc.gauss3(7, 4, 11))
    xs = np.concatenate([orc.gauss3(1, 0, t) for t in range(1, 4001)])
    assert abs(xs.mean()) < 0.05 and abs(xs.std() - 1.0) < 0.05


def test_nose_hoover_thermostats(orc):
    desc, fr = W.lj_fcc(ncell=4, t_star=0.5)
    T = 1.0 / 8.617333262e-5
    s = oracle_system(orc, desc, fr, thermostat=1, temperature=T, tau=20 * desc["dt"])
    s.build_list()
    s.compute_forces()
    _, hist = s.run(600, history=True)
    n = desc["n_atoms"]
    t_kin = 2 * hist[-200:, 1] / ((3 * n - 3) * 8.617333262e-5)
    assert t_kin.mean() == pytest.approx(T, rel=0.15)
