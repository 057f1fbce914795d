"""Known-answer tests of the oracle's per-type LJ tables and special pairs,
restating the reference's own cases (CPU only):

- tests/cpu/potentials/test_pair_lj_types.cpp: a single-type table equals
  the scalar path; unlike pairs mix by Lorentz-Berthelot; an explicit cross
  term overrides mixing; a type without an LJ site does not interact;
- tests/cpu/dynamics/test_lj_exclusions.cpp: on an all-trans united-atom
  chain, 1-2/1-3/1-4 exclusions remove the huge bonded LJ energy;
- coul_long.cpp:159-196: a special pair keeps erfc and subtracts
  (1 - f) k_e q_i q_j / r.
"""
import math

import numpy as np
import pytest

KE = 14.399645
RC, SKIN, BOX = 8.5, 1.0, 40.0


def lj_ref(eps, sigma, r, rc):
    s6 = (sigma / r) ** 6
    s6c = (sigma / rc) ** 6
    return 4 * eps * (s6 * s6 - s6) - 4 * eps * (s6c * s6c - s6c)


def _system(orc, pos, q=None, has_lj=1, eps=1.0, sigma=1.0, has_coul=0, alpha=0.3):
    n = len(pos)
    d = orc.make_desc(n, (BOX, BOX, BOX), nl_cutoff=RC, skin=SKIN, has_lj=has_lj,
                      lj_eps=eps, lj_sigma=sigma, lj_rc=RC, has_coul=has_coul,
                      coul_alpha=alpha, coul_rc=RC)
    s = orc.OracleSystem(d)
    p = np.asarray(pos, dtype=np.float64) + BOX / 2
    s.set_state(p[:, 0], p[:, 1], p[:, 2], q=q)
    return s


def _energy(s):
    s.build_list()
    s.compute_forces()
    sc = s.scalars()
    return sc["e_lj"] + sc["e_coul"]


def test_single_type_table_equals_scalar_path(orc):
    eps, sigma, r = 0.0104, 3.4, 4.0
    plain = _system(orc, [[0, 0, 0], [r, 0, 0]], eps=eps, sigma=sigma)
    e_plain = _energy(plain)
    table = _system(orc, [[0, 0, 0], [r, 0, 0]], eps=123.0, sigma=9.9)
    table.set_lj_types([(0, 0, eps, sigma)], [0, 0])
    assert e_plain == pytest.approx(lj_ref(eps, sigma, r, RC), abs=1e-13)
    assert _energy(table) == pytest.approx(e_plain, abs=1e-12)


def test_unlike_pairs_mix_by_lorentz_berthelot(orc):
    e1, s1, e2, s2, r = 0.01, 3.0, 0.04, 4.0, 4.2
    coeffs = [(0, 0, e1, s1), (1, 1, e2, s2)]
    for types, (e, sg) in (([0, 1], (math.sqrt(e1 * e2), 0.5 * (s1 + s2))),
                           ([0, 0], (e1, s1)), ([1, 1], (e2, s2))):
        s = _system(orc, [[0, 0, 0], [r, 0, 0]])
        s.set_lj_types(coeffs, types)
        assert _energy(s) == pytest.approx(lj_ref(e, sg, r, RC), abs=1e-13)


def test_explicit_cross_term_overrides_mixing(orc):
    r = 5.5
    s = _system(orc, [[0, 0, 0], [r, 0, 0]])
    s.set_lj_types([(0, 0, 0.01, 3.0), (1, 1, 0.04, 4.0), (0, 1, 0.9, 5.0)], [0, 1])
    assert _energy(s) == pytest.approx(lj_ref(0.9, 5.0, r, RC), abs=1e-12)


def test_type_without_lj_site_does_not_interact(orc):
    # types: 0 = O (LJ site), 1 = H (none); only O-O is set
    coeffs = [(0, 0, 0.0065, 3.15), (1, 1, 0.0, 1.0)]
    coeffs_no_h = [(0, 0, 0.0065, 3.15)]
    for types, r in (([1, 1], 0.96), ([0, 1], 1.0)):
        s = _system(orc, [[0, 0, 0], [r, 0, 0]])
        s.set_lj_types(coeffs_no_h, types)
        # H has no diagonal: every pair involving H has eps = 0
        assert _energy(s) == pytest.approx(0.0, abs=1e-14)
    oo = _system(orc, [[0, 0, 0], [3.5, 0, 0]])
    oo.set_lj_types(coeffs, [0, 0])
    e = _energy(oo)
    assert e == pytest.approx(lj_ref(0.0065, 3.15, 3.5, RC), abs=1e-13)
    assert e < 0.0


def test_bad_type_coefficient_rejected(orc):
    s = _system(orc, [[0, 0, 0], [3.0, 0, 0]])
    with pytest.raises(ValueError):
        s.set_lj_types([(0, 0, 0.01, 0.0)], [0, 0])


def chain(n, bond=1.529, angle_deg=111.7):
    """All-trans zigzag chain in the xy plane."""
    th = math.radians(angle_deg) / 2
    dx, dy = bond * math.sin(th), bond * math.cos(th)
    return [[k * dx - n * dx / 2, (k % 2) * dy, 0.0] for k in range(n)]


def special_pairs(n_atoms, bonds):
    """1-2, 1-3, 1-4 partners from bond topology (nearest class wins)."""
    adj = [set() for _ in range(n_atoms)]
    for a, b in bonds:
        adj[a].add(b)
        adj[b].add(a)
    out = {}
    for i in range(n_atoms):
        seen = {i: 0}
        frontier = [i]
        for depth in (1, 2, 3):
            nxt = []
            for u in frontier:
                for v in adj[u]:
                    if v not in seen:
                        seen[v] = depth
                        nxt.append(v)
            frontier = nxt
        for j, dpt in seen.items():
            if j > i and dpt > 0:
                out[(i, j)] = dpt
    return out


def test_chain_exclusions_remove_bonded_lj(orc):
    n = 20
    pos = chain(n)
    bonds = [(k, k + 1) for k in range(n - 1)]
    sp = special_pairs(n, bonds)
    eps, sigma = 0.00395, 4.01
    plain = _system(orc, pos, eps=eps, sigma=sigma)
    e_plain = _energy(plain)
    excl = _system(orc, pos, eps=eps, sigma=sigma)
    pairs = np.array(list(sp.keys()), dtype=np.int32)
    excl.set_special(pairs, np.zeros(len(pairs)), np.ones(len(pairs)))
    e_excl = _energy(excl)
    assert e_plain > 1e3
    assert abs(e_excl) < 1.0
    # 1-4 at half strength (Amber-like): exactly half the 1-4 terms come back
    half = _system(orc, pos, eps=eps, sigma=sigma)
    s_lj = np.array([0.0 if sp[(int(a), int(b))] < 3 else 0.5 for a, b in pairs])
    half.set_special(pairs, s_lj, np.ones(len(pairs)))
    p = np.asarray(pos)
    e14 = sum(lj_ref(eps, sigma, float(np.linalg.norm(p[a] - p[b])), RC)
              for (a, b), dpt in sp.items() if dpt == 3)
    assert _energy(half) == pytest.approx(e_excl + 0.5 * e14, rel=1e-12)


@pytest.mark.parametrize("f", [0.0, 0.5, 0.8333])
def test_coulomb_special_pair_compensation(orc, f):
    r, alpha = 1.2, 0.3
    s = _system(orc, [[0, 0, 0], [r, 0, 0]], q=[1.0, -1.0], has_lj=0, has_coul=1, alpha=alpha)
    s.set_special(np.array([[0, 1]]), np.array([1.0]), np.array([f]))
    s.build_list()
    s.compute_forces()
    sc = s.scalars()
    pref = KE * (1.0) * (-1.0) / r
    want = pref * math.erfc(alpha * r) - (1.0 - f) * pref
    assert sc["e_coul"] == pytest.approx(want, rel=1e-13)
    fx = s.state()["fx"]
    fc = pref * (math.erfc(alpha * r) + 2 / math.sqrt(math.pi) * alpha * r
                 * math.exp(-(alpha * r) ** 2)) - (1.0 - f) * pref
    # force on atom 0 along -x (dx = x0 - x1 = -r)
    assert fx[0] == pytest.approx(fc / r * (-r) / r, rel=1e-12)
