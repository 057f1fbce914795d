"""Per-type LJ tables and special (bonded) pairs on the GPU, against the
oracle (k_pair_general): a three-type LJ mixture, and SPC/E-like water with
PME, intramolecular 1-2/1-3 exclusions and LJ on oxygen only; the pair set
is unchanged by the special-class bits; batches mix general and plain
systems with results equal to each system alone."""
import math

import numpy as np
import pytest

from conftest import oracle_system, rms_rel


def _mixture(n_cells=8, seed=5):
    rng = np.random.default_rng(seed)
    a = 1.6796  # FCC at rho* = 0.8442
    from atomiverse_b200 import workloads as W
    pos = W.fcc_sites(n_cells, a) + rng.uniform(-0.06, 0.06, size=(4 * n_cells ** 3, 3))
    n = len(pos)
    L = n_cells * a
    types = rng.integers(0, 3, size=n).astype(np.int32)
    coeffs = [(0, 0, 1.0, 1.0), (1, 1, 0.5, 0.88), (0, 1, 1.5, 0.8),  # explicit cross term
              (2, 2, 0.0, 1.0)]                                         # type 2: no LJ site
    desc = dict(n_atoms=n, box=(L, L, L), nl_cutoff=2.5, nl_skin=0.3, lj_enabled=1,
                lj_epsilon=1.0, lj_sigma=1.0, lj_cutoff=2.5, dt=0.02, stress_required=1)
    frame = dict(x=np.mod(pos[:, 0], L), y=np.mod(pos[:, 1], L), z=np.mod(pos[:, 2], L),
                 mass=np.ones(n), type=types)
    return desc, frame, coeffs


def _water(m=10, seed=7):
    """SPC/E-like rigid geometry on a cubic lattice, random orientations."""
    from atomiverse_b200 import workloads as W
    rng = np.random.default_rng(seed)
    d_oh, ang = 1.0, math.radians(109.47)
    spacing = 3.1
    L = m * spacing
    pos, typ, q, mass, bonds = [], [], [], [], []
    tag = 1
    for i in range(m):
        for j in range(m):
            for k in range(m):
                o = (np.array([i, j, k]) + 0.5) * spacing
                R, _ = np.linalg.qr(rng.normal(size=(3, 3)))
                h1 = o + R @ np.array([d_oh, 0, 0])
                h2 = o + R @ np.array([d_oh * math.cos(ang), d_oh * math.sin(ang), 0])
                pos += [o, h1, h2]
                typ += [0, 1, 1]
                q += [-0.8476, 0.4238, 0.4238]
                mass += [15.9994, 1.008, 1.008]
                bonds += [(tag, tag + 1), (tag, tag + 2)]
                tag += 3
    pos = np.mod(np.array(pos), L)
    n = len(pos)
    rc = 9.0
    alpha = W.recommend_alpha(rc, 1e-5)
    desc = dict(n_atoms=n, box=(L, L, L), nl_cutoff=rc, nl_skin=1.0, lj_enabled=1,
                lj_epsilon=0.0067, lj_sigma=3.166, lj_cutoff=rc, coul_enabled=1,
                coul_alpha=alpha, coul_cutoff=rc, pme_enabled=1, pme_alpha=alpha,
                pme_order=4, pme_grid=(32, 32, 32), dt=1.0, stress_required=1)
    frame = dict(x=pos[:, 0].copy(), y=pos[:, 1].copy(), z=pos[:, 2].copy(),
                 charge=np.array(q), mass=np.array(mass), type=np.array(typ, dtype=np.int32),
                 tag=np.arange(1, n + 1, dtype=np.int64))
    coeffs = [(0, 0, 0.0067, 3.166)]  # hydrogens carry no LJ site
    special = dict(lj=(0.0, 0.0, 0.0), coul=(0.0, 0.0, 0.0), bonds=bonds)
    return desc, frame, coeffs, special


def _special_pairs(n, bonds, lj, coul):
    """(pairs, s_lj, s_coul) by index from tag bonds (tags 1..n), 1-2/1-3/1-4."""
    adj = [set() for _ in range(n)]
    for a, b in bonds:
        adj[a - 1].add(b - 1)
        adj[b - 1].add(a - 1)
    pairs, sl, sc = [], [], []
    for i in range(n):
        seen = {i: 0}
        frontier = [i]
        for d in (1, 2, 3):
            nxt = []
            for u in frontier:
                for v in adj[u]:
                    if v not in seen:
                        seen[v] = d
                        nxt.append(v)
            frontier = nxt
        for j, d in seen.items():
            if j > i and d > 0 and (lj[d - 1] != 1.0 or coul[d - 1] != 1.0):
                pairs.append((i, j))
                sl.append(lj[d - 1])
                sc.append(coul[d - 1])
    return np.array(pairs, dtype=np.int32).reshape(-1, 2), np.array(sl), np.array(sc)


def _forces(out):
    return np.stack([out["fx"], out["fy"], out["fz"]], axis=1)


def _oracle(orc, desc, frame, coeffs, special=None):
    o = oracle_system(orc, desc, frame)
    o.set_lj_types(coeffs, frame["type"])
    if special is not None:
        p, sl, sc = _special_pairs(desc["n_atoms"], special["bonds"], special["lj"],
                                   special["coul"])
        o.set_special(p, sl, sc)
    o.build_list()
    o.compute_forces()
    return _forces(o.state()), o.scalars(), o


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [(0, 1e-6), (1, 5e-6)])
def test_lj_mixture_matches_oracle(atvb, ctx, orc, precision, tol):
    desc, frame, coeffs = _mixture()
    fo, so, _ = _oracle(orc, desc, frame, coeffs)
    s = atvb.System(ctx, dict(desc, precision=precision), frame, lj_types=coeffs)
    s.compute_forces()
    out, sc = s.download()
    assert rms_rel(_forces(out), fo) <= tol
    assert sc["energy_lj"] == pytest.approx(so["e_lj"], rel=10 * tol)
    assert np.allclose(sc["stress"], so["virial"], rtol=10 * tol, atol=1e-9 * np.abs(so["virial"]).max())


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [(0, 1e-6), (1, 5e-6)])
def test_water_with_exclusions_and_pme_matches_oracle(atvb, ctx, orc, precision, tol):
    desc, frame, coeffs, special = _water()
    fo, so, o = _oracle(orc, desc, frame, coeffs, special)
    s = atvb.System(ctx, dict(desc, precision=precision), frame, lj_types=coeffs,
                    special_bonds=special)
    s.compute_forces()
    out, sc = s.download()
    assert rms_rel(_forces(out), fo) <= tol
    assert sc["energy_coul"] == pytest.approx(so["e_coul"], rel=10 * tol)
    assert sc["energy_lj"] == pytest.approx(so["e_lj"], rel=10 * tol)
    assert sc["energy_recip"] + sc["energy_const"] == pytest.approx(
        so["e_recip"] + so["e_const"], rel=10 * tol)
    # the listed pair set is the plain FP64 one (class bits are not indices)
    if precision == 0:
        pi, pj = s.pairs()
        got = set(zip(np.minimum(pi, pj).tolist(), np.maximum(pi, pj).tolist()))
        oi, oj = o.pairs()
        want = set(zip(np.minimum(oi, oj).tolist(), np.maximum(oi, oj).tolist()))
        assert got == want


@pytest.mark.gpu
def test_general_and_plain_systems_batch_equals_alone(atvb, ctx):
    from atomiverse_b200 import workloads as W
    desc_m, frame_m, coeffs = _mixture(n_cells=6)
    desc_w, frame_w, coeffs_w, special = _water(m=8)
    plain = W.lj_fcc(ncell=5, seed=3, precision=1)
    items = [(dict(desc_m, precision=1), frame_m, dict(lj_types=coeffs)),
             (dict(desc_w, precision=1), frame_w, dict(lj_types=coeffs_w, special_bonds=special)),
             (plain[0], plain[1])]
    b = atvb.Batch(ctx, items)
    b.compute_forces()
    b.step(10)
    for k, it in enumerate(items):
        ob, _ = b.download(k)
        opts = it[2] if len(it) > 2 else {}
        s = atvb.System(ctx, it[0], it[1], **opts)
        s.compute_forces()
        s.step(10)
        oa, _ = s.download()
        s.close()
        for key in ("x", "y", "z", "vx", "vy", "vz"):
            assert np.array_equal(ob[key], oa[key]), (k, key)
    b.close()


@pytest.mark.gpu
def test_configuration_after_upload_is_refused(atvb, ctx):
    desc, frame, coeffs = _mixture(n_cells=4)
    s = atvb.System(ctx, desc, frame)
    with pytest.raises(atvb.AtvbError) as e:
        args, keep = atvb._lj_type_args(coeffs)
        atvb.check(s.lib.atvb_system_set_lj_types(s._h, *args))
    assert e.value.code == 4
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_cpp_water_matches_python(atvb, ctx, tmp_path, precision):
    """md::MD with per-type PairLJCut, special bonds and PME (C++ mirror)
    gives bit for bit what the Python layer gives for the same frame."""
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    desc, frame, coeffs, special = _water(m=8)  # box 24.8 > 2 (rc + skin)
    n, bonds = desc["n_atoms"], special["bonds"]
    path = tmp_path / "water.bin"
    with open(path, "wb") as fh:
        fh.write(np.array([n, len(bonds)], dtype=np.int64).tobytes())
        fh.write(np.array(list(desc["box"]) + [desc["coul_alpha"], desc["coul_cutoff"]]).tobytes())
        fh.write(np.array([desc["pme_grid"][0]], dtype=np.int64).tobytes())
        for k in ("x", "y", "z", "charge", "mass"):
            fh.write(np.ascontiguousarray(frame[k], dtype=np.float64).tobytes())
        fh.write(frame["type"].astype(np.int32).tobytes())
        fh.write(np.array(bonds, dtype=np.int64).tobytes())
    exe = str(tmp_path / "md_water")
    lib_dir = os.path.join(root, "atomiverse_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(root, "include"),
                    os.path.join(root, "tests", "cpp", "md_water.cpp"), "-o", exe,
                    "-L", lib_dir, "-latvb", "-Wl,-rpath," + lib_dir], check=True)
    r = subprocess.run([exe, str(path), "20", str(precision)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = r.stdout.split()
    d = dict(desc, precision=precision, dt=0.5, stress_required=0)
    s = atvb.System(ctx, d, frame, lj_types=coeffs, special_bonds=special)
    fr = {k: np.array(v, copy=True) for k, v in frame.items()}
    sc = s.run(fr, 20)
    s.close()
    csum = 0.0
    for x, y, z in zip(fr["x"].tolist(), fr["y"].tolist(), fr["z"].tolist()):
        csum += x + 2.0 * y + 3.0 * z
    assert int(out[0]) == sc["step"] == 20
    assert float(out[1]) == sc["energy_lj"]
    assert float(out[2]) == sc["energy_coul"]
    assert float(out[3]) == sc["energy_recip"]
    assert float(out[4]) == pytest.approx(csum, rel=1e-15, abs=0)
