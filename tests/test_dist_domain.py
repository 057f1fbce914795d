"""Domain decomposition of one system (atomiverse_b200/domain.py) on gloo
ranks on CPU: x slabs, halo plans, migration and the slab transposes of the
PME mesh.  Each rank evaluates what the single-GPU library evaluates for a
sub-domain -- real-space pair forces of its owned atoms against owned +
ghost atoms (the CPU oracle on that atom set), B-spline spreading into its
mesh planes, the transforms along y/z, along x after the transpose, the
influence function, and the interpolation -- with numpy and the oracle's
splines standing in for the kernels.  Two ranks give the forces, energy and
virial of one rank, and both give the oracle's for the whole periodic
system (the check of the reference's tests/mpi/test_pme_nacl_parity.cpp:
97,178, made here against the oracle); five velocity-Verlet steps with
migration and fresh halos every step follow the oracle's trajectory."""
import datetime
import os
import socket

import numpy as np
import pytest

from atomiverse_b200 import domain
from atomiverse_b200 import workloads as W

QQR2E, FTM2V = 14.399645, 1.0 / 103.6427          # metal units (oracle)
RC, SKIN, K, ORDER = 9.0, 1.0, 24, 4


def _case():
    desc, frame = W.rocksalt_melt(ncell=8, seed=41, grid=(K, K, K), rc=RC, skin=SKIN)
    return desc, frame


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


# ---- per-rank arithmetic (stands in for the library's kernels) --------------

def _oracle_pairs(orc, desc, x, y, z, q, m, box):
    """Real-space LJ + Coulomb forces, energy and virial of an atom set in
    `box` (the oracle, no PME)."""
    from conftest import oracle_system
    d = dict(desc, n_atoms=len(x), box=tuple(box), pme_enabled=0)
    fr = {"x": x, "y": y, "z": z, "charge": q, "mass": m}
    s = oracle_system(orc, d, fr)
    s.build_list()
    s.compute_forces()
    st, sc = s.state(), s.scalars()
    s.close()
    return np.stack([st["fx"], st["fy"], st["fz"]], 1), sc["e_lj"] + sc["e_coul"], \
        np.array(sc["virial"])


def _pair_rank(orc, desc, dom, own, gh):
    """Forces on the owned atoms (full shell), and this rank's share of the
    pair energy / virial: E_oo + E_og / 2 = (E_all - E_gg + E_oo) / 2."""
    L = dom.L
    box3 = (3 * L[0], L[1], L[2])            # x open: no wrap across the shell
    cat = np.concatenate([own, gh], axis=0)
    cols = lambda a: (a[:, 0] + L[0], a[:, 1], a[:, 2], a[:, 3], a[:, 5])
    f_all, e_all, v_all = _oracle_pairs(orc, desc, *cols(cat), box3)
    e_oo, v_oo = 0.0, np.zeros(6)
    if len(own):
        _, e_oo, v_oo = _oracle_pairs(orc, desc, *cols(own), box3)
    e_gg, v_gg = 0.0, np.zeros(6)
    if len(gh):
        _, e_gg, v_gg = _oracle_pairs(orc, desc, *cols(gh), box3)
    return f_all[:len(own)], 0.5 * (e_all - e_gg + e_oo), 0.5 * (v_all - v_gg + v_oo)


def _splines(orc, u):
    base = np.floor(u).astype(np.int64)
    th = np.empty((len(u), ORDER))
    dth = np.empty((len(u), ORDER))
    for i, f in enumerate(u - base):
        th[i], dth[i] = orc.bspline(f, ORDER)
    return base, th, dth


def _fractional(L, Kd, x):
    # the oracle's reduction: u = (x / L) K, then folded into [0, K)
    u = (1.0 / L) * x * Kd
    return u - np.floor(u / Kd) * Kd


def _pme_rank(orc, desc, dom, own, gh):
    """Reciprocal forces on the owned atoms and this rank's share of the
    reciprocal energy and virial, on the slab decomposition."""
    L, alpha = dom.L, desc["pme_alpha"]
    K0, K1, K2 = dom.K
    Kh = K2 // 2 + 1
    cat = np.concatenate([own, gh], axis=0)
    # x stays unwrapped: a ghost is its atom's plane index moved by whole
    # periods (column 6 holds the atom's own x)
    image = np.rint((cat[:, 0] - cat[:, 6]) / L[0]).astype(np.int64)
    u = [_fractional(L[0], K0, cat[:, 6]), _fractional(L[1], K1, cat[:, 1]),
         _fractional(L[2], K2, cat[:, 2])]
    sp = [_splines(orc, ud) for ud in u]
    b0 = sp[0][0] + image * K0
    q = cat[:, 3]
    # spread into this rank's planes [P0, P1): each (atom image, plane) once
    n_p = dom.P1 - dom.P0
    grid = np.zeros((n_p, K1, K2))
    for a in range(ORDER):
        g0 = b0 - (ORDER - 1) + a
        ok = (g0 >= dom.P0) & (g0 < dom.P1)
        for b in range(ORDER):
            g1 = (sp[1][0] - (ORDER - 1) + b) % K1
            for c in range(ORDER):
                g2 = (sp[2][0] - (ORDER - 1) + c) % K2
                w = q * sp[0][1][:, a] * sp[1][1][:, b] * sp[2][1][:, c]
                np.add.at(grid, (g0[ok] - dom.P0, g1[ok], g2[ok]), w[ok])
    # forward: z, y on the slab; transpose; x
    S = np.fft.fft(np.fft.rfft(grid, axis=2), axis=1)
    S = np.fft.fft(dom.to_pencils(S), axis=0)
    # influence on this rank's modes (pme_influence.h:159-199)
    bm = [orc.spline_moduli(k, ORDER) for k in (K0, K1, K2)]
    m1 = np.arange(dom.M1[dom.r], dom.M1[dom.r + 1])
    h = lambda m, Kd: np.where(m <= Kd // 2, m, m - Kd)
    mx = (h(np.arange(K0), K0) / L[0])[:, None, None]
    my = (h(m1, K1) / L[1])[None, :, None]
    mz = (h(np.arange(Kh), K2) / L[2])[None, None, :]
    msq = mx * mx + my * my + mz * mz
    zero = msq == 0.0
    inv = np.where(zero, 0.0, 1.0 / np.where(zero, 1.0, msq))
    pi2a2 = np.pi ** 2 / alpha ** 2
    H = np.where(zero, 0.0, np.exp(-pi2a2 * msq) * inv *
                 bm[0][:, None, None] * bm[1][m1][None, :, None] * bm[2][:Kh][None, None, :])
    m2 = np.arange(Kh)
    wt = np.where((m2 == 0) | (2 * m2 == K2), 1.0, 2.0)[None, None, :]
    ug = wt * H * np.abs(S) ** 2
    vt = -2.0 * (inv + pi2a2)
    vir = np.array([(ug * (1 + vt * mx * mx)).sum(), (ug * (1 + vt * my * my)).sum(),
                    (ug * (1 + vt * mz * mz)).sum(), (ug * vt * mx * my).sum(),
                    (ug * vt * mx * mz).sum(), (ug * vt * my * mz).sum()])
    vol = L.prod()
    escale = QQR2E / (2.0 * np.pi * vol)
    e_rec = ug.sum() * escale
    # inverse: x; transpose back; y, z (unnormalised, as the oracle)
    conv = np.fft.ifft(H * S, axis=0) * K0
    conv = np.fft.ifft(dom.to_slabs(conv), axis=1) * K1
    conv = np.fft.irfft(conv, n=K2, axis=2) * K2
    # interpolation of the owned atoms: planes [P0 - order, P1)
    ext = np.concatenate([dom.lower_planes(conv, ORDER), conv], axis=0)
    no = len(own)
    g = np.zeros((no, 3))
    for a in range(ORDER):
        g0 = b0[:no] - (ORDER - 1) + a - (dom.P0 - ORDER)
        assert g0.min() >= 0 and g0.max() < ext.shape[0]
        for b in range(ORDER):
            g1 = (sp[1][0][:no] - (ORDER - 1) + b) % K1
            for c in range(ORDER):
                g2 = (sp[2][0][:no] - (ORDER - 1) + c) % K2
                cv = ext[g0, g1, g2]
                t = [sp[d][1][:no, k] for d, k in ((0, a), (1, b), (2, c))]
                dt = [sp[d][2][:no, k] for d, k in ((0, a), (1, b), (2, c))]
                g[:, 0] += cv * dt[0] * t[1] * t[2]
                g[:, 1] += cv * t[0] * dt[1] * t[2]
                g[:, 2] += cv * t[0] * t[1] * dt[2]
    fscale = QQR2E / (np.pi * vol)
    f = -fscale * q[:no, None] * g * (np.array([K0, K1, K2]) / L)[None, :]
    return f, e_rec, vir * escale


def _forces(orc, desc, dom, own):
    """All forces on the owned rows, and this rank's shares of energy and
    virial.  Rows: x y z q tag mass x_own vx vy vz."""
    plan = dom.halo_plan(own[:, 0])
    gh = dom.exchange(plan, own)
    fp, ep, vp = _pair_rank(orc, desc, dom, own, gh)
    fr, er, vr = _pme_rank(orc, desc, dom, own, gh)
    return fp + fr, ep + er, vp + vr


def _allsum(v):
    import torch
    import torch.distributed as dist
    t = torch.as_tensor(np.atleast_1d(np.asarray(v, dtype=np.float64))).clone()
    dist.all_reduce(t)
    return t.numpy()


def _worker(rank, ws, port, q):
    import torch.distributed as dist
    import oracle as orc
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=120))
    try:
        orc.set_threads(2)
        desc, frame = _case()
        dom = domain.Slabs(desc["box"], RC + SKIN, ws, rank, K=(K, K, K), order=ORDER)
        n = desc["n_atoms"]
        xyz = [np.mod(np.asarray(frame[k], dtype=np.float64), dom.L[i])
               for i, k in enumerate("xyz")]
        full = np.stack(xyz + [frame["charge"], np.arange(1, n + 1, dtype=np.float64),
                               frame["mass"], xyz[0], frame["vx"], frame["vy"], frame["vz"]], 1)
        own = full[dom.owner(full[:, 0]) == rank]
        out = {}
        f, e, v = _forces(orc, desc, dom, own)
        qq = _allsum([np.sum(own[:, 3] ** 2), np.sum(own[:, 3])])
        vol, a = dom.L.prod(), desc["pme_alpha"]
        e_const = -QQR2E * a / np.sqrt(np.pi) * qq[0] - \
            QQR2E * np.pi / (2.0 * vol * a * a) * qq[1] ** 2
        out["energy"] = float(_allsum(e)[0]) + e_const
        out["virial"] = _allsum(v)
        tags = dom.alltoallv([own[:, [4]] if d == 0 else np.zeros((0, 1)) for d in range(ws)])
        fs = dom.alltoallv([f if d == 0 else np.zeros((0, 3)) for d in range(ws)])
        if rank == 0:
            o = np.argsort(tags[:, 0])
            out["tags"], out["f"] = tags[o, 0], fs[o]
        # migration: random moves of up to 1.5 A; every atom is owned once
        rng = np.random.default_rng(7)
        moved = own.copy()
        moved[:, 0] += rng.uniform(-1.5, 1.5, len(own))
        mig = dom.migrate(moved)
        assert np.all(dom.owner(mig[:, 0]) == rank)
        assert np.all((mig[:, 0] >= 0) & (mig[:, 0] < dom.L[0]))
        alltags = dom.alltoallv([mig[:, [4]] if d == 0 else np.zeros((0, 1)) for d in range(ws)])
        if rank == 0:
            out["migrated_tags"] = np.sort(alltags[:, 0])
        # five velocity-Verlet steps (metal units, NVE), migration and fresh
        # halos every step
        dt = desc["dt"]
        dtf = 0.5 * dt * FTM2V
        cur, fc = own.copy(), f
        for _ in range(5):
            m = cur[:, 5][:, None]
            cur[:, 7:10] += dtf / m * fc
            cur[:, 0:3] += dt * cur[:, 7:10]
            cur[:, 1] = np.mod(cur[:, 1], dom.L[1])
            cur[:, 2] = np.mod(cur[:, 2], dom.L[2])
            cur = dom.migrate(cur)
            cur[:, 6] = cur[:, 0]
            fc, _, _ = _forces(orc, desc, dom, cur)
            cur[:, 7:10] += dtf / cur[:, 5][:, None] * fc
        st = dom.alltoallv([cur if d == 0 else np.zeros((0, cur.shape[1])) for d in range(ws)])
        if rank == 0:
            o = np.argsort(st[:, 4])
            out["traj"] = st[o]
            q.put(out)
    finally:
        dist.destroy_process_group()


def _run(ws):
    import torch.multiprocessing as mp
    q = mp.get_context("spawn").Queue()
    procs = mp.spawn(_worker, args=(ws, _free_port(), q), nprocs=ws, join=False)
    out = q.get(timeout=600)          # before joining: the queue must drain
    while not procs.join():
        pass
    return out


def test_slab_geometry_and_checks():
    desc, _ = _case()
    d = domain.Slabs(desc["box"], RC + SKIN, 2, 1, K=(K, K, K), order=ORDER)
    assert (d.P0, d.P1) == (12, 24) and d.M1 == [0, 12, 24]
    assert domain.max_ranks(desc["box"], RC + SKIN) == 2
    with pytest.raises(ValueError):
        domain.Slabs(desc["box"], RC + SKIN, 3, 0)          # slabs narrower than rlist
    with pytest.raises(ValueError):
        domain.Slabs(desc["box"], 3.0, 2, 0, K=(6, 6, 6))   # mesh too coarse for the shell
    x = np.array([0.0, 11.27, 11.28, 22.55, -0.1, 22.6])
    assert d.owner(x).tolist() == [0, 0, 1, 1, 1, 0]


def test_two_ranks_equal_one_rank_and_the_oracle(orc):
    from conftest import oracle_system, rms_rel
    r1, r2 = _run(1), _run(2)
    desc, frame = _case()
    n = desc["n_atoms"]
    assert np.array_equal(r2["tags"], np.arange(1, n + 1))
    assert np.array_equal(r2["migrated_tags"], np.arange(1, n + 1))
    o = oracle_system(orc, dict(desc, thermostat=0), frame)     # the loop below is NVE
    o.build_list()
    o.compute_forces()
    st, sc = o.state(), o.scalars()
    fo = np.stack([st["fx"], st["fy"], st["fz"]], 1)
    assert rms_rel(r2["f"], r1["f"]) < 1e-12
    assert rms_rel(r2["f"], fo) < 1e-10
    assert r2["energy"] == pytest.approx(sc["energy"], rel=1e-10)
    assert r2["energy"] == pytest.approx(r1["energy"], rel=1e-12)
    vir = np.array(sc["virial"])
    assert np.allclose(r2["virial"], vir, rtol=1e-9, atol=1e-9 * np.abs(vir).max())
    # five NVE steps: positions and velocities follow the oracle
    o.run(5)
    st = o.state()
    L = desc["box"][0]
    for k, c in (("x", 0), ("y", 1), ("z", 2)):
        d = r2["traj"][:, c] - st[k]
        d -= L * np.rint(d / L)
        assert np.abs(d).max() < 1e-9, k
    v = r2["traj"][:, 7:10]
    vo = np.stack([st["vx"], st["vy"], st["vz"]], 1)
    assert rms_rel(v, vo) < 1e-8
    o.close()
