"""MTK NPT on the GPU (md::NoseHooverNPT) against the oracle:

- the reference's npt_lj_mtk regression (216 LJ atoms, 80 steps, no force
  pass before the first step): cell volume, positions and the conserved
  extended Hamiltonian match the oracle, and the volume is the reference's
  own V = 269.425432;
- a charged LJ melt with PME under 16 kbar: the cell, PME prefactors and
  neighbour bins follow the cell every step;
- one uncoupled axis keeps its edge;
- an NPT system batched with a Nose-Hoover one gives what each gives alone.
"""
import numpy as np
import pytest

from conftest import oracle_system

KB = 8.617333262e-5


def _lj_cube(n_side=6, rho=0.8):
    n = n_side ** 3
    L = (n / rho) ** (1.0 / 3.0)
    a = L / n_side
    idx = np.array([(ix, iy, iz) for ix in range(n_side) for iy in range(n_side)
                    for iz in range(n_side)])
    pos = (idx + 0.5) * a
    ix, iy, iz = idx[:, 0], idx[:, 1], idx[:, 2]
    desc = dict(n_atoms=n, box=(L, L, L), nl_cutoff=2.5, nl_skin=0.3, lj_enabled=1,
                lj_epsilon=1.0, lj_sigma=1.0, lj_cutoff=2.5, dt=0.005)
    frame = dict(x=pos[:, 0].copy(), y=pos[:, 1].copy(), z=pos[:, 2].copy(),
                 vx=0.02 * ((ix + iy + iz) % 3 - 1.0), vy=0.02 * ((ix + 2 * iy) % 3 - 1.0),
                 vz=0.02 * ((2 * ix + iz) % 3 - 1.0), mass=np.ones(n))
    return desc, frame


def _melt(ncell=6):
    from atomiverse_b200 import workloads as W
    desc, frame = W.rocksalt_melt(ncell=ncell, rc=5.5, grid=(20, 20, 20))
    desc = dict(desc, thermostat=0, stress_required=1)
    return desc, frame


def _pos(out):
    return np.stack([out["x"], out["y"], out["z"]], axis=1)


def _oracle_npt(orc, desc, frame, npt, steps, setup=False):
    o = oracle_system(orc, desc, frame)
    o.set_npt(npt["T_target"], npt["tau_T"], npt["P_target"], npt["tau_P"],
              couple=npt.get("couple_axis", (True, True, True)))
    if setup:
        o.build_list()
        o.compute_forces()
    o.run(steps)
    return o


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [(0, 1e-10), (1, 1e-6)])
def test_npt_lj_regression_matches_oracle(atvb, ctx, orc, precision, tol):
    desc, frame = _lj_cube()
    npt = dict(T_target=1.0 / KB, tau_T=0.1, P_target=0.0, tau_P=1.0, dt=0.005)
    s = atvb.System(ctx, dict(desc, precision=precision), frame, npt=npt)
    s.step(80)
    out, sc = s.download()
    s.close()
    o = _oracle_npt(orc, desc, frame, npt, 80)
    ost = o.npt_state()
    V, Vo = float(np.prod(sc["box"])), float(np.prod(ost["box"]))
    assert V == pytest.approx(Vo, rel=tol)
    assert V == pytest.approx(269.425432, abs=max(1e-6, tol * V))
    assert sc["conserved"] == pytest.approx(ost["conserved"], rel=10 * tol)
    d = _pos(out) - _pos(o.state())
    d -= np.rint(d / sc["box"]) * sc["box"]
    assert np.abs(d).max() < 1e3 * tol * sc["box"][0]
    assert sc["status"] == 0 and sc["step"] == 80


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [(0, 1e-9), (1, 2e-6)])
def test_npt_pme_melt_matches_oracle(atvb, ctx, orc, precision, tol):
    desc, frame = _melt()
    npt = dict(T_target=1200.0, tau_T=100.0, P_target=1e-5, tau_P=1000.0, dt=2.0)
    s = atvb.System(ctx, dict(desc, precision=precision), frame, npt=npt)
    s.compute_forces()
    s.step(20)
    out, sc = s.download()
    s.close()
    o = _oracle_npt(orc, desc, frame, npt, 20, setup=True)
    ost, osc = o.npt_state(), o.scalars()
    assert sc["box"][0] != desc["box"][0]
    assert np.allclose(sc["box"], ost["box"], rtol=tol, atol=0)
    assert sc["conserved"] == pytest.approx(ost["conserved"], rel=10 * tol)
    assert sc["energy_recip"] + sc["energy_const"] == pytest.approx(
        osc["e_recip"] + osc["e_const"], rel=100 * tol)
    d = _pos(out) - _pos(o.state())
    d -= np.rint(d / sc["box"]) * sc["box"]
    assert np.abs(d).max() < 1e3 * tol * sc["box"][0]


@pytest.mark.gpu
def test_npt_uncoupled_axis_keeps_edge(atvb, ctx, orc):
    desc, frame = _lj_cube()
    npt = dict(T_target=1.0 / KB, tau_T=0.1, P_target=0.0, tau_P=1.0, dt=0.005,
               couple_axis=(True, True, False))
    s = atvb.System(ctx, desc, frame, npt=npt)
    s.compute_forces()
    s.step(30)
    _, sc = s.download()
    s.close()
    assert sc["box"][2] == desc["box"][2]
    assert sc["box"][0] != desc["box"][0]
    o = _oracle_npt(orc, desc, frame, npt, 30, setup=True)
    assert np.allclose(sc["box"], o.npt_state()["box"], rtol=1e-10, atol=0)


@pytest.mark.gpu
def test_npt_batch_equals_alone(atvb, ctx):
    from atomiverse_b200 import workloads as W
    d1, f1 = _lj_cube()
    npt = dict(T_target=1.0 / KB, tau_T=0.1, P_target=0.0, tau_P=1.0, dt=0.005)
    d2, f2 = _melt()
    npt2 = dict(T_target=1200.0, tau_T=100.0, P_target=1e-5, tau_P=1000.0, dt=2.0)
    d3, f3 = W.lj_fcc(ncell=5, seed=3)
    items = [(d1, f1, dict(npt=npt)), (d2, f2, dict(npt=npt2)), (d3, f3)]
    b = atvb.Batch(ctx, items)
    b.compute_forces()
    b.step(15)
    for k, it in enumerate(items):
        ob, sb = b.download(k)
        opts = it[2] if len(it) > 2 else {}
        s = atvb.System(ctx, it[0], it[1], **opts)
        s.compute_forces()
        s.step(15)
        oa, sa = s.download()
        s.close()
        for key in ("x", "y", "z", "vx", "vy", "vz"):
            assert np.array_equal(ob[key], oa[key]), (k, key)
        assert np.array_equal(sb["box"], sa["box"])
        assert sb["conserved"] == sa["conserved"]
    b.close()


@pytest.mark.gpu
def test_cpp_npt_regression(atvb, tmp_path):
    """The reference's npt_lj_mtk case through the C++ mirror
    (md::NoseHooverNPT): the reference CPU build's V = 269.425432."""
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = str(tmp_path / "md_npt")
    lib_dir = os.path.join(root, "atomiverse_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(root, "include"),
                    os.path.join(root, "tests", "cpp", "md_npt.cpp"), "-o", exe,
                    "-L", lib_dir, "-latvb", "-Wl,-rpath," + lib_dir], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    V, H, status = r.stdout.split()
    assert float(V) == pytest.approx(269.425432, abs=1e-6)
    assert np.isfinite(float(H)) and int(status) == 0


@pytest.mark.gpu
def test_python_md_mirror_npt(atvb, ctx):
    """md.MD with NoseHooverNPT as its integrator moves frame["box"]."""
    desc, frame = _lj_cube()
    fr = dict(frame, box=desc["box"])
    sim = atvb.MD(ctx=ctx)
    sim.set_neighbor(atvb.NeighborList(2.5, 0.3)).set_evaluator(atvb.PairLJCut(1.0, 1.0, 2.5))
    sim.set_integrator(atvb.NoseHooverNPT(1.0 / KB, 0.1, 0.0, 1.0, 0.005))
    sim.run(fr, 40)
    sim.run(fr, 40)
    assert float(np.prod(fr["box"])) == pytest.approx(269.425432, abs=1e-6)


@pytest.mark.gpu
def test_npt_cell_leaving_the_planned_range_is_replanned(atvb, ctx, orc):
    """A dilute LJ system compressed at high pressure shrinks far beyond the
    90 % its first bins were planned for; between step calls the library
    re-plans bins (and the list) for the current cell, and the run matches
    the oracle, which rebuilds every step, to rounding level."""
    from atomiverse_b200 import workloads as W
    desc, frame = W.lj_fcc(ncell=7, rho=0.5, t_star=1.0, seed=9)
    L0 = desc["box"][0]
    npt = dict(T_target=1.0 / KB, tau_T=1.0, P_target=5.0, tau_P=5.0, dt=desc["dt"])
    s = atvb.System(ctx, desc, frame, npt=npt)
    s.compute_forces()
    for _ in range(200):
        s.step(3)            # 3 steps shrink an edge by at most 1.5 %
        sc = s.scalars()
        assert sc["status"] == 0
    out, sc = s.download()
    s.close()
    assert sc["box"][0] < 0.85 * L0              # beyond the first plan's range
    o = _oracle_npt(orc, desc, frame, npt, 600, setup=True)
    assert np.allclose(sc["box"], o.npt_state()["box"], rtol=1e-8, atol=0)


def _baro_case(thermostat=1, precision=0):
    from atomiverse_b200 import workloads as W
    desc, frame = W.lj_fcc(ncell=6, t_star=1.0, seed=3, thermostat=thermostat, precision=precision)
    return dict(desc, tau=50.0), frame, dict(P_target=0.5, tau_P=20.0, dt=desc["dt"],
                                             bulk_modulus=10.0)


@pytest.mark.gpu
@pytest.mark.parametrize("thermostat,precision,tol", [(1, 0, 1e-10), (2, 0, 1e-10), (1, 1, 1e-6)])
def test_berendsen_barostat_matches_oracle(atvb, ctx, orc, thermostat, precision, tol):
    """md::Barostat (Berendsen) beside Nose-Hoover or Langevin: cell and
    positions follow the oracle over 200 steps."""
    desc, frame, baro = _baro_case(thermostat, precision)
    s = atvb.System(ctx, desc, frame, barostat=baro)
    s.compute_forces()
    s.step(200)
    out, sc = s.download()
    s.close()
    o = oracle_system(orc, desc, frame)
    o.set_barostat(baro["P_target"], baro["tau_P"], baro["bulk_modulus"])
    o.build_list()
    o.compute_forces()
    o.run(200)
    box = o.npt_state()["box"]
    assert sc["box"][0] != desc["box"][0]
    assert np.allclose(sc["box"], box, rtol=tol, atol=0)
    d = _pos(out) - _pos(o.state())
    d -= np.rint(d / sc["box"]) * sc["box"]
    assert np.abs(d).max() < 1e4 * tol * box[0]
    assert sc["status"] == 0


@pytest.mark.gpu
def test_berendsen_batch_equals_alone_and_resumes(atvb, ctx):
    desc, frame, baro = _baro_case(1, 1)
    from atomiverse_b200 import workloads as W
    d2, f2 = W.lj_fcc(ncell=5, seed=4)
    items = [(desc, frame, dict(barostat=baro)), (d2, f2)]
    b = atvb.Batch(ctx, items)
    b.compute_forces()
    b.step(30)
    ob, sb = b.download(0)
    b.close()
    s = atvb.System(ctx, desc, frame, barostat=baro)
    s.compute_forces()
    s.step(12)
    blob = s.save()
    s.close()
    r = atvb.System(ctx, desc, None, barostat=baro)
    r.restore(blob)
    r.step(18)
    oa, sa = r.download()
    r.close()
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(ob[k], oa[k]), k
    assert np.array_equal(sb["box"], sa["box"])


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["nve_limit", "deform"])
def test_nve_limit_and_deform_match_oracle(atvb, ctx, orc, kind):
    """md::NVELimit (speed cap) and md::Deform (engineering strain) against
    the oracle over 150 steps (FP64)."""
    from atomiverse_b200 import workloads as W
    desc, frame = W.lj_fcc(ncell=6, t_star=3.0 if kind == "nve_limit" else 1.0, seed=3)
    if kind == "nve_limit":
        opts, xmax = dict(nve_limit=0.002), 0.002
    else:
        opts = dict(deform=(2, 2e-3))
    s = atvb.System(ctx, desc, frame, **opts)
    s.compute_forces()
    s.step(150)
    out, sc = s.download()
    s.close()
    o = oracle_system(orc, desc, frame)
    if kind == "nve_limit":
        o.set_nve_limit(xmax)
    else:
        o.set_deform(2, 2e-3)
    o.build_list()
    o.compute_forces()
    o.run(150)
    box = o.npt_state()["box"]
    assert np.allclose(sc["box"], box, rtol=1e-12, atol=0)
    d = _pos(out) - _pos(o.state())
    d -= np.rint(d / sc["box"]) * sc["box"]
    assert np.abs(d).max() < 1e-8
    if kind == "deform":
        assert sc["box"][2] > desc["box"][2] * 1.01
    else:
        v = np.sqrt(out["vx"] ** 2 + out["vy"] ** 2 + out["vz"] ** 2)
        assert v.max() <= xmax / desc["dt"] * (1 + 1e-12)


@pytest.mark.gpu
def test_python_md_mirror_nve_limit_deform(atvb, ctx):
    """md.MD with NVELimit as its integrator and Deform bound beside it runs
    the same steps as System(nve_limit=, deform=) on the same description,
    bit for bit."""
    from atomiverse_b200 import workloads as W
    desc, frame = W.lj_fcc(ncell=6, t_star=3.0, seed=5)
    sim = atvb.MD(ctx=ctx)
    sim.set_neighbor(atvb.NeighborList(desc["nl_cutoff"], desc["nl_skin"]))
    sim.set_evaluator(atvb.PairLJCut(desc["lj_epsilon"], desc["lj_sigma"], desc["lj_cutoff"]))
    sim.set_integrator(atvb.NVELimit(desc["dt"], 0.002))
    sim.set_thermostat(atvb.Deform(1, 1e-3, desc["dt"]))
    n = len(frame["x"])
    ref = atvb.System(ctx, sim.desc(n, desc["box"]), None, nve_limit=0.002, deform=(1, 1e-3))
    fa = {k: np.array(v) for k, v in frame.items()}
    s = ref.run(fa, 60)
    ref.close()
    fb = dict({k: np.array(v) for k, v in frame.items()}, box=desc["box"])
    sm = sim.run(fb, 60)
    assert sm["box"][1] > desc["box"][1] * 1.002
    assert np.array_equal(np.asarray(sm["box"]), np.asarray(s["box"]))
    assert sm["energy"] == s["energy"] and sm["kinetic"] == s["kinetic"]
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(fa[k], fb[k]), k
    v = np.sqrt(fb["vx"] ** 2 + fb["vy"] ** 2 + fb["vz"] ** 2)
    assert v.max() <= 0.002 / desc["dt"] * (1 + 1e-12)


@pytest.mark.gpu
def test_rows_widen_between_calls_under_compression(atvb, ctx, orc):
    """A Langevin gas (rho* = 0.2, T* = 1) squeezed along z to a fifth of its
    edge by Deform in calls of 40 steps, with no synchronisation between
    them: the longest neighbour row goes from 18 to ~104 entries, past the 96
    the rows were sized for.  Between calls (and between the pieces a call is
    cut into so that the shrinking cell never leaves its bins) the rows are
    widened once a build fills 80 % of them, so no build overflows (status 0)
    and the run matches the oracle."""
    from atomiverse_b200 import workloads as W
    desc, frame = W.lj_fcc(ncell=11, rho=0.2, t_star=1.0, seed=12, thermostat=2,
                           damp_tau=0.5)
    steps, chunk = 1000, 40
    rate = -0.8 / (steps * desc["dt"])
    s = atvb.System(ctx, desc, frame, deform=(2, rate))
    s.compute_forces()
    first = s.scalars()["max_neighbors"]
    for _ in range(steps // chunk):
        s.step(chunk)
    out, sc = s.download()
    s.close()
    o = oracle_system(orc, desc, frame)
    o.set_deform(2, rate)
    o.build_list()
    o.compute_forces()
    o.run(steps)
    d = _pos(out) - _pos(o.state())
    d -= np.rint(d / sc["box"]) * sc["box"]
    err = np.abs(d).max()
    e_rel = abs(sc["energy"] / o.scalars()["energy"] - 1.0)
    assert first < 40 and sc["max_neighbors"] > 96, (first, sc["max_neighbors"])
    assert sc["status"] == 0
    assert np.allclose(sc["box"], o.npt_state()["box"], rtol=1e-12, atol=0)
    assert err < 1e-6 and e_rel < 1e-8, (err, e_rel)
