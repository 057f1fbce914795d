"""Batching and serving forms on the GPU.

- a batch of uneven systems gives each system bit-for-bit the result it gets
  alone (per-system lane counts, per-item fixed-point energy flushes);
- the autotuner leaves the forces and energies as a plain force pass with
  the chosen lane count would;
- the number of launches per step does not grow with the number of systems;
- a served request gives the same result alone and in a mix, under a tight
  or a loose device-memory budget; admission, cancel and oversize errors;
- the reference-shaped C++ API (md.hpp) drives the library end to end.
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEYS = ("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz")


def _mix(W, precision):
    """Three LJ fluids of different sizes (two under Langevin) and one small
    rock-salt melt with PME."""
    out = []
    for c, seed, thermo in ((4, 11, 2), (5, 12, 0), (6, 13, 2)):
        out.append(W.lj_fcc(ncell=c, seed=seed, precision=precision, thermostat=thermo,
                            t_star=1.0))
    out.append(W.rocksalt_melt(ncell=8, seed=14, rc=10.2, grid=(24, 24, 24),
                               precision=precision))
    return out


def _alone(A, ctx, desc, frame, n_steps, lanes=0):
    s = A.System(ctx, desc, frame)
    if lanes:
        s.set_pair_lanes(lanes)
    s.compute_forces()
    if n_steps:
        s.step(n_steps)
    out, sc = s.download()
    s.close()
    return out, sc


def _same(a, b, keys=KEYS):
    for k in keys:
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_batch_equals_alone_bitwise(atvb, ctx, precision):
    from atomiverse_b200 import workloads as W
    items = _mix(W, precision)
    b = atvb.Batch(ctx, items)
    b.compute_forces()
    b.step(30)
    for k, (d, f) in enumerate(items):
        ob, sb = b.download(k)
        oa, sa = _alone(atvb, ctx, d, f, 30)
        _same(ob, oa)
        assert sb["energy"] == sa["energy"]
        assert sb["kinetic"] == sa["kinetic"]
        assert sb["step"] == 30
    b.close()


@pytest.mark.gpu
def test_autotune_keeps_results(atvb, ctx):
    from atomiverse_b200 import workloads as W
    items = _mix(W, 1)
    b = atvb.Batch(ctx, items)
    g = b.autotune()
    assert g in (1, 2, 4, 8, 16, 32)
    for k, (d, f) in enumerate(items):
        ob, sb = b.download(k)
        oa, sa = _alone(atvb, ctx, d, f, 0, lanes=g)
        _same(ob, oa, ("fx", "fy", "fz"))
        assert sb["energy"] == sa["energy"]
        assert np.array_equal(sb["stress"], sa["stress"])
    b.close()


@pytest.mark.gpu
def test_launches_do_not_grow_with_systems(atvb, ctx):
    from atomiverse_b200 import workloads as W
    sizes = [(4, 1), (5, 2), (6, 3), (4, 4), (5, 5), (6, 6)]
    six = [W.lj_fcc(ncell=c, seed=s, precision=1) for c, s in sizes]
    twelve = six + [W.lj_fcc(ncell=c, seed=s + 10, precision=1) for c, s in sizes]
    counts = []
    for items in (six[:1], six, twelve):
        b = atvb.Batch(ctx, items)
        b.step(1)
        counts.append(b.launch_count())
        b.close()
    one, n6, n12 = counts
    assert one > 0
    assert n6 == n12                  # twice the systems, same launches
    assert n6 <= one + 5              # at most one extra pair launch per lane class


def _serve(atvb, ctx, reqs, budget, chunk=7, max_ticks=200):
    srv = atvb.Server(ctx, budget)
    ids = [srv.submit(d, f, n) for d, f, n in reqs]
    peak_running = 0
    for _ in range(max_ticks):
        srv.tick(chunk)
        st = srv.stats()
        peak_running = max(peak_running, st["running"])
        assert st["bytes"] <= budget
        if st["queued"] == 0 and st["running"] == 0:
            break
    outs = []
    for rid in ids:
        assert srv.poll(rid)["state"] == 2
        out, res = srv.collect(rid)
        outs.append((out, res))
    srv.close()
    return outs, peak_running


@pytest.mark.gpu
@pytest.mark.parametrize("tight", [False, True])
def test_served_result_equals_alone(atvb, ctx, tight):
    from atomiverse_b200 import workloads as W
    mix = _mix(W, 1)
    reqs = [(mix[0][0], mix[0][1], 40), (mix[3][0], mix[3][1], 25),
            (mix[2][0], mix[2][1], 33)]
    sizes = [atvb.request_bytes(d) for d, _, _ in reqs]
    budget = max(sizes) if tight else 2 * sum(sizes)
    outs, peak = _serve(atvb, ctx, reqs, budget)
    if tight:
        # the largest request cannot share the budget with any other one
        assert peak < len(reqs)
    else:
        assert peak == len(reqs)          # all overlap on the device
    for (d, f, n), (out, res) in zip(reqs, outs):
        assert res["steps_done"] == n
        assert res["scalars"]["step"] == n
        alone, sa = _alone(atvb, ctx, d, f, n)
        _same(out, alone)
        assert res["scalars"]["energy"] == sa["energy"]
        assert res["t_submit"] <= res["t_start"] <= res["t_done"]


@pytest.mark.gpu
def test_served_arrivals_while_running_equal_alone(atvb, ctx):
    """Continuous batching with arrivals: requests submitted while others are
    already on the GPU join the running batch at the next tick, run beside
    them, and each result is still the one it gets alone, bit for bit."""
    from atomiverse_b200 import workloads as W
    mix = _mix(W, 1)
    reqs = [(mix[0][0], mix[0][1], 60), (mix[3][0], mix[3][1], 30),
            (mix[2][0], mix[2][1], 25), (mix[1][0], mix[1][1], 20)]
    budget = 2 * sum(atvb.request_bytes(d) for d, _, _ in reqs)
    srv = atvb.Server(ctx, budget)
    ids = [srv.submit(*reqs[0])]
    srv.tick(5)                                  # the first request is running
    assert srv.poll(ids[0])["state"] == 1
    ids.append(srv.submit(*reqs[1]))             # arrives mid-run
    srv.tick(5)
    st = srv.stats()
    assert st["running"] == 2                    # both on the device together
    ids.append(srv.submit(*reqs[2]))
    srv.tick(5)
    ids.append(srv.submit(*reqs[3]))
    peak = 0
    for _ in range(200):
        srv.tick(5)
        st = srv.stats()
        peak = max(peak, st["running"])
        if st["queued"] == 0 and st["running"] == 0:
            break
    assert peak >= 2
    outs = [srv.collect(r) for r in ids]
    srv.close()
    # the late arrivals started before the first request finished
    assert outs[1][1]["t_start"] < outs[0][1]["t_done"]
    for (d, f, n), (out, res) in zip(reqs, outs):
        assert res["steps_done"] == n
        alone, sa = _alone(atvb, ctx, d, f, n)
        _same(out, alone)
        assert res["scalars"]["energy"] == sa["energy"]


@pytest.mark.gpu
def test_server_admission_cancel_and_errors(atvb, ctx):
    from atomiverse_b200 import workloads as W
    d1, f1 = W.lj_fcc(ncell=5, seed=21, precision=1)
    d2, f2 = W.lj_fcc(ncell=6, seed=22, precision=1)
    b1, b2 = atvb.request_bytes(d1), atvb.request_bytes(d2)
    srv = atvb.Server(ctx, max(b1, b2))
    with pytest.raises(atvb.AtvbError) as e:      # bigger than the whole budget
        big, fb = W.lj_fcc(ncell=12, seed=23, precision=1)
        srv.submit(big, fb, 10)
    assert e.value.code == 5
    r1 = srv.submit(d1, f1, 50)
    r2 = srv.submit(d2, f2, 50)
    srv.tick(5)
    assert srv.poll(r1)["state"] == 1 and srv.poll(r2)["state"] == 0
    srv.cancel(r2)
    assert srv.poll(r2)["state"] == 3
    srv.cancel(r1)                                 # a running request frees its slot
    assert srv.poll(r1)["state"] == 3
    assert srv.stats()["bytes"] == 0
    with pytest.raises(atvb.AtvbError) as e:
        srv.poll(12345)
    assert e.value.code == 6
    srv.close()


@pytest.mark.gpu
def test_cpp_md_example(atvb):
    exe = os.path.join(ROOT, "tests", "cpp", "md_example")
    lib_dir = os.path.join(ROOT, "atomiverse_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "md_example.cpp"), "-o", exe,
                    "-L", lib_dir, "-latvb", "-Wl,-rpath," + lib_dir], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    step, e1, e2, ke = int(out[0]), float(out[1]), float(out[2]), float(out[3])
    assert step == 100
    assert ke > 0
    assert abs(e2 - e1) <= 1e-3 * abs(e1)          # NVE: total energy conserved


@pytest.mark.gpu
def test_cpp_thermo_output(atvb, tmp_path):
    """md::MD::set_thermo(25, file): cpu::thermo_print's columns on stdout and
    in the file; steps carry the driver's zero-based iteration index, which
    runs on across run() calls (md.cuh:170), so 2 x 50 steps print 0, 25,
    50, 75."""
    exe = str(tmp_path / "md_example")
    lib_dir = os.path.join(ROOT, "atomiverse_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "md_example.cpp"), "-o", exe,
                    "-L", lib_dir, "-latvb", "-Wl,-rpath," + lib_dir], check=True)
    dat = tmp_path / "thermo.dat"
    lines = subprocess.run([exe, "25", str(dat)], capture_output=True, text=True,
                           check=True).stdout.splitlines()
    assert lines[0].split() == ["Step", "Temp", "PotEng", "KinEng", "TotEng"]
    rows = [[float(v) for v in ln.split()] for ln in lines[1:5]]
    assert [int(r[0]) for r in rows] == [0, 25, 50, 75]
    final = [float(v) for v in lines[5].split()]
    n = 4 * 6 ** 3
    for r in rows:
        assert r[4] == pytest.approx(r[2] + r[3], abs=2e-6)         # TotEng = Pot + Kin
        assert r[1] == pytest.approx(2 * r[3] / ((3 * n - 3) * 8.617333262e-5), rel=1e-4)
        assert r[4] == pytest.approx(final[2], rel=1e-3)             # NVE
    body = dat.read_text().splitlines()
    assert body[0] == "# Step Temp PotEng KinEng TotEng"
    assert [int(b.split()[0]) for b in body[1:]] == [0, 25, 50, 75]


@pytest.mark.gpu
def test_python_md_thermo(atvb, ctx, capsys):
    """md.MD.set_thermo(5): rows for steps 0, 5, .., 25 across two run()
    calls of 23 and 7 steps, the header once, values from the energy ring."""
    from atomiverse_b200 import workloads as W
    desc, frame = W.lj_fcc(ncell=5, seed=4)
    sim = atvb.MD(ctx=ctx)
    sim.set_neighbor(atvb.NeighborList(desc["nl_cutoff"], desc["nl_skin"]))
    sim.set_evaluator(atvb.PairLJCut(desc["lj_epsilon"], desc["lj_sigma"], desc["lj_cutoff"]))
    sim.set_integrator(atvb.VelocityVerlet(desc["dt"]))
    sim.set_thermo(5)
    fr = dict(frame, box=desc["box"])
    sim.run(fr, 23)
    sim.run(fr, 7)
    out = capsys.readouterr().out.splitlines()
    assert out[0].split() == ["Step", "Temp", "PotEng", "KinEng", "TotEng"]
    rows = [ln.split() for ln in out[1:]]
    assert [int(r[0]) for r in rows] == [0, 5, 10, 15, 20, 25]
    hist = sim._system.history(30)
    for r in rows:
        pe, ke, st = hist[int(r[0])]
        assert int(st) == int(r[0])
        assert float(r[2]) == pytest.approx(pe, abs=1e-6)
        assert float(r[3]) == pytest.approx(ke, abs=1e-6)


@pytest.mark.gpu
def test_server_resident_atom_limit(atvb, ctx):
    from atomiverse_b200 import workloads as W
    reqs = [W.lj_fcc(ncell=c, seed=30 + c, precision=1) for c in (5, 6, 4)]  # 500, 864, 256 atoms
    srv = atvb.Server(ctx, 1 << 34)
    srv.set_limits(900)
    ids = [srv.submit(d, f, 12) for d, f in reqs]
    sizes = {rid: d["n_atoms"] for rid, (d, _) in zip(ids, reqs)}
    for _ in range(50):
        srv.tick(4)
        running = [rid for rid in ids if srv.poll(rid)["state"] == 1]
        assert len(running) == 1 or sum(sizes[r] for r in running) <= 900
        if all(srv.poll(rid)["state"] == 2 for rid in ids):
            break
    assert all(srv.poll(rid)["state"] == 2 for rid in ids)
    with pytest.raises(atvb.AtvbError):
        srv.set_limits(-1)
    srv.close()
