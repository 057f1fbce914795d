"""Checkpoints (state I/O): save a system mid-run, restore it into a fresh
system, step on -- the trajectory equals the one that never stopped, bit for
bit, for every integrator and both precisions (neighbour rows, their order
and the lane count are those of the saved run).  Bad blobs are refused."""
import numpy as np
import pytest

KB = 8.617333262e-5
KEYS = ("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz")


def _cases():
    from atomiverse_b200 import workloads as W
    from test_gpu_general import _water
    out = []
    d, f = W.rocksalt_melt(ncell=6, rc=5.5, grid=(20, 20, 20))          # NH + PME
    out.append(("pme_nh_fp64", d, f, {}))
    out.append(("pme_nh_mixed", dict(d, precision=1), f, {}))
    d, f = W.lj_fcc(ncell=6, precision=1, thermostat=2, t_star=1.0)     # Langevin
    out.append(("lj_langevin_mixed", d, f, {}))
    d, f = W.lj_fcc(ncell=5, seed=11)    # hot enough for list rebuilds in 40 steps
    npt = dict(T_target=1.44 / KB, tau_T=5.0, P_target=0.0, tau_P=50.0, dt=d["dt"])
    out.append(("lj_npt_fp64", d, f, dict(npt=npt)))
    out.append(("lj_npt_mixed", dict(d, precision=1), f, dict(npt=npt)))
    d, f, coeffs, special = _water(m=8)
    out.append(("water_general_fp64", dict(d, dt=0.5), f,
                dict(lj_types=coeffs, special_bonds=special)))
    return out


CASES = _cases()


@pytest.mark.gpu
@pytest.mark.parametrize("name,desc,frame,opts", CASES, ids=[c[0] for c in CASES])
def test_restore_continues_bit_for_bit(atvb, ctx, name, desc, frame, opts):
    a = atvb.System(ctx, desc, frame, **opts)
    a.compute_forces()
    a.step(40)
    oa, sa = a.download()
    a.close()
    b = atvb.System(ctx, desc, frame, **opts)
    b.compute_forces()
    b.step(15)
    blob = b.save()
    b.close()
    c = atvb.System(ctx, desc, None, **opts)
    c.restore(blob)
    c.step(25)
    oc, sc = c.download()
    c.close()
    for k in KEYS:
        assert np.array_equal(oa[k], oc[k]), (name, k)
    for k in ("step", "energy", "kinetic", "conserved", "rebuilds"):
        assert sa[k] == sc[k], (name, k)
    assert np.array_equal(sa["box"], sc["box"])
    assert sa["rebuilds"] > 0


@pytest.mark.gpu
def test_batch_restore_and_bad_blobs(atvb, ctx):
    from atomiverse_b200 import workloads as W
    d1, f1 = W.lj_fcc(ncell=5, seed=7)
    d2, f2 = W.rocksalt_melt(ncell=6, rc=5.5, grid=(20, 20, 20), precision=1)
    s = atvb.System(ctx, d2, f2)
    s.compute_forces()
    s.step(10)
    blob = s.save()
    s.step(10)
    want, _ = s.download()
    s.close()
    b = atvb.Batch(ctx, [(d1, f1), (d2, None)])
    b.restore(1, blob)
    b.step(10)
    got, _ = b.download(1)
    for k in KEYS:
        assert np.array_equal(want[k], got[k]), k
    with pytest.raises(atvb.AtvbError) as e:
        b.restore(1, blob)                         # already running
    assert e.value.code == 4
    b.close()
    other = atvb.System(ctx, d1)                   # different system
    with pytest.raises(atvb.AtvbError) as e:
        other.restore(blob)
    assert e.value.code == 1
    with pytest.raises(atvb.AtvbError):
        other.restore(blob[:100])                  # truncated
    bad = bytearray(blob)
    bad[0:8] = b"NOTACKPT"
    same = atvb.System(ctx, d2)
    with pytest.raises(atvb.AtvbError):
        same.restore(bytes(bad))
    same.restore(blob)                             # the good one still works
    other.close()
    same.close()


@pytest.mark.gpu
def test_server_resumable_segments(atvb, ctx):
    """Serve a request in segments -- run, suspend, resume; keep a finished
    request's state and extend it; move a running request to a second
    server by checkpoint -- every path ends where one uninterrupted run of
    the same steps ends, bit for bit."""
    from atomiverse_b200 import workloads as W
    d1, f1 = W.lj_fcc(ncell=5, seed=21, precision=1)
    d2, f2 = W.rocksalt_melt(ncell=6, rc=5.5, grid=(20, 20, 20), precision=1)
    ref = {}
    for key, (d, f) in {"lj": (d1, f1), "melt": (d2, f2)}.items():
        s = atvb.System(ctx, d, f)
        s.compute_forces()
        s.step(30)
        ref[key] = s.download()[0]
        s.close()
    srv = atvb.Server(ctx, 1 << 34)
    srv.keep_checkpoints(True)
    a = srv.submit(d1, f1, 30)                    # one segment of 30
    b = srv.submit(d2, f2, 12)                    # 12, then 18 more
    c = srv.submit(d2, f2, 30)                    # suspended at 10, resumed
    srv.tick(10)
    srv.suspend(c)
    assert srv.poll(c)["state"] == 5
    srv.tick(2)
    assert srv.poll(b)["state"] == 2
    srv.resume(b, 18)
    srv.resume(c, 20)
    blob, done_at = None, 0
    for _ in range(20):
        srv.tick(6)
        pa = srv.poll(a)
        if blob is None and pa["state"] == 1 and pa["steps_done"] >= 15:
            blob, done_at = srv.checkpoint(a), pa["steps_done"]   # a running request
        if all(srv.poll(r)["state"] == 2 for r in (a, b, c)):
            break
    for rid, key in ((a, "lj"), (b, "melt"), (c, "melt")):
        out, res = srv.collect(rid)
        for k in KEYS:
            assert np.array_equal(out[k], ref[key][k]), (rid, k)
    assert blob is not None
    srv2 = atvb.Server(ctx, 1 << 34)               # migrate: finish a's copy elsewhere
    m = srv2.submit_checkpoint(d1, blob, 30 - done_at)
    for _ in range(10):
        srv2.tick(6)
        if srv2.poll(m)["state"] == 2:
            break
    out, _ = srv2.collect(m)
    for k in KEYS:
        assert np.array_equal(out[k], ref["lj"][k]), k
    srv.close()
    srv2.close()


@pytest.mark.gpu
def test_cpp_checkpoint_resume(atvb, tmp_path):
    """md::MD::checkpoint / restore continue an NPT run bit for bit; the
    snapshot ring delivered the frames of steps 20, 40, 60, 80."""
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = str(tmp_path / "md_resume")
    lib_dir = os.path.join(root, "atomiverse_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(root, "include"),
                    os.path.join(root, "tests", "cpp", "md_resume.cpp"), "-o", exe,
                    "-L", lib_dir, "-latvb", "-Wl,-rpath," + lib_dir], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.split() == ["OK", "4"]
