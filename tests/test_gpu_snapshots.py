"""Trajectory snapshots: the step graph publishes positions and velocities
every k steps into a host-mapped ring (seqlock per slot); polling needs no
device synchronisation.  Frames equal what a download at that step gives,
bit for bit; frames overwritten before a poll are counted as dropped."""
import numpy as np
import pytest

KB = 8.617333262e-5


@pytest.mark.gpu
def test_snapshots_equal_downloads(atvb, ctx):
    from atomiverse_b200 import workloads as W
    desc, frame = W.rocksalt_melt(ncell=6, rc=5.5, grid=(20, 20, 20))   # NH + PME
    s = atvb.System(ctx, desc, frame)
    with pytest.raises(atvb.AtvbError) as e:
        s.poll_snapshots()
    assert e.value.code == 4
    s.set_snapshots(every=5, depth=16)
    s.compute_forces()
    s.step(20)
    out, sc = s.download()                       # synchronises
    frames, dropped = s.poll_snapshots()
    assert dropped == 0
    assert [f[0] for f in frames] == [5, 10, 15, 20]
    step, box, fr = frames[-1]
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(fr[k], out[k]), k
    assert np.array_equal(box, sc["box"])
    assert s.poll_snapshots()[0] == []           # nothing new
    ref = atvb.System(ctx, desc, frame)
    ref.compute_forces()
    ref.step(10)
    o10, _ = ref.download()
    ref.close()
    for k in ("x", "vx"):
        assert np.array_equal(frames[1][2][k], o10[k]), k
    s.close()


@pytest.mark.gpu
def test_snapshot_ring_overrun_and_npt_cell(atvb, ctx):
    from test_gpu_npt import _lj_cube
    desc, frame = _lj_cube()
    npt = dict(T_target=1.0 / KB, tau_T=0.1, P_target=0.0, tau_P=1.0, dt=0.005)
    s = atvb.System(ctx, desc, frame, npt=npt)
    s.set_snapshots(every=1, depth=2)
    s.step(10)
    _, sc = s.download()
    frames, dropped = s.poll_snapshots()
    assert [f[0] for f in frames] == [9, 10]
    assert dropped == 8
    assert np.array_equal(frames[-1][1], sc["box"])
    assert frames[-1][1][0] != desc["box"][0]    # the cell moved
    s.set_snapshots(every=0, depth=0)            # off
    s.step(3)
    with pytest.raises(atvb.AtvbError):
        s.poll_snapshots()
    s.close()
