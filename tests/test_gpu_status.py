"""No silent wrong physics: every condition under which a step ran on wrong
or non-finite physics raises a sticky status bit, and the calls that report
state (scalars, download, run) then fail with ATVB_ERR_PHYSICS.

Each condition is made on the host: a pinned row capacity below what the
rows need, a one-entry near-cutoff queue, a NaN coordinate in the uploaded
frame (the force kernels map it to an ordinary in-range fixed-point
coordinate, so nothing on the device reads out of bounds).  The reference's
cuda::StopOnNaN (criterion.cuh:166-178) stops a run whose state is no
longer finite; StopOnNaN here halts the system on the device.
"""
import numpy as np
import pytest

from atomiverse_b200 import workloads as W
from conftest import oracle_system, rms_rel

pytestmark = pytest.mark.gpu


def _pairs_set(pi, pj):
    a = np.minimum(pi, pj).astype(np.int64)
    b = np.maximum(pi, pj).astype(np.int64)
    return np.unique(a * (1 << 32) + b)


def _hot_lj(ncell=8, seed=5, precision=0):
    # a hot, small-skin fluid: the list is rebuilt every few steps
    desc, frame = W.lj_fcc(ncell=ncell, t_star=2.5, seed=seed, skin=0.1,
                           precision=precision)
    desc["stress_required"] = 1
    return desc, frame


def test_row_overflow_is_flagged_and_healed(atvb, ctx, orc):
    desc, frame = _hot_lj()
    s = atvb.System(ctx, desc, frame)
    s.compute_forces()
    m = s.scalars()["max_neighbors"]
    # pin the rows shorter than the longest one: every build cuts rows
    s.set_capacity(row_capacity=m - 8)
    s.step(40)
    with pytest.raises(atvb.PhysicsError) as ei:
        s.scalars()
    sc = ei.value.result
    assert sc["status_bits"] & 1 and sc["status"] == 3
    with pytest.raises(atvb.PhysicsError):
        s.download()
    out, sc = s.download(check=False)
    assert sc["step"] == 40 and sc["status_bits"] & 1
    # unpinned: the next call widens the rows and builds again at once
    s.set_capacity(row_capacity=0)
    s.clear_status()
    s.step(3)
    sc = s.scalars()                      # no bit: nothing was cut since
    assert sc["status_bits"] == 0
    # the healed list equals the oracle's at the current positions
    s.compute_forces()
    out, sc = s.download()
    gi, gj = s.pairs()
    ref = oracle_system(orc, desc, out)
    ref.build_list()
    ref.compute_forces()
    oi, oj = ref.pairs()
    assert np.array_equal(_pairs_set(gi, gj), _pairs_set(oi, oj))
    rs = ref.state()
    f = np.stack([out["fx"], out["fy"], out["fz"]], 1)
    fr = np.stack([rs["fx"], rs["fy"], rs["fz"]], 1)
    assert rms_rel(f, fr) < 1e-10


def test_pinned_capacity_refuses_a_short_force_pass(atvb, ctx):
    desc, frame = _hot_lj()
    s = atvb.System(ctx, desc, frame)
    m = s.scalars()["max_neighbors"]
    s.set_capacity(row_capacity=m - 8)
    s.clear_status()
    with pytest.raises(atvb.AtvbError) as ei:
        s.compute_forces()                # outside a step: refused, not cut
    assert ei.value.code == 3


def test_near_queue_overflow_is_flagged(atvb, ctx):
    # mixed LJ: pairs within the FP32 error band of the cutoff are queued
    # for an exact decision; a one-entry queue loses some
    desc, frame = W.lj_fcc(ncell=20, seed=9, precision=1)
    s = atvb.System(ctx, desc, frame)
    s.set_capacity(nearq_capacity=1)
    s.compute_forces()
    s.step(30)
    sc = s.scalars(check=False)
    assert sc["status_bits"] & 4
    with pytest.raises(atvb.PhysicsError):
        s.scalars()
    # a default-sized queue loses nothing
    s2 = atvb.System(ctx, desc, frame)
    s2.compute_forces()
    s2.step(30)
    assert s2.scalars()["status_bits"] == 0


def test_nan_position_is_flagged(atvb, ctx):
    desc, frame = _hot_lj(ncell=6)
    frame = {k: (v.copy() if hasattr(v, "copy") else v) for k, v in frame.items()}
    frame["x"][17] = np.nan
    s = atvb.System(ctx, desc, frame)
    s.step(5)
    sc = s.scalars(check=False)
    assert sc["status_bits"] & 8 and not sc["halted"] and sc["step"] == 5
    with pytest.raises(atvb.PhysicsError):
        s.download()


def test_stop_on_nan_halts_the_system(atvb, ctx):
    desc, frame = _hot_lj(ncell=6)
    frame = {k: (v.copy() if hasattr(v, "copy") else v) for k, v in frame.items()}
    frame["vy"][3] = np.inf
    s = atvb.System(ctx, desc, frame)
    s.set_stop_on_nan(True)
    s.step(5)
    out, sc = s.download(check=False)
    # the first step's drift met the infinite velocity: that step is the last
    assert sc["halted"] and sc["status_bits"] & 8 and sc["step"] == 1
    with pytest.raises(atvb.PhysicsError):
        s.step(2)                         # a halted system refuses to step
    # the reference-shaped API: MD.add_criterion(StopOnNaN()) -> PhysicsError
    md = atvb.MD(ctx=ctx)
    md.set_neighbor(atvb.NeighborList(desc["nl_cutoff"], desc["nl_skin"]))
    md.set_evaluator(atvb.PairLJCut(1.0, 1.0, desc["lj_cutoff"]))
    md.set_integrator(atvb.VelocityVerlet(desc["dt"]))
    md.add_criterion(atvb.StopOnNaN())
    fr = {k: (v.copy() if hasattr(v, "copy") else v) for k, v in frame.items()}
    fr["box"] = desc["box"]
    with pytest.raises(atvb.PhysicsError):
        md.run(fr, 4)                     # (run() downloads into fr's arrays)
    # clearing the status resumes a system whose state was repaired
    s2 = atvb.System(ctx, desc, frame)
    s2.set_stop_on_nan(True)
    s2.step(2)
    assert s2.scalars(check=False)["halted"]
    _, good = _hot_lj(ncell=6)            # a finite state, freshly made
    good["vy"] = np.zeros_like(good["vy"])
    s2.upload(good)
    s2.clear_status()
    s2.step(3)
    assert s2.scalars()["step"] == 3


def test_step_timed_runs_in_pieces_like_step(atvb, ctx):
    # 1,200 steps cross the 1,000-step piece boundary (row check and cell
    # re-plan between pieces): step_timed must give the trajectory of step
    desc, frame = _hot_lj(ncell=5, seed=3, precision=1)
    a = atvb.System(ctx, desc, frame)
    b = atvb.System(ctx, desc, frame)
    a.compute_forces()
    b.compute_forces()
    total, per = a.step_timed(1200)
    b.step(1200)
    oa, sa = a.download()
    ob, sb = b.download()
    assert len(per) == 1200 and total > 0 and np.all(per > 0)
    assert abs(per.sum() - total) < 1e-3 * total + 1e-3
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(oa[k], ob[k])
    assert sa["step"] == sb["step"] == 1200


def test_force_beyond_fixed_point_is_flagged(atvb, ctx):
    # mixed LJ: two atoms 0.05 sigma apart carry a pair force far beyond the
    # range of the 64-bit fixed-point row sums (2^31 eV/A)
    desc, frame = W.lj_fcc(ncell=6, seed=4, precision=1)
    frame = {k: (v.copy() if hasattr(v, "copy") else v) for k, v in frame.items()}
    frame["x"][1], frame["y"][1], frame["z"][1] = frame["x"][0] + 0.05, frame["y"][0], frame["z"][0]
    s = atvb.System(ctx, desc, frame)
    s.compute_forces()
    sc = s.scalars(check=False)
    assert sc["status_bits"] & 16
    with pytest.raises(atvb.PhysicsError):
        s.scalars()
    # the same system without the overlap raises nothing
    desc2, frame2 = W.lj_fcc(ncell=6, seed=4, precision=1)
    s2 = atvb.System(ctx, desc2, frame2)
    s2.compute_forces()
    s2.step(5)
    assert s2.scalars()["status_bits"] == 0
