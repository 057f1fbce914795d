"""Mixed-precision build: fixed-point force accumulation and exact cutoff
decisions near the LJ cutoff (GPU).

- pair forces are summed per pair in 64-bit fixed point, so the force on
  every atom is the same whatever the number of lanes per atom;
- a pair whose FP32 distance lies within rounding of the LJ cutoff (where the
  shifted LJ force jumps by ~0.039 eps/sigma at 2.5 sigma) is settled on the
  FP64 positions, so no atom carries a whole flipped pair force: the largest
  per-atom force error stays far below the jump.
"""
import numpy as np
import pytest

from conftest import rms_rel


def _forces(out):
    return np.stack([out["fx"], out["fy"], out["fz"]], axis=1)


def _thermalised(atvb, ctx, desc, frame, steps):
    s = atvb.System(ctx, desc, frame)
    s.compute_forces()
    s.step(steps)
    snap, _ = s.download()
    s.close()
    return dict(frame, **{k: snap[k] for k in ("x", "y", "z", "vx", "vy", "vz")})


@pytest.mark.gpu
def test_mixed_forces_do_not_depend_on_lanes(atvb, ctx):
    from atomiverse_b200 import workloads as W
    desc, frame = W.rocksalt_melt(ncell=10, rc=10.0, grid=(30, 30, 30), precision=1)
    ref = None
    for lanes in (1, 4, 32):
        s = atvb.System(ctx, desc, frame)
        s.set_pair_lanes(lanes)
        s.compute_forces()
        out, _ = s.download()
        s.close()
        f = _forces(out)
        if ref is None:
            ref = f
        else:
            assert np.array_equal(f, ref), lanes


@pytest.mark.gpu
def test_mixed_lj_cutoff_decisions_match_fp64(atvb, ctx):
    from atomiverse_b200 import workloads as W
    desc, frame = W.lj_fcc(ncell=24, t_star=0.72, seed=2028)     # 55,296 atoms
    frame = _thermalised(atvb, ctx, desc, frame, 300)
    s64 = atvb.System(ctx, desc, frame)
    s64.compute_forces()
    f64 = _forces(s64.download()[0])
    s64.close()
    sm = atvb.System(ctx, dict(desc, precision=1), frame)
    sm.compute_forces()
    f32 = _forces(sm.download()[0])
    sm.close()
    err = np.linalg.norm(f32 - f64, axis=1)
    assert rms_rel(f32, f64) <= 2e-6
    # one flipped pair would put ~0.039 eps/sigma on two atoms
    assert err.max() < 2e-3
