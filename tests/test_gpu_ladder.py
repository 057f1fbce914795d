"""The full replica ladder (512 LJ systems, 256-32,768 atoms, seed 2029,
Langevin, mixed precision) advanced as one batch: every system equals the
same system run alone, bit for bit, and sampled systems' pair forces agree
with the CPU FP64 oracle within the mixed build's tolerance."""
import numpy as np
import pytest

from atomiverse_b200 import workloads as W
from conftest import oracle_system, rms_rel

pytestmark = pytest.mark.gpu

STEPS = 4


def test_full_ladder_batch_equals_alone(atvb, ctx, orc):
    items = W.ladder(n_systems=512, precision=atvb.MIXED)
    b = atvb.Batch(ctx, items)
    b.compute_forces()
    b.step(STEPS)
    batched = [b.download(k, keys=("x", "y", "z", "vx", "vy", "vz"))[0]
               for k in range(len(items))]
    launches = b.launch_count()
    b.close()
    # one launch per kernel per step for all 512 systems (not per system)
    assert launches < 40 * STEPS
    for k, (desc, frame) in enumerate(items):
        s = atvb.System(ctx, desc, frame)
        s.compute_forces()
        s.step(STEPS)
        alone, sc = s.download(keys=("x", "y", "z", "vx", "vy", "vz"))
        s.close()
        assert sc["step"] == STEPS
        for c in ("x", "y", "z", "vx", "vy", "vz"):
            assert np.array_equal(batched[k][c], alone[c]), (k, c)
    # sampled systems: mixed pair forces at the reached positions vs the oracle
    for k in (0, 255, 511):
        desc, frame = items[k]
        snap = dict(frame, **{c: batched[k][c] for c in ("x", "y", "z")})
        s = atvb.System(ctx, desc, snap)
        s.compute_forces()
        out, _ = s.download()
        s.close()
        o = oracle_system(orc, dict(desc, thermostat=0), snap)
        o.build_list()
        o.compute_forces()
        st = o.state()
        o.close()
        f = np.stack([out["fx"], out["fy"], out["fz"]], 1)
        fr = np.stack([st["fx"], st["fy"], st["fz"]], 1)
        assert rms_rel(f, fr) <= 5e-6, k
