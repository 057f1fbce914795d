"""The PME grid transforms in each of their forms, against the CPU FP64
oracle: the register four-step forms (every line length up to 256 that
splits into two factors of at most 16), the generic Stockham kernels (an
odd K2, so a full complex z line; an axis longer than 256), and a batch of
PME systems with different meshes, where each system must get bit for bit
the result it gets alone (its transforms depend on its own mesh only)."""
import numpy as np
import pytest

from atomiverse_b200 import workloads as W
from conftest import oracle_system, rms_rel

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-6
MIXED_TOL = 5e-6


def _case(grid, ncell=8, seed=21, precision=0):
    desc, frame = W.rocksalt_melt(ncell=ncell, seed=seed, grid=grid, rc=10.2,
                                  precision=precision)
    desc["stress_required"] = 1
    return desc, frame


def _f(o):
    return np.stack([o["fx"], o["fy"], o["fz"]], 1)


def _gpu(atvb, ctx, desc, frame):
    s = atvb.System(ctx, desc, frame)
    s.compute_forces()
    out, sc = s.download()
    s.close()
    return out, sc


def _oracle(orc, desc, frame):
    o = oracle_system(orc, desc, frame)
    o.build_list()
    o.compute_forces()
    st, sc = o.state(), o.scalars()
    o.close()
    return st, sc


@pytest.mark.parametrize("grid", [
    (24, 30, 32),    # register forms on every axis (z lines of 16)
    (20, 24, 27),    # odd K2: the generic z passes, register y and x
    (270, 24, 28),   # x longer than 256: the generic x pass
    (42, 36, 50),    # register forms with radix-7 and radix-5 factors
])
def test_forms_match_oracle_fp64(atvb, ctx, orc, grid):
    desc, frame = _case(grid)
    out, sc = _gpu(atvb, ctx, desc, frame)
    ref, rsc = _oracle(orc, desc, frame)
    assert rms_rel(_f(out), _f(ref)) <= FP64_TOL
    assert sc["energy"] == pytest.approx(rsc["energy"], rel=1e-9, abs=1e-7)
    assert np.allclose(sc["stress"], rsc["virial"], rtol=1e-8,
                       atol=1e-8 * np.abs(rsc["virial"]).max())


@pytest.mark.parametrize("grid", [(24, 30, 32), (20, 24, 27)])
def test_forms_match_oracle_mixed(atvb, ctx, orc, grid):
    desc, frame = _case(grid, precision=1)
    out, sc = _gpu(atvb, ctx, desc, frame)
    ref, rsc = _oracle(orc, desc, frame)
    assert rms_rel(_f(out), _f(ref)) <= MIXED_TOL
    assert sc["energy"] == pytest.approx(rsc["energy"], rel=2e-5)


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_of_meshes_equals_alone(atvb, ctx, precision):
    items = [_case(g, ncell=c, seed=s, precision=precision) for g, c, s in (
        ((24, 24, 24), 8, 31), ((30, 30, 30), 10, 32), ((20, 24, 27), 8, 33),
        ((24, 24, 24), 8, 34))]
    b = atvb.Batch(ctx, items)
    b.compute_forces()
    b.step(5)
    for k, (d, f) in enumerate(items):
        ob, sb = b.download(k)
        s = atvb.System(ctx, d, f)
        s.compute_forces()
        s.step(5)
        oa, sa = s.download()
        s.close()
        for key in ("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz"):
            assert np.array_equal(ob[key], oa[key]), (k, key)
        assert sb["energy"] == sa["energy"]
    b.close()
