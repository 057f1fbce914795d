"""atvb_pair_forces_static: the allocation-free pair-force entry point.

Compared with the library's main path (atvb_system_compute_forces on a
system without PME, whose pair forces and LJ / real-space Coulomb energies
are the same physics) on two calls in a row with different inputs, with
the CPU FP64 oracle directly, in its LJ-only (no charge array),
Coulomb-only and no-energy forms, plus the up-front rejections.  This file
sorts last so it also runs after every other GPU test in the same process.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import oracle_system, rms_rel


def _case(atvb, ncell, seed, rc=10.0):
    from atomiverse_b200 import workloads as W
    desc, frame = W.rocksalt_melt(ncell=ncell, seed=seed, rc=rc, skin=1.0)
    desc["pme_enabled"] = 0
    desc.pop("pme_grid", None)
    return desc, frame


def _static(atvb, torch, desc, frame, stream=None, charges=True, energy=True):
    dev = torch.device("cuda:0")
    t = {k: torch.as_tensor(np.ascontiguousarray(frame[k]), dtype=torch.float64, device=dev)
         for k in ("x", "y", "z", "charge")}
    n = desc["n_atoms"]
    f = [torch.full((n,), float("nan"), dtype=torch.float64, device=dev) for _ in range(3)]
    e = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
    d = atvb.make_desc(**desc)
    lib = atvb.load()
    rc = lib.atvb_pair_forces_static(
        C.byref(d), t["x"].data_ptr(), t["y"].data_ptr(), t["z"].data_ptr(),
        t["charge"].data_ptr() if charges else None, f[0].data_ptr(), f[1].data_ptr(),
        f[2].data_ptr(), e.data_ptr() if energy else None, stream)
    atvb.check(rc)
    torch.cuda.synchronize()
    return np.stack([a.cpu().numpy() for a in f], axis=1), e.cpu().numpy()


def _oracle(orc, desc, frame):
    o = oracle_system(orc, dict(desc, pme_enabled=0), frame)
    o.build_list()
    o.compute_forces()
    st, sc = o.state(), o.scalars()
    o.close()
    return np.stack([st["fx"], st["fy"], st["fz"]], axis=1), sc


@pytest.mark.gpu
@pytest.mark.parametrize("ncell", [12, 8])  # 3 cells per axis; 2 cells (whole-axis walk)
def test_static_matches_main_path_two_calls(atvb, ctx, ncell):
    torch = pytest.importorskip("torch")
    for seed in (3, 4):
        desc, frame = _case(atvb, ncell, seed)
        sys_ = atvb.System(ctx, desc, frame)
        sys_.compute_forces()
        out, sc = sys_.download()
        ref = np.stack([out["fx"], out["fy"], out["fz"]], axis=1)
        del sys_
        f, e = _static(atvb, torch, desc, frame)
        assert np.all(np.isfinite(f))
        assert rms_rel(f, ref) <= 1e-6
        assert e[0] == pytest.approx(sc["energy_lj"], rel=1e-9, abs=1e-6)
        assert e[1] == pytest.approx(sc["energy_coul"], rel=1e-9, abs=1e-6)


@pytest.mark.gpu
def test_static_repeats_bitwise_and_honours_stream(atvb, ctx):
    torch = pytest.importorskip("torch")
    desc, frame = _case(atvb, 12, 5)
    f1, e1 = _static(atvb, torch, desc, frame)
    s = torch.cuda.Stream()
    f2, e2 = _static(atvb, torch, desc, frame, stream=s.cuda_stream)
    assert np.array_equal(f1, f2)
    assert np.array_equal(e1, e2)


def test_static_rejects_oversize_and_bad_boxes(atvb):
    """Every rejection happens on the host before any CUDA call, so this
    runs without a GPU."""
    lib = atvb.load()
    desc, _ = _case(atvb, 12, 3)
    null = [None] * 9

    def call(**over):
        d = dict(desc)
        d.update(over)
        return lib.atvb_pair_forces_static(C.byref(atvb.make_desc(**d)), *null)

    assert call(n_atoms=65537) == 1          # more atoms than the scratch holds
    assert call(box=(500.0, 500.0, 500.0), lj_cutoff=1.0, coul_cutoff=1.0) == 1  # > 65536 cells
    assert call(box=(15.0, 40.0, 40.0)) == 1  # edge below twice the cutoff
    assert call(pme_enabled=1) == 1
    assert call(precision=1) == 1
    assert call() == 1                        # valid description, NULL arrays
    assert "NULL" in lib.atvb_last_error().decode()
    assert lib.atvb_pair_forces_static(None, *null) == 1


@pytest.mark.gpu
def test_static_matches_oracle(atvb, ctx, orc):
    """Against the CPU FP64 oracle directly (LJ + real-space Coulomb)."""
    torch = pytest.importorskip("torch")
    desc, frame = _case(atvb, 12, 6)
    fref, sc = _oracle(orc, desc, frame)
    f, e = _static(atvb, torch, desc, frame)
    assert rms_rel(f, fref) <= 1e-6
    assert e[0] == pytest.approx(sc["e_lj"], rel=1e-9, abs=1e-6)
    assert e[1] == pytest.approx(sc["e_coul"], rel=1e-9, abs=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["lj_only", "coul_only", "no_energy"])
def test_static_partial_forms(atvb, ctx, orc, form):
    """LJ only with no charge array, Coulomb only, and no energy output:
    forces against the main path and the oracle, twice in a row."""
    torch = pytest.importorskip("torch")
    for seed in (7, 8):
        desc, frame = _case(atvb, 12, seed)
        if form == "lj_only":
            desc["coul_enabled"] = 0
        elif form == "coul_only":
            desc["lj_enabled"] = 0
        sys_ = atvb.System(ctx, desc, frame)
        sys_.compute_forces()
        out, sc = sys_.download()
        sys_.close()
        ref = np.stack([out["fx"], out["fy"], out["fz"]], axis=1)
        fref, osc = _oracle(orc, desc, frame)
        f, e = _static(atvb, torch, desc, frame, charges=(form != "lj_only"),
                       energy=(form != "no_energy"))
        assert np.all(np.isfinite(f))
        assert rms_rel(f, ref) <= 1e-6
        assert rms_rel(f, fref) <= 1e-6
        if form == "no_energy":
            assert np.all(np.isnan(e))         # the energy buffer is not touched
        else:
            assert e[0] == pytest.approx(sc["energy_lj"], rel=1e-9, abs=1e-6)
            assert e[1] == pytest.approx(sc["energy_coul"], rel=1e-9, abs=1e-6)
