"""User components through the reference's plugin boundary: a C++ program
built against include/atomiverse_b200/md.hpp plugs a harmonic wall (its own
CUDA kernel) into the force phase with MD::on(md::Phase::force).add(c,
order); the library runs it at every step and adds its forces and energy.
The trajectory matches the CPU FP64 oracle with the same wall term, build
and destroy run once, the step index is cumulative across run() calls, and
the plan's stress verdict reaches set_stress_required."""
import os
import subprocess

import numpy as np
import pytest

from atomiverse_b200 import workloads as W
from conftest import oracle_system, rms_rel

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    exe = str(tmp_path / "md_wall")
    lib_dir = os.path.join(ROOT, "atomiverse_b200")
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "md_wall.cu"), "-o", exe,
                    "-L", lib_dir, "-latvb", "-Xlinker", "-rpath," + lib_dir], check=True)
    return exe


def test_cpp_harmonic_wall_component_matches_oracle(atvb, ctx, orc, tmp_path):
    desc, frame = W.lj_fcc(ncell=8, seed=17)
    n, L = desc["n_atoms"], desc["box"][0]
    zw, kw = 0.6 * L, 0.5
    path = tmp_path / "frame.bin"
    with open(path, "wb") as fh:
        fh.write(np.array([n], dtype=np.int64).tobytes())
        fh.write(np.array(list(desc["box"][:3]) + [desc["dt"], desc["lj_cutoff"],
                                                   desc["nl_skin"], zw, kw]).tobytes())
        for k in ("x", "y", "z", "vx", "vy", "vz", "mass"):
            fh.write(np.ascontiguousarray(frame[k], dtype=np.float64).tobytes())
    exe = _build(tmp_path)
    out_path = tmp_path / "out.bin"
    r = subprocess.run([exe, str(path), "20", "30", str(out_path)], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    energy, kinetic, builds, destroys, last, stress = r.stdout.split()
    assert (int(builds), int(destroys)) == (1, 1)
    assert int(last) == 49                         # cumulative over the two run() calls
    assert int(stress) == 1                        # StepProbe requires the virial
    got = np.fromfile(out_path, dtype=np.float64).reshape(9, n)

    # run(frame, n) starts from the frame's forces (zero here), as the
    # reference's setup_pass does (driver.cuh:344-359): no force pass first
    o = oracle_system(orc, dict(desc, wall_axis=2, wall_pos=zw, wall_k=kw), frame)
    o.build_list()
    o.run(50)
    ref, rsc = o.state(), o.scalars()
    o.close()
    for ax, k in enumerate("xyz"):
        d = got[ax] - ref[k]
        d -= L * np.rint(d / L)
        assert np.abs(d).max() < 1e-8, (k, np.abs(d).max())
    f = got[6:9].T
    fr = np.stack([ref["fx"], ref["fy"], ref["fz"]], 1)
    assert rms_rel(f, fr) < 1e-8
    assert float(energy) == pytest.approx(rsc["energy"], rel=1e-9)
    assert float(kinetic) == pytest.approx(rsc["kinetic"], rel=1e-9)

    # without the wall the trajectory is a different one: the component acted
    o2 = oracle_system(orc, desc, frame)
    o2.build_list()
    o2.run(50)
    free = o2.state()
    o2.close()
    assert np.abs(free["z"] - ref["z"]).max() > 1e-4
