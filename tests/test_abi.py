"""The C ABI library: it loads, exports exactly what include/atvb.h declares,
and validates inputs on the host (CPU only; no kernel is launched)."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "atvb.h")


def _declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(atvb_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(atvb):
    lib_path = atvb.library_path()
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(atvb_\w+)", out))
    declared = _declared()
    assert declared, "no declarations parsed"
    missing = [s for s in declared if s not in exported]
    assert not missing, missing


def test_python_binding_covers_header(atvb):
    from atomiverse_b200 import _abi
    assert sorted(_abi.SIGNATURES) == _declared()


def test_abi_version_and_error_string(atvb):
    lib = atvb.load()
    assert lib.atvb_abi_version() == 1
    assert lib.atvb_last_error() is not None


def test_host_validation_without_gpu(atvb):
    """atvb_request_bytes runs the host-side geometry checks only."""
    good = atvb.make_desc(4000, (16.8, 16.8, 16.8), nl_cutoff=2.5, nl_skin=0.3,
                          lj_enabled=1, lj_epsilon=1.0, lj_sigma=1.0, lj_cutoff=2.5, dt=0.05)
    assert atvb.request_bytes(good) > 4000 * 100
    tri = atvb.make_desc(10, (20.0, 1.0, 0.0, 0.0, 20.0, 0.0, 0.0, 0.0, 20.0), nl_cutoff=2.5,
                         dt=1.0)
    with pytest.raises(atvb.AtvbError) as e:
        atvb.request_bytes(tri)
    assert e.value.code == 1 and "orthorhombic" in str(e.value)
    small = atvb.make_desc(10, (5.0, 5.0, 5.0), nl_cutoff=2.5, nl_skin=0.3, dt=1.0)
    with pytest.raises(atvb.AtvbError):
        atvb.request_bytes(small)


def test_ctx_without_device_fails_cleanly(atvb):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(atvb.AtvbError) as e:
        atvb.Context(0)
    assert e.value.code == 2


def test_cpp_header_compiles():
    """The C ABI header is plain C and compiles as C and C++."""
    for lang, cc in (("c", "gcc"), ("c++", "g++")):
        r = subprocess.run([cc, "-x", lang, "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
                            "-"], input='#include "atvb.h"\nint main(void){return 0;}\n',
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def test_cpp_mirror_compiles():
    """The header-only C++ mirror compiles with every component bound, and
    so does each C++ driver program under tests/cpp."""
    snippet = r'''
#include <atomiverse_b200/md.hpp>
int main() {
    using namespace atvb_cpp;
    md::MD a(0, ATVB_FP64);
    a.set_neighbor(NeighborList(2.5, 0.3)).set_evaluator(PairLJCut(1.0, 1.0, 2.5))
     .set_integrator(md::NVELimit(0.005, 0.01));
    a.set_thermostat(md::Deform(2, 1e-3, 0.005));
    a.set_barostat(md::Barostat(0.0, 1.0, 0.005));
    md::MD b(0, ATVB_MIXED);
    b.set_neighbor(NeighborList(2.5, 0.3)).set_evaluator(PairLJCut(1.0, 1.0, 2.5))
     .set_integrator(md::NoseHooverNPT(100.0, 0.1, 0.0, 1.0, 0.005));
    return 0;
}
'''
    r = subprocess.run(["g++", "-std=c++17", "-x", "c++", "-fsyntax-only", "-I",
                        os.path.join(ROOT, "include"), "-"], input=snippet,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    cpp = os.path.join(ROOT, "tests", "cpp")
    for name in sorted(os.listdir(cpp)):
        if name.endswith(".cpp"):
            r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I",
                                os.path.join(ROOT, "include"), os.path.join(cpp, name)],
                               capture_output=True, text=True)
            assert r.returncode == 0, (name, r.stderr)
