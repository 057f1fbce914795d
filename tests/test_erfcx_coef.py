"""The compile-time erfcx polynomial used by the pair kernels (CPU only).

erfcx_coef.h holds one polynomial in u = A t + B, t = 1 / (1 + P x), for
erfcx(x) = exp(x^2) erfc(x) on 0 <= x <= 6.  Evaluated the way the kernels
do (Horner, in the storage type), it must match SciPy's erfcx within the
error written in the header, and that error must be small enough for each
build: ~1 ulp for FP64, below 1e-6 for the FP32 (mixed) build.
"""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "atomiverse_b200", "csrc", "erfcx_coef.h")


def _parse():
    txt = open(HDR).read()
    const = {k: float(v) for k, v in re.findall(r"constexpr double (kErfcx[A-Za-z]+) = ([-0-9.e+]+);", txt)}
    arrays = {}
    for name, body in re.findall(r"(kErfcx[DF])\[\d+\] = \{(.*?)\};", txt, flags=re.S):
        arrays[name] = [float(v.rstrip("f")) for v in re.findall(r"[-0-9.e+]+f?", body)]
    errs = [float(e) for e in re.findall(r"Horner evaluation: ([0-9.e+-]+)", txt)]
    return const, arrays, errs


def _horner(c, x, P, A, B, dtype):
    t = (1.0 / (1.0 + P * x)).astype(dtype)
    u = (dtype(A) * t + dtype(B)).astype(dtype)
    cc = np.array(c, dtype=dtype)
    acc = np.full_like(u, cc[-1])
    for k in range(len(cc) - 2, -1, -1):
        acc = (acc * u + cc[k]).astype(dtype)
    return acc


def test_erfcx_polynomials_match_scipy():
    special = pytest.importorskip("scipy.special")
    const, arrays, errs = _parse()
    assert const["kErfcxXmax"] == 6.0
    x = np.linspace(0.0, 6.0, 200001)
    ref = special.erfcx(x)
    e64 = np.max(np.abs(_horner(arrays["kErfcxD"], x, const["kErfcxP"], const["kErfcxA"],
                                const["kErfcxB"], np.float64) / ref - 1))
    e32 = np.max(np.abs(_horner(arrays["kErfcxF"], x, const["kErfcxP"], const["kErfcxA"],
                                const["kErfcxB"], np.float32) / ref - 1))
    assert e64 < 4e-15
    assert e32 < 1e-6
    # the header states what its generator measured
    assert errs[0] < 2e-15 and errs[1] < 1e-6


def test_erfc_from_erfcx_and_exp():
    """erfc(x) = exp(-x^2) erfcx(x): the identity the kernels rely on."""
    special = pytest.importorskip("scipy.special")
    const, arrays, _ = _parse()
    x = np.linspace(0.0, 6.0, 5001)
    got = np.exp(-x * x) * _horner(arrays["kErfcxD"], x, const["kErfcxP"], const["kErfcxA"],
                                   const["kErfcxB"], np.float64)
    assert np.max(np.abs(got / special.erfc(x) - 1)) < 1e-13


def test_table_driven_exp_constants():
    """exp_neg64's table (2^(j/64)) and split ln2/64, evaluated the way the
    kernel does (Tang's table-driven reduction, degree-5 Taylor), stay
    within 2 ulp of exp(-z) on [0, 708]; the head of ln2/64 has enough
    trailing zero bits that n * head is exact."""
    txt = open(HDR).read()
    c = {k: float(v) for k, v in re.findall(r"constexpr double (kExp[A-Za-z0-9]+) = ([-0-9.e+]+);", txt)}
    body = re.search(r"kExp2Tab\[64\] = \{(.*?)\};", txt, flags=re.S).group(1)
    tab = np.array([float(v) for v in re.findall(r"[-0-9.e+]+", body)])
    assert len(tab) == 64
    assert np.allclose(tab, 2.0 ** (np.arange(64) / 64.0), rtol=2e-16, atol=0)
    hi, lo, inv = c["kExpLn2By64Hi"], c["kExpLn2By64Lo"], c["kExp64ByLn2"]
    m, _ = np.frexp(hi)
    assert float(m * 2 ** 29).is_integer()           # <= 29 significant bits
    assert abs((hi + lo) - np.log(2) / 64) < 1e-18
    z = np.concatenate([np.linspace(0.0, 40.0, 200001), np.linspace(40.0, 700.0, 20001)])
    w = -z
    n = np.rint(w * inv)
    r = (w - n * hi) - n * lo
    p = np.full_like(r, 1.0 / 120.0)
    for k in (1.0 / 24.0, 1.0 / 6.0, 0.5, 1.0, 1.0):
        p = p * r + k
    ni = n.astype(np.int64)
    val = tab[ni & 63] * p * np.ldexp(1.0, ni >> 6)
    assert np.max(np.abs(val / np.exp(-z) - 1.0)) < 5e-16   # 2 ulp incl. numpy's own exp


def test_short_range_erfcx_set_matches_scipy():
    """The short FP64 set (alpha * cutoff <= 3.2) evaluated as the kernel
    does (even/odd Horner chains in u^2) stays within 2e-15 of SciPy."""
    special = pytest.importorskip("scipy.special")
    txt = open(HDR).read()
    c = {k: float(v) for k, v in re.findall(r"constexpr double (kErfcxS[A-Za-z]+) = ([-0-9.e+]+);", txt)}
    body = re.search(r"kErfcxS\[\d+\] = \{(.*?)\};", txt, flags=re.S).group(1)
    cs = np.array([float(v) for v in re.findall(r"[-0-9.e+]+", body)])
    x = np.linspace(0.0, c["kErfcxSXmax"], 50001)
    t = 1.0 / (1.0 + c["kErfcxSP"] * x)
    u = c["kErfcxSA"] * t + c["kErfcxSB"]
    v = u * u
    ce, co = cs[0::2], cs[1::2]
    e = np.full_like(u, ce[-1])
    for k in range(len(ce) - 2, -1, -1):
        e = e * v + ce[k]
    o = np.full_like(u, co[-1])
    for k in range(len(co) - 2, -1, -1):
        o = o * v + co[k]
    got = e + u * o
    assert np.max(np.abs(got / special.erfcx(x) - 1.0)) < 2e-15
    assert len(cs) < 20                      # shorter than the full-range set
