"""Generate golden PME vectors from the reference's OWN header-only PME
math (include/atomiverse/cpu/longrange/pme_spline.h, pme_influence.h),
compiled from the reference tree by oracle/ref_build.sh.

The reference leaves the 3D FFT to FFTW (src/cpu/longrange/pme.cpp:203-210:
FFTW_FORWARD then unnormalised FFTW_BACKWARD); numpy's fftn / ifftn*N are
the same transforms.  Run from the repository root:

    oracle/ref_build.sh <reference tree> && python tests/golden/make_golden.py

Writes tests/golden/pme_reference.npz (small: a few KB).
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402


def dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def ref_pme(lib, pos, q, L, alpha, K, order):
    n = len(q)
    x, y, z = [np.ascontiguousarray(pos[:, k]) for k in range(3)]
    Lh = np.asarray(L, dtype=np.float64)
    Kh = np.asarray(K, dtype=np.int32)
    grid = np.zeros(2 * int(np.prod(K)))
    lib.ref_spread(n, dp(x), dp(y), dp(z), dp(q), dp(Lh), ip(Kh), order, dp(grid))
    g = grid.view(np.complex128).reshape(K)
    Q = np.fft.fftn(g)  # FFTW_FORWARD
    Qi = np.ascontiguousarray(Q.reshape(-1)).view(np.float64).copy()
    e = np.zeros(1)
    w = np.zeros(6)
    lib.ref_influence(dp(Qi), dp(Lh), ip(Kh), order, alpha, dp(e), dp(w))
    conv = np.fft.ifftn(Qi.view(np.complex128).reshape(K)) * np.prod(K)  # unnormalised backward
    ci = np.ascontiguousarray(conv.reshape(-1)).view(np.float64).copy()
    f = [np.zeros(n) for _ in range(3)]
    lib.ref_interpolate(n, dp(x), dp(y), dp(z), dp(q), dp(Lh), ip(Kh), order, dp(ci),
                        dp(f[0]), dp(f[1]), dp(f[2]))
    vol = float(np.prod(L))
    qq = float((q * q).sum())
    qt = float(q.sum())
    e_self = -14.399645 * alpha / np.sqrt(np.pi) * qq
    e_net = -14.399645 * np.pi / (2 * vol * alpha * alpha) * qt * qt
    return e[0] + e_self + e_net, np.stack(f, 1), w, grid


def main():
    lib = oracle.ref_pme_lib()
    if lib is None:
        raise SystemExit("build oracle/_ref first: oracle/ref_build.sh <reference tree>")
    out = {}
    # bspline / moduli / FFT sizes (pme_spline.h)
    for n in (4, 5, 6, 8):
        th = np.zeros((5, n))
        dth = np.zeros((5, n))
        for k, fr in enumerate((0.0, 0.1, 0.33, 0.5, 0.999)):
            a, b = np.zeros(n), np.zeros(n)
            lib.ref_bspline(fr, n, dp(a), dp(b))
            th[k], dth[k] = a, b
        out[f"bspline_{n}_theta"] = th
        out[f"bspline_{n}_dtheta"] = dth
    for K, n in ((12, 4), (24, 6), (30, 4), (49, 5)):
        m = np.zeros(K)
        lib.ref_spline_moduli(K, n, dp(m))
        out[f"moduli_{K}_{n}"] = m
    out["good_fft_size"] = np.array([[k, lib.ref_good_fft_size(k)] for k in
                                     (1, 11, 13, 15, 16, 23, 49, 97, 181, 193)])
    # the FD fixture of tests/cpu/longrange/test_pme_coul.cpp:194-244
    pos = np.array([[1.0, 1.0, 1.0], [3.2, 1.4, 1.1], [1.3, 3.1, 2.4], [2.7, 2.2, 3.6]])
    q = np.array([0.6, -0.4, 0.5, -0.7])
    e, f, w, grid = ref_pme(lib, pos, q, (8.0, 8.0, 8.0), 0.45, (12, 12, 12), 6)
    out.update(fd_pos=pos, fd_q=q, fd_energy=np.array([e]), fd_force=f, fd_virial=w)
    # a jittered, non-cubic 54-ion salt at order 4
    rng = np.random.default_rng(5)
    g = np.arange(3)
    ijk = np.stack(np.meshgrid(g, g, np.arange(6), indexing="ij"), -1).reshape(-1, 3)
    L = (8.46, 8.46, 16.92)
    pos = np.mod(ijk * 2.82 + rng.uniform(-0.3, 0.3, ijk.shape), L)
    q = np.where(ijk.sum(1) % 2 == 0, 1.0, -1.0)
    e, f, w, grid = ref_pme(lib, pos, q, L, 0.55, (10, 10, 18), 4)
    out.update(salt_pos=pos, salt_q=q, salt_L=np.array(L), salt_energy=np.array([e]),
               salt_force=f, salt_virial=w)
    np.savez_compressed(os.path.join(HERE, "pme_reference.npz"), **out)
    print("wrote", os.path.join(HERE, "pme_reference.npz"))


if __name__ == "__main__":
    main()
