"""CPU FP64 oracle for the MD hot path -- TEST INFRASTRUCTURE ONLY.

Python (ctypes) view of ``liboracle.so`` (built from ``atvb_oracle.c`` by
``oracle/Makefile``).  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this package, and only as the
checker; the product library ``atomiverse_b200`` never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PME_PATH = os.path.join(HERE, "_ref", "libref_pme.so")

THERMO_NONE, THERMO_NH, THERMO_LANGEVIN, THERMO_NPT = 0, 1, 2, 3
NSCALARS = 15
NPT_NSTATE = 13


class OrcNpt(C.Structure):
    _fields_ = [
        ("T_start", C.c_double),
        ("T_stop", C.c_double),
        ("tau_T", C.c_double),
        ("P_target", C.c_double),
        ("tau_P", C.c_double),
        ("drag", C.c_double),
        ("mtchain", C.c_int),
        ("mpchain", C.c_int),
        ("couple", C.c_int * 3),
        ("nfirst", C.c_int64),
        ("nlast", C.c_int64),
    ]


class OrcDesc(C.Structure):
    _fields_ = [
        ("n", C.c_int),
        ("L", C.c_double * 3),
        ("nl_cutoff", C.c_double),
        ("skin", C.c_double),
        ("nl_every", C.c_int),
        ("nl_delay", C.c_int),
        ("nl_check", C.c_int),
        ("has_lj", C.c_int),
        ("lj_eps", C.c_double),
        ("lj_sigma", C.c_double),
        ("lj_rc", C.c_double),
        ("has_coul", C.c_int),
        ("coul_alpha", C.c_double),
        ("coul_rc", C.c_double),
        ("has_pme", C.c_int),
        ("pme_alpha", C.c_double),
        ("pme_K", C.c_int * 3),
        ("pme_order", C.c_int),
        ("dt", C.c_double),
        ("thermostat", C.c_int),
        ("T", C.c_double),
        ("tau", C.c_double),
        ("damp", C.c_double),
        ("seed", C.c_uint32),
        ("need_virial", C.c_int),
        ("T_stop", C.c_double),
        ("lang_nfirst", C.c_int64),
        ("lang_nlast", C.c_int64),
        ("wall_axis", C.c_int),
        ("wall_pos", C.c_double),
        ("wall_k", C.c_double),
    ]


_lib = None


# where the reference source tree sits in the build container (it is absent
# on GPU machines, which use the prebuilt oracle/_ref)
REFERENCE_ROOT = os.environ.get("ATVB_REFERENCE_ROOT", "/root/reference")


def build() -> str:
    """Compile liboracle.so (and the reference PME wrapper when the
    reference tree is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    subprocess.run([os.path.join(HERE, "ref_build.sh"), REFERENCE_ROOT], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int32)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(OrcDesc)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_get_threads.restype = C.c_int
        L.orc_set_state.argtypes = [C.c_void_p] + [dp] * 11 + [C.POINTER(C.c_int64)]
        L.orc_get_state.argtypes = [C.c_void_p] + [dp] * 9
        L.orc_scalars.argtypes = [C.c_void_p, dp]
        L.orc_build_list.restype = C.c_int64
        L.orc_build_list.argtypes = [C.c_void_p]
        L.orc_get_pairs.argtypes = [C.c_void_p, ip, ip]
        L.orc_compute_forces.argtypes = [C.c_void_p]
        L.orc_run.restype = C.c_int
        L.orc_run.argtypes = [C.c_void_p, C.c_int, dp]
        L.orc_bspline.argtypes = [C.c_double, C.c_int, dp, dp]
        L.orc_good_fft_size.restype = C.c_int
        L.orc_good_fft_size.argtypes = [C.c_int]
        L.orc_spline_moduli.argtypes = [C.c_int, C.c_int, dp]
        L.orc_fft3d.argtypes = [C.c_int, C.c_int, C.c_int, dp, C.c_int]
        L.orc_ewald_recip.argtypes = [C.c_int, dp, dp, dp, dp, dp, C.c_double,
                                      C.c_double, dp, dp, dp, dp, dp]
        L.orc_pme.argtypes = [C.c_int, dp, dp, dp, dp, dp, C.c_double,
                              C.POINTER(C.c_int), C.c_int, dp, dp, dp, dp, dp]
        L.orc_gauss3.argtypes = [C.c_uint32, C.c_int64, C.c_int64, dp]
        L.orc_set_lj_types.restype = C.c_int
        L.orc_set_lj_types.argtypes = [C.c_void_p, C.c_int, ip, ip, dp, dp, ip]
        L.orc_set_special.argtypes = [C.c_void_p, C.c_int, ip, ip, dp, dp]
        L.orc_set_npt.restype = C.c_int
        L.orc_set_npt.argtypes = [C.c_void_p, C.POINTER(OrcNpt)]
        L.orc_npt_state.argtypes = [C.c_void_p, dp]
        L.orc_set_barostat.restype = C.c_int
        L.orc_set_barostat.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double]
        L.orc_set_nve_limit.restype = C.c_int
        L.orc_set_nve_limit.argtypes = [C.c_void_p, C.c_double]
        L.orc_set_deform.restype = C.c_int
        L.orc_set_deform.argtypes = [C.c_void_p, C.c_int, C.c_double]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def threads() -> int:
    return lib().orc_get_threads()


def make_desc(n, L, **kw) -> OrcDesc:
    d = OrcDesc()
    d.n = int(n)
    for k in range(3):
        d.L[k] = float(L[k])
    d.nl_cutoff = kw.get("nl_cutoff", 2.5)
    d.skin = kw.get("skin", 0.3)
    d.nl_every = kw.get("nl_every", 1)
    d.nl_delay = kw.get("nl_delay", 0)
    d.nl_check = kw.get("nl_check", 1)
    d.has_lj = int(kw.get("has_lj", 0))
    d.lj_eps = kw.get("lj_eps", 1.0)
    d.lj_sigma = kw.get("lj_sigma", 1.0)
    d.lj_rc = kw.get("lj_rc", d.nl_cutoff)
    d.has_coul = int(kw.get("has_coul", 0))
    d.coul_alpha = kw.get("coul_alpha", 0.0)
    d.coul_rc = kw.get("coul_rc", d.nl_cutoff)
    d.has_pme = int(kw.get("has_pme", 0))
    d.pme_alpha = kw.get("pme_alpha", d.coul_alpha)
    K = kw.get("pme_K", (0, 0, 0))
    for k in range(3):
        d.pme_K[k] = int(K[k])
    d.pme_order = int(kw.get("pme_order", 4))
    d.dt = kw.get("dt", 1.0)
    d.thermostat = int(kw.get("thermostat", THERMO_NONE))
    d.T = kw.get("T", 0.0)
    d.tau = kw.get("tau", 100.0)
    d.damp = kw.get("damp", 100.0)
    d.seed = int(kw.get("seed", 0))
    d.need_virial = int(kw.get("need_virial", 1))
    d.T_stop = kw.get("T_stop", d.T)
    d.lang_nfirst = int(kw.get("lang_nfirst", 0))
    d.lang_nlast = int(kw.get("lang_nlast", 0))
    d.wall_axis = int(kw.get("wall_axis", -1))
    d.wall_pos = kw.get("wall_pos", 0.0)
    d.wall_k = kw.get("wall_k", 0.0)
    return d


class OracleSystem:
    """One system in the CPU oracle (state + half list + scalars)."""

    def __init__(self, desc: OrcDesc):
        self.desc = desc
        self.n = desc.n
        self._h = lib().orc_create(C.byref(desc))

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    __del__ = close

    def set_state(self, x, y, z, vx=None, vy=None, vz=None, fx=None, fy=None,
                  fz=None, mass=None, q=None, tag=None):
        arrs = [_f64(a) for a in (x, y, z, vx, vy, vz, fx, fy, fz, mass, q)]
        self._keep = arrs
        t = None if tag is None else np.ascontiguousarray(tag, dtype=np.int64)
        lib().orc_set_state(self._h, *[_dp(a) for a in arrs],
                            t.ctypes.data_as(C.POINTER(C.c_int64)) if t is not None else None)

    def state(self):
        out = [np.zeros(self.n) for _ in range(9)]
        lib().orc_get_state(self._h, *[_dp(a) for a in out])
        return dict(zip(("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz"), out))

    def scalars(self):
        s = np.zeros(NSCALARS)
        lib().orc_scalars(self._h, _dp(s))
        keys = ("energy", "e_lj", "e_coul", "e_recip", "e_const", "kinetic")
        d = {k: float(s[i]) for i, k in enumerate(keys)}
        d["virial"] = s[6:12].copy()
        d["xi"] = float(s[12])
        d["step"] = int(s[13])
        d["rebuilds"] = int(s[14])
        return d

    def set_lj_types(self, coeffs, types):
        """coeffs: [(type_i, type_j, eps, sigma), ...]; types: per-atom type."""
        ti = np.array([c[0] for c in coeffs], dtype=np.int32)
        tj = np.array([c[1] for c in coeffs], dtype=np.int32)
        e = np.array([c[2] for c in coeffs], dtype=np.float64)
        sg = np.array([c[3] for c in coeffs], dtype=np.float64)
        t = np.ascontiguousarray(types, dtype=np.int32)
        self._keep_t = (ti, tj, e, sg, t)
        ip = C.POINTER(C.c_int32)
        nt = lib().orc_set_lj_types(self._h, len(coeffs), ti.ctypes.data_as(ip),
                                    tj.ctypes.data_as(ip), _dp(e), _dp(sg),
                                    t.ctypes.data_as(ip))
        if nt < 0:
            raise ValueError("bad LJ type coefficient")
        return nt

    def set_special(self, pairs, s_lj, s_coul):
        """pairs: (m, 2) atom indices; s_lj, s_coul: (m,) scales."""
        p = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
        a = np.ascontiguousarray(p[:, 0])
        b = np.ascontiguousarray(p[:, 1])
        sl = np.ascontiguousarray(s_lj, dtype=np.float64)
        sc = np.ascontiguousarray(s_coul, dtype=np.float64)
        self._keep_s = (a, b, sl, sc)
        ip = C.POINTER(C.c_int32)
        lib().orc_set_special(self._h, len(a), a.ctypes.data_as(ip), b.ctypes.data_as(ip),
                              _dp(sl), _dp(sc))

    def set_npt(self, T, tau_T, P, tau_P, drag=0.0, mtchain=3, mpchain=3,
                couple=(True, True, True), T_stop=-1.0, span=(0, 0)):
        """MTK NPT in place of velocity Verlet + thermostat; P in eV/A^3."""
        p = OrcNpt(float(T), float(T_stop), float(tau_T), float(P), float(tau_P),
                   float(drag), int(mtchain), int(mpchain),
                   (C.c_int * 3)(*[int(bool(c)) for c in couple]), int(span[0]),
                   int(span[1]))
        if lib().orc_set_npt(self._h, C.byref(p)) != 0:
            raise ValueError("bad NPT parameters")

    def set_barostat(self, P, tau_P, bulk_modulus=1.0):
        """Berendsen barostat at end_of_step (P in eV/A^3)."""
        if lib().orc_set_barostat(self._h, float(P), float(tau_P), float(bulk_modulus)) != 0:
            raise ValueError("bad barostat parameters")

    def set_nve_limit(self, xmax):
        if lib().orc_set_nve_limit(self._h, float(xmax)) != 0:
            raise ValueError("bad xmax")

    def set_deform(self, axis, rate):
        if lib().orc_set_deform(self._h, int(axis), float(rate)) != 0:
            raise ValueError("bad deform axis")

    def npt_state(self) -> dict:
        o = np.zeros(NPT_NSTATE)
        lib().orc_npt_state(self._h, _dp(o))
        return {"box": o[0:3].copy(), "conserved": float(o[3]), "eps_dot": o[4:7].copy(),
                "eta_t": float(o[7]), "eta_t_dot": float(o[8]), "eta_b": float(o[9]),
                "eta_b_dot": float(o[10]), "T_live": float(o[11]), "KE_global": float(o[12])}

    def build_list(self) -> int:
        return int(lib().orc_build_list(self._h))

    def pairs(self):
        n = self.build_list()
        pi = np.zeros(n, dtype=np.int32)
        pj = np.zeros(n, dtype=np.int32)
        lib().orc_get_pairs(self._h, pi.ctypes.data_as(C.POINTER(C.c_int32)),
                            pj.ctypes.data_as(C.POINTER(C.c_int32)))
        return pi, pj

    def compute_forces(self):
        lib().orc_compute_forces(self._h)

    def run(self, n_steps: int, history: bool = False):
        hist = np.zeros(2 * max(n_steps, 1)) if history else None
        nreb = lib().orc_run(self._h, int(n_steps), _dp(hist))
        if history:
            return nreb, hist.reshape(-1, 2)[:n_steps]
        return nreb


def bspline(frac, n):
    th = np.zeros(n)
    dth = np.zeros(n)
    lib().orc_bspline(float(frac), int(n), _dp(th), _dp(dth))
    return th, dth


def good_fft_size(n):
    return int(lib().orc_good_fft_size(int(n)))


def spline_moduli(K, n):
    out = np.zeros(K)
    lib().orc_spline_moduli(int(K), int(n), _dp(out))
    return out


def fft3d(a: np.ndarray, sign: int) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.complex128).copy()
    K0, K1, K2 = a.shape
    lib().orc_fft3d(K0, K1, K2, a.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)), int(sign))
    return a


def ewald_recip(x, y, z, q, L, alpha, accuracy=1e-8):
    n = len(x)
    arrs = [_f64(a) for a in (x, y, z, q)]
    Lh = np.asarray(L, dtype=np.float64)
    e = np.zeros(1)
    f = [np.zeros(n) for _ in range(3)]
    w = np.zeros(6)
    lib().orc_ewald_recip(n, *[_dp(a) for a in arrs], _dp(Lh), float(alpha), float(accuracy),
                          _dp(e), *[_dp(a) for a in f], _dp(w))
    return float(e[0]), np.stack(f, axis=1), w


def pme(x, y, z, q, L, alpha, K, order):
    n = len(x)
    arrs = [_f64(a) for a in (x, y, z, q)]
    Lh = np.asarray(L, dtype=np.float64)
    Kh = (C.c_int * 3)(*[int(k) for k in K])
    e = np.zeros(1)
    f = [np.zeros(n) for _ in range(3)]
    w = np.zeros(6)
    lib().orc_pme(n, *[_dp(a) for a in arrs], _dp(Lh), float(alpha), Kh, int(order),
                  _dp(e), *[_dp(a) for a in f], _dp(w))
    return float(e[0]), np.stack(f, axis=1), w


def gauss3(seed, step, tag):
    out = np.zeros(3)
    lib().orc_gauss3(int(seed) & 0xFFFFFFFF, int(step), int(tag), _dp(out))
    return out


def ref_pme_lib():
    """The reference's own PME headers compiled by ref_build.sh, or None."""
    if not os.path.exists(REF_PME_PATH):
        return None
    L = C.CDLL(REF_PME_PATH)
    dp = C.POINTER(C.c_double)
    ipp = C.POINTER(C.c_int)
    L.ref_bspline.argtypes = [C.c_double, C.c_int, dp, dp]
    L.ref_good_fft_size.restype = C.c_int
    L.ref_good_fft_size.argtypes = [C.c_int]
    L.ref_spline_moduli.argtypes = [C.c_int, C.c_int, dp]
    L.ref_spread.argtypes = [C.c_int, dp, dp, dp, dp, dp, ipp, C.c_int, dp]
    L.ref_influence.argtypes = [dp, dp, ipp, C.c_int, C.c_double, dp, dp]
    L.ref_interpolate.argtypes = [C.c_int, dp, dp, dp, dp, dp, ipp, C.c_int, dp, dp, dp, dp]
    return L
