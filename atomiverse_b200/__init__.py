"""atomiverse_b200 -- B200-native classical-MD hot path behind a C ABI.

The compute path is libatvb.so (hand-written CUDA for sm_100a, see csrc/);
this module is a thin ctypes view of its C ABI (include/atvb.h) plus the
reference-shaped component API (NeighborList, PairLJCut, CoulLong,
KSpacePME, VelocityVerlet, NoseHoover, FixLangevin, MD) that assembles a
system description.  There is no CPU fallback: every call goes to the GPU
library, and importing the package fails loudly if the library is missing.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import (FP64, LANGEVIN, MIXED, NOSE_HOOVER, NVE, AtvbError, PhysicsError,
                   Scalars, SoaView, SystemDesc, check, check_status, load)

__all__ = [
    "FP64", "MIXED", "NVE", "NOSE_HOOVER", "LANGEVIN", "AtvbError", "PhysicsError",
    "Context", "System", "Batch", "Server", "make_desc",
    "NeighborList", "PairLJCut", "CoulLong", "KSpacePME", "VelocityVerlet",
    "NoseHoover", "FixLangevin", "NoseHooverNPT", "Barostat", "NVELimit", "Deform", "MD",
    "StopOnNaN",
    "library_path",
]

FRAME_KEYS = ("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz", "mass", "charge")
KB_EV_PER_K = 8.617333262e-5   # units.h:138
HISTORY_DEFAULT = 4096         # per-step energy ring of a system (history_capacity 0)


def library_path() -> str:
    return _abi.LIB_PATH


def make_desc(n_atoms, box, **kw) -> SystemDesc:
    """Flat system record; keywords are the atvb_system_desc field names."""
    d = SystemDesc()
    d.n_atoms = int(n_atoms)
    b = list(box)
    if len(b) == 3:
        b = [b[0], 0, 0, 0, b[1], 0, 0, 0, b[2]]
    for k in range(9):
        d.box[k] = float(b[k])
    d.nl_skin = -1.0
    d.nl_every = 1
    d.nl_delay = 0
    d.nl_check = 1
    d.pme_order = 4
    d.dt = 1.0
    for k, v in kw.items():
        if k == "pme_grid":
            for i in range(3):
                d.pme_grid[i] = int(v[i])
        elif k == "box":
            continue
        else:
            if not hasattr(d, k):
                raise TypeError(f"unknown system field {k!r}")
            setattr(d, k, v)
    return d


def _soa(frame: dict, n: int, writable: bool = False) -> tuple[SoaView, list]:
    """SoaView over numpy arrays in `frame` (float64, contiguous)."""
    v = SoaView()
    keep = []
    for k in FRAME_KEYS:
        a = frame.get(k)
        if a is None:
            continue
        if writable:
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
                raise TypeError(f"frame[{k!r}] must be a contiguous float64 array")
        else:
            a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape[0] != n:
            raise ValueError(f"frame[{k!r}] has {a.shape[0]} rows, expected {n}")
        keep.append(a)
        setattr(v, k, a.ctypes.data_as(C.POINTER(C.c_double)))
    t = frame.get("tag")
    if t is not None:
        t = np.ascontiguousarray(t, dtype=np.int64)
        keep.append(t)
        v.tag = t.ctypes.data_as(C.POINTER(C.c_int64))
    ty = frame.get("type")
    if ty is not None and not writable:
        ty = np.ascontiguousarray(ty, dtype=np.int32)
        keep.append(ty)
        v.type = ty.ctypes.data_as(C.POINTER(C.c_int32))
    return v, keep


def _lj_type_args(coeffs):
    """ctypes arguments for (type_i, type_j, epsilon, sigma) coefficients."""
    ti = np.array([c[0] for c in coeffs], dtype=np.int32)
    tj = np.array([c[1] for c in coeffs], dtype=np.int32)
    e = np.array([c[2] for c in coeffs], dtype=np.float64)
    sg = np.array([c[3] for c in coeffs], dtype=np.float64)
    ip, dp = C.POINTER(C.c_int32), C.POINTER(C.c_double)
    return (len(coeffs), ti.ctypes.data_as(ip), tj.ctypes.data_as(ip),
            e.ctypes.data_as(dp), sg.ctypes.data_as(dp)), (ti, tj, e, sg)


def _special_args(special):
    """ctypes arguments for dict(lj=(s12, s13, s14), coul=(...), bonds=[(tag_a, tag_b)])."""
    lj = (C.c_double * 3)(*[float(x) for x in special.get("lj", (1.0, 1.0, 1.0))])
    co = (C.c_double * 3)(*[float(x) for x in special.get("coul", (1.0, 1.0, 1.0))])
    b = np.asarray(special.get("bonds", []), dtype=np.int64).reshape(-1, 2)
    a0 = np.ascontiguousarray(b[:, 0])
    a1 = np.ascontiguousarray(b[:, 1])
    lp = C.POINTER(C.c_int64)
    return (lj, co, len(a0), a0.ctypes.data_as(lp), a1.ctypes.data_as(lp)), (lj, co, a0, a1)


def scalars_dict(s: Scalars) -> dict:
    return {
        "energy": s.energy, "energy_pair": s.energy_pair, "energy_lj": s.energy_lj,
        "energy_coul": s.energy_coul, "energy_recip": s.energy_recip,
        "energy_const": s.energy_const, "kinetic": s.kinetic, "conserved": s.conserved,
        "stress": np.array(list(s.stress)), "nh_xi": s.nh_xi, "step": s.step,
        "rebuilds": s.rebuilds, "max_neighbors": s.max_neighbors, "status": s.status,
        "status_bits": s.status_bits, "halted": bool(s.halted),
        "list_pairs": s.list_pairs, "box": np.array(list(s.box)), "pressure": s.pressure,
    }


def _baro_args(b) -> tuple:
    """Barostat (or a dict of its fields) -> (P_target, tau_P, bulk_modulus)."""
    if isinstance(b, dict):
        b = Barostat(**b)
    return float(b.P_target), float(b.tau_P), float(b.bulk_modulus)


def _npt_desc(npt) -> "_abi.NptDesc":
    """NoseHooverNPT (or a dict of its fields) -> atvb_npt_desc."""
    if isinstance(npt, dict):
        npt = NoseHooverNPT(**npt)
    d = _abi.NptDesc()
    d.T_start = float(npt.T_target)
    d.T_stop = float(npt.T_stop)
    d.tau_T = float(npt.tau_T)
    d.P_target = float(npt.P_target)
    d.tau_P = float(npt.tau_P)
    d.drag = float(npt.drag)
    d.mtchain = int(npt.mtchain)
    d.mpchain = int(npt.mpchain)
    for a in range(3):
        d.couple[a] = 1 if npt.couple_axis[a] else 0
    d.nfirst = int(npt.nfirst)
    d.nlast = int(npt.nlast)
    return d


class Context:
    """One CUDA device (cuda::Context)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        opts = _abi.DeviceOpts()
        opts.device = device
        h = C.c_void_p()
        check(self.lib.atvb_ctx_create(C.byref(opts), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self.lib.atvb_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class System:
    """One MD system on the device (cuda::md::MD + its components)."""

    def __init__(self, ctx: Context, desc: SystemDesc | dict, frame: dict | None = None,
                 lj_types=None, special_bonds=None, npt=None, barostat=None,
                 nve_limit=None, deform=None):
        """lj_types: [(type_i, type_j, epsilon, sigma), ...] (PairLJCut's
        per-type form; per-atom types in frame["type"]); special_bonds:
        dict(lj=(s12, s13, s14), coul=(s12, s13, s14), bonds=[(tag_a, tag_b), ...]);
        npt: a NoseHooverNPT (MTK NPT in place of velocity Verlet, desc NVE);
        barostat: a Barostat (Berendsen, beside the thermostat); nve_limit:
        xmax [A] (NVELimit); deform: (axis, strain_rate) (Deform).
        All are applied before the frame is uploaded."""
        self.ctx = ctx
        self.lib = ctx.lib
        if isinstance(desc, dict):
            desc = make_desc(**desc)
        self.desc = desc
        self.n = desc.n_atoms
        h = C.c_void_p()
        check(self.lib.atvb_system_create(ctx._h, C.byref(desc), C.byref(h)))
        self._h = h
        if lj_types is not None:
            args, keep = _lj_type_args(lj_types)
            check(self.lib.atvb_system_set_lj_types(self._h, *args))
        if special_bonds is not None:
            args, keep = _special_args(special_bonds)
            check(self.lib.atvb_system_set_special_bonds(self._h, *args))
        if npt is not None:
            check(self.lib.atvb_system_set_npt(self._h, C.byref(_npt_desc(npt))))
        if barostat is not None:
            check(self.lib.atvb_system_set_barostat(self._h, *_baro_args(barostat)))
        if nve_limit is not None:
            check(self.lib.atvb_system_set_nve_limit(self._h, float(nve_limit)))
        if deform is not None:
            check(self.lib.atvb_system_set_deform(self._h, int(deform[0]), float(deform[1])))
        if frame is not None:
            self.upload(frame)

    def close(self):
        if getattr(self, "_h", None):
            self.lib.atvb_system_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def upload(self, frame: dict):
        v, keep = _soa(frame, self.n)
        check(self.lib.atvb_system_upload(self._h, C.byref(v)))
        del keep

    def compute_forces(self):
        check(self.lib.atvb_system_compute_forces(self._h))

    def set_snapshots(self, every: int, depth: int = 8):
        """Publish positions/velocities every `every` steps into a host ring."""
        check(self.lib.atvb_system_set_snapshots(self._h, int(every), int(depth)))

    def poll_snapshots(self, max_frames: int = 64) -> tuple[list, int]:
        """Frames published since the last poll (no device sync):
        [(step, box, {x, y, z, vx, vy, vz})], dropped."""
        n, m = self.n, int(max_frames)
        arrs = [np.zeros(m * n) for _ in range(6)]
        steps = np.zeros(m, dtype=np.int64)
        box = np.zeros(3 * m)
        cnt, drop = C.c_int32(), C.c_int64()
        dp = C.POINTER(C.c_double)
        check(self.lib.atvb_system_snapshot_poll(
            self._h, m, steps.ctypes.data_as(C.POINTER(C.c_int64)), box.ctypes.data_as(dp),
            *[a.ctypes.data_as(dp) for a in arrs], C.byref(cnt), C.byref(drop)))
        keys = ("x", "y", "z", "vx", "vy", "vz")
        frames = [(int(steps[f]), box[3 * f:3 * f + 3].copy(),
                   {k: arrs[j][f * n:(f + 1) * n].copy() for j, k in enumerate(keys)})
                  for f in range(cnt.value)]
        return frames, int(drop.value)

    def save(self) -> bytes:
        """Checkpoint: the whole resumable state as bytes."""
        nb = C.c_int64()
        check(self.lib.atvb_system_checkpoint_size(self._h, C.byref(nb)))
        buf = C.create_string_buffer(nb.value)
        check(self.lib.atvb_system_save(self._h, buf, nb.value))
        return buf.raw

    def restore(self, blob: bytes):
        """Resume from save()'s bytes, in place of the first upload."""
        check(self.lib.atvb_system_restore(self._h, blob, len(blob)))

    def step(self, n: int):
        check(self.lib.atvb_system_step(self._h, int(n)))

    def step_timed(self, n: int) -> tuple[float, np.ndarray]:
        """n steps timed with CUDA events on the system's stream: (total
        ms, per-step ms)."""
        per = np.zeros(int(n))
        tot = C.c_double()
        check(self.lib.atvb_system_step_timed(
            self._h, int(n), per.ctypes.data_as(C.POINTER(C.c_double)), C.byref(tot)))
        return tot.value, per

    def download(self, keys=FRAME_KEYS, check: bool = True) -> tuple[dict, dict]:
        """Frame and scalars.  A sticky status bit (wrong or non-finite
        physics in some step) raises PhysicsError unless check=False; its
        `result` carries the (frame, scalars) anyway."""
        out = {k: np.zeros(self.n) for k in keys}
        v, keep = _soa(out, self.n, writable=True)
        s = Scalars()
        rc = self.lib.atvb_system_download(self._h, C.byref(v), C.byref(s))
        return check_status(rc, (out, scalars_dict(s)), check)

    def scalars(self, check: bool = True) -> dict:
        """SystemScalars; raises PhysicsError on a sticky status bit unless
        check=False (the dict's status_bits then tells which)."""
        s = Scalars()
        rc = self.lib.atvb_system_scalars(self._h, C.byref(s))
        return check_status(rc, scalars_dict(s), check)

    def clear_status(self):
        """Reset the sticky status bits (and a StopOnNaN halt)."""
        _abi.check(self.lib.atvb_system_clear_status(self._h))

    def set_stop_on_nan(self, on: bool = True):
        """cuda::StopOnNaN: stop integrating at a non-finite state."""
        _abi.check(self.lib.atvb_system_set_stop_on_nan(self._h, 1 if on else 0))

    def set_langevin_ramp(self, T_stop: float, nfirst: int, nlast: int):
        """FixLangevin's setpoint ramp (fix_langevin.cpp:94-104): from the
        descriptor's temperature to T_stop over steps [nfirst, nlast]."""
        _abi.check(self.lib.atvb_system_set_langevin_ramp(self._h, float(T_stop), int(nfirst),
                                                          int(nlast)))

    def set_capacity(self, row_capacity: int = 0, nearq_capacity: int = 0):
        """Pin the neighbour row length / size the near-cutoff queue (0: auto)."""
        _abi.check(self.lib.atvb_system_set_capacity(self._h, int(row_capacity),
                                                     int(nearq_capacity)))

    def run(self, frame: dict, n_steps: int, check: bool = True) -> dict:
        """MD::run(frame, n): upload on first use, step, download into frame."""
        for k in FRAME_KEYS:
            if k not in frame:
                frame[k] = np.zeros(self.n)
            frame[k] = np.ascontiguousarray(frame[k], dtype=np.float64)
        v, keep = _soa(frame, self.n, writable=True)
        s = Scalars()
        rc = self.lib.atvb_system_run(self._h, C.byref(v), int(n_steps), C.byref(s))
        return check_status(rc, scalars_dict(s), check)

    def history(self, max_steps: int = 4096) -> np.ndarray:
        buf = np.zeros(3 * max_steps)
        cnt = C.c_int32()
        check(self.lib.atvb_system_energy_history(
            self._h, buf.ctypes.data_as(C.POINTER(C.c_double)), int(max_steps), C.byref(cnt)))
        return buf[: 3 * cnt.value].reshape(-1, 3)

    def pairs(self) -> tuple[np.ndarray, np.ndarray]:
        cnt = C.c_int64()
        check(self.lib.atvb_system_pairs(self._h, None, None, 0, C.byref(cnt)))
        pi = np.zeros(cnt.value, dtype=np.int32)
        pj = np.zeros(cnt.value, dtype=np.int32)
        check(self.lib.atvb_system_pairs(
            self._h, pi.ctypes.data_as(C.POINTER(C.c_int32)),
            pj.ctypes.data_as(C.POINTER(C.c_int32)), cnt.value, C.byref(cnt)))
        return pi, pj

    def set_pair_lanes(self, lanes: int):
        check(self.lib.atvb_system_set_pair_lanes(self._h, int(lanes)))

    def profile(self, enable: bool):
        check(self.lib.atvb_system_profile(self._h, 1 if enable else 0))

    def profile_read(self) -> dict:
        buf = (_abi.KernelTime * 64)()
        cnt = C.c_int32()
        check(self.lib.atvb_system_profile_read(self._h, buf, 64, C.byref(cnt)))
        return {buf[k].name.decode(): (buf[k].total_ms, buf[k].launches) for k in range(cnt.value)}

    def launch_count(self) -> int:
        n = C.c_int64()
        check(self.lib.atvb_system_launch_count(self._h, C.byref(n)))
        return n.value

    def stream(self) -> int:
        return self.lib.atvb_system_stream(self._h) or 0


class Batch:
    """Many independent systems advanced by one launch per kernel."""

    def __init__(self, ctx: Context, items: list):
        """items: (desc, frame) or (desc, frame, options) with options the
        System keywords lj_types / special_bonds / npt."""
        self.ctx = ctx
        self.lib = ctx.lib
        descs = [make_desc(**it[0]) if isinstance(it[0], dict) else it[0] for it in items]
        arr = (SystemDesc * len(descs))(*descs)
        self.sizes = [d.n_atoms for d in descs]
        h = C.c_void_p()
        check(self.lib.atvb_batch_create(ctx._h, arr, len(descs), C.byref(h)))
        self._h = h
        for k, it in enumerate(items):
            opts = it[2] if len(it) > 2 and it[2] else {}
            if opts.get("lj_types") is not None:
                args, keep = _lj_type_args(opts["lj_types"])
                check(self.lib.atvb_batch_set_lj_types(self._h, k, *args))
            if opts.get("special_bonds") is not None:
                args, keep = _special_args(opts["special_bonds"])
                check(self.lib.atvb_batch_set_special_bonds(self._h, k, *args))
            if opts.get("npt") is not None:
                check(self.lib.atvb_batch_set_npt(self._h, k, C.byref(_npt_desc(opts["npt"]))))
            if opts.get("barostat") is not None:
                check(self.lib.atvb_batch_set_barostat(self._h, k, *_baro_args(opts["barostat"])))
            if opts.get("nve_limit") is not None:
                check(self.lib.atvb_batch_set_nve_limit(self._h, k, float(opts["nve_limit"])))
            if opts.get("deform") is not None:
                a, r = opts["deform"]
                check(self.lib.atvb_batch_set_deform(self._h, k, int(a), float(r)))
        for k, it in enumerate(items):
            if it[1] is not None:
                self.upload(k, it[1])

    def close(self):
        if getattr(self, "_h", None):
            self.lib.atvb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def upload(self, k: int, frame: dict):
        v, keep = _soa(frame, self.sizes[k])
        check(self.lib.atvb_batch_upload(self._h, int(k), C.byref(v)))

    def compute_forces(self):
        check(self.lib.atvb_batch_compute_forces(self._h))

    def save(self, k: int) -> bytes:
        nb = C.c_int64()
        check(self.lib.atvb_batch_checkpoint_size(self._h, int(k), C.byref(nb)))
        buf = C.create_string_buffer(nb.value)
        check(self.lib.atvb_batch_save(self._h, int(k), buf, nb.value))
        return buf.raw

    def restore(self, k: int, blob: bytes):
        check(self.lib.atvb_batch_restore(self._h, int(k), blob, len(blob)))

    def step(self, n: int):
        check(self.lib.atvb_batch_step(self._h, int(n)))

    def download(self, k: int, keys=FRAME_KEYS, check: bool = True) -> tuple[dict, dict]:
        out = {key: np.zeros(self.sizes[k]) for key in keys}
        v, keep = _soa(out, self.sizes[k], writable=True)
        s = Scalars()
        rc = self.lib.atvb_batch_download(self._h, int(k), C.byref(v), C.byref(s))
        return check_status(rc, (out, scalars_dict(s)), check)

    def clear_status(self, k: int):
        _abi.check(self.lib.atvb_batch_clear_status(self._h, int(k)))

    def set_stop_on_nan(self, k: int, on: bool = True):
        _abi.check(self.lib.atvb_batch_set_stop_on_nan(self._h, int(k), 1 if on else 0))

    def set_langevin_ramp(self, k: int, T_stop: float, nfirst: int, nlast: int):
        _abi.check(self.lib.atvb_batch_set_langevin_ramp(self._h, int(k), float(T_stop),
                                                         int(nfirst), int(nlast)))

    def autotune(self) -> int:
        g = C.c_int32()
        check(self.lib.atvb_batch_autotune(self._h, C.byref(g)))
        return g.value

    def launch_count(self) -> int:
        n = C.c_int64()
        check(self.lib.atvb_batch_launch_count(self._h, C.byref(n)))
        return n.value

    def profile(self, enable: bool):
        check(self.lib.atvb_batch_profile(self._h, int(bool(enable))))

    def profile_read(self) -> dict:
        buf = (_abi.KernelTime * 64)()
        cnt = C.c_int32()
        check(self.lib.atvb_batch_profile_read(self._h, buf, 64, C.byref(cnt)))
        return {buf[k].name.decode(): (buf[k].total_ms, buf[k].launches) for k in range(cnt.value)}


class Server:
    """Continuous batching of MD segments under a device-memory budget."""

    def __init__(self, ctx: Context, budget_bytes: int, max_active: int = 0):
        self.ctx = ctx
        self.lib = ctx.lib
        h = C.c_void_p()
        check(self.lib.atvb_server_create(ctx._h, int(budget_bytes), int(max_active), C.byref(h)))
        self._h = h
        self.sizes = {}

    def close(self):
        if getattr(self, "_h", None):
            self.lib.atvb_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def submit(self, desc, frame: dict, n_steps: int) -> int:
        if isinstance(desc, dict):
            desc = make_desc(**desc)
        v, keep = _soa(frame, desc.n_atoms)
        rid = C.c_int64()
        check(self.lib.atvb_server_submit(self._h, C.byref(desc), C.byref(v), int(n_steps),
                                          C.byref(rid)))
        self.sizes[rid.value] = desc.n_atoms
        return rid.value

    def cancel(self, rid: int):
        check(self.lib.atvb_server_cancel(self._h, int(rid)))

    def set_limits(self, max_resident_atoms: int = 0):
        check(self.lib.atvb_server_set_limits(self._h, int(max_resident_atoms)))

    def tick(self, chunk: int = 50):
        check(self.lib.atvb_server_tick(self._h, int(chunk)))

    def poll(self, rid: int) -> dict:
        r = _abi.RequestResult()
        check(self.lib.atvb_server_poll(self._h, int(rid), C.byref(r)))
        return {"id": r.id, "state": r.state, "steps_done": r.steps_done,
                "t_submit": r.t_submit, "t_start": r.t_start, "t_done": r.t_done,
                "scalars": scalars_dict(r.scalars)}

    def collect(self, rid: int) -> tuple[dict, dict]:
        n = self.sizes[rid]
        out = {k: np.zeros(n) for k in FRAME_KEYS[:9]}
        v, keep = _soa(out, n, writable=True)
        r = _abi.RequestResult()
        check(self.lib.atvb_server_collect(self._h, int(rid), C.byref(v), C.byref(r)))
        res = {"id": r.id, "state": r.state, "steps_done": r.steps_done,
               "t_submit": r.t_submit, "t_start": r.t_start, "t_done": r.t_done,
               "scalars": scalars_dict(r.scalars)}
        return out, res

    def keep_checkpoints(self, on: bool = True):
        check(self.lib.atvb_server_keep_checkpoints(self._h, int(bool(on))))

    def suspend(self, rid: int):
        check(self.lib.atvb_server_suspend(self._h, int(rid)))

    def resume(self, rid: int, more_steps: int):
        check(self.lib.atvb_server_resume(self._h, int(rid), int(more_steps)))

    def checkpoint(self, rid: int) -> bytes:
        nb = C.c_int64()
        check(self.lib.atvb_server_checkpoint(self._h, int(rid), None, 0, C.byref(nb)))
        buf = C.create_string_buffer(nb.value)
        check(self.lib.atvb_server_checkpoint(self._h, int(rid), buf, nb.value, C.byref(nb)))
        return buf.raw

    def submit_checkpoint(self, desc, blob: bytes, n_steps: int) -> int:
        if isinstance(desc, dict):
            desc = make_desc(**desc)
        rid = C.c_int64()
        check(self.lib.atvb_server_submit_checkpoint(self._h, C.byref(desc), blob, len(blob),
                                                     int(n_steps), C.byref(rid)))
        self.sizes[rid.value] = desc.n_atoms
        return rid.value

    def stats(self) -> dict:
        q, r, d = C.c_int64(), C.c_int64(), C.c_int64()
        b = C.c_size_t()
        check(self.lib.atvb_server_stats(self._h, C.byref(q), C.byref(r), C.byref(d), C.byref(b)))
        return {"queued": q.value, "running": r.value, "done": d.value, "bytes": b.value}


def request_bytes(desc) -> int:
    if isinstance(desc, dict):
        desc = make_desc(**desc)
    b = C.c_size_t()
    check(load().atvb_request_bytes(C.byref(desc), C.byref(b)))
    return b.value


# ---------------------------------------------------------------------------
# Reference-shaped component API (cuda::NeighborList, cuda::PairLJCut, ...).
# Each component only records its constructor arguments; MD.build() folds
# them into one system description for the fused device step.
# ---------------------------------------------------------------------------

@dataclass
class NeighborList:
    """NeighborList(cutoff, skin=-1 -> 0.3*cutoff, every, delay, check)
    (neighbor_list.cuh:98; cpu/neighbor/neighbor_list.h:79)."""
    cutoff: float
    skin: float = -1.0
    every: int = 1
    delay: int = 0
    check: bool = True


@dataclass
class PairLJCut:
    """PairLJCut(epsilon, sigma, cutoff) (pair_lj_cut.cuh:25)."""
    epsilon: float
    sigma: float
    cutoff: float


@dataclass
class CoulLong:
    """CoulLong(alpha, cutoff) (coul_long.cuh:24)."""
    alpha: float
    cutoff: float


@dataclass
class KSpacePME:
    """KSpacePME(alpha, grid_spacing=1.0, order=6) (pme.cuh:26); `grid`
    fixes the mesh instead of the spacing rule."""
    alpha: float
    grid_spacing: float = 1.0
    order: int = 6
    grid: tuple | None = None


@dataclass
class VelocityVerlet:
    dt: float


@dataclass
class NoseHoover:
    """NoseHoover(T, tau, dt) (nose_hoover.cu:29)."""
    T: float
    tau: float
    dt: float


@dataclass
class FixLangevin:
    """FixLangevin(T_start, T_stop, damp, dt, seed) + set_run_span(nfirst,
    nlast) (fix_langevin.h; cuda/dynamics/fix_langevin.cuh:69-80): the
    setpoint ramps linearly from T_start to T_stop over the span (T_stop < 0:
    constant)."""
    T_start: float
    T_stop: float
    damp: float
    dt: float
    seed: int = 0
    nfirst: int = 0
    nlast: int = 0

    def set_run_span(self, nfirst: int, nlast: int):
        self.nfirst, self.nlast = int(nfirst), int(nlast)
        return self


@dataclass
class NoseHooverNPT:
    """NoseHooverNPT(T_target, tau_T, P_target, tau_P, dt, drag=0, mtchain=3,
    mpchain=3, couple_axis=(True, True, True), T_stop=-1) + set_run_span
    (cuda/dynamics/nose_hoover_npt.cuh:60-70): MTK NPT, P_target in eV/A^3.
    An integrator: it replaces VelocityVerlet and the thermostat."""
    T_target: float
    tau_T: float
    P_target: float
    tau_P: float
    dt: float
    drag: float = 0.0
    mtchain: int = 3
    mpchain: int = 3
    couple_axis: tuple = (True, True, True)
    T_stop: float = -1.0
    nfirst: int = 0
    nlast: int = 0

    def set_run_span(self, nfirst: int, nlast: int):
        self.nfirst, self.nlast = int(nfirst), int(nlast)
        return self


@dataclass
class NVELimit:
    """NVELimit(dt, xmax) (cuda/dynamics/nve_limit.cuh): velocity Verlet with
    each half kick's speed capped at xmax / dt.  An integrator."""
    dt: float
    xmax: float


@dataclass
class Deform:
    """Deform(axis, strain_rate, dt) (cuda/dynamics/deform.cuh): constant
    engineering strain along one axis; bound with set_thermostat."""
    axis: int
    strain_rate: float
    dt: float


@dataclass
class Barostat:
    """Barostat(P_target, tau_P, dt, bulk_modulus=1.0) (Berendsen,
    cpu/dynamics/barostat.h:86): end-of-step pressure coupling beside the
    thermostat; P_target and bulk_modulus in eV/A^3."""
    P_target: float
    tau_P: float
    dt: float
    bulk_modulus: float = 1.0


@dataclass
class StopOnNaN:
    """cuda::StopOnNaN (include/atomiverse/cuda/driver/criterion.cuh:166-178):
    abandon the run once the state is no longer finite.  Attached with
    MD.add_criterion; the device halts the system at the step where a
    position or velocity turned non-finite and run() raises PhysicsError."""
    name: str = "stop_on_nan"


@dataclass
class MD:
    """cuda::md::MD: categorical setters, build(), run(frame, n)
    (include/atomiverse/cuda/dynamics/md.cuh:118-385)."""
    ctx: Context | None = None
    precision: int = FP64
    _neighbor: NeighborList | None = None
    _evaluators: list = field(default_factory=list)
    _integrator: VelocityVerlet | None = None
    _thermostats: list = field(default_factory=list)
    _stress: bool = False
    _system: System | None = None
    _thermo: tuple | None = None          # (every, file or None, header printed)
    _criteria: list = field(default_factory=list)

    def add_criterion(self, c):
        """Driver::add_criterion (driver.cuh:151); StopOnNaN is the one the
        device path evaluates."""
        if not isinstance(c, StopOnNaN):
            raise TypeError(f"unsupported criterion {type(c).__name__}")
        self._criteria.append(c)
        if self._system is not None:
            self._system.set_stop_on_nan(True)
        return self

    def set_neighbor(self, nl: NeighborList):
        self._neighbor = nl
        return self

    def set_evaluator(self, ev):
        self._evaluators.append(ev)
        return self

    def set_integrator(self, integ):
        if self._integrator is not None and self._integrator != integ:
            raise ValueError("set_integrator already configured")
        self._integrator = integ
        return self

    def set_thermostat(self, th):
        """Plural (md.cuh:229-233): Nose-Hoover / Langevin, or any component
        bound at its default slot (Deform, Barostat)."""
        self._thermostats.append(th)
        return self

    def set_barostat(self, b: "Barostat"):
        """LAMMPS `fix press/berendsen` (md.cuh:239-243)."""
        return self.set_thermostat(b)

    def set_thermo(self, every: int, filename: str | None = None):
        """Thermo output every `every` steps (md.cuh:249-262, cuda::Thermo in
        record/thermo.cuh): Step, Temp (2 KE / (Ndof k_B), Ndof = 3N - 3),
        PotEng, KinEng, TotEng in the columns of cpu::thermo_print
        (record/thermo.cpp:56-81), read from the device's per-step energy
        ring after each run.  Step is the driver's zero-based iteration
        index, continued across run() calls (md.cuh:170); a row is printed
        where it is a multiple of `every` (driver.cu:128).  Singular: a
        different cadence throws."""
        every = int(every) if int(every) > 0 else 1      # 0 is every step
        if self._thermo is not None:
            if self._thermo[0] == every:
                return self
            raise ValueError(f"set_thermo already configured with {self._thermo[0]}, "
                             f"rejected re-call with {every}")
        fh = None
        if filename:
            fh = open(filename, "w")
            fh.write("# Step Temp PotEng KinEng TotEng\n")
        self._thermo = [every, fh, False]
        return self

    def _thermo_rows(self, hist: np.ndarray, n_atoms: int):
        every, fh, header = self._thermo
        ndof = 3 * n_atoms - 3
        for pe, ke, step in hist:
            step = int(step)
            if step % every:
                continue
            temp = 2.0 * ke / (ndof * KB_EV_PER_K) if ndof > 0 else 0.0
            if not header:
                print(f"{'Step':>8s} {'Temp':>12s} {'PotEng':>14s} {'KinEng':>14s} {'TotEng':>14s}")
                header = self._thermo[2] = True
            print(f"{step:8d} {temp:12.4f} {pe:14.6f} {ke:14.6f} {pe + ke:14.6f}")
            if fh is not None:
                fh.write(f"{step} {temp:.6f} {pe:.6f} {ke:.6f} {pe + ke:.6f}\n")
        if fh is not None:
            fh.flush()

    def set_stress_required(self, on: bool = True):
        self._stress = on
        return self

    def desc(self, n_atoms: int, box) -> SystemDesc:
        if self._integrator is None:
            raise ValueError("MD needs an integrator (set_integrator)")
        if self._neighbor is None and self._evaluators:
            raise ValueError("a pair evaluator needs a NeighborList: "
                             "add sim.set_neighbor(NeighborList(cutoff))")
        kw = dict(precision=self.precision, dt=self._integrator.dt,
                  stress_required=int(self._stress))
        nl = self._neighbor
        kw.update(nl_cutoff=nl.cutoff, nl_skin=nl.skin, nl_every=nl.every,
                  nl_delay=nl.delay, nl_check=int(nl.check))
        for ev in self._evaluators:
            if isinstance(ev, PairLJCut):
                kw.update(lj_enabled=1, lj_epsilon=ev.epsilon, lj_sigma=ev.sigma,
                          lj_cutoff=ev.cutoff)
            elif isinstance(ev, CoulLong):
                kw.update(coul_enabled=1, coul_alpha=ev.alpha, coul_cutoff=ev.cutoff)
            elif isinstance(ev, KSpacePME):
                kw.update(pme_enabled=1, pme_alpha=ev.alpha,
                          pme_grid_spacing=ev.grid_spacing, pme_order=ev.order)
                if ev.grid is not None:
                    kw["pme_grid"] = tuple(ev.grid)
            else:
                raise TypeError(f"unsupported evaluator {type(ev).__name__}")
        for th in self._thermostats:
            if isinstance(th, (Barostat, Deform)):
                continue              # applied after create (System barostat= / deform=)
            if isinstance(th, NoseHoover):
                kw.update(thermostat=NOSE_HOOVER, temperature=th.T, tau=th.tau)
            elif isinstance(th, FixLangevin):
                kw.update(thermostat=LANGEVIN, temperature=th.T_start, damp=th.damp,
                          seed=th.seed)
            else:
                raise TypeError(f"unsupported thermostat {type(th).__name__}")
        return make_desc(n_atoms, box, **kw)

    def run(self, frame: dict, n_steps: int, box=None) -> dict:
        if self._system is None:
            if self.ctx is None:
                self.ctx = Context(0)
            n = len(frame["x"])
            npt = self._integrator if isinstance(self._integrator, NoseHooverNPT) else None
            baro = next((t for t in self._thermostats if isinstance(t, Barostat)), None)
            dfm = next((t for t in self._thermostats if isinstance(t, Deform)), None)
            lim = self._integrator.xmax if isinstance(self._integrator, NVELimit) else None
            self._system = System(self.ctx, self.desc(n, box if box is not None else frame["box"]),
                                  npt=npt, barostat=baro, nve_limit=lim,
                                  deform=(dfm.axis, dfm.strain_rate) if dfm else None)
            if self._criteria:
                self._system.set_stop_on_nan(True)
            lang = next((t for t in self._thermostats if isinstance(t, FixLangevin)), None)
            if lang is not None and lang.T_stop >= 0 and lang.T_stop != lang.T_start:
                self._system.set_langevin_ramp(lang.T_stop, lang.nfirst, lang.nlast)
        if self._thermo is None:
            sc = self._system.run(frame, n_steps)
        else:
            # in pieces no longer than the energy ring, printing each piece
            cap = HISTORY_DEFAULT
            left = int(n_steps)
            while True:
                k = min(left, cap)
                sc = self._system.run(frame, k)
                if k > 0:
                    self._thermo_rows(self._system.history(k), len(frame["x"]))
                left -= k
                if left <= 0:
                    break
        frame["box"] = tuple(sc["box"])   # the cell moves under NPT
        return sc
