"""Python mirror of the serving C ABI (nnpe_server_*): a stream of independent MD replicas on one GPU.

The server's worker thread (serve.cu) admits requests as slots and HBM free up, keeps a
CUDA-graph launch of `chunk_steps` steps in flight on every resident replica and retires finished
ones; this module only marshals systems into requests and reads results back.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from .systems import System

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


class ServeConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("max_replicas", C.c_int), ("hbm_budget", C.c_int64), ("chunk_steps", C.c_int),
                ("pair_cutoff", C.c_double), ("skin", C.c_double), ("neigh_cap", C.c_int), ("dt", C.c_double),
                ("fp64_state", C.c_int), ("thermostat", C.c_int), ("thermo_frac", C.c_double), ("ntype", C.c_int),
                ("nbin", C.c_int), ("force", _fp), ("potential", _fp), ("nbtyp", C.c_int), ("bcoef", _fp),
                ("natyp", C.c_int), ("acoef", _fp), ("ndtyp", C.c_int), ("dcoef", _fp), ("nnp_kind", C.c_int),
                ("nnp_cutoff", C.c_double), ("nnp_nbin", C.c_int), ("nnp_scale", C.c_double), ("e1", C.c_int),
                ("e2", C.c_int), ("h1", C.c_int), ("h2", C.c_int), ("coef_p", _fp), ("coef_w", _fp), ("coef_d", _fp),
                ("coef_r", _fp), ("embw", _fp), ("fitw", _fp), ("nnp_bf16", C.c_int), ("autotune", C.c_int)]


class Request(C.Structure):
    _fields_ = [("natom", C.c_int), ("bl", C.c_double), ("typ", _ip), ("mass", _fp), ("q", _fp), ("x", _fp), ("v", _fp),
                ("mol_id", _ip), ("intra_id", _ip), ("atom_moltype", _ip), ("nmoltype", C.c_int), ("nmax", C.c_int),
                ("special", _ip), ("nbond", C.c_int), ("bonds", _ip), ("nangle", C.c_int), ("angles", _ip),
                ("ndih", C.c_int), ("dihs", _ip), ("nsteps", C.c_int), ("temperature", C.c_double),
                ("seed", C.c_uint64)]


class RequestStats(C.Structure):
    _fields_ = [("id", C.c_int64), ("natom", C.c_int), ("nsteps", C.c_int), ("status", C.c_int),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double), ("bytes", C.c_int64),
                ("erg", C.c_double), ("ekin", C.c_double), ("temperature", C.c_double)]


_SIGS = {
    "nnpe_server_create": (C.c_int, [C.POINTER(ServeConfig), C.POINTER(C.c_void_p)]),
    "nnpe_server_submit": (C.c_int, [C.c_void_p, C.POINTER(Request), C.POINTER(C.c_int64)]),
    "nnpe_server_wait": (C.c_int, [C.c_void_p, C.c_int64, C.c_double, C.POINTER(RequestStats)]),
    "nnpe_server_result": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.POINTER(RequestStats)]),
    "nnpe_server_drain": (C.c_int, [C.c_void_p, C.c_double]),
    "nnpe_server_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int),
                                   C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int)]),
    "nnpe_server_error": (C.c_char_p, [C.c_void_p]),
    "nnpe_server_footprint": (C.c_int64, [C.c_void_p, C.c_int, C.c_double]),
    "nnpe_server_destroy": (None, [C.c_void_p]),
}


class ServeError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"nnpe serving error {code}: {msg}")
        self.code = code


def _stats(st: RequestStats) -> Dict[str, float]:
    return {k: getattr(st, k) for k, _ in RequestStats._fields_}


class Server:
    """Persistent request loop on one GPU. Force field: pair table (F, U as [npair][nbin+1]),
    bonded coefficients in their stored forms, optional network model (nnp_model.NnpModel)."""

    def __init__(self, device: int = 0, *, ntype: int, table: Optional[Tuple[np.ndarray, np.ndarray]] = None,
                 bcoef: Sequence = (), acoef: Sequence = (), dcoef: Sequence = (), nnp=None, nnp_cutoff: float = 6.0,
                 nnp_nbin: int = 750, bf16: bool = True, pair_cutoff: float = 10.0, skin: float = 2.0,
                 neigh_cap: int = 1024, dt: float = 0.5, fp64: bool = True, thermostat: bool = True,
                 thermo_frac: float = 0.1, max_replicas: int = 64, hbm_budget: int = 64 << 30, chunk_steps: int = 20,
                 autotune: bool = False):
        self.lib = _lib.load()
        for name, (res, args) in _SIGS.items():
            fn = getattr(self.lib, name)
            fn.restype = res
            fn.argtypes = args
        self._keep = []
        cfg = ServeConfig()
        cfg.device, cfg.max_replicas, cfg.hbm_budget, cfg.chunk_steps = device, max_replicas, int(hbm_budget), chunk_steps
        cfg.pair_cutoff, cfg.skin, cfg.neigh_cap, cfg.dt = pair_cutoff, skin, neigh_cap, dt
        cfg.fp64_state, cfg.thermostat, cfg.thermo_frac, cfg.ntype = int(fp64), int(thermostat), thermo_frac, ntype
        cfg.autotune = int(autotune)
        if table is not None:
            F, U = (np.ascontiguousarray(a, np.float32) for a in table)
            cfg.nbin, cfg.force, cfg.potential = F.shape[1] - 1, self._f(F), self._f(U)
        for nm, arr in (("b", bcoef), ("a", acoef), ("d", dcoef)):
            a = np.ascontiguousarray(np.reshape(arr, (-1, 4)), np.float32) if len(arr) else np.zeros((1, 4), np.float32)
            setattr(cfg, f"n{nm}typ", len(a))
            setattr(cfg, f"{nm}coef", self._f(a))
        cfg.nnp_kind = -1
        if nnp is not None:
            cfg.nnp_kind = 1 if nnp.kind == "embed" else 0
            cfg.nnp_cutoff, cfg.nnp_nbin, cfg.nnp_scale = nnp_cutoff, nnp_nbin, nnp.scale
            cfg.e1, cfg.e2, cfg.h1, cfg.h2, cfg.nnp_bf16 = nnp.e1, nnp.e2, nnp.h1, nnp.h2, int(bf16)
            for f in ("coef_p", "coef_w", "coef_d", "coef_r", "embw", "fitw"):
                a = getattr(nnp, f)
                if a is not None:
                    setattr(cfg, f, self._f(np.ascontiguousarray(a, np.float32)))
        h = C.c_void_p()
        rc = self.lib.nnpe_server_create(C.byref(cfg), C.byref(h))
        if rc:
            raise ServeError(rc, "nnpe_server_create failed")
        self.h = h
        self._keep.clear()   # the server holds its own copies

    def _f(self, a):
        a = np.ascontiguousarray(a, np.float32)
        self._keep.append(a)
        return a.ctypes.data_as(_fp)

    def submit(self, s: System, nsteps: int, temperature: float = 300.0, seed: int = 1) -> int:
        mol_id, intra = s.mol_id_intra()
        nmax = max(m.n_atom for m in s.moltypes)
        spec = np.zeros((len(s.moltypes), nmax, nmax), np.int32)
        for k, m in enumerate(s.moltypes):
            spec[k, :m.n_atom, :m.n_atom] = m.special()
        b, a, d = s.topology()
        keep = []

        def ip(x):
            x = np.ascontiguousarray(x, np.int32).ravel()
            if x.size == 0:
                x = np.zeros(1, np.int32)
            keep.append(x)
            return x.ctypes.data_as(_ip)

        def fp(x):
            x = np.ascontiguousarray(x, np.float32).ravel()
            keep.append(x)
            return x.ctypes.data_as(_fp)

        r = Request()
        r.natom, r.bl = s.natom, float(s.bl)
        r.typ, r.mass, r.q, r.x, r.v = ip(s.typ), fp(s.mass), fp(s.q), fp(s.x), fp(s.v)
        r.mol_id, r.intra_id, r.atom_moltype = ip(mol_id), ip(intra), ip(s.mol_type[mol_id])
        r.nmoltype, r.nmax, r.special = len(s.moltypes), nmax, ip(spec)
        r.nbond, r.bonds, r.nangle, r.angles, r.ndih, r.dihs = len(b), ip(b), len(a), ip(a), len(d), ip(d)
        r.nsteps, r.temperature, r.seed = nsteps, temperature, seed
        rid = C.c_int64(0)
        rc = self.lib.nnpe_server_submit(self.h, C.byref(r), C.byref(rid))
        if rc:
            raise ServeError(rc, "submit rejected")
        return rid.value

    def wait(self, rid: int, timeout: float = -1.0) -> Dict[str, float]:
        st = RequestStats()
        rc = self.lib.nnpe_server_wait(self.h, rid, timeout, C.byref(st))
        if rc:
            raise ServeError(rc, self.lib.nnpe_server_error(self.h).decode())
        return _stats(st)

    def result(self, rid: int, natom: int):
        x = np.zeros(natom * 3, np.float32)
        v = np.zeros(natom * 3, np.float32)
        st = RequestStats()
        rc = self.lib.nnpe_server_result(self.h, rid, x.ctypes.data, v.ctypes.data, C.byref(st))
        if rc:
            raise ServeError(rc, self.lib.nnpe_server_error(self.h).decode())
        return x.reshape(-1, 3), v.reshape(-1, 3), _stats(st)

    def stats(self, rid: int) -> Dict[str, float]:
        st = RequestStats()
        self.lib.nnpe_server_result(self.h, rid, None, None, C.byref(st))
        return _stats(st)

    def footprint(self, natom: int, bl: float) -> int:
        """Device bytes admission reserves for a request of natom atoms in a box of edge bl."""
        return int(self.lib.nnpe_server_footprint(self.h, natom, bl))

    def drain(self, timeout: float = -1.0):
        rc = self.lib.nnpe_server_drain(self.h, timeout)
        if rc:
            raise ServeError(rc, "drain timed out")

    def info(self) -> Dict[str, int]:
        done, queued, peak_b, inuse = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        res, peak_r = C.c_int(), C.c_int()
        self.lib.nnpe_server_info(self.h, C.byref(done), C.byref(queued), C.byref(res), C.byref(inuse), C.byref(peak_b),
                                  C.byref(peak_r))
        return dict(done=done.value, queued=queued.value, resident=res.value, bytes_in_use=inuse.value,
                    peak_bytes=peak_b.value, peak_resident=peak_r.value)

    def close(self):
        if getattr(self, "h", None):
            self.lib.nnpe_server_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
