"""Python mirror of the reference's force-step interfaces over the C ABI.

``Engine`` holds one ``nnpe_ctx`` (one periodic system in HBM) and exposes the reference's
objects' operations under their own names: ENVIRON (system), NEIGHLIST (list build/isvalid),
LJTableCoulDSF (pair table + forces), BOND/ANGLE/DIHEDRAL, VERLET, GR/SQ and the step loop.
Arrays cross the boundary in atom-id order. A non-zero status raises ``NNPEError`` carrying the
library's message (the reference ends the process in the same situations, util.cpp:117-124).
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _lib
from .systems import System


class NNPEError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"nnpe error {code}: {msg}")
        self.code = code


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def _i32(a):
    return np.ascontiguousarray(a, np.int32)


def bond_coef(b0, ka=0.0, kb=0.0, kc=0.0) -> np.ndarray:
    out = np.zeros(4, np.float32)
    _lib.load().nnpe_bond_coef(b0, ka, kb, kc, out)
    return out


def angle_coef(theta0, ka=0.0, kb=0.0, kc=0.0) -> np.ndarray:
    out = np.zeros(4, np.float32)
    _lib.load().nnpe_angle_coef(theta0, ka, kb, kc, out)
    return out


def dihedral_coef(c0=0.0, c1=0.0, c2=0.0, c3=0.0) -> np.ndarray:
    out = np.zeros(4, np.float32)
    _lib.load().nnpe_dihedral_coef(c0, c1, c2, c3, out)
    return out


class Engine:
    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = C.c_void_p()
        rc = self.lib.nnpe_create(device, C.byref(h))
        if rc:
            raise NNPEError(rc, "nnpe_create failed (no CUDA device?)")
        self.h = h
        self.natom = 0
        self.npair = 0

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.nnpe_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ok(self, rc):
        if rc:
            raise NNPEError(rc, self.lib.nnpe_last_error(self.h).decode())

    # ---- ENVIRON ---------------------------------------------------------------------------
    def set_system(self, s: System):
        mol_id, intra = s.mol_id_intra()
        nmax = max(m.n_atom for m in s.moltypes)
        spec = np.zeros((len(s.moltypes), nmax, nmax), np.int32)
        for k, m in enumerate(s.moltypes):
            spec[k, :m.n_atom, :m.n_atom] = m.special()
        amt = s.mol_type[mol_id]
        self._ok(self.lib.nnpe_set_system(self.h, s.natom, s.ntype, float(s.bl), _i32(s.typ), _f32(s.mass), _f32(s.q),
                                          _f32(s.x).ravel(), _i32(mol_id), _i32(intra), _i32(amt), len(s.moltypes),
                                          nmax, spec.ravel()))
        self.natom = s.natom
        self.npair = s.npair
        self._ok(self.lib.nnpe_set_velocities(self.h, _f32(s.v).ravel()))

    def load_system_file(self, path: str):
        self._ok(self.lib.nnpe_load_system_file(self.h, path.encode()))
        self.natom = self.lib.nnpe_natom(self.h)
        self.npair = self.lib.nnpe_npair(self.h)

    def set_positions(self, x):
        self._ok(self.lib.nnpe_set_positions(self.h, _f32(x).ravel()))

    def set_velocities(self, v):
        self._ok(self.lib.nnpe_set_velocities(self.h, _f32(v).ravel()))

    def setup(self, pair_cutoff=10.0, skin=2.0, gr_cutoff=None, neigh_cap=2048):
        self._ok(self.lib.nnpe_setup(self.h, pair_cutoff, skin, gr_cutoff or pair_cutoff, neigh_cap))

    # ---- LJTableCoulDSF --------------------------------------------------------------------
    def set_box(self, bl: float):
        """BL_MANAGER::setBL: a new cubic box length (grid, stencils and ghost limit follow)."""
        self._ok(self.lib.nnpe_set_box(self.h, bl))

    def set_pair_table(self, F, U):
        """F, U: [npair, nbin] or [npair, nbin+1] (the extra zero column is added)."""
        F = np.asarray(F, np.float32); U = np.asarray(U, np.float32)
        if F.shape[1] == U.shape[1] and not np.all(F[:, -1] == 0):
            F = np.concatenate([F, np.zeros((F.shape[0], 1), np.float32)], 1)
            U = np.concatenate([U, np.zeros((U.shape[0], 1), np.float32)], 1)
        self._ok(self.lib.nnpe_pair_set_table(self.h, F.shape[1] - 1, _f32(F).ravel(), _f32(U).ravel()))
        self.nbin = F.shape[1] - 1

    def load_pair_table(self, nbin: int, path: str):
        self._ok(self.lib.nnpe_pair_load_table(self.h, nbin, path.encode()))

    def pair_exact(self, on: bool):
        self._ok(self.lib.nnpe_pair_exact(self.h, int(on)))

    def pair_enable(self, on: bool):
        self._ok(self.lib.nnpe_pair_enable(self.h, int(on)))

    # ---- BOND / ANGLE / DIHEDRAL -----------------------------------------------------------
    def set_bonded(self, s: System, bcoef: Sequence, acoef: Sequence, dcoef: Sequence = ()):
        b, a, d = s.topology()
        bc = _f32(np.reshape(bcoef, (-1, 4))) if len(bcoef) else np.zeros((1, 4), np.float32)
        ac = _f32(np.reshape(acoef, (-1, 4))) if len(acoef) else np.zeros((1, 4), np.float32)
        dc = _f32(np.reshape(dcoef, (-1, 4))) if len(dcoef) else np.zeros((1, 4), np.float32)
        self._ok(self.lib.nnpe_bonded_set(self.h, len(b), _i32(b).ravel(), len(bc), bc.ravel(), len(a), _i32(a).ravel(),
                                          len(ac), ac.ravel(), len(d), _i32(d).ravel(), len(dc), dc.ravel()))

    # ---- NNPOTENTIAL_TBL / network term ---------------------------------------------------
    def nnp_set(self, m, cutoff=6.0, nbin=750):
        """Install a network term (nnp_model.NnpModel) sharing the pair list."""
        kind = 1 if m.kind == "embed" else 0
        keep = []

        def ptr(a):
            if a is None:
                return None
            a = np.ascontiguousarray(a, np.float32)
            keep.append(a)
            return a.ctypes.data

        self._ok(self.lib.nnpe_nnp_set(self.h, kind, cutoff, nbin, m.scale, m.e1, m.e2, m.h1, m.h2, ptr(m.coef_p),
                                       ptr(m.coef_w), ptr(m.coef_d), ptr(m.coef_r), ptr(m.embw), ptr(m.fitw)))

    def nnp_load(self, cutoff: float, nbin: int, paramfile: str, wtfile: str):
        self._ok(self.lib.nnpe_nnp_load(self.h, cutoff, nbin, paramfile.encode(), wtfile.encode()))

    def nnp_enable(self, on: bool):
        self._ok(self.lib.nnpe_nnp_enable(self.h, int(on)))

    def nnp_precision(self, bf16: bool):
        self._ok(self.lib.nnpe_nnp_precision(self.h, int(bf16)))

    # ---- SQD (direct S(q)) -------
    def sqd_setup(self, nq: int, qmax: float) -> int:
        n = C.c_int(0)
        self._ok(self.lib.nnpe_sqd_setup(self.h, nq, qmax, C.byref(n)))
        self._sqd_nq = nq
        return n.value

    def sqd_compute(self):
        """S(q) of the current positions: (mean |G| per bin, sq [nq][npair], vectors per bin)."""
        self._ok(self.lib.nnpe_sqd_compute(self.h))
        nq, npair = self._sqd_nq, int(self.lib.nnpe_npair(self.h))
        q = np.zeros(nq)
        sq = np.zeros(nq * npair)
        cnt = np.zeros(nq, np.int32)
        self._ok(self.lib.nnpe_sqd_get(self.h, q.ctypes.data, sq.ctypes.data, cnt.ctypes.data))
        return q, sq.reshape(nq, npair), cnt

    def sqd_dump(self, path: str, append: bool = False):
        self._ok(self.lib.nnpe_sqd_dump(self.h, path.encode(), int(append)))

    def nnp_autotune(self, reps: int = 5, use_cache: bool = True):
        """Tune the tensor-core kernels' grid sizes on the current state; returns (desc, force) CTAs."""
        gd, gf = C.c_int(0), C.c_int(0)
        self._ok(self.lib.nnpe_nnp_autotune(self.h, reps, int(use_cache), C.byref(gd), C.byref(gf)))
        return gd.value, gf.value

    def nnp_grids(self, grid_desc: int = 0, grid_force: int = 0):
        self._ok(self.lib.nnpe_nnp_grids(self.h, grid_desc, grid_force))

    def nnp_get_grids(self):
        gd, gf = C.c_int(0), C.c_int(0)
        self._ok(self.lib.nnpe_nnp_get_grids(self.h, C.byref(gd), C.byref(gf)))
        return gd.value, gf.value

    def nnp_get(self):
        din, kind = C.c_int(0), C.c_int(0)
        self._ok(self.lib.nnpe_nnp_info(self.h, C.byref(din), C.byref(kind)))
        G = np.zeros(self.natom * din.value, np.float32)
        dG = np.zeros(self.natom * din.value, np.float32)
        e = np.zeros(self.natom)
        self._ok(self.lib.nnpe_nnp_get(self.h, G.ctypes.data, dG.ctypes.data, e.ctypes.data))
        return G.reshape(self.natom, -1), dG.reshape(self.natom, -1), e

    # ---- VERLET / thermostat ---------------------------------------------------------------
    def verlet(self, dt=1.0, fp64=True):
        self._ok(self.lib.nnpe_verlet_setup(self.h, dt, int(fp64)))

    def thermostat(self, kind="none", t_start=300.0, t_end=None, interval=1, frac=0.1, seed=1, total_steps=0):
        k = {"none": 0, "andersen": 1, "csvr": 2}[kind]
        self._ok(self.lib.nnpe_thermostat(self.h, k, t_start, t_end if t_end is not None else t_start,
                                          interval if k else 0, frac, seed))
        self._ok(self.lib.nnpe_set_total_steps(self.h, total_steps))

    # ---- NEIGHLIST -------------------------------------------------------------------------
    def list_build(self):
        self._ok(self.lib.nnpe_list_build(self.h))

    def list_isvalid(self) -> bool:
        v = C.c_int(0)
        self._ok(self.lib.nnpe_list_isvalid(self.h, C.byref(v)))
        return bool(v.value)

    def list_info(self) -> Dict[str, int]:
        ng, nb, gx = C.c_int(0), C.c_int(0), C.c_int(0)
        ne = C.c_int64(0)
        self._ok(self.lib.nnpe_list_info(self.h, C.byref(ng), C.byref(ne), C.byref(nb), C.byref(gx)))
        return dict(nghost=ng.value, entries=ne.value, nbuild=nb.value, num_gx=gx.value)

    def set_prune(self, delta: float) -> None:
        """Dynamic list pruning margin in A (<= 0 or >= skin: off, the kernels read the full list)."""
        self._ok(self.lib.nnpe_set_prune(self.h, float(delta)))

    def prune_info(self) -> Dict[str, float]:
        d, a, n, ne = C.c_double(0), C.c_int(0), C.c_int(0), C.c_int64(0)
        self._ok(self.lib.nnpe_prune_info(self.h, C.byref(d), C.byref(a), C.byref(n), C.byref(ne)))
        return dict(delta=d.value, active=bool(a.value), nprune=n.value, entries=ne.value)

    def verify_grid(self) -> None:
        """ENVIRON::verify_grid on the device's cell sort (raises on a violation)."""
        self._ok(self.lib.nnpe_verify_grid(self.h))

    def list_records(self) -> np.ndarray:
        n = self.list_info()["entries"]
        rec = np.zeros(4 * max(n, 1), np.int32)
        got = C.c_int64(0)
        self._ok(self.lib.nnpe_list_get(self.h, max(n, 1), rec, C.byref(got)))
        return rec[: 4 * got.value].reshape(-1, 4)

    # ---- forces and state ------------------------------------------------------------------
    def compute_forces(self, ev=True):
        e, w = C.c_double(0), C.c_double(0)
        self._ok(self.lib.nnpe_compute_forces(self.h, int(ev), C.byref(e), C.byref(w)))
        return (e.value, w.value) if ev else None

    def forces(self, kind=0) -> np.ndarray:
        f = np.zeros(self.natom * 3, np.float32)
        self._ok(self.lib.nnpe_get_forces(self.h, kind, f))
        return f.reshape(-1, 3)

    def positions(self, f64=False) -> np.ndarray:
        x = np.zeros(self.natom * 3, np.float64 if f64 else np.float32)
        self._ok((self.lib.nnpe_get_positions_f64 if f64 else self.lib.nnpe_get_positions)(self.h, x))
        return x.reshape(-1, 3)

    def velocities(self, f64=False) -> np.ndarray:
        v = np.zeros(self.natom * 3, np.float64 if f64 else np.float32)
        self._ok((self.lib.nnpe_get_velocities_f64 if f64 else self.lib.nnpe_get_velocities)(self.h, v))
        return v.reshape(-1, 3)

    def atom_energy(self) -> np.ndarray:
        e = np.zeros(self.natom)
        self._ok(self.lib.nnpe_get_atom_energy(self.h, e))
        return e

    def device_errors(self) -> int:
        b = C.c_int(0)
        self._ok(self.lib.nnpe_device_errors(self.h, C.byref(b)))
        return b.value

    # ---- the step loop ---------------------------------------------------------------------
    def run(self, nsteps: int, log_interval: int = 1, graph: bool = False, max_log: Optional[int] = None) -> List[dict]:
        cap = max_log if max_log is not None else (nsteps // max(log_interval, 1) + 2)
        buf = (_lib.Thermo * max(cap, 1))()
        n = C.c_int(0)
        fn = self.lib.nnpe_run_graph if graph else self.lib.nnpe_run
        self._ok(fn(self.h, nsteps, log_interval, buf, max(cap, 1), C.byref(n)))
        return [{k: getattr(buf[i], k) for k, _ in _lib.Thermo._fields_} for i in range(n.value)]

    # ---- GR / SQ ---------------------------------------------------------------------------
    def gr_setup(self, nbin_inner: int, nq: int = 512, qmax: float = 20.0, gr_interval: int = 0, gr_interval_long: int = 0):
        self._ok(self.lib.nnpe_gr_setup(self.h, nbin_inner, nq, qmax, gr_interval, gr_interval_long))
        self.nq = nq

    def gr_tally(self, inner: bool = False):
        self._ok(self.lib.nnpe_gr_tally(self.h, int(inner)))

    def gr_counts(self, inner: bool = False) -> np.ndarray:
        nb = self.lib.nnpe_gr_nbin(self.h, int(inner))
        c = np.zeros(self.npair * nb, np.uint64)
        g = np.zeros(self.npair * nb)
        self._ok(self.lib.nnpe_gr_get(self.h, int(inner), c, g))
        return c.reshape(self.npair, nb)

    def gr(self, inner: bool = False) -> np.ndarray:
        nb = self.lib.nnpe_gr_nbin(self.h, int(inner))
        c = np.zeros(self.npair * nb, np.uint64)
        g = np.zeros(self.npair * nb)
        self._ok(self.lib.nnpe_gr_get(self.h, int(inner), c, g))
        return g.reshape(self.npair, nb)

    def sq(self, inner: bool = False):
        s = np.zeros(self.npair * self.nq)
        q = np.zeros(self.nq)
        self._ok(self.lib.nnpe_sq_compute(self.h, int(inner), s, q))
        return s.reshape(self.npair, self.nq), q

    # ---- RMDF ------------------------------------------------------------------------------
    def rmdf_set(self, sqex, wt, ff, strength: float, gamma: float):
        """sqex, wt: [n_sq][nq]; ff: [n_sq][nq][ntype] (the target files' columns)."""
        sqex = np.ascontiguousarray(sqex, np.float64).reshape(-1, self.nq)
        wt = np.ascontiguousarray(wt, np.float64).reshape(-1, self.nq)
        ff = np.ascontiguousarray(ff, np.float64)
        self.n_sq = sqex.shape[0]
        self._ok(self.lib.nnpe_rmdf_set(self.h, self.n_sq, sqex.ravel(), wt.ravel(), ff.ravel(), strength, gamma))

    def rmdf_load(self, files, strength: float, gamma: float):
        arr = (C.c_char_p * len(files))(*[f.encode() for f in files])
        self.n_sq = len(files)
        self._ok(self.lib.nnpe_rmdf_load(self.h, len(files), arr, strength, gamma))

    def rmdf_step(self, potential: bool = False) -> float:
        """compute_Qspace + compute_Rspace (+ compute_Potential); returns erg_exp."""
        e = C.c_double(0)
        self._ok(self.lib.nnpe_rmdf_step(self.h, 7 if potential else 3, C.byref(e)))
        return e.value

    def rmdf_get(self):
        s = np.zeros(self.n_sq * self.nq)
        d = np.zeros(self.n_sq * self.nq)
        f = np.zeros(self.npair * self.nq)
        self._ok(self.lib.nnpe_rmdf_get(self.h, s.ctypes.data, d.ctypes.data, f.ctypes.data))
        return s.reshape(self.n_sq, self.nq), d.reshape(self.n_sq, self.nq), f.reshape(self.npair, self.nq)

    def pair_table(self):
        nb1 = self.nbin + 1
        F = np.zeros(self.npair * nb1, np.float32)
        U = np.zeros(self.npair * nb1, np.float32)
        self._ok(self.lib.nnpe_pair_get_table(self.h, F, U))
        return F.reshape(self.npair, nb1), U.reshape(self.npair, nb1)
