"""ORACLE bindings (test infrastructure only): ctypes access to the C restatement and a runner
for the reference harness ``_ref/ref_dump``."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
BUILD_DIR = os.path.join(HERE, "_build")

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_libs: Dict[str, C.CDLL] = {}


# Where the reference's sources are read from (the only place that names it; REFSRC overrides it).
REFSRC_DEFAULT = "/root/reference/src"


def refsrc() -> str:
    return os.environ.get("REFSRC", REFSRC_DEFAULT)


def build(quiet: bool = True) -> None:
    """Compile the restatement (always) and the reference harness (when its sources exist)."""
    targets = ["restate"]
    src = refsrc()
    if os.path.isdir(src):
        targets.append("ref")
    subprocess.run(["make", "-C", HERE, "-j8", f"REFSRC={src}"] + targets, check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def _lib(prec: str) -> C.CDLL:
    if prec in _libs:
        return _libs[prec]
    path = os.path.join(BUILD_DIR, f"liboracle_{prec}.so")
    lib = C.CDLL(path)
    real = _f32p if prec == "f32" else _f64p
    lib.orc_create.restype = C.c_void_p
    lib.orc_create.argtypes = [C.c_int, C.c_int, C.c_double, _i32p, _f32p, _i32p, _i32p, _i32p, C.c_int, C.c_int, _i32p]
    lib.orc_destroy.argtypes = [C.c_void_p]
    lib.orc_rebuild.argtypes = [C.c_void_p, _f32p, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int]
    lib.orc_list_size.restype = C.c_long
    lib.orc_list_size.argtypes = [C.c_void_p]
    lib.orc_nghost.argtypes = [C.c_void_p]
    lib.orc_num_gx.argtypes = [C.c_void_p]
    lib.orc_get_list.argtypes = [C.c_void_p, _i32p]
    lib.orc_get_sorted.argtypes = [C.c_void_p, _i32p, _i32p, _f64p]
    lib.orc_pair_forces.argtypes = [C.c_void_p, _f32p, _f32p, C.c_int, C.c_double, _f64p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.orc_bonded.argtypes = [C.c_void_p, C.c_int, _i32p, _f32p, C.c_int, _i32p, _f32p, C.c_int, _i32p, _f32p,
                               _f64p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.orc_gr_counts.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_double, _i64p, C.POINTER(C.c_int)]
    lib.orc_nnp_tbl.argtypes = [C.c_void_p, C.c_double, C.c_int, _f32p, _f32p, _f32p, _f32p, C.c_int, C.c_int, _f32p,
                                _f64p, _f64p, _f64p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.orc_nnp_emb.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_int, _f32p, C.c_int, C.c_int, _f32p,
                                _f64p, _f64p, _f64p, _f64p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.orc_nnp_tables.argtypes = [C.c_int, C.c_double, C.c_int, _f32p, _f32p, _f32p, _f32p, real, real, real, real]
    lib.orc_sq.argtypes = [C.c_int, C.c_double, C.c_int, C.c_double, C.c_int, C.c_double, C.c_int, _f64p, _f64p, _f64p]
    _libs[prec] = lib
    return lib


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def _i32(a):
    return np.ascontiguousarray(a, np.int32)


class Restated:
    """One system in the C restatement (``prec`` = "f32" follows the reference's float
    arithmetic, "f64" is the FP64 oracle)."""

    def __init__(self, sysm, prec: str = "f64"):
        self.lib = _lib(prec)
        self.sysm = sysm
        mol_id, intra = sysm.mol_id_intra()
        nmax = max(m.n_atom for m in sysm.moltypes)
        spec = np.zeros((len(sysm.moltypes), nmax, nmax), np.int32)
        for k, m in enumerate(sysm.moltypes):
            spec[k, :m.n_atom, :m.n_atom] = m.special()
        amt = sysm.mol_type[mol_id]
        # the reference reads BL with %f into a float (environ.cpp:42)
        self.h = self.lib.orc_create(sysm.natom, sysm.ntype, float(np.float32(sysm.bl)), _i32(sysm.typ), _f32(sysm.q), _i32(mol_id),
                                     _i32(intra), _i32(amt), len(sysm.moltypes), nmax, spec.ravel())

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def rebuild(self, x, cutoff, skin, comm, cap=2048, max_nbin=126) -> int:
        return self.lib.orc_rebuild(self.h, _f32(x).ravel(), cutoff, skin, comm, cap, max_nbin)

    @property
    def nghost(self) -> int:
        return self.lib.orc_nghost(self.h)

    def list_records(self) -> np.ndarray:
        n = self.lib.orc_list_size(self.h)
        rec = np.zeros(4 * n, np.int32)
        self.lib.orc_get_list(self.h, rec)
        return rec.reshape(-1, 4)

    def pair_forces(self, F, U, cutoff):
        """F, U: [npair, nbin+1] float tables (loadPotential layout)."""
        F = _f32(F); U = _f32(U)
        f = np.zeros(self.sysm.natom * 3)
        e, w = C.c_double(0), C.c_double(0)
        self.lib.orc_pair_forces(self.h, F.ravel(), U.ravel(), F.shape[1] - 1, cutoff, f, C.byref(e), C.byref(w))
        return f.reshape(-1, 3), e.value, w.value

    def bonded(self, bcoef, acoef, dcoef):
        b, a, d = self.sysm.topology()
        f = np.zeros(self.sysm.natom * 3)
        e, w = C.c_double(0), C.c_double(0)
        self.lib.orc_bonded(self.h, len(b), _i32(b).ravel(), _f32(bcoef).ravel(), len(a), _i32(a).ravel(),
                            _f32(acoef).ravel(), len(d), _i32(d).ravel(), _f32(dcoef).ravel(), f, C.byref(e), C.byref(w))
        return f.reshape(-1, 3), e.value, w.value

    def gr_counts(self, gr_cutoff, skin, nbin_inner, r_inner):
        dr = np.float32(r_inner) / np.float32(nbin_inner)
        nmax = int(np.float32(gr_cutoff) * (np.float32(nbin_inner) / np.float32(r_inner))) + 2
        cnt = np.zeros(self.sysm.npair * nmax, np.int64)
        nb = C.c_int(0)
        rc = self.lib.orc_gr_counts(self.h, gr_cutoff, skin, nbin_inner, r_inner, cnt, C.byref(nb))
        assert rc == 0
        return cnt[: self.sysm.npair * nb.value].reshape(self.sysm.npair, nb.value)

    def nnp_tbl(self, cutoff, nbin, coef_p, coef_w, coef_d, coef_r, h1, h2, fitw):
        n = self.sysm.natom
        G = np.zeros(n * 20); dG = np.zeros(n * 20); f = np.zeros(n * 3)
        ep, en, w = C.c_double(0), C.c_double(0), C.c_double(0)
        self.lib.orc_nnp_tbl(self.h, cutoff, nbin, _f32(coef_p).ravel(), _f32(coef_w).ravel(), _f32(coef_d).ravel(),
                             _f32(coef_r).ravel(), h1, h2, _f32(fitw).ravel(), G, dG, f, C.byref(ep), C.byref(en), C.byref(w))
        return dict(G=G.reshape(n, 20), dEdG=dG.reshape(n, 20), f=f.reshape(n, 3), e_pair=ep.value, e_net=en.value, vir=w.value)

    def nnp_emb(self, cutoff, scale, e1, e2, embw, h1, h2, fitw):
        n = self.sysm.natom
        din = 4 * e2
        G = np.zeros(n * din); dG = np.zeros(n * din); ea = np.zeros(n); f = np.zeros(n * 3)
        en, w = C.c_double(0), C.c_double(0)
        self.lib.orc_nnp_emb(self.h, cutoff, scale, e1, e2, _f32(embw).ravel(), h1, h2, _f32(fitw).ravel(), G, dG, ea, f,
                             C.byref(en), C.byref(w))
        return dict(G=G.reshape(n, din), dEdG=dG.reshape(n, din), e_atom=ea, f=f.reshape(n, 3), e_net=en.value, vir=w.value)


def sq(natom, bl, gr, dr, nq, qmax, prec="f64"):
    gr = np.ascontiguousarray(gr, np.float64)
    npair, nbin = gr.shape
    out = np.zeros(npair * nq); qq = np.zeros(nq)
    _lib(prec).orc_sq(natom, bl, nbin, dr, nq, qmax, npair, gr.ravel(), out, qq)
    return out.reshape(npair, nq), qq


# ----------------------------------------------------------------------------------------------
# reference harness
# ----------------------------------------------------------------------------------------------

def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "ref_dump"))


def run_ref_dump(cfg: Dict[str, str], workdir: str, fast: bool = False, env: Optional[dict] = None,
                 timeout: float = 600, threads: int = 27) -> Dict[str, np.ndarray]:
    """Write ``cfg`` (key -> value text) and run the reference harness; returns its arrays.
    fast: the timing build (-O3 AVX2, float network in the shim); threads: 27 (the reference's
    3x3x3 layout) or 8 (its 2x2x2 layout), timing build only."""
    os.makedirs(workdir, exist_ok=True)
    cfg = dict(cfg)
    cfg.setdefault("out", workdir)
    path = os.path.join(workdir, "ref.cfg")
    with open(path, "w") as f:
        for k, v in cfg.items():
            if isinstance(v, list):
                for item in v:
                    f.write(f"{k} {item}\n")
            else:
                f.write(f"{k} {v}\n")
    if threads not in (27, 8) or (threads == 8 and not fast):
        raise ValueError("the harness is built for 27 threads, and for 8 in its timing build")
    exe = os.path.join(REF_DIR, ("ref_dump_fast8" if threads == 8 else "ref_dump_fast") if fast else "ref_dump")
    subprocess.run([exe, path], check=True, cwd=workdir, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                   env=env, timeout=timeout)
    return read_ref_dump(workdir)


def read_ref_dump(d: str) -> Dict[str, np.ndarray]:
    out: Dict[str, np.ndarray] = {}
    info = {}
    with open(os.path.join(d, "info.txt")) as f:
        for line in f:
            k, v = line.split()
            info[k] = float(v) if "." in v else int(v)
    out["info"] = info
    recs = []
    for t in range(int(info["threads"])):
        p = os.path.join(d, f"fulllist_t{t}.i32")
        if os.path.exists(p):
            recs.append(np.fromfile(p, np.int32).reshape(-1, 4))
    if recs:
        out["fulllist"] = np.concatenate(recs)
    for name, dt in [("force.f32", np.float32), ("f.f32", np.float32), ("x.f32", np.float32), ("v.f32", np.float32),
                     ("f_classical.f32", np.float32), ("desc.f32", np.float32), ("dedg.f32", np.float32),
                     ("gr_counts.i64", np.int64), ("gr_inner_counts.i64", np.int64), ("gr.f32", np.float32),
                     ("sq.f32", np.float32), ("qq.f32", np.float32), ("rr.f32", np.float32), ("log_e.f64", np.float64),
                     ("log_w.f64", np.float64), ("log_k.f64", np.float64), ("log_enn.f64", np.float64),
                     ("log_exp.f64", np.float64), ("rmdf_erg.f64", np.float64), ("rmdf_sq.f32", np.float32),
                     ("tbl_force.f32", np.float32), ("tbl_pot.f32", np.float32), ("sqd_q.f32", np.float32),
                     ("sqd_sq.f32", np.float32), ("sqd_count.i32", np.int32)]:
        p = os.path.join(d, name)
        if os.path.exists(p):
            out[name.split(".")[0]] = np.fromfile(p, dt)
    return out


# ----------------------------------------------------------------------------------------------
# RMDF restated in FP64 (grsq.cpp:899-1377)
# ----------------------------------------------------------------------------------------------

def rmdf_setup(typ, ntype, nbin, dr, nq, qmax, sqex, wt, ff, strength):
    """RMDF ctor (grsq.cpp:899-1059): per target n the weights sqwt/fwt [n][P][nq] from the
    scattering factors and type counts, wt*strength, and the transforms ftmx/potmx [nbin][nq]
    on the reference's float grids rr=(i+.5F)dr (grsq.cpp:53), qq=(i+.5F)dq (grsq.cpp:272)."""
    sqex = np.atleast_2d(np.asarray(sqex, np.float64))
    wt = np.atleast_2d(np.asarray(wt, np.float64)) * strength
    ff = np.asarray(ff, np.float64).reshape(sqex.shape[0], nq, ntype)
    cnt = np.bincount(np.asarray(typ), minlength=ntype).astype(np.float64)
    natom = cnt.sum()
    P = ntype * (ntype + 1) // 2
    nsq = sqex.shape[0]
    sqwt = np.zeros((nsq, P, nq)); fwt = np.zeros((nsq, P, nq))
    for n in range(nsq):
        cifi2 = (ff[n] @ cnt / natom) ** 2                       # grsq.cpp:993-997
        ip = 0
        for j in range(ntype):
            ni = cnt[j] / natom ** 2
            for k in range(j, ntype):
                fw = ff[n, :, j] * ff[n, :, k] / cifi2
                sqwt[n, ip] = fw * cnt[k] * ni * (1 if k == j else 2)   # grsq.cpp:1003-1006
                fwt[n, ip] = fw * wt[n]
                ip += 1
    dq = np.float32(np.float32(qmax) / np.float32(nq))
    qq = ((np.arange(nq, dtype=np.float32) + np.float32(0.5)) * dq).astype(np.float64)
    rr = ((np.arange(nbin, dtype=np.float32) + np.float32(0.5)) * np.float32(dr)).astype(np.float64)
    qr = rr[:, None] * qq[None, :]
    j0 = np.sin(qr) / qr
    return dict(sqwt=sqwt, fwt=fwt, sqex=sqex, wt=wt, potmx=j0, ftmx=(j0 - np.cos(qr)) / rr[:, None] ** 2,
                natom=natom, P=P, nsq=nsq)


def rmdf_update(st, sq_partial, deltasq, gamma):
    """compute_Qspace (grsq.cpp:1061-1118): returns erg_exp, new deltasq [n][nq], force_q [P][nq], S_n."""
    sq_partial = np.asarray(sq_partial, np.float64)
    sqn = np.einsum("pq,npq->nq", sq_partial, st["sqwt"])
    d = sqn - st["sqex"]
    erg = float((d * d * st["wt"]).sum()) * st["natom"] * 0.25
    dsq = deltasq + gamma * (d - deltasq)
    fq = np.einsum("nq,npq->pq", dsq, st["fwt"])
    return erg, dsq, fq, sqn


def rmdf_tables(st, fq, Fbase, Ubase, potential=True):
    """compute_Rspace / compute_Potential (grsq.cpp:1120-1210): base + force_q x transform."""
    F = np.array(Fbase, np.float64); U = np.array(Ubase, np.float64)
    nbin = st["ftmx"].shape[0]
    F[:, :nbin] += fq @ st["ftmx"].T
    if potential:
        U[:, :nbin] += fq @ st["potmx"].T
    return F, U


# ----------------------------------------------------------------------------------------------
# SQD (direct S(q) over reciprocal lattice vectors, grsq.cpp:362-585) restated in FP64
# ----------------------------------------------------------------------------------------------

def sqd_gvectors(bl, nq, qmax):
    """The reference's G set and bins (grsq.cpp:362-470): half-space integer triples (k>0; k=0,j>0;
    k=j=0,i>0) with i^2+j^2+k^2 <= (int)(qmax/g)^2, g = 2 pi/L, the cutoff, |G| and the bin edges in
    its float arithmetic. Returns (ijk int[ngv][3], |G| float32[ngv], bin int[ngv])."""
    f = np.float32
    g = f(f(2 * np.pi) / f(bl))
    ratio = f(f(qmax) / g)
    kc = int(ratio)
    cut = int(f(ratio * ratio))
    r = np.arange(-kc, kc + 1)
    I, J, K = np.meshgrid(r, r, r, indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    n2 = I * I + J * J + K * K
    half = (K > 0) | ((K == 0) & (J > 0)) | ((K == 0) & (J == 0) & (I > 0))
    sel = half & (n2 <= cut)
    ijk = np.stack([I[sel], J[sel], K[sel]], 1)
    gscl = (np.sqrt(n2[sel].astype(np.float32)) * g).astype(np.float32)
    dq = f(f(qmax) / f(nq))
    edges = (np.arange(nq, dtype=np.float32) * dq).astype(np.float32)   # i*dq in float, i = 0..nq-1
    b = np.searchsorted(edges, gscl, side="right") - 1                   # largest i with edge_i <= |G|
    return ijk, gscl, np.clip(b, 0, nq - 1)


def sqd(x, typ, ntype, bl, nq, qmax, chunk=4096):
    """FP64 restatement of SQD::compute: per G and type, S_t = sum sin(G.x), C_t = sum cos(G.x);
    per bin and type pair (t1 <= t2), sq = mean over the bin's G of (S1 S2 + C1 C2) * N/(n1 n2)
    minus N/n1 when t1 == t2. Returns (q = mean |G| per bin, sq [nq][npair], count per bin)."""
    ijk, gscl, b = sqd_gvectors(bl, nq, qmax)
    x = np.asarray(x, np.float64)
    typ = np.asarray(typ)
    n = np.bincount(typ, minlength=ntype).astype(np.float64)
    N = float(len(typ))
    pairs = [(i, j) for i in range(ntype) for j in range(i, ntype)]
    acc = np.zeros((nq, len(pairs)))
    G = ijk.astype(np.float64) * (2 * np.pi / float(np.float32(bl)))
    for s0 in range(0, len(G), chunk):
        ph = G[s0:s0 + chunk] @ x.T
        sn, cs = np.sin(ph), np.cos(ph)
        S = np.stack([sn[:, typ == t].sum(1) for t in range(ntype)], 1)
        Cc = np.stack([cs[:, typ == t].sum(1) for t in range(ntype)], 1)
        for p, (i, j) in enumerate(pairs):
            np.add.at(acc[:, p], b[s0:s0 + chunk], S[:, i] * S[:, j] + Cc[:, i] * Cc[:, j])
    count = np.bincount(b, minlength=nq)
    qsum = np.bincount(b, weights=gscl.astype(np.float64), minlength=nq)
    q = np.where(count > 0, qsum / np.maximum(count, 1), 0.0)
    sq = np.zeros((nq, len(pairs)))
    for p, (i, j) in enumerate(pairs):
        fac = N / (n[i] * n[j])
        base = N / n[j] if i == j else 0.0
        sq[:, p] = np.where(count > 0, acc[:, p] / np.maximum(count, 1) * fac - base, 0.0)
    return q, sq, count
