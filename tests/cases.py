"""Seeded parity cases shared by the golden-fixture generator and the tests.

Each case is a small system in the reference's own formats, with the water model of the
3000-atom / 96k-atom workloads (O-H bond 1.0 A with k=450 kcal/mol/A^2, H-O-H 109.47 deg
harmonic in cos(theta) with kc=62 kcal/mol, tabulated O-O LJ at 10 A with 1000 bins, DSF
Coulomb, 2 A skin) or the two-species LJ+Coulomb mixture of the g(r)/S(q) workload.
"""
from __future__ import annotations

import hashlib
import math
import os
from typing import Dict

import numpy as np

from nnpengine_b200 import systems as S

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

WATER_BOND_K = 450.0
WATER_ANGLE_KC = 62.0


def water_case(n_side=6, bl=18.624, seed=1, temperature=300.0, nmol=None, jitter=0.0):
    """jitter > 0 displaces atoms by seeded N(0, jitter) so that bonds and angles are off their
    equilibrium (the lattice start sits exactly on it, where FP32 bonded forces are rounding noise)."""
    s = S.water_box(n_side, bl, seed=seed, temperature=temperature, nmol=nmol)
    if jitter > 0:
        rng = np.random.default_rng(seed + 1000)
        s.x = (s.x + rng.normal(0, jitter, s.x.shape)).astype(np.float32)
    r, F, U = S.water_lj_table(10.0, 1000)
    return s, (r, F, U)


MIX_SIGMA, MIX_EPS = (3.0, 3.4), (0.15, 0.25)


def mixture_table(eps_scale=1.0):
    return S.lj_table(2, MIX_SIGMA, tuple(eps_scale * e for e in MIX_EPS), 10.0, 1000)


def rescaled(s, bl):
    """System s with box length bl and positions scaled by bl / s.bl (float32)."""
    import dataclasses
    return dataclasses.replace(s, bl=float(bl), x=(np.asarray(s.x, np.float64) * (bl / s.bl)).astype(np.float32))


def mixture_case(natom=2000, rho=0.035, seed=4):
    s = S.lj_mixture(natom, rho, 0.6, seed=seed)
    return s, mixture_table()


def water3000_case():
    """The 3000-atom box of the plain workload: 1000 molecules on a 10^3 lattice in 31.04 A, seed 2."""
    return water_case(n_side=10, bl=31.04, seed=2)


def mixture30k_case():
    """The 30,000-atom liquid of the g(r)/S(q) workload: 60/40 at 0.035 A^-3 (94.99 A box), seed 4."""
    return mixture_case(natom=30000, rho=0.035, seed=4)


PEROXIDE_BOND = ((0.97, 450.0), (1.45, 300.0))     # (b0, k) of bond types O-H, O-O
PEROXIDE_ANGLE = (100.0, 50.0)                     # (theta0, kc) of H-O-O, harmonic in cos(theta)
PEROXIDE_DIHEDRAL = (1.0, 1.5, -0.8, 0.3)          # c0 + c1 cos(phi) + c2 cos(2 phi) + c3 cos(3 phi)


def peroxide_case(jitter=0.05):
    """512 H2O2 molecules (2048 atoms) in a 30.4 A box, seed 9, atoms displaced by seeded N(0, jitter)."""
    s = S.peroxide_box(8, 30.4, seed=9)
    if jitter > 0:
        rng = np.random.default_rng(1009)
        s.x = (s.x + rng.normal(0, jitter, s.x.shape)).astype(np.float32)
    return s, S.water_lj_table(10.0, 1000)


def peroxide_bonded_cfg():
    """The peroxide bonded terms as the reference harness's config lines (BOND/ANGLE/DIHEDRAL::setParam)."""
    return {"bond": [f"{b0} {k}" for b0, k in PEROXIDE_BOND], "angle": [f"{PEROXIDE_ANGLE[0]} 0 0 {PEROXIDE_ANGLE[1]}"],
            "dihedral": [" ".join(str(c) for c in PEROXIDE_DIHEDRAL)]}


def bond_row(b0, ka=0.0, kb=0.0, kc=0.0):
    """BOND::setParam's coefficient row (bond.cpp:27-33): (b0, 2 ka, kb, 2 kc) in float."""
    f = np.float32
    return np.array([f(b0), f(ka) * f(2), f(kb), f(kc) * f(2)], np.float32)


def angle_row(theta0, ka=0.0, kb=0.0, kc=0.0):
    """ANGLE::setParam's row (angle.cpp:26-32): (cos theta0, 2 ka, kb, 2 kc) in float."""
    f = np.float32
    return np.array([cos_theta0(theta0), f(ka) * f(2), f(kb), f(kc) * f(2)], np.float32)


def dihedral_row(c0, c1, c2, c3):
    """DIHEDRAL::setParam's row (dihedral.cpp:27-35): (c0 - c2, c1 - 3 c3, 4 c2, 12 c3) in float."""
    f = np.float32
    c0, c1, c2, c3 = f(c0), f(c1), f(c2), f(c3)
    return np.array([c0 - c2, c1 - f(3) * c3, c2 * f(2) * f(2), c3 * f(4) * f(3)], np.float32)


def peroxide_coefs():
    """The peroxide terms as coefficient rows (the setParam transforms): (bond rows, angle rows,
    dihedral rows)."""
    return ([bond_row(b0, 0, 0, k) for b0, k in PEROXIDE_BOND], [angle_row(PEROXIDE_ANGLE[0], 0, 0, PEROXIDE_ANGLE[1])],
            [dihedral_row(*PEROXIDE_DIHEDRAL)])


def table_as_loaded(F, U):
    """The tables as the reference holds them after reading the %.9e text: float32, extra zero column."""
    F = np.asarray(F, np.float64).astype(np.float32)
    U = np.asarray(U, np.float64).astype(np.float32)
    z = np.zeros((F.shape[0], 1), np.float32)
    return np.concatenate([F, z], 1), np.concatenate([U, z], 1)


def write_inputs(s, table, d) -> Dict[str, str]:
    """Write the reference-format inputs of a case into directory d."""
    os.makedirs(d, exist_ok=True)
    init = os.path.join(d, "init.txt")
    S.write_init_file(init, s)
    tab = os.path.join(d, "table.txt")
    r, F, U = table
    S.write_pair_table(tab, r, F, U)
    vel = os.path.join(d, "v.bin")
    S.write_velocity_file(vel, s.v)
    return dict(init=init, table=tab, vel=vel)


def list_keys(rec: np.ndarray, natom: int):
    """Per-atom sorted neighbour keys (id_j, image, special) and a digest per atom."""
    rec = np.asarray(rec, np.int64)
    key = (rec[:, 1] * 27 + rec[:, 2]) * 4 + rec[:, 3]
    order = np.lexsort((key, rec[:, 0]))
    i_sorted, k_sorted = rec[order, 0], key[order]
    counts = np.bincount(i_sorted, minlength=natom)
    starts = np.concatenate([[0], np.cumsum(counts)])
    digests = np.zeros(natom, np.uint64)
    for a in range(natom):
        h = hashlib.blake2b(k_sorted[starts[a]:starts[a + 1]].tobytes(), digest_size=8).digest()
        digests[a] = np.frombuffer(h, np.uint64)[0]
    return counts, digests


def block_digests(digests, block=1000):
    """One 64-bit digest per block of `block` atoms over the per-atom list digests (a checksum of
    checksums that keeps large fixtures small)."""
    d = np.asarray(digests, np.uint64)
    out = []
    for k in range(0, len(d), block):
        h = hashlib.blake2b(d[k:k + block].tobytes(), digest_size=8).digest()
        out.append(np.frombuffer(h, np.uint64)[0])
    return np.array(out, np.uint64)


def x_digest(x):
    return np.frombuffer(hashlib.blake2b(np.ascontiguousarray(x, np.float32).tobytes(), digest_size=8).digest(),
                         np.uint64)[0]


def rel_rms(a, b):
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def cos_theta0(theta0_deg: float) -> np.float32:
    """cos(theta_0) as ANGLE::setParam computes it (angle.cpp:28): the argument theta*pi/180 in
    float, the cosine correctly rounded to float (the library's nnpe_angle_coef gives the same
    bits). Plain numpy, so that the reference's timing process loads no library of this project."""
    f = np.float32
    arg = f(f(theta0_deg) * f(3.141592653589793238462643383279502884)) / f(180)
    return f(math.cos(float(arg)))


def water_bonded_raw():
    """Raw (pre-setParam) bond/angle/dihedral coefficients of the water model, as the reference's
    NNP weight file stores them (pair_nnp.cpp:507-512): setParam() doubles entries 1 and 3."""
    return (np.array([[1.0, 0, 0, WATER_BOND_K]], np.float32),
            np.array([[cos_theta0(109.47), 0, 0, WATER_ANGLE_KC]], np.float32), np.zeros((1, 4), np.float32))


def write_nnp_inputs(m, d):
    """Model file, paramfile and reference-layout weight file of a network model into d."""
    from nnpengine_b200 import nnp_model as NM
    os.makedirs(d, exist_ok=True)
    model = os.path.join(d, "model.nnpe")
    param = os.path.join(d, "nnp.param")
    wt = os.path.join(d, "nnp.wt")
    NM.write_model(model, m)
    NM.write_paramfile(param, model, 3, m.din)
    b, a, dd = water_bonded_raw()
    NM.write_weight_file(wt, m, b, a, dd)
    return dict(model=model, param=param, wt=wt)


def write_run_input(d, mode, s, table=None, nnp_paths=None, temps=(0.0, 0.0), steps=(20, 5, 20, 5, 10),
                    rmdf=None, nbin=1000, cutoffs=(10.0, 2.0, 10.0), nq=512, qmax=20.0, sqd=None, append=False):
    """The run input file of the reference's `classical` or `nnp_run` mode (run.cpp:25-50) for a
    case in directory d; rmdf = (strength, gamma, target file) or None (no target: n_sq 0, which
    the reference reads but cannot run, so its harness runs use one target of strength 0);
    sqd = (q_max, nq) writes the direct S(q) of the final state, None skips it; append: the output
    lines ask for appending (running averages of the g(r), S(q), SQD and RMDF dumps)."""
    os.makedirs(d, exist_ok=True)
    init = os.path.join(d, "init.txt")
    S.write_init_file(init, s)
    lines = [init, "%g %g %g" % cutoffs]
    if mode == "classical":
        tab = os.path.join(d, "table.txt")
        S.write_pair_table(tab, table[0], table[1], table[2])
        lines += [f"{nbin} {tab}", "1", f"1.0 {WATER_BOND_K}", "1", f"109.47 0 0 {WATER_ANGLE_KC}", "0"]
    else:
        lines += ["1", "1", "0", nnp_paths["param"], nnp_paths["wt"], str(nbin)]
    lines.append(f"{nbin} {nq} {qmax}")
    if rmdf is None:
        lines += ["0 1", "0", "*"]
    else:
        lines += [f"{rmdf[0]} {rmdf[1]}", f"1 {rmdf[2]}", os.path.join(d, "no_such_delta.txt")]
    lines.append(f"{temps[0]} {temps[1]}")
    lines.append(" ".join(str(v) for v in steps))
    out = {k: os.path.join(d, k + ".out") for k in ("xyz", "gr", "sq", "sqd", "sqx", "force")}
    ap = int(bool(append))
    sqd_line = f"{out['sqd']} {ap} {sqd[0]} {sqd[1]}" if sqd else "* 0 20 10"   # file append q_max nq
    lines += [f"{out['xyz']} {ap}", f"{out['gr']} {ap}", f"{out['sq']} {ap}", sqd_line, f"{out['sqx']} {ap}"]
    if mode == "classical":
        lines.append(f"{out['force']} {ap}")
    path = os.path.join(d, "run.in")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path, out


def read_dump(path):
    """An output file of the reference's formats as numbers: xyz frames (ENVIRON::dump,
    environ.cpp:178-188) -> (frames [n][natom][3], types [natom], box half-lengths); the other
    dumps (GR/SQ/SQD::dump, RMDF::dumpSQ, dumpForce) -> (accumulation count from the '# n'
    header or 0, rows [m][cols])."""
    with open(path) as f:
        lines = [ln.split() for ln in f if ln.strip()]
    if lines and lines[0][0].isdigit() and len(lines) > 1 and lines[1][:4] == ["x", "y", "z", "w"]:
        frames, k = [], 0
        while k < len(lines):
            n = int(lines[k][0])
            box = (float(lines[k + 1][4]), float(lines[k + 1][5]))
            rows = lines[k + 2:k + 2 + n]
            frames.append([[float(v) for v in r[1:4]] for r in rows])
            types = [int(r[0][1:]) for r in rows]
            k += 2 + n
        return np.array(frames), np.array(types), box
    num = 0
    if lines and lines[0][0] == "#":
        num = int(lines[0][1])
        lines = lines[1:]
    return num, np.array([[float(v) for v in r] for r in lines])


def parse_log(text):
    """The step lines of the reference's log (run.cpp:383-390): md_step temp press erg dif nbuild."""
    rows = []
    for line in text.splitlines():
        f = line.split()
        if len(f) == 6 and f[0].lstrip("-").isdigit():
            rows.append([float(v) for v in f])
    return np.array(rows)
