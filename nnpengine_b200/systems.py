"""Seeded synthetic systems written in NNPEngine's own input formats.

The reference reads four kinds of text input, and the drop-in reads the same files:

* the initial configuration (``ENVIRON::initialize``, environ.cpp:22-141): a header
  ``nmoltype nmol``, one molecule-file path per molecule type, ``ntype natom BL``, then one
  line per atom ``moltype typ mass charge x y z`` in molecule order;
* the LAMMPS-like molecule file (``MOLECULE::from_file``, molecule.cpp:25-134) with 1-based
  bond/angle/dihedral records whose first integer after the id is a 1-based type;
* the pair table (``LJTableCoulDSF::loadPotential``, pair.cpp:197-263): ``nbin`` rows of
  ``r F_00/r U_00 F_01/r U_01 ...`` at ``r=(i+.5)dr``;
* the run file of the ``classical`` driver (run.cpp:25-50, 65-190, 397-452).

Every generator takes an explicit seed; nothing reads the clock or ``random_device``.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import List, Optional, Sequence, Tuple

import numpy as np

# Unit constants of the reference (environ.h:60-83): A, kcal/mol, fs, e, amu.
ELECTRIC_K = 332.06371
ACCEL_F = 4.184e-4
EKIN_F = 1195.0286802753603
KT_M_SQRT = 0.0009118367518929329
EK_T = 335.47968899917714
EV_GPA = 6.9476954570553735

# Special-class scale factors (molecule.h:11).
SPECIAL_LJ = (1.0, 0.0, 0.0, 0.5)
SPECIAL_COUL = (1.0, 0.0, 0.0, 5.0 / 6.0)


@dataclasses.dataclass
class MoleculeType:
    """One molecule type: atom count plus 0-based (type, atoms...) topology records."""
    n_atom: int
    bonds: List[Tuple[int, int, int]] = dataclasses.field(default_factory=list)
    angles: List[Tuple[int, int, int, int]] = dataclasses.field(default_factory=list)
    dihedrals: List[Tuple[int, int, int, int, int]] = dataclasses.field(default_factory=list)

    def special(self) -> np.ndarray:
        """special[i][j] in {0,1,2,3} exactly as MOLECULE::from_file builds it (molecule.cpp:98-131)."""
        sp = np.zeros((self.n_atom, self.n_atom), dtype=np.int32)
        for _, a, b in self.bonds:
            sp[a, b] = sp[b, a] = 1
        for _, a, _, c in self.angles:
            sp[a, c] = sp[c, a] = 2
        for _, a, _, _, d in self.dihedrals:
            sp[a, d] = sp[d, a] = 3
        return sp


@dataclasses.dataclass
class System:
    """A periodic system in atom-id order (the order of the configuration file)."""
    bl: float
    ntype: int
    typ: np.ndarray        # int32 [natom]
    mass: np.ndarray       # float32 [natom]
    q: np.ndarray          # float32 [natom]
    x: np.ndarray          # float32 [natom,3]
    v: np.ndarray          # float32 [natom,3]
    moltypes: List[MoleculeType]
    mol_type: np.ndarray   # int32 [nmol]
    name: str = "system"

    @property
    def natom(self) -> int:
        return int(self.typ.shape[0])

    @property
    def nmol(self) -> int:
        return int(self.mol_type.shape[0])

    @property
    def npair(self) -> int:
        return self.ntype * (self.ntype + 1) // 2

    def mol_id_intra(self) -> Tuple[np.ndarray, np.ndarray]:
        mol_id = np.empty(self.natom, np.int32)
        intra = np.empty(self.natom, np.int32)
        k = 0
        for m, mt in enumerate(self.mol_type):
            n = self.moltypes[mt].n_atom
            mol_id[k:k + n] = m
            intra[k:k + n] = np.arange(n)
            k += n
        assert k == self.natom
        return mol_id, intra

    def topology(self):
        """Expanded bond/angle/dihedral lists in atom ids (BOND::autoGenerate, bond.cpp:66-86)."""
        bonds, angles, dihs = [], [], []
        k = 0
        for mt in self.mol_type:
            m = self.moltypes[mt]
            bonds += [(t, a + k, b + k) for t, a, b in m.bonds]
            angles += [(t, a + k, b + k, c + k) for t, a, b, c in m.angles]
            dihs += [(t, a + k, b + k, c + k, d + k) for t, a, b, c, d in m.dihedrals]
            k += m.n_atom
        return (np.array(bonds, np.int32).reshape(-1, 3), np.array(angles, np.int32).reshape(-1, 4),
                np.array(dihs, np.int32).reshape(-1, 5))


def pairtype(ntype: int) -> np.ndarray:
    """pairtype[i][j] enumeration of ENVIRON::initialize (environ.cpp:130-138)."""
    pt = np.zeros((ntype, ntype), np.int32)
    n = 0
    for i in range(ntype):
        for j in range(i, ntype):
            pt[i, j] = pt[j, i] = n
            n += 1
    return pt


def _random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform random rotation matrices from unit quaternions (Shoemake's method)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    q0 = np.sqrt(1 - u1) * np.sin(2 * np.pi * u2)
    q1 = np.sqrt(1 - u1) * np.cos(2 * np.pi * u2)
    q2 = np.sqrt(u1) * np.sin(2 * np.pi * u3)
    q3 = np.sqrt(u1) * np.cos(2 * np.pi * u3)
    w, x, y, z = q3, q0, q1, q2
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z); R[:, 0, 1] = 2 * (x * y - z * w); R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w); R[:, 1, 1] = 1 - 2 * (x * x + z * z); R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w); R[:, 2, 1] = 2 * (y * z + x * w); R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def maxwell_boltzmann(rng: np.random.Generator, mass: np.ndarray, temperature: float) -> np.ndarray:
    """Velocities with the spread ENVIRON::initV uses: sqrt(T/m)*kT_m_sqrt (environ.cpp:190-205)."""
    sd = np.sqrt(temperature / mass.astype(np.float64)) * KT_M_SQRT
    v = rng.standard_normal((mass.shape[0], 3)) * sd[:, None]
    v -= (v * mass[:, None]).sum(0) / mass.sum()
    return v.astype(np.float32)


WATER = MoleculeType(n_atom=3, bonds=[(0, 0, 1), (0, 0, 2)], angles=[(0, 1, 0, 2)])
WATER_MASS = (15.9994, 1.008)
WATER_Q = (-0.8476, 0.4238)
WATER_LJ = (3.166, 0.1553)          # O-O sigma [A], epsilon [kcal/mol]; H carries no LJ
WATER_R_OH = 1.0
WATER_THETA = 109.47


def water_box(n_side: int, bl: float, seed: int, temperature: float = 300.0,
              nmol: Optional[int] = None, name: str = "water") -> System:
    """Rigid-geometry 3-site water on a cubic lattice with seeded random orientations.

    ``n_side**3`` lattice sites of spacing ``bl/n_side``; when ``nmol`` is smaller, a seeded
    subset of sites is occupied (96,000 atoms = 32,000 molecules on a 32^3 lattice).
    """
    rng = np.random.default_rng(seed)
    nsite = n_side ** 3
    nmol = nsite if nmol is None else nmol
    sites = np.arange(nsite) if nmol == nsite else np.sort(rng.choice(nsite, nmol, replace=False))
    ix, iy, iz = np.unravel_index(sites, (n_side, n_side, n_side))
    a = bl / n_side
    centers = np.stack([ix, iy, iz], 1) * a - bl / 2 + a / 2
    th = math.radians(WATER_THETA) / 2
    local = np.array([[0.0, 0.0, 0.0],
                      [WATER_R_OH * math.sin(th), 0.0, WATER_R_OH * math.cos(th)],
                      [-WATER_R_OH * math.sin(th), 0.0, WATER_R_OH * math.cos(th)]])
    R = _random_rotations(rng, nmol)
    x = (centers[:, None, :] + np.einsum("mij,aj->mai", R, local)).reshape(-1, 3)
    x -= np.rint(x / bl) * bl
    typ = np.tile(np.array([0, 1, 1], np.int32), nmol)
    mass = np.array(WATER_MASS, np.float32)[typ]
    q = np.array(WATER_Q, np.float32)[typ]
    v = maxwell_boltzmann(rng, mass, temperature)
    return System(bl=float(bl), ntype=2, typ=typ, mass=mass, q=q, x=x.astype(np.float32), v=v,
                  moltypes=[WATER], mol_type=np.zeros(nmol, np.int32), name=name)


# Hydrogen peroxide H-O-O-H (atom order H1 O1 O2 H2): the smallest molecule with a dihedral, for
# the bonded terms' parity. Types as water (O 0, H 1), so the water pair table applies. Bond types
# 0 (O-H) and 1 (O-O), angle type 0 (H-O-O), dihedral type 0 (H-O-O-H).
PEROXIDE = MoleculeType(n_atom=4, bonds=[(0, 0, 1), (1, 1, 2), (0, 2, 3)], angles=[(0, 0, 1, 2), (0, 1, 2, 3)],
                        dihedrals=[(0, 0, 1, 2, 3)])
PEROXIDE_Q = (-0.41, 0.41)
PEROXIDE_R_OO, PEROXIDE_R_OH, PEROXIDE_THETA, PEROXIDE_PHI = 1.45, 0.97, 100.0, 115.0


def peroxide_box(n_side: int, bl: float, seed: int, temperature: float = 300.0, name: str = "peroxide") -> System:
    """H2O2 molecules on a cubic lattice of n_side^3 sites with seeded random orientations."""
    rng = np.random.default_rng(seed)
    nmol = n_side ** 3
    ix, iy, iz = np.unravel_index(np.arange(nmol), (n_side,) * 3)
    a = bl / n_side
    centers = np.stack([ix, iy, iz], 1) * a - bl / 2 + a / 2
    th, ph = math.radians(PEROXIDE_THETA), math.radians(PEROXIDE_PHI)
    o1, o2 = np.array([-PEROXIDE_R_OO / 2, 0, 0]), np.array([PEROXIDE_R_OO / 2, 0, 0])
    # H1 on O1 at angle theta from the O1->O2 axis in the xz plane; H2 on O2 rotated by the dihedral
    h1 = o1 + PEROXIDE_R_OH * np.array([math.cos(th), 0.0, math.sin(th)])
    h2 = o2 + PEROXIDE_R_OH * np.array([-math.cos(th), math.sin(th) * math.sin(ph), math.sin(th) * math.cos(ph)])
    local = np.stack([h1, o1, o2, h2])
    R = _random_rotations(rng, nmol)
    x = (centers[:, None, :] + np.einsum("mij,aj->mai", R, local)).reshape(-1, 3)
    x -= np.rint(x / bl) * bl
    typ = np.tile(np.array([1, 0, 0, 1], np.int32), nmol)
    mass = np.array(WATER_MASS, np.float32)[typ]
    q = np.array(PEROXIDE_Q, np.float32)[typ]
    v = maxwell_boltzmann(rng, mass, temperature)
    return System(bl=float(bl), ntype=2, typ=typ, mass=mass, q=q, x=x.astype(np.float32), v=v,
                  moltypes=[PEROXIDE], mol_type=np.zeros(nmol, np.int32), name=name)


ATOM = MoleculeType(n_atom=1)


def lj_mixture(natom: int, rho: float, frac_a: float, seed: int, temperature: float = 300.0,
               masses=(39.948, 39.948), charges=(0.5, -0.5), name: str = "mixture") -> System:
    """Two-species atomic liquid: jittered cubic-lattice subset at number density ``rho``."""
    rng = np.random.default_rng(seed)
    bl = (natom / rho) ** (1.0 / 3.0)
    n_side = int(math.ceil(natom ** (1.0 / 3.0)))
    sites = np.sort(rng.choice(n_side ** 3, natom, replace=False))
    ix, iy, iz = np.unravel_index(sites, (n_side,) * 3)
    a = bl / n_side
    x = np.stack([ix, iy, iz], 1) * a - bl / 2 + a / 2 + rng.uniform(-0.1, 0.1, (natom, 3)) * a
    x -= np.rint(x / bl) * bl
    na = int(round(frac_a * natom))
    typ = np.ones(natom, np.int32)
    typ[rng.permutation(natom)[:na]] = 0
    mass = np.array(masses, np.float32)[typ]
    q = np.array(charges, np.float32)[typ]
    v = maxwell_boltzmann(rng, mass, temperature)
    return System(bl=float(bl), ntype=2, typ=typ, mass=mass, q=q, x=x.astype(np.float32), v=v,
                  moltypes=[ATOM], mol_type=np.zeros(natom, np.int32), name=name)


# ----------------------------------------------------------------------------------------------
# pair tables
# ----------------------------------------------------------------------------------------------

def lj_table(ntype: int, sigma: Sequence[float], eps: Sequence[float], cutoff: float, nbin: int,
             mixing: str = "geometric_eps_arith_sigma", r_floor_frac: float = 0.5):
    """F(r)/r and U(r) tables of a plain 12-6 LJ, one column pair per type pair.

    Returns (r[nbin], force[npair,nbin], potential[npair,nbin]) at ``r=(i+.5)dr`` (the grid
    loadPotential checks, pair.cpp:224-229). Below ``r_floor_frac*sigma`` the value is held at
    that radius so that the table stays finite in FP32.
    """
    dr = cutoff / nbin
    r = (np.arange(nbin) + 0.5) * dr
    pt = pairtype(ntype)
    npair = ntype * (ntype + 1) // 2
    F = np.zeros((npair, nbin))
    U = np.zeros((npair, nbin))
    for i in range(ntype):
        for j in range(i, ntype):
            s = 0.5 * (sigma[i] + sigma[j])
            e = math.sqrt(eps[i] * eps[j])
            if e == 0.0 or s == 0.0:
                continue
            rr = np.maximum(r, r_floor_frac * s)
            sr6 = (s / rr) ** 6
            U[pt[i, j]] = 4 * e * (sr6 * sr6 - sr6)
            F[pt[i, j]] = 24 * e * (2 * sr6 * sr6 - sr6) / (rr * rr)
    return r, F, U


def water_lj_table(cutoff: float = 10.0, nbin: int = 1000):
    """O-O LJ of the water model (sigma 3.166 A, epsilon 0.1553 kcal/mol); O-H and H-H zero."""
    return lj_table(2, (WATER_LJ[0], 0.0), (WATER_LJ[1], 0.0), cutoff, nbin)


# ----------------------------------------------------------------------------------------------
# writers (reference formats)
# ----------------------------------------------------------------------------------------------

def write_molecule_file(path: str, mt: MoleculeType) -> None:
    """LAMMPS-like molecule file with 1-based ids and types (molecule.cpp:25-96)."""
    with open(path, "w") as f:
        f.write(f"{mt.n_atom} atoms\n{len(mt.bonds)} bonds\n{len(mt.angles)} angles\n"
                f"{len(mt.dihedrals)} dihedrals\n\n")
        if mt.bonds:
            f.write("Bonds\n\n")
            for k, (t, a, b) in enumerate(mt.bonds):
                f.write(f"{k + 1} {t + 1} {a + 1} {b + 1}\n")
            f.write("\n")
        if mt.angles:
            f.write("Angles\n\n")
            for k, (t, a, b, c) in enumerate(mt.angles):
                f.write(f"{k + 1} {t + 1} {a + 1} {b + 1} {c + 1}\n")
            f.write("\n")
        if mt.dihedrals:
            f.write("Dihedrals\n\n")
            for k, (t, a, b, c, d) in enumerate(mt.dihedrals):
                f.write(f"{k + 1} {t + 1} {a + 1} {b + 1} {c + 1} {d + 1}\n")


def write_init_file(path: str, sysm: System) -> None:
    """Initial configuration in the ENVIRON::initialize format (environ.h:109-114)."""
    d = os.path.dirname(os.path.abspath(path))
    base = os.path.splitext(os.path.basename(path))[0]
    molfiles = []
    for k, mt in enumerate(sysm.moltypes):
        mp = os.path.join(d, f"{base}.mol{k}")
        write_molecule_file(mp, mt)
        molfiles.append(mp)
    mol_id, _ = sysm.mol_id_intra()
    lines = [f"{len(sysm.moltypes)} {sysm.nmol}\n"]
    lines += [m + "\n" for m in molfiles]
    lines.append(f"{sysm.ntype} {sysm.natom} {sysm.bl:.9g}\n")
    mt_of_atom = sysm.mol_type[mol_id]
    for i in range(sysm.natom):
        lines.append(f"{mt_of_atom[i]} {sysm.typ[i]} {float(sysm.mass[i]):.9g} {float(sysm.q[i]):.9g} "
                     f"{float(sysm.x[i, 0]):.9g} {float(sysm.x[i, 1]):.9g} {float(sysm.x[i, 2]):.9g}\n")
    with open(path, "w") as f:
        f.writelines(lines)


def write_pair_table(path: str, r, F, U) -> None:
    """``r F_00/r U_00 F_01/r U_01 ...`` rows, %.9e (float round-trips exactly)."""
    npair, nbin = F.shape
    with open(path, "w") as f:
        for i in range(nbin):
            f.write(f"{r[i]:.9e}" + "".join(f" {F[p, i]:.9e} {U[p, i]:.9e}" for p in range(npair)) + "\n")


def write_velocity_file(path: str, v: np.ndarray) -> None:
    np.asarray(v, np.float32).tofile(path)


def write_sq_target(path: str, q, sqex, wt, ff) -> None:
    """RMDF target file (grsq.cpp:897): ``q S_exp wt f_0 ... f_{ntype-1}`` per q point, %.9e."""
    ff = np.asarray(ff, np.float64)
    with open(path, "w") as f:
        for i in range(len(q)):
            f.write(f"{q[i]:.9e} {sqex[i]:.9e} {wt[i]:.9e}" + "".join(f" {v:.9e}" for v in ff[i]) + "\n")


def synthetic_sq_target(nq: int = 512, qmax: float = 20.0, ntype: int = 2, q_min: float = 0.3, seed: int = 0):
    """A smooth seeded stand-in for a measured structure factor on the SQ grid q_i = (i+.5) qmax/nq:
    S_exp(q) = a sin(b q) exp(-c q), weight 1 from q_min up (0 below), scattering factors constant
    per type. Returns q, S_exp, wt, ff[nq][ntype] (float32 values, as the reference reads them)."""
    rng = np.random.default_rng(seed)
    q = ((np.arange(nq, dtype=np.float32) + np.float32(0.5)) * np.float32(qmax / nq)).astype(np.float32)
    a, b, c = rng.uniform(0.05, 0.15), rng.uniform(0.8, 1.2), rng.uniform(0.05, 0.15)
    sqex = (a * np.sin(b * q) * np.exp(-c * q)).astype(np.float32)
    wt = (q >= q_min).astype(np.float32)
    ff = np.tile(np.linspace(1.0, 0.6, ntype, dtype=np.float32), (nq, 1))
    return q, sqex, wt, ff


WATER_MOLAR_MASS = 18.01528   # g/mol
AVOGADRO_A3 = 0.602214076     # N_A * 1e-24 (g/cm^3 -> g/mol per A^3)


def water_request_box(natom: int, density: float, seed: int, temperature: float) -> System:
    """Water box of about `natom` atoms (rounded down to whole molecules, at least one) at `density`
    g/cm^3: the cubic box holding that many molecules, molecules on the smallest cubic lattice that
    fits them (a seeded subset of its sites), Maxwell-Boltzmann velocities at `temperature`."""
    nmol = max(1, natom // 3)
    bl = (nmol * WATER_MOLAR_MASS / (density * AVOGADRO_A3)) ** (1.0 / 3.0)
    n_side = int(math.ceil(nmol ** (1.0 / 3.0) - 1e-9))
    return water_box(n_side, bl, seed=seed, temperature=temperature, nmol=nmol)


def serving_trace(nreq: int = 256, seed: int = 3, natom_range=(300, 30000), density_range=(0.95, 1.05),
                  temp_range=(250.0, 400.0), steps_range=(100, 5000), rate: float = 20.0):
    """Seeded request stream of the served-replica workload: atom counts log-uniform in natom_range,
    densities and temperatures uniform, step counts uniform integers, Poisson arrivals at `rate`
    per second. Returns a list of dicts (arrival time in s, natom, density, temperature, nsteps, seed)."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(natom_range[0]), np.log(natom_range[1])
    natom = np.exp(rng.uniform(lo, hi, nreq)).astype(int)
    dens = rng.uniform(*density_range, nreq)
    temp = rng.uniform(*temp_range, nreq)
    steps = rng.integers(steps_range[0], steps_range[1] + 1, nreq)
    arrive = np.cumsum(rng.exponential(1.0 / rate, nreq))
    return [dict(t=float(arrive[k]), natom=int(natom[k]), density=float(dens[k]), temperature=float(temp[k]),
                 nsteps=int(steps[k]), seed=int(1000 + k)) for k in range(nreq)]
