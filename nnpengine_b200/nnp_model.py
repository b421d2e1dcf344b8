"""Seeded network models in the reference's NNP input formats.

The reference's NNPOTENTIAL_TBL reads (pair_nnp.cpp:457-519):

* a paramfile: the model location, then one input spec ``name dtype index d0 d1 d2 d3`` (-2 means
  nmol, 0 ends the dims) and two output specs ``name index``;
* a float32 weight file: bond (nbtyp x 4), angle (natyp x 4) and dihedral (ndtyp x 4)
  coefficients in raw form, then coef_p [npair][4][6], coef_w, coef_d, coef_r [npair][4][20].

Here the model location names an NNPE model file: a text header ending in a line ``end``,
followed by float32 weights:

    nnpe-model 1
    descriptor embed <e1> <e2> <scale>     | descriptor gauss 20
    fitting <h1> <h2>
    ntype <ntype>
    slots <n> <type of each atom of the molecule>
    end
    [embed: per species W1[e1] b1[e1] W2[e1][e2] b2[e2]]
    per species A1[din][h1] c1[h1] A2[h1][h2] c2[h2] A3[h2] c3

Weights are Xavier-normal (std sqrt(2/(fan_in+fan_out))), biases zero, from an explicit seed.
"""
from __future__ import annotations

import dataclasses
from typing import Optional

import numpy as np


def _xavier(rng, fan_in, fan_out, shape):
    return (rng.standard_normal(shape) * np.sqrt(2.0 / (fan_in + fan_out))).astype(np.float32)


@dataclasses.dataclass
class NnpModel:
    kind: str                      # "embed" or "gauss"
    ntype: int
    npair: int
    h1: int
    h2: int
    fitw: np.ndarray               # per species blocks, float32
    e1: int = 32
    e2: int = 64
    scale: float = 1.0 / 16.0
    embw: Optional[np.ndarray] = None
    coef_p: Optional[np.ndarray] = None   # [npair,4,6]
    coef_w: Optional[np.ndarray] = None   # [npair,4,20]
    coef_d: Optional[np.ndarray] = None
    coef_r: Optional[np.ndarray] = None

    @property
    def din(self) -> int:
        return 4 * self.e2 if self.kind == "embed" else 20


def fitting_weights(rng, ntype, din, h1, h2):
    blocks = []
    for _ in range(ntype):
        blocks += [_xavier(rng, din, h1, (din, h1)).ravel(), np.zeros(h1, np.float32),
                   _xavier(rng, h1, h2, (h1, h2)).ravel(), np.zeros(h2, np.float32),
                   _xavier(rng, h2, 1, (h2,)), np.zeros(1, np.float32)]
    return np.concatenate(blocks).astype(np.float32)


def embed_model(ntype=2, npair=3, e1=32, e2=64, h1=128, h2=128, seed=5, scale=1.0 / 16.0) -> NnpModel:
    """The 1->32->64 radial embedding + 256->128->128->1 fitting network of the 96k-atom workload."""
    rng = np.random.default_rng(seed)
    emb = []
    for _ in range(ntype):
        emb += [_xavier(rng, 1, e1, (e1,)), np.zeros(e1, np.float32), _xavier(rng, e1, e2, (e1, e2)).ravel(),
                np.zeros(e2, np.float32)]
    embw = np.concatenate(emb).astype(np.float32)
    fitw = fitting_weights(rng, ntype, 4 * e2, h1, h2)
    return NnpModel(kind="embed", ntype=ntype, npair=npair, h1=h1, h2=h2, fitw=fitw, e1=e1, e2=e2, scale=scale,
                    embw=embw, coef_p=np.zeros((npair, 4, 6), np.float32), coef_w=np.zeros((npair, 4, 20), np.float32),
                    coef_d=np.zeros((npair, 4, 20), np.float32), coef_r=np.zeros((npair, 4, 20), np.float32))


def gauss_model(ntype=2, npair=3, h1=32, h2=32, seed=6, pair_part=True) -> NnpModel:
    """A tabulated-descriptor model of the reference's own kind: 20 Gaussians per (pair type,
    special class) with coef_w in [0.025,0.075], coef_d in [-2,-0.5], coef_r in [0,5]; pair part
    coef_p (eps, sigma, c8, c10, c12, q_ij) per special class (zero for 1-2/1-3, as the
    reference's own models set them)."""
    rng = np.random.default_rng(seed)
    cw = rng.uniform(0.025, 0.075, (npair, 4, 20)).astype(np.float32)
    cd = rng.uniform(-2.0, -0.5, (npair, 4, 20)).astype(np.float32)
    cr = rng.uniform(0.0, 5.0, (npair, 4, 20)).astype(np.float32)
    cp = np.zeros((npair, 4, 6), np.float32)
    if pair_part:
        c8 = c10 = c12 = 1 / np.sqrt(3.0)
        for p in range(npair):
            eps, sig, qij = [(0.1553 * 4 / np.sqrt(3), 3.166, 0.2), (0.02, 2.5, -0.1), (0.01, 2.0, 0.05)][p % 3]
            base = np.array([eps, sig, c8, c10, c12, qij], np.float32)
            cp[p, 0] = base
            cp[p, 3] = base * np.array([0.5, 1, 1, 1, 1, 0.5], np.float32)
    fitw = fitting_weights(rng, ntype, 20, h1, h2)
    return NnpModel(kind="gauss", ntype=ntype, npair=npair, h1=h1, h2=h2, fitw=fitw, coef_p=cp, coef_w=cw, coef_d=cd,
                    coef_r=cr)


def write_model(path: str, m: NnpModel, slots=(0, 1, 1)) -> None:
    with open(path, "wb") as f:
        f.write(b"nnpe-model 1\n")
        if m.kind == "embed":
            f.write(f"descriptor embed {m.e1} {m.e2} {m.scale:.9g}\n".encode())
        else:
            f.write(b"descriptor gauss 20\n")
        f.write(f"fitting {m.h1} {m.h2}\nntype {m.ntype}\nnpair {m.npair}\n".encode())
        f.write(("slots %d %s\n" % (len(slots), " ".join(str(s) for s in slots))).encode())
        f.write(b"end\n")
        if m.kind == "embed":
            f.write(np.ascontiguousarray(m.embw, np.float32).tobytes())
        f.write(np.ascontiguousarray(m.fitw, np.float32).tobytes())


def write_paramfile(path: str, model_path: str, atoms_per_mol: int = 3, din: int = 20) -> None:
    """pair_nnp.cpp:457-482: model location, one input spec, two output specs."""
    with open(path, "w") as f:
        f.write(f"{model_path}\n")
        f.write(f"serving_default_input_1 f 0 -2 {atoms_per_mol} {din} 0\n")
        f.write("StatefulPartitionedCall 0\nStatefulPartitionedCall 1\n")


def write_weight_file(path: str, m: NnpModel, bond_raw, angle_raw, dih_raw=None) -> None:
    """pair_nnp.cpp:505-519 order: bonded coefficients in raw form (setParam() converts them),
    then coef_p, coef_w, coef_d, coef_r."""
    parts = [np.asarray(bond_raw, np.float32).ravel(), np.asarray(angle_raw, np.float32).ravel()]
    if dih_raw is not None:
        parts.append(np.asarray(dih_raw, np.float32).ravel())
    parts += [m.coef_p.ravel(), m.coef_w.ravel(), m.coef_d.ravel(), m.coef_r.ravel()]
    np.concatenate(parts).astype(np.float32).tofile(path)
