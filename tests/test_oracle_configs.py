"""The oracle (C restatement) against the reference's own C++ at the workloads' sizes: the
3000-atom water box, the 30,000-atom two-species liquid and a 2048-atom system with dihedrals
(fixtures from tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

import cases
from oracle import orc

pytestmark = pytest.mark.skipif(not os.path.exists(os.path.join(orc.BUILD_DIR, "liboracle_f32.so")),
                                reason="oracle not built")


def golden(name):
    return np.load(os.path.join(cases.GOLDEN, name))


def water_rows():
    return (cases.bond_row(1.0, 0, 0, cases.WATER_BOND_K)[None], cases.angle_row(109.47, 0, 0, cases.WATER_ANGLE_KC)[None],
            np.zeros((1, 4), np.float32))


def test_water3000_list_forces_gr():
    g = golden("water3000.npz")
    s, table = cases.water3000_case()
    np.testing.assert_array_equal(s.x, g["x"])
    F, U = cases.table_as_loaded(table[1], table[2])
    o = orc.Restated(s, "f32")
    assert o.rebuild(s.x, 10, 2, 12) == 0
    assert o.nghost == int(g["nghost"])
    counts, digests = cases.list_keys(o.list_records(), s.natom)
    np.testing.assert_array_equal(counts, g["list_counts"])
    np.testing.assert_array_equal(digests, g["list_digests"])
    np.testing.assert_array_equal(o.gr_counts(10, 2, 1000, 10), g["gr_counts"])
    f, e, w = o.pair_forces(F, U, 10.0)
    fb, eb, wb = o.bonded(*water_rows())
    assert cases.rel_rms(f + fb, g["force"]) < 1e-5
    o64 = orc.Restated(s, "f64")
    assert o64.rebuild(s.x, 10, 2, 12) == 0
    f64, e64, _ = o64.pair_forces(F, U, 10.0)
    fb64, eb64, _ = o64.bonded(*water_rows())
    assert cases.rel_rms(f64 + fb64, g["force"]) < 1e-5
    # the reference sums its energy in float
    assert abs(e64 + eb64 - g["erg_f32"][0]) / abs(g["erg_f32"][0]) < 1e-4


def test_mixture30k_list_and_gr_counts():
    g = golden("mixture30k.npz")
    s, table = cases.mixture30k_case()
    assert cases.x_digest(s.x) == g["x_digest"]     # the seeded generator reproduces the reference's input
    o = orc.Restated(s, "f32")
    assert o.rebuild(s.x, 10, 2, 17) == 0
    assert o.nghost == int(g["nghost"])
    counts, digests = cases.list_keys(o.list_records(), s.natom)
    np.testing.assert_array_equal(counts, g["list_counts"])
    np.testing.assert_array_equal(cases.block_digests(digests), g["list_block_digests"])
    np.testing.assert_array_equal(o.gr_counts(15, 2, 1000, 10), g["gr_counts"])


def test_peroxide_dihedral_forces():
    g = golden("peroxide2048.npz")
    s, table = cases.peroxide_case()
    np.testing.assert_array_equal(s.x, g["x"])
    b, a, d = cases.peroxide_coefs()
    for prec, tol in (("f32", 1e-5), ("f64", 1e-5)):
        o = orc.Restated(s, prec)
        assert o.rebuild(s.x, 10, 2, 12) == 0
        fb, eb, _ = o.bonded(np.array(b), np.array(a), np.array(d))
        assert cases.rel_rms(fb, g["f_bonded"]) < tol
        assert abs(eb - g["erg_bonded"][0]) / abs(g["erg_bonded"][0]) < 1e-5
    # the dihedral carries force: dropping it moves the bonded forces well past the bar
    o = orc.Restated(s, "f64")
    o.rebuild(s.x, 10, 2, 12)
    fnd, _, _ = o.bonded(np.array(b), np.array(a), np.zeros((1, 4), np.float32))
    assert cases.rel_rms(fnd, g["f_bonded"]) > 1e-3


def test_rescaled_boxes_list_and_forces():
    """The restatement at the box lengths of the variable-box fixture: pair set bit-exact, forces."""
    g = golden("box648.npz")
    s, table = cases.water_case()
    F, U = cases.table_as_loaded(table[1], table[2])
    for tag in ("small", "large"):
        sb = cases.rescaled(s, float(g[f"{tag}_bl"]))
        np.testing.assert_array_equal(sb.x, g[f"{tag}_x"])
        o = orc.Restated(sb, "f32")
        assert o.rebuild(sb.x, 10, 2, 12) == 0
        assert o.nghost == int(g[f"{tag}_nghost"])
        counts, digests = cases.list_keys(o.list_records(), sb.natom)
        np.testing.assert_array_equal(counts, g[f"{tag}_list_counts"])
        np.testing.assert_array_equal(digests, g[f"{tag}_list_digests"])
        f, _, _ = o.pair_forces(F, U, 10.0)
        fb, _, _ = o.bonded(*water_rows())
        assert cases.rel_rms(f + fb, g[f"{tag}_force"]) < 1e-5
