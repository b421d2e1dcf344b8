"""The variable-box path (nnpe_set_box, the reference's BL_MANAGER::setBL run.cpp:688-712): one
context set up at the 648-atom water box's length, moved to a smaller box, a larger one (its grid
has more cells, so the grid arrays are reallocated) and back; at each box the pair set is the
reference's bit for bit and the forces match the reference and the FP64 oracle."""
import os

import numpy as np
import pytest

import cases
from nnpengine_b200 import engine as E
from nnpengine_b200.engine import Engine

pytestmark = pytest.mark.gpu


def test_set_box_matches_reference_at_each_box():
    from oracle import orc
    g, g0 = (np.load(os.path.join(cases.GOLDEN, n)) for n in ("box648.npz", "water648.npz"))
    s, table = cases.water_case()
    F, U = cases.table_as_loaded(table[1], table[2])
    e = Engine(0)
    e.set_system(s)
    e.set_velocities(np.zeros_like(s.v))
    e.setup(10.0, 2.0, 10.0, 2048)
    e.set_pair_table(F, U)
    rows = ([cases.bond_row(1.0, 0, 0, cases.WATER_BOND_K)], [cases.angle_row(109.47, 0, 0, cases.WATER_ANGLE_KC)])
    e.set_bonded(s, *rows)
    e.verlet(1.0, True)
    gx = e.list_info()["num_gx"]
    for tag in ("small", "large", None):
        if tag:
            bl, x = float(g[f"{tag}_bl"]), g[f"{tag}_x"]
            ref = dict(nghost=g[f"{tag}_nghost"], counts=g[f"{tag}_list_counts"], digests=g[f"{tag}_list_digests"],
                       force=g[f"{tag}_force"])
        else:
            bl, x = s.bl, s.x
            ref = dict(nghost=g0["nghost"], counts=g0["list_counts"], digests=g0["list_digests"], force=g0["force"])
        e.set_box(bl)
        e.set_positions(x)
        e.list_build()
        info = e.list_info()
        if tag == "large":
            assert info["num_gx"] > gx          # the grid grew
        assert info["nghost"] == int(ref["nghost"])
        counts, digests = cases.list_keys(e.list_records(), s.natom)
        np.testing.assert_array_equal(counts, ref["counts"])
        np.testing.assert_array_equal(digests, ref["digests"])
        erg, _ = e.compute_forces(True)
        f = e.forces()
        assert cases.rel_rms(f, ref["force"]) < 1e-5
        sb = cases.rescaled(s, bl) if tag else s
        o = orc.Restated(sb, "f64")
        assert o.rebuild(sb.x, 10, 2, 12) == 0
        fp, ep, _ = o.pair_forces(F, U, 10.0)
        fb, eb, _ = o.bonded(np.array(rows[0]), np.array(rows[1]), np.zeros((1, 4), np.float32))
        assert cases.rel_rms(f, fp + fb) < 1e-5
        assert abs(erg - (ep + eb)) / abs(ep + eb) < 1e-6
    assert e.device_errors() == 0
    e.close()
