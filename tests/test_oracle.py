"""The oracle (C restatement) against the golden vectors produced by the reference's own C++."""
import os

import numpy as np
import pytest

import cases
from oracle import orc

pytestmark = pytest.mark.skipif(not os.path.exists(os.path.join(orc.BUILD_DIR, "liboracle_f32.so")),
                                reason="oracle not built")


def _water():
    g = np.load(os.path.join(cases.GOLDEN, "water648.npz"))
    s, table = cases.water_case()
    np.testing.assert_array_equal(s.x, g["x"])      # the seeded generator is reproducible
    return s, table, g


def _bonded():
    from nnpengine_b200.systems import WATER
    return (np.array([[1.0, 0, 0, 2 * cases.WATER_BOND_K]], np.float32),
            np.array([[np.cos(np.float32(109.47) * np.float32(np.pi) / np.float32(180)), 0, 0,
                       2 * cases.WATER_ANGLE_KC]], np.float32),
            np.zeros((1, 4), np.float32))


def test_restated_list_matches_reference_bit_exact():
    s, table, g = _water()
    o = orc.Restated(s, "f32")
    assert o.rebuild(s.x, 10, 2, 12) == 0
    assert o.nghost == int(g["nghost"])
    counts, digests = cases.list_keys(o.list_records(), s.natom)
    np.testing.assert_array_equal(counts, g["list_counts"])
    np.testing.assert_array_equal(digests, g["list_digests"])


def test_restated_forces_match_reference():
    s, table, g = _water()
    F, U = cases.table_as_loaded(table[1], table[2])
    o = orc.Restated(s, "f32")
    o.rebuild(s.x, 10, 2, 12)
    f, e, w = o.pair_forces(F, U, 10.0)
    fb, eb, wb = o.bonded(*_bonded())
    assert cases.rel_rms(f + fb, g["force"]) < 1e-5
    # the reference accumulates its energy in float; the restatement sums the same terms in double
    assert abs((e + eb) - g["erg_f32"][0]) / abs(g["erg_f32"][0]) < 1e-4
    assert abs((w + wb) - g["vir_f32"][0]) / abs(g["vir_f32"][0]) < 1e-4


def test_fp64_oracle_close_to_fp32():
    s, table, g = _water()
    F, U = cases.table_as_loaded(table[1], table[2])
    o = orc.Restated(s, "f64")
    o.rebuild(s.x, 10, 2, 12)
    f, e, w = o.pair_forces(F, U, 10.0)
    fb, eb, wb = o.bonded(*_bonded())
    assert cases.rel_rms(f + fb, g["force"]) < 1e-5


def test_restated_gr_counts_bit_exact():
    s, table, g = _water()
    o = orc.Restated(s, "f32")
    o.rebuild(s.x, 10, 2, 12)
    np.testing.assert_array_equal(o.gr_counts(10, 2, 1000, 10), g["gr_counts"])


def test_restated_mixture_gr_and_sq():
    gm = np.load(os.path.join(cases.GOLDEN, "mixture2000.npz"))
    s, table = cases.mixture_case()
    np.testing.assert_array_equal(s.x, gm["x"])
    o = orc.Restated(s, "f32")
    assert o.rebuild(s.x, 10, 2, 17) == 0
    counts, digests = cases.list_keys(o.list_records(), s.natom)
    np.testing.assert_array_equal(counts, gm["list_counts"])
    np.testing.assert_array_equal(digests, gm["list_digests"])
    cnt = o.gr_counts(15, 2, 1000, 10)
    np.testing.assert_array_equal(cnt, gm["gr_counts"])
    # S(q) of the reference's float g(r): FP64 transform agrees with its float transform
    sq, qq = orc.sq(s.natom, float(np.float32(s.bl)), gm["gr_f32"].astype(np.float64), np.float32(10) / np.float32(1000), 512, 20.0)
    np.testing.assert_allclose(qq, gm["qq"], rtol=1e-6)
    scale = np.abs(gm["sq_f32"]).max()
    assert np.abs(sq - gm["sq_f32"]).max() < 1e-3 * scale


@pytest.mark.skipif(not orc.ref_available(), reason="reference harness not built")
def test_reference_harness_reproducible(tmp_path):
    """Re-running the reference gives the committed fixture (seeded inputs, deterministic sums)."""
    s, table, g = _water()
    f = cases.write_inputs(s, table, str(tmp_path))
    v0 = str(tmp_path / "v0.bin")
    np.zeros((s.natom, 3), np.float32).tofile(v0)
    r = orc.run_ref_dump({"init": f["init"], "table": f"1000 {f['table']}", "cutoff": 10, "skin": 2, "gr_cutoff": 10,
                          "bond": [f"1.0 {cases.WATER_BOND_K}"], "angle": [f"109.47 0 0 {cases.WATER_ANGLE_KC}"],
                          "velocity": v0, "mode": "snapshot"}, str(tmp_path / "o"))
    np.testing.assert_array_equal(r["force"].reshape(-1, 3), g["force"])
    np.testing.assert_array_equal(r["gr_counts"].reshape(3, -1), g["gr_counts"])


def test_restated_nnp_tbl_matches_reference():
    """The restated NNPOTENTIAL_TBL (tables, descriptor, fitting net, back-projection) against the
    reference's own C++ with the shim network."""
    from nnpengine_b200 import nnp_model as NM
    g = np.load(os.path.join(cases.GOLDEN, "nnp_gauss648.npz"))
    s, _ = cases.water_case()
    m = NM.gauss_model()
    o = orc.Restated(s, "f32")
    assert o.rebuild(s.x, 6, 2, 8) == 0
    r = o.nnp_tbl(6.0, 750, m.coef_p, m.coef_w, m.coef_d, m.coef_r, m.h1, m.h2, m.fitw)
    np.testing.assert_allclose(r["G"], g["desc"], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(r["dEdG"], g["dedg"], rtol=1e-4, atol=1e-6)
    assert abs(r["e_net"] - g["enn"][0]) / abs(g["enn"][0]) < 1e-6
    fb, _, _ = o.bonded(*[np.asarray(x) * np.array([1, 2, 1, 2], np.float32) for x in cases.water_bonded_raw()[:2]],
                        np.zeros((1, 4), np.float32))
    assert cases.rel_rms(r["f"] + fb, g["force"]) < 1e-5


def test_embedding_nnp_forces_are_energy_gradient():
    """The FP64 oracle's embedding-network forces equal -dE/dx by central differences, on
    atoms of both species (a pair enters G_i through the net of t_j and G_j through that of t_i)."""
    from nnpengine_b200 import nnp_model as NM
    s, _ = cases.water_case(jitter=0.05)
    m = NM.embed_model()
    o = orc.Restated(s, "f64")

    def run(x):
        assert o.rebuild(x, 6, 2, 8) == 0
        return o.nnp_emb(6.0, m.scale, m.e1, m.e2, m.embw, m.h1, m.h2, m.fitw)

    x0 = s.x.astype(np.float32)
    f = run(x0)["f"]
    h = np.float32(2e-3)
    for atom in (0, 1, 2, 301):
        for d in range(3):
            xp, xm = x0.copy(), x0.copy()
            xp[atom, d] += h
            xm[atom, d] -= h
            step = float(xp[atom, d]) - float(xm[atom, d])
            grad = (run(xp)["e_net"] - run(xm)["e_net"]) / step
            assert abs(grad + f[atom, d]) < 2e-4 * np.abs(f[atom]).max() + 1e-6, (atom, d, grad, f[atom, d])


def test_restated_rmdf_matches_reference():
    """The FP64 RMDF restatement on the reference's own float S(q) reproduces the reference's
    refined tables to within its float accumulation (512 terms added to the base value)."""
    g = np.load(os.path.join(cases.GOLDEN, "rmdf2000.npz"))
    s, table = cases.mixture_case()
    F, U = cases.table_as_loaded(table[1], table[2])
    st = orc.rmdf_setup(s.typ, 2, 1000, np.float32(10) / np.float32(1000), 512, 20.0, g["sqex"][None], g["wt"][None],
                        g["ff"][None], 0.02)
    erg, dsq, fq, sqn = orc.rmdf_update(st, g["sq_f32"], np.zeros((1, 512)), 0.5)
    Fo, Uo = orc.rmdf_tables(st, fq, F, U)
    assert abs(erg - g["rmdf_erg"][0]) < 1e-6 * abs(g["rmdf_erg"][0])
    np.testing.assert_allclose(sqn[0], g["rmdf_sq"], rtol=1e-5, atol=1e-6 * np.abs(sqn).max())
    for o, r in ((Fo, g["tbl_force"]), (Uo, g["tbl_pot"])):
        u = np.spacing(np.maximum(np.abs(o), np.abs(r)).astype(np.float32)).astype(np.float64)
        assert (np.abs(o - r) / u).max() <= 1024
    # the target file round-trips through the reference's reader format
    from nnpengine_b200 import systems as S
    q, sqex, wt, ff = S.synthetic_sq_target(512, 20.0, 2, seed=7)
    np.testing.assert_array_equal(sqex, g["sqex"])


@pytest.mark.parametrize("name,ntype", [("sqd648", 2), ("sqd2000", 2)])
def test_restated_sqd_matches_reference(name, ntype):
    """The FP64 SQD restatement on the positions the reference used reproduces its G set per bin
    exactly, its mean |G| to float rounding, and its S(q) to the reference's float accumulation."""
    g = np.load(os.path.join(cases.GOLDEN, name + ".npz"))
    nq = int(g["nq"])
    q, sq, cnt = orc.sqd(g["x"], g["typ"], ntype, float(g["bl"]), nq, float(g["qmax"]))
    np.testing.assert_array_equal(cnt, g["count"])
    assert int(cnt.sum()) == int(g["ngv"])
    m = cnt > 0
    np.testing.assert_allclose(q[m], g["q"][m], rtol=1e-5)
    scale = max(1.0, float(np.abs(g["sq"]).max()))
    assert np.abs(sq[m] - g["sq"][m]).max() < 1e-4 * scale


def test_sqd_vector_set_is_a_half_space_within_the_cutoff():
    """The restated G set holds exactly one of each +-G pair with 0 < |n|^2 <= (int)(q_max/g)^2, and
    its bins follow |G| (the structure the device set-up also builds)."""
    bl, nq, qmax = 18.624, 60, 6.0
    ijk, gscl, b = orc.sqd_gvectors(bl, nq, qmax)
    keys = {tuple(v) for v in ijk}
    assert len(keys) == len(ijk)
    assert not any(tuple(-v) in keys for v in ijk)
    g = np.float32(np.float32(2 * np.pi) / np.float32(bl))
    cut = int(np.float32(np.float32(qmax) / g) ** 2)
    n2 = (ijk ** 2).sum(1)
    assert n2.min() > 0 and n2.max() <= cut
    r = np.arange(-int(np.float32(qmax) / g), int(np.float32(qmax) / g) + 1)
    full = sum(1 for i in r for j in r for k in r if 0 < i * i + j * j + k * k <= cut)
    assert 2 * len(ijk) == full
    order = np.argsort(gscl, kind="stable")
    assert np.all(np.diff(b[order]) >= 0)
    assert b.min() >= 0 and b.max() <= nq - 1
