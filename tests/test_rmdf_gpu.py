"""RMDF (reverse-MD / FMIRL table refinement, grsq.cpp:899-1377) on the device vs the reference
(golden vectors from its own C++) and vs the FP64 oracle.

The reference accumulates each table entry in float from the base value over 512 q terms, so its
tables carry up to a few hundred float ulps of rounding where the table is large (small r), and its
S(q) is a float transform (1e-3 relative of the device's FP64 one), which moves the refinement
term by the same fraction. The bars: against the reference, 1024 ulps of the table value plus 1e-3
of the largest table change; against the FP64 oracle run on the device's own S(q), 2 ulps (the
final FP64 -> FP32 rounding).
"""
import os

import numpy as np
import pytest

import cases
from nnpengine_b200.engine import Engine

pytestmark = pytest.mark.gpu

STRENGTH, GAMMA = 0.02, 0.5


def golden(name):
    return np.load(os.path.join(cases.GOLDEN, name))


def ulps(a, b):
    u = np.spacing(np.maximum(np.abs(a), np.abs(b)).astype(np.float32)).astype(np.float64)
    return np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)) / u


def close_to_reference(ours, ref, base):
    slack = 1e-3 * np.abs(np.asarray(ref, np.float64) - base).max()
    u = np.spacing(np.maximum(np.abs(ours), np.abs(ref)).astype(np.float32)).astype(np.float64)
    return bool(np.all(np.abs(np.asarray(ours, np.float64) - ref) <= 1024 * u + slack))


def mixture_engine(v=None):
    s, table = cases.mixture_case()
    F, U = cases.table_as_loaded(table[1], table[2])
    e = Engine(0)
    e.set_system(s)
    e.set_velocities(np.zeros_like(s.v) if v is None else v)
    e.setup(10.0, 2.0, 15.0, 2048)
    e.set_pair_table(F, U)
    return s, (F, U), e


def test_rmdf_update_matches_reference_and_oracle():
    from oracle import orc
    g = golden("rmdf2000.npz")
    s, (F, U), e = mixture_engine()
    e.list_build()
    e.gr_setup(1000, 512, 20.0)
    e.gr_tally(inner=False)
    sq, q = e.sq(False)
    e.rmdf_set(g["sqex"][None], g["wt"][None], g["ff"][None], STRENGTH, GAMMA)
    erg = e.rmdf_step(potential=True)
    sqn, dsq, fq = e.rmdf_get()
    Fg, Ug = e.pair_table()
    # FP64 oracle on the device's own S(q)
    st = orc.rmdf_setup(s.typ, 2, 1000, np.float32(10) / np.float32(1000), 512, 20.0, g["sqex"][None], g["wt"][None],
                        g["ff"][None], STRENGTH)
    erg_o, dsq_o, fq_o, sqn_o = orc.rmdf_update(st, sq, np.zeros((1, 512)), GAMMA)
    Fo, Uo = orc.rmdf_tables(st, fq_o, F, U)
    assert abs(erg - erg_o) < 1e-9 * abs(erg_o)
    np.testing.assert_allclose(fq, fq_o, rtol=1e-9, atol=1e-12 * np.abs(fq_o).max())
    assert ulps(Fg, Fo).max() <= 2 and ulps(Ug, Uo).max() <= 2
    # the reference (float S(q), float table accumulation)
    assert abs(erg - g["rmdf_erg"][0]) < 1e-3 * abs(g["rmdf_erg"][0])
    np.testing.assert_allclose(sqn[0], g["rmdf_sq"], rtol=1e-3, atol=1e-3 * np.abs(g["rmdf_sq"]).max())
    assert close_to_reference(Fg, g["tbl_force"], F) and close_to_reference(Ug, g["tbl_pot"], U)
    # the refinement moved the table, and only inside the table's range (the extra column stays 0)
    assert np.abs(Fg - F).max() > 1e-3 and np.all(Fg[:, -1] == 0)


def test_rmdf_in_step_loop_matches_reference():
    g = golden("rmdf2000.npz")
    s, (F, U), e = mixture_engine(v=cases.mixture_case()[0].v)
    e.verlet(1.0, False)
    e.pair_exact(True)
    e.gr_setup(1000, 512, 20.0, gr_interval=5, gr_interval_long=10)
    e.rmdf_set(g["sqex"][None], g["wt"][None], g["ff"][None], STRENGTH, GAMMA)
    log = e.run(21, log_interval=5)
    assert [r["step"] for r in log] == [0, 5, 10, 15, 20]
    ex = np.array([r["erg_exp"] for r in log])
    np.testing.assert_allclose(ex, g["md_exp"], rtol=1e-3)
    assert cases.rel_rms(e.positions(), g["md_x"]) < 1e-5
    assert cases.rel_rms(e.velocities(), g["md_v"]) < 1e-3
    Fg, Ug = e.pair_table()
    assert close_to_reference(Fg, g["md_tbl_force"], F)
    assert close_to_reference(Ug, g["md_tbl_pot"], U)


def test_rmdf_graph_replay_bit_identical():
    g = golden("rmdf2000.npz")
    out = []
    for graph in (False, True):
        s, _, e = mixture_engine(v=cases.mixture_case()[0].v)
        e.gr_setup(1000, 512, 20.0, gr_interval=2, gr_interval_long=4)
        e.rmdf_set(g["sqex"][None], g["wt"][None], g["ff"][None], STRENGTH, GAMMA)
        log = e.run(12, log_interval=3, graph=graph)
        out.append((e.positions(f64=True), e.pair_table(), [r["erg_exp"] for r in log]))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1][0], out[1][1][0])
    np.testing.assert_array_equal(out[0][1][1], out[1][1][1])
    assert out[0][2] == out[1][2]
