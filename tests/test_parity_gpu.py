"""CUDA force step vs the reference (golden vectors from its own C++) and vs the FP64 oracle.

Bars: neighbour pair sets and g(r) counts bit-exact; per-atom forces within 1e-5 relative RMS of
the reference; energies within 1e-6 relative of the FP64 oracle (FP64 device reductions).
"""
import os

import numpy as np
import pytest

import cases
from nnpengine_b200 import engine as E
from nnpengine_b200.engine import Engine, NNPEError

pytestmark = pytest.mark.gpu

FORCE_RTOL = 1e-5
ENERGY_RTOL = 1e-6


def water_engine(fp64=False, cap=2048, v=None, exact=False):
    s, table = cases.water_case()
    F, U = cases.table_as_loaded(table[1], table[2])
    e = Engine(0)
    e.set_system(s)
    if v is not None:
        e.set_velocities(v)
    e.setup(10.0, 2.0, 10.0, cap)
    e.set_pair_table(F, U)
    e.set_bonded(s, [E.bond_coef(1.0, 0, 0, cases.WATER_BOND_K)], [E.angle_coef(109.47, 0, 0, cases.WATER_ANGLE_KC)])
    e.verlet(1.0, fp64)
    e.pair_exact(exact)
    return s, (F, U), e


def golden(name):
    return np.load(os.path.join(cases.GOLDEN, name))


def fp64_oracle_water(s, F, U):
    from oracle import orc
    o = orc.Restated(s, "f64")
    assert o.rebuild(s.x, 10, 2, 12) == 0
    f, e, w = o.pair_forces(F, U, 10.0)
    fb, eb, wb = o.bonded(E.bond_coef(1.0, 0, 0, cases.WATER_BOND_K)[None],
                          E.angle_coef(109.47, 0, 0, cases.WATER_ANGLE_KC)[None], np.zeros((1, 4), np.float32))
    return f + fb, e + eb, w + wb


def test_neighbour_list_bit_exact():
    g = golden("water648.npz")
    s, _, e = water_engine()
    e.list_build()
    info = e.list_info()
    assert info["nghost"] == int(g["nghost"])
    counts, digests = cases.list_keys(e.list_records(), s.natom)
    np.testing.assert_array_equal(counts, g["list_counts"])
    np.testing.assert_array_equal(digests, g["list_digests"])


@pytest.mark.parametrize("exact", [True, False])
def test_forces_and_energy(exact):
    g = golden("water648.npz")
    s, (F, U), e = water_engine(exact=exact)
    e.list_build()
    erg, vir = e.compute_forces(ev=True)
    f = e.forces()
    assert cases.rel_rms(f, g["force"]) < FORCE_RTOL
    f64, e64, w64 = fp64_oracle_water(s, F, U)
    assert cases.rel_rms(f, f64) < FORCE_RTOL
    assert abs(erg - e64) / abs(e64) < ENERGY_RTOL
    assert abs(vir - w64) / abs(w64) < ENERGY_RTOL


def test_force_evaluation_deterministic():
    s, _, e = water_engine()
    e.list_build()
    e.compute_forces(ev=True)
    f1 = e.forces().copy()
    e.list_build()
    e.compute_forces(ev=True)
    np.testing.assert_array_equal(e.forces(), f1)


def test_gr_counts_bit_exact():
    g = golden("water648.npz")
    s, _, e = water_engine()
    e.list_build()
    e.gr_setup(1000, 512, 20.0)
    e.gr_tally(inner=False)
    np.testing.assert_array_equal(e.gr_counts(False).astype(np.int64), g["gr_counts"])
    e.gr_tally(inner=True)
    np.testing.assert_array_equal(e.gr_counts(True).astype(np.int64), g["gr_inner_counts"])


def test_mixture_gr_counts_and_sq():
    gm = golden("mixture2000.npz")
    from oracle import orc
    s, table = cases.mixture_case()
    F, U = cases.table_as_loaded(table[1], table[2])
    e = Engine(0)
    e.set_system(s)
    e.set_velocities(np.zeros_like(s.v))
    e.setup(10.0, 2.0, 15.0, 2048)
    e.set_pair_table(F, U)
    e.list_build()
    counts, digests = cases.list_keys(e.list_records(), s.natom)
    np.testing.assert_array_equal(counts, gm["list_counts"])
    np.testing.assert_array_equal(digests, gm["list_digests"])
    e.gr_setup(1000, 512, 20.0)
    e.gr_tally(inner=False)
    cnt = e.gr_counts(False).astype(np.int64)
    np.testing.assert_array_equal(cnt, gm["gr_counts"])
    # FP64 normalisation: agrees with the reference's float g(r) to float resolution
    gr = e.gr(False)
    np.testing.assert_allclose(gr, gm["gr_f32"], rtol=2e-6, atol=2e-6)
    # FP64 S(q) vs the FP64 transform of the same g(r) in the oracle, and vs the reference's float S(q)
    sq, q = e.sq(False)
    sq_o, qq = orc.sq(s.natom, float(np.float32(s.bl)), gr, np.float32(10) / np.float32(1000), 512, 20.0)
    np.testing.assert_allclose(q, qq, rtol=1e-12)
    assert np.abs(sq - sq_o).max() < 1e-9 * np.abs(sq_o).max()
    assert np.abs(sq - gm["sq_f32"]).max() < 1e-3 * np.abs(gm["sq_f32"]).max()


def test_nve_trajectory_fp32_matches_reference():
    g = golden("water648.npz")
    s, _, e = water_engine(fp64=False, exact=True)
    log = e.run(21, log_interval=1)
    assert len(log) == 21
    x, v = e.positions(), e.velocities()
    # chaotic growth of summation-order differences stays far below these bounds over 20 fs
    assert cases.rel_rms(x, g["md_x"]) < 1e-5
    assert cases.rel_rms(v, g["md_v"]) < 1e-3
    erg = np.array([r["erg"] for r in log])
    np.testing.assert_allclose(erg, g["md_erg"], rtol=1e-4)
    ekin = np.array([r["ekin"] for r in log])
    np.testing.assert_allclose(ekin, g["md_ekin"], rtol=1e-4)
    assert log[-1]["nbuild"] == int(g["md_nbuild"])


def test_graph_replay_bit_identical():
    s, _, e1 = water_engine(fp64=True)
    l1 = e1.run(30, log_interval=5)
    s, _, e2 = water_engine(fp64=True)
    l2 = e2.run(30, log_interval=5, graph=True)
    np.testing.assert_array_equal(e1.positions(f64=True), e2.positions(f64=True))
    np.testing.assert_array_equal(e1.velocities(f64=True), e2.velocities(f64=True))
    assert [r["erg"] for r in l1] == [r["erg"] for r in l2]


def test_nve_energy_conservation_fp64():
    s, _, e = water_engine(fp64=True)
    e.verlet(0.5, True)
    log = e.run(401, log_interval=50)
    etot = np.array([r["erg"] + r["ekin"] for r in log])
    # 200 fs of NVE from a lattice start: total energy drifts by far less than the kinetic scale
    assert np.abs(etot - etot[0]).max() < 0.02 * abs(log[0]["ekin"]) + 1.0


def test_andersen_thermostat_temperature():
    s, _, e = water_engine(fp64=True)
    e.thermostat("andersen", 300.0, 300.0, interval=1, frac=0.1, seed=7, total_steps=300)
    log = e.run(300, log_interval=10)
    t = np.array([r["temperature"] for r in log[10:]])
    assert 200 < t.mean() < 450


def test_list_overflow_is_reported():
    s, _, e = water_engine(cap=64)
    with pytest.raises(NNPEError) as ei:
        e.list_build()
    assert ei.value.code == 3 and "nei_list overflow" in str(ei.value)
