"""The CUDA force step at the workloads' own sizes, against the reference's C++ (golden vectors from
tests/golden/make_golden.py) and the FP64 oracle:

* the 3000-atom water box (plain workload): pair set and g(r) counts bit-exact, forces within 1e-5
  relative RMS of the reference and of FP64, energy and virial within 1e-6 of FP64; 100 NVE steps
  tracking the reference's trajectory; 1000 NVE steps agreeing with its energy statistics;
* the same box after the reference's 5 ps of equilibration with the network term added: the FP32
  network within 1e-5 of FP64 (forces) and 1e-6 (energy), the BF16 tensor-core network within 1 %
  of the FP64 force RMS;
* the 96,000-atom box: the BF16 and FP32 network force errors against FP64;
* the 30,000-atom two-species liquid (g(r)/S(q) workload): pair set and g(r) counts bit-exact;
* a 2048-atom H2O2 system: the dihedral term against the reference and FP64;
* the FP32 network's forces against a finite difference of the GPU's own FP64-summed energy.
"""
import os

import numpy as np
import pytest

import cases
from nnpengine_b200 import nnp_model as NM
from nnpengine_b200 import systems as S
from nnpengine_b200.engine import Engine

pytestmark = pytest.mark.gpu

FORCE_RTOL = 1e-5
ENERGY_RTOL = 1e-6
BF16_FORCE_BAR = 1e-2


def golden(name):
    return np.load(os.path.join(cases.GOLDEN, name))


def water_rows():
    return ([cases.bond_row(1.0, 0, 0, cases.WATER_BOND_K)], [cases.angle_row(109.47, 0, 0, cases.WATER_ANGLE_KC)])


def engine_for(s, table, v=None, exact=False, fp64=True, gr_cutoff=10.0, bonded=None, nnp=None):
    F, U = cases.table_as_loaded(table[1], table[2])
    e = Engine(0)
    e.set_system(s)
    e.set_velocities(np.zeros_like(s.v) if v is None else v)
    e.setup(10.0, 2.0, gr_cutoff, 2048)
    e.set_pair_table(F, U)
    if bonded is not None:
        e.set_bonded(s, *bonded)
    if nnp is not None:
        e.nnp_set(nnp, 6.0, 750)
    e.verlet(1.0, fp64)
    e.pair_exact(exact)
    return e, (F, U)


def fp64_classical(s, x, F, U, rows, dcoef=None):
    from oracle import orc
    o = orc.Restated(s, "f64")
    assert o.rebuild(x, 10, 2, 12) == 0
    f, e, w = o.pair_forces(F, U, 10.0)
    b, a = rows
    d = np.zeros((1, 4), np.float32) if dcoef is None else np.array(dcoef)
    fb, eb, wb = o.bonded(np.array(b), np.array(a), d)
    return f + fb, e + eb, w + wb


def min_image_rms(a, b, bl):
    d = np.asarray(a, np.float64) - np.asarray(b, np.float64)
    d -= np.rint(d / bl) * bl
    return float(np.sqrt((d ** 2).sum(1).mean()))


# ---- the 3000-atom water box ------------------------------------------------------------------

def test_water3000_snapshot_bit_exact_list_gr_and_forces():
    g = golden("water3000.npz")
    s, table = cases.water3000_case()
    np.testing.assert_array_equal(s.x, g["x"])
    for exact in (True, False):
        e, (F, U) = engine_for(s, table, exact=exact, bonded=water_rows())
        e.list_build()
        info = e.list_info()
        assert info["nghost"] == int(g["nghost"])
        counts, digests = cases.list_keys(e.list_records(), s.natom)
        np.testing.assert_array_equal(counts, g["list_counts"])
        np.testing.assert_array_equal(digests, g["list_digests"])
        erg, vir = e.compute_forces(ev=True)
        f = e.forces()
        assert cases.rel_rms(f, g["force"]) < FORCE_RTOL
        f64, e64, w64 = fp64_classical(s, s.x, F, U, water_rows())
        assert cases.rel_rms(f, f64) < FORCE_RTOL
        assert abs(erg - e64) / abs(e64) < ENERGY_RTOL
        assert abs(vir - w64) / abs(w64) < ENERGY_RTOL
        e.gr_setup(1000, 512, 20.0)
        e.gr_tally(inner=False)
        np.testing.assert_array_equal(e.gr_counts(False).astype(np.int64), g["gr_counts"])
        e.gr_tally(inner=True)
        np.testing.assert_array_equal(e.gr_counts(True).astype(np.int64), g["gr_inner_counts"])
        e.close()


def test_water3000_100_steps_track_reference():
    """FP32 state in the reference's float sequence: 100 NVE steps at 1 fs from the lattice start
    with Maxwell-Boltzmann velocities. Two builds of the reference itself (27 and 8 threads, other
    summation orders) differ by 2e-5 A in position and 5e-5 in relative velocity RMS here; the
    trajectories separate chaotically after about 200 fs."""
    g = golden("water3000.npz")
    s, table = cases.water3000_case()
    e, _ = engine_for(s, table, v=s.v, exact=True, fp64=False, bonded=water_rows())
    log = e.run(101, log_interval=10)
    assert min_image_rms(e.positions(), g["md100_x"], s.bl) < 1e-3
    assert cases.rel_rms(e.velocities(), g["md100_v"]) < 1e-3
    np.testing.assert_allclose([r["erg"] for r in log], g["md100_erg"], rtol=1e-4)
    np.testing.assert_allclose([r["ekin"] for r in log], g["md100_ekin"], rtol=1e-4)
    assert abs(log[-1]["nbuild"] - int(g["md100_nbuild"])) <= 1
    e.close()


@pytest.mark.parametrize("fp64", [False, True])
def test_water3000_1000_steps_energy_statistics(fp64):
    """1000 NVE steps at 1 fs (the plain workload's run), FP32 state in the reference's sequence or
    FP64 state: the mean potential and kinetic energies over the last 500 fs within 2 % of the
    reference's, and the total-energy change over steps 100..1000 within twice the reference's plus
    10 kcal/mol. (Two builds of the reference agree to 0.5 % in the means; the lattice start
    releases about 4.5e3 kcal/mol in the first 100 fs.)"""
    g = golden("water3000.npz")
    s, table = cases.water3000_case()
    e, _ = engine_for(s, table, v=s.v, exact=not fp64, fp64=fp64, bonded=water_rows())
    log = e.run(1001, log_interval=10)
    erg = np.array([r["erg"] for r in log])
    ekin = np.array([r["ekin"] for r in log])
    assert len(erg) == len(g["md1000_erg"])
    assert e.device_errors() == 0
    ref_e, ref_k = g["md1000_erg"], g["md1000_ekin"]
    assert abs(erg[50:].mean() - ref_e[50:].mean()) < 0.02 * abs(ref_e[50:].mean())
    assert abs(ekin[50:].mean() - ref_k[50:].mean()) < 0.02 * abs(ref_k[50:].mean())
    d_ref = (ref_e + ref_k)[-1] - (ref_e + ref_k)[10]
    d_gpu = (erg + ekin)[-1] - (erg + ekin)[10]
    assert abs(d_gpu) < 2 * abs(d_ref) + 10.0
    e.close()


def _network_errors(s, x, m, table=None):
    """GPU network term (FP32 and BF16) against the FP64 oracle at positions x; with a table, the
    whole force (LJ/DSF + bonded + network) too."""
    from oracle import orc
    sx = S.System(**{**s.__dict__, "x": np.asarray(x, np.float32)})
    out = {}
    o6 = orc.Restated(sx, "f64")
    assert o6.rebuild(sx.x, 6, 2, 8) == 0
    r = o6.nnp_emb(6.0, m.scale, m.e1, m.e2, m.embw, m.h1, m.h2, m.fitw)
    e = Engine(0)
    e.set_system(sx)
    e.set_velocities(np.zeros_like(sx.v))
    e.setup(6.0, 2.0, 6.0, 2048)
    e.pair_enable(False)
    e.set_bonded(sx, [], [], [])
    e.nnp_set(m, 6.0, 750)
    for prec in ("fp32", "bf16"):
        e.nnp_precision(prec == "bf16")
        e.list_build()
        erg, _ = e.compute_forces(True)
        assert e.device_errors() == 0
        out[prec] = (cases.rel_rms(e.forces(), r["f"]), abs(erg - r["e_net"]) / abs(r["e_net"]))
    e.close()
    if table is not None:
        et, (F, U) = engine_for(sx, table, bonded=water_rows(), nnp=m)
        et.nnp_precision(False)
        et.list_build()
        erg, _ = et.compute_forces(True)
        f64, e64, _ = fp64_classical(sx, sx.x, F, U, water_rows())
        out["total_fp32"] = (cases.rel_rms(et.forces(), f64 + r["f"]), abs(erg - (e64 + r["e_net"])) / abs(e64 + r["e_net"]))
        et.close()
    return out


def test_water3000_equilibrated_network_vs_fp64():
    """The network workload's starting state: the reference's 5 ps at 1 fs under its Andersen
    thermostat at 300 K from the lattice start, then the radial-embedding network at 6 A."""
    g = golden("water3000.npz")
    s, table = cases.water3000_case()
    out = _network_errors(s, g["eq_x"], NM.embed_model(), table)
    print("3000-atom equilibrated state, rel. force / energy error vs FP64:", out)
    assert out["fp32"][0] < FORCE_RTOL and out["fp32"][1] < ENERGY_RTOL
    assert out["total_fp32"][0] < FORCE_RTOL and out["total_fp32"][1] < ENERGY_RTOL
    assert out["bf16"][0] < BF16_FORCE_BAR and out["bf16"][1] < BF16_FORCE_BAR


def test_water96k_network_error_vs_fp64():
    """The 96,000-atom box of the headline workload (lattice start, atoms displaced by N(0, 0.05 A)
    so that every pair distance is off the lattice's): the BF16 tensor-core network within 1 % of
    the FP64 force RMS, the FP32 network within 1e-5."""
    s = S.water_box(32, 99.3, seed=2, nmol=32000)
    rng = np.random.default_rng(77)
    x = (s.x + rng.normal(0, 0.05, s.x.shape)).astype(np.float32)
    out = _network_errors(s, x, NM.embed_model())
    print("96k atoms, rel. force / energy error vs FP64:", out)
    assert out["fp32"][0] < FORCE_RTOL and out["fp32"][1] < ENERGY_RTOL
    assert out["bf16"][0] < BF16_FORCE_BAR and out["bf16"][1] < BF16_FORCE_BAR


# ---- the 30,000-atom liquid -------------------------------------------------------------------

def test_mixture30k_bit_exact_list_and_gr_counts():
    g = golden("mixture30k.npz")
    s, table = cases.mixture30k_case()
    assert cases.x_digest(s.x) == g["x_digest"]
    e, (F, U) = engine_for(s, table, gr_cutoff=15.0)
    e.list_build()
    assert e.list_info()["nghost"] == int(g["nghost"])
    counts, digests = cases.list_keys(e.list_records(), s.natom)
    np.testing.assert_array_equal(counts, g["list_counts"])
    np.testing.assert_array_equal(cases.block_digests(digests), g["list_block_digests"])
    e.gr_setup(1000, 512, 20.0)
    e.gr_tally(inner=False)
    np.testing.assert_array_equal(e.gr_counts(False).astype(np.int64), g["gr_counts"])
    e.gr_tally(inner=True)
    np.testing.assert_array_equal(e.gr_counts(True).astype(np.int64), g["gr_inner_counts"])
    erg, _ = e.compute_forces(ev=True)
    f64, e64, _ = fp64_classical(s, s.x, F, U, ([np.zeros(4, np.float32)], [np.zeros(4, np.float32)]))
    assert cases.rel_rms(e.forces(), f64) < FORCE_RTOL
    assert abs(erg - e64) / abs(e64) < ENERGY_RTOL
    e.close()


# ---- dihedrals --------------------------------------------------------------------------------

def test_peroxide_dihedral_parity():
    g = golden("peroxide2048.npz")
    s, table = cases.peroxide_case()
    np.testing.assert_array_equal(s.x, g["x"])
    b, a, d = cases.peroxide_coefs()
    e, (F, U) = engine_for(s, table, bonded=(b, a, d))
    e.list_build()
    erg, vir = e.compute_forces(ev=True)
    assert cases.rel_rms(e.forces(), g["force"]) < FORCE_RTOL
    f64, e64, w64 = fp64_classical(s, s.x, F, U, (b, a), d)
    assert cases.rel_rms(e.forces(), f64) < FORCE_RTOL
    assert abs(erg - e64) / abs(e64) < ENERGY_RTOL
    assert abs(vir - w64) / abs(w64) < ENERGY_RTOL
    # the bonded terms alone, dihedral included
    e.pair_enable(False)
    erg_b, _ = e.compute_forces(ev=True)
    assert cases.rel_rms(e.forces(), g["f_bonded"]) < FORCE_RTOL
    assert abs(erg_b - g["erg_bonded"][0]) / abs(g["erg_bonded"][0]) < 1e-5
    e.close()
    # 20 NVE steps at 0.5 fs in the reference's float sequence
    e, _ = engine_for(s, table, v=s.v, exact=True, fp64=False, bonded=(b, a, d))
    e.verlet(0.5, False)
    log = e.run(21, log_interval=1)
    assert cases.rel_rms(e.positions(), g["md_x"]) < 1e-5
    assert cases.rel_rms(e.velocities(), g["md_v"]) < 1e-3
    np.testing.assert_allclose([r["erg"] for r in log], g["md_erg"], rtol=1e-4)
    e.close()


# ---- the network's forces are the gradient of its energy (GPU only) ---------------------------

def test_network_forces_are_gradient_of_gpu_energy():
    """Central differences of the GPU's own network energy (FP32 network, per-atom energies summed
    in FP64) against the GPU's forces, on 8 atoms x 3 directions of the jittered 648-atom water box:
    ties the hand-written backward to the forward without the oracle. The FP32 energy carries about
    2e-6 kcal/mol of rounding noise from evaluation to evaluation, so the step is 0.02 A, where a
    central difference resolves the forces (RMS 0.04 kcal/mol/A) to about 2e-3 of their RMS; a wrong
    term in the backward would be off by order one."""
    s, _ = cases.water_case(jitter=0.05)
    m = NM.embed_model()
    e = Engine(0)
    e.set_system(s)
    e.set_velocities(np.zeros_like(s.v))
    e.setup(6.0, 2.0, 6.0, 2048)
    e.pair_enable(False)
    e.set_bonded(s, [], [], [])
    e.nnp_set(m, 6.0, 750)
    e.nnp_precision(False)
    e.list_build()
    e.compute_forces(True)
    f0 = e.forces().astype(np.float64)
    frms = np.sqrt((f0 ** 2).sum(1).mean())
    rng = np.random.default_rng(3)
    h = np.float32(2e-2)
    worst = 0.0
    for a in rng.choice(s.natom, 8, replace=False):
        for dim in range(3):
            ep = []
            for sign in (1, -1):
                x = s.x.copy()
                x[a, dim] = np.float32(s.x[a, dim] + sign * h)
                e.set_positions(x)
                e.list_build()
                erg, _ = e.compute_forces(True)
                ep.append((erg, x[a, dim]))
            fd = -(ep[0][0] - ep[1][0]) / (float(ep[0][1]) - float(ep[1][1]))
            worst = max(worst, abs(fd - f0[a, dim]) / frms)
    print(f"finite difference vs forces: worst {worst:.2e} of the force RMS {frms:.3f}")
    assert worst < 5e-3
    e.close()
