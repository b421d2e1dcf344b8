"""Network term on the GPU: the reference's tabulated NNP against its own C++ (golden vectors),
the embedding network against the FP64 oracle, and the BF16 tensor-core form's stated error."""
import os

import numpy as np
import pytest

import cases
from nnpengine_b200 import engine as E
from nnpengine_b200 import nnp_model as NM
from nnpengine_b200.engine import Engine

pytestmark = pytest.mark.gpu


def nnp_engine(s, model=None, files=None, lj_table=None, cutoff=6.0, nbin=750):
    e = Engine(0)
    e.set_system(s)
    e.set_velocities(np.zeros_like(s.v))
    if lj_table is not None:
        e.setup(10.0, 2.0, 10.0, 2048)
        e.set_pair_table(*lj_table)
    else:
        e.setup(cutoff, 2.0, cutoff, 2048)
        e.pair_enable(False)
    b, a, d = cases.water_bonded_raw()
    e.set_bonded(s, [b[0] * np.array([1, 2, 1, 2], np.float32)], [a[0] * np.array([1, 2, 1, 2], np.float32)], [d[0]])
    if files is not None:
        e.nnp_load(cutoff, nbin, files["param"], files["wt"])
    else:
        e.nnp_set(model, cutoff, nbin)
    return e


def test_gauss_nnp_matches_reference(tmp_path):
    g = np.load(os.path.join(cases.GOLDEN, "nnp_gauss648.npz"))
    s, _ = cases.water_case()
    m = NM.gauss_model()
    files = cases.write_nnp_inputs(m, str(tmp_path))
    e = nnp_engine(s, files=files)
    e.list_build()
    erg, vir = e.compute_forces(True)
    G, dG, ea = e.nnp_get()
    np.testing.assert_allclose(G, g["desc"], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(dG, g["dedg"], rtol=1e-4, atol=1e-6)
    assert abs(ea.sum() - g["enn"][0]) / abs(g["enn"][0]) < 1e-5
    assert cases.rel_rms(e.forces(), g["force"]) < 1e-5


def test_embed_nnp_fp32_matches_fp64_oracle():
    from oracle import orc
    s, table = cases.water_case(jitter=0.05)
    m = NM.embed_model()
    e = nnp_engine(s, model=m)
    e.list_build()
    erg, vir = e.compute_forces(True)
    G, dG, ea = e.nnp_get()
    o = orc.Restated(s, "f64")
    assert o.rebuild(s.x, 6, 2, 8) == 0
    r = o.nnp_emb(6.0, m.scale, m.e1, m.e2, m.embw, m.h1, m.h2, m.fitw)
    assert cases.rel_rms(G, r["G"]) < 1e-5
    assert cases.rel_rms(dG, r["dEdG"]) < 1e-4
    assert abs(ea.sum() - r["e_net"]) / abs(r["e_net"]) < 1e-5
    fb, _, _ = o.bonded(*[x * np.array([1, 2, 1, 2], np.float32) for x in cases.water_bonded_raw()[:2]],
                        np.zeros((1, 4), np.float32))
    f = e.forces()
    assert cases.rel_rms(f, r["f"] + fb) < 1e-5


def test_embed_nnp_plus_lj_composed():
    """Tabulated LJ/Coulomb at 10 A plus the network at 6 A on one 12 A list."""
    from oracle import orc
    s, table = cases.water_case(jitter=0.05)
    F, U = cases.table_as_loaded(table[1], table[2])
    m = NM.embed_model()
    e = nnp_engine(s, model=m, lj_table=(F, U))
    e.list_build()
    erg, vir = e.compute_forces(True)
    o = orc.Restated(s, "f64")
    assert o.rebuild(s.x, 10, 2, 12) == 0
    fp, ep, wp = o.pair_forces(F, U, 10.0)
    r = o.nnp_emb(6.0, m.scale, m.e1, m.e2, m.embw, m.h1, m.h2, m.fitw)
    fb, eb, wb = o.bonded(*[x * np.array([1, 2, 1, 2], np.float32) for x in cases.water_bonded_raw()[:2]],
                          np.zeros((1, 4), np.float32))
    ref = fp + r["f"] + fb
    assert cases.rel_rms(e.forces(), ref) < 1e-5
    assert abs(erg - (ep + r["e_net"] + eb)) / abs(ep + r["e_net"] + eb) < 1e-5


def _bf16_vs_fp64(s, m, e):
    from oracle import orc
    o = orc.Restated(s, "f64")
    assert o.rebuild(s.x, 6, 2, 8) == 0
    r = o.nnp_emb(6.0, m.scale, m.e1, m.e2, m.embw, m.h1, m.h2, m.fitw)
    G, dG, ea = e.nnp_get()
    return r, G, dG, ea


def test_embed_nnp_bf16_tensor_core_error_vs_fp64():
    """BF16 operands on tcgen05 (FP32 accumulate): network force RMSE within 1% of the force RMS
    against the FP64 oracle (the stated bar), descriptor and energy errors reported the same way."""
    s, _ = cases.water_case(jitter=0.05)
    m = NM.embed_model()
    e = nnp_engine(s, model=m)
    e.pair_enable(False)
    e.set_bonded(s, [], [], [])
    e.nnp_precision(True)
    e.list_build()
    erg, vir = e.compute_forces(True)
    assert e.device_errors() == 0
    r, G, dG, ea = _bf16_vs_fp64(s, m, e)
    f = e.forces()
    err_G = cases.rel_rms(G, r["G"])
    err_dG = cases.rel_rms(dG, r["dEdG"])
    err_f = cases.rel_rms(f, r["f"])
    err_e = abs(ea.sum() - r["e_net"]) / abs(r["e_net"])
    print(f"BF16 vs FP64: G {err_G:.2e} dE/dG {err_dG:.2e} force {err_f:.2e} energy {err_e:.2e}")
    assert err_G < 1e-2
    assert err_dG < 3e-2
    assert err_f < 1e-2
    assert err_e < 1e-2


def test_embed_nnp_bf16_deterministic():
    s, _ = cases.water_case(jitter=0.05)
    m = NM.embed_model()
    e = nnp_engine(s, model=m)
    e.nnp_precision(True)
    e.list_build()
    e.compute_forces(True)
    f1 = e.forces().copy()
    e.compute_forces(True)
    np.testing.assert_array_equal(e.forces(), f1)


def test_embed_nnp_bf16_md_steps():
    """A few MD steps on the tensor-core path: finite, no device errors, graph replay matches."""
    s, table = cases.water_case(jitter=0.05)
    F, U = cases.table_as_loaded(table[1], table[2])
    m = NM.embed_model()
    logs = []
    for graph in (False, True):
        e = nnp_engine(s, model=m, lj_table=(F, U))
        e.set_velocities(s.v)
        e.nnp_precision(True)
        e.verlet(0.5, True)
        logs.append((e.run(20, log_interval=5, graph=graph), e.positions(f64=True)))
        assert e.device_errors() == 0
    assert all(np.isfinite(r["erg"]) for r in logs[0][0])
    np.testing.assert_array_equal(logs[0][1], logs[1][1])


@pytest.mark.parametrize("rho", [0.003, 0.2])
def test_embed_nnp_bf16_sparse_and_dense_pair_counts(rho):
    """The tensor-core kernels cut each CTA's pairs into tiles of up to two atom segments: a dilute
    mixture (most atoms have no neighbour inside 6 A, tiles hold one or two short segments) and a
    dense one (about 180 neighbours, an atom's pairs span two or three tiles) both reproduce the
    FP64 oracle within the BF16 bar, and atoms without pairs get a zero descriptor."""
    from nnpengine_b200 import systems as S
    s = S.lj_mixture(600, rho, 0.6, seed=5)
    m = NM.embed_model()
    e = Engine(0)
    e.set_system(s)
    e.set_velocities(np.zeros_like(s.v))
    e.setup(6.0, 2.0, 6.0, 2048)
    e.pair_enable(False)
    e.nnp_set(m, 6.0, 750)
    e.nnp_precision(True)
    e.list_build()
    e.compute_forces(True)
    assert e.device_errors() == 0
    r, G, dG, ea = _bf16_vs_fp64(s, m, e)
    lone = np.all(r["G"] == 0, axis=1)
    if rho < 0.01:
        assert lone.sum() > 100
    else:
        assert not lone.any()
    assert np.all(G[lone] == 0)
    assert cases.rel_rms(G, r["G"]) < 1e-2
    assert cases.rel_rms(e.forces(), r["f"]) < 1e-2
    e.compute_forces(True)   # deterministic
    G2, _, _ = e.nnp_get()
    np.testing.assert_array_equal(G, G2)


def test_autotuned_grids_same_bits_for_same_grid_and_bf16_bar_across_grids():
    """The grid autotuner picks grid sizes among its candidates; a second context given the same grids
    reproduces the forces bit for bit, and the default grids agree to well inside the BF16 bar."""
    s, _ = cases.water_case(jitter=0.05)
    m = NM.embed_model()
    tuned = nnp_engine(s, model=m)
    tuned.set_bonded(s, [], [], [])   # the network term alone, as the FP64 oracle has it
    tuned.nnp_precision(True)
    gd, gf = tuned.nnp_autotune(reps=2, use_cache=False)
    sms = 148
    assert 1 <= gd <= min(s.natom, 4 * sms) and 1 <= gf <= min(s.natom, 2 * sms)
    assert tuned.nnp_get_grids() == (gd, gf)
    tuned.compute_forces(True)
    f_tuned = tuned.forces().copy()
    fixed = nnp_engine(s, model=m)
    fixed.set_bonded(s, [], [], [])
    fixed.nnp_precision(True)
    fixed.nnp_grids(gd, gf)
    fixed.list_build()
    fixed.compute_forces(True)
    np.testing.assert_array_equal(fixed.forces(), f_tuned)
    default = nnp_engine(s, model=m)
    default.set_bonded(s, [], [], [])
    default.nnp_precision(True)
    default.list_build()
    default.compute_forces(True)
    assert default.nnp_get_grids() == (min(s.natom, 4 * sms), min(s.natom, 2 * sms))
    assert cases.rel_rms(default.forces(), f_tuned) < 2e-3
    r, _, _, _ = _bf16_vs_fp64(s, m, fixed)
    assert cases.rel_rms(f_tuned, r["f"]) < 1e-2
    for e in (tuned, fixed, default):
        assert e.device_errors() == 0


@pytest.mark.parametrize("rho", [0.003, 0.2])
def test_embed_nnp_fp32_sparse_and_dense_pair_counts(rho):
    """The FP32 kernels take each atom's pairs species by species in ballot-compacted chunks of up to
    32 (the force kernel in groups of 16): a dilute mixture (most atoms without a pair inside 6 A)
    and a dense one (about 180 pairs per atom, several chunks per species) both match the FP64
    oracle at the plain form's bars, and atoms without pairs get a zero descriptor."""
    from nnpengine_b200 import systems as S
    s = S.lj_mixture(600, rho, 0.6, seed=5)
    m = NM.embed_model()
    e = Engine(0)
    e.set_system(s)
    e.set_velocities(np.zeros_like(s.v))
    e.setup(6.0, 2.0, 6.0, 2048)
    e.pair_enable(False)
    e.nnp_set(m, 6.0, 750)
    e.nnp_precision(False)
    e.list_build()
    erg, _ = e.compute_forces(True)
    assert e.device_errors() == 0
    r, G, dG, ea = _bf16_vs_fp64(s, m, e)
    lone = np.all(r["G"] == 0, axis=1)
    if rho < 0.01:
        assert lone.sum() > 100
    else:
        assert not lone.any()
    assert np.all(G[lone] == 0)
    assert cases.rel_rms(G, r["G"]) < 1e-5
    assert cases.rel_rms(e.forces(), r["f"]) < 1e-5
    assert abs(ea.sum() - r["e_net"]) < 1e-5 * abs(r["e_net"])
    e.compute_forces(True)   # deterministic
    np.testing.assert_array_equal(e.nnp_get()[0], G)
