"""Dynamic pruning of the neighbour list: the pair and network kernels read a copy of the list that
keeps the entries within the force cutoff + delta, remade after every rebuild and whenever an atom
has moved delta/2 since the copy was made. The pairs that interact are those of the full list, so
forces with and without pruning differ only by the order of the FP32 sums (the network's pair list
is the same, entry for entry)."""
import dataclasses

import numpy as np
import pytest

import cases
from nnpengine_b200 import engine as E
from nnpengine_b200 import nnp_model as NM

pytestmark = pytest.mark.gpu

SUM_ORDER_RTOL = 1e-6   # FP32 per-atom sums over the same pairs in another order


def _water(s, table, delta, fp64=True, nnp=None):
    F, U = cases.table_as_loaded(table[1], table[2])
    e = E.Engine(0)
    e.set_system(s)
    e.setup(10.0, 2.0, 10.0, 2048)
    e.set_pair_table(F, U)
    e.set_bonded(s, [E.bond_coef(1.0, 0, 0, cases.WATER_BOND_K)], [E.angle_coef(109.47, 0, 0, cases.WATER_ANGLE_KC)])
    if nnp is not None:
        e.nnp_set(nnp, 6.0, 750)
        e.nnp_precision(False)
    e.verlet(1.0, fp64)
    e.set_prune(delta)
    return e


def _min_image(d, bl):
    return d - np.rint(d / bl) * bl


def test_default_is_on_and_switches():
    s, table = cases.water_case()
    e = _water(s, table, 0.5)
    assert e.prune_info()["active"] and abs(e.prune_info()["delta"] - 0.5) < 1e-7
    e.set_prune(0.0)
    assert not e.prune_info()["active"]
    e.set_prune(2.5)                                  # not below the 2 A skin: off
    assert not e.prune_info()["active"]
    e.set_prune(0.5)
    assert e.prune_info()["active"]
    e.close()


def test_md_with_pruning_remakes_the_copy_and_keeps_the_forces():
    """300 steps at 1 fs from 300 K: the copy is remade more often than the list is rebuilt (0.25 A
    against 1 A of motion), and at the end the forces over the copy equal those over the full list
    to FP32 summation order; the energies and virial (FP64 per pair) agree closely."""
    s, table = cases.water3000_case()
    e = _water(s, table, 0.5)
    e.run(300, log_interval=300, graph=True)
    info, lst = e.prune_info(), e.list_info()
    assert info["active"] and info["nprune"] > lst["nbuild"] >= 1, (info, lst)
    erg1, vir1 = e.compute_forces(True)
    f1 = e.forces()
    e.set_prune(0.0)
    erg0, vir0 = e.compute_forces(True)
    f0 = e.forces()
    assert e.device_errors() == 0
    assert cases.rel_rms(f1, f0) < SUM_ORDER_RTOL
    assert abs(erg1 - erg0) < 1e-9 * abs(erg0) and abs(vir1 - vir0) < 1e-9 * abs(vir0)
    e.close()


def test_trajectory_with_and_without_pruning():
    """200 steps with and without pruning from the same state: the two runs differ only by FP32
    summation order in the forces, which the dynamics amplifies; they stay within the 1e-3 A RMS
    that the GPU keeps against the reference's own trajectory over 100 steps."""
    s, table = cases.water3000_case()
    a = _water(s, table, 0.5)
    b = _water(s, table, 0.0)
    la = a.run(200, log_interval=100, graph=True)
    lb = b.run(200, log_interval=100, graph=True)
    assert a.prune_info()["nprune"] > 1 and b.prune_info()["nprune"] == 0
    d = _min_image(a.positions(f64=True) - b.positions(f64=True), float(s.bl))
    assert np.sqrt((d ** 2).sum(1).mean()) < 1e-3
    for ra, rb in zip(la, lb):
        assert abs(ra["erg"] - rb["erg"]) < 1e-5 * abs(rb["erg"])
    a.close()
    b.close()


def test_host_positions_trigger_the_copy():
    """nnpe_force_step: a displacement past delta/2 (0.3 A) but short of skin/2 remakes the copy
    without a rebuild, and the forces still equal those over the full list."""
    s, table = cases.water_case(jitter=0.05)
    x0 = np.ascontiguousarray(s.x, np.float32)
    a = _water(s, table, 0.5, fp64=False)
    b = _water(s, table, 0.0, fp64=False)

    def step(e, x):
        f = np.zeros_like(x)
        assert e.lib.nnpe_force_step(e.h, x.ctypes.data, f.ctypes.data, None, None) == 0, e.lib.nnpe_last_error(e.h)
        return f

    step(a, x0)
    step(b, x0)
    n0, nb0 = a.prune_info()["nprune"], a.list_info()["nbuild"]
    rng = np.random.default_rng(5)
    u = rng.normal(size=x0.shape)
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    x1 = (x0 + np.float32(0.3) * u.astype(np.float32)).astype(np.float32)
    fa, fb = step(a, x1), step(b, x1)
    assert a.list_info()["nbuild"] == nb0                 # no rebuild at 0.3 A
    assert a.prune_info()["nprune"] == n0 + 1             # the copy was remade
    assert cases.rel_rms(fa, fb) < SUM_ORDER_RTOL
    x2 = (x1 + np.float32(0.1) * u.astype(np.float32)).astype(np.float32)
    fa, fb = step(a, x2), step(b, x2)
    assert a.prune_info()["nprune"] == n0 + 1             # 0.1 A since the copy: kept
    assert cases.rel_rms(fa, fb) < SUM_ORDER_RTOL
    a.close()
    b.close()


def test_network_pairs_unchanged_by_pruning():
    """With the network on, its pair list is compacted from the copy in list order: the same entries
    in the same order as from the full list, so the FP32 network forces are bit-identical."""
    s, table = cases.water_case(jitter=0.05)
    m = NM.embed_model()
    a = _water(s, table, 0.5, nnp=m)
    a.run(50, log_interval=50, graph=True)
    x = a.positions()
    a.pair_enable(False)
    a.compute_forces(False)
    fa = a.forces()
    a.set_prune(0.0)
    a.compute_forces(False)
    fb = a.forces()
    assert a.device_errors() == 0
    np.testing.assert_array_equal(fa, fb)
    assert np.isfinite(x).all()
    a.close()
