"""ENVIRON::verify_grid (environ.cpp:638-683) ported: the checker on host arrays with planted
mistakes (CPU), and the device's own cell sort after list builds (GPU)."""
import ctypes as C

import numpy as np
import pytest

import cases
from nnpengine_b200 import _lib


def _grid(bl, cutoff=10.0, skin=2.0):
    # the grid constants in float, as nnpe_setup derives them (run.cpp:76-79, environ.cpp:143-155)
    f = np.float32
    comm = f(skin) + f(cutoff)
    g_dx = f(f(0.5) * (f(skin) + f(cutoff)))
    g_rdx = f(1) / g_dx
    g_offset = comm + f(f(bl) * f(0.5))
    num_gx = int(np.ceil(np.float64(f(g_offset * f(2)) * g_rdx)))
    return g_offset, g_rdx, num_gx


def _cell(x, g_offset, g_rdx, num_gx):
    a = ((np.float32(g_offset) + x.astype(np.float32)).astype(np.float32) * np.float32(g_rdx)).astype(np.float32)
    a = np.trunc(a).astype(np.int64)
    return (a[:, 0] * num_gx * num_gx + a[:, 1] * num_gx + a[:, 2]).astype(np.int32)


def _sorted_system(n=400, bl=20.0, seed=3):
    rng = np.random.default_rng(seed)
    g_offset, g_rdx, num_gx = _grid(bl)
    x = rng.uniform(-bl / 2, bl / 2, (n, 3)).astype(np.float32)
    near = np.where(x[:, 0] > bl / 2 - 12)[0]                    # images of the atoms near +x
    img = (x[near] - np.array([bl, 0, 0], np.float32)).astype(np.float32)
    cr, ci = _cell(x, g_offset, g_rdx, num_gx), _cell(img, g_offset, g_rdx, num_gx)
    orr, oi = np.argsort(cr, kind="stable"), np.argsort(ci, kind="stable")
    pos = np.zeros((n + len(img), 4), np.float32)
    pos[:n, :3], pos[n:, :3] = x[orr], img[oi]
    cell = np.concatenate([cr[orr], ci[oi]]).astype(np.int32)
    NG = num_gx ** 3
    cnt, gcnt = np.bincount(cr, minlength=NG), np.bincount(ci, minlength=NG)
    cend = np.cumsum(cnt).astype(np.int32)
    cstart = (cend - cnt).astype(np.int32)
    gcend = (n + np.cumsum(gcnt)).astype(np.int32)
    gcstart = (gcend - gcnt).astype(np.int32)
    return dict(natom=n, nimage=len(img), num_gx=num_gx, g_offset=g_offset, g_rdx=g_rdx, cstart=cstart,
                cend=cend, gcstart=gcstart, gcend=gcend, cell=cell, pos=pos)


def _verify(d):
    lib = _lib.load()
    bad, what = C.c_int64(0), C.c_int(0)
    rc = lib.nnpe_verify_grid_arrays(d["natom"], d["nimage"], d["num_gx"], float(d["g_offset"]), float(d["g_rdx"]),
                                     d["cstart"], d["cend"], d["gcstart"], d["gcend"], d["cell"],
                                     np.ascontiguousarray(d["pos"]), C.byref(bad), C.byref(what))
    return rc, what.value, bad.value


def test_verify_grid_accepts_a_correct_sort_and_finds_planted_mistakes():
    d = _sorted_system()
    assert _verify(d) == (0, 0, -1)
    n = d["natom"]
    # two real atoms of different cells swapped (positions and stored cells together)
    e = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    i, j = 0, n - 1
    assert e["cell"][i] != e["cell"][j]
    e["pos"][[i, j]] = e["pos"][[j, i]]
    e["cell"][[i, j]] = e["cell"][[j, i]]
    assert _verify(e)[:2] == (5, 4)
    # an atom moved across a cell boundary without a new sort
    e = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    e["pos"][3, 0] += np.float32(6.5)
    assert _verify(e) == (5, 5, 3)
    # ranges that do not start at 0 / natom, or are not contiguous
    e = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    e["gcstart"][0] += 1
    assert _verify(e)[:2] == (5, 1)
    e = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    k = int(np.nonzero(np.diff(e["cstart"]))[0][0])
    e["cend"][k] += 1
    assert _verify(e) == (5, 2, k + 1)


@pytest.mark.gpu
def test_device_cell_sort_passes_verify_grid():
    """The device's sort of real atoms and images satisfies verify_grid after a build: the water box
    at its start and after 100 steps of motion, and the two-species liquid."""
    from nnpengine_b200 import engine as E
    s, table = cases.water_case(jitter=0.05)
    F, U = cases.table_as_loaded(table[1], table[2])
    e = E.Engine(0)
    e.set_system(s)
    e.setup(10.0, 2.0, 10.0, 2048)
    e.set_pair_table(F, U)
    e.set_bonded(s, [E.bond_coef(1.0, 0, 0, cases.WATER_BOND_K)], [E.angle_coef(109.47, 0, 0, cases.WATER_ANGLE_KC)])
    e.verlet(1.0, True)
    e.list_build()
    e.verify_grid()
    e.run(100, log_interval=100, graph=True)
    e.list_build()
    e.verify_grid()
    assert e.device_errors() == 0
    e.close()
    s, table = cases.mixture_case()
    F, U = cases.table_as_loaded(table[1], table[2])
    e = E.Engine(0)
    e.set_system(s)
    e.setup(10.0, 2.0, 15.0, 2048)
    e.set_pair_table(F, U)
    e.list_build()
    e.verify_grid()
    assert e.device_errors() == 0
    e.close()
