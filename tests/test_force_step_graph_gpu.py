"""nnpe_force_step runs its device part as a cached CUDA graph. Changes made between calls (the pair
kernel's exact mode, the pair term switched off and on, energies requested or not) must reach the
next call: each call is compared bit for bit with the eager, allocation-free step of a second
context that was set up the same way and changed the same way."""
import ctypes as C

import numpy as np
import pytest

import cases
from nnpengine_b200 import engine as E

pytestmark = pytest.mark.gpu


def _engine(s, table):
    F, U = cases.table_as_loaded(table[1], table[2])
    e = E.Engine(0)
    e.set_system(s)
    e.setup(10.0, 2.0, 10.0, 2048)
    e.set_pair_table(F, U)
    e.set_bonded(s, [E.bond_coef(1.0, 0, 0, cases.WATER_BOND_K)], [E.angle_coef(109.47, 0, 0, cases.WATER_ANGLE_KC)])
    return e


def _step(e, fn, x, ev):
    f = np.zeros_like(x)
    erg, vir = C.c_double(0), C.c_double(0)
    rc = fn(e.h, x.ctypes.data, f.ctypes.data, C.byref(erg) if ev else None, C.byref(vir) if ev else None)
    assert rc == 0, e.lib.nnpe_last_error(e.h)
    return f, erg.value, vir.value


def test_graph_force_step_follows_changes_between_calls():
    s, table = cases.water_case(jitter=0.05)
    g, ref = _engine(s, table), _engine(s, table)
    x0 = np.ascontiguousarray(s.x, np.float32)
    rng = np.random.default_rng(5)
    changes = [
        lambda e: None,
        lambda e: e.pair_exact(True),
        lambda e: None,
        lambda e: e.pair_exact(False),
        lambda e: e.pair_enable(False),
        lambda e: e.pair_enable(True),
    ]
    # positions per call: calls 0-1 share one set (fast vs exact pair math), calls 3-5 another
    # (exact off, pair term off, back on)
    xa = (x0 + rng.normal(0, 0.01, x0.shape)).astype(np.float32)
    xb = (x0 + rng.normal(0, 0.01, x0.shape)).astype(np.float32)
    xs = [xa, xa, (x0 + rng.normal(0, 0.01, x0.shape)).astype(np.float32), xb, xb, xb]
    seen = []
    for k, change in enumerate(changes):
        change(g)
        change(ref)
        x = xs[k]
        ev = k % 2 == 1
        fg, eg, vg = _step(g, g.lib.nnpe_force_step, x, ev)
        fr, er, vr = _step(ref, ref.lib.nnpe_force_step_noalloc, x, ev)
        np.testing.assert_array_equal(fg, fr)
        assert eg == er and vg == vr
        seen.append(fg)
    # the changes did change the forces: exact vs fast pair math (rounding), and no pair term at all
    assert not np.array_equal(seen[0], seen[1])
    assert np.abs(seen[4] - seen[5]).max() > 1.0
    np.testing.assert_array_equal(seen[3], seen[5])
