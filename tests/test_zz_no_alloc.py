"""nnpe_force_step_noalloc (static staging, no device allocation) against nnpe_force_step on the
same system and positions, through the C ABI."""
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


def _step(e, fn, x):
    f = np.zeros_like(x)
    erg, vir = C.c_double(0), C.c_double(0)
    rc = fn(e.h, x.ctypes.data, f.ctypes.data, C.byref(erg), C.byref(vir))
    return rc, f, erg.value, vir.value


def _device_bytes(e):
    b = C.c_int64(0)
    assert e.lib.nnpe_device_bytes(e.h, C.byref(b)) == 0
    return b.value


def test_force_step_noalloc_matches_force_step():
    s, table = cases.water_case(jitter=0.05)
    ref, stat = _engine(s, table), _engine(s, table)
    x1 = np.ascontiguousarray(s.x, np.float32)
    x2 = (x1 + np.random.default_rng(11).normal(0, 0.02, x1.shape)).astype(np.float32)
    bytes_before = _device_bytes(stat)
    for x in (x1, x2):   # two calls in a row on each context
        rc_a, fa, ea, va = _step(ref, ref.lib.nnpe_force_step, x)
        rc_b, fb, eb, vb = _step(stat, stat.lib.nnpe_force_step_noalloc, x)
        assert rc_a == 0, ref.lib.nnpe_last_error(ref.h)
        assert rc_b == 0, stat.lib.nnpe_last_error(stat.h)
        np.testing.assert_array_equal(fa, fb)
        assert ea == eb and va == vb
        assert np.abs(fb).max() > 0
    # the point of the entry point: the context's device-byte ledger did not move, while the
    # allocating step's context grew by its two staging buffers
    assert _device_bytes(stat) == bytes_before
    assert _device_bytes(ref) >= bytes_before + 2 * 4 * 3 * s.natom


def test_force_step_noalloc_rejects_systems_over_its_limit():
    s, _ = cases.mixture_case(140000, 0.035)
    e = E.Engine(0)
    e.set_system(s)
    x = np.zeros((s.natom, 3), np.float32)
    f = np.zeros_like(x)
    rc = e.lib.nnpe_force_step_noalloc(e.h, x.ctypes.data, f.ctypes.data, None, None)
    assert rc == 1   # NNPE_EARG
    assert b"131072" in e.lib.nnpe_last_error(e.h)
