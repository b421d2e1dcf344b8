"""nnpe_force_step with host-owned coordinates that the host never folds into the box: the library
folds its own copy at each list build, and the host's positions must keep mapping onto that copy
(no list rebuild on every call once an atom has crossed a face, forces equal to those of the folded
coordinates)."""
import dataclasses

import numpy as np
import pytest

import cases
from nnpengine_b200 import engine as E

pytestmark = pytest.mark.gpu


def _engine(s, table, x=None):
    F, U = cases.table_as_loaded(table[1], table[2])
    e = E.Engine(0)
    if x is not None:
        s = dataclasses.replace(s, x=np.ascontiguousarray(x, np.float32))
    e.set_system(s)
    e.setup(10.0, 2.0, 10.0, 2048)
    e.set_pair_table(F, U)
    e.set_bonded(s, [E.bond_coef(1.0, 0, 0, cases.WATER_BOND_K)], [E.angle_coef(109.47, 0, 0, cases.WATER_ANGLE_KC)])
    return e


def _forces(e, x):
    f = np.zeros_like(x)
    rc = e.lib.nnpe_force_step(e.h, x.ctypes.data, f.ctypes.data, None, None)
    assert rc == 0, e.lib.nnpe_last_error(e.h)
    return f


def test_unfolded_host_coordinates_across_faces():
    s, table = cases.water_case(jitter=0.05)
    bl = float(s.bl)
    x0 = np.ascontiguousarray(s.x, np.float32)
    rng = np.random.default_rng(21)
    u = rng.normal(size=x0.shape)
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    e = _engine(s, table)
    nb0 = None
    checked = 0
    for k in range(40):
        x = (x0 + np.float32(0.06 * k) * u.astype(np.float32)).astype(np.float32)   # never folded
        f = _forces(e, x)
        if k == 0:
            nb0 = e.list_info()["nbuild"]
        if k in (10, 25, 39):
            xf = (x - bl * np.rint(x / bl)).astype(np.float32)
            ref = _engine(s, table, x=xf)
            assert cases.rel_rms(f, _forces(ref, xf)) < 1e-5
            checked += 1
    crossed = np.any(np.abs(x) > bl / 2, axis=1).sum()
    assert crossed > 0                              # some atoms left the box in host coordinates
    builds = e.list_info()["nbuild"] - nb0
    assert 1 <= builds <= 6, builds                 # 2.3 A of motion per atom at 1 A per build, not one per call
    assert checked == 3
