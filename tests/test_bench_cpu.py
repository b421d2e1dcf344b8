"""Host-side checks of the bench's reference arm and of the coefficient rows the tests build."""
import os
import subprocess
import sys

import numpy as np
import pytest

import cases
from oracle import orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not os.path.exists(os.path.join(orc.REF_DIR, "ref_dump_fast8")), reason="reference harness not built")
def test_reference_arm_process_loads_no_product_library():
    """The reference arm times the reference's own code: its process maps the oracle's harness
    binaries only, never this project's libnnpe.so."""
    code = ("import sys; sys.path.insert(0, %r); import bench; "
            "r = bench.cpu_reference(bench.WORKLOADS['water3k-classical'], 5); "
            "maps = open('/proc/self/maps').read(); "
            "print('LOADED' if 'libnnpe' in maps else 'CLEAN', r[0] > 0, len(r[3]))") % ROOT
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    assert out.stdout.split() == ["CLEAN", "True", "2"], out.stdout


def test_coefficient_rows_match_the_library_setparam():
    """cases' numpy setParam transforms give the library's rows bit for bit (nnpe_*_coef)."""
    from nnpengine_b200 import engine as E
    for t, kc in ((109.47, 62.0), (100.0, 50.0), (120.0, 1.5)):
        np.testing.assert_array_equal(cases.angle_row(t, 0.25, 0.5, kc), E.angle_coef(t, 0.25, 0.5, kc))
    np.testing.assert_array_equal(cases.bond_row(1.45, 2.0, 0.5, 300.0), E.bond_coef(1.45, 2.0, 0.5, 300.0))
    np.testing.assert_array_equal(cases.dihedral_row(*cases.PEROXIDE_DIHEDRAL), E.dihedral_coef(*cases.PEROXIDE_DIHEDRAL))
