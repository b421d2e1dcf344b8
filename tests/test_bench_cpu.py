"""Host-side checks of the bench's reference arm, of its clock sampler (against a stand-in for
nvidia-smi) and of the coefficient rows the tests build."""
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



FAKE_SMI = """#!%s
import time
time.sleep(0.3)   # the real tool's start-up delay
while True:
    print("0, 1965, 1965, 500.0, 0x0, Not Active, Not Active, Not Active, %s", flush=True)
    time.sleep(0.05)
"""


def _fake_smi(tmp_path, power_cap=False):
    """A stand-in for nvidia-smi's query loop (clocks at max; sw_power_cap active or not)."""
    p = tmp_path / "nvidia-smi"
    p.write_text(FAKE_SMI % (sys.executable, "Active" if power_cap else "Not Active"))
    p.chmod(0o755)
    return str(tmp_path)


def test_clock_sampler_covers_short_and_long_timed_regions(tmp_path, monkeypatch):
    """A timed region shorter than the sampler's interval (the default 20-step run) still gets
    the samples next to it; a long one gets its own samples."""
    import time
    import bench
    monkeypatch.setenv("PATH", _fake_smi(tmp_path) + os.pathsep + os.environ["PATH"])
    for region_s in (0.02, 0.6):
        with bench.ClockSampler(0) as c:
            time.sleep(region_s)
        s = c.summary()
        assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0 and s["reasons"] == []
        assert s["samples"] >= 2
        assert ("note" in s) == (region_s < 0.1)


def test_clock_sampler_reports_an_active_reason(tmp_path, monkeypatch):
    import time
    import bench
    monkeypatch.setenv("PATH", _fake_smi(tmp_path, power_cap=True) + os.pathsep + os.environ["PATH"])
    with bench.ClockSampler(0) as c:
        time.sleep(0.02)
    assert c.summary()["reasons"] == ["sw_power_cap"]
