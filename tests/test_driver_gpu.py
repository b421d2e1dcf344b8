"""The C++ run-file driver (nnpe_run, the reference's `classical` and `nnp_run` step loops on the
device) against the reference's own executable on the same input files.

Both runs start at 0 K, so their first log line (forces and energies of the starting
configuration, the kinetic energy after the first updateV, the RMDF penalty of the first g(r)
step) does not depend on the reference's unseeded random generator; later lines do (its Andersen
thermostat picks atoms at random), so for those the driver's log is checked for its form and the
output files for the reference's layout.
"""
import os
import subprocess

import numpy as np
import pytest

import cases
from nnpengine_b200 import build
from nnpengine_b200 import nnp_model as NM
from nnpengine_b200 import systems as S

pytestmark = pytest.mark.gpu

STRENGTH, GAMMA = 0.02, 0.5


def run_case(tmp_path, mode):
    d = str(tmp_path / mode)
    os.makedirs(d, exist_ok=True)
    s, table = cases.water_case()
    q, sqex, wt, ff = S.synthetic_sq_target(512, 20.0, 2, seed=7)
    tpath = os.path.join(d, "sq_target.txt")
    S.write_sq_target(tpath, q, sqex, wt, ff)
    if mode == "classical":
        path, files = cases.write_run_input(d, mode, s, table, rmdf=(STRENGTH, GAMMA, tpath))
    else:
        paths = cases.write_nnp_inputs(NM.gauss_model(), d)
        path, files = cases.write_run_input(d, mode, s, nnp_paths=paths, rmdf=(STRENGTH, GAMMA, tpath), nbin=750,
                                            cutoffs=(6.0, 2.0, 6.0))
    r = subprocess.run([build.DRIVER, mode, path, "--seed", "5", "--fp32-state"], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return cases.parse_log(r.stdout), files


@pytest.mark.parametrize("mode", ["classical", "nnp_run"])
def test_driver_first_log_line_matches_reference(tmp_path, mode):
    g = np.load(os.path.join(cases.GOLDEN, "driver648.npz"))
    log, files = run_case(tmp_path, mode)
    ref = g[f"{mode}_log"]
    assert log.shape == ref.shape                       # the same log steps
    np.testing.assert_array_equal(log[:, 0], ref[:, 0])
    step0, ref0 = log[0], ref[0]
    np.testing.assert_allclose(step0[1], ref0[1], rtol=1e-4)     # temperature after the first updateV
    np.testing.assert_allclose(step0[2], ref0[2], rtol=1e-4)     # pressure
    # potential energy: the reference sums it in float per thread; on this box its total of ~15
    # kcal/mol is the small difference of terms of ~1e4, and the float sums carry ~1e-3 of that
    np.testing.assert_allclose(step0[3], ref0[3], rtol=1e-5, atol=0.02)
    np.testing.assert_allclose(step0[4], ref0[4], rtol=1e-3)     # RMDF penalty (float vs FP64 S(q))
    assert step0[5] == ref0[5]                                   # list builds
    assert np.all(np.isfinite(log))
    lines = [sum(1 for _ in open(files[k])) if os.path.exists(files[k]) else 0
             for k in ("xyz", "gr", "sq", "sqx", "force")]
    np.testing.assert_array_equal(lines, g[f"{mode}_lines"])


def test_reference_style_loop_through_adapter_matches_step_loop(tmp_path):
    """run.cpp's classical loop written against nnpe.hpp (one device call per reference call) gives
    the same bits as the library's own step loop on the same system."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_abi import _build_adapter_loop
    from nnpengine_b200 import engine as E
    exe = _build_adapter_loop(str(tmp_path))
    s, table = cases.water_case()
    f = cases.write_inputs(s, table, str(tmp_path / "in"))
    xout = str(tmp_path / "x.f32")
    sqd_out = str(tmp_path / "sqd_adapter.txt")
    r = subprocess.run([exe, f["init"], f["table"], "20", "5", xout, sqd_out], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    log = cases.parse_log(r.stdout)
    x_adapter = np.fromfile(xout, np.float32).reshape(-1, 3)
    e = E.Engine(0)
    e.load_system_file(f["init"])
    e.setup(10.0, 2.0, 10.0, 2048)
    e._ok(e.lib.nnpe_pair_load_table(e.h, 1000, f["table"].encode()))
    e._ok(e.lib.nnpe_bonded_autogen(e.h, 1, E.bond_coef(1.0, 0, 0, cases.WATER_BOND_K), 1,
                                    E.angle_coef(109.47, 0, 0, cases.WATER_ANGLE_KC), 0, np.zeros(4, np.float32)))
    e.verlet(1.0, True)
    ref = e.run(21, log_interval=5)
    np.testing.assert_array_equal(x_adapter, e.positions())
    np.testing.assert_allclose(log[:, 3], [r["erg"] for r in ref], rtol=1e-6)
    e.sqd_setup(60, 6.0)   # the adapter's SQD of the same final state: the same file
    e.sqd_compute()
    e.sqd_dump(str(tmp_path / "sqd_engine.txt"))
    assert open(sqd_out).read() == open(str(tmp_path / "sqd_engine.txt")).read()
    e.close()


@pytest.mark.parametrize("mode", ["classical", "nnp_run"])
def test_driver_output_files_match_reference_values(tmp_path, mode):
    """The output files' contents, value by value, against the reference executable's on the same
    run file: total_steps 0 at 0 K (nothing depends on the reference's unseeded generator), run
    twice with the append flags on, so the g(r), S(q) and RMDF S(q) files hold running averages of
    count 2 and the xyz file two frames (ENVIRON::dump environ.cpp:178-188, GR::dump
    grsq.cpp:221-256, SQ::dump grsq.cpp:324-360, RMDF::dumpSQ grsq.cpp:1380-1416, dumpForce
    pair.cpp:421-437)."""
    g = np.load(os.path.join(cases.GOLDEN, "dumps648.npz"))
    d = str(tmp_path / mode)
    os.makedirs(d, exist_ok=True)
    s, table = cases.water_case()
    q, sqex, wt, ff = S.synthetic_sq_target(512, 20.0, 2, seed=7)
    tpath = os.path.join(d, "sq_target.txt")
    S.write_sq_target(tpath, q, sqex, wt, ff)
    kw = dict(rmdf=(STRENGTH, GAMMA, tpath), steps=(0, 1, 1000, 1, 1), append=True)
    if mode == "classical":
        path, files = cases.write_run_input(d, mode, s, table, **kw)
    else:
        paths = cases.write_nnp_inputs(NM.gauss_model(), d)
        path, files = cases.write_run_input(d, mode, s, nnp_paths=paths, nbin=750, cutoffs=(6.0, 2.0, 6.0), **kw)
    for _ in range(2):
        r = subprocess.run([build.DRIVER, mode, path, "--seed", "5", "--fp32-state"], capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
    frames, types, box = cases.read_dump(files["xyz"])
    np.testing.assert_array_equal(frames, g[f"{mode}_xyz"])          # FP32 positions, printed %.15e
    np.testing.assert_array_equal(types, g[f"{mode}_xyz_types"])
    np.testing.assert_allclose(box, g[f"{mode}_xyz_box"], rtol=1e-7)
    for k, rtol, atol_frac in (("gr", 2e-6, 2e-6), ("sq", 0, 1e-3), ("sqx", 0, 1e-3), ("force", 1e-4, 1e-4)):
        if f"{mode}_{k}" not in g:
            assert not os.path.exists(files[k])
            continue
        num, rows = cases.read_dump(files[k])
        ref = g[f"{mode}_{k}"]
        assert num == int(g[f"{mode}_{k}_num"])
        assert rows.shape == ref.shape, (k, rows.shape, ref.shape)
        np.testing.assert_allclose(rows[:, 0], ref[:, 0], rtol=1e-6)        # r or q grid
        vals, rvals = rows[:, 1:], ref[:, 1:]
        np.testing.assert_allclose(vals, rvals, rtol=rtol, atol=atol_frac * np.abs(rvals).max(), err_msg=k)
