"""Direct S(q) (SQD) on the GPU against the reference's own output (golden fixtures made by its C++)
and the FP64 restatement: the same G vectors in every bin, the same mean |G|, S(q) within FP32
summation; the dump format and its running average; the run-file driver's sqd line."""
import dataclasses
import os
import subprocess

import numpy as np
import pytest

import cases
from nnpengine_b200 import engine as E
from oracle import orc

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _engine(name):
    g = np.load(os.path.join(cases.GOLDEN, name + ".npz"))
    s, _ = cases.water_case(jitter=0.05) if name == "sqd648" else cases.mixture_case()
    s = dataclasses.replace(s, x=np.ascontiguousarray(g["x"], np.float32))
    e = E.Engine(0)
    e.set_system(s)
    e.setup(10.0, 2.0, 10.0, 2048)
    return e, s, g


@pytest.mark.parametrize("name", ["sqd648", "sqd2000"])
def test_sqd_matches_reference_and_fp64(name):
    e, s, g = _engine(name)
    nq, qmax = int(g["nq"]), float(g["qmax"])
    assert e.sqd_setup(nq, qmax) == int(g["ngv"])
    q, sq, cnt = e.sqd_compute()
    np.testing.assert_array_equal(cnt, g["count"])
    m = cnt > 0
    np.testing.assert_allclose(q[m], g["q"][m], rtol=1e-5)
    q64, sq64, cnt64 = orc.sqd(g["x"], s.typ, s.ntype, float(s.bl), nq, qmax)
    np.testing.assert_array_equal(cnt, cnt64)
    np.testing.assert_allclose(q, q64, rtol=1e-12, atol=0)
    scale = max(1.0, float(np.abs(sq64).max()))
    err64 = np.abs(sq - sq64)[m].max() / scale
    err_ref = np.abs(sq - g["sq"])[m].max() / scale
    print(f"{name}: SQD vs FP64 {err64:.2e}, vs the reference's float {err_ref:.2e} (of max |S| {scale:.3g})")
    assert err64 < 2e-5
    assert err_ref < 1e-4
    assert np.all(sq[~m] == 0)


def test_sqd_after_list_build_and_determinism():
    """After a list build the atoms are sorted by cell and folded into the box: the sums run in
    another order over periodic images of the same positions."""
    e, s, g = _engine("sqd648")
    nq, qmax = int(g["nq"]), float(g["qmax"])
    e.sqd_setup(nq, qmax)
    _, sq0, _ = e.sqd_compute()
    _, sq0b, _ = e.sqd_compute()
    np.testing.assert_array_equal(sq0, sq0b)
    e.list_build()
    _, sq1, _ = e.sqd_compute()
    scale = max(1.0, float(np.abs(sq0).max()))
    assert np.abs(sq1 - sq0).max() < 2e-5 * scale


def test_sqd_dump_and_running_average(tmp_path):
    e, s, g = _engine("sqd648")
    nq, qmax = int(g["nq"]), float(g["qmax"])
    e.sqd_setup(nq, qmax)
    q, sq, cnt = e.sqd_compute()
    path = str(tmp_path / "sqd.txt")
    e.sqd_dump(path)
    lines = open(path).read().splitlines()
    assert lines[0] == "# 1"
    rows = np.array([[float(v) for v in ln.split()] for ln in lines[1:]])
    m = cnt > 0
    assert rows.shape == (int(m.sum()), 1 + sq.shape[1])
    np.testing.assert_allclose(rows[:, 0], q[m], rtol=1e-14)
    np.testing.assert_allclose(rows[:, 1:], sq[m], rtol=1e-14, atol=1e-14)
    e.sqd_dump(path, append=True)   # the same values averaged in: unchanged, count 2
    lines2 = open(path).read().splitlines()
    assert lines2[0] == "# 2"
    rows2 = np.array([[float(v) for v in ln.split()] for ln in lines2[1:]])
    np.testing.assert_allclose(rows2, rows, rtol=1e-13, atol=1e-13)


def test_run_file_driver_writes_sqd(tmp_path):
    s, table = cases.water_case(jitter=0.05)
    d = str(tmp_path)
    path, out = cases.write_run_input(d, "classical", s, table, steps=(5, 5, 5, 5, 5), sqd=(6.0, 60))
    exe = os.path.join(ROOT, "nnpengine_b200", "lib", "nnpe_run")
    r = subprocess.run([exe, "classical", path, "--seed", "3"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = open(out["sqd"]).read().splitlines()
    assert lines[0] == "# 1"
    rows = np.array([[float(v) for v in ln.split()] for ln in lines[1:]])
    q64, _, cnt64 = orc.sqd(s.x, s.typ, s.ntype, float(s.bl), 60, 6.0)
    m = cnt64 > 0
    assert rows.shape == (int(m.sum()), 4)
    np.testing.assert_allclose(rows[:, 0], q64[m], rtol=1e-12)
    assert np.all(np.isfinite(rows))
