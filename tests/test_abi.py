"""The C-ABI library: it loads, exports every declared symbol, and fails cleanly without a GPU."""
import ctypes as C
import os

import numpy as np
import pytest

from nnpengine_b200 import _lib, systems


def test_library_exports_declared_symbols():
    lib = _lib.load()
    declared = _lib.declared_symbols()
    assert len(declared) > 30
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing


def test_coef_helpers_match_reference_set_param():
    from nnpengine_b200 import engine
    np.testing.assert_array_equal(engine.bond_coef(1.0, 0, 0, 450.0), np.array([1, 0, 0, 900], np.float32))
    a = engine.angle_coef(109.47, 0, 0, 62.0)
    assert a[0] == np.float32(np.cos(np.float32(109.47) * np.float32(np.pi) / np.float32(180)))
    np.testing.assert_array_equal(engine.dihedral_coef(1, 2, 3, 4), np.array([1 - 3, 2 - 12, 12, 48], np.float32))


def test_create_without_device_reports_error():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.load()
    h = C.c_void_p()
    assert lib.nnpe_create(0, C.byref(h)) != 0


def test_water_files_roundtrip(tmp_path):
    s = systems.water_box(3, 9.312, seed=3)
    p = tmp_path / "init.txt"
    systems.write_init_file(str(p), s)
    lines = [l for l in open(p).read().splitlines() if l.strip()]
    nmt, nmol = map(int, lines[0].split())
    assert (nmt, nmol) == (1, 27)
    ntype, natom, bl = lines[2].split()
    assert int(natom) == 81 and abs(float(bl) - 9.312) < 1e-6
    x = np.array([[float(v) for v in l.split()[4:7]] for l in lines[3:]], np.float32)
    np.testing.assert_array_equal(x, s.x)
    mol = open(str(p).replace("init.txt", "init.mol0")).read()
    assert "3 atoms" in mol and "Bonds" in mol and "Angles" in mol


def test_serving_struct_layout_matches_header(tmp_path):
    """The ctypes mirrors of nnpe_serve_config / nnpe_request / nnpe_request_stats have the C
    header's sizes and field offsets (compiled here with gcc against include/nnpe.h)."""
    import os
    import shutil
    import subprocess
    from nnpengine_b200 import serve
    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    inc = os.path.join(os.path.dirname(_lib.__file__), "..", "include")
    structs = {"nnpe_serve_config": serve.ServeConfig, "nnpe_request": serve.Request,
               "nnpe_request_stats": serve.RequestStats}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "nnpe.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", inc, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


def _build_adapter_loop(out_dir):
    import os
    import subprocess
    from nnpengine_b200 import build
    here = os.path.dirname(os.path.abspath(__file__))
    inc = os.path.join(here, "..", "include")
    exe = os.path.join(out_dir, "adapter_loop")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", inc, os.path.join(here, "adapter_loop.cpp"),
                    "-L", build.OUT, "-lnnpe", "-Wl,-rpath," + build.OUT, "-o", exe], check=True)
    return exe


def test_reference_classes_adapter_compiles(tmp_path):
    """A loop written like run.cpp against the reference's class names compiles and links against
    include/nnpe.hpp and libnnpe.so (it runs in the GPU tests)."""
    import shutil
    if not shutil.which("g++"):
        pytest.skip("no C++ compiler")
    assert os.path.exists(_build_adapter_loop(str(tmp_path)))


def test_run_file_driver_built():
    from nnpengine_b200 import build
    assert os.path.exists(build.DRIVER) and os.access(build.DRIVER, os.X_OK)
