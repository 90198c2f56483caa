"""The pybind11 binding INTEGRATION.md gives a maintainer who keeps the
reference's compiled `_dda_model` module (python_bindings/PythonBindings.cpp)
compiles as written against include/tdda.h, links against libtdda.so and
imports; its constructor maps the reference's arguments onto tdda_params and
raises RuntimeError on invalid input (checked before any device work, so this
runs without a GPU)."""
import importlib.util
import os
import re
import shutil
import subprocess
import sys
import sysconfig

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "topo-dda_b200", "dda_model")


def _sketch():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", text, re.S)
    src = [b for b in blocks if "PYBIND11_MODULE" in b]
    assert len(src) == 1
    return src[0]


def test_pybind_sketch_compiles_and_imports(tmp_path):
    pybind11 = pytest.importorskip("pybind11")
    if shutil.which("g++") is None or not os.path.exists(os.path.join(LIBDIR, "libtdda.so")):
        pytest.skip("g++ or the built library is missing")
    src = tmp_path / "binding.cpp"
    src.write_text("#include <array>\n#include <complex>\n#include <stdexcept>\n" + _sketch())
    ext = sysconfig.get_config_var("EXT_SUFFIX")
    out = tmp_path / f"_dda_model{ext}"
    cmd = ["g++", "-O1", "-shared", "-fPIC", "-std=c++17", "-I", pybind11.get_include(),
           "-I", sysconfig.get_paths()["include"], "-I", os.path.join(ROOT, "include"), str(src),
           "-o", str(out), "-L", LIBDIR, "-l:libtdda.so", f"-Wl,-rpath,{LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    spec = importlib.util.spec_from_file_location("_dda_model", out)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    assert hasattr(mod, "DDAModel")
    for name in ("solveElectricField", "calculateObjective", "calculateGradients", "setParameters",
                 "getParameters", "getDielectrics", "getElectricField"):
        assert hasattr(mod.DDAModel, name), name
    geo = np.zeros(3 * 8, dtype=np.int32)
    with pytest.raises(RuntimeError, match="symmetryType"):
        mod.DDAModel(0.0, 50.0, 0.5, "piecewise", [100], [2.0], False, "none", [0.0, 0.0], False,
                     "IntegratedE", [2.0], geo, np.zeros(24), 2, 2, 2, 8, [0, 0, 1], 1.0, [1, 0, 0], 542.0,
                     [1.0 + 0j, 3.5 + 0.01j], 1.0, 0, 0, 2.0, 2.0, "FCD", 25.0, np.zeros(4), np.zeros(4), 0.1,
                     False)
