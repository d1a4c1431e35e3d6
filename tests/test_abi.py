"""CPU tests of the C ABI: the library builds, loads and exports every
symbol include/lu_b200.h declares; host-only entry points work."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_symbols():
    txt = open(os.path.join(ROOT, "include", "lu_b200.h")).read()
    return sorted(set(re.findall(r"^\s*LU_API\s+(?:int|int64_t|size_t|const char\*)\s+(lu_\w+)\s*\(", txt, re.M)))


def test_library_loads_and_exports_header_symbols():
    from charmlu_b200 import _lib
    L = _lib.load()
    syms = _header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(L, s), s
    assert sorted(_lib.EXPORTS) == syms
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (lu_\w+)$", out, re.M))
    assert exported == set(syms), exported ^ set(syms)
    # the only other exports are unit-test hooks of internal kernels
    others = set(re.findall(r" T (\w+)$", out, re.M)) - exported
    assert all(o.startswith("lub_test_") for o in others), others


def test_status_strings_and_config_defaults():
    from charmlu_b200 import _lib
    L = _lib.load()
    assert L.lu_status_string(0) == b"ok"
    assert b"timed out" in L.lu_status_string(-3)
    assert b"singular" in L.lu_status_string(7)
    c = _lib.LuConfig()
    assert L.lu_config_default(ctypes.byref(c), 2048, 128) == 0
    assert c.n == 2048 and c.block_size == 128 and c.pivot_batch == 32  # b/4, benchmark.C:98
    assert c.ir_target == 16.0
    assert L.lu_workspace_bytes(ctypes.byref(c)) > 0
    assert L.lu_config_default(None, 1, 1) == -1


def test_create_rejects_bad_config_without_gpu():
    from charmlu_b200 import _lib
    L = _lib.load()
    c = _lib.LuConfig()
    L.lu_config_default(ctypes.byref(c), 48, 12)
    h = ctypes.c_void_p()
    c.block_size = 0
    assert L.lu_create(ctypes.byref(c), ctypes.byref(h)) == -1
    c.block_size = 7  # odd block sizes break the 16-byte TMA coordinate rule for FP64
    assert L.lu_create(ctypes.byref(c), ctypes.byref(h)) == -1


def test_matgen_host_matches_oracle():
    import oracle
    import charmlu_b200 as lu
    v = lu.matgen(32, seed=9934835, skip=5)
    ref, _ = oracle.matgen(32, seed=9934835, skip=5)
    np.testing.assert_array_equal(v, ref)


def test_product_does_not_import_oracle():
    pkg = os.path.join(ROOT, "charmlu_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
                txt = open(os.path.join(dirpath, f)).read()
                assert "import oracle" not in txt and "from oracle" not in txt, f
                assert "liboracle" not in txt, f


def _header_param_counts():
    """Parameter count of every LU_API declaration in include/lu_b200.h."""
    txt = open(os.path.join(ROOT, "include", "lu_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    out = {}
    for m in re.finditer(r"LU_API\s+(?:int|int64_t|size_t|const char\*)\s+(lu_\w+)\s*\(([^)]*)\)", txt):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_bindings_match_header_parameter_counts():
    """The ctypes signature table declares as many arguments as the header
    does for every entry point (an ABI change without its binding fails
    here, on CPU)."""
    from charmlu_b200 import _lib
    L = _lib.load()
    counts = _header_param_counts()
    assert set(counts) == set(_lib.EXPORTS)
    for name, k in counts.items():
        argtypes = getattr(L, name).argtypes
        assert argtypes is not None and len(argtypes) == k, (name, k, argtypes)


def test_create_rejects_bad_refinement_settings_without_gpu():
    from charmlu_b200 import _lib
    L = _lib.load()
    h = ctypes.c_void_p()
    for field, bad in (("gmres_restart", -1), ("gmres_restart", 5000), ("ir_stall", -2), ("gmres_tol", 1.5),
                       ("gmres_tol", -1e-3), ("gmres_tol", float("nan"))):
        c = _lib.LuConfig()
        L.lu_config_default(ctypes.byref(c), 256, 64)
        setattr(c, field, bad)
        assert L.lu_create(ctypes.byref(c), ctypes.byref(h)) == -1, (field, bad)


def test_config_struct_layout_matches_header():
    """sizeof and field offsets of lu_config / lu_refine_info as the C
    compiler lays them out equal the ctypes mirrors'."""
    import tempfile
    from charmlu_b200 import _lib
    fields = {"lu_config": _lib.LuConfig, "lu_refine_info": _lib.LuRefineInfo}
    src = ["#include <stdio.h>", "#include <stddef.h>", '#include "lu_b200.h"', "int main(void) {"]
    for name, cls in fields.items():
        src.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for f, _ in cls._fields_:
            src.append(f'printf("{name}.{f} %zu\\n", offsetof({name}, {f}));')
    src.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        c_path, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        open(c_path, "w").write("\n".join(src))
        subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), c_path, "-o", exe])
        out = dict(line.split() for line in subprocess.check_output([exe], text=True).splitlines())
    for name, cls in fields.items():
        assert int(out[name]) == ctypes.sizeof(cls), name
        for f, _ in cls._fields_:
            assert int(out[f"{name}.{f}"]) == getattr(cls, f).offset, (name, f)
