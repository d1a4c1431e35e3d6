"""The public header compiles as C and as C++ (its extern "C" block), and a
program built against it links to liblu_b200.so and runs the entry points
that need no GPU. This is what a maintainer's host driver does first."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "charmlu_b200")
CUDA_LIB = "/usr/local/cuda/lib64"


@pytest.mark.parametrize("compiler,std", [("gcc", "-std=c11"), ("g++", "-std=c++17")])
def test_header_compiles_links_and_runs(tmp_path, compiler, std):
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} not found")
    src = os.path.join(ROOT, "tests", "cpp", "abi_use.c")
    exe = str(tmp_path / f"abi_use_{compiler}")
    lang = ["-x", "c++"] if compiler == "g++" else []
    cmd = [compiler, std, "-Wall", "-Werror", *lang, src, "-x", "none", "-I", os.path.join(ROOT, "include"),
           "-L", LIBDIR, "-llu_b200", "-L", CUDA_LIB, "-lcudart", f"-Wl,-rpath,{LIBDIR}",
           f"-Wl,-rpath,{CUDA_LIB}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    txt = out.stdout
    assert "n=2048 b=128 batch=32 layout=0 target=16" in txt
    assert "status(0)=ok" in txt
    assert "bad_layout=-1" in txt
