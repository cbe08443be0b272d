"""The drop-in C++ headers (include/compat) compile on the host: every header
in one translation unit, plus the C++ ImageFitter smoke program."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
COMPAT = ROOT / "include" / "compat"


def _cxx():
    return shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def test_all_compat_headers_compile(tmp_path):
    headers = sorted(p.relative_to(COMPAT).as_posix() for p in COMPAT.rglob("*.h"))
    assert len(headers) >= 15
    src = tmp_path / "all.cpp"
    src.write_text("".join(f'#include "{h}"\n' for h in headers) + "int main() { return 0; }\n")
    r = subprocess.run([_cxx(), "-std=c++17", "-I", str(COMPAT), "-I", str(ROOT / "include"),
                        "-c", str(src), "-o", str(tmp_path / "all.o")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_cpp_fitter_smoke_builds(tmp_path):
    from diffsplat_b200 import build as B
    lib = B.build()
    exe = tmp_path / "fitter_smoke"
    r = subprocess.run([_cxx(), "-std=c++17", "-I", str(COMPAT), "-I", str(ROOT / "include"),
                        str(ROOT / "tests" / "cpp" / "fitter_smoke.cpp"), "-L", str(lib.parent),
                        "-ldiffsplat_b200", "-Xlinker", "-rpath", "-Xlinker", str(lib.parent),
                        "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
