"""CPU tests of the C ABI library and host-side logic (no GPU calls)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    syms = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        syms |= set(re.findall(r"\b(ds_[a-z0-9_]+)\s*\(", txt))
    return syms


def test_library_builds_and_exports_every_declared_symbol():
    from diffsplat_b200 import build as B
    lib_path = B.build()
    lib = C.CDLL(str(lib_path))
    syms = declared_symbols()
    assert len(syms) > 30
    missing = [s for s in sorted(syms) if not hasattr(lib, s)]
    assert not missing, missing


def test_status_strings_and_version():
    from diffsplat_b200 import _lib as L
    assert L.lib().ds_abi_version() == 1
    assert L.lib().ds_status_string(L.DS_ERR_ISECT_OVERFLOW) == b"intersection buffer overflow"
    assert L.lib().ds_status_string(L.DS_ERR_INTERNAL) == b"device-side consistency check failed"
    assert L.lib().ds_status_string(99) == b"unknown status"


def test_ctypes_struct_layouts_match_header(tmp_path):
    """Sizes and field offsets of the ctypes mirrors equal what the C compiler
    computes from include/diffsplat_b200.h."""
    import subprocess
    from diffsplat_b200 import _lib as L
    structs = {"ds_gaussian3d": L.Gaussian3D, "ds_splat3d": L.Splat3D, "ds_splat2d": L.Splat2D,
               "ds_adam_group": L.AdamGroup, "ds_fitter_config": L.FitterConfig,
               "ds_batch_config": L.BatchConfig, "ds_batch_instance": L.BatchInstance,
               "ds_densify_params": L.DensifyParams}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "diffsplat_b200.h"',
             "int main(void) {"]
    expect = []
    for cname, py in structs.items():
        lines.append(f'printf("%zu\\n", sizeof({cname}));')
        expect.append(C.sizeof(py))
        for fname, _ in py._fields_:
            lines.append(f'printf("%zu\\n", offsetof({cname}, {fname}));')
            expect.append(getattr(py, fname).offset)
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    assert got == expect


def test_scenes_are_deterministic():
    from diffsplat_b200.scenes import plain_small
    a, b = plain_small(3), plain_small(3)
    assert np.array_equal(a.params, b.params) and np.array_equal(a.target, b.target)
    assert not np.array_equal(plain_small(4).params, a.params)
    assert a.target.min() >= 0 and a.target.max() <= 1
    assert np.allclose(a.target * 255, np.round(a.target * 255), atol=1e-4)


def test_pinhole_pv_maps_pixels():
    from diffsplat_b200.scenes import pinhole_pv
    pv = pinhole_pv(256, 128, 200.0, 200.0, 128.0, 64.0).astype(np.float64)
    M = pv.reshape(4, 4).T
    u, v, z = 40.0, 100.0, 3.0
    p = np.array([(u - 128) * z / 200, (v - 64) * z / 200, z, 1.0])
    c = M @ p
    ndc = c[:3] / c[3]
    assert np.isclose((ndc[0] + 1) * 0.5 * 256, u) and np.isclose((1 - ndc[1]) * 0.5 * 128, v)
    assert -1 < ndc[2] < 1 and np.isclose(c[3], z)
