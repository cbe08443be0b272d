"""Writes the golden PLY fixtures with the reference's own PLYSaver
(src/io/ply_io.cpp, built into oracle/_ref/libdsref_ply.so by
`make -C oracle ref REF=<reference tree>`):

  tests/golden/ref_sh0.ply, ref_sh3.ply   written by PLYSaver::save
  tests/golden/ply_records.npz            the in-memory records they were
                                          written from (Gaussian3D rows,
                                          59 floats) and what PLYLoader::load
                                          reads back from each file

    python tests/golden/make_golden_ply.py
"""
from pathlib import Path
import sys

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from oracle import ref_ply  # noqa: E402


def records(n: int, bands: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    rec = rng.normal(size=(n, 59)).astype(np.float32)
    rec[:, 13 + 3 * bands:58] = 0.0  # only 3 * bands SH-rest floats are stored
    return rec


def main() -> None:
    out = {}
    for name, bands in (("sh0", 0), ("sh3", 15)):
        rec = records(48, bands, seed=100 + bands)
        path = HERE / f"ref_{name}.ply"
        ref_ply.save(path, rec, bands)
        back, deg = ref_ply.load(path)
        out[f"{name}_records"] = rec
        out[f"{name}_loaded"] = back
        out[f"{name}_degree"] = np.int32(deg)
    np.savez(HERE / "ply_records.npz", **out)


if __name__ == "__main__":
    main()
