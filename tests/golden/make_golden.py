"""Regenerate the committed fixtures of tests/golden/.

    python tests/golden/make_golden.py --reference <path of the reference checkout>

* kh_grid_y.txt     -- the 66 GY values stored in the reference's
                       KH_test/grid.h5 (/grids/y), read straight from the
                       HDF5 file's contiguous data block.
* KH_test_input.dat, KH_test_input_chan.dat -- the reference's KH_test run
                       parameters, byte for byte (input-file parser tests).
* KH_test_grid.h5    -- the reference's KH_test/grid.h5, byte for byte: a file
                       the HDF5 library wrote, for the tests of diablo_b200.h5.
* oracle_kh_small.npz -- CPU-oracle regression vectors: a 24x17x16 shear
                       layer, initial Fourier state and the state after 3
                       time steps (dealiased block), plus the statistics.
"""
from __future__ import annotations

import argparse
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def read_grid_h5(path: str, n: int) -> np.ndarray:
    """Find the n little-endian doubles of /grids/y: the contiguous data block
    that ends the file (HDF5 stores a small contiguous dataset at the end)."""
    raw = open(path, "rb").read()
    v = np.frombuffer(raw[len(raw) - 8 * n:], dtype="<f8").copy()
    if not (np.all(np.diff(v) > 0) and abs(v[0] + v[-1]) < 1e-12):
        raise ValueError("unexpected grid.h5 layout")
    return v


def oracle_fixture(path: str) -> None:
    from diablo_b200 import grid as G, ics, params as P
    from oracle.oracle import Oracle

    p = P.kelvin_helmholtz(24, 17, 16)
    g = G.channel_grid(G.uniform_gy(p.ny, -10.0, 10.0))
    o = Oracle(p, g, 0.05)
    u, th = ics.shear_layer(p, g, seed=99, amp=1e-2)
    o.init_from_physical(u, th)
    blk = lambda a: a[..., : p.tnkz + 1, : p.nkx + 1].copy()
    init = {f"init_cu{c}": blk(o.cu[c]) for c in range(3)}
    init["init_cth"] = blk(o.cth)
    o.step(3)
    out = {f"cu{c}": blk(o.cu[c]) for c in range(3)}
    out.update(cth=blk(o.cth), cp=blk(o.cp), cf0=blk(o.cf[0]), cf1=blk(o.cf[1]), cf2=blk(o.cf[2]),
               cfth=blk(o.cfth), stats=o.stats(), gy=g.gy, gyf=g.gyf)
    np.savez_compressed(path, u=u, th=th, **init, **out)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the reference checkout (holds diablo_2.0/)")
    a = ap.parse_args()
    kh = os.path.join(a.reference, "diablo_2.0", "KH_test")
    gy = read_grid_h5(os.path.join(kh, "grid.h5"), 66)
    np.savetxt(os.path.join(HERE, "kh_grid_y.txt"), gy, fmt="%.17e")
    shutil.copyfile(os.path.join(kh, "input.dat"), os.path.join(HERE, "KH_test_input.dat"))
    shutil.copyfile(os.path.join(kh, "input_chan.dat"), os.path.join(HERE, "KH_test_input_chan.dat"))
    shutil.copyfile(os.path.join(kh, "grid.h5"), os.path.join(HERE, "KH_test_grid.h5"))
    oracle_fixture(os.path.join(HERE, "oracle_kh_small.npz"))
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
