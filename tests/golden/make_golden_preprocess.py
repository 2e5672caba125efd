"""Writes tests/golden/preprocess.npz: seeded tilt stacks and what the
reference ICONPreProcess (built from its sources by oracle/build_ref.sh into
oracle/_ref/ICONPreProcess) writes for them, with and without the variance
normalisation.  Runs on the CPU.

    python tests/golden/make_golden_preprocess.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from feilab_b200 import mrc  # noqa: E402

CASES = {
    # name: (nz, ny, nx, thickness, seed)
    "p1": (7, 48, 64, 100, 3),
    "p2": (9, 75, 90, 250, 4),
}


def stack_for(nz, ny, nx, seed):
    rng = np.random.default_rng(seed)
    base = rng.gamma(3.0, 2.0, size=(nz, ny, nx))
    yy, xx = np.mgrid[0:ny, 0:nx]
    blob = 6.0 * np.exp(-((xx - nx / 3) ** 2 + (yy - ny / 2) ** 2) / (2 * (nx / 8) ** 2))
    return (base + blob[None] + rng.normal(0, 0.3, size=(nz, ny, nx))).astype(np.float32)


def main():
    exe = os.path.join(ROOT, "oracle", "_ref", "ICONPreProcess")
    out = {}
    with tempfile.TemporaryDirectory() as d:
        for name, (nz, ny, nx, th, seed) in CASES.items():
            st = stack_for(nz, ny, nx, seed)
            tilts = np.linspace(-60, 60, nz).astype(np.float32)
            fin, tlt = os.path.join(d, "in.mrc"), os.path.join(d, "t.tlt")
            mrc.write(fin, st)
            mrc.write_tlt(tlt, tilts)
            f1, f2 = os.path.join(d, "o1.mrc"), os.path.join(d, "o2.mrc")
            subprocess.run([exe, "-i", fin, "-o", f1], check=True, stdout=subprocess.DEVNULL)
            subprocess.run([exe, "-i", fin, "-t", tlt, "-th", str(th), "-o", f2], check=True, stdout=subprocess.DEVNULL)
            out[name + "_stack"] = st
            out[name + "_tilts"] = tilts
            out[name + "_thickness"] = np.int32(th)
            out[name + "_mode_only"] = mrc.read(f1)[1]
            out[name + "_normalized"] = mrc.read(f2)[1]
            out[name + "_header"] = np.frombuffer(open(f2, "rb").read(1024), np.uint8)
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "preprocess.npz"), **out)
    print("wrote tests/golden/preprocess.npz")


if __name__ == "__main__":
    main()
