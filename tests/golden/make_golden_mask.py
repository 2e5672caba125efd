"""Writes tests/golden/mask.npz: what the reference ICONMask3 (built from its
sources by oracle/build_ref.sh into oracle/_ref/ICONMask3) makes of the
slices and FRC files that the reference ICON-GPU (oracle/_ref/ICON-GPU)
writes for a small seeded tilt series.  Needs a GPU (both tools are CUDA).

    python tests/golden/make_golden_mask.py [--out DIR]

ICONMask3 works on square slices, so ICON-GPU runs with thickness = nx.
Cases: radius from the cross-validation FRC files; an explicit radius with a
Gaussian width; a cropped thickness with a z shift; no mask (assembly only).
"""
import argparse
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from feilab_b200 import mrc, synth  # noqa: E402

NX, S, SLICES = 64, 8, (0, 7)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    args = ap.parse_args()
    ref = os.path.join(ROOT, "oracle", "_ref")
    tilts = synth.tilt_angles(-60, 60, 3)
    ph = synth.make_phantom((NX, S, NX), 25, 0, seed=55)
    rows = synth.add_noise(synth.project(ph, tilts, ys=list(range(S))), 0.5, 55).numpy()
    out = {"tilts": tilts.astype(np.float32), "rows": rows.astype(np.float32)}
    with tempfile.TemporaryDirectory() as d:
        stack, tlt, res = os.path.join(d, "stack.mrc"), os.path.join(d, "t.tlt"), os.path.join(d, "res")
        os.makedirs(res)
        mrc.write_tilt_series(stack, rows)
        mrc.write_tlt(tlt, tilts)
        subprocess.run([os.path.join(ref, "ICON-GPU"), "-i", stack, "-t", tlt, "-o", res, "-s", f"{SLICES[0]},{SLICES[1]}",
                        "-iter", "2,10,2", "-d", "2", "-thr", "0", "-g", "0"], check=True, stdout=subprocess.DEVNULL)
        rec, cv = os.path.join(res, "reconstruction"), os.path.join(res, "crossValidation")
        out["mids"] = np.stack([mrc.read(os.path.join(rec, f"mid{s:05d}.mrc"))[1][0] for s in range(S)])
        out["mid_header"] = np.frombuffer(open(os.path.join(rec, "mid00000.mrc"), "rb").read(1024), np.uint8)
        for fn in ("crossV.frc", "fullRec.frc"):
            out[fn.replace(".", "_")] = np.loadtxt(os.path.join(cv, fn)).astype(np.float64)
        cases = {
            "frc": ["-th", str(NX), "-cf", os.path.join(cv, "crossV.frc"), "-ff", os.path.join(cv, "fullRec.frc")],
            "radius": ["-th", str(NX), "-r", "12", "-gw", "6"],
            "crop": ["-th", "40", "-z", "5", "-r", "15"],
            "nomask": ["-th", "48", "-nm", "1"],
        }
        for name, extra in cases.items():
            vol = os.path.join(d, f"{name}.mrc")
            cmd = [os.path.join(ref, "ICONMask3"), "-i", rec, "-s", f"{SLICES[0]},{SLICES[1]}", "-t", tlt, "-o", vol] + extra
            # the reference returns 1 after a successful no-mask assembly
            # (ICONCrossVMaskIn2D_weightOnlyOnSampled.cu:777-782)
            p = subprocess.run(cmd, stdout=subprocess.DEVNULL)
            if p.returncode not in (0, 1) or not os.path.exists(vol):
                raise RuntimeError(f"ICONMask3 failed for case {name}: rc {p.returncode}")
            h, v = mrc.read(vol)
            out[f"vol_{name}"] = v
            out[f"hdr_{name}"] = np.frombuffer(open(vol, "rb").read(1024), np.uint8)
            out[f"args_{name}"] = np.array(" ".join(extra))
    os.makedirs(args.out, exist_ok=True)
    np.savez_compressed(os.path.join(args.out, "mask.npz"), **out)
    print("wrote", os.path.join(args.out, "mask.npz"))


if __name__ == "__main__":
    main()
