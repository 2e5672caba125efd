"""Makes the golden fixtures of tests/golden/ from the reference itself.

Run on a machine with a B200 after oracle/build_ref.sh has built
oracle/_ref/ref_harness and oracle/_ref/ICON-GPU from the reference sources:

    python tests/golden/make_golden.py [--out DIR] [--cases a,b,c,cli]

For every case below it writes <case>.npz holding the inputs (tilt angles,
projection rows, test vectors, iteration schedule) and what the reference's
own routines returned for them (stage outputs of ref_harness).  For the
"cli" case it also runs the reference ICON-GPU command-line tool on an MRC
tilt series and keeps its output files.  The npz files go to tests/golden/
by default, where they are committed; tests compare the oracle and the CUDA
path with them.  Inputs are generated here once, so the tests never regenerate them.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from feilab_b200 import mrc, synth  # noqa: E402

MAGIC = 0x49434F4E


def _case_inputs(name):
    rng = np.random.default_rng(abs(hash(name)) % (2 ** 32) if False else {"a": 11, "b": 22, "c": 33, "cli": 44}[name])
    if name == "a":
        nx, thick, S = 64, 48, 3
        tilts = synth.tilt_angles(-60, 60, 4)
        sched, dtype_, thr = (2, 6, 2), 2, 0.0
        ph = synth.make_phantom((nx, S, thick), 20, seed=101)
        rows = synth.add_noise(synth.project(ph, tilts), 0.5, 101).numpy()
    elif name == "b":
        nx, thick, S = 50, 37, 2
        t = np.linspace(-55, 55, 25).astype(np.float32)
        t = t + rng.uniform(-0.7, 0.7, t.shape).astype(np.float32)
        tilts = np.delete(t, [5, 17]).astype(np.float32)
        sched, dtype_, thr = (0, 8, 0), 1, 0.03
        ph = synth.make_phantom((nx, S, thick), 12, seed=202)
        rows = -synth.add_noise(synth.project(ph, tilts), 0.5, 202).numpy() * 0.01
    elif name == "c":
        nx, thick, S = 256, 128, 1
        tilts = synth.tilt_angles(-60, 60, 2)
        sched, dtype_, thr = (10, 170, 20), 2, 0.0
        ph = synth.make_phantom((nx, 32, thick), 200, seed=1001)
        rows = synth.add_noise(synth.project(ph, tilts, ys=[17]), 0.5, 1001).numpy()
    elif name == "cli":
        nx, thick, S = 64, 40, 4
        tilts = synth.tilt_angles(-60, 60, 5)
        sched, dtype_, thr = (1, 5, 1), 2, 0.0
        ph = synth.make_phantom((nx, S, thick), 15, seed=404)
        rows = synth.add_noise(synth.project(ph, tilts), 0.5, 404).numpy()
    else:
        raise ValueError(name)
    nz = len(tilts)
    M = nx * nz
    img_r = rng.standard_normal((nx, thick)).astype(np.float32)
    img_c = (rng.standard_normal((nx, thick)) + 1j * rng.standard_normal((nx, thick))).astype(np.complex64)
    fvec = (rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(np.complex64)
    return dict(nx=nx, thickness=thick, S=S, tilts=np.asarray(tilts, np.float32), rows=np.asarray(rows, np.float32),
                sched=np.array(sched, np.int32), data_type=dtype_, threshold=np.float32(thr),
                img_r=img_r, img_c=img_c, f=fvec)


def _write_case(path, c):
    nz = len(c["tilts"])
    hd = np.array([MAGIC, c["nx"], c["thickness"], nz, c["S"], *c["sched"], c["data_type"], 0], np.int32)
    with open(path, "wb") as f:
        f.write(hd.tobytes())
        f.write(np.float32(c["threshold"]).tobytes())
        f.write(c["tilts"].astype(np.float32).tobytes())
        f.write(c["rows"].astype(np.float32).tobytes())
        f.write(c["img_r"].astype(np.float32).tobytes())
        f.write(c["img_c"].astype(np.complex64).tobytes())
        f.write(c["f"].astype(np.complex64).tobytes())


def _read_out(path, c):
    nx, N1, S = c["nx"], c["thickness"], c["S"]
    M, NN = nx * len(c["tilts"]), nx * N1
    a = np.fromfile(path, np.float32)
    o, res = 0, {}

    def take(n):
        nonlocal o
        v = a[o:o + n]
        o += n
        return v
    res["ref_fwd_r"] = take(2 * M).view(np.complex64).copy()
    res["ref_fwd_c"] = take(2 * M).view(np.complex64).copy()
    res["ref_adj"] = take(2 * NN).view(np.complex64).reshape(nx, N1).copy()
    b, A, m, rp = [], [], [], []
    for _ in range(S):
        b.append(take(2 * M).view(np.complex64))
        A.append(take(2 * NN).view(np.complex64).reshape(nx, N1))
        m.append(take(NN).reshape(nx, N1))
        rp.append(take(nx))
    assert o == a.size, (o, a.size)
    res["ref_b"], res["ref_Ahwb"] = np.stack(b), np.stack(A)
    res["ref_m"], res["ref_reproj"] = np.stack(m), np.stack(rp)
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--ref", default=os.path.join(ROOT, "oracle", "_ref"))
    ap.add_argument("--cases", default="a,b,c,cli")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    harness = os.path.join(args.ref, "ref_harness")
    icon = os.path.join(args.ref, "ICON-GPU")
    for name in args.cases.split(","):
        c = _case_inputs(name)
        work = os.path.join(args.out, "work_" + name)
        os.makedirs(work, exist_ok=True)
        cpath, opath = os.path.join(work, "case.bin"), os.path.join(work, "out.bin")
        _write_case(cpath, c)
        subprocess.run([harness, cpath, opath, work], check=True, stdout=subprocess.DEVNULL)
        res = _read_out(opath, c)
        extra = {}
        if name == "cli":
            stack, tlt, odir = os.path.join(work, "stack.mrc"), os.path.join(work, "cli.tlt"), os.path.join(work, "res")
            mrc.write_tilt_series(stack, c["rows"])
            mrc.write_tlt(tlt, c["tilts"])
            os.makedirs(odir, exist_ok=True)
            a, b, cc = c["sched"]
            cmd = [icon, "-i", stack, "-t", tlt, "-o", odir, "-s", f"0,{c['S'] - 1}", "-iter", f"{a},{b},{cc}",
                   "-d", str(c["data_type"]), "-thr", str(float(c["threshold"])), "-g", "0", "-thi", str(c["thickness"])]
            p = subprocess.run(cmd, capture_output=True, text=True)
            extra["cli_returncode"] = np.int32(p.returncode)
            extra["cli_stdout"] = np.frombuffer(p.stdout.encode(), np.uint8)
            for y in range(c["S"]):
                raw = open(os.path.join(odir, "reconstruction", f"mid{y:05d}.mrc"), "rb").read()
                extra[f"cli_mid{y:05d}"] = np.frombuffer(raw, np.uint8)
            for fn in ("GroundTruth.mrc", "fullRec_reProjection.mrc", "crossV_reprojection.mrc", "fullRec.frc", "crossV.frc"):
                fp = os.path.join(odir, "crossValidation", fn)
                if os.path.exists(fp):
                    extra["cli_" + fn.replace(".", "_")] = np.frombuffer(open(fp, "rb").read(), np.uint8)
        np.savez_compressed(os.path.join(args.out, f"{name}.npz"), **{k: np.asarray(v) for k, v in c.items()}, **res, **extra)
        shutil.rmtree(work, ignore_errors=True)
        print("golden case", name, "written")


if __name__ == "__main__":
    main()
