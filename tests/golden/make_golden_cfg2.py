"""Makes tests/golden/cfg2.npz: the production workload's parity fixture.

Sixteen seeded, randomly chosen xz-slices of the 1024 x 1024 x 300 series
(300 ellipsoids + 3000 Gaussian blobs on a 0.1 background, 61 tilts -60..60
step 2, SNR 0.1; feilab_b200.synth.series("cfg2")), reconstructed with the
full production schedule (-iter 10,280,10, data type 2, threshold 0):

  phase "reference" (a machine with a B200, after oracle/build_ref.sh):
      python tests/golden/make_golden_cfg2.py --phase reference --out DIR
    generates the rows on the CPU, runs the reference's own routines
    (oracle/_ref/ref_harness: readSlicePart ... Iteration3, compiled from the
    reference sources) and writes DIR/cfg2_ref.npz (rows, tilts, schedule,
    ref_m, ref_reproj);
  phase "oracle" (any machine; about 4 minutes on 8 cores):
      python tests/golden/make_golden_cfg2.py --phase oracle --ref DIR/cfg2_ref.npz
    adds the FP64 oracle's solve of the same rows for the same iteration
    count and writes tests/golden/cfg2.npz.  The FP64 result is stored as its
    difference from the reference's, quantised to int16 (fp64_minus_ref_q,
    step fp64_minus_ref_step): m_fp64 = ref_m + q * step, exact to ~5e-11 of
    the image's largest value (m_fp64() below rebuilds it).

The rows are stored, so the tests never regenerate them.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

SCHED = (10, 280, 10)
DATA_TYPE, THRESHOLD = 2, 0.0
NSLICES, SLICE_SEED = 16, 20260


def slice_indices():
    """The 16 slices: seeded random y in 0..1023, sorted."""
    rng = np.random.default_rng(SLICE_SEED)
    return np.sort(rng.choice(1024, NSLICES, replace=False)).astype(np.int32)


def phase_reference(out_dir, ref_dir):
    from feilab_b200 import synth
    from make_golden import _read_out, _write_case
    ys = slice_indices()
    rows, tilts, thick, _ = synth.series("cfg2", device="cpu", ys=[int(y) for y in ys])
    rows = rows.numpy().astype(np.float32)
    nx, nz, S = rows.shape[2], len(tilts), rows.shape[0]
    rng = np.random.default_rng(7)
    c = dict(nx=nx, thickness=thick, S=S, tilts=np.asarray(tilts, np.float32), rows=rows,
             sched=np.array(SCHED, np.int32), data_type=DATA_TYPE, threshold=np.float32(THRESHOLD),
             img_r=rng.standard_normal((nx, thick)).astype(np.float32),
             img_c=np.zeros((nx, thick), np.complex64), f=np.zeros(nx * nz, np.complex64))
    work = os.path.join(out_dir, "work_cfg2")
    os.makedirs(work, exist_ok=True)
    cpath, opath = os.path.join(work, "case.bin"), os.path.join(work, "out.bin")
    _write_case(cpath, c)
    subprocess.run([os.path.join(ref_dir, "ref_harness"), cpath, opath, work], check=True, stdout=subprocess.DEVNULL)
    res = _read_out(opath, c)
    np.savez_compressed(os.path.join(out_dir, "cfg2_ref.npz"), ys=ys, nx=nx, thickness=thick, S=S, tilts=c["tilts"],
                        rows=rows, sched=c["sched"], data_type=DATA_TYPE, threshold=np.float32(THRESHOLD),
                        ref_m=res["ref_m"].astype(np.float32), ref_reproj=res["ref_reproj"].astype(np.float32))
    shutil.rmtree(work, ignore_errors=True)
    print("cfg2_ref.npz written:", S, "slices, y =", ys.tolist())


def phase_oracle(ref_path, out_path):
    from oracle.oracle import OraclePlan
    z = dict(np.load(ref_path))
    p = OraclePlan(int(z["nx"]), int(z["thickness"]), z["tilts"], "f64")
    m64 = p.reconstruct(z["rows"], tuple(int(v) for v in z["sched"]), int(z["data_type"]), float(z["threshold"]))
    d = m64 - z["ref_m"].astype(np.float64)
    step = max(float(np.abs(d).max()), 1e-300) / 32000.0
    z["fp64_minus_ref_q"] = np.round(d / step).astype(np.int16)
    z["fp64_minus_ref_step"] = np.float64(step)
    np.savez_compressed(out_path, **z)
    back = m_fp64(z)
    rel = [np.linalg.norm(m64[s] - z["ref_m"][s]) / np.linalg.norm(m64[s]) for s in range(len(m64))]
    enc = float(np.abs(back - m64).max() / np.abs(m64).max())
    print(f"cfg2.npz written; reference vs FP64 oracle: max relative L2 {max(rel):.3e}; encoding error {enc:.1e}")


def m_fp64(z):
    """The FP64 oracle's result (float64) from a loaded cfg2.npz."""
    return z["ref_m"].astype(np.float64) + z["fp64_minus_ref_q"].astype(np.float64) * float(z["fp64_minus_ref_step"])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--phase", choices=["reference", "oracle"], required=True)
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--ref", default=os.path.join(ROOT, "oracle", "_ref"),
                    help="reference phase: directory of ref_harness; oracle phase: the cfg2_ref.npz to complete")
    args = ap.parse_args()
    if args.phase == "reference":
        os.makedirs(args.out, exist_ok=True)
        phase_reference(args.out, args.ref)
    else:
        phase_oracle(args.ref, os.path.join(args.out, "cfg2.npz"))


if __name__ == "__main__":
    main()
