"""Train the warm-start network for one geometry on synthetic tilt series.

    python -m feilab_b200.train_warmstart --out feilab_b200/weights/warmstart_1024x300.npz
    python -m feilab_b200.train_warmstart --nx 512 --thickness 256 --seeds 20 --per-seed 1000 \
        --schedule 10,480,10 --batch 32 --epochs 20 --heldout 1024 --out feilab_b200/weights/warmstart_512x256.npz

Training slices come from phantoms of the 1024x1024x300 / 61-tilt kind
(300 ellipsoids + 3000 Gaussian blobs on a 0.1 background, SNR 0.1) with
seeds disjoint from the benchmark's phantom.  The input of a slice is its
back-projection A^H W b (IconPlan.prepare_rhs), the target the plain ICON
solution after the full schedule (IconPlan.solve from m = 0), so that the
network predicts where the reference's iteration ends.  The output gain is
set so that targets have unit RMS in network units.  Adam with a cosine
learning-rate decay; a held-out phantom reports the prediction error, the
iterations cold and warm solves need to bring the ICON update below a
relative-step tolerance (IconPlan.solve_until), and the FRC of the warm
result against the cold one.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np


def make_data(plan, seeds, per_seed, sched, data_type, threshold, batch, log):
    """Inputs A^H W b and plain-ICON targets of per_seed slices of each
    phantom: the 1024x1024x300 series itself at that size, else a phantom of
    its kind with plan.N0 x per_seed x plan.N1 voxels."""
    import torch
    from . import synth
    As, Ms = [], []
    for sd in seeds:
        if (plan.N0, plan.N1) == (1024, 300):
            g = np.random.default_rng(sd)
            ys = sorted(g.choice(1024, size=per_seed, replace=False).tolist())
            rows, tilts, th, _ = synth.series("cfg2", device="cuda", ys=ys, seed=sd)
        else:
            rows, tilts = synth.cfg2_kind(plan.N0, per_seed, plan.N1, sd, device="cuda")
        for s0 in range(0, per_seed, batch):
            r = rows[s0:s0 + batch].contiguous()
            A = plan.prepare_rhs(r)
            m = plan.solve(A, sched, data_type, threshold)
            As.append(A)
            Ms.append(m)
        torch.cuda.synchronize()
        log(f"data: seed {sd}, {per_seed} slices")
    return torch.cat(As), torch.cat(Ms)


def frc_mean(a, b, nring=None):
    """Per-slice mean over frequency rings (up to Nyquist) of the Fourier ring
    correlation of two image stacks (S, N0, N1)."""
    import torch
    fa, fb = torch.fft.fft2(a.double()), torch.fft.fft2(b.double())
    S, N0, N1 = a.shape
    ky = torch.fft.fftfreq(N0, device=a.device)[:, None]
    kx = torch.fft.fftfreq(N1, device=a.device)[None, :]
    r = torch.sqrt(kx * kx + ky * ky)
    nring = nring or min(N0, N1) // 2
    idx = torch.clamp((r * 2 * nring).long(), max=nring)
    out = []
    for s in range(S):
        num = torch.zeros(nring + 1, dtype=torch.float64, device=a.device)
        da = torch.zeros_like(num)
        db = torch.zeros_like(num)
        num.index_add_(0, idx.flatten(), (fa[s] * fb[s].conj()).real.flatten())
        da.index_add_(0, idx.flatten(), (fa[s].abs() ** 2).flatten())
        db.index_add_(0, idx.flatten(), (fb[s].abs() ** 2).flatten())
        f = num[:nring] / torch.sqrt(da[:nring] * db[:nring]).clamp_min(1e-300)
        out.append(float(f.mean()))
    return np.array(out)


def rms_ratio(A, M):
    a = A.real.double().pow(2).mean(dim=(1, 2)).sqrt()
    m = M.double().pow(2).mean(dim=(1, 2)).sqrt()
    return (m / a).cpu().numpy()


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--seeds", type=int, default=16, help="training phantoms")
    ap.add_argument("--per-seed", type=int, default=256, help="slices per phantom")
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--init-seed", type=int, default=1)
    ap.add_argument("--tol", type=float, default=1e-3, help="relative-step tolerance of the evaluation")
    ap.add_argument("--eval-only", default=None, help="load weights from this file instead of training")
    ap.add_argument("--heldout", type=int, default=64, help="held-out slices")
    ap.add_argument("--log", default=None)
    ap.add_argument("--nx", type=int, default=1024)
    ap.add_argument("--thickness", type=int, default=300)
    ap.add_argument("--schedule", default="10,280,10", help="schedule of the target solves")
    args = ap.parse_args(argv)

    import torch
    from . import icon, synth, warmstart

    logf = open(args.log, "a") if args.log else None

    def log(msg):
        line = f"[{time.strftime('%H:%M:%S')}] {msg}"
        print(line, flush=True)
        if logf:
            logf.write(line + "\n")
            logf.flush()

    sched, data_type, threshold = tuple(int(v) for v in args.schedule.split(",")), 2, 0.0
    tilts = synth.tilt_angles(-60, 60, 2)
    plan = icon.IconPlan(args.nx, args.thickness, tilts, capacity=128)
    plan.set_operator("toeplitz")
    t0 = time.time()
    A, M = make_data(plan, [5001 + k for k in range(args.seeds)], args.per_seed, sched, data_type, threshold, 128, log)
    Ah, Mh = make_data(plan, [9001], args.heldout, sched, data_type, threshold, 64, log)
    log(f"data ready: {A.shape[0]} training, {Ah.shape[0]} held-out slices in {time.time() - t0:.1f} s")

    n = A.shape[0]
    net = warmstart.Network(plan, capacity=args.batch)
    if args.eval_only:
        z = np.load(args.eval_only)
        net.set_params(z["params"], float(z["gain"]))
        log(f"loaded {args.eval_only}")
    else:
        gain = float(np.median(rms_ratio(A, M)))
        net.init(args.init_seed)
        net.set_gain(gain)
        steps_per_epoch = n // args.batch
        total = steps_per_epoch * args.epochs
        gen = torch.Generator().manual_seed(args.init_seed)
        step = 0
        t1 = time.time()
        for ep in range(args.epochs):
            perm = torch.randperm(n, generator=gen)
            losses = []
            for k in range(steps_per_epoch):
                idx = perm[k * args.batch:(k + 1) * args.batch].cuda()
                lr = args.lr * 0.5 * (1 + math.cos(math.pi * step / total))
                losses.append(net.train_step(A.index_select(0, idx).contiguous(), M.index_select(0, idx).contiguous(),
                                             lr))
                step += 1
            log(f"epoch {ep}: mean loss {np.mean(losses):.5f} (last {losses[-1]:.5f}), {time.time() - t1:.1f} s")
        if warmstart.device_error():
            raise RuntimeError("tensor-core kernel reported a timed-out wait")

    # Held-out evaluation.
    err = []
    for s0 in range(0, Ah.shape[0], args.batch):
        a = Ah[s0:s0 + args.batch].contiguous()
        m = Mh[s0:s0 + args.batch]
        p = net.predict(a)
        err.append(((p - m).norm(dim=(1, 2)) / m.norm(dim=(1, 2))).cpu().numpy())
    err = np.concatenate(err)
    hb = Ah[:args.batch].contiguous()
    tol = args.tol
    a, b, c = sched
    m_cold = plan.solve(hb, sched, data_type, threshold)
    _, n_cold, st_cold = plan.solve_until(hb, tol, sched, data_type, threshold, check_every=10)
    m0 = net.predict(hb)
    m_warm, n_warm, st_warm = plan.solve_until(hb, tol, sched, data_type, threshold, m0=m0, check_every=10)
    frc = frc_mean(m_warm, m_cold)
    rel = ((m_warm - m_cold).norm(dim=(1, 2)) / m_cold.norm(dim=(1, 2))).cpu().numpy()
    log(f"held-out: prediction rel. error median {np.median(err):.4f}; to relative step {tol:g}: cold {n_cold} "
        f"iterations (step {st_cold.max():.2e}), warm {n_warm} (step {st_warm.max():.2e}); warm vs cold: "
        f"rel. L2 median {np.median(rel):.4f}, mean FRC min {frc.min():.4f}")
    # Iterations to the cold-start result: ICON iterations k of the schedule
    # (a, k, c) after which the result has FRC >= 0.99 against the full cold
    # solve (a, b, c), for cold and warm starts.
    curve = []
    for k in [k for k in (0, 10, 20, 40, 70, 100, 150, 200, 280, 380, 480) if k <= b]:
        mc = plan.solve(hb, (a, k, c), data_type, threshold)
        mw = plan.solve(hb, (a, k, c), data_type, threshold, m0=m0)
        fc, fw = frc_mean(mc, m_cold), frc_mean(mw, m_cold)
        curve.append((k, float(fc.min()), float(fw.min())))
        log(f"  ICON iterations {k:3d}: FRC vs full cold solve, min over slices: cold {fc.min():.4f}  warm {fw.min():.4f}")
    f0 = frc_mean(m0, m_cold)
    log(f"  prediction itself: FRC vs full cold solve, min over slices {f0.min():.4f}, median {np.median(f0):.4f}")
    curve0 = []
    for k in (0, 10, 20, 40, 70, 100, 150):
        mw = plan.solve(hb, (0, k, c), data_type, threshold, m0=m0)
        fw = frc_mean(mw, m_cold)
        curve0.append((k, float(fw.min())))
        log(f"  warm without the first INFR phase, ICON iterations {k:3d}: FRC min {fw.min():.4f}")
    k_cold = next((k for k, fc, fw in curve if fc >= 0.99), b)
    k_warm = next((k for k, fc, fw in curve if fw >= 0.99), b)
    log(f"  ICON iterations to FRC >= 0.99: cold {k_cold}, warm {k_warm}")
    # Every held-out slice to the tolerance: cold (icon_solve_until from
    # m = 0) against warm (network start, icon_solve_warm with its acceptance
    # test and cold redo), device-timed, FRC against the full cold solve.
    full = {}
    cap = plan.capacity
    for tol_f, name in [(t, nm) for t in sorted({tol, 0.02, 0.03}) for nm in ("cold", "warm")]:
        its, redone, frcs = [], 0, []
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        outs = []
        for s0 in range(0, Ah.shape[0], cap):
            a = Ah[s0:s0 + cap].contiguous()
            if name == "cold":
                m, it, _ = plan.solve_until(a, tol_f, sched, data_type, threshold, check_every=10)
            else:
                m0 = torch.empty_like(a.real).contiguous()
                for q in range(0, a.shape[0], args.batch):
                    net.predict(a[q:q + args.batch].contiguous(), out=m0[q:q + args.batch])
                m, why, it = plan.solve_warm(a, m0, tol_f, sched, data_type, threshold, check_every=10)
                redone += int((why != 0).sum())
            its.append(it)
            outs.append(m)
        e1.record()
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) / 1e3
        for q, m in enumerate(outs):
            frcs.append(frc_mean(m, Mh[q * cap:q * cap + m.shape[0]]))
        frcs = np.concatenate(frcs)
        full.setdefault(str(tol_f), {})[name] = dict(
            slices_per_s=float(Ah.shape[0] / sec), iterations=its, redone_cold=redone,
            frc_vs_full_cold_min=float(frcs.min()), frc_vs_full_cold_median=float(np.median(frcs)))
        log(f"  all {Ah.shape[0]} held-out slices to tolerance {tol_f:g}, {name}: {full[str(tol_f)][name]}")
    params, g = net.get_params()
    meta = dict(nx=args.nx, thickness=args.thickness, tilts="-60..60 step 2", schedule=list(sched), data_type=data_type,
                threshold=threshold, train_slices=int(n), epochs=args.epochs, batch=args.batch, lr=args.lr,
                heldout_rel_error=float(np.median(err)), heldout_tol=tol, heldout_iters_cold=n_cold,
                heldout_iters_warm=n_warm, heldout_frc_min=float(frc.min()), frc_curve=curve,
                icon_iters_to_frc099_cold=k_cold, icon_iters_to_frc099_warm=k_warm,
                prediction_frc_min=float(f0.min()), frc_curve_warm_no_first_infr=curve0, heldout_slices=int(Ah.shape[0]),
                heldout_to_tol=full)
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    np.savez(args.out, params=params, gain=np.float32(g), meta=json.dumps(meta))
    log(f"saved {args.out}: {json.dumps(meta)}")


if __name__ == "__main__":
    main()
