"""Benchmark of the ICON reconstruction path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the production configuration of the headline metric): a seeded
synthetic tilt series 1024 (x) x 1024 (y) x 300 (z) of 300 ellipsoids and 3000
Gaussian blobs on a 0.1 background, 61 tilts -60..+60 deg step 2 stored sorted
by angle, Gaussian noise SNR 0.1, thickness 300, 300 ICON iterations per
xz-slice (schedule 10,280,10, data type 2, threshold 0).  A step reconstructs
one batch of SLICES_PER_STEP slices: input stage (1-D row NUFFTs, W, adjoint)
plus 300 iterations.  Per step the working set (~20 GB) is far larger than
the 126 MB L2, so no flush is needed between steps.

The iterations' normal operator A^H W A is, by default (--operator toeplitz),
the Toeplitz form: a convolution with the exact kernel of the node set on
the oversampled grid (two 2-D FFT round trips per iteration, no
interpolation); with --operator nufft it is the reference's Gaussian-window
NUFFT pair (three NUFFTs per iteration).  Both are timed in every run (the
other one over min(K, 5) steps), both carry a parity record against the
reference and the FP64 oracle, and the NUFFT pair's HBM GB/s comes from the
nufft run.

value: slices/s with the projection rows already in HBM (device-timed with
CUDA events on the launch stream, max over ranks).  e2e: the same through
icon_reconstruct_host, host (pinned) rows in and host slices out, the copies
inside the timed region.  Under torchrun each rank reconstructs its own
slices (weak scaling; slices are independent, there is no collective on the
data path).

--impl reference: the reference has no CPU implementation of this path, so
the CPU arm is the oracle's float port of it (oracle/icon_oracle_core.c, the
reference's own algorithm restated in C, OpenMP over slices on all host
cores) on a bounded sample of the same workload: one slice per host thread,
the 300-iteration schedule cut into 20 pieces of 15 iterations (the input
stage goes with the first), one piece per step, the image carried from step
to step, so 20 steps run one whole reconstruction of the sample.  value =
slices x (steps / 20) / measured time.  The repo arm's cpu_baseline runs the
same sample through all 20 pieces, timed as a whole.

window_kb4: the same workload with the Kaiser-Bessel window of half-width 4
(8 taps per dimension instead of the reference's 14-tap Gaussian): both
operators' slices/s, its NUFFT pair and its parity record.

Also in the repo arm's line: reference_gpu (the reference's own ICON-GPU,
compiled from its sources for sm_100a into oracle/_ref/, run by wall clock
on a 64-slice stack of the workload, and the agreement of its slices with
this build's) and parity (this build's result on the 16 slices of
tests/golden/cfg2.npz against the reference's and the FP64 oracle's results
for the same 300 iterations).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "slices/s to fixed residual: warm-start vs plain ICON, 1 B200; NUFFT HBM GB/s"
NX, NY, THICK = 1024, 1024, 300
SCHED = (10, 280, 10)
DATA_TYPE, THRESHOLD = 2, 0.0
SLICES_PER_STEP = 256   # one launch takes 32 groups of 8 slices (1.4% faster than 16 groups)
WORKLOAD = ("plain ICON, 1024x1024x300 phantom (300 ellipsoids + 3000 blobs, background 0.1), "
            "61 tilts -60..60 step 2, SNR 0.1, thickness 300, 300 iterations (10,280,10)")
# NUFFT forward+adjoint pair, algorithmic bytes per slice (model of the
# reference's staged NUFFT: B_fwdR + B_adj, complex 8 B, real 4 B).
N0, N1, n0, n1, M = NX, THICK, 2048, 1024, NX * 61
PAIR_MODEL_BYTES = (4 * N0 * N1 + 16 * N0 * n1 + 16 * n0 * n1 + 8 * M) + (8 * M + 16 * n0 * n1 + 16 * N0 * n1 + 8 * N0 * N1)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def bf16_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return {"peak_tflops": float(json.load(open(p))["bf16_tflops"]), "peak_source": "measured (cuBLAS bf16 burst)"}
    return {"peak_tflops": 1590.0, "peak_source": "fallback"}


# Traced kernel kind -> (committed ncu summary, line holding its per-slot DRAM bytes).
PROFILE_LINES = {"ypass_toep": ("ypass_toep_cfg2.txt", "dram_bytes_per_slot"),
                 "ypass_toep_quad": ("ypass_toep_cfg2.txt", "dram_bytes_per_slot_mode1"),
                 "xtoep_mid": ("xtoep_cfg2.txt", "dram_bytes_per_slot"),
                 "xtoep_fwd": ("xtoep_cfg2.txt", "dram_bytes_per_slot_mode0")}


def dram_traffic_from_profile(kind):
    """Per-slot DRAM bytes of a kernel from a committed ncu summary
    (profiles/<kind>_cfg2.txt, or the file PROFILE_LINES names; a line
    '<key>: <float>')."""
    name, key = PROFILE_LINES.get(kind, (f"{kind}_cfg2.txt", "dram_bytes_per_slot"))
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith(key + ":"):
            return float(line.split(":", 1)[1])
    return None


class ClockSampler:
    def __init__(self, uuid):
        self.uuid = uuid
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 8 or (self.uuid and f[0] != self.uuid):
                    continue
                rows.append(f)
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[4 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def make_rows(ys, device):
    from feilab_b200 import synth
    rows, tilts, thick, desc = synth.series("cfg2", device=device, ys=ys)
    return rows, tilts


NPIECES, PIECE_ITERS = 20, 15    # the 300-iteration schedule in timed pieces


def schedule_piece(k, sched=SCHED, per=PIECE_ITERS):
    """(INFR before, ICON, INFR after) counts of iterations [k*per, (k+1)*per)
    of the schedule (Iteration2.cu:129-132)."""
    a, b, c = sched
    lo, hi = k * per, (k + 1) * per

    def ov(x0, x1):
        return max(0, min(hi, x1) - max(lo, x0))
    return ov(0, a), ov(a, a + b), ov(a + b, a + b + c)


class CpuSchedule:
    """The oracle's float port on a sample of slices (OpenMP over slices), run
    piece by piece: step() runs the next piece of the schedule (piece 0 starts
    with the input stage and m = 0); the image is carried between pieces, so
    NPIECES steps make one whole reconstruction; then the next step starts a
    new one."""

    def __init__(self, tilts, rows_np, nthreads=0):
        from oracle.oracle import OraclePlan
        self.p = OraclePlan(NX, THICK, tilts, "f32")
        self.rows = np.ascontiguousarray(rows_np, np.float32)
        self.S = self.rows.shape[0]
        self.nthreads = nthreads
        self.k = 0
        self.A = self.m = None

    def step(self):
        if self.k == 0:
            self.A = self.p.rhs_batch(self.rows, self.nthreads)
            self.m = np.zeros((self.S, NX, THICK), np.float32)
        self.p.solve_batch(self.A, self.m, schedule_piece(self.k), DATA_TYPE, THRESHOLD, self.nthreads)
        self.k = (self.k + 1) % NPIECES

    @property
    def threads(self):
        return self.p.threads_used


def cpu_rows(tilts, rows_dev=None):
    """One slice per host thread: the first slices of the workload."""
    ncpu = os.cpu_count() or 1
    if rows_dev is not None:
        return rows_dev.reshape(-1, len(tilts), NX)[:ncpu].cpu().numpy()
    rows, _ = make_rows(list(range(ncpu)), "cpu")
    return rows.numpy()


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from feilab_b200 import synth
    tilts = synth.tilt_angles(-60, 60, 2)
    rows_np = cpu_rows(tilts)
    cs = CpuSchedule(tilts, rows_np)
    for _ in range(args.warmup):
        cs.step()
    cs.k = 0                                   # the timed steps start a reconstruction
    times = []
    t_all = time.perf_counter()
    for _ in range(args.steps):
        t0 = time.perf_counter()
        cs.step()
        times.append(time.perf_counter() - t0)
    total = time.perf_counter() - t_all
    value = cs.S * (args.steps / NPIECES) / total
    sample = (f"{cs.S} slices of the workload (one per host thread); step i runs iterations "
              f"{PIECE_ITERS}*(i mod {NPIECES}) .. +{PIECE_ITERS} of the {sum(SCHED)}-iteration schedule "
              f"(the input stage with the first), the image carried between steps; {args.steps} timed steps = "
              f"{args.steps / NPIECES:g} reconstructions of the sample; value = slices x steps/{NPIECES} / measured time")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "slices/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3,
            "ms_per_step_minmax": [round(min(times) * 1e3, 1), round(max(times) * 1e3, 1)],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "implementation": "oracle float port of the reference algorithm "
                       "(no CPU build of the path exists in the reference)"},
            "cpu_baseline": {"value": value, "unit": "slices/s", "cores": cs.threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "slices/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline_full(tilts, rows_np):
    """One whole reconstruction (input stage + 300 iterations) of one slice per
    host thread by the oracle's float port, timed as a whole."""
    cs = CpuSchedule(tilts, rows_np)
    t0 = time.perf_counter()
    for _ in range(NPIECES):
        cs.step()
    t = time.perf_counter() - t0
    return {"value": cs.S / t, "unit": "slices/s", "cores": cs.threads, "kind": "port",
            "seconds": round(t, 2),
            "sample": f"{cs.S} slices of the workload (one per host thread), input stage + all {sum(SCHED)} "
                      f"iterations, measured wall time"}


def reference_gpu_leg(tilts, rows_dev, plan, nslices=64):
    """The reference ICON-GPU (oracle/_ref/ICON-GPU, built from the reference
    sources for sm_100a) on an MRC stack of `nslices` slices of the workload,
    -iter 10,280,10 -d 2 -thr 0 -thi 300 -skipCV 1 -g 0, timed by wall clock
    around the process; its slice files against this build's slices."""
    from feilab_b200 import mrc
    exe = os.path.join(ROOT, "oracle", "_ref", "ICON-GPU")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/ICON-GPU not built (oracle/build_ref.sh needs the reference sources)"}
    rows = rows_dev[:nslices].contiguous()
    rows_np = rows.cpu().numpy()
    with tempfile.TemporaryDirectory() as d:
        stack, tlt, out = os.path.join(d, "stack.mrc"), os.path.join(d, "s.tlt"), os.path.join(d, "out")
        os.makedirs(out)
        mrc.write_tilt_series(stack, rows_np)
        mrc.write_tlt(tlt, tilts)
        a, b, c = SCHED
        cmd = [exe, "-i", stack, "-t", tlt, "-o", out, "-s", f"0,{nslices - 1}", "-iter", f"{a},{b},{c}",
               "-d", str(DATA_TYPE), "-thr", str(THRESHOLD), "-g", "0", "-thi", str(THICK), "-skipCV", "1"]
        t0 = time.perf_counter()
        p = subprocess.run(cmd, capture_output=True, text=True)
        wall = time.perf_counter() - t0
        if p.returncode != 0:
            return {"unavailable": f"ICON-GPU exited with {p.returncode}: {p.stderr[-200:]}"}
        per = []
        for line in p.stdout.splitlines():
            if line.startswith("slice") and "finished" in line and "time" in line:
                try:
                    per.append(float(line.rsplit("time", 1)[1].strip()))
                except ValueError:
                    pass
        ref = np.stack([mrc.read(os.path.join(out, "reconstruction", f"mid{y:05d}.mrc"))[1][0].T
                        for y in range(nslices)])            # (S, N0, N1), Y fastest
    A = plan.prepare_rhs(rows)
    ours = plan.solve(A, SCHED, DATA_TYPE, THRESHOLD).cpu().numpy()
    rel = [float(np.linalg.norm(ours[s] - ref[s]) / max(np.linalg.norm(ref[s]), 1e-30)) for s in range(nslices)]
    res = {"value": nslices / wall, "unit": "slices/s", "slices": nslices, "wall_s": round(wall, 2),
           "command": "ICON-GPU -s 0,%d -iter %d,%d,%d -d %d -thr %g -g 0 -thi %d -skipCV 1" %
                      (nslices - 1, a, b, c, DATA_TYPE, THRESHOLD, THICK),
           "rel_l2_vs_this_build_max": max(rel), "rel_l2_vs_this_build_mean": float(np.mean(rel))}
    if per:
        res["solve_s_per_slice_mean"] = float(np.mean(per))
        res["value_solve_only"] = 1.0 / float(np.mean(per))
    return res


def parity_leg(plan_factory, operator):
    """This build's reconstruction of the 16 slices of tests/golden/cfg2.npz
    (seeded random slices of the workload, full schedule) with the given
    normal operator, against the reference's result (ref_harness) and the
    FP64 oracle's, same iterations."""
    import torch
    from feilab_b200.train_warmstart import frc_mean
    path = os.path.join(ROOT, "tests", "golden", "cfg2.npz")
    if not os.path.exists(path):
        return {"unavailable": "tests/golden/cfg2.npz not present"}
    z = np.load(path)
    S = int(z["S"])
    plan = plan_factory(S)
    plan.set_operator(operator)
    rows = torch.from_numpy(np.ascontiguousarray(z["rows"])).cuda()
    m = plan.solve(plan.prepare_rhs(rows), tuple(int(v) for v in z["sched"]), int(z["data_type"]),
                   float(z["threshold"])).cpu()
    plan.close()
    m64 = torch.from_numpy(z["ref_m"].astype(np.float64) +
                           z["fp64_minus_ref_q"].astype(np.float64) * float(z["fp64_minus_ref_step"]))
    mref = torch.from_numpy(z["ref_m"].astype(np.float32))

    def rel(a, b):
        return [float(((a[s].double() - b[s].double()).norm() / b[s].double().norm()).item()) for s in range(S)]
    r64, rref = rel(m, m64), rel(m, mref)
    return {"slices": S, "iterations": int(sum(int(v) for v in z["sched"])), "y": z["ys"].tolist(),
            "rel_l2_vs_fp64_max": max(r64), "rel_l2_vs_fp64_mean": float(np.mean(r64)),
            "frc_vs_fp64_min": float(frc_mean(m, m64).min()),
            "rel_l2_vs_reference_max": max(rref), "rel_l2_vs_reference_mean": float(np.mean(rref)),
            "frc_vs_reference_min": float(frc_mean(m, mref).min()),
            "reference_vs_fp64_max": max(rel(mref, m64))}


def run_ours(args):
    import torch
    import torch.distributed as dist
    from feilab_b200 import icon, sharding

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)

    S = SLICES_PER_STEP
    nsteps = args.warmup + args.steps
    # This rank's slices: disjoint y ranges per rank (weak scaling).
    ys = sharding.rank_slices(rank, world, nsteps, S, NY)
    rows, tilts = make_rows(ys, dev)
    rows = rows.view(nsteps, S, len(tilts), NX).contiguous()
    plan = icon.IconPlan(NX, THICK, tilts, capacity=S, device=local)
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return sharding.max_over_ranks(x, world, device=dev)

    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass

    def timed_device(op, steps, plan=plan):
        """Device-resident rows in, `steps` timed steps (input stage +
        schedule), CUDA events on the launch stream, max over ranks."""
        plan.set_operator(op)
        for i in range(args.warmup):
            plan.solve(plan.prepare_rhs(rows[i]), SCHED, DATA_TYPE, THRESHOLD)
        barrier()
        plan.trace(True)
        plan.trace_read()
        launches0 = plan.launch_count()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(uuid) as clk:
            barrier()
            ev0.record(stream)
            for i in range(args.warmup, args.warmup + steps):
                plan.solve(plan.prepare_rhs(rows[i]), SCHED, DATA_TYPE, THRESHOLD)
            ev1.record(stream)
            barrier()
        launches = plan.launch_count() - launches0
        trace = plan.trace_read()
        plan.trace(False)
        t = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
        return {"value": sharding.job_rate(world, S, steps, t), "t": t, "steps": steps, "trace": trace,
                "launches": launches, "clocks": clk.summary()}

    h_rows = torch.empty((nsteps, S, len(tilts), NX), dtype=torch.float32, pin_memory=True)
    h_rows.copy_(rows.cpu())
    h_out = torch.empty((S, NX, THICK), dtype=torch.float32, pin_memory=True)

    def timed_e2e(op):
        """The same through icon_reconstruct_host: pinned host rows in, host
        slices out, the copies inside the timed region."""
        plan.set_operator(op)
        for i in range(args.warmup):
            plan.reconstruct_host(h_rows[i], SCHED, DATA_TYPE, THRESHOLD, out=h_out, stream=stream.cuda_stream)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(args.warmup, nsteps):
            plan.reconstruct_host(h_rows[i], SCHED, DATA_TYPE, THRESHOLD, out=h_out, stream=stream.cuda_stream)
        e1.record(stream)
        barrier()
        return sharding.job_rate(world, S, args.steps, max_over_ranks(e0.elapsed_time(e1) / 1e3))

    slots = plan.B * ((S + plan.B - 1) // plan.B)

    def kernel_table(trace):
        total_ms = sum(v[1] for v in trace.values())
        return {k: {"launches": v[0], "ms": round(v[1], 3), "share": round(v[1] / total_ms, 4),
                    "gbs": round(v[2] / (v[1] / 1e3) / 1e9, 1) if v[1] > 0 and v[2] > 0 else None}
                for k, v in trace.items() if v[0] > 0}

    peak, peak_kind = measured_peaks()
    # The headline operator is timed over the K steps, device-resident and end
    # to end; the other operator over min(K, 5) steps, device-resident.
    ops = [args.operator] + [o for o in ("nufft", "toeplitz") if o != args.operator]
    runs = {}
    for op in ops:
        headline = op == args.operator
        runs[op] = timed_device(op, args.steps if headline else min(args.steps, 5))
        runs[op]["e2e"] = timed_e2e(op) if headline else None
    head = runs[args.operator]
    value, t_dev, trace, e2e = head["value"], head["t"], head["trace"], head["e2e"]

    # ---- roofline of the headline operator's dominant kernel ---------------
    dom = max((k for k in trace if trace[k][0] > 0), key=lambda k: trace[k][1])
    cnt, ms, by = trace[dom]
    achieved = (by / cnt) / (ms / cnt / 1e3) / 1e9
    traffic_slot = dram_traffic_from_profile(dom)
    # NUFFT pair (forward R2C + adjoint) per slice-iteration: the model bytes
    # of the reference's staged NUFFT over the time of our fused kernels, from
    # the run with the NUFFT operator.
    def pair(run):
        tn = run["trace"]
        fwd_ms = (tn["xpass_fwd"][1] + tn["ypass_fwd"][1] + tn["interp_fin"][1]) / 2.0
        adj_ms = tn["ypass_adj"][1] + tn["xpass_adj"][1]
        slice_iters = slots * run["steps"] * sum(SCHED)
        pair_s = (fwd_ms + adj_ms) / 1e3 / slice_iters
        pair_gbs = PAIR_MODEL_BYTES / pair_s / 1e9
        return {"model_bytes_per_slice": PAIR_MODEL_BYTES, "gbs": round(pair_gbs, 1),
                "frac": round(pair_gbs / peak, 4), "us_per_slice": round(pair_s * 1e6, 3)}
    # FP32 work of the dominant Toeplitz y-pass (its bound is the FP32 pipe, not
    # DRAM): per slot two complex FFTs of n1 points (5 n log2 n flops each) per
    # grid row, against the SIMT FP32 peak of the device at the sampled clock.
    fp32 = None
    if dom == "ypass_toep":
        import math
        props = torch.cuda.get_device_properties(local)
        mhz = (head["clocks"] or {}).get("sm_max_mhz") or 1965.0
        peak_tf = props.multi_processor_count * 128 * 2 * mhz * 1e6 / 1e12
        flops = slots * n0 * 2 * 5 * n1 * math.log2(n1)
        tf = flops / (ms / cnt / 1e3) / 1e12
        fp32 = {"model_flops_per_launch": flops, "achieved_tflops": round(tf, 2), "peak_tflops": round(peak_tf, 1),
                "frac": round(tf / peak_tf, 4), "peak_source": "SMs x 128 FP32 lanes x 2 x max SM clock"}

    line = {"metric": METRIC, "value": value, "unit": "slices/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_dev / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "slices_per_step": S, "iterations": sum(SCHED), "nx": NX, "thickness": THICK,
                       "tilts": len(tilts), "slices_per_group": plan.B, "parallelism": f"slices sharded over {world} GPU(s)",
                       "operator": args.operator,
                       "l2": "inputs larger than L2 (per-step working set ~20 GB), no flush needed",
                       "stop": "fixed iteration count (the reference has no residual test)"},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                         "traffic": (traffic_slot * slots if traffic_slot else None),
                         "algorithmic_bytes_per_launch": by / cnt, "fp32": fp32},
            "nufft_pair": pair(runs["nufft"]),
            "kernels": kernel_table(trace),
            "e2e": {"value": e2e, "unit": "slices/s", "h2d_bytes_per_step": int(S * len(tilts) * NX * 4),
                    "d2h_bytes_per_step": int(S * NX * THICK * 4)},
            "gpu_launches": int(head["launches"]),
            "device_error": plan.device_error(),   # bounded TMA waits that ran out (0: none)
            "clocks": head["clocks"],
            "operators": {op: {"value": r["value"], "e2e": r["e2e"], "steps": r["steps"],
                               "ms_per_step": r["t"] / r["steps"] * 1e3,
                               "kernels": kernel_table(r["trace"]), "clocks": r["clocks"]} for op, r in runs.items()}}
    plan.set_operator(args.operator)
    if not args.no_kb:
        # The Kaiser-Bessel window mode (half-width 4, 8 taps): both operators
        # over min(K, 3) steps on the same rows, its NUFFT pair, and its result
        # on the parity slices against the reference's and the FP64 oracle's
        # (both Gaussian).
        kplan = icon.IconPlan(NX, THICK, tilts, capacity=S, device=local, window="kb4")
        kruns = {op: timed_device(op, min(args.steps, 3), plan=kplan) for op in ("toeplitz", "nufft")}
        kplan.close()
        line["window_kb4"] = {op: {"value": r["value"], "steps": r["steps"], "ms_per_step": r["t"] / r["steps"] * 1e3,
                                   "kernels": kernel_table(r["trace"])} for op, r in kruns.items()}
        line["window_kb4"]["nufft_pair"] = pair(kruns["nufft"])
        if rank == 0:
            line["window_kb4"]["parity"] = {
                op: parity_leg(lambda n: icon.IconPlan(NX, THICK, tilts, capacity=n, device=local, window="kb4"), op)
                for op in ops}
    if not args.no_warm:
        line["warm_start"] = warm_start_leg(args, plan, rows, stream, barrier, max_over_ranks, world, S)
    if rank == 0:
        line["parity"] = {op: parity_leg(lambda n: icon.IconPlan(NX, THICK, tilts, capacity=n, device=local), op)
                          for op in ops}
    if rank == 0 and world == 1 and args.uneven_scale > 0:
        line["uneven_batch"] = uneven_leg(args, args.uneven_scale)
    if rank == 0 and world == 1 and args.loo_scale > 0:
        line["loo_sweep"] = loo_leg(args, args.loo_scale)
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        line["reference_gpu"] = reference_gpu_leg(tilts, rows[0], plan)
        if "value" in line["reference_gpu"]:
            line["reference_gpu"]["speedup_e2e"] = round(e2e / line["reference_gpu"]["value"], 2)
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline_full(tilts, cpu_rows(tilts, rows))
    if rank == 0:
        print(json.dumps(line), flush=True)
    plan.close()
    if world > 1:
        dist.destroy_process_group()


WARM_TOLS, WARM_CHECK = (0.03, 0.02), 10   # relative-step tolerances of the warm and cold solves


def conv_rates(dev):
    """CUDA-event TFLOP/s of the network's tensor-core 3x3 convolution
    (icon_ws_conv3x3: tcgen05.mma fed by TMA, BF16 in, FP32 accumulate) on
    the shapes of its levels for 32 images of 304 x 1024."""
    import torch
    from feilab_b200 import warmstart
    out = {}
    for c, H, W in ((16, 304, 1024), (32, 152, 512), (64, 76, 256), (128, 38, 128)):
        x = torch.randn((32, H, W, c), device=dev).to(torch.bfloat16)
        w = (0.05 * torch.randn((9, c, c), device=dev)).to(torch.bfloat16)
        for _ in range(3):
            warmstart.conv3x3(x, w)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 20
        e0.record()
        for _ in range(reps):
            warmstart.conv3x3(x, w)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        tf = 2.0 * 32 * H * W * c * c * 9 / (ms / 1e3) / 1e12
        out[f"{c}ch_{H}x{W}"] = {"ms": round(ms, 4), "tflops": round(tf, 1)}
    return out


def warm_start_leg(args, plan, rows, stream, barrier, max_over_ranks, world, S):
    """The learned warm start against the plain solve on the same slices,
    both stopped at each relative-step tolerance of WARM_TOLS: cold = input stage
    + icon_solve_until from m = 0; warm = input stage + network +
    icon_solve_warm (the warm solve to the tolerance, the per-slice
    acceptance test and the cold redo of rejected slices).  Device-resident
    rows, CUDA events; the FRC of both against the full-schedule cold result,
    the slices the acceptance test sent back, and the held-out comparison
    stored with the weights."""
    import torch
    from feilab_b200 import sharding, warmstart
    from feilab_b200.train_warmstart import frc_mean
    try:
        params, gain, meta = warmstart.load_weights(nx=NX, thickness=THICK)
    except OSError as e:
        return {"unavailable": f"no trained weights: {e}"}
    cap = 32
    net = warmstart.Network(plan, capacity=cap)
    net.set_params(params, gain)

    def run(tol):
        def cold(i):
            A = plan.prepare_rhs(rows[i])
            m, it, _ = plan.solve_until(A, tol, SCHED, DATA_TYPE, THRESHOLD, check_every=WARM_CHECK)
            return A, m, it, None

        def warm(i):
            A = plan.prepare_rhs(rows[i])
            m0 = torch.empty((S, NX, THICK), dtype=torch.float32, device=A.device)
            for s0 in range(0, S, cap):
                net.predict(A[s0:s0 + cap], out=m0[s0:s0 + cap])
            m, why, it = plan.solve_warm(A, m0, tol, SCHED, DATA_TYPE, THRESHOLD, check_every=WARM_CHECK)
            return A, m, it, why

        res = {}
        for name, fn in (("cold_to_tol", cold), ("warm_to_tol", warm)):
            for i in range(min(args.warmup, 1)):
                fn(i)
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            its, redone = [], 0
            for i in range(args.warmup, args.warmup + steps):
                A, m, it, why = fn(i)
                its.append(it)
                if why is not None:
                    redone += int((why != 0).sum())
            e1.record(stream)
            barrier()
            t = max_over_ranks(e0.elapsed_time(e1) / 1e3)
            res[name] = {"value": sharding.job_rate(world, S, steps, t), "unit": "slices/s", "iterations": its,
                         "m_last": m}
            if why is not None:
                res[name]["redone_cold"] = redone
                res[name]["slices"] = S * steps
        # both against the full-schedule cold result of the last step's slices
        m_full = plan.solve(A, SCHED, DATA_TYPE, THRESHOLD)
        torch.cuda.synchronize()
        for name in res:
            f = frc_mean(res[name].pop("m_last")[:16].double().cpu(), m_full[:16].double().cpu())
            res[name]["frc_vs_full_cold_min"] = round(float(f.min()), 4)
        res["gain"] = round(res["warm_to_tol"]["value"] / res["cold_to_tol"]["value"], 3)
        return res, A

    steps = min(args.steps, 3)
    by_tol = {}
    for tol in WARM_TOLS:
        by_tol[str(tol)], A = run(tol)
    # inference alone
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    m0 = torch.empty((S, NX, THICK), dtype=torch.float32, device=A.device)
    f0.record(stream)
    for s0 in range(0, S, cap):
        net.predict(A[s0:s0 + cap], out=m0[s0:s0 + cap])
    f1.record(stream)
    torch.cuda.synchronize()
    net.close()
    return {"check_every": WARM_CHECK, "by_tolerance": by_tol,
            "inference_ms_per_slice": round(f0.elapsed_time(f1) / S, 4),
            "conv_tensor_core": {**conv_rates(A.device), **bf16_peak()},
            "heldout_icon_iterations_to_frc_0.99": {"cold": meta.get("icon_iters_to_frc099_cold"),
                                                    "warm": meta.get("icon_iters_to_frc099_warm")},
            "heldout_prediction_frc_min": meta.get("prediction_frc_min"),
            "weights": f"feilab_b200/weights/warmstart_{NX}x{THICK}.npz (trained on {meta.get('train_slices')} slices)"}


TUNE_CACHE = os.path.join(ROOT, "feilab_b200", "tune", "b200_uneven.txt")


def uneven_leg(args, slice_scale):
    """The uneven multi-series workload (24 seeded series: widths 256-2048,
    64-512 slices times slice_scale, thickness 100-400, tilt ranges +-45..70
    with 10% of the tilts dropped, SNR 0.1-0.5; the full schedule 10,280,10)
    through icon_batch: all series at once from CUDA graphs with the tuned
    slices per group and per launch (tuning from the committed cache file,
    shapes missing from it timed here), against the same series one after
    another (same plans, direct launches).  Wall time around the host call,
    pinned rows in and slices out, so copies are inside."""
    import torch
    from feilab_b200 import icon, synth
    t0 = time.perf_counter()
    ser = synth.uneven_batch(24, seed=3003, slice_scale=slice_scale, device="cuda")
    gen_s = time.perf_counter() - t0
    shapes = [(d["nx"], d["thickness"], d["tilts"], d["slices"]) for d in ser]
    rows = [d["rows"].cpu().pin_memory() for d in ser]
    del ser
    torch.cuda.empty_cache()
    if args.tune_write:
        cache, tune = args.tune_write, 2
    else:
        cache, tune = (TUNE_CACHE if os.path.exists(TUNE_CACHE) else None), 1
    t0 = time.perf_counter()
    b = icon.IconBatch(shapes, operator="toeplitz", tune_cache=cache, tune=tune)
    setup_s = time.perf_counter() - t0
    out = [torch.empty((sl, nx, th), dtype=torch.float32, pin_memory=True) for nx, th, _, sl in shapes]
    total = sum(sl for *_, sl in shapes)
    res = {}
    for mode, conc in (("concurrent_graphs", True), ("one_series_at_a_time", False)):
        # warm-up: every graph kind of the schedule captured, every chunk size met
        b.reconstruct(rows, (2, 2, 2), DATA_TYPE, THRESHOLD, out=out, concurrent=conc)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.reconstruct(rows, SCHED, DATA_TYPE, THRESHOLD, out=out, concurrent=conc)
        t = time.perf_counter() - t0
        res[mode] = {"value": total / t, "unit": "slices/s", "seconds": round(t, 3)}
    tun = [b.tuning(k) for k in range(len(shapes))]
    b.close()
    # The same concurrent run with the built-in defaults (8 slices per group
    # where the size allows, 128 slices per launch): what the tuning gains.
    b = icon.IconBatch(shapes, operator="toeplitz", tune_cache=None, tune=0)
    b.reconstruct(rows, (2, 2, 2), DATA_TYPE, THRESHOLD, out=out, concurrent=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b.reconstruct(rows, SCHED, DATA_TYPE, THRESHOLD, out=out, concurrent=True)
    t = time.perf_counter() - t0
    res["concurrent_default_tuning"] = {"value": total / t, "unit": "slices/s", "seconds": round(t, 3)}
    b.close()
    return {"workload": f"24 seeded series, slice_scale {slice_scale}", "slices": total,
            "series": [{"nx": nx, "thickness": th, "tilts": len(t), "slices": sl, "group": tu["group"],
                        "chunk": tu["chunk"], "tuned": tu["tuned"]} for (nx, th, t, sl), tu in zip(shapes, tun)],
            **res, "speedup_concurrent": round(res["concurrent_graphs"]["value"] /
                                               res["one_series_at_a_time"]["value"], 3),
            "speedup_tuning": round(res["concurrent_graphs"]["value"] /
                                    res["concurrent_default_tuning"]["value"], 3),
            "setup_s": round(setup_s, 2), "generate_s": round(gen_s, 2),
            "iterations": sum(SCHED), "operator": "toeplitz"}


def loo_leg(args, slice_scale):
    """Leave-one-out cross validation of the 1024-wide, 61-tilt workload
    (SNR 0.1, thickness 300, the full 10,280,10 schedule) on 512 * slice_scale
    slices: every tilt left out in turn, 61 x slices solves.  The batched
    sweep (icon_loo_sweep: one plan over all tilts, one slice group per
    (omitted tilt, 8 slices) with that tilt's weights at 0, all solves in one
    batched schedule) against the plain sweep (a plan rebuilt without each
    tilt, its slices solved and reprojected at the omitted angle, as the
    reference's Lib_2D_crossV2 does for its one tilt), both cold-started and
    with the Toeplitz operator; wall time around each, per-tilt FRC of both."""
    import torch
    from feilab_b200 import icon, tools
    S = max(8, int(round(512 * slice_scale)))
    rows, tilts = make_rows(list(range(S)), "cuda")
    rows = rows.cpu().numpy()
    nz = len(tilts)
    t0 = time.perf_counter()
    frc_b, _, _ = tools.loo_sweep(rows, THICK, tilts, SCHED, DATA_TYPE, THRESHOLD, capacity=SLICES_PER_STEP,
                                  operator="toeplitz")
    t_b = time.perf_counter() - t0
    cap = min(SLICES_PER_STEP, S)
    frc_p = np.zeros_like(frc_b)
    t0 = time.perf_counter()
    for k in range(nz):
        keep = [i for i in range(nz) if i != k]
        p = icon.IconPlan(NX, THICK, tilts[keep], capacity=cap)
        p.set_operator("toeplitz")
        rp = np.zeros((S, NX), np.float32)
        for s0 in range(0, S, cap):
            n = min(cap, S - s0)
            r = torch.from_numpy(np.ascontiguousarray(rows[s0:s0 + n][:, keep])).cuda()
            m = p.solve(p.prepare_rhs(r), SCHED, DATA_TYPE, THRESHOLD)
            rp[s0:s0 + n] = p.reproject(m, float(tilts[k])).cpu().numpy()
        p.close()
        frc_p[k] = tools.frc(rows[:, k, :], rp)
    t_p = time.perf_counter() - t0
    mean_b, mean_p = frc_b[:, 1:].mean(axis=1), frc_p[:, 1:].mean(axis=1)
    return {"workload": f"1024 wide x {S} slices x {nz} tilts (-60..60 step 2), SNR 0.1, thickness {THICK}, "
                        f"{sum(SCHED)} iterations, every tilt left out in turn", "solves": nz * S,
            "batched": {"seconds": round(t_b, 2), "solves_per_s": round(nz * S / t_b, 1)},
            "plain_per_tilt_plans": {"seconds": round(t_p, 2), "solves_per_s": round(nz * S / t_p, 1)},
            "speedup": round(t_p / t_b, 3),
            "frc_mean_per_tilt": {"batched_min": round(float(mean_b.min()), 4),
                                  "batched_max": round(float(mean_b.max()), 4),
                                  "max_abs_diff_vs_plain": float(np.abs(frc_b - frc_p).max())},
            "frc_mean_per_tilt_batched": [round(float(v), 4) for v in mean_b],
            "operator": "toeplitz", "start": "m = 0 (a warm start would leak the held-out projection)"}


def run_profile_case(args):
    """Small case for ncu captures: --profile-slices slices of the workload
    (32 by default: the grid intermediate of every kernel, 157 MB, is larger
    than L2; under 1 GB on the device in all), the input stage and 2
    iterations; prints the traced kernel times."""
    import torch
    from feilab_b200 import icon
    torch.cuda.set_device(0)
    S = args.profile_slices
    rows, tilts = make_rows(list(range(S)), "cuda")
    plan = icon.IconPlan(NX, THICK, tilts, capacity=S)
    plan.set_operator(args.operator)
    plan.trace(True)
    A = plan.prepare_rhs(rows)
    plan.solve(A, (0, 2, 0), DATA_TYPE, THRESHOLD)
    torch.cuda.synchronize()
    for k, v in plan.trace_read().items():
        if v[0]:
            print(f"{k:12s} launches {v[0]:4d}  ms {v[1]:9.3f}  algorithmic GB/s {v[2] / (v[1] / 1e3) / 1e9 if v[2] else 0:8.1f}")
    plan.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-reference-gpu", action="store_true", help="skip the reference ICON-GPU leg")
    ap.add_argument("--no-kb", action="store_true", help="skip the Kaiser-Bessel window leg")
    ap.add_argument("--no-warm", action="store_true", help="skip the warm-start leg")
    ap.add_argument("--operator", default="toeplitz", choices=["nufft", "toeplitz"],
                    help="normal operator of the headline run (the other is timed beside it)")
    ap.add_argument("--uneven-scale", type=float, default=0.25,
                    help="slice-count scale of the 24-series uneven batch leg (0 skips it; 1 is the full workload)")
    ap.add_argument("--uneven-only", action="store_true", help="run the uneven batch leg only and print it")
    ap.add_argument("--loo-scale", type=float, default=1.0 / 16,
                    help="slice-count scale of the leave-one-out leg (512 slices x scale; 0 skips it)")
    ap.add_argument("--loo-only", action="store_true", help="run the leave-one-out leg only and print it")
    ap.add_argument("--tune-write", default=None,
                    help="tuning cache file to read and extend (time every shape missing from it)")
    ap.add_argument("--profile", action="store_true", help="run the small ncu case only")
    ap.add_argument("--profile-slices", type=int, default=32, help="slices of the --profile case")
    args = ap.parse_args()
    if args.profile:
        run_profile_case(args)
        return
    if args.uneven_only:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps({"uneven_batch": uneven_leg(args, args.uneven_scale)}), flush=True)
        return
    if args.loo_only:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps({"loo_sweep": loo_leg(args, args.loo_scale)}), flush=True)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
