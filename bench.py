"""Benchmark: orientation-solves/s of the DDA-FFT hot path on B200.

Workload (one orientation-solve = one iteration of the reference's sample loop,
main.cpp:806-985): a 64^3 ellipsoid with b/a = 0.7, c/a = 0.5, x = 6, m = 1.55+0.005i,
CM polarisability, CG, Error_max 1e-3, Max_Step 20, 1 scattering plane, theta 0..180 step
10, Monte-Carlo orientations from the reference's own sampler (seed 7).  Both incident
polarisations are solved to Error_max, then CabsCext, the far field at 19 angles and the
Jones -> Mueller conversion.  One step = one batch of --batch orientations (2 x batch
right-hand sides) in one batched call of libddagpu.

Printed line (rank 0): value = batched orientation-solves/s with the occupancy resident
in HBM (device time, CUDA events on the library's stream, max over ranks); e2e = the same
through the public C ABI with the host occupancy uploaded and the results read back every
step; plain_gpu = the drop-in path (one ddagpu_dda_fft call per polarisation); roofline =
the matvec (K1+K2+K3) on the same batch; cpu_baseline = the reference's own sample loop on
the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GRID, X, MAT, BA, CA, SEED = 64, 6.0, (1.55, 0.005), 0.7, 0.5, 7
METRIC = "orientation-solves/s at 64^3, batched+mixed vs plain GPU at Error_max 1e-3"
WORKLOAD = ("MC orientations (seed 7) of a 64^3 ellipsoid b/a=0.7 c/a=0.5, x=6, m=1.55+0.005i, "
            "CM, CG, Error_max 1e-3, Max_Step 20, 1 plane, 19 angles, both polarisations")


def ellipsoid_occ(n=GRID, b_a=BA, c_a=CA):
    """iGenerateEllipsoid (particle.cpp:408-444): cell centres inside the ellipsoid."""
    f = np.float32
    c = f(f(n) / f(2.0) - f(0.5))
    a = f(n)
    b, cc = f(a * f(b_a)), f(a * f(c_a))
    a2, b2, c2 = f(a / f(2)) ** 2, f(b / f(2)) ** 2, f(cc / f(2)) ** 2
    i = np.arange(n, dtype=f)[:, None, None] - c
    j = np.arange(n, dtype=f)[None, :, None] - c
    k = np.arange(n, dtype=f)[None, None, :] - c
    return (((i * i) / a2 + (j * j) / b2) + (k * k) / c2 <= f(1.0)).astype(np.int8)


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        """Start sampling every 50 ms and return once the first sample has arrived (so that
        sampling is running when the timed region begins); samples from then on count."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        self.first = len(self.lines)

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        """Stop sampling; a timed region shorter than the sampling period still gets the
        sample taken right after it (waited for, up to 0.5 s)."""
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        t0 = time.time()
        while len(self.lines) <= self.first and time.time() - t0 < 0.5 and self.proc.poll() is None:
            time.sleep(0.005)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[self.first:]:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ reference / CPU arm
def cpu_reference(n_samples: int, threads: int):
    """The reference's own sample loop (oracle/_ref, physicist2018/dda-fft compiled from its
    sources) on this workload; returns (orientation-solves/s, kind, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as P
    if os.path.exists(P.REF_SO):
        R = P.RefLib()
        cfg = P.make_run_cfg(grid=GRID, target=2, b_a=BA, c_a=CA, x=X, materials=(MAT,),
                             orientation=1, seed=SEED)
        secs, *_ = R.run_samples(cfg, n_samples, threads)
        return n_samples / secs, "reference", secs, threads
    O = P.Oracle()   # the FP64 restatement, single thread
    t0 = time.perf_counter()
    P.orientation_solves(O, GRID, X, [MAT], n_samples, target=2, b_a=BA, c_a=CA, orientation=1,
                         seed=SEED)
    secs = time.perf_counter() - t0
    return n_samples / secs, "port", secs, 1


def cross_check(ctx, occ, n):
    """Both arms on the same orientations: the first n draws of worker 0's stream (seed 7),
    through this library and through the reference's own single-threaded sample loop (the
    reference arm's workers draw from their own streams, so their orientation sets differ;
    the cost per orientation does not).  Largest relative differences of Cext and Cabs."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as P
    import dda_fft_b200 as D
    if not os.path.exists(P.REF_SO):
        return None
    cfg = P.make_run_cfg(grid=GRID, target=2, b_a=BA, c_a=CA, x=X, materials=(MAT,), orientation=1,
                         seed=SEED)
    *_, (ca, ce, _) = P.RefLib().run_samples(cfg, n, 1, each=True)
    r = ctx.orientation_solves(D.BatchConfig(occ=occ, materials=[MAT]), D.mc_rotations(SEED, n))
    return {"orientations": n, "reference": "float build, worker 0 stream",
            "cext_max_rel": float(np.max(np.abs(r["cext"] - ce) / np.abs(ce))),
            "cabs_max_rel": float(np.max(np.abs(r["cabs"] - ca) / np.abs(ca)))}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    per_step = max(2 * threads, 8)
    for _ in range(args.warmup):
        cpu_reference(max(threads, 1), threads)
    vals, total_s, total_n, kind, used = [], 0.0, 0, "reference", threads
    for _ in range(args.steps):
        v, kind, secs, used = cpu_reference(per_step, threads)
        vals.append(v)
        total_s += secs
        total_n += per_step
    value = total_n / total_s
    sample = f"{per_step} orientation-solves per step on {used} host threads (setup excluded)"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "orientation-solves/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * total_s / max(args.steps, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "grid": GRID, "orientations_per_step": per_step},
        "cpu_baseline": {"value": value, "unit": "orientation-solves/s", "cores": used,
                         "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "orientation-solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


# ------------------------------------------------------------------------- our arm
def matvec_bytes(n: int, nrhs: int) -> float:
    """Algorithmic HBM bytes of one matvec launch on an n^3 lattice: the Green-tensor
    octant read once (384 B per cell) and, per right-hand side, the field read and written
    plus the three passes over the half-padded spectrum (624 B per cell)."""
    return 384.0 * n ** 3 + 624.0 * n ** 3 * nrhs


def load_traffic(nrhs: int):
    """DRAM bytes per matvec from the committed ncu summary, scaled to nrhs."""
    path = os.path.join(ROOT, "profiles", "matvec_traffic.json")
    try:
        t = json.load(open(path))
        per_rhs = t["dram_bytes_per_rhs"]
        return float(t.get("dram_bytes_fixed", 0.0) + per_rhs * nrhs)
    except Exception:
        return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=64, help="orientations per step")
    ap.add_argument("--plain", type=int, default=8, help="orientations timed on the plain path")
    ap.add_argument("--cpu-samples", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the other configurations appended to the headline line")
    ap.add_argument("--profile-matvec", type=int, default=0, metavar="NRHS",
                    help="only run the matvec on NRHS right-hand sides (for ncu captures)")
    ap.add_argument("--grid", type=int, default=GRID)
    ap.add_argument("--variant", type=int, nargs=2, default=None, metavar=("X", "YZ"),
                    help="launch variants of the specialised passes instead of autotuning")
    ap.add_argument("--no-graph", action="store_true",
                    help="host-driven solver loop instead of one graph launch per batch (for "
                         "per-kernel launch lists: profilers list graph-launched kernels apart)")
    ap.add_argument("--workload", default="orientations",
                    choices=["orientations", "precision", "adjoint", "realizations", "plain",
                             "solver_graph"])
    args = ap.parse_args()
    if args.profile_matvec:
        return profile_matvec(args)
    if args.workload == "precision":
        return precision_run(args)
    if args.workload == "adjoint":
        return adjoint_run(args)
    if args.workload == "plain":
        return plain_run(args)
    if args.workload == "solver_graph":
        return solver_graph_run(args)
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "realizations":
        return realizations_run(args)
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import torch.distributed as dist
    import dda_fft_b200 as D

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    # under torchrun the process group exists whatever the rank count (the reduction of the
    # job's sums then goes through NCCL even on one rank)
    distributed = "RANK" in os.environ and "WORLD_SIZE" in os.environ
    torch.cuda.set_device(local)
    dev = local
    if distributed:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device(f"cuda:{local}"))

    B, K, W = args.batch, args.steps, args.warmup
    occ = ellipsoid_occ()
    kd = 2 * X / GRID
    ctx = D.Context(GRID, kd, max_rhs=2 * B, device=dev)
    if args.variant:
        ctx.set_fast_variant(*args.variant)
    else:
        ctx.autotune(2 * B)      # pass variants and tiling for this batch (set-up, not timed)
    if args.no_graph:
        ctx.set_solver_graph(False)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr, device=dev)
    # every rank draws its own contiguous run of the reference's MC stream (worker 0)
    total = (W + K) * B * world
    rot_all = D.mc_rotations(SEED, total)
    mine = rot_all[rank * (W + K) * B:(rank + 1) * (W + K) * B]
    cfg_host = D.BatchConfig(occ=occ, materials=[MAT], nplanes=1)
    cfg_res = D.BatchConfig(occ=None, materials=[MAT], nplanes=1)

    def barrier():
        if distributed:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def maxrank(v):
        if not distributed:
            return v
        t = torch.tensor([v], device=f"cuda:{dev}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # warm-up (also uploads the occupancy, which stays resident, and runs the final
    # reduction once so that its first-use set-up is not timed)
    from dda_fft_b200.shard import reduce_sums
    for w in range(W):
        r = ctx.orientation_solves(cfg_host if w == 0 else cfg_res, mine[w * B:(w + 1) * B])
    reduce_sums({"count": B, "cabs": float(r["cabs"].sum()), "cext": float(r["cext"].sum()),
                 "mueller": r["mueller"].sum(axis=0)}, r["mueller"].shape[1], device=f"cuda:{dev}")

    # ---- value: occupancy resident, device time
    sums = {"cabs": 0.0, "cext": 0.0, "mueller": None}
    clk = ClockSampler(dev)
    barrier()
    l0 = ctx.kernel_launches
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(K):
        r = ctx.orientation_solves(cfg_res, mine[(W + k) * B:(W + k + 1) * B])
        sums["cabs"] += float(r["cabs"].sum())
        sums["cext"] += float(r["cext"].sum())
        m = r["mueller"].sum(axis=0)
        sums["mueller"] = m if sums["mueller"] is None else sums["mueller"] + m
    # the job's one exchange: the sums over every rank's samples (dda_fft_b200.shard)
    job = reduce_sums({"count": K * B, "cabs": sums["cabs"], "cext": sums["cext"],
                       "mueller": sums["mueller"]}, sums["mueller"].shape[0],
                      device=f"cuda:{dev}")
    e1.record(stream)
    barrier()
    clocks = clk.stop()
    launches = ctx.kernel_launches - l0
    ms = maxrank(e0.elapsed_time(e1))
    value = K * B * world / (ms / 1000.0)

    # ---- e2e: public API with host buffers every step
    barrier()
    t0 = time.perf_counter()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for k in range(K):
        ctx.orientation_solves(cfg_host, mine[(W + k) * B:(W + k + 1) * B])
    f1.record(stream)
    barrier()
    wall = time.perf_counter() - t0
    ms_e2e = maxrank(max(f0.elapsed_time(f1), wall * 1000.0))
    e2e = K * B * world / (ms_e2e / 1000.0)
    nA = D.num_angles(0, 180, 10)
    h2d = occ.nbytes + B * 72 + 64
    d2h = B * (16 + nA * 16 * 8) + 2 * B * 8

    # ---- plain drop-in path: one ddagpu_dda_fft per polarisation + Mueller
    plain = None
    if rank == 0 and args.plain > 0:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        pctx = D.Context(GRID, kd, max_rhs=2, device=dev)
        alpha = np.array([0, _cm_alpha(kd, complex(*MAT))], np.complex64)
        th = np.deg2rad(np.arange(nA) * 10.0)
        ksc0 = np.stack([np.sin(th), np.zeros_like(th), np.cos(th)], 1)
        rots = mine[:args.plain]

        def one(T):
            kinc = T @ np.array([0, 0, 1.0])
            e = [T @ np.array([1.0, 0, 0]), T @ np.array([0, 1.0, 0])]
            ksc = (ksc0 @ T.T)[None]
            esc = [pctx.dda_fft(occ, alpha, [0, 1], kd, kinc, e[q], ksc, trace=False)["esc"]
                   for q in range(2)]
            pctx.mueller(kinc, e[0], e[1], ksc, (T @ np.array([0, 1.0, 0]))[None], esc[0], esc[1])
        one(rots[0])
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for T in rots:
            one(T)
        torch.cuda.synchronize(dev)
        plain = len(rots) / (time.perf_counter() - t0)
        pctx.close()

    # ---- roofline: the matvec (K1+K2+K3) on the batch, device-resident
    nrhs = 2 * B
    n3 = GRID ** 3
    x = torch.randn(nrhs, 3, GRID, GRID, GRID, dtype=torch.complex64, device=f"cuda:{dev}")
    y = torch.empty_like(x)
    torch.cuda.synchronize(dev)
    for _ in range(3):
        ctx.convolution_dev(x, y, nrhs)
    reps = 10
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    for _ in range(reps):
        ctx.convolution_dev(x, y, nrhs)
    g1.record(stream)
    torch.cuda.synchronize(dev)
    mv_ms = g0.elapsed_time(g1) / reps
    alg_bytes = matvec_bytes(GRID, nrhs)
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except Exception:
        peak, peak_src = 6650.0, "fallback"
    achieved = alg_bytes / (mv_ms / 1000.0) / 1e9
    traffic = load_traffic(nrhs)
    del x, y

    # ---- CPU baseline (rank 0, N = 1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        ns = args.cpu_samples or max(24 * threads, 64)   # about 10 s of the host's threads
        v, kind, secs, used = cpu_reference(ns, threads)
        cpu = {"value": v, "unit": "orientation-solves/s", "cores": used, "kind": kind,
               "sample": f"{ns} orientation-solves of the same workload, {secs:.1f} s wall "
                         f"(setup excluded)"}
        cpu["cross_check"] = cross_check(ctx, occ, 8)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "orientation-solves/s", "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": GRID, "orientations_per_step": B,
                       "rhs_per_step": 2 * B, "parallelism": f"orientations sharded over {world} GPU(s)",
                       "l2": "working set per step >> L2 (126 MB): no flush needed",
                       "tiling": list(ctx.tiling()), "fast_passes": ctx.fast_kernels,
                       "fast_variant": list(ctx.fast_variant),
                       "solve_graph": not args.no_graph},
            "e2e": {"value": e2e, "unit": "orientation-solves/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "plain_gpu": {"value": plain, "unit": "orientation-solves/s",
                          "path": "ddagpu_dda_fft per polarisation + ddagpu_mueller"},
            "speedup_vs_plain": (value / plain) if plain else None,
            "roofline": {"kernel": "matvec K1+K2+K3", "bound": "hbm", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_src, "traffic": traffic,
                         "algorithmic_bytes": alg_bytes, "ms_per_launch": mv_ms,
                         "rhs_per_launch": nrhs},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": launches,
            "check": {"cext_mean": job["cext"] / job["count"], "cabs_mean": job["cabs"] / job["count"],
                      "samples": job["count"]},
        }
    ctx.close()
    if distributed:
        dist.destroy_process_group()
    if rank == 0:
        if world == 1 and not args.no_extras:
            line["other_configs"] = other_configs(args)
        print(json.dumps(line), flush=True)


def other_configs(args):
    """The other configurations, measured in the same run after the headline (one GPU):
    the plain mid configuration (per-sample time, far field by kz groups and direct), the
    realisations of the three lattice sizes as one group graph (device and end-to-end
    rates, the 128^3 matvec's roofline fraction) and the differentiation configuration's
    adjoint pass (backward / forward time and matvecs).  Each runs its own workload
    function with shortened step counts; its JSON line is condensed here."""
    import contextlib
    import io
    runs = (("plain_mid", plain_run, {"steps": 5, "warmup": 2, "no_cpu": True}),
            ("realizations", realizations_run, {"steps": 3, "warmup": 3, "no_cpu": True}),
            ("adjoint", adjoint_run, {"grid": 64}))
    keep = {"plain_mid": lambda r: {"ms_per_sample": r["graph"]["ms_per_sample"],
                                    "ms_per_sample_direct_farfield": r["graph_direct_farfield"]["ms_per_sample"],
                                    "ms_per_sample_host_loop": r["host_loop"]["ms_per_sample"],
                                    "cext": r["cext"], "cabs": r["cabs"], "workload": r["workload"]},
            "realizations": lambda r: {"value": r["value"], "unit": r["unit"], "e2e": r["e2e"]["value"],
                                       "graph_launches_per_step": r["config"]["graph_launches_per_step"],
                                       "matvec_roofline_frac": r["roofline"]["frac"],
                                       "matvec_kernel": r["roofline"]["kernel"], "steps": r["steps"]},
            "adjoint": lambda r: {k: r[k] for k in ("workload", "dipoles", "forward_s", "backward_s",
                                                    "backward_over_forward", "forward_matvecs",
                                                    "backward_matvecs")}}
    out = {}
    for name, fn, kw in runs:
        a = argparse.Namespace(**vars(args))
        a.__dict__.update(kw)
        buf = io.StringIO()
        try:
            with contextlib.redirect_stdout(buf):
                fn(a)
            out[name] = keep[name](json.loads(buf.getvalue().strip().splitlines()[-1]))
        except Exception as e:   # reported in the line, never fatal to the headline
            out[name] = {"error": repr(e)[:300]}
    return out


def profile_matvec(args):
    """Launch the matvec (K1+K2+K3) args.steps times on NRHS device-resident fields."""
    import torch
    import dda_fft_b200 as D
    n, nrhs = args.grid, args.profile_matvec
    ctx = D.Context(n, 2 * X / n, max_rhs=nrhs)
    if args.variant:
        ctx.set_fast_variant(*args.variant)
    else:
        ctx.autotune(nrhs)
    x = torch.randn(nrhs, 3, n, n, n, dtype=torch.complex64, device="cuda")
    y = torch.empty_like(x)
    torch.cuda.synchronize()
    for _ in range(args.warmup + args.steps):
        ctx.convolution_dev(x, y, nrhs)
    torch.cuda.synchronize()
    print(json.dumps({"profile_matvec": nrhs, "grid": n, "launches": ctx.kernel_launches,
                      "fast_variant": list(ctx.fast_variant)}))
    ctx.close()


def precision_run(args):
    """The precision configuration: 128^3 sphere, x = 16, m = 1.6+0.0005i, theta 0..180 step
    2, both polarisations.  The FP64 reference is the FP64 GPU solve (the reference's CG in
    double, to a discrepancy of 3e-10); beside it: the plain float BiCGStab (the reference's
    method, Error_max 1e-5, 100 steps), the FP64 BiCGStab (which diverges on this system),
    and the precision pattern -- FP32 FFT matvec, FP64 fields, residuals and test -- at the
    configuration's Error_max 1e-5, at 1e-8 and at 1e-9.  Errors of Cext, Cabs (averaged over the two
    polarisations) and of the Mueller matrix against the FP64 solve; one JSON line."""
    import dda_fft_b200 as D
    n, x, m = 128, 16.0, complex(1.6, 0.0005)
    kd = 2 * x / n
    occ = ellipsoid_occ(n, 1.0, 1.0)
    alpha = np.array([0, _cm_alpha(kd, m)], np.complex64)      # one system for every solve
    th = np.deg2rad(np.arange(91) * 2.0)
    ksc = np.stack([np.sin(th), np.zeros_like(th), np.cos(th)], 1)
    E = ((1, 0, 0), (0, 1, 0))
    out = {"workload": "precision: 128^3 sphere x=16 m=1.6+0.0005i, 91 angles, both polarisations"}
    with D.Context(n, kd, max_rhs=2) as ctx:
        def mueller(esc):
            return ctx.mueller((0, 0, 1), E[0], E[1], ksc[None], [(0, 1, 0)],
                               np.asarray(esc[0]).reshape(1, -1, 3), np.asarray(esc[1]).reshape(1, -1, 3))
        t0 = time.perf_counter()
        ref = [ctx.solve_fp64(occ, alpha.astype(np.complex128), [0, 1], kd, (0, 0, 1), e, ksc, solver=0,
                              max_step=12000, err_max=3e-10, trace=False) for e in E]
        out["fp64_cg"] = {"seconds": time.perf_counter() - t0, "steps": [r["steps"] for r in ref],
                          "err": [r["err"] for r in ref]}
        b64 = ctx.solve_fp64(occ, alpha.astype(np.complex128), [0, 1], kd, (0, 0, 1), E[0], None, solver=2,
                             max_step=1000, err_max=1e-9)
        out["fp64_bicgstab"] = {"steps": b64["steps"], "err_min": b64["err_min"], "err_final": b64["err"],
                                "trace_every_100": [float(v) for v in b64["trace"][::100]]}
        ctx.release_fp64()
        Mr = mueller([r["esc"] for r in ref])
        cr = {q: 0.5 * (ref[0][q] + ref[1][q]) for q in ("cext", "cabs")}

        def errors(res):
            M = mueller([r["esc"] for r in res])
            c = {q: 0.5 * (res[0][q] + res[1][q]) for q in ("cext", "cabs")}
            sig = np.abs(Mr) > 1e-3 * np.abs(Mr).max()
            return {"cext_rel": abs(c["cext"] - cr["cext"]) / abs(cr["cext"]),
                    "cabs_rel": abs(c["cabs"] - cr["cabs"]) / abs(cr["cabs"]),
                    "mueller_over_m11_max": float((np.abs(M - Mr) / Mr[..., :1, :1]).max()),
                    "mueller_significant_rel_median": float(np.median(np.abs(M - Mr)[sig] / np.abs(Mr)[sig]))}
        t0 = time.perf_counter()
        plain = [ctx.dda_fft(occ, alpha, [0, 1], kd, (0, 0, 1), e, ksc[None], solver=2, max_step=100,
                             err_max=1e-5) for e in E]
        out["plain_float_bicgstab"] = {"seconds": time.perf_counter() - t0,
                                       "err_min": [r["err_min"] for r in plain], **errors(plain)}
        for em in (1e-5, 1e-8, 1e-9):
            t0 = time.perf_counter()
            res = [ctx.dda_fft_refined(occ, alpha, [0, 1], kd, (0, 0, 1), e, ksc[None], solver=0,
                                       err_max=em, max_outer=30) for e in E]
            out[f"mixed_cg_{em:g}"] = {"seconds": time.perf_counter() - t0,
                                       "iterations": [r["inner_steps"] for r in res],
                                       "matvecs": [r["matvecs"] for r in res],
                                       "err": [r["err"] for r in res], **errors(res)}
    print(json.dumps(out), flush=True)


def adjoint_run(args):
    """The differentiation configuration: two-material porous 64^3 cube (packing 0.3,
    materials 1.5+0.01i / 1.7+0.1i at 0.7 / 0.3, seed 11), x = 5, CMRR, CG; forward pass
    (both polarisations) and the adjoint gradient of Cabs + M11(180 deg) for every dipole;
    one JSON line with the times and matvec counts of both passes."""
    import torch
    from dda_fft_b200.adjoint import GPUBackend, Problem, observables, porous_target
    n = args.grid
    filled, m = porous_target(n, seed=11)
    P = Problem(filled, kd=2 * 5.0 / n, model="cmrr")
    G = GPUBackend(P, err_max=1e-8)
    m_re = torch.tensor(m.real, requires_grad=True)
    m_im = torch.tensor(m.imag, requires_grad=True)
    observables(m_re, m_im, P, G)                       # warm-up
    mv0 = G.matvecs
    t0 = time.perf_counter()
    f = observables(m_re, m_im, P, G)
    t1 = time.perf_counter()
    mv1 = G.matvecs
    (f[0] + f[1]).backward()
    t2 = time.perf_counter()
    mv2 = G.matvecs
    print(json.dumps({"workload": f"adjoint: {n}^3 porous two-material cube, x=5, CMRR, CG",
                      "dipoles": int(P.ndip), "cabs": float(f[0].detach()),
                      "m11_180": float(f[1].detach()),
                      "forward_s": t1 - t0, "backward_s": t2 - t1,
                      "backward_over_forward": (t2 - t1) / (t1 - t0),
                      "forward_matvecs": mv1 - mv0, "backward_matvecs": mv2 - mv1,
                      "grad_norm_re": float(np.linalg.norm(m_re.grad.numpy())),
                      "grad_norm_im": float(np.linalg.norm(m_im.grad.numpy()))}), flush=True)
    G.close()


def plain_run(args):
    """The plain-method mid configuration: 64^3 sphere, x = 8, m = 1.5+0.01i, LDR,
    BiCGStab, Error_max 1e-3, Max_Step 100, 12 planes, theta 0..180 step 1 (2172
    directions), fixed orientation: one sample (both polarisations) through the batched
    entry point, with the solver loop as a CUDA graph and on the host (far field by kz
    groups), with the graph and the direct far field, the matvec on 2 right-hand sides,
    and the reference's own sample loop on one host thread (the configuration has one
    sample, so one worker)."""
    import torch
    import dda_fft_b200 as D
    n, x, mat = 64, 8.0, (1.5, 0.01)
    kd = 2 * x / n
    occ = ellipsoid_occ(n, 1.0, 1.0)
    cfg = D.BatchConfig(occ=occ, materials=[mat], polarizability=5, solver=2, max_step=100,
                        err_max=1e-3, nplanes=12, theta_step=1.0)
    out = {"workload": "plain mid: 64^3 sphere x=8 m=1.5+0.01i LDR BiCGStab 1e-3, 12 planes, "
                       "2172 directions, one sample"}
    rot = D.fixed_rotation(0, 0, 0)[None]
    with D.Context(n, kd, max_rhs=2) as ctx:
        st = torch.cuda.ExternalStream(ctx.stream_ptr)
        for graph, ff in ((True, 0), (False, 0), (True, 1)):
            ctx.set_solver_graph(graph)
            ctx.set_farfield_mode(ff)
            for _ in range(max(args.warmup, 1)):
                r = ctx.orientation_solves(cfg, rot)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            reps = max(args.steps, 1)
            l0 = ctx.kernel_launches
            e0.record(st)
            for _ in range(reps):
                r = ctx.orientation_solves(cfg, rot)
            e1.record(st)
            torch.cuda.synchronize()
            key = ("graph" if graph else "host_loop") + ("_direct_farfield" if ff else "")
            out[key] = {"ms_per_sample": e0.elapsed_time(e1) / reps, "steps": r["max_steps"],
                        "kernels_per_sample": (ctx.kernel_launches - l0) / reps}
            if ff == 0:
                out["cext"], out["cabs"] = float(r["cext"][0]), float(r["cabs"][0])
        ctx.set_farfield_mode(0)
        xx = torch.randn(2, 3, n, n, n, dtype=torch.complex64, device="cuda")
        yy = torch.empty_like(xx)
        for _ in range(3):
            ctx.convolution_dev(xx, yy, 2)
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(st)
        for _ in range(20):
            ctx.convolution_dev(xx, yy, 2)
        g1.record(st)
        torch.cuda.synchronize()
        mv_ms = g0.elapsed_time(g1) / 20
        out["matvec_2rhs"] = {"ms": mv_ms, "GBs_algorithmic": matvec_bytes(n, 2) / mv_ms / 1e6}
    if not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as P
        rc = P.make_run_cfg(grid=n, target=1, x=x, materials=(mat,), polarizability=5, solver=2,
                            max_step=100, nplanes=12, theta_step=1.0)
        secs, *_ = P.RefLib().run_samples(rc, 1, 1)
        out["reference_cpu_s_per_sample"] = secs
    print(json.dumps(out), flush=True)


def solver_graph_run(args):
    """Solves that iterate (BiCGStab to Error_max 1e-6 on ellipsoids b/a 0.8, c/a 0.6,
    x = n/8, m = 1.6+0.002i): wall time per batched call with iterations 2.. recorded as
    one CUDA graph launch vs the host loop that reads the active flags every iteration."""
    import torch
    import dda_fft_b200 as D
    out = {"workload": "BiCGStab to 1e-6, ellipsoid 0.8/0.6, x = n/8, m = 1.6+0.002i"}
    for n, no in ((16, 1), (32, 1), (32, 8), (64, 1), (64, 16)):
        x = n / 8.0
        cfg = D.BatchConfig(occ=ellipsoid_occ(n, 0.8, 0.6), materials=[(1.6, 0.002)], solver=2,
                            err_max=1e-6, max_step=300)
        rot = D.mc_rotations(SEED, no)
        row = {}
        with D.Context(n, 2 * x / n, max_rhs=2 * no) as ctx:
            for g in (False, True):
                ctx.set_solver_graph(g)
                for _ in range(max(args.warmup, 1)):
                    r = ctx.orientation_solves(cfg, rot)
                torch.cuda.synchronize()
                t = time.perf_counter()
                for _ in range(max(args.steps, 1)):
                    r = ctx.orientation_solves(cfg, rot)
                torch.cuda.synchronize()
                row["graph_ms" if g else "host_loop_ms"] = (time.perf_counter() - t) / max(args.steps, 1) * 1e3
            row["steps"] = r["max_steps"]
        out[f"{n}^3 x {2 * no} rhs"] = row
    print(json.dumps(out), flush=True)


AGG_SIZES, AGG_N, AGG_R, AGG_LR, AGG_RHO = (32, 64, 128), 64, 3.0, 0.0, 0.25
AGG_METRIC = "realization-solves/s, agglomerates on lattices drawn from {32,64,128}^3"
AGG_WORKLOAD = ("64 agglomerate realisations (monomer radius 3 cells, length ratio 0, packing "
                "0.25; realisation k placed from the random stream of worker k of seed 7) on "
                "lattice edges drawn from {32, 64, 128} by the reference's generator seeded 7; "
                "x=6, m=1.55+0.005i, CM, CG, Error_max 1e-3, Max_Step 20, fixed orientation, "
                "1 plane, 19 angles, both polarisations")


def xorshift_draws(seed: int, count: int):
    """dda_srand / dda_rand (randomize.cpp:44-58): count draws after seeding."""
    m = (1 << 64) - 1
    s = seed or 0x9E3779B97F4A7C15
    out = []
    for _ in range(count):
        s ^= s >> 12
        s = (s ^ (s << 25)) & m
        s ^= s >> 27
        out.append(((s * 2685821657736338717) & m) >> 33)
    return out


def agglomerate_sizes():
    return [AGG_SIZES[v % len(AGG_SIZES)] for v in xorshift_draws(SEED, AGG_N)]


def realizations_reference(args, sizes):
    """The reference's own sample loop (oracle/_ref) on agglomerates of each lattice size,
    a bounded sample of realisations per size on all host threads; the job time is
    estimated as the sum over sizes of (realisations of that size) / (measured rate)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as P
    threads = os.cpu_count() or 1
    R = P.RefLib()
    per = {}
    for n in AGG_SIZES:
        ns = args.cpu_samples or threads
        cfg = P.make_run_cfg(grid=n, target=6, x=X, materials=(MAT,), seed=SEED,
                             monomer_radius=AGG_R, monomer_ratio=AGG_LR, packing=AGG_RHO)
        secs, *_ = R.run_samples(cfg, ns, threads)
        per[n] = (ns, secs)
    total = sum(sizes.count(n) * per[n][1] / per[n][0] for n in AGG_SIZES)
    value = len(sizes) / total
    sample = ", ".join(f"{per[n][0]} realisations at {n}^3 in {per[n][1]:.1f} s"
                       for n in AGG_SIZES) + f" on {threads} threads (Green tensor set-up excluded)"
    return value, threads, sample, total


def realizations_run(args):
    """The realisation half of the batching configuration: every realisation is placed on
    the host (the reference's float geometry, one thread per realisation), rasterised on
    the GPU into the batch of its lattice size and solved for both polarisations; the three
    lattice sizes are one group (ddagpu_group), so a step is one graph launch with a branch
    per lattice.  value: the GPU part (monomer lists to Mueller matrices); e2e: placement
    included."""
    from concurrent.futures import ThreadPoolExecutor
    sizes = agglomerate_sizes()
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return
        value, cores, sample, total = realizations_reference(args, sizes)
        print(json.dumps({
            "impl": "reference", "metric": AGG_METRIC, "value": value,
            "unit": "realization-solves/s", "n_gpus": args.gpus, "steps": 1, "warmup": 0,
            "ms_per_step": 1000 * total, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": AGG_WORKLOAD, "sizes": {str(n): sizes.count(n) for n in AGG_SIZES}},
            "cpu_baseline": {"value": value, "unit": "realization-solves/s", "cores": cores,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": "realization-solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}), flush=True)
        return
    import torch
    import dda_fft_b200 as D
    K, W = args.steps, args.warmup
    groups = {n: [k for k, s in enumerate(sizes) if s == n] for n in AGG_SIZES}
    counts = {n: D.Agglomerate.count((n, n, n), AGG_RHO, AGG_R, AGG_LR) for n in AGG_SIZES}
    ctxs = {n: D.Context(n, 2 * X / n, max_rhs=2 * max(len(g), 1)) for n, g in groups.items() if g}
    for n, c in ctxs.items():
        c.autotune(2 * len(groups[n]))
    cfg = D.BatchConfig(occ=None, materials=[MAT])
    pool = ThreadPoolExecutor(max_workers=os.cpu_count() or 4)
    members = sorted(ctxs)
    grp = D.Group([ctxs[n] for n in members])

    def place(step, k):
        n = sizes[k]
        return D.Agglomerate(SEED, step * AGG_N + k).place(n, AGG_R, AGG_R * AGG_LR, counts[n])

    def step_device(mons):
        """one graph launch for the three lattice sizes, monomers already placed"""
        res = grp.agglomerate_solves(cfg, [[mons[k] for k in groups[n]] for n in members])
        return dict(zip(members, res))

    def place_step(step):
        # the largest lattices' realisations first: their placement is the longest
        order = sorted(range(AGG_N), key=lambda k: -sizes[k])
        return dict(zip(order, pool.map(lambda k: place(step, k), order)))

    placed = [list(pool.map(lambda k: place(s, k), range(AGG_N))) for s in range(W + K)]
    for s in range(W):
        step_device(placed[s])
    clk = ClockSampler(0)
    launches0 = sum(c.kernel_launches for c in ctxs.values())
    runs0 = grp.graph_runs
    torch.cuda.synchronize()
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    res = None
    for s in range(W, W + K):
        res = step_device(placed[s])
    torch.cuda.synchronize()
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    launches = sum(c.kernel_launches for c in ctxs.values()) - launches0
    graph_launches = grp.graph_runs - runs0
    ms = e0.elapsed_time(e1)
    value = K * AGG_N / (ms / 1000.0)
    # end to end: step s + 1's realisations are placed on the host threads while step s
    # solves on the GPU (the library call releases the interpreter lock)
    ahead = ThreadPoolExecutor(max_workers=1)
    t0 = time.perf_counter()
    nxt = ahead.submit(place_step, W)
    for s in range(W, W + K):
        now = nxt.result()
        if s + 1 < W + K:
            nxt = ahead.submit(place_step, s + 1)
        step_device(now)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    ahead.shutdown()
    e2e = K * AGG_N / e2e_s
    nA = D.num_angles(0, 180, 10)
    h2d = sum(counts[s] * 13 * 4 for s in sizes) + AGG_N * 200
    d2h = AGG_N * (16 + nA * 16 * 8 + 4)
    # roofline: the matvec on the largest lattice's batch
    nbig = max(n for n, g in groups.items() if g)
    nrhs = 2 * len(groups[nbig])
    ctx = ctxs[nbig]
    x = torch.randn(nrhs, 3, nbig, nbig, nbig, dtype=torch.complex64, device="cuda")
    y = torch.empty_like(x)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr, device=0)
    for _ in range(3):
        ctx.convolution_dev(x, y, nrhs)
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    for _ in range(5):
        ctx.convolution_dev(x, y, nrhs)
    g1.record(stream)
    torch.cuda.synchronize()
    mv_ms = g0.elapsed_time(g1) / 5
    del x, y
    try:
        peak, src = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), "measured"
    except Exception:
        peak, src = 6650.0, "fallback"
    achieved = matvec_bytes(nbig, nrhs) / (mv_ms / 1000.0) / 1e9
    cpu = None
    if not args.no_cpu:
        v, cores, sample, _ = realizations_reference(args, sizes)
        cpu = {"value": v, "unit": "realization-solves/s", "cores": cores, "kind": "reference",
               "sample": sample}
    info = {n: {"realizations": len(groups[n]), "max_steps": r["max_steps"],
                "mean_dipoles": float(np.mean(r["ndip"])), "rolled_back": r["rolled_back"]}
            for n, r in res.items()}
    print(json.dumps({
        "metric": AGG_METRIC, "value": value, "unit": "realization-solves/s", "n_gpus": 1,
        "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": AGG_WORKLOAD, "groups": info,
                   "graph_launches_per_step": graph_launches / K,
                   "l2": "working set per step >> L2 (126 MB): no flush needed"},
        "e2e": {"value": e2e, "unit": "realization-solves/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "includes": "host placement of every realisation, the next step's overlapping "
                            "this step's solve"},
        "roofline": {"kernel": f"matvec K1+K2+K3 at {nbig}^3", "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": src, "traffic": None, "ms_per_launch": mv_ms,
                     "rhs_per_launch": nrhs, "kernels": "specialised" if ctx.fast_kernels else "generic"},
        "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": launches}), flush=True)
    grp.close()
    for c in ctxs.values():
        c.close()
    pool.shutdown()


def _cm_alpha(d0, m):
    """Polarizability_CM (dda_func.cpp:1631-1637)."""
    return d0 ** 3 * (0.75 / np.pi) * (m * m - 1) / (m * m + 2)


if __name__ == "__main__":
    main()
