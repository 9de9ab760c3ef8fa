#!/usr/bin/env python
"""Benchmark of the B200 channel-dns time step.

Workload: Re_tau = 180 channel, 128 x 129 x 128 base grid (NXS = NZS = 64,
NYS = 126), 196 x 193 x 196 dealiased product grid, 4 pi x 2 x 2 pi, fixed
mean pressure gradient, DT = 5e-5, FP64.  Initial field: seeded Reichardt
log-law mean profile plus a divergence-free perturbation with a k^-5/3
envelope at 10 % rms (synthetic, cdns/fields.py).

  value   steps/s with the state resident in HBM: K graph-replayed steady
          steps (it > W >= 3) timed with CUDA events on the library stream,
          max over ranks, x ranks.
  e2e     steps/s through the C ABI with host buffers: upload of the state
          from pinned memory, K steps called one by one from iteration 1
          (setup included) each reading back its pressure gradient, and the
          download of velocity and pressure, timed with the same events.
  roofline  the dominant stage's algorithmic HBM bytes per launch over its
          CUDA-event duration (per-stage pass after the timed region).
  cpu_baseline  the reference's own sources (oracle/_ref, built with the
          project FFTW/MPI shims) on this host's cores, bounded sample.

  pencil  the workload as an 8-rank pencil decomposition (one channel over
          several GPUs) with every rank emulated on this GPU: per-rank stage
          times and the bytes each rank exchanges per step (--pencil P).

``--impl reference`` times the reference CPU solver alone on the same
workload.  With torchrun (N > 1) every rank advances its own channel
(replicas, no collective in the data path; scaling "weak").
"""
from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "channel-dns_b200"))

METRIC = ("Reτ180 128×129×128 steps/s: FP64 vs FP32/FP64 (err≤1e-6); "
          "adjoint/fwd cost")
PI = math.acos(-1.0)
WORKLOAD = {"workload": "retau180_fp64_step", "grid": "128x129x128", "product_grid": "196x193x196",
            "domain": "4pi x 2 x 2pi", "Re_tau": 180, "DT": 5e-5, "forcing": "fixed dp/dx",
            "precision": "fp64", "l2_policy": "inputs larger than L2 (about 1.9 GB of stage traffic per step)"}


def workload_mesh():
    import cdns
    mesh = cdns.Mesh(128, 128, 128, 64, 126, 64, 196, 192, 196, 4.0 * PI, 2.0 * PI)
    params = cdns.Params(Re=180.0, DT=5e-5, INDEX_GRAD_PRE=1)
    return mesh, params


def stage_bytes(mesh):
    """Algorithmic HBM bytes per launch of each stage (16 B per complex value;
    every stage reads and writes its operands once)."""
    nkx, nkz, ncy = mesh.NXS + 1, 2 * mesh.NZS + 1, mesh.NYS + 1
    ny2 = mesh.NY2 + 1
    Ns = nkz * ncy * nkx
    Ny = nkz * ny2 * nkx
    Nz = mesh.NZ2 * ny2 * nkx
    return {
        "curl": 16 * (3 * Ns + 3 * Ns),
        "y_synthesis": 16 * (6 * Ns + 6 * Ny),
        "z_backward": 16 * 6 * (Ny + Nz),
        "x_cross": 16 * 9 * Nz,
        "z_forward": 16 * 3 * (Nz + Ny),
        "y_analysis": 16 * (3 * Ny + 3 * Ns),
        # R from u, u_prev, N, N_prev (12), influence + B-problem fields (12),
        # tau pivots ad_p, ad_v (1 complex-equivalent), writes u, p (4)
        "solve": 16 * 29 * Ns,
    }


# Source files behind each stage's kernel: a recorded DRAM-traffic figure is
# only reported while these files are unchanged since its ncu capture.
STAGE_SOURCES = {
    "curl": ["chebyshev.cu", "warp_columns.cuh"],
    "y_synthesis": ["chebyshev.cu", "transforms.cu", "reg_fft.cuh"],
    "z_backward": ["transforms.cu", "reg_fft.cuh", "fft_lines.cuh"],
    "x_cross": ["transforms.cu", "reg_fft.cuh", "fft_lines.cuh"],
    "z_forward": ["transforms.cu", "reg_fft.cuh", "fft_lines.cuh"],
    "y_analysis": ["chebyshev.cu", "transforms.cu", "reg_fft.cuh"],
    "solve": ["solver.cu", "warp_columns.cuh"],
}
TRAFFIC_PROFILE = os.path.join(ROOT, "profiles", "dram_traffic_retau180.md")


def stage_source_hash(stage: str) -> str:
    import hashlib
    h = hashlib.sha256()
    for name in STAGE_SOURCES[stage] + ["cdns_kernels.cuh", "cdns_common.cuh"]:
        with open(os.path.join(ROOT, "channel-dns_b200", "csrc", name), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:16]


def ncu_traffic(stage: str):
    """(DRAM bytes read + written per launch, note) of a stage's kernel from
    the committed ncu summary: lines ``traffic: stage=<s> bytes=<n>
    sources=<sha>`` in profiles/dram_traffic_retau180.md.  None when the
    stage has no recorded capture or its sources changed since it."""
    import re
    try:
        text = open(TRAFFIC_PROFILE).read()
    except OSError:
        return None, "no ncu capture recorded"
    for m in re.finditer(r"^traffic: stage=(\w+) bytes=(\d+) sources=(\w+)", text, re.M):
        if m.group(1) == stage:
            if m.group(3) != stage_source_hash(stage):
                return None, "stale: kernel sources changed since the ncu capture"
            return int(m.group(2)), "ncu dram__bytes_read.sum + dram__bytes_write.sum, " \
                                    "profiles/dram_traffic_retau180.md"
    return None, "no ncu capture recorded for this stage"


def step_bytes_model(mesh):
    """Stage-pass model of the whole step: the sum of the stage bytes."""
    return sum(stage_bytes(mesh).values())


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(prefix="cdns_clocks_", suffix=".csv")
        os.close(fd)
        self.fh = open(self.path, "w")
        self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                      "-lms", "200", "-i", str(self.dev)], stdout=self.fh,
                                     stderr=subprocess.DEVNULL)

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def reference_arm_time(steps: int, warmup: int, threads: int, reps: int = 1):
    """Steady steps/s of the reference CPU solver: T(n1 + steps) - T(n1),
    each run from the same restart (setup and final output cancel); the
    median of `reps` such pairs (tests/tools/bench_hybrid.py:52-88 takes the
    median of 3)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_io  # the reference sources built in oracle/_ref (checker / baseline only)
    import cdns
    from cdns.fields import divergence_free_field
    mesh, params = workload_mesh()
    u0 = divergence_free_field(mesh, params, seed=1, amp=0.1, spectrum="k53", mean="loglaw")

    class _M:
        pass

    m = _M()
    for k in ("NX", "NY", "NZ", "NXS", "NYS", "NZS", "NX2", "NY2", "NZ2", "XL", "ZL"):
        setattr(m, k, getattr(mesh, k))
    m.nkz, m.ncy, m.nkx = 2 * mesh.NZS + 1, mesh.NYS + 1, mesh.NXS + 1

    class _P:
        pass

    p = _P()
    p.Re, p.DT, p.G_pre, p.a_pre0, p.b_pre0 = 180.0, 5e-5, 0.0, 0.0, 1.0
    p.a_V, p.b_V, p.INDEX_GRAD_PRE, p.THETA, p.V_Microblow0 = (1.0, 1.0, 1.0), (0.0, 0.0, 0.0), 1, 0.0, 0.0
    if ref_io.available():
        n1 = max(warmup, 2)
        steady, whole = [], []
        for _ in range(max(reps, 1)):
            _, _, t1 = ref_io.run_steps(m, p, u0, n1, threads=threads)
            _, _, t2 = ref_io.run_steps(m, p, u0, n1 + steps, threads=threads)
            steady.append(steps / max(t2 - t1, 1e-9))
            whole.append((n1 + steps) / max(t2, 1e-9))
        return statistics.median(steady), {
            "kind": "reference", "cores": threads,
            "sample": f"reference sources + project FFT shim (oracle/_ref), "
                      f"T({n1 + steps} steps) - T({n1} steps) from one restart, {threads} threads, "
                      f"median of {len(steady)}",
            "runs": [round(v, 4) for v in steady],
            # the reference's own --timing counts every step of a run, the two
            # setup steps (EqSolvePV::setup at iterations 1-2) included
            "with_setup": {"value": statistics.median(whole), "unit": "steps/s", "steps": n1 + steps}}
    # the numpy restatement, single thread, one steady step
    import numpy as np
    import channel_oracle as orc
    om = orc.Mesh(*(getattr(mesh, k) for k in ("NX", "NY", "NZ", "NXS", "NYS", "NZS", "NX2", "NY2", "NZ2")),
                  mesh.XL, mesh.ZL)
    op = orc.Parm(Re=180.0, DT=5e-5)
    sim = orc.Simulation(om, op, u0)
    with np.errstate(all="ignore"):
        sim.run(2)
        t = time.perf_counter()
        sim.run(steps)
        dt = time.perf_counter() - t
    return steps / dt, {"kind": "port", "cores": 1,
                        "sample": f"numpy oracle, {steps} steady steps after 2 setup steps"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    steps = max(1, args.steps)
    # the reference runs about 10 steps/s here: three timed pairs while that
    # stays within a minute or so, one pair for longer runs
    v, info = reference_arm_time(steps, args.warmup, threads, reps=3 if steps <= 100 else 1)
    line = {"metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": args.gpus, "steps": steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(WORKLOAD), "impl": "reference",
            "cpu_baseline": dict(info, value=v, unit="steps/s"),
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def ensemble_case(n: int, re: float):
    """Channel member: N x (N+1) x N base grid, NXS=NZS=N/2, NYS=N-2, 3/2 product
    grid, 4pi x 2 x 2pi, fixed pressure gradient."""
    import cdns
    n2 = 3 * n // 2
    mesh = cdns.Mesh(n, n, n, n // 2, n - 2, n // 2, n2, n2, n2, 4.0 * math.pi, 2.0 * math.pi)
    params = cdns.Params(Re=re, DT=5e-5, G_pre=0.0, a_pre0=0.0, b_pre0=1.0, a_V=(1.0, 1.0, 1.0),
                         b_V=(0.0, 0.0, 0.0), INDEX_GRAD_PRE=1, THETA=0.0, V_Microblow0=0.0)
    return mesh, params


def run_ensemble(members: int, K: int, W: int, precision: int, device: int, seed: int, world: int = 1,
                 rank: int = 0, dist=None) -> dict:
    """Ensemble form: `members` channels with N drawn from {32, 48, 64, 96} and
    Re_tau from U[100, 180] (seeded, cdns.ensemble.members), laminar profile +
    5 % divergence-free perturbation on |k| <= 4; K graph-replayed steady steps
    after W warm-up steps, timed with CUDA events on the batch stream.  On N
    GPUs the members are partitioned over the ranks by estimated bytes per step
    (replicas only: no data crosses ranks); the time is the max over ranks."""
    import numpy as np
    import torch
    import cdns
    from cdns.ensemble import imbalance, rank_members
    from cdns.fields import divergence_free_field
    mine = rank_members(members, world, rank)
    cases = [ensemble_case(n, re) for _, n, re in mine]
    batch = cdns.Batch([c[0] for c in cases], [c[1] for c in cases], device=device, precision=precision)
    for ctx, (i, _, _), (mesh, params) in zip(batch.members, mine, cases):
        u = divergence_free_field(mesh, params, seed=seed + i, amp=0.05, kmax=4)
        ctx.set_velocity(np.stack(u, axis=-1))
    batch.run(1, W)
    batch.synchronize()
    stream = torch.cuda.ExternalStream(batch.stream_ptr(), device=device)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    batch.run(W + 1, K)
    e1.record(stream)
    batch.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    sizes = np.array([n for _, n, _ in mine], dtype=np.int64)
    points = int(sum(int(n) * (int(n) + 1) * int(n) for n in sizes))
    tunings = {}
    for ctx, n in zip(batch.members, sizes):
        tunings.setdefault(str(int(n)), ctx.tuning())
    batch.close()
    if dist is not None:
        t = torch.tensor([ms, float(points)], device=f"cuda:{device}", dtype=torch.float64)
        tmax = t.clone()
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        ms, points = float(tmax[0].item()), int(t[1].item())
    res = np.array([re for _, _, re in mine])
    return {"members": members, "steps": K, "ms_per_batch_step": ms / K,
            "grid_points_steps_per_s": points * K / (ms / 1000.0), "grid_points": points,
            "members_per_rank": len(mine), "partition_imbalance": imbalance(members, world),
            "sizes": {str(n): int((sizes == n).sum()) for n in (32, 48, 64, 96)},
            "re_tau_range": [float(res.min()), float(res.max())] if len(res) else None, "tuning": tunings}


def run_adjoint(device: int, seed: int, reps: int = 3) -> dict:
    """Adjoint form: a 64 x 65 x 64 channel (96 x 97 x 96 product grid) at
    Re_tau 180 from a log-law mean plus a k^-5/3 perturbation (10 % rms), the
    wall shear stress averaged over 50 steps, wall blowing/suction on the
    |k| <= 8 modes (0.01 per mode), checkpoints every 10 steps.  The forward
    run (cdns_run, iterations 1..50) and the gradient run (cdns_adjoint_run:
    forward sweep, recomputation and reverse steps) are timed with CUDA events
    on the context stream, best of `reps`; a 4th-order central difference
    along one velocity and one control direction checks the gradient."""
    import numpy as np
    import torch
    import cdns
    from cdns.fields import blowing_suction, divergence_free_field
    mesh, params = ensemble_case(64, 180.0)
    N, KC = 50, 10
    u0 = np.stack(divergence_free_field(mesh, params, seed=seed, amp=0.1, spectrum="k53", mean="loglaw"), axis=-1)
    bc0 = blowing_suction(mesh, seed + 1, amp=1e-2)
    ctx = cdns.Context(mesh, params, device=device)
    ctx.set_velocity_bc(bc0)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=device)

    def timed(fn):
        best = float("inf")
        for _ in range(reps):
            ctx.set_velocity(u0)
            ctx.synchronize()
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            out = fn()
            b.record(stream)
            torch.cuda.synchronize()
            best = min(best, a.elapsed_time(b))
        return best, out

    def forward():
        ctx.run(1, N)
        ctx.synchronize()

    ms_fwd, _ = timed(forward)

    def forward_steady():
        ctx.run(3, N)   # 50 steady steps (graph replay), the setup already in place
        ctx.synchronize()

    ctx.set_velocity(u0)
    ctx.run(1, 2)
    ctx.synchronize()
    ms_steady, _ = timed(forward_steady)
    ms_sweep, _ = timed(lambda: ctx.adjoint_run(N, KC, gradient=False))
    ms_grad, (J0, gu, gb) = timed(lambda: ctx.adjoint_run(N, KC))
    # central-difference spot check (4th order) along a velocity and a control direction
    du = np.stack(divergence_free_field(mesh, params, seed=seed + 2, amp=0.05, kmax=8), axis=-1)
    du[mesh.NZS, :, 0, 0] = np.random.default_rng(seed + 3).standard_normal(mesh.NYS + 1) * 0.3
    dc = blowing_suction(mesh, seed + 4)
    errs = []
    for d_u, d_c, h in ((du, 0.0 * bc0, 1e-2), (0.0 * u0, dc, 1e-4)):
        def J(t):
            ctx.set_velocity(u0 + t * d_u)
            return ctx.adjoint_run(N, KC, control=bc0 + t * d_c, gradient=False)[0]
        fd = (J(-2 * h) - 8 * J(-h) + 8 * J(h) - J(2 * h)) / (12 * h)
        ad = float(np.sum(np.real(np.conj(gu) * d_u)) + np.sum(np.real(np.conj(gb) * d_c)))
        errs.append(abs(fd - ad) / abs(ad))
    out = {"workload": "adjoint_64x65x64_retau180_wall_shear_50_steps_checkpoint_10",
           "steps": N, "checkpoint_interval": KC, "objective": J0,
           "forward_ms": ms_fwd, "gradient_ms": ms_grad, "forward_sweep_ms": ms_sweep,
           "cost_ratio": ms_grad / ms_fwd, "reverse_ratio": (ms_grad - ms_sweep) / ms_fwd,
           "forward_steady_ms": ms_steady, "cost_ratio_steady": ms_grad / ms_steady,
           "fd_rel_err": errs, "device_bytes": ctx.device_bytes(),
           "note": "cost_ratio = gradient run (forward sweep + recomputation + reverse steps) / forward run "
                   "(cdns_run of iterations 1..50, with its two setups); cost_ratio_steady divides by 50 "
                   "steady graph-replayed steps without setup; reverse_ratio excludes the forward sweep"}
    ctx.close()
    return out


def run_pencil(ranks: int, steps: int, warmup: int, device: int, seed: int, exchange: str = "copy") -> dict:
    """The workload as a `ranks`-way pencil decomposition with every rank in
    this process on one GPU (cdns.pencil.LocalPencil): each rank's three stages
    per step timed with CUDA events on its stream, one rank at a time, the
    exchanges between stages done by device copies (not timed: across GPUs
    they are NVLink all-to-alls).  Reports per-rank stage times, their maximum
    (a rank's device time per step) and sum (the decomposition's total
    device work against the single-context step), and the bytes each rank
    sends to other ranks per step."""
    import numpy as np
    import torch
    from cdns import pencil
    from cdns.fields import divergence_free_field
    mesh, params = workload_mesh()
    u0 = np.stack(divergence_free_field(mesh, params, seed=seed, amp=0.1, spectrum="k53", mean="loglaw"),
                  axis=-1)
    lp = pencil.LocalPencil(mesh, params, ranks, device, exchange=exchange)
    try:
        lp.set_velocity(u0)
        lp.run(1, warmup)
        streams = [m.torch_stream() for m in lp.members]
        ms = np.zeros((ranks, 3))
        for it in range(warmup + 1, warmup + 1 + steps):
            for st in range(3):
                for r, m in enumerate(lp.members):
                    a = torch.cuda.Event(enable_timing=True)
                    b = torch.cuda.Event(enable_timing=True)
                    a.record(streams[r])
                    m.stage(it, st)
                    b.record(streams[r])
                    m.synchronize()
                    ms[r, st] += a.elapsed_time(b)
                if st < 2 and exchange == "copy":
                    lp._exchange(st)
        ms /= steps
        sent = [sum(8 * (sum(m.exchange_counts(e)[0]) - m.exchange_counts(e)[0][r]) for e in (0, 1))
                for r, m in enumerate(lp.members)]
        finite = bool(np.isfinite(lp.get_velocity()).all())
    finally:
        lp.close()
    per_rank = ms.sum(axis=1)
    if exchange == "peer":
        sent = [0] * ranks   # peer loads and stores instead of exchange buffers
    return {"ranks": ranks, "steps": steps, "exchange": exchange, "layout": pencil.layout(mesh, ranks),
            "stage_ms": [[round(float(x), 5) for x in row] for row in ms],
            "rank_max_ms": float(per_rank.max()), "rank_sum_ms": float(per_rank.sum()),
            "bytes_to_peers_per_step": max(sent), "finite": finite,
            "emulated": "all ranks in one process on one GPU, stages one rank at a time, "
                        "exchanges by device copies (untimed)"}


def _rounded(x, digits: int = 6):
    """Floats to `digits` significant digits (keeps the bench line short)."""
    if isinstance(x, float):
        return float(f"{x:.{digits}g}") if math.isfinite(x) else x
    if isinstance(x, dict):
        return {k: _rounded(v, digits) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [_rounded(v, digits) for v in x]
    return x


def compact_mixed(m):
    if not m:
        return m
    return {k: m[k] for k in ("value", "unit", "ms_per_step", "speedup_vs_fp64", "rel_l2_vs_fp64_after_1000_steps",
                              "statistics_rel_l2_vs_fp64") if k in m}


def compact_ensemble(e):
    if not e:
        return e
    return {label: {k: r[k] for k in ("members", "grid_points", "ms_per_batch_step", "grid_points_steps_per_s")}
            for label, r in e.items()}


def compact_adjoint(a):
    if not a:
        return a
    return {k: a[k] for k in ("steps", "checkpoint_interval", "forward_ms", "gradient_ms", "cost_ratio",
                              "cost_ratio_steady", "fd_rel_err") if k in a}


def compact_pencil(pa):
    if not pa:
        return pa
    out = {k: pa[k] for k in ("ranks", "rank_max_ms", "rank_sum_ms", "overhead", "bytes_to_peers_per_step",
                              "error") if k in pa}
    if "fused_exchange" in pa:
        out["fused_exchange"] = {k: pa["fused_exchange"][k] for k in ("rank_max_ms", "overhead")}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=0, help="steps of the e2e pass (default: min(K, 200))")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed FP32/FP64 arm")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the ensemble-batch arm")
    ap.add_argument("--ensemble-members", type=int, default=64)
    ap.add_argument("--ensemble-steps", type=int, default=200)
    ap.add_argument("--no-adjoint", action="store_true", help="skip the discrete-adjoint arm")
    ap.add_argument("--no-output", action="store_true", help="skip the statistics-sampling arm")
    ap.add_argument("--pencil", type=int, default=8,
                    help="also time a P-rank pencil decomposition of the workload on this GPU (0: skip)")
    ap.add_argument("--detail", default="", help="also write the full results (tuning, per-stage and "
                                                 "per-rank times) to this JSON file")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")

    import numpy as np
    import torch
    import cdns
    from cdns.fields import divergence_free_field

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()

    mesh, params = workload_mesh()
    u0 = divergence_free_field(mesh, params, seed=1 + rank, amp=0.1, spectrum="k53", mean="loglaw")
    host_u = torch.from_numpy(np.stack(u0, axis=-1)).pin_memory()
    host_v = torch.empty_like(host_u).pin_memory()
    host_p = torch.empty(host_u.shape[:-1], dtype=torch.complex128).pin_memory()
    ctx = cdns.Context(mesh, params, device=local)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=local)
    K, W = args.steps, args.warmup

    # ---- device-resident throughput ------------------------------------
    clocks = ClockSampler(local)
    clocks.start()
    ctx.set_velocity(host_u.numpy())
    # iterations 1-2 each run EqSolvePV::setup (its g changes): timed apart, not in `value`
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    ctx.run(1, 2)
    s1.record(stream)
    ctx.run(3, W - 2)
    ctx.synchronize()
    setup_ms = s0.elapsed_time(s1)
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.run(W + 1, K)
    e1.record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms_total = e0.elapsed_time(e1)
    t = torch.tensor([ms_total], device=f"cuda:{local}", dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    ms_per_step = ms_max / K
    value = world * K / (ms_max / 1000.0)

    # ---- per-stage timing (roofline of the dominant stage) ---------------
    ctx.profile_begin()
    nprof = 20
    ctx.run(W + K + 1, nprof)
    stage_ms, nst = ctx.profile_end()
    per_launch = {k: v / nst for k, v in stage_ms.items()}
    sb = stage_bytes(mesh)
    top = max(per_launch, key=per_launch.get)
    peak, peak_kind = measured_peak()
    achieved = sb[top] / (per_launch[top] * 1e-3) / 1e9
    step_model = step_bytes_model(mesh)

    # ---- statistics sampled every step (device-side output reduction) ------
    output = None
    if not args.no_output:
        KS = min(K, 200)
        ctx.statistics_reset()
        ctx.set_velocity(host_u.numpy())
        ctx.run(1, W)
        ctx.statistics_sample()
        ctx.synchronize()
        torch.cuda.synchronize()
        o0 = torch.cuda.Event(enable_timing=True)
        o1 = torch.cuda.Event(enable_timing=True)
        o2 = torch.cuda.Event(enable_timing=True)
        o0.record(stream)
        for it in range(W + 1, W + KS + 1):
            ctx.step(it)
            ctx.statistics_sample()
        o1.record(stream)
        for _ in range(KS):
            ctx.statistics_sample()
        o2.record(stream)
        ctx.synchronize()
        torch.cuda.synchronize()
        ms_sampled = o0.elapsed_time(o1) / KS
        ms_sample = o1.elapsed_time(o2) / KS
        ny1, nzc, nxc = mesh.NY + 1, mesh.NZ, mesh.NX
        ns = (2 * mesh.NZS + 1) * (mesh.NYS + 1) * (mesh.NXS + 1)
        ncol = (2 * mesh.NZS + 1) * (mesh.NXS + 1)
        # divergence (u, v, w, p in; p, div out) + y synthesis (5 fields) + z (5) + fused x/moments (5 in)
        red_bytes = 16 * (6 * ns + 5 * ns + 2 * 5 * ny1 * ncol + 2 * 5 * ny1 * nzc * (mesh.NXS + 1))
        t0 = time.perf_counter()
        for _ in range(20):
            ctx.output_reduce()
        ms_sync = (time.perf_counter() - t0) * 1e3 / 20
        output = {"workload": "statistics sampled every step (to_physical + Statistics::reduce + accumulate "
                              "on the 128x129x128 coarse grid)",
                  "steps_per_s_sampled": world * 1000.0 / ms_sampled, "ms_per_sampled_step": ms_sampled,
                  "ms_per_sample": ms_sample, "sample_overhead_vs_step": ms_sample / ms_per_step,
                  "sample_bytes": red_bytes,
                  "sample_hbm_frac": red_bytes / (ms_sample * 1e-3) / 1e9 / peak,
                  "output_reduce_call_ms": ms_sync,
                  "note": "output_reduce_call_ms: the synchronous call (plane sums and diagnostics to the "
                          "host), host wall clock; the others CUDA events on the context stream"}

    # ---- mixed FP32/FP64 arm: throughput and error after 1000 steps ------
    mixed = None
    if not args.no_mixed:
        cm = cdns.Context(mesh, params, device=local, precision=cdns.PRECISION_MIXED)
        sm_ = torch.cuda.ExternalStream(cm.stream_ptr(), device=local)
        cm.set_velocity(host_u.numpy())
        cm.run(1, W)
        cm.synchronize()
        barrier()
        torch.cuda.synchronize()
        m0 = torch.cuda.Event(enable_timing=True)
        m1 = torch.cuda.Event(enable_timing=True)
        m0.record(sm_)
        cm.run(W + 1, K)
        m1.record(sm_)
        cm.synchronize()
        torch.cuda.synchronize()
        barrier()
        tm = torch.tensor([m0.elapsed_time(m1)], device=f"cuda:{local}", dtype=torch.float64)
        if dist is not None:
            dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        mixed_ms = float(tm.item()) / K
        cm.profile_begin()
        cm.run(W + K + 1, nprof)
        mstage, mst = cm.profile_end()
        # error against the FP64 path after 1000 steps from the same field, with
        # a statistics sample after every step (mean profile, Reynolds stresses)
        nerr = 1000
        stats = []
        for c_ in (ctx, cm):
            c_.set_velocity(host_u.numpy())
            c_.statistics_reset()
            for it in range(1, nerr + 1):
                c_.step(it)
                c_.statistics_sample()
            c_.synchronize()
            stats.append(c_.statistics_read()[2])
        v64, v32 = ctx.get_velocity(), cm.get_velocity()
        errs = [float(np.linalg.norm(v32[..., k] - v64[..., k]) / np.linalg.norm(v64[..., k])) for k in range(3)]

        def rel(a, b):
            return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

        def stresses(mn):
            return [mn[4] - mn[0] ** 2, mn[5] - mn[1] ** 2, mn[6] - mn[2] ** 2, mn[7] - mn[0] * mn[1]]
        stat_errs = {"mean_U": rel(stats[1][0], stats[0][0])}
        for name, a, b in zip(("uu", "vv", "ww", "uv"), stresses(stats[1]), stresses(stats[0])):
            stat_errs["reynolds_" + name] = rel(a, b)
        mixed = {"value": world * 1000.0 / mixed_ms, "unit": "steps/s", "ms_per_step": mixed_ms,
                 "speedup_vs_fp64": ms_per_step / mixed_ms,
                 "rel_l2_vs_fp64_after_1000_steps": errs,
                 "statistics_rel_l2_vs_fp64": stat_errs,
                 "stage_ms": {k: round(v / mst, 5) for k, v in mstage.items()},
                 "arithmetic": "fine-grid stages stored FP32; curl, Chebyshev accumulation, "
                               "tau solves, corrections and mean flow FP64"}
        cm.close()

    # ---- ensemble arm: independent channels of seeded sizes in one batch ---
    ensemble = None
    if not args.no_ensemble:
        ensemble = {}
        for label, prec in (("fp64", cdns.PRECISION_FP64), ("mixed", cdns.PRECISION_MIXED)):
            ensemble[label] = run_ensemble(args.ensemble_members, args.ensemble_steps, W, prec, local,
                                           1000, world, rank, dist)

    # ---- discrete-adjoint arm: gradient cost against the forward run ------
    adjoint = None
    if not args.no_adjoint:
        adjoint = run_adjoint(local, 2000 + rank)

    # ---- pencil decomposition, emulated on this GPU (opt-in) ---------------
    pencil_arm = None
    if args.pencil > 0 and world == 1:
        try:
            pencil_arm = run_pencil(args.pencil, min(K, 20), W, local, 1)
            pencil_arm["single_ms"] = ms_per_step
            pencil_arm["overhead"] = pencil_arm["rank_sum_ms"] / ms_per_step
            fused = run_pencil(args.pencil, min(K, 20), W, local, 1, exchange="peer")
            pencil_arm["fused_exchange"] = {k: fused[k] for k in ("stage_ms", "rank_max_ms", "rank_sum_ms", "finite")}
            pencil_arm["fused_exchange"]["overhead"] = fused["rank_sum_ms"] / ms_per_step
        except Exception as exc:  # an auxiliary arm must not hide the main line
            pencil_arm = {"ranks": args.pencil, "error": str(exc)[:200]}

    # ---- end to end through the C ABI with host buffers -------------------
    KE = args.e2e_steps or min(K, 200)
    ctx2 = cdns.Context(mesh, params, device=local)
    s2 = torch.cuda.ExternalStream(ctx2.stream_ptr(), device=local)
    barrier()
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(s2)
    ctx2.set_velocity(host_u.numpy())
    dp = None
    for it in range(1, KE + 1):
        ctx2.step(it)
        dp = ctx2.dpdx()
    ctx2.synchronize()
    v_np = ctx2.get_velocity(out=host_v.numpy())
    p_np = ctx2.get_pressure(out=host_p.numpy())
    f1.record(s2)
    torch.cuda.synchronize()
    e2e_ms = f0.elapsed_time(f1)
    t = torch.tensor([e2e_ms], device=f"cuda:{local}", dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_ms = float(t.item())
    e2e_value = world * KE / (e2e_ms / 1000.0)
    state_bytes = host_u.numel() * 16
    h2d = state_bytes / KE
    d2h = 16 + (host_u.numel() + host_p.numel()) * 16 / KE
    finite = bool(np.isfinite(v_np).all() and np.isfinite(p_np).all())

    # ---- CPU baseline (rank 0, N = 1) ----------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            v_cpu, info = reference_arm_time(10, 2, os.cpu_count() or 1, reps=3)
            cpu = dict(info, value=v_cpu, unit="steps/s")
        except Exception as exc:  # the baseline must not hide the GPU line
            cpu = {"value": None, "unit": "steps/s", "error": str(exc)[:200]}

    if rank == 0:
        traffic, traffic_note = ncu_traffic(top)
        detail = {"tuning": ctx.tuning(), "mixed": mixed, "ensemble": ensemble, "adjoint": adjoint,
                  "statistics": output, "pencil": pencil_arm, "cpu_baseline": cpu,
                  "stage_ms": per_launch}
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(WORKLOAD),
            "parallelism": f"replicas{world}",
            "throughput": {"grid_points_steps_per_s": value * 128 * 129 * 128,
                           "product_points_steps_per_s": value * 196 * 193 * 196,
                           "step_model_bytes": step_model,
                           "step_roofline_frac": (step_model / (ms_per_step * 1e-3) / 1e9) / peak},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_note,
                         "kernel": top, "algorithmic_bytes": sb[top], "launch_ms": per_launch[top],
                         "peak_source": peak_kind,
                         "stage_ms": {k: round(v, 4) for k, v in per_launch.items()}},
            "cpu_baseline": None if cpu is None else {
                k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample", "error") if k in cpu},
            "mixed": compact_mixed(mixed),
            "ensemble": compact_ensemble(ensemble),
            "adjoint": compact_adjoint(adjoint),
            "statistics": None if output is None else {
                k: output[k] for k in ("steps_per_s_sampled", "ms_per_sample", "sample_hbm_frac")},
            "pencil": compact_pencil(pencil_arm),
            "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": KE, "finite": finite,
                    "protocol": "upload + steps 1..K (setup included) one call each with dpdx readback + download"},
            "clocks": clk,
            "setup_steps": {"ms": setup_ms, "steps": 2},
            "gpu_launches": len(per_launch) * K,   # one kernel per stage per step
        }
        print(json.dumps(_rounded(line)), flush=True)
        if args.detail:
            with open(args.detail, "w") as fh:
                json.dump(_rounded(dict(line, detail=detail)), fh, indent=1)
    ctx.close()
    ctx2.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
