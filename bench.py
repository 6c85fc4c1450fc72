#!/usr/bin/env python
"""Benchmark: particle-steps/s of the SPMHD particle update on B200.

Workload (default): 3-D MHD blast, 128^3 = 2,097,152 particles on a cubic
lattice in the periodic unit cube [-0.5, 0.5]^3, rho = 1, p = 0.1 except
p = 10 for r < 0.1, B = (1/sqrt2, 1/sqrt2, 0), gamma = 5/3, cubic spline
kernel with hfact 1.2 (configs/mhdblast.toml), Cullen-Dehnen alpha in
[0.1, 1], artificial viscosity / conduction / resistivity 1, cleaning 1/1.
Synthetic seeded inputs of that shape; no dataset is involved.

One "step" is one predictor-evaluate-corrector step of the whole particle
set (neighbour sort, iterated density, fused force pass, FP64 dt reduction,
fused corrector-predictor), after the reference's 3-RHS warm-up.  The K
timed steps run as one captured CUDA graph (``mhd_advance``); the kernel
breakdown comes from K more steps of the same kernels run uncaptured.  Inputs
(state 35 fields x 2.1M x 8 B ~ 590 MB) exceed the 126 MB L2, so no flush
is needed between steps.

The same line carries the batched form (``batched_form``): 64 independent
2-D Orszag-Tang instances of uneven size advanced 100 steps in one captured
graph launch after the autotuner, against the plain FP64 path run instance
by instance.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
    python bench.py --workload ot128|briowu   # the 2-D Orszag-Tang and Brio-Wu measurements

Multi-GPU: "replicas only" -- every rank advances its own independent blast
(the per-instance update does not shard without a halo exchange); value is
the particle-steps of all ranks over the max-over-ranks time.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "pysph-mhd_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "particle-steps/s on 1 B200, FP32/batched vs plain FP64 at stated L2 error"
UNIT = "particle-steps/s"

# Algorithmic bytes per particle of the fused force pass: its seven record
# planes of four values (FP32: 16 B each, FP64: 32 B), each neighbour's
# counted once (ideal reuse), the seven FP64 epilogue inputs (rho omega cs
# psipred p epred h) and the 16 FP64 outputs (au av aw ae ah div div_for_psi
# dt_cfl dt_adapt aBevol x3 apsi divBsymm divBdiff alphaloc).
FORCE_BYTES_PER_PARTICLE = {"fp64": 7 * 32 + 7 * 8 + 16 * 8, "fp32": 7 * 16 + 7 * 8 + 16 * 8}
# Floating-point operations of one neighbour pair of k_force_pass
# (csrc/mhd_force.cu), counted statically from its source: +, -, *, /,
# sqrt, rsqrt and reciprocal count 1, a fused multiply-add 2; comparisons,
# max/min and int -> float conversions are not counted.  Cubic kernel, the
# pair inside the kernel's outer segment (1 < q <= 2, 7 of 8 pairs on a
# lattice), the viscosity branch not taken.  FP32: geometry 12, the two
# kernel gradients 15, omega factors, dv and v.x 10, Cullen-Dehnen moments
# 55, signal speed 3, pressure coefficient 5, Maxwell projections 12,
# momentum 27 (three Kahan adds), div v 6, conduction speed 7, energy terms
# 15, field projections and resistive speed 27, dissipation 6, induction
# and cleaning terms 9 + 27, energy sum 13, div B sums 14 -- 253, of which
# 40 are the compensation of the ten Kahan sums; FP64 (plain sums) 223.  A
# list entry beyond the cut-off costs its geometry (12).  The density pass:
# 33 per pair in FP32 (geometry 10, kernel 8, two Kahan sums 15).
FORCE_FLOPS_PER_PAIR = {"fp32": 253, "fp64": 223}
FORCE_FLOPS_PER_CANDIDATE = 12
DENSITY_FLOPS_PER_PAIR = {"fp32": 33, "fp64": 25}


def blast_case(n: int, precision: str = "fp64", hot_radius: float = 0.1):
    dx = 1.0 / n
    ax = -0.5 + (np.arange(n) + 0.5) * dx
    x, y, z = np.meshgrid(ax, ax, ax, indexing="ij")
    x, y, z = x.ravel(), y.ravel(), z.ravel()
    cnt = x.size
    gamma = 5.0 / 3.0
    p = np.where(x * x + y * y + z * z < hot_radius * hot_radius, 10.0, 0.1)
    b = 1.0 / math.sqrt(2.0)
    ic = dict(x=x, y=y, z=z, u=np.zeros(cnt), v=np.zeros(cnt), w=np.zeros(cnt), rho=np.ones(cnt),
              h=np.full(cnt, 1.2 * dx), m=np.full(cnt, dx ** 3), e=p / (gamma - 1.0), Bx=np.full(cnt, b),
              By=np.full(cnt, b), Bz=np.zeros(cnt), alpha1=np.full(cnt, 0.1), gid=np.arange(cnt, dtype=np.float64))
    prm = dict(dim=3, kernel="cubic", hfact=1.2, density="iterate", gamma=gamma, mu0=1.0, av=1.0, ac=1.0, ar=1.0,
               clean_speed=1.0, clean_damp=1.0, timestep_factor=1.0, tf=1e30, lo=[-0.5] * 3, hi=[0.5] * 3,
               periodic=[True] * 3, alpha_min=0.1, alpha_max=1.0, precision=precision)
    return ic, prm


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.samples = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.idx), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[5 + k].lower() == "active"})
        pw = [float(s[3]) for s in self.samples if s[3].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples), "power_w_max": max(pw) if pw else None}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "of measured"
    return 6650.0, "of fallback"


def profiled_traffic(n, precision):
    """DRAM bytes per force-pass launch from the committed ncu summary, scaled
    to n particles (traffic grows in proportion to the particles processed)."""
    path = os.path.join(ROOT, "profiles", "force_pass_blast96_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    per = d.get(precision, {}).get("dram_bytes_per_particle")
    return None if per is None else float(per) * n


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def oracle_rate(n_side, steps, warm_steps=0):
    """Particle-steps/s of the C oracle (the reference restated, OpenMP over all
    host threads) on the blast at n_side^3: the 3-RHS warm-up and
    `warm_steps` steps untimed, then `steps` timed.  Returns the rate, the
    timed seconds, the particle count and the density passes of each timed
    step."""
    import oracle

    oracle.build()
    ic, prm = blast_case(n_side)
    s = oracle.State(ic)
    o = oracle.Oracle(prm, exact_order=False, nthreads=cpu_cores())
    o.warmup(s)
    dt = o.initial_dt(s)
    for _ in range(warm_steps):
        o.step(s, dt)
        dt = o.min_dt(s)
    passes = []
    t0 = time.perf_counter()
    for _ in range(steps):
        passes.append(o.step(s, dt))
        dt = o.min_dt(s)
    el = time.perf_counter() - t0
    return s.n * steps / el, el, s.n, passes


def blast_workload(n_side):
    """The workload name both arms put in config.workload."""
    return (f"3-D MHD blast {n_side}^3 = {n_side ** 3} particles, cubic kernel hfact 1.2, alpha [0.1, 1], "
            f"periodic unit cube")


def oracle_sample(n_side, warm, steps, el, passes):
    return (f"C oracle (reference equations restated, FP64, OpenMP {cpu_cores()} threads): 3-D blast at {n_side}^3 "
            f"= {n_side ** 3} particles, the 3-RHS warm-up and {warm} steps untimed, then {steps} timed PEC steps "
            f"({el:.1f} s; density passes per step {passes})")


def run_reference(args, rank):
    if rank != 0:
        return
    n_side = args.ref_n or args.n
    rate, el, n, passes = oracle_rate(n_side, args.steps, args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": blast_workload(args.n), "timed_workload": blast_workload(n_side),
                   "form": "fp64 (the oracle)", "sample_particles": n},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cpu_cores(), "kind": "port",
                         "sample": oracle_sample(n_side, args.warmup, args.steps, el, passes)},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _timed(args, prec, dev, barrier, dist, world):
    """W untimed + K timed fused steps of the blast in one precision form.

    The timed steps are one captured run (``mhd_advance``: a CUDA graph of K
    fused steps, grids planned on the device); the per-kernel breakdown and
    the pair counts come from K more steps of the same kernels run uncaptured
    with CUDA events around every launch (outside the timed region)."""
    import ctypes

    import torch

    from src import _abi
    from src.batch import BatchEngine
    from src.engine import params_from_dict

    ic, prm = blast_case(args.n, prec)
    n = args.n ** 3
    lib = _abi.load()
    eng = BatchEngine(params_from_dict(prm), [ic])
    eng.warmup()
    eng.begin(eng.initial_dt())
    eng.advance(args.warmup, finish=False)
    # capture the K-step graph once (runs K steps; the state stays valid)
    eng.advance(args.steps, finish=False)
    torch.cuda.synchronize()
    snap = eng.snapshot()
    replays0 = eng.replays
    launches0 = eng.launches()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    listed, rebuilt = ctypes.c_int64(), ctypes.c_int64()
    lib.mhd_list_counts(eng.ctx, ctypes.byref(listed), ctypes.byref(rebuilt), st)
    clocks = ClockSampler(dev.index or 0)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    eng.advance(args.steps, finish=False, snapshot=snap)
    e1.record()
    torch.cuda.synchronize()
    barrier()
    clocks.stop()
    ms = e0.elapsed_time(e1)
    lib.mhd_list_counts(eng.ctx, ctypes.byref(listed), ctypes.byref(rebuilt), st)
    launches = eng.launches() - launches0
    replays = eng.replays - replays0
    ms_max = ms
    if dist:
        import torch.distributed as tdist

        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        ms_max = float(t.item())
    # kernel breakdown (uncaptured, identical kernels)
    ms_k = (ctypes.c_double * len(_abi.TIMING_KINDS))()
    cnt_k = (ctypes.c_int64 * len(_abi.TIMING_KINDS))()
    pairs, cands = ctypes.c_int64(), ctypes.c_int64()
    lib.mhd_pair_counts(eng.ctx, ctypes.byref(pairs), ctypes.byref(cands), st)
    lib.mhd_timing_enable(eng.ctx, 1)
    lib.mhd_timing_read(eng.ctx, ms_k, cnt_k)
    e0.record()
    eng.advance(args.steps, finish=False, capture=False)
    e1.record()
    torch.cuda.synchronize()
    ms_unc = e0.elapsed_time(e1)
    lib.mhd_timing_read(eng.ctx, ms_k, cnt_k)
    lib.mhd_pair_counts(eng.ctx, ctypes.byref(pairs), ctypes.byref(cands), st)
    lib.mhd_timing_enable(eng.ctx, 0)
    if args.profile_steps > 0:
        # steady-state steps bracketed for a profiler started with
        # --profile-from-start off (outside every timed region)
        torch.cuda.profiler.start()
        eng.advance(args.profile_steps, finish=False, capture=False)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
    eng.rhs()
    passes = int(eng.last_stats.density_passes)
    eng.close()
    kern = {k: {"ms_total": ms_k[i], "launches": int(cnt_k[i])} for i, k in enumerate(_abi.TIMING_KINDS)}
    return {"value": world * n * args.steps / (ms_max * 1e-3), "ms_per_step": ms_max / args.steps,
            "ms_per_step_uncaptured": ms_unc / args.steps, "kernels": kern, "launches": launches,
            "replays": replays, "clocks": clocks.summary(), "pairs": pairs.value, "candidates": cands.value,
            "passes": passes, "lists_rebuilt": rebuilt.value / max(listed.value, 1)}


def _batched(args, dev, rank=0, world=1):
    """The batched form: 64 independent 2-D Orszag-Tang instances (N ~ U{32..256},
    B0 x U[0.8, 1.2], seed 0) advanced 100 steps as one captured graph after
    the autotuner, against the plain FP64 path run instance by instance.
    With N ranks the instances are shared out by particle count
    (src.parallel.shard_instances); each rank runs its share in FP32, the
    value is all particle-steps over the slowest rank's time, and the ranks'
    per-instance checksums are gathered."""
    import ctypes

    import torch

    from src import _abi
    from src.parallel import checksum, gather_instances, max_over_ranks, shard_instances

    from src.batch import BatchEngine
    from src.cases.orstang import orszag_tang_batch
    from src.config import load_config
    from src.engine import Engine, params_from_dict
    from src.particle_array import ParticleArray
    from src.run import CASES

    cfg = load_config(os.path.join(PKG, "configs", "orstang2d.toml"), {k: v.config_type for k, v in CASES.items()})
    inst, prm, sizes, scales = orszag_tang_batch(cfg, n_inst=args.batch_instances, seed=0)
    total = int(sum(len(a["x"]) for a in inst))
    n_all = len(inst)
    share = shard_instances([len(a["x"]) for a in inst], world)[rank]
    inst = [inst[k] for k in share]
    steps = args.batch_steps
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out, final = {}, {}
    for prec in ("fp32", "fp64") if world == 1 else ("fp32",):
        eng = BatchEngine(params_from_dict(prm, prec), inst)
        eng.warmup()
        eng.begin(eng.initial_dt())
        t0 = time.perf_counter()
        tuned = eng.tune(steps=4)
        tune_s = time.perf_counter() - t0
        snap = eng.snapshot()
        eng.advance(steps, finish=True, snapshot=snap)  # capture + first run
        eng.restore(snap)
        torch.cuda.synchronize()
        l0, r0 = eng.launches(), eng.replays
        ev0.record()
        eng.advance(steps, finish=True, snapshot=snap)
        ev1.record()
        ev1.synchronize()
        ms = max_over_ranks(ev0.elapsed_time(ev1), dev)
        out[prec] = {"value": total * steps / (ms * 1e-3), "ms": ms, "gpu_launches": eng.launches() - l0,
                     "graph_launches": 1, "replays": eng.replays - r0, "tune_s": tune_s,
                     "tuned": {"stencil": tuned["stencil"], "force_shape": tuned["force_shape"]}}
        final[prec] = eng.pa.pull("rho", "u", "v", "Bx", "By", "gid", order="gid")
        if world > 1:
            sums = gather_instances({k: checksum(eng.pull_instance(i, "rho", "u", "v", "Bx", "By"))
                                     for i, k in enumerate(share)}, n_all)
        # where the captured run's time goes: the same kernels run uncaptured
        # for a few steps with CUDA events around each family (the density
        # iteration host-checked there, so its passes are the needed ones)
        lib = _abi.load()
        ms_k = (ctypes.c_double * len(_abi.TIMING_KINDS))()
        cnt_k = (ctypes.c_int64 * len(_abi.TIMING_KINDS))()
        lib.mhd_timing_enable(eng.ctx, 1)
        lib.mhd_timing_read(eng.ctx, ms_k, cnt_k)
        k_unc = 5
        eng.restore(snap)
        eng.advance(k_unc, finish=False, capture=False)
        lib.mhd_timing_read(eng.ctx, ms_k, cnt_k)
        lib.mhd_timing_enable(eng.ctx, 0)
        out[prec]["kernels_ms_per_step"] = {k: ms_k[i] / k_unc for i, k in enumerate(_abi.TIMING_KINDS)}
        out[prec]["captured_ms_per_step"] = ms / steps
        out[prec]["launches_per_step"] = out[prec]["gpu_launches"] / steps
        eng.close()
    if world > 1:
        return {"workload": f"{n_all} x 2-D Orszag-Tang (seed 0), {total} particles, {steps} steps, instances "
                            f"shared out over {world} ranks by particle count",
                "particles": total, "steps": steps, "fp32": out["fp32"], "ranks": world,
                "instance_checksums_sum": float(sum(sums))}
    # plain FP64 path, one instance at a time (K steps each, summed device time)
    k_loop = args.batch_loop_steps
    loop_ms = 0.0
    for a in inst:
        eng = Engine(params_from_dict(prm, "fp64"), ParticleArray("fluid", dict(a), device=dev))
        eng.warmup()
        eng.begin(eng.initial_dt())
        torch.cuda.synchronize()
        ev0.record()
        eng.advance(k_loop, finish=False)
        ev1.record()
        ev1.synchronize()
        loop_ms += ev0.elapsed_time(ev1)
        eng.close()
    loop = total * k_loop / (loop_ms * 1e-3)
    # the plain FP64 path at its fastest one instance at a time: each
    # instance alone on the device planner, its `steps` steps captured once
    # and timed as one graph launch (summed device time over the instances)
    cap_ms, cap_launches = 0.0, 0
    for a in inst:
        eng = BatchEngine(params_from_dict(prm, "fp64"), [dict(a)])
        eng.warmup()
        eng.begin(eng.initial_dt())
        snap = eng.snapshot()
        eng.advance(steps, finish=True, snapshot=snap)  # capture + first run
        eng.restore(snap)
        torch.cuda.synchronize()
        l0 = eng.launches()
        ev0.record()
        eng.advance(steps, finish=True, snapshot=snap)
        ev1.record()
        ev1.synchronize()
        cap_ms += ev0.elapsed_time(ev1)
        cap_launches += eng.launches() - l0
        eng.close()
    captured = total * steps / (cap_ms * 1e-3)
    # control: the FP64 batch again with every x moved by 1e-10 of its
    # instance's spacing -- the spread that rounding of any kind reaches on
    # these unjittered lattices (their Cullen-Dehnen limiter starts as
    # roundoff over roundoff)
    rng = np.random.default_rng(1)
    moved = [dict(a_, x=a_["x"] + 1e-10 * rng.uniform(-1.0, 1.0, len(a_["x"])) / np.sqrt(len(a_["x"])))
             for a_ in inst]
    eng = BatchEngine(params_from_dict(prm, "fp64"), moved)
    eng.warmup()
    eng.begin(eng.initial_dt())
    eng.advance(steps, finish=True, capture=False)
    final["fp64_moved"] = eng.pa.pull("rho", "u", "v", "Bx", "By", "gid", order="gid")
    eng.close()

    def rel(keys, a_name="fp32", b_name="fp64"):
        a, b = final[a_name], final[b_name]
        num = sum(float(np.sum((a[k] - b[k]) ** 2)) for k in keys)
        den = sum(float(np.sum(b[k] ** 2)) for k in keys)
        return math.sqrt(num / den)

    return {"workload": f"{len(inst)} x 2-D Orszag-Tang, N x N with N ~ U{{32..256}} (seed 0; sizes "
                        f"{int(sizes.min())}..{int(sizes.max())}), B0 x U[0.8, 1.2], quintic hfact 1.2, "
                        f"{total} particles, {steps} steps in one captured graph launch",
            "particles": total, "steps": steps, "fp32": out["fp32"], "fp64": out["fp64"],
            "fp64_instance_loop": {"value": loop, "steps_per_instance": k_loop, "ms": loop_ms,
                                   "how": "each instance uncaptured through Engine.advance, host-checked density "
                                          "iteration"},
            "fp64_instance_captured": {"value": captured, "steps_per_instance": steps, "ms": cap_ms,
                                       "gpu_launches": cap_launches, "graph_launches": len(inst),
                                       "how": "each instance alone as one captured graph of all its steps"},
            "speedup_fp32_vs_fp64_loop": out["fp32"]["value"] / loop,
            "speedup_fp64_vs_fp64_loop": out["fp64"]["value"] / loop,
            "speedup_fp32_vs_fp64_captured": out["fp32"]["value"] / captured,
            "speedup_fp64_vs_fp64_captured": out["fp64"]["value"] / captured,
            "fp32_vs_fp64_rel_l2": {"rho": rel(["rho"]), "v": rel(["u", "v"]), "B": rel(["Bx", "By"])},
            "fp64_moved_1e-10dx_vs_fp64_rel_l2": {"rho": rel(["rho"], "fp64_moved"), "v": rel(["u", "v"], "fp64_moved"),
                                                  "B": rel(["Bx", "By"], "fp64_moved")}}


def _accuracy(args, dev, steps):
    """rel L2 of the FP32 form against the FP64 path after `steps` steps."""
    from src.engine import Engine, params_from_dict
    from src.particle_array import ParticleArray

    out = {}
    for prec in ("fp64", "fp32"):
        ic, prm = blast_case(args.n, prec)
        eng = Engine(params_from_dict(prm), ParticleArray("fluid", ic, device=dev))
        eng.warmup()
        eng.begin(eng.initial_dt())
        eng.advance(steps)
        out[prec] = eng.pa.pull("rho", "u", "v", "w", "Bx", "By", "Bz", "e", "gid", order="gid")
        eng.close()
    a, b = out["fp32"], out["fp64"]

    def rel(keys):
        num = sum(float(np.sum((a[k] - b[k]) ** 2)) for k in keys)
        den = sum(float(np.sum(b[k] ** 2)) for k in keys)
        return math.sqrt(num / den)

    return {"steps": steps, "rel_l2_rho": rel(["rho"]), "rel_l2_v": rel(["u", "v", "w"]),
            "rel_l2_B": rel(["Bx", "By", "Bz"]), "rel_l2_e": rel(["e"]), "target": 1e-4}


def _derivative(args, dev):
    """The derivative form: gradient of the final magnetic energy of the 2-D
    circularly polarised Alfven wave (configs/alfven2d.toml: 64 x 128,
    amplitude 0.1, single density pass) after `steps` steps with respect to
    (amplitude, alpha_max), by the checkpointed adjoint and by forward mode,
    against central differences of the FP64 drop-in path with the same
    (frozen) step sizes.  The adjoint is timed twice: the first call (CUDA
    module loading, context set-up) and a second, steady-state one.  The
    Alfven wave does not compress, so its alpha_max gradient is zero; a
    second configuration -- a 3-D blast whose shock drives alpha_loc to the
    clip -- checks a non-zero alpha_max gradient against differences."""
    import torch

    from src.config import load_config
    from src.derivative import alfven_case, magnetic_energy_adjoint, magnetic_energy_and_gradient
    from src.engine import Engine, params_from_dict
    from src.particle_array import ParticleArray
    from src.run import CASES

    cfg = load_config(os.path.join(PKG, "configs", "alfven2d.toml"), {k: v.config_type for k, v in CASES.items()})
    steps, every = args.derivative_steps, 16
    times = []
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        la, ga, dts = magnetic_energy_adjoint(cfg, 0.1, 1.0, steps, every=every)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    t1 = time.perf_counter()
    lt, gt, _ = magnetic_energy_and_gradient(cfg, 0.1, 1.0, steps, dts=dts)
    torch.cuda.synchronize()
    t2 = time.perf_counter()

    def energy(o):
        return float(np.sum(o["m"] * (o["Bx"] ** 2 + o["By"] ** 2 + o["Bz"] ** 2) / (2.0 * o["rho"])))

    def drop_in(ic, prm, step_sizes):
        eng = Engine(params_from_dict(dict(prm, density="single")), ParticleArray("fluid", dict(ic), device=dev))
        eng.warmup()
        for dt in step_sizes:
            eng.step(dt)
        o = eng.pa.pull("Bx", "By", "Bz", "m", "rho")
        eng.close()
        return energy(o)

    def loss(a, am):
        ic, _, prm = alfven_case(cfg, a, am)
        return drop_in(ic, prm, dts)

    ea = 1e-4 * 0.1
    fd_a = (loss(0.1 + ea, 1.0) - loss(0.1 - ea, 1.0)) / (2.0 * ea)
    fd_m = (loss(0.1, 1.1) - loss(0.1, 0.9)) / 0.2
    out = {"workload": f"2-D circularly polarised Alfven wave, 64 x 128 lattice, periodic box 1 x 2, rho 1, p 0.1, "
                       f"B_par 1, amplitude 0.1, Wendland C6 hfact 1.9, artificial viscosity 1, single density "
                       f"pass; final magnetic energy after {steps} steps (frozen step sizes)",
           "loss": la, "grad_adjoint": {"amplitude": float(ga[0]), "alpha_max": float(ga[1])},
           "grad_forward_mode": {"amplitude": float(gt[0]), "alpha_max": float(gt[1])},
           "central_differences": {"amplitude": fd_a, "alpha_max": fd_m, "step_amplitude": ea, "step_alpha_max": 0.1},
           "rel_err_adjoint_vs_fd_amplitude": abs(ga[0] - fd_a) / abs(fd_a),
           "checkpoint_every": every, "adjoint_s": times[1], "adjoint_first_call_s": times[0],
           "forward_mode_s": t2 - t1,
           "note": "alpha_loc stays ~1e-9 in this linear wave, so the alpha_max clip is inactive and "
                   "dL/dalpha_max = 0 exactly (also by differences); alpha_max_active checks a non-zero one"}
    out["alpha_max_active"] = _derivative_alpha_active(args, dev, drop_in)
    return out


def _derivative_alpha_active(args, dev, drop_in, n=16, steps=40, every=8, alpha_max=0.6):
    """Adjoint gradient of the final magnetic energy of a small 3-D blast
    (n^3 lattice, p = 10 inside r < 0.25, alpha in [0.1, alpha_max]) with
    respect to (s, alpha_max), e -> e (1 + 0.01 s), against central
    differences of the drop-in path: the shock drives alpha_loc to the clip,
    so dL/dalpha_max is not zero."""
    import torch

    from src.derivative import AdjointEngine, TangentEngine, TangentState
    from src.engine import params_from_dict

    ic, prm = blast_case(n, "fp64", hot_radius=0.25)
    prm = dict(prm, alpha_max=alpha_max, density="single")
    params = params_from_dict(prm)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    te = TangentEngine(params, TangentState(dict(ic), {"e": [0.01 * ic["e"], None]}), alpha_max_seed=[0.0, 1.0])
    te.warmup()
    ae = AdjointEngine(params, te.ts.n)
    values = {f: te.ts[f][:, 0].contiguous() for f in ae.fields}
    values["m"] = te.ts["m"][:, 0].contiguous()
    values["itype"] = te.ts["itype"]
    tan0 = torch.stack([te.ts[f][:, 1:].clone() for f in ae.fields])
    la, used, cps = ae.forward(values, steps, [te.initial_dt()] + [-1.0] * (steps - 1), every)
    lam, dam = ae.backward(values, steps, used, every, cps)
    ga = torch.einsum("fn,fnd->d", lam, tan0).cpu().numpy()
    ga[1] += dam
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    te.run(steps, used)
    clipped = int((te.ts.value("alphaloc") == alpha_max).sum())
    ae.close()
    te.close()

    def loss(scale_e, am):
        return drop_in(dict(ic, e=ic["e"] * (1.0 + 0.01 * scale_e)), dict(prm, alpha_max=am), used)

    h = 1e-6
    fd_e = (loss(h, alpha_max) - loss(-h, alpha_max)) / (2 * h)
    fd_m = (loss(0.0, alpha_max + h) - loss(0.0, alpha_max - h)) / (2 * h)
    return {"workload": f"3-D blast {n}^3 = {n ** 3} particles, p 10 inside r < 0.25 (0.1 outside), cubic hfact "
                        f"1.2, alpha in [0.1, {alpha_max}], single density pass; final magnetic energy after "
                        f"{steps} steps (frozen step sizes), parameters (s: e -> e (1 + 0.01 s), alpha_max)",
            "loss": la, "grad_adjoint": {"s": float(ga[0]), "alpha_max": float(ga[1])},
            "central_differences": {"s": fd_e, "alpha_max": fd_m, "step": h},
            "rel_err_adjoint_vs_fd": {"s": abs(ga[0] - fd_e) / abs(fd_e), "alpha_max": abs(ga[1] - fd_m) / abs(fd_m)},
            "alphaloc_at_clip_final": clipped, "checkpoint_every": every, "adjoint_s": t1 - t0}


def _app_case(name, nx=None, precision=None):
    """A case of the application layer from its TOML config (initial state and
    kernel parameters)."""
    from dataclasses import replace

    from src.config import load_config
    from src.run import CASES

    cfg = load_config(os.path.join(PKG, "configs", f"{name}.toml"), {k: v.config_type for k, v in CASES.items()})
    if nx is not None:
        cfg = replace(cfg, case=replace(cfg.case, nx=nx))
    app = CASES[cfg.case.name](cfg)
    ic = app.create_mhd_particles()
    prm = app.scheme.kernel_params(app.create_domain(), app.tf)
    if precision:
        prm = dict(prm, precision=precision)
    return ic, prm, cfg


def _morton(cx, cy, cz, bits):
    """Interleaved bits of three cell coordinates (x lowest)."""
    key = np.zeros(cx.shape, dtype=np.int64)
    for b in range(bits):
        key |= ((cx >> b) & 1) << (3 * b)
        key |= ((cy >> b) & 1) << (3 * b + 1)
        key |= ((cz >> b) & 1) << (3 * b + 2)
    return key


def cell_order_locality(n: int, seed: int = 0):
    """How far apart in memory the neighbours of a warp's 32 consecutive
    particles lie under the linear cell order the sort uses (x fastest, then
    y, then z) and under a Morton (Z-curve) order of the same cells: per warp,
    the distinct neighbour records its list entries name (each a record load
    that L1 can serve to the other lanes) and the distinct 128-byte lines of
    one 16-byte record plane they touch.  On the blast lattice (n^3, 0.1 %
    jitter, cubic kernel, h = 1.2 dx, the grid's cells of the list cut-off /
    2), neighbours by the reach R h (1 + 2 %) of the list build.  CPU only."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    dx = 1.0 / n
    ax = (np.arange(n) + 0.5) * dx
    pos = np.stack(np.meshgrid(ax, ax, ax, indexing="ij"), -1).reshape(-1, 3)
    pos = (pos + 0.001 * dx * rng.uniform(-1, 1, pos.shape)) % 1.0
    reach = 2.0 * 1.2 * dx * 1.02
    nc = int(np.floor(1.0 / (reach / 2)))
    c = np.minimum((pos * nc).astype(np.int64), nc - 1)
    keys = {"linear": (c[:, 2] * nc + c[:, 1]) * nc + c[:, 0],
            "morton": _morton(c[:, 0], c[:, 1], c[:, 2], int(np.ceil(np.log2(nc))))}
    pairs = cKDTree(pos, boxsize=1.0).query_pairs(reach, output_type="ndarray")
    i = np.concatenate([pairs[:, 0], pairs[:, 1], np.arange(len(pos))])
    j = np.concatenate([pairs[:, 1], pairs[:, 0], np.arange(len(pos))])
    out = {"workload": f"blast lattice {n}^3 = {len(pos)} particles, {nc}^3 cells, "
                       f"{len(i) / len(pos):.1f} neighbours per particle (self included)"}
    for name, key in keys.items():
        order = np.argsort(key, kind="stable")
        rank = np.empty_like(order)
        rank[order] = np.arange(len(order))
        wi, wj = rank[i] // 32, rank[j]  # warp of i, new index of j
        recs = np.unique(wi * len(pos) + wj)
        lines = np.unique(wi * len(pos) + wj // 8)
        warps = (len(pos) + 31) // 32
        out[name] = {"records_per_warp": len(recs) / warps, "lines_per_warp": len(lines) / warps,
                     "list_entries_per_warp": len(i) / warps,
                     "mean_abs_index_distance": float(np.mean(np.abs(rank[i] - rank[j])))}
    return out


def run_workload(args):
    """The other measured configurations, one JSON line each:
    ot128  -- 2-D Orszag-Tang 128^2, quintic, 50 steps: FP64 on the GPU and the
              CPU oracle (FP64, OpenMP) on the same case;
    briowu -- 2-D Brio-Wu 4096 x 128 slab to t = 0.1: the FP32 form against the
              FP64 path, relative L2 error per field."""
    import torch

    from src.batch import BatchEngine
    from src.engine import params_from_dict

    def run_gpu(ic, prm, steps=None, until=None):
        """`steps` captured fused steps (timed on a replay of the captured
        run), or steps until t = `until` as the reference's solver loop takes
        them: captured chunks of 100 while more than 150 steps of the current
        dt remain, then single steps up to the one clipped to `until`."""
        eng = BatchEngine(params_from_dict(prm), [ic])
        eng.warmup()
        eng.begin(eng.initial_dt())
        done = 0
        if steps is not None:
            snap = eng.snapshot()
            eng.advance(steps, finish=True, snapshot=snap)  # capture + first run
            eng.restore(snap)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            eng.advance(steps, finish=True, snapshot=snap)
            done = steps
        else:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            while True:
                t, dt = (float(a[0]) for a in eng.clocks())
                if t + dt >= until * (1.0 - 1e-14) or dt <= 0.0:
                    eng.advance(1, finish=True, capture=False)
                    done += 1
                    break
                if (until - t) > 150.0 * dt:
                    eng.advance(100, finish=False)
                    done += 100
                else:
                    eng.advance(1, finish=False, capture=False)
                    done += 1
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        t, dt = (float(a[0]) for a in eng.clocks())
        out = eng.pa.pull("x", "rho", "u", "v", "w", "Bx", "By", "Bz", "e", "gid", order="gid")
        eng.close()
        return out, el, done, t + dt

    if args.workload == "ot128":
        import oracle

        ic, prm, _ = _app_case("orstang2d", precision="fp64")
        n = len(ic["x"])
        steps = 50
        gpu, el, _, _ = run_gpu(ic, prm, steps=steps)
        oracle.build()
        s = oracle.State(dict(ic, gid=np.arange(n, dtype=float)))
        o = oracle.Oracle(prm, exact_order=False, nthreads=cpu_cores())
        o.warmup(s)
        t0 = time.perf_counter()
        o.run(s, steps, tf=prm["tf"])
        cel = time.perf_counter() - t0
        rel = {k: float(np.linalg.norm(gpu[k] - s[k]) / max(np.linalg.norm(s[k]), 1e-300))
               for k in ("rho", "u", "v", "Bx", "By")}
        print(json.dumps({"workload": f"2-D Orszag-Tang 128^2 = {n} particles, quintic hfact 1.2, {steps} steps, FP64",
                          "gpu_fp64": {"value": n * steps / el, "unit": UNIT},
                          "cpu_oracle_fp64": {"value": n * steps / cel, "unit": UNIT, "cores": cpu_cores()},
                          "gpu_vs_cpu_rel_l2": rel}), flush=True)
    else:
        # The FP32 form against the FP64 path, and as a control the FP64 path
        # against itself with the free particles' x moved by 1e-10 of the left
        # spacing: a shock tube's post-shock particle noise amplifies any
        # perturbation, so the control's error is the floor that rounding of
        # either kind reaches.  Errors per particle and of the x profile
        # (means over 500 bins across [-0.5, 0.5], the quantity a shock-tube
        # plot shows).
        ic, prm, cfg = _app_case("mhdshock2d")
        n = len(ic["x"])
        dx = 0.5 / cfg.case.nx
        free = ic["itype"] == 1
        pert = dict(ic, x=ic["x"] + np.where(free, 1e-10 * dx * np.random.default_rng(0).uniform(-1, 1, n), 0.0))
        fields = ("rho", "u", "v", "e", "By", "Bx")
        edges = np.linspace(-0.5, 0.5, 501)

        def profile(o, k):
            idx = np.clip(np.digitize(o["x"], edges) - 1, 0, 499)
            inside = (o["x"] >= -0.5) & (o["x"] < 0.5)
            s = np.bincount(idx[inside], o[k][inside], 500)
            c = np.bincount(idx[inside], None, 500)
            return s / np.maximum(c, 1)

        def errors(a, b):
            part = {k: float(np.linalg.norm(a[k] - b[k]) / max(np.linalg.norm(b[k]), 1e-300)) for k in fields}
            prof = {}
            for k in fields:
                pa_, pb_ = profile(a, k), profile(b, k)
                prof[k] = float(np.linalg.norm(pa_ - pb_) / max(np.linalg.norm(pb_), 1e-300))
            return {"particles": part, "x_profile": prof}

        report = {}
        for until in (0.02, prm["tf"]):
            res = {}
            for name, prec, init in (("fp64", "fp64", ic), ("fp32", "fp32", ic), ("fp64_perturbed", "fp64", pert)):
                res[name] = run_gpu(init, dict(prm, precision=prec, tf=until), until=until)
            report[f"t={until}"] = {
                "steps": {k: r[2] for k, r in res.items()}, "t_end": {k: r[3] for k, r in res.items()},
                "rate": {k: n * r[2] / r[1] for k, r in res.items()},
                "fp32_vs_fp64": errors(res["fp32"][0], res["fp64"][0]),
                "fp64_perturbed_vs_fp64": errors(res["fp64_perturbed"][0], res["fp64"][0])}
        print(json.dumps({"workload": f"2-D Brio-Wu {n} particles (4096 x 128 left lattice, right at density 1/8), "
                                      f"gamma 2, quintic hfact 1.0", "unit": UNIT, "runs": report}), flush=True)


def run_b200(args, rank, world):
    import ctypes

    import torch

    from src import _abi

    dist = world > 1
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if dist:
        import datetime

        import torch.distributed as tdist

        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    def barrier():
        if dist:
            import torch.distributed as tdist

            tdist.barrier()

    n = args.n ** 3
    head = _timed(args, args.precision, dev, barrier, dist, world)
    other = "fp64" if args.precision == "fp32" else None
    base = _timed(args, other, dev, barrier, dist, world) if (other and not args.no_fp64) else None
    acc = _accuracy(args, dev, args.accuracy_steps) if (rank == 0 and not dist and args.accuracy_steps > 0) else None

    lib = _abi.load()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    peak = ctypes.c_double()
    lib.mhd_probe_fma_peak(1 if args.precision == "fp32" else 0, ctypes.byref(peak), st)
    kern = head["kernels"]
    force_ms = kern["force"]["ms_total"] / max(kern["force"]["launches"], 1)
    bytes_per_launch = FORCE_BYTES_PER_PARTICLE[args.precision] * n
    hbm_peak, peak_src = measured_peaks()
    achieved_gbs = bytes_per_launch / (force_ms * 1e-3) / 1e9
    # pairs counts the self pair of every particle, which does no arithmetic
    pairs_ns = head["pairs"] - n * args.steps
    flops = (FORCE_FLOPS_PER_PAIR[args.precision] * pairs_ns
             + FORCE_FLOPS_PER_CANDIDATE * (head["candidates"] - head["pairs"])) / args.steps
    achieved_tf = flops / (force_ms * 1e-3) / 1e12

    e2e = run_e2e(args, dev, barrier, dist, world)
    batched = _batched(args, dev, rank, world) if args.batch_instances > 0 else None
    derivative = _derivative(args, dev) if (rank == 0 and not dist and args.derivative_steps > 0) else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the reference arm's measurement on a bounded sample of its steps:
        # the same workload and the same untimed lead-in, fewer timed steps
        n_side = args.ref_n or args.n
        k = min(args.cpu_steps, args.steps)
        rate, el, ns, passes = oracle_rate(n_side, k, args.warmup)
        cpu = {"value": rate, "unit": UNIT, "cores": cpu_cores(), "kind": "port",
               "sample": oracle_sample(n_side, args.warmup, k, el, passes)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32 pair arithmetic, f64 h-iteration/epilogue/dt",
            "data": "synthetic",
            "config": {"workload": blast_workload(args.n), "form": args.precision,
                       "parallelism": "replicas" if world > 1 else "single", "l2_flush": "inputs (~0.6 GB) > L2",
                       "density_passes_per_rhs": head["passes"], "timed_run": "one captured graph of K fused steps",
                       "replays": head["replays"], "ms_per_step_uncaptured": head["ms_per_step_uncaptured"],
                       "neighbours_mean": head["pairs"] / (n * args.steps),
                       "list_entries_mean": head["candidates"] / (n * args.steps),
                       "lists_rebuilt_fraction": head["lists_rebuilt"]},
            "fp64_path": None if base is None else {"value": base["value"], "ms_per_step": base["ms_per_step"],
                                                    "kernels_ms_per_step": {k: v["ms_total"] / args.steps for k, v
                                                                            in base["kernels"].items()}},
            "speedup_vs_fp64": None if base is None else head["value"] / base["value"],
            "accuracy_vs_fp64": acc,
            "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved_gbs / hbm_peak, "traffic": profiled_traffic(n, args.precision),
                         "kernel": "k_force_pass", "peak_source": peak_src, "bytes_per_launch": bytes_per_launch,
                         "launch_ms": force_ms},
            "roofline_compute": {"bound": "fp32_simt" if args.precision == "fp32" else "fp64_simt",
                                 "achieved": achieved_tf, "peak": peak.value / 1e12, "unit": "TFLOP/s",
                                 "frac": achieved_tf * 1e12 / peak.value,
                                 "peak_source": "measured FMA probe on this GPU", "flops_per_launch": flops},
            "kernels_ms_per_step": {k: v["ms_total"] / args.steps for k, v in kern.items()},
            "gpu_launches": head["launches"],
            "clocks": head["clocks"],
            "e2e": e2e,
            "batched_form": batched,
            "derivative_form": derivative,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if dist:
        import torch.distributed as tdist

        tdist.barrier()
        tdist.destroy_process_group()


def run_e2e(args, dev, barrier=lambda: None, dist=False, world=1):
    """The metric end to end through the reference-facing application:
    ``MHDApplication`` built from configs/mhdblast3d.toml (the same 128^3
    blast), its warm-up, then ``MHDSolver.solve`` for K steps with the
    fused loop (``execution.fused``: captured chunks, device dt).  Timed:
    the host -> device copy of the run's inputs (the carried state and the
    last rates; every other property is written before it is read) from
    pinned host memory, the
    K steps, and the device -> host copy of OUTPUT_PROPERTIES at the dump
    every 20 steps (a post-step callback; no files are written).  One
    untimed solve first captures the chunk's graph, which the timed solve
    reuses."""
    from dataclasses import replace

    import torch

    from src.config import load_config
    from src.particles import OUTPUT_PROPERTIES
    from src.run import CASES

    cfg = load_config(os.path.join(PKG, "configs", "mhdblast3d.toml"), {k: v.config_type for k, v in CASES.items()})
    pfreq = 20
    cfg = replace(cfg, case=replace(cfg.case, nx=args.n),
                  solver=replace(cfg.solver, max_steps=args.steps, pfreq=pfreq),
                  execution=replace(cfg.execution, precision=args.precision, fused=True))
    app = CASES[cfg.case.name](cfg)
    app.diagnostics = False  # the diagnostic outputs no equation reads, as in the device-timed value
    app.setup(device=dev)
    app._warm_initial_derivatives(app.solver)  # start-up, excluded as in the metric
    app._compute_initial_dt(app.solver)
    pa = app.particles[0]
    n = pa.n
    solver = app.solver
    solver.output_directory = None
    t0, dt0 = solver.t, solver.dt
    # the run's inputs, what it reads before writing: the last right-hand
    # side's dt_adapt (the first step size is their minimum) and rates, and
    # what the predictor opening a chunk (initialize + stage1: positions, h,
    # the evolved fields, alpha1 and c_s of the alpha switch, the particle
    # type) and the sort of the right-hand side after it (mass and gid
    # besides) read.  Every other property -- rho, p and B (the prologue's),
    # the predicted fields, h0, omega, converged, rho_sum -- is written
    # before it is read.  The timed run starts with the untimed run's end
    # state in every property it does not push, so its outputs equalling
    # the untimed run's, bit for bit (checked below), show none of them is
    # read.
    inputs = ["x", "y", "z", "h", "m", "gid", "itype", "u", "v", "w", "e", "Bevolx", "Bevoly", "Bevolz", "psi",
              "alpha1", "cs", "au", "av", "aw", "ae", "ah", "aBevolx", "aBevoly", "aBevolz", "apsi", "alphaloc",
              "dt_adapt"]
    host = {k: torch.empty(n, dtype=pa.properties[k].dtype, pin_memory=True) for k in inputs}
    for k in inputs:
        host[k].copy_(pa.properties[k])
    out = {k: torch.empty(n, dtype=pa.properties[k].dtype, pin_memory=True) for k in OUTPUT_PROPERTIES}
    d2h = [0]

    def pull(sv):
        if sv.count % pfreq == 0 or sv.count >= sv.max_steps:
            for k in OUTPUT_PROPERTIES:
                out[k].copy_(pa.properties[k], non_blocking=True)
                d2h[0] += out[k].numel() * out[k].element_size()
            torch.cuda.synchronize()

    solver.post_step_callbacks.append(pull)

    def run_once():
        for k, t in host.items():
            pa.properties[k].copy_(t, non_blocking=True)
        solver.t, solver.dt, solver.count = t0, dt0, 0
        solver.initial_acceleration_is_current = True
        solver.solve()
        torch.cuda.synchronize()

    run_once()  # captures the chunk's graph
    first = {k: v.clone() for k, v in out.items()}
    d2h[0] = 0
    h2d = sum(t.numel() * t.element_size() for t in host.values())
    barrier()
    torch.cuda.synchronize()
    t_start = time.perf_counter()
    run_once()
    el = time.perf_counter() - t_start
    steps = solver.count
    for k in out:
        if not torch.equal(out[k], first[k]):
            raise RuntimeError(f"end-to-end run: {k} differs from the untimed run's (an input not pushed)")
    if dist:
        # every rank's replica, timed as the slowest rank
        import torch.distributed as tdist

        t = torch.tensor([el], device=dev, dtype=torch.float64)
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        el = float(t.item())
    barrier()
    app.engine.close()
    return {"value": world * n * steps / el, "unit": UNIT, "h2d_bytes_per_step": world * h2d / steps,
            "d2h_bytes_per_step": world * (d2h[0] + 8 * steps) / steps,
            "path": "MHDApplication (configs/mhdblast3d.toml) -> MHDSolver.solve, fused loop: pinned-host inputs "
                    "(the 28 properties the run reads before writing: state, type, last rates and dt_adapt) pushed, "
                    "K steps in captured chunks with device dt, OUTPUT_PROPERTIES pulled at the dump every 20 steps "
                    "(equal, bit for bit, to an untimed run's); diagnostic outputs off"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=("b200", "reference"))
    ap.add_argument("--n", type=int, default=128, help="lattice side of the blast (n^3 particles)")
    ap.add_argument("--ref-n", type=int, default=0, help="lattice side of the CPU runs (0: the workload's)")
    ap.add_argument("--cpu-steps", type=int, default=5, help="timed oracle steps of the cpu_baseline sample")
    ap.add_argument("--precision", default="fp32", choices=("fp64", "fp32"),
                    help="form timed as the headline value (the FP64 path is timed beside it)")
    ap.add_argument("--accuracy-steps", type=int, default=100)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="uncaptured steps run between cudaProfilerStart/Stop after the timing (0: none)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-instances", type=int, default=64, help="batched form instances (0 skips it)")
    ap.add_argument("--batch-steps", type=int, default=100)
    ap.add_argument("--batch-loop-steps", type=int, default=10, help="steps per instance of the FP64 loop")
    ap.add_argument("--derivative-steps", type=int, default=200, help="derivative form steps (0 skips it)")
    ap.add_argument("--workload", default="blast", choices=("blast", "ot128", "briowu", "cell_order"),
                    help="blast: the benchmark line; ot128 / briowu: the other measured configurations; "
                         "cell_order: memory locality of neighbour gathers, linear vs Morton cell order (CPU)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.workload == "cell_order":
        if rank == 0:
            print(json.dumps(cell_order_locality(args.n if args.n != 128 else 64)))
    elif args.workload != "blast":
        if rank == 0:
            run_workload(args)
    elif args.impl == "reference":
        run_reference(args, rank)
    else:
        run_b200(args, rank, world)


if __name__ == "__main__":
    main()
