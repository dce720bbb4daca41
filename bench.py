"""Benchmark of the Fisher-Kolmogorov RD hot path on B200.

One step = one pass of the fused RD kernel (ReactionDiffusionOperator<3> +
UpdateTumor<3>) over the 256^3-equivalent frozen uniform topology of the
adaptive FP32 configuration: 32768 blocks of 8^3 cells, FP32 storage (the
reference's default Real), Dw = 0.2 cm^2/day, rho = 0.05/day, seeded synthetic
anatomy.  ``value`` is whole-job cell-updates/s with the fields resident in
HBM; ``e2e`` is the same metric through the public API with host buffers
(H2D and D2H of phi, the state, inside every timed step; the anatomy p_w, p_g
is fixed for a whole calibration and stays resident like a model's weights;
``e2e.all_fields`` uploads p_w and p_g every step as well).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gbfk|reference]

Multi-GPU: one process per GPU (torchrun); a single solve does not shard
(256^3 fits one GPU), so N GPUs run N independent replicas ("weak").
``--impl reference`` times the reference's own CPU operators (oracle/_ref,
threaded TBB stand-in) on the host cores instead.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import re
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from gliomasolver_b200.anatomy import make_case  # noqa: E402
from gliomasolver_b200.schedule import make_schedule  # noqa: E402

METRIC = "RD cell-updates/s & % HBM roofline"
UNIT = "cell-updates/s"
# the step kernel each GBFK_STEP_* choice launches
KERNEL_NAMES = {"pipelined": "rd_step_tma_kernel<{real}> (persistent, TMA-fed)",
                "block": "rd_step_kernel<{real},0> (one CTA per block)"}
N_GRID = 256
DW, RHO, TEND, L_CM = 0.2, 0.05, 300.0, 25.6
SEED = 0
CPU_SAMPLE_N = 64
PROFILE_SUMMARY = ROOT / "profiles" / "rd_step_f32_n256.md"


def workload_config(n, precision):
    return {
        "workload": f"fused RD step (ReactionDiffusionOperator<3> + UpdateTumor<3>), {n}^3 uniform frozen "
                    f"topology, {(n // 8) ** 3} blocks of 8^3, {'FP32' if precision == 'f32' else 'FP64'} storage",
        "n": n, "blocks": (n // 8) ** 3, "precision": precision,
        "Dw_cm2_day": DW, "rho_day": RHO, "L_cm": L_CM, "anatomy_seed": SEED,
        "l2": "inputs larger than L2: phi in/out + p_w + p_g = %d MB per step" % (16 * n ** 3 // 2 ** 20),
    }


def heavy_blocks(pw, pg):
    """Blocks that read p_w and p_g in the pipelined step: a cell with tissue
    (p_w + p_g > 0) in the block or in its face halo (periodic)."""
    t = (pw + pg) > 0
    halo = t.copy()
    for ax in range(3):
        halo |= np.roll(t, 1, axis=ax) | np.roll(t, -1, axis=ax)
    n = t.shape[0]
    b = n // 8
    return int(halo.reshape(b, 8, b, 8, b, 8).any(axis=(1, 3, 5)).sum())


def fp64_lines(stream, local, steps):
    """FP64 storage (the reference built with Real = double): config 1 in full
    (64^3, 739 steps to T = 150 d) against the reference's own output (the
    golden fixture: SHA-256 and relative L2 of a subsample), and the 256^3
    workload of the headline line in FP64.  CUDA events on the stream."""
    import hashlib

    import torch

    from gliomasolver_b200 import BlockPool

    peak, _ = measured_peak()
    out = {}
    with np.load(ROOT / "tests" / "golden" / "config1_n64_f64.npz") as z:
        fx = {k: z[k] for k in z.files}
    n = int(fx["n"])
    pw, pg, c0, _ = make_case(n, int(fx["seed"]))
    with BlockPool((n // 8) ** 3, "f64", device=local, stream=stream.cuda_stream) as pool:
        pool.set_uniform(n // 8)
        for name, a in (("p_w", pw), ("p_g", pg), ("phi", c0)):
            pool.upload_dense(name, a)
        pool.rd_step(float(fx["Dw"]), float(fx["Dg"]), float(fx["rho"]), float(fx["dt"]), 1)  # face coefficients
        pool.upload_dense("phi", c0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        pool.rd_step(float(fx["Dw"]), float(fx["Dg"]), float(fx["rho"]), float(fx["dt"]), int(fx["nsteps"]))
        e1.record(stream)
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) / 1e3
        phi = pool.download_dense("phi")
    sub = phi[::4, ::4, ::4]
    k = int(fx["nsteps"])
    out["config1_n64"] = {
        "workload": f"config 1: {n}^3 uniform, FP64, {k} steps to T = 150 d (fields L2-resident: 8 MB)",
        "steps": k, "seconds": sec, "cell_updates_per_s": n ** 3 * k / sec,
        "algorithmic_gbs": 32 * n ** 3 * k / sec / 1e9, "hbm_frac_algorithmic": 32 * n ** 3 * k / sec / 1e9 / peak,
        "rel_l2_vs_reference": float(np.linalg.norm(sub - fx["out_sub"]) / np.linalg.norm(fx["out_sub"])),
        "sha256_equal_to_reference": hashlib.sha256(np.ascontiguousarray(phi).tobytes()).hexdigest()
        == str(fx["output_sha"])}
    n = N_GRID
    pw, pg, c0, _ = make_case(n, SEED)
    s = make_schedule(DW, RHO, TEND, L_CM, n // 8, "f64")
    with BlockPool((n // 8) ** 3, "f64", device=local, stream=stream.cuda_stream) as pool:
        pool.set_uniform(n // 8)
        for name, a in (("p_w", pw), ("p_g", pg), ("phi", c0)):
            pool.upload_dense(name, a)
        pool.rd_step(s.Dw, s.Dg, s.rho, s.dt, 5)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        pool.rd_step(s.Dw, s.Dg, s.rho, s.dt, steps)
        e1.record(stream)
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) / 1e3
        heavy = heavy_blocks(pw, pg)
    per = sec / steps
    out["uniform_n256"] = {
        "workload": f"the headline workload in FP64: {n}^3 uniform frozen topology, {steps} steps",
        "ms_per_step": 1e3 * per, "cell_updates_per_s": n ** 3 / per,
        "algorithmic_gbs": 32 * n ** 3 / per / 1e9, "algorithmic_frac": 32 * n ** 3 / per / 1e9 / peak,
        "minimum_bytes_gbs": 8 * (2 * n ** 3 + 2 * 512 * heavy) / per / 1e9,
        "minimum_bytes_frac": 8 * (2 * n ** 3 + 2 * 512 * heavy) / per / 1e9 / peak}
    return out


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def profiled_traffic(kind):
    """dram bytes per launch of the step kernel `kind` ("pipelined" / "block")
    at the default workload, from the committed ncu summary."""
    if not PROFILE_SUMMARY.exists():
        return None
    m = re.search(r"dram_bytes_per_launch\[%s\]:\s*([0-9.eE+]+)" % kind, PROFILE_SUMMARY.read_text())
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_reference_run(steps, warmup, n_sample=CPU_SAMPLE_N, precision="f32", target_s=None, threads=None):
    """The reference's own operators on the host cores (oracle/_ref; all of
    them, or ``threads``), else the oracle restatement on one core.  Returns
    (record, kind, cores, n, steps)."""
    from oracle import oracle as O

    pw, pg, c0, _ = make_case(n_sample, SEED)
    s = make_schedule(DW, RHO, TEND, L_CM, n_sample // 8, precision)
    cores = threads or os.cpu_count() or 1
    if O.ref_available(precision):
        if target_s is not None:
            probe = O.ref_time(pw, pg, c0, s.Dw, s.Dg, s.rho, s.dt, 3, precision, threads=cores, warmup=1)
            per = probe["seconds"] / 3
            steps = int(max(3, min(2000, target_s / max(per, 1e-6))))
        rec = O.ref_time(pw, pg, c0, s.Dw, s.Dg, s.rho, s.dt, steps, precision, threads=cores, warmup=warmup)
        return rec, "reference", rec["threads"], n_sample, steps
    R = np.float32 if precision == "f32" else np.float64
    a, b, c = (x.astype(R) for x in (pw, pg, c0))
    if target_s is not None:
        t = time.perf_counter()
        O.rd_steps_dense(a, b, c, s.Dw, s.Dg, s.rho, s.h, s.dt, 1)
        steps = int(max(1, min(500, target_s / max(time.perf_counter() - t, 1e-6))))
    O.rd_steps_dense(a, b, c, s.Dw, s.Dg, s.rho, s.h, s.dt, warmup)
    t = time.perf_counter()
    O.rd_steps_dense(a, b, c, s.Dw, s.Dg, s.rho, s.h, s.dt, steps)
    dt = time.perf_counter() - t
    cells = n_sample ** 3
    return {"cells": cells, "steps": steps, "seconds": dt, "threads": 1,
            "cell_updates_per_s": cells * steps / dt}, "port", 1, n_sample, steps


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    # the GPU arm's own workload when its K + W steps fit in about two minutes of
    # the host cores, else a smaller grid of the same anatomy as each step's sample
    n_sample = 32
    for n_try in (N_GRID, CPU_SAMPLE_N):
        rec, kind, cores, n_s, steps = cpu_reference_run(3, 1, n_try, args.precision)
        if rec["seconds"] / rec["steps"] * (args.steps + args.warmup) <= 120:
            n_sample = n_try
            break
    rec, kind, cores, n_s, steps = cpu_reference_run(args.steps, args.warmup, n_sample, args.precision)
    value = rec["cell_updates_per_s"]
    grid = (f"{N_GRID}^3 uniform grid (the GPU arm's workload)" if n_s == N_GRID else
            f"{n_s}^3 uniform grid of the same synthetic anatomy (same brain fraction as {N_GRID}^3)")
    sample = f"{grid}, {steps} timed steps after {args.warmup} warm-up steps, stepping loop only"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * rec["seconds"] / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": args.precision,
        "data": "synthetic", "config": workload_config(N_GRID, args.precision),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def batched_stage(args, stream, local, nsamples=512, bpd=16, seed=1):
    """Config 3: a TMCMC stage of 512 forward solves on 128^3 (FP32, one
    seeded anatomy, Dw log-U[0.02,0.3], rho log-U[0.002,0.2], T U[30,300] d,
    x0 a white-matter voxel), batched vs the same 512 solves one after the
    other through gbfk_rd_step on one BlockPool.  With several ranks each
    runs its share of the samples (shard.stage_shards, balanced by steps) and
    the times are the max over ranks.  Returns the JSON record."""
    import torch

    from gliomasolver_b200 import BlockPool
    from gliomasolver_b200.anatomy import make_anatomy, tumor_ic
    from gliomasolver_b200.shard import max_over_ranks, stage_shards
    from gliomasolver_b200.tmcmc import Batch, sample_stage, to_gbfk_samples

    n = 8 * bpd
    p_w, p_g, _ = make_anatomy(n, SEED)
    pw32, pg32 = p_w.astype(np.float32), p_g.astype(np.float32)
    full = sample_stage(nsamples, p_w, seed=seed)
    _, full_scheds = to_gbfk_samples(full, bpd, "f32", L_CM)
    all_steps = np.array([sc.nsteps for sc in full_scheds])
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    mine = stage_shards(all_steps, world)[rank]
    stage = [full[i] for i in mine]
    samples, scheds = to_gbfk_samples(stage, bpd, "f32", L_CM)
    steps = all_steps
    cells = n ** 3
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    with Batch(bpd, max(len(stage), 1), "f32", device=local, stream=stream.cuda_stream) as b:
        b.set_anatomy(0, pw32, pg32)
        b.set_samples(samples)
        l0 = b.launches
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record(stream)
        b.run(0)
        e1.record(stream)
        torch.cuda.synchronize()
        t_batch = max_over_ranks(e0.elapsed_time(e1) / 1e3)
        batch_launches = b.launches - l0
        spc = b.samples_per_cta
        tile = list(b.tile_shape)
        graphs = b.graph_count

    with BlockPool(bpd ** 3, "f32", device=local, stream=stream.cuda_stream) as pool:
        pool.set_uniform(bpd)
        pool.upload_dense("p_w", pw32)
        pool.upload_dense("p_g", pg32)
        ics = [tumor_ic(n, st.x0, p_w, p_g).astype(np.float32) for st in stage]
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record(stream)
        for ic, sc in zip(ics, scheds):
            pool.upload_dense("phi", ic)
            pool.rd_step(sc.Dw, sc.Dg, sc.rho, sc.dt, sc.nsteps)
        e1.record(stream)
        torch.cuda.synchronize()
        t_seq = max_over_ranks(e0.elapsed_time(e1) / 1e3)

    return {
        "workload": f"{nsamples} TMCMC samples, {n}^3 uniform, FP32, one seeded anatomy; Dw log-U[0.02,0.3], "
                    "rho log-U[0.002,0.2], T U[30,300] d, x0 in white matter",
        "samples": nsamples, "steps_total": int(steps.sum()), "steps_min": int(steps.min()),
        "steps_max": int(steps.max()),
        "batched_s": t_batch, "batched_samples_per_s": nsamples / t_batch,
        "batched_cell_updates_per_s": float(steps.sum()) * cells / t_batch,
        "sequential_s": t_seq, "sequential_samples_per_s": nsamples / t_seq,
        "speedup_vs_sequential": t_seq / t_batch,
        "samples_per_cta": spc, "tile_shape": tile, "cuda_graphs": graphs, "batched_launches": batch_launches,
        "ranks": world,
        "empty_blocks": "the batch steps the empty blocks (no tissue in them or their face halos; +0 from the "
                        "initial condition on) once, then skips them: both state buffers hold their final +0; "
                        "the sequential solves step every block",
        "timing": "CUDA events on the stream: batched = face coefficients + initial conditions + all steps; "
                  "sequential = per sample an H2D of c0, face coefficients and its steps",
    }


def adjoint_sample(stream, local, bpd=16, nsnap=64, check=True):
    """Config 4: forward + discrete adjoint at 128^3, FP32 state, FP64 loss and
    gradient sums, 64 checkpoint buffers, about 10^4 steps (Dw = 0.2, T = 300 d);
    observations from a seeded FP64 ground-truth run (rho = 0.012) thresholded
    at 0.7 / 0.25 with 2% label noise; gradients taken at Dw = 0.18, rho = 0.014.
    rho*T ~ 4 keeps a tumour front: with rho*T >> 1 the tumour saturates the
    brain (every cell exactly 0 or 1), the loss is locally constant and all
    gradients are 0.  Timed against one plain forward solve of the same steps.
    Untimed checks: the same problem with FP64 state against central
    differences of FP64 forward solves (relative step 1e-4 for Dw and rho,
    1e-7 for x0), and the FP32 gradients against the FP64 ones."""
    import torch

    from gliomasolver_b200 import BlockPool
    from gliomasolver_b200.anatomy import make_anatomy, pick_origin, tumor_ic
    from gliomasolver_b200.gradcheck import check_gradients, synthetic_observations

    n = 8 * bpd
    p_w, p_g, _ = make_anatomy(n, SEED)
    s = make_schedule(0.2, 0.012, 300.0, L_CM, bpd, "f32")
    s64 = make_schedule(0.2, 0.012, 300.0, L_CM, bpd, "f64")
    x_gt = pick_origin(p_w, SEED)[0]
    x0 = [float(min(1.0, v + 2.0 / n)) for v in x_gt]
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    with BlockPool(bpd ** 3, "f64", device=local, stream=stream.cuda_stream) as pool64:
        pool64.set_uniform(bpd)
        pool64.upload_dense("p_w", p_w)
        pool64.upload_dense("p_g", p_g)
        masks = synthetic_observations(pool64, tumor_ic(n, x_gt, p_w, p_g), s64.Dw, s64.rho, s64.dt, s64.nsteps,
                                       seed=SEED + 17)
        Dw64 = float(np.float64(0.18) / np.float64(L_CM * L_CM))
        chk = check_gradients(pool64, p_w, p_g, Dw64, 0.014, s.dt, s.nsteps, x0, 2.0 / n,
                              nsnapshots=nsnap) if check else None
    with BlockPool(bpd ** 3, "f32", device=local, stream=stream.cuda_stream) as pool:
        pool.set_uniform(bpd)
        pool.upload_dense("p_w", p_w.astype(np.float32))
        pool.upload_dense("p_g", p_g.astype(np.float32))
        pool.set_observations(*masks)
        Dw = float(np.float32(np.float32(0.18) / np.float32(L_CM * L_CM)))
        Dg = float(np.float32(0.1 * Dw))
        # warm-up (face coefficients, first allocations)
        pool.forward_adjoint(Dw, Dg, 0.014, s.dt, 20, x0=x0, sigma=2.0 / n, nsnapshots=nsnap)
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record(stream)
        res = pool.forward_adjoint(Dw, Dg, 0.014, s.dt, s.nsteps, x0=x0, sigma=2.0 / n, nsnapshots=nsnap)
        e1.record(stream)
        torch.cuda.synchronize()
        t_adj = e0.elapsed_time(e1) / 1e3
        # the same gradient with the checkpoint budget of the whole HBM: every
        # state of the first sweep kept (or as many as 80% of the free memory
        # holds), so that nothing is recomputed
        all_states = None
        free, _ = torch.cuda.mem_get_info(local)
        nall = int(min(s.nsteps, 0.8 * free // (n ** 3 * 4)))
        if nall > nsnap:
            pool.forward_adjoint(Dw, Dg, 0.014, s.dt, 20, x0=x0, sigma=2.0 / n, nsnapshots=nall)  # allocation
            torch.cuda.synchronize()
            e0, e1 = ev(), ev()
            e0.record(stream)
            res_all = pool.forward_adjoint(Dw, Dg, 0.014, s.dt, s.nsteps, x0=x0, sigma=2.0 / n, nsnapshots=nall)
            e1.record(stream)
            torch.cuda.synchronize()
            all_states = {"checkpoints": nall, "checkpoint_gb": nall * n ** 3 * 4 / 1e9,
                          "forward_steps_run": res_all["forward_steps"], "gradient_s": e0.elapsed_time(e1) / 1e3,
                          "same_gradients_as_64": all(res_all[k] == res[k] for k in ("loss", "dDw", "drho")) and
                          list(res_all["dx0"]) == list(res["dx0"])}
        pool.upload_dense("phi", tumor_ic(n, x0, p_w, p_g).astype(np.float32))
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record(stream)
        pool.rd_step(Dw, Dg, 0.014, s.dt, s.nsteps)
        e1.record(stream)
        torch.cuda.synchronize()
        t_fwd = e0.elapsed_time(e1) / 1e3
    out = {
        "workload": f"forward + discrete adjoint, {n}^3 uniform, FP32 state, FP64 loss/gradient sums, "
                    f"{nsnap} checkpoint buffers, {s.nsteps} steps",
        "steps": s.nsteps, "forward_steps_run": res["forward_steps"], "adjoint_steps": res["adjoint_steps"],
        "gradient_s": t_adj, "gradient_samples_per_s": 1.0 / t_adj,
        "plain_forward_s": t_fwd, "plain_forward_samples_per_s": 1.0 / t_fwd,
        "gradient_cost_in_forward_solves": t_adj / t_fwd,
        "forward_steps_note": "the gradient's forward steps run only the blocks with tissue once every empty block "
                              "holds its final +0; the plain forward solve steps every block",
        "all_states": None if all_states is None else dict(
            all_states, gradient_cost_in_forward_solves=all_states["gradient_s"] / t_fwd),
        "loss": res["loss"], "dDw": res["dDw"], "drho": res["drho"], "dx0": list(res["dx0"]),
    }
    if chk is not None:
        a64 = chk["adjoint"]
        rel32 = {k: abs(res[k] - a64[k]) / max(abs(a64[k]), 1e-300) for k in ("dDw", "drho")}
        rel32["loss"] = abs(res["loss"] - chk["loss"]) / abs(chk["loss"])
        rel32["dx0"] = float(np.linalg.norm(np.array(res["dx0"]) - np.array(a64["dx0"])) / np.linalg.norm(a64["dx0"]))
        out["fp64_check"] = {
            "what": "FP64 state, same problem: adjoint vs central differences of FP64 forward solves (relative "
                    "step 1e-4 for Dw, rho; 1e-7 for x0); crossings = voxels that cross a likelihood threshold "
                    "between the two runs of a quotient",
            "adjoint": a64, "fd": chk["fd"], "rel_err": chk["rel_err"], "crossings": chk["crossings"],
            "fd_resolution": chk["fd_resolution"], "chain_rule_rel_err": chk["chain_rule_rel_err"],
            "term_cancellation": chk["term_cancellation"],
            "forward_steps_run": chk["forward_steps"]}
        out["fp32_vs_fp64_rel"] = rel32
    return out


def adjoint_batch(stream, local, nsamples=16, bpd=32, seed=5, hbm_cap=160e9, max_steps=None):
    """Config 5: forward + discrete adjoint for 16 samples at 256^3, FP32 state,
    each sample with its own seeded anatomy (brain scale U[0.8, 1.2]) and
    parameters sampled as in config 3 (Dw log-U[0.02,0.3], rho
    log-U[0.002,0.2], T U[30,300] d, x0 in white matter).  Observations: the
    sample's own forward run thresholded at 0.7 / 0.25 with 2% label noise;
    gradients at Dw * 1.1, rho * 0.9.  The samples run one after the other
    (one gbfk_forward_adjoint call each, on one context whose buffers are
    allocated before the timed calls).  The checkpoint budget is admitted by
    a 160 GB HBM cap (less what the device has free beside the other
    buffers): min(steps, cap / 67 MB) checkpoints per sample.  Sample 0 is
    repeated in FP64 for the FP32-vs-FP64 gradient error."""
    import torch

    from gliomasolver_b200 import BlockPool
    from gliomasolver_b200.anatomy import tumor_ic
    from gliomasolver_b200.gradcheck import config5_sample

    n = 8 * bpd
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    t_total, steps_total, fwd_total, recs = 0.0, 0, 0, []
    peak, _ = measured_peak()

    def open_pool(prec):
        R = np.float32 if prec == "f32" else np.float64
        pool = BlockPool(bpd ** 3, prec, device=local, stream=stream.cuda_stream)
        pool.set_uniform(bpd)
        z = np.zeros((n, n, n), dtype=R)
        pool.upload_dense("p_w", z)
        pool.upload_dense("p_g", z)
        pool.upload_dense("phi", z)
        pool.set_observations(z.astype(float), z.astype(float))
        torch.cuda.synchronize()
        free, _total = torch.cuda.mem_get_info(local)
        fbytes = n ** 3 * np.dtype(R).itemsize
        cap = min(hbm_cap, free - 8 * fbytes - 4e9)
        cap_snap = max(1, int(cap // fbytes))
        # allocate the checkpoints (and the work fields) once, outside the timed
        # calls; halve the budget if the device refuses it
        from gliomasolver_b200 import GbfkError
        from gliomasolver_b200._lib import STATUS_CODES
        while True:
            try:
                pool.forward_adjoint(1e-4, 1e-5, 0.01, 1e-3, 2, nsnapshots=cap_snap)
                break
            except GbfkError as e:
                if e.code != STATUS_CODES["GBFK_E_OOM"] or cap_snap <= 64:
                    raise
                cap_snap //= 2
        torch.cuda.synchronize()
        return pool, cap_snap

    def one(pool, cap_snap, prec, p_w, p_g, st, rng, masks=None, magnitudes=False):
        R = np.float32 if prec == "f32" else np.float64
        s = make_schedule(st.Dw_cm2_day, st.rho_day, st.tend_day, L_CM, bpd, prec)
        if max_steps is not None and s.nsteps > max_steps:
            s = dataclasses.replace(s, nsteps=max_steps)
        pool.upload_dense("p_w", p_w.astype(R))
        pool.upload_dense("p_g", p_g.astype(R))
        if masks is None:
            pool.upload_dense("phi", tumor_ic(n, st.x0, p_w, p_g).astype(R))
            pool.rd_step(s.Dw, s.Dg, s.rho, s.dt, s.nsteps)
            u = pool.download_dense("phi").astype(np.float64)
            masks = [(u > 0.7).astype(float), (u > 0.25).astype(float)]
            for m in masks:
                flip = rng.random(m.shape) < 0.02
                m[flip] = 1 - m[flip]
        pool.set_observations(*masks)
        Dw = float(R(R(st.Dw_cm2_day * 1.1) / R(L_CM * L_CM)))
        Dg = float(R(0.1 * Dw))
        nsnap = min(s.nsteps, cap_snap)
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record(stream)
        res = pool.forward_adjoint(Dw, Dg, st.rho_day * 0.9, s.dt, s.nsteps, x0=st.x0, sigma=2.0 / n,
                                   nsnapshots=max(1, nsnap), term_magnitudes=magnitudes)
        e1.record(stream)
        torch.cuda.synchronize()
        return res, e0.elapsed_time(e1) / 1e3, s.nsteps, masks, nsnap

    first = None
    pool, cap32 = open_pool("f32")
    try:
        for i in range(nsamples):
            p_w, p_g, st, rng = config5_sample(i, n, seed)
            res, t, k, masks, nsnap = one(pool, cap32, "f32", p_w, p_g, st, rng)
            t_total += t
            steps_total += k
            fwd_total += res["forward_steps"]
            recs.append({"steps": k, "checkpoints": nsnap, "forward_steps_run": res["forward_steps"], "seconds": t,
                         "loss": res["loss"], "dDw": res["dDw"], "drho": res["drho"]})
            if first is None:
                first = (p_w, p_g, st, res, masks)
    finally:
        pool.close()
    p_w, p_g, st, r32, masks = first
    pool, cap64 = open_pool("f64")
    try:
        r64 = one(pool, cap64, "f64", p_w, p_g, st, None, masks, magnitudes=True)[0]
    finally:
        pool.close()
    rel = {k: abs(r32[k] - r64[k]) / max(abs(r64[k]), 1e-300) for k in ("loss", "dDw", "drho")}
    # sum of |term| over |sum of terms| in the FP64 run: a relative change e of
    # the terms moves a gradient by up to e times this, relatively
    cancel = {"dDw": r64["dDw_abs"] / max(abs(r64["dDw"]), 1e-300),
              "drho": r64["drho_abs"] / max(abs(r64["drho"]), 1e-300)}
    alg = 9 * 4 * (n ** 3) * steps_total  # (4 forward + 5 adjoint) words per cell and step, FP32
    return {
        "workload": f"{nsamples} samples, forward + discrete adjoint at {n}^3, FP32 state, own anatomy each "
                    f"(scale U[0.8,1.2]), config-3 parameter sampling, checkpoints admitted by a "
                    f"{hbm_cap / 1e9:.0f} GB HBM cap (up to {cap32} of 67 MB), one sample per call"
                    + (f"; horizons capped at {max_steps} steps (T' = min(T, {max_steps} dt))" if max_steps else ""),
        "max_steps_per_sample": max_steps,
        "samples": nsamples, "steps_total": steps_total, "forward_steps_run": fwd_total, "seconds": t_total,
        "gradient_samples_per_s": nsamples / t_total,
        "roofline": {"achieved": alg / t_total / 1e9, "peak": peak, "unit": "GB/s", "frac": alg / t_total / 1e9 / peak,
                     "algorithmic_bytes": "9 words (forward 4 + adjoint 5) x cells x steps; recomputation not counted"},
        "fp32_vs_fp64_rel": rel, "term_cancellation_fp64": cancel,
        "fp32_vs_fp64_rel_over_cancellation": {k: rel[k] / cancel[k] for k in cancel},
        "per_sample": recs,
    }


def adaptive_forward(steps, precision="f32"):
    """Config 2 on the resident drop-in (dropin/_build/glioma_adaptive_*): the
    reference's MRAG grid as the block tree, the leaves on the GPU for the
    whole run; level 2 to 5 (256^3-equivalent), Dw = 0.2 cm^2/day,
    rho = 0.05/day, re-adapting every 20 steps (one refinement loop at 1e-3,
    compression to convergence at 1e-4), ``steps`` steps of the T = 300 d
    schedule (36364 in all).  Host wall clock around synchronous calls."""
    import tempfile

    exe = ROOT / "dropin" / "_build" / f"glioma_adaptive_{precision}"
    if not exe.exists():
        return {"unavailable": "dropin/_build is built only where the reference sources are"}
    n = 256
    pw, pg, c0, _ = make_case(n, SEED)
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            f.write(np.int32(n).tobytes())
            for a in (pw, pg, c0):
                f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
        t0 = time.perf_counter()
        r = subprocess.run([str(exe), fin, "5", "1e-3", "1e-4", str(steps), "20", fout], capture_output=True,
                           text=True, timeout=1800)
        wall = time.perf_counter() - t0
    if r.returncode != 0:
        return {"failed": r.stderr[-500:]}
    rec = json.loads(r.stdout.strip().splitlines()[-1])
    cu = rec["cell_updates"]
    keep = ("step_seconds", "adapt_seconds", "first_upload_seconds", "topology_changes", "uploads", "upload_seconds",
            "detail_sweeps", "details_seconds", "plan_seconds", "splits", "split_seconds", "collapses",
            "collapse_seconds", "near_decisions", "min_margin_refine", "min_margin_compress")
    out = {"workload": f"config 2 adaptive forward, levels 2-5 (256^3-equivalent), {precision.upper()} storage, "
                       f"re-adapt every 20 steps, first {steps} of the 36364 steps of T = 300 d",
           "steps": steps, "blocks_min": min(rec["blocks"]), "blocks_max": max(rec["blocks"]),
           "cell_updates": cu, "stepping_cell_updates_per_s": cu / rec["step_seconds"],
           "run_cell_updates_per_s": cu / (rec["step_seconds"] + rec["adapt_seconds"]), "process_wall_s": wall}
    out.update({k: rec[k] for k in keep})
    out["timing"] = ("host wall clock around synchronous calls; adapt = device details + the reference grid's "
                     "own plan and tree update (plan_seconds) + device split/collapse + ghost-list upload")
    return out


def gpu_arm(args):
    import torch
    import torch.distributed as dist

    from gliomasolver_b200 import BlockPool
    from gliomasolver_b200.build import build_library
    from gliomasolver_b200.shard import max_over_ranks

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus and world > 1:
        print(f"WORLD_SIZE={world} but --gpus {args.gpus}", file=sys.stderr)
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    build_library()

    n, prec = args.n, args.precision
    R = np.float32 if prec == "f32" else np.float64
    pw, pg, c0, _ = make_case(n, SEED)
    pw, pg, c0 = (a.astype(R) for a in (pw, pg, c0))
    s = make_schedule(DW, RHO, TEND, L_CM, n // 8, prec)
    cells = n ** 3
    # an explicit stream: the library treats a NULL handle (torch's legacy
    # default stream) as "create a private stream", which events on the
    # default stream would not see
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    pool = BlockPool((n // 8) ** 3, prec, device=local, stream=stream.cuda_stream)
    assert stream.cuda_stream != 0
    pool.set_uniform(n // 8)
    pool.step_kernel = args.step_kernel
    pool.upload_dense("p_w", pw)
    pool.upload_dense("p_g", pg)
    pool.upload_dense("phi", c0)

    def barrier():
        if world > 1:
            dist.barrier()

    # ---- device-resident throughput -------------------------------------
    for _ in range(args.warmup):
        pool.rd_step(s.Dw, s.Dg, s.rho, s.dt, 1)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    launches0 = pool.launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    pool.rd_step(s.Dw, s.Dg, s.rho, s.dt, args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    launches = pool.launches - launches0
    clk = clocks.stop()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    ms_per_step = ms / args.steps
    value = world * cells * args.steps / (ms / 1e3)

    # ---- roofline of the fused kernel (one launch per step) --------------
    word = 4 if prec == "f32" else 8
    alg_bytes = 4 * word * cells  # read phi, p_w, p_g; write phi
    kernel_s = (ms / 1e3) / max(launches, 1) if launches == args.steps else (ms / 1e3) / args.steps
    achieved = alg_bytes / kernel_s / 1e9
    peak, peak_kind = measured_peak()
    traffic = profiled_traffic(pool.step_kernel) if (n, prec) == (N_GRID, "f32") else None
    # the fewest bytes the exact shortcuts allow: phi in and out for every
    # cell, p_w and p_g only for blocks with tissue in a cell or a face halo
    heavy = heavy_blocks(pw, pg)
    min_bytes = word * (2 * cells + 2 * 512 * heavy)
    roofline = {"kernel": KERNEL_NAMES[pool.step_kernel].format(real="float" if prec == "f32" else "double"),
                "bound": "hbm", "unit": "GB/s", "peak": peak,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "traffic": traffic, "algorithmic_bytes_per_launch": alg_bytes,
                "algorithmic_achieved": achieved, "algorithmic_frac": achieved / peak,
                "minimum_bytes_per_launch": min_bytes, "heavy_blocks": heavy,
                "traffic_over_minimum": (traffic / min_bytes) if traffic else None}
    if traffic:
        # DRAM bytes of a warm launch (ncu) over the CUDA-event launch time: the
        # HBM fraction.  The algorithmic figure (4 words per cell-update) exceeds
        # what DRAM moves because empty blocks read no p_w, p_g or coefficients.
        roofline.update({"achieved": traffic / kernel_s / 1e9, "frac": traffic / kernel_s / 1e9 / peak,
                         "frac_basis": "DRAM bytes per warm launch (ncu) / CUDA-event launch time"})
    else:
        roofline.update({"achieved": achieved, "frac": achieved / peak,
                         "frac_basis": "algorithmic bytes (4 words per cell-update) / CUDA-event launch time"})

    # ---- end to end through the public API with host buffers -------------
    e2e_steps = max(1, min(args.steps, 50))
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    hpw, hpg, hphi = pin(pw), pin(pg), pin(c0)
    hout = torch.empty((n, n, n), dtype=torch.float32 if prec == "f32" else torch.float64).pin_memory().numpy()
    def e2e_run(all_fields):
        barrier()
        torch.cuda.synchronize()
        e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2.record(stream)
        for _ in range(e2e_steps):
            if all_fields:
                pool.upload_dense("p_w", hpw)
                pool.upload_dense("p_g", hpg)
                pool.upload_dense("phi", hphi)
                pool.rd_step(s.Dw, s.Dg, s.rho, s.dt, 1)
                pool._check(pool.lib.gbfk_download_dense(pool.ctx, 0, hout.ctypes.data, n))
            else:
                # host-to-host steps: each step's output copy overlaps the next input copy
                pool.rd_step_host(hphi, hout, s.Dw, s.Dg, s.rho, s.dt, 1)
        if not all_fields:
            pool.join_copies()
        e3.record(stream)
        torch.cuda.synchronize()
        pool.sync()
        return max_over_ranks(e2.elapsed_time(e3))

    # the state goes in and out every step; the anatomy (p_w, p_g), fixed for
    # a whole calibration like a model's weights, stays resident
    pool.upload_dense("p_w", hpw)
    pool.upload_dense("p_g", hpg)
    # warm-up: the first host-to-host call allocates its pinned staging
    # buffers and copy streams
    pool.rd_step_host(hphi, hout, s.Dw, s.Dg, s.rho, s.dt, 1)
    pool.join_copies()
    ms_e2e = e2e_run(False)
    ms_e2e_all = e2e_run(True)
    e2e = {"value": world * cells * e2e_steps / (ms_e2e / 1e3), "unit": UNIT,
           "h2d_bytes_per_step": word * cells, "d2h_bytes_per_step": word * cells,
           "steps": e2e_steps,
           "api": "BlockPool.rd_step_host (gbfk_rd_step_host: H2D of phi from a pinned host buffer, one step, "
                  "D2H of phi to a pinned host buffer; the output copy of a step overlaps the next step's input "
                  "copy); p_w, p_g uploaded once before the timed region",
           "all_fields": {"value": world * cells * e2e_steps / (ms_e2e_all / 1e3), "unit": UNIT,
                          "h2d_bytes_per_step": 3 * word * cells, "d2h_bytes_per_step": word * cells,
                          "api": "BlockPool.upload_dense x3 (p_w, p_g, phi) + rd_step + gbfk_download_dense"}}

    batch = None
    adj = None
    adj5 = None
    adaptive = None
    fp64 = fp64_lines(stream, local, args.steps) if prec == "f32" and n == N_GRID and not args.no_fp64 else None
    if args.adaptive_steps > 0 and rank == 0:
        adaptive = adaptive_forward(args.adaptive_steps, prec)
    if not args.no_batch:
        batch = batched_stage(args, stream, local)
    if not args.no_batch or args.adjoint_sample:
        adj = adjoint_sample(stream, local, check=not args.no_adjoint_check)
    if args.adjoint_batch_steps != 0 and rank == 0:
        adj5 = adjoint_batch(stream, local, max_steps=args.adjoint_batch_steps if args.adjoint_batch_steps > 0 else None)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rec, kind, cores, n_s, st = cpu_reference_run(0, 2, N_GRID if n == N_GRID else CPU_SAMPLE_N, prec,
                                                       target_s=15.0)
        cpu = {"value": rec["cell_updates_per_s"], "unit": UNIT, "cores": cores, "kind": kind,
               "sample": f"{n_s}^3 grid of the same synthetic anatomy, {st} steps of the stepping loop "
                         f"({rec['seconds']:.1f} s) on {cores} host threads",
               "cpu_model": cpu_model(), "host_threads": os.cpu_count()}
        # the same reference on one core, and its FP64 build on all cores
        r1, k1, c1, n1, st1 = cpu_reference_run(0, 1, CPU_SAMPLE_N, prec, target_s=6.0, threads=1)
        cpu["one_core"] = {"value": r1["cell_updates_per_s"], "unit": UNIT, "cores": c1, "kind": k1,
                           "sample": f"{n1}^3 grid, {st1} steps ({r1['seconds']:.1f} s) on 1 host thread"}
        other = "f64" if prec == "f32" else "f32"
        r2, k2, c2, n2, st2 = cpu_reference_run(0, 1, N_GRID if n == N_GRID else CPU_SAMPLE_N, other,
                                                target_s=8.0)
        cpu[other] = {"value": r2["cell_updates_per_s"], "unit": UNIT, "cores": c2, "kind": k2,
                      "sample": f"{n2}^3 grid, {st2} steps ({r2['seconds']:.1f} s) on {c2} host threads, "
                                f"the reference built with Real = {'double' if other == 'f64' else 'float'}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": prec, "data": "synthetic", "config": workload_config(n, prec),
            "parallelism": "replicas" if world > 1 else "single",
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk,
            "batched_stage": batch, "forward_adjoint": adj, "forward_adjoint_16x256": adj5,
            "adaptive_forward": adaptive, "fp64": fp64,
            "not_in_value": "face_kernel (harmonic means, once per topology and (Dw, Dg): about 190 us at 256^3) "
                            "runs in the warm-up, outside the timed steps",
        }
        print(json.dumps(line), flush=True)
    pool.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="gbfk", choices=["gbfk", "reference"])
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    ap.add_argument("--n", type=int, default=N_GRID)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched TMCMC-stage measurement")
    ap.add_argument("--adjoint-sample", action="store_true",
                    help="run the config-4 gradient sample even with --no-batch")
    ap.add_argument("--no-adjoint-check", action="store_true",
                    help="skip the FP64 central-difference check of the config-4 gradients")
    ap.add_argument("--adjoint-batch-steps", type=int, default=3000,
                    help="config 5 (16 gradient samples at 256^3): cap on each sample's steps (-1: the full "
                         "horizons, a few minutes; 0: skip)")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 lines (config 1, 256^3)")
    ap.add_argument("--adaptive-steps", type=int, default=400,
                    help="steps of the config-2 adaptive run on the resident drop-in (0: skip)")
    ap.add_argument("--step-kernel", default="auto", choices=["auto", "block", "pipelined", "run"],
                    help="step kernel of the resident solve (auto: pipelined on uniform power-of-two grids)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)
    return gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
