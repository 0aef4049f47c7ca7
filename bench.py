#!/usr/bin/env python
"""Throughput of the FIT-TD step on the plain-method-at-scale workload.

One step = one full leapfrog step of the brick-box workload
(:func:`magnelio_b200.workloads.brick_box`): E update with the CPML psi
recursion on six 10-layer slabs, the lumped gap source, H update with its
CPML part, and three 64-frequency running-DFT E-field monitors on the
mid-planes, for one field set of ``size^3`` cells.  The metric is
Gcell-updates/s = cells x steps / device time (CUDA events on the engine's
stream), summed over GPUs.  Multi-GPU runs are independent replicas (one
problem per GPU, no exchange), timed as the max over ranks.

``--impl reference`` times the CPU port of the reference's algorithm
(``oracle/``) on the host cores instead, on a bounded sample of steps of the
same workload.
"""

from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "Gcell-updates/s"
BYTES_PER_CELL = 96  # E(3) H(3) read+write, alpha/beta E/H (12) read, float32
FIELD_BYTES_PER_CELL = 48  # the field part of it, per field set
TILE_VARIANT_BASE = 7  # fused-step variants from here on are the TMA tile form
SLAB_VARIANT_BASE = 16  # and from here on the slab step (CPML inside the tile march)
COEF_BYTES_PER_CELL = 48  # the coefficient part, shared by a batch of field sets
BYTES_PER_CPML_CELL = 32  # 2 psi_E + 2 psi_H read+write per slab cell per face, float32


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic(kernel_key: str, n: int, cpml_cells: int = 0):
    """DRAM bytes of one step from a committed ncu summary, if one exists:
    bytes per cell x n^3 (and, for the tile step, bytes per CPML slab cell of
    its CPML passes)."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    v = d.get(kernel_key)
    if v is None:
        return None
    if isinstance(v, dict):
        return float(v["per_cell"]) * n**3 + float(v["per_cpml_face_cell"]) * cpml_cells
    return float(v) * n**3


class ClockSampler:
    """nvidia-smi clock / throttle sampling around the timed region.

    Sampling starts when the object is made (every 50 ms, with a timestamp)
    and is given time to come up; ``window()`` brackets the timed region and
    ``stop()`` keeps the samples inside it.  A region shorter than the
    sampling interval keeps the sample nearest to its middle."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    STARTUP_S = 0.5

    def __init__(self, local_rank: int):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        idx = vis.split(",")[local_rank] if vis else str(local_rank)
        self.proc = None
        self.t0 = self.t1 = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={idx}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            time.sleep(self.STARTUP_S)
        except OSError:
            self.proc = None

    def window(self, start: bool) -> None:
        if start:
            self.t0 = datetime.datetime.now()
        else:
            self.t1 = datetime.datetime.now()

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        return self.summarise(out.strip().splitlines(), self.t0, self.t1)

    @staticmethod
    def summarise(lines, t0, t1) -> dict:
        """Median SM clock, max clock and active throttle reasons of the
        csv ``lines`` (timestamp first) taken between ``t0`` and ``t1``."""
        rows = []
        for line in lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f")
                rows.append((ts, float(parts[2]), float(parts[3]), parts[6:10]))
            except ValueError:
                continue
        inside = rows
        where = "timed region"
        if t0 is not None and t1 is not None and rows:
            inside = [r for r in rows if t0 <= r[0] <= t1]
            if not inside:
                mid = t0 + (t1 - t0) / 2
                inside = [min(rows, key=lambda r: abs((r[0] - mid).total_seconds()))]
                where = "nearest to the timed region (shorter than the 50 ms sampling interval)"
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = set()
        for r in inside:
            for nm, v in zip(names, r[3]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        sm = [r[1] for r in inside]
        smax = [r[2] for r in inside]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "sampled": where}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _max_over_ranks(x: float, world: int, local: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    # NCCL reduces on the rank's GPU; gloo (the CPU tests of this path) on the host
    device = "cpu" if dist.get_backend() == "gloo" else f"cuda:{local}"
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1


def cpu_port_rate(prob, budget_s: float = 20.0, max_steps: int = 200, warmup: int = 2):
    """Gcell-updates/s of the CPU port of the reference's step (C + OpenMP
    on every host thread, float32 as the reference's default precision) on
    the full-size workload: whole steps, timed until ``budget_s`` elapses."""
    from oracle.cport import CPortRun

    threads = cpu_threads()
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    run = CPortRun(prob, "single", max_steps + warmup + 1)
    run.run(warmup)
    n = 0
    t0 = time.perf_counter()
    while n < max_steps:
        run.run(1)
        n += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    cells = prob.nx * prob.ny * prob.nz
    return cells * n / dt / 1e9, n, dt, threads


def parity_prefix(prob, tuned, steps: int, device: int) -> dict:
    """Checker line: the timed workload's first ``steps`` steps on the
    engine (the tuned stencil, float32) against the float64 C port of the
    reference step on the host cores (``oracle/prefix_parity.py``)."""
    from oracle.prefix_parity import Fp64Prefix

    t0 = time.perf_counter()
    ref = Fp64Prefix(prob, steps)
    eng = prob.build_engine("single", device=device)
    try:
        if tuned is not None:
            from magnelio_b200 import autotune

            autotune.apply(eng, tuned)
        eng.step(steps)
        e, h = eng.read_fields()
        out = ref.compare(e, h, eng.read_dft)
        out["stencil"] = eng.stencil_config()
    finally:
        eng.close()
    out["seconds"] = round(time.perf_counter() - t0, 1)
    return out


def run_reference(args, world, rank, local):
    if rank != 0:
        return 0
    from magnelio_b200 import workloads

    prob = workloads.brick_box(args.size, steps=args.steps + args.warmup + 8)
    budget = min(args.cpu_budget * 6, 120.0)
    rate, n, secs, threads = cpu_port_rate(prob, budget_s=budget, max_steps=max(args.steps, 1), warmup=min(args.warmup, 3))
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": METRIC, "n_gpus": world,
        "steps": n, "warmup": min(args.warmup, 3), "ms_per_step": secs / n * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded brick box)",
        "config": _config(args, prob),
        "cpu_baseline": {"value": rate, "unit": METRIC, "cores": threads, "kind": "port",
                         "sample": f"{n} full steps of the {args.size}^3 workload (of {args.steps} asked, "
                                   f"bounded to {budget:.0f} s) after {min(args.warmup, 3)} warm-up steps; "
                                   f"C+OpenMP port, float32, {threads} threads"},
        "e2e": {"value": rate, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _config(args, prob):
    from magnelio_b200 import workloads

    return {
        "workload": f"brick_box_{args.size}",
        "grid": f"{prob.nx}x{prob.ny}x{prob.nz} non-uniform (0.8-1.2 mm, centre-graded)",
        "bricks": "32 dielectric, eps_r U[1,10], cat-1 conformal fill U[0,1]",
        "cpml": f"10 layers x 6 faces ({workloads.cells_in_cpml(prob)} slab cells)",
        "source": "lumped z gap, 50 ohm, modulated Gaussian 1-7.5 GHz",
        "monitors": "3 mid-plane E-field DFT monitors x 64 freq, every step",
        "field_sets": getattr(args, "batch", 1),
        "coefficients": "float32" if getattr(args, "coef", "native") == "native" else f"{args.coef} storage, float32 arithmetic",
        "parallelism": "replicas" if args.gpus > 1 else "single",
        "l2": "inputs larger than L2 (working set >1 GB per GPU)",
    }


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--batch", type=int, default=1, help="field sets sharing one coefficient set")
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU-port timing")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sweep", type=int, nargs="*", default=[512],
                    help="more grid sizes timed after the headline one (N=1 only; none: --sweep)")
    ap.add_argument("--parity-steps", type=int, default=300,
                    help="steps of the float64 parity prefix on the timed workload (0: none)")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (keep the default stencil plan)")
    ap.add_argument("--stencil", default=None, metavar="KIND:VARIANT[:ICHUNK]",
                    help="run this stencil form instead of the autotuner's pick (e.g. fused:16)")
    ap.add_argument("--workload", choices=("brick_box", "slab", "cross", "wr90"), default="brick_box",
                    help="brick_box (plain method at scale), slab (dispersive slab, TF/SF plane wave, 384x384x192) "
                         "or cross (four-port junction, eight excitations batched vs one at a time)")
    ap.add_argument("--precision-study", action="store_true",
                    help="R/T of the slab workload per precision variant against its float64 run")
    ap.add_argument("--study-size", type=int, nargs=3, default=(96, 96, 128))
    ap.add_argument("--serving", action="store_true",
                    help="serve the S-parameter request stream (batched and one excitation at a time) instead")
    ap.add_argument("--serving-requests", type=int, default=256)
    ap.add_argument("--serving-ports", choices=("modal", "lumped"), default="modal",
                    help="waveguide ports with 1-3 modes on both ends (the configuration), or lumped ports only")
    ap.add_argument("--serving-stencil", default=None, metavar="BATCHED[,PLAIN]",
                    help="stencil forms of the served handles, KIND:VARIANT or 'default' each (batched, then "
                         "one-excitation handles; the loop's own choice when absent)")
    ap.add_argument("--serving-coef", choices=("native", "f16"), default="native",
                    help="coefficient storage of the served handles (f16: 16-bit with per-component scales)")
    ap.add_argument("--serving-scale", type=float, default=1.0,
                    help="scale factor on the request grid sizes and step counts (1 = the full stream)")
    ap.add_argument("--coef", choices=("native", "f16", "bf16"), default="native",
                    help="coefficient storage of the stencil kernels (16-bit forms round the coefficients)")
    ap.add_argument("--dist-backend", choices=("nccl", "gloo"), default="nccl",
                    help="process-group backend for N > 1 (gloo: host-only runs of the replica path)")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    world, rank, local = _dist()
    if world > 1:
        import torch
        import torch.distributed as dist

        if args.dist_backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(args.dist_backend, timeout=datetime.timedelta(seconds=120))
    try:
        if args.impl == "reference":
            return run_reference(args, world, rank, local)
        if args.serving:
            return run_serving(args, world, rank, local)
        if args.precision_study:
            return run_precision_study(args, world, rank, local)
        if args.workload == "slab":
            return run_slab(args, world, rank, local)
        if args.workload == "cross":
            return run_cross(args, world, rank, local)
        if args.workload == "wr90":
            return run_wr90(args, world, rank, local)
        return run_b200(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


def run_serving(args, world, rank, local):
    """Serving workload: Poisson stream of waveguide-section S-parameter
    requests (mean gap 20 ms), served with continuous batching and, for
    comparison, one excitation per handle at a time."""
    from magnelio_b200 import serving

    sc = args.serving_scale
    cells = (max(8**3, int(32**3 * sc)), max(8**3, int(192**3 * sc)))
    steps = (max(100, int(6000 * sc)), max(100, int(12000 * sc)))
    reqs = serving.request_stream(args.serving_requests, seed=2027 + rank, mean_gap=0.020, cells=cells, steps=steps,
                                  port_kind=args.serving_ports)
    stencil = serving.serving_stencil
    if args.serving_stencil:
        forms = [None if f in ("default", "") else (f.split(":")[0], int(f.split(":")[1]))
                 for f in args.serving_stencil.split(",")]
        forms = forms + forms[-1:] if len(forms) == 1 else forms

        def stencil(batch, _f=forms):
            return _f[0] if batch > 1 else _f[1]
    coef = None if args.serving_coef == "native" else args.serving_coef
    # S-matrices from the device post-step: the V/I histories never leave the GPU
    batched = serving.ServingLoop(device=local, max_slots=8, slice_steps=512, records=False, stencil=stencil,
                                  coef=coef).run(reqs)
    plain = serving.ServingLoop(device=local, slice_steps=512, records=False, stencil=stencil,
                                coef=coef).run(reqs, plain=True)
    # the slowest replica bounds the whole job
    solves = -_max_over_ranks(-batched.solves_per_s, world, local)
    if rank == 0:
        line = {
            "metric": "S-param solves/s", "value": solves * world, "unit": "solves/s", "n_gpus": world,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded waveguide-section request stream)",
            "config": {"workload": "serving_stream", "requests": len(reqs), "arrivals": "Poisson, mean gap 20 ms",
                       "cells": list(cells), "steps": list(steps),
                       "ports": ("2-4: waveguide ports on both ends with 1-3 TE modes each (modes solved and DTBC "
                                 "tables built on the device per request), the rest 50 ohm lumped"
                                 if args.serving_ports == "modal" else "2-4 lumped, 50 ohm"),
                       "s_matrix": "device post-step (fitb_s_params)",
                       "max_slots": 8, "slice_steps": 512,
                       "stencil": {"batched": str(stencil(2) or "engine default (batched two-pass)"),
                                   "plain": str(stencil(1) or "engine default")},
                       "coefficients": "float32" if coef is None else f"{coef} storage, float32 arithmetic"},
            "p50_s": batched.p50, "p99_s": batched.p99, "wall_s": batched.wall,
            "mean_active": batched.mean_active, "peak_device_bytes": batched.peak_bytes,
            "plain": plain.summary(), "ratio_vs_plain": batched.solves_per_s / max(plain.solves_per_s, 1e-12),
        }
        print(json.dumps(line), flush=True)
    return 0


def run_precision_study(args, world, rank, local):
    """Slab reflection / transmission per precision variant (float32 fields
    with float32, float16 or bfloat16 coefficients, Kahan-compensated DFT
    bins or not) against the float64 run of the same problem."""
    from magnelio_b200 import precision

    nx, ny, nz = args.study_size
    res = precision.precision_study(nx, ny, nz, args.steps, device=local)
    if rank == 0:
        line = {"metric": "slab R/T deviation from float64", "unit": "linear |dT|, |dR|; degrees",
                "higher_is_better": False, "n_gpus": world, "steps": args.steps,
                "config": {"workload": f"dispersive_slab_{nx}x{ny}x{nz}", "poles": "2 Lorentz pairs, 8 and 14 GHz",
                           "source": "TF/SF Gaussian plane wave +z, f_max 20 GHz", "band": "1-20 GHz, 64 freqs"},
                "variants": {k: {m: v[m] for m in ("dR", "dT", "dT_phase_deg")} for k, v in res.items()
                             if k != "freqs"}}
        print(json.dumps(line), flush=True)
    return 0


def run_cross(args, world, rank, local):
    """Batching configuration: WR-90 cross junction (200 x 200 x 40 cells,
    PEC corner blocks, 4 waveguide ports x 2 DTBC modes), the eight port x
    mode excitations for the full 12000 steps as one batch of eight field
    sets, then the same eight one at a time; device time of each.  The
    problem (port modes, DTBC kernels, waveforms) was set up by the
    reference's own analysis and is stored with the tests."""
    sys.path.insert(0, str(ROOT / "tests"))
    from conftest import load_golden

    from magnelio_b200 import autotune

    prob, _d, n_full = load_golden("cfg3_cross_full")
    steps = n_full if args.steps >= n_full else args.steps
    cells = prob.nx * prob.ny * prob.nz
    n_exc = prob.batch

    def one_excitation(b):
        q = load_golden("cfg3_cross_full")[0]
        q.batch = 1
        for mp in q.modal:
            mp.excitation = [mp.excitation[b]]
        q.e0, q.h0 = [None], [None]
        return q

    tuned = tuned1 = None
    if not args.no_tune:
        tuned = autotune.tune_problem(prob, "single", batch_widths=(n_exc,), device=local, iters=5)
        tuned1 = autotune.tune_problem(one_excitation(0), "single", batch_widths=(1,), device=local, iters=5)

    def build(q, t):
        e = q.build_engine("single", device=local)
        if t is not None:
            autotune.apply(e, t)
        return e

    eng = build(prob, tuned)
    eng.step(args.warmup)
    eng.close()
    eng = build(prob, tuned)
    ms_batched = eng.step_timed(steps)
    stencil_cfg = eng.stencil_config()
    units = eng.slab_units()
    eng.close()
    ms_seq = 0.0
    for b in range(n_exc):
        e1 = build(one_excitation(b), tuned1)
        ms_seq += e1.step_timed(steps)
        stencil1 = e1.stencil_config()
        e1.close()
    ms_batched = _max_over_ranks(ms_batched, world, local)
    ms_seq = _max_over_ranks(ms_seq, world, local)
    solve_steps = n_full
    if rank == 0:
        line = {
            "metric": "batched S-param solves/s", "unit": "solves/s", "n_gpus": world, "steps": steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "reference-built port setup (stored), eight DTBC excitations",
            "value": world * 1e3 / (ms_batched / steps * solve_steps),
            "gcell_updates_per_s": cells * n_exc * steps * world / (ms_batched * 1e-3) / 1e9,
            "sequential": {"solves_per_s": world * 1e3 / (ms_seq / steps * solve_steps),
                           "gcell_updates_per_s": cells * n_exc * steps * world / (ms_seq * 1e-3) / 1e9},
            "ratio_vs_sequential": ms_seq / ms_batched,
            "config": {"workload": f"cross_junction_{prob.nx}x{prob.ny}x{prob.nz}", "field_sets": n_exc,
                       "solve": f"all {n_exc} excitations x {solve_steps} steps", "stencil": stencil_cfg,
                       "stencil_sequential": stencil1,
                       "units": units if units["dead"] or sum(units["slots"]) else None,
                       "autotune": None if tuned is None else [list(r[:3]) + [round(r[4], 4)] for r in tuned.table]},
        }
        print(json.dumps(line), flush=True)
    return 0


def run_wr90(args, world, rank, local):
    """Plain-method configuration: the WR-90 section (29 x 13 x 51 cells, two
    3-mode DTBC ports) set up by the reference's own analysis (stored with
    the tests), all six port x mode excitations for the full 8000 steps as
    one batch, the 6 x 6 S-matrix on 501 frequencies from the device
    post-step, compared with the reference's S-matrix (|dS| and phase in
    each excitation's band)."""
    sys.path.insert(0, str(ROOT / "tests"))
    from conftest import load_golden
    from magnelio_b200 import autotune, sparams

    prob, d, n_full = load_golden("cfg1_wr90")
    c = sparams.load_cfg1(d)
    cells = prob.nx * prob.ny * prob.nz
    tuned = None
    if not args.no_tune:
        tuned = autotune.tune_problem(prob, "single", batch_widths=(prob.batch,), device=local, iters=5)
    times, S = [], None
    for rep in range(2):  # the first solve warms the graphs and clocks
        eng = prob.build_engine("single", device=local)
        if tuned is not None:
            autotune.apply(eng, tuned)
        ms = eng.step_timed(n_full)
        t0 = time.perf_counter()
        S, A = eng.s_parameters(c["f"], np.stack(c["maps"]), c["icot"], c["excited"], return_incident=True)
        post_ms = (time.perf_counter() - t0) * 1e3
        cfg = eng.stencil_config()
        eng.close()
        times.append((ms, post_ms))
    ms, post_ms = times[-1]
    ref, A_ref = sparams.s_matrix(c["V"], c["I"], c["dt"], c["f"], c["maps"], c["icot"], c["excited"],
                                  return_incident=True)
    band = np.abs(A_ref) >= 1e-2 * np.max(np.abs(A_ref), axis=0, keepdims=True)
    sel = np.isfinite(ref) & (np.abs(ref) <= 1.05) & band[:, None, :]
    dS = float(np.abs(S - ref)[sel].max())
    big = sel & (np.abs(ref) > 0.05)
    dphi = float(np.degrees(np.abs(np.angle(S[big] / ref[big]))).max())
    ms = _max_over_ranks(ms, world, local)
    if rank == 0:
        line = {
            "metric": "S-matrix solves/s", "unit": "solves/s", "n_gpus": world, "steps": n_full,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "reference-built WR-90 setup (stored): two 3-mode DTBC ports, six excitations",
            "value": world * 1e3 / (ms + post_ms), "ms_per_step": ms / n_full,
            "gcell_updates_per_s": cells * prob.batch * n_full / (ms * 1e-3) / 1e9,
            "s_post_ms": post_ms,
            "parity": {"dS_max": dS, "phase_max_deg": dphi, "vs": "reference S-matrix (float64 analysis)",
                       "bins": int(sel.sum())},
            "config": {"workload": f"wr90_{prob.nx}x{prob.ny}x{prob.nz}", "field_sets": prob.batch,
                       "solve": f"all {prob.batch} excitations x {n_full} steps, S on {len(c['f'])} frequencies",
                       "stencil": cfg},
        }
        print(json.dumps(line), flush=True)
    return 0


def run_slab(args, world, rank, local):
    """The precision configuration's workload at full size: 384 x 384 x 192
    cells, two-pole Lorentz slab (ADE on device), TF/SF plane wave, CPML on
    six faces (separate passes after the ADE update), two DFT planes."""
    from magnelio_b200 import autotune, workloads

    nx, ny, nz = 384, 384, 192
    prob = workloads.dispersive_slab(nx, ny, nz)
    tuned = None
    if not args.no_tune:
        tuned = autotune.tune_problem(prob, "single", device=local, coef=args.coef, iters=5)
    eng = prob.build_engine("single", device=local)
    if args.coef != "native":
        eng.set_coefficient_storage(args.coef)
    if tuned is not None:
        autotune.apply(eng, tuned)
    stencil_cfg = eng.stencil_config()
    cells = nx * ny * nz
    sampler = ClockSampler(local)
    eng.step(args.warmup)
    eng.sync()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    l0 = eng.launch_count
    sampler.window(True)
    ms = eng.step_timed(args.steps)
    sampler.window(False)
    launches = eng.launch_count - l0
    clocks = sampler.stop()
    ms = _max_over_ranks(ms, world, local)
    value = cells * args.steps * world / (ms * 1e-3) / 1e9
    # end to end through the public API: one fitb_step per step, the
    # transmission plane's bins read back at the end
    eng.sync()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        eng.step(1)
    bins = eng.read_dft(1, "Ex")
    e2e_s = _max_over_ranks(time.perf_counter() - t0, world, local)
    e2e = cells * args.steps * world / e2e_s / 1e9
    t_e, t_h = eng.time_stencil(20)
    coef_bytes = COEF_BYTES_PER_CELL if args.coef == "native" else COEF_BYTES_PER_CELL // 2
    # stencil launches without their CPML (it runs as passes after the ADE update)
    alg_bytes = (FIELD_BYTES_PER_CELL + coef_bytes) * cells
    achieved = alg_bytes / ((t_e + t_h) * 1e-3) / 1e9
    peak, peak_kind = _peaks()
    eng.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded dispersive slab, host-built setup)",
            "config": {"workload": f"dispersive_slab_{nx}x{ny}x{nz}", "cpml": "10 layers x 6 faces",
                       "dispersion": f"2 Lorentz pairs, {sum(b.idx.size for d in prob.dispersion for b in d.blocks)} states",
                       "source": "TF/SF Gaussian plane wave +z, f_max 20 GHz",
                       "monitors": "2 E-field DFT planes x 64 freq, every step",
                       "stencil": stencil_cfg, "l2": "inputs larger than L2"},
            "roofline": {"bound": "hbm", "kernel": "update_E + update_H (one stencil step, no CPML)",
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "algorithmic_bytes": alg_bytes, "ms_E": t_e,
                         "ms_H": t_h, "step_share": (t_e + t_h) / (ms / args.steps)},
            "cpu_baseline": None,
            "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(bins.size * 8 / args.steps),
                    "how": "one fitb_step per step, the transmission plane's bins read back at the end"},
            "gpu_launches": launches, "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    return 0


SWEEP_CANDIDATES = (("stream", 0, 0), ("fused", 7, 0), ("fused", 16, 0), ("fused", 17, 0), ("fused", 18, 0),
                    ("fused", 19, 0), ("fused", 20, 0), ("fused", 21, 0), ("fused", 22, 0), ("fused", 23, 0),
                    ("fused", 24, 0), ("fused", 25, 0))


def sweep_point(n: int, args, local: int) -> dict:
    """One more grid size of the same workload, timed the same way as the
    headline (device time of graph-replayed steps, clocks sampled over the
    timed region), with the stencil tuned over the fastest forms."""
    from magnelio_b200 import autotune, workloads

    total = args.warmup + args.steps + 8
    prob = workloads.brick_box(n, steps=total)
    tuned = autotune.tune_problem(prob, "single", device=local, candidates=SWEEP_CANDIDATES, iters=3)
    eng = prob.build_engine("single", device=local)
    try:
        autotune.apply(eng, tuned)
        sampler = ClockSampler(local)
        eng.step(args.warmup)
        eng.sync()
        sampler.window(True)
        ms = eng.step_timed(args.steps)
        sampler.window(False)
        clocks = sampler.stop()
        t_e, t_h = eng.time_stencil(10)
        cfg = eng.stencil_config()
    finally:
        eng.close()
    cpml_cells = workloads.cells_in_cpml(prob)
    alg = BYTES_PER_CELL * n**3 + BYTES_PER_CPML_CELL * cpml_cells
    peak, peak_kind = _peaks()
    achieved = alg / ((t_e + t_h) * 1e-3) / 1e9
    return {"size": n, "value": n**3 * args.steps / (ms * 1e-3) / 1e9, "unit": METRIC,
            "ms_per_step": ms / args.steps, "stencil": cfg,
            "roofline": {"achieved": achieved, "peak": peak, "peak_kind": peak_kind, "frac": achieved / peak,
                         "algorithmic_bytes": alg, "ms_stencil": t_e + t_h},
            "clocks": clocks}


def run_b200(args, world, rank, local):
    from magnelio_b200 import workloads

    n = args.size
    total = args.warmup + 2 * args.steps + 64
    prob = workloads.brick_box(n, steps=total)
    B = args.batch
    if B > 1:
        # B field sets of the same mesh, each driven by its own amplitude
        prob.batch = B
        v = prob.lumped[0].v_src[0]
        prob.lumped[0].v_src = [v * (1.0 + 0.1 * b) for b in range(B)]
    tuned = None
    if args.stencil:
        from magnelio_b200 import autotune

        parts = args.stencil.split(":")
        tuned = autotune.TuneResult(kind=parts[0], variant=int(parts[1]) if len(parts) > 1 else 0,
                                    ichunk=int(parts[2]) if len(parts) > 2 else 0, batch=B, ms=0.0, gcells=0.0)
    elif not args.no_tune:
        # stencil form, march depth: fastest on this GPU for this grid / batch
        from magnelio_b200 import autotune

        tuned = autotune.tune_problem(prob, "single", batch_widths=(B,), device=local, coef=args.coef, iters=5)
    eng = prob.build_engine("single", device=local)
    if args.coef != "native":
        eng.set_coefficient_storage(args.coef)
    if tuned is not None:
        from magnelio_b200 import autotune

        autotune.apply(eng, tuned)
    stencil_cfg = eng.stencil_config()
    coef_bytes = COEF_BYTES_PER_CELL if args.coef == "native" else COEF_BYTES_PER_CELL // 2
    cells = n**3 * B
    # warm-up (graph capture, clocks)
    sampler = ClockSampler(local)
    eng.step(args.warmup)
    eng.sync()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    l0 = eng.launch_count
    sampler.window(True)
    ms = eng.step_timed(args.steps)
    sampler.window(False)
    launches = eng.launch_count - l0
    clocks = sampler.stop()
    ms = _max_over_ranks(ms, world, local)
    value = cells * args.steps * world / (ms * 1e-3) / 1e9

    # end to end through the public API: every step streams its source
    # sample host->device from pinned memory and reads its recorded V/I back
    import torch

    pinned = torch.empty(args.steps, dtype=torch.float64, pin_memory=True)
    base = eng.steps_done
    pinned.copy_(torch.from_numpy(np.ascontiguousarray(prob.lumped[0].v_src[0][base:base + args.steps])))
    stride = pinned.element_size()
    eng.sync()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    # the step's V/I land in page-locked host memory; the host waits for step
    # s - 1's values while step s runs (one step of read-behind)
    nch = eng.n_channels
    vi_host = torch.empty((2, args.steps, max(nch, 1)), dtype=torch.float64, pin_memory=True)
    row = max(nch, 1) * 8
    t0 = time.perf_counter()
    prev = None
    for s in range(args.steps):
        eng.push_lumped_samples(0, 0, base + s, 1, pinned.data_ptr() + s * stride)
        eng.step(1)
        t = eng.read_vi_async(0, base + s, 1, vi_host[0].data_ptr() + s * row, vi_host[1].data_ptr() + s * row)
        if prev is not None:
            eng.wait_ticket(prev)
        prev = t
    eng.wait_ticket(prev)
    eng.sync()
    e2e_s = _max_over_ranks(time.perf_counter() - t0, world, local)
    e2e = cells * args.steps * world / e2e_s / 1e9
    # the values read are the recorder's
    V_ref, I_ref = eng.read_vi(0, base, args.steps)
    assert np.array_equal(vi_host[0].numpy()[:, :nch], V_ref) and np.array_equal(vi_host[1].numpy()[:, :nch], I_ref)

    # stencil roofline: E and H updates timed alone (advances the fields,
    # after all measured runs)
    t_e, t_h = eng.time_stencil(20)
    t_pair = t_e + t_h
    cpml_cells = workloads.cells_in_cpml(prob)
    alg_bytes = (FIELD_BYTES_PER_CELL * B + coef_bytes) * n**3 + BYTES_PER_CPML_CELL * B * cpml_cells
    achieved = alg_bytes / (t_pair * 1e-3) / 1e9
    peak, peak_kind = _peaks()
    tile = stencil_cfg["kind"] == "fused" and TILE_VARIANT_BASE <= stencil_cfg["variant"] < SLAB_VARIANT_BASE
    slab = stencil_cfg["kind"] == "fused" and stencil_cfg["variant"] >= SLAB_VARIANT_BASE
    if slab:
        kernel = "k_step_slab (one stencil step, CPML inside the march)"
        traffic = _traffic("slab_step", n, cpml_cells) if B == 1 else None
    elif tile:
        kernel = "k_step_tile + CPML passes (one stencil step)"
        traffic = _traffic("tile_step", n, cpml_cells) if B == 1 else None
    else:
        kernel = "update_E + update_H (one stencil step)"
        traffic = _traffic("update_E+update_H", n) if stencil_cfg["kind"] == "stream" and B == 1 else None
    roofline = {"bound": "hbm", "kernel": kernel, "achieved": achieved,
                "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "algorithmic_bytes": alg_bytes, "ms_E": t_e, "ms_H": t_h,
                "step_share": t_pair / (ms / args.steps)}
    eng.close()

    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and B == 1:
        rate, ns, secs, threads = cpu_port_rate(prob, budget_s=args.cpu_budget)
        cpu = {"value": rate, "unit": METRIC, "cores": threads, "kind": "port",
               "sample": f"{ns} full steps of the {n}^3 workload after 2 warm-up steps "
                         f"(C+OpenMP port, float32, {threads} threads, {secs:.1f} s)"}
        if args.parity_steps > 0:
            parity = parity_prefix(prob, tuned, args.parity_steps, local)
    sweep = None
    if rank == 0 and world == 1 and B == 1 and args.sweep:
        sweep = [sweep_point(m, args, local) for m in args.sweep if m != n]
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded brick box, host-built coefficients)",
            "config": dict(_config(args, prob), stencil=stencil_cfg,
                           autotune=None if tuned is None or not tuned.table
                           else [list(r[:3]) + [round(r[4], 4)] for r in tuned.table]),
            "roofline": roofline, "cpu_baseline": cpu, "parity": parity, "sweep": sweep,
            "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": 8, "d2h_bytes_per_step": 16 * nch,
                    "how": "per step: pinned H2D of the source sample, one fitb_step, async D2H of the step's V/I "
                           "into pinned memory (fitb_read_vi_async), the host waiting for the previous step's "
                           "values while the step runs"},
            "gpu_launches": launches, "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
