#!/usr/bin/env python
"""Benchmark of the KPM moment loop (the LSQT hot path) on B200.

One step = one KPM moment set: mu_m = <phi|T_m(H/E_max)|phi>, m < 3000, over the
honeycomb graphene lattice of 2,097,152 sites (4-orbital cell x 1024x512, t = -2.7 eV,
Anderson W = 1.0 eV, seed 3, E_max 8.7 eV) for one random-phase vector per GPU, in the
plain FP64 form (the reference's arithmetic, bit-identical per site) with the operator
in its default device format (coded: one byte per ELL entry). value = site-moments/s
over all ranks (sites x moments x steps / max-over-ranks device time).

Also reported, on the same line:
  roofline      the dominant kernel (the fused Chebyshev step + moment partial sums)
  e2e           the same metric through the public API with host buffers
  forms         graphene 2M in every form: FP64 on the ELL arrays, FP32 storage with
                1/16/32 vectors per launch, symmetric (doubled) sets in FP64 and FP32,
                each with its byte model and roofline fraction; `target_ratios` states the
                FP32/FP64 ratios like for like (direct/direct, doubled/doubled) next to
                their byte-model ceilings
  evolution     the Bessel evolution of one 1 fs MSD step (evolve, evolvex)
  batch         the realisation batch (8 uneven square lattices, 64 vectors, FP32)
  cubic256      the 3D Anderson lattice 256^3 (z = 6): FP64 and 16-vector FP32 side by
                side (DOS rate, one VAC and one MSD correlation step, errors)
  precision     graphene 4M, 5000 moments: error of the FP32, FP32X and FP32R forms
                against FP64 for the DOS and 20 VAC steps (peak-relative and pointwise)
  precision_msd graphene 2M, 3000 moments: the same for 20 MSD steps of 1 fs
  cpu_baseline  the reference's CPU path (oracle/_ref) on this host: one core, and
                one process per core

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
Multi-GPU runs are launched with torchrun, one rank per GPU (independent replicas).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "KPM site-moments/s + HBM GB/s: batched FP32/FP64-acc vs plain FP64 at ≤1e-6 err"
UNIT = "site-moments/s"
WORKLOAD = "graphene2m"
# Algorithmic bytes per site-moment of the fused step (uniform rows, z = 3): per
# neighbour entry 1 B in the coded format (a table row number; the table of distinct
# (j - i, hopping, xx) entries sits in shared memory) or 20 B in the ELL format (index
# 4 B + complex hopping 16 B); on-site potential 8 B; four complex vector streams
# (T_{m-2} read, T_{m-1} read once, T_m write, left read).
Z = 3


def entry_bytes(coded):
    return 1 if coded else 4 + 16


def fp64_bytes_per_site(z=Z, coded=True):
    return z * entry_bytes(coded) + 8 + 4 * 16


def fp32_bytes_per_site_vector(V, z=Z, coded=True):
    return (z * entry_bytes(coded) + 8) / V + 4 * 8


# FP32X storage: FP32 plus a BF16 residual, 12 bytes per complex element, in all four
# streams (the loop's copy of left is FP32X too).
def fp32x_bytes_per_site_vector(V, z=Z, coded=True):
    return (z * entry_bytes(coded) + 8) / V + 4 * 12


# A step of a symmetric (doubled) moment set reads T_{k-1} and T_{k-2} and writes T_k
# (no left stream) and yields two moments.
def fp64_pair_bytes_per_site_step(z=Z, coded=True):
    return z * entry_bytes(coded) + 8 + 3 * 16


def fp32_pair_bytes_per_site_vector_step(V, z=Z, coded=True):
    return (z * entry_bytes(coded) + 8) / V + 3 * 8


# Evolution terms (per site and term): k_cheb2 reads T_{m-1} (gathered once), T_{m-2},
# reads and writes the accumulator and writes T_m; k_cheb2x does the same for the
# state and its [X, .] partner (the coded format keeps xx in its table).
def cheb2_bytes_per_site(z=Z, coded=True):
    return z * entry_bytes(coded) + 8 + 5 * 16


def cheb2x_bytes_per_site(z=Z, coded=True):
    return z * (entry_bytes(coded) + (0 if coded else 8)) + 8 + 10 * 16


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ----------------------------------------------------------------------------- plumbing
def dist():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as td
        torch.cuda.set_device(local)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                              device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as td
        td.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as td
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during a timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.index), "-f", self.path],
                stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        rows = []
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        os.remove(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ----------------------------------------------------------------------------- CPU side
def reference_dir(src, dst):
    """A copy of an input directory the reference binaries accept (no seed keywords)."""
    os.makedirs(dst, exist_ok=True)
    for f in os.listdir(src):
        if f.endswith(".in"):
            shutil.copy(os.path.join(src, f), dst)
    with open(os.path.join(src, "para.in")) as f:
        lines = [l for l in f if l.split() and l.split()[0] not in
                 ("seed", "disorder_seed", "phase_seed")]
    with open(os.path.join(dst, "para.in"), "w") as f:
        f.writelines(lines)
    return dst


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def time_reference(ref_dir, n_moments, reps, procs):
    """Run the reference's find_moments_chebyshev (oracle/_ref/ref_driver) in `procs`
    independent processes at once; returns per-rep max-over-process seconds."""
    import oracle
    if not oracle.have_ref():
        return None, "reference build oracle/_ref not present"
    ps = [subprocess.Popen([oracle.REF_DRIVER, "time", ref_dir, str(n_moments), str(reps)],
                           stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
          for _ in range(procs)]
    per = []
    for p in ps:
        out, _ = p.communicate()
        if p.returncode != 0:
            return None, f"ref_driver exited {p.returncode}"
        per.append(json.loads(out.strip().splitlines()[-1])["reps_s"])
    return [max(p[r] for p in per) for r in range(reps)], None


def cpu_baseline_configs(tmp, names=("graphene4m", "cubic256"), n_moments_sample=16,
                         reps=2):
    """The reference's CPU moment loop on the larger workloads (one process: its 1-core
    rate), a bounded sample of moments each; the rate per site-moment does not depend
    on the count."""
    from gpuqt_b200 import workloads as W
    out = {}
    for name in names:
        rd = reference_dir(W.config_dir(os.path.join(tmp, "cpu"), name),
                           os.path.join(tmp, "cpu_ref", name))
        t, why = time_reference(rd, n_moments_sample, reps, 1)
        if t is None:
            out[name] = {"value_1_core": None, "why": why}
            continue
        out[name] = {"value_1_core": W.config_sites(name) * n_moments_sample /
                                     statistics.mean(t),
                     "unit": UNIT, "sample": f"{n_moments_sample} moments per call, {reps} "
                                             f"calls, one process, the reference's fixed "
                                             f"seed"}
    return out


def cpu_baseline_line(ref_dir, n_sites, n_moments_sample=64, reps=3):
    """The reference's CPU moment loop on this host: one process (the reference is
    serial: its 1-core rate) and one process per core at once (the host's aggregate,
    independent vectors)."""
    procs = min(host_cores(), 64)
    t1, why = time_reference(ref_dir, n_moments_sample, reps, 1)
    if t1 is None:
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": why}
    t, why = time_reference(ref_dir, n_moments_sample, reps, procs)
    if t is None:
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": why}
    one_core = n_sites * n_moments_sample / statistics.mean(t1)
    return {"value": procs * n_sites * n_moments_sample / statistics.mean(t), "unit": UNIT,
            "cores": procs, "kind": "reference", "cpu_model": cpu_model(),
            "value_1_core": one_core,
            "sample": f"reference find_moments_chebyshev (oracle/_ref, g++ -O3, serial) on "
                      f"the same lattice (its fixed seed 12345678), {n_moments_sample} "
                      f"moments per call; value: {procs} independent processes at once, "
                      f"{reps} calls each, mean of the slowest process; value_1_core: one "
                      f"process alone, {reps} calls"}


# ----------------------------------------------------------------------------- arms
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from gpuqt_b200 import workloads as W
    tmp = tempfile.mkdtemp(prefix="gqt_bench_ref_")
    try:
        src = W.config_dir(tmp, WORKLOAD)
        rd = reference_dir(src, os.path.join(tmp, "ref"))
        n = W.config_sites(WORKLOAD)
        sample = 64
        procs = min(host_cores(), 64)
        t, why = time_reference(rd, sample, args.warmup + args.steps, procs)
        if t is None:
            print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)
            return
        timed = t[args.warmup:]
        mean = statistics.mean(timed)
        value = procs * n * sample / mean
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": mean * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(workload_config(WORKLOAD),
                           moments=sample, seed=12345678,
                           sample=f"{sample} of the workload's 3000 moments per process and "
                                  f"step (the rate per site-moment does not depend on the "
                                  f"count); the reference's fixed seed 12345678 instead of "
                                  f"seed 3 (same lattice and disorder strength)",
                           form="reference CPU path (its own objects, g++ -O3), FP64",
                           parallelism=f"{procs} host processes (independent vectors)"),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "reference",
                             "cpu_model": cpu_model(),
                             "sample": f"{sample}-moment find_moments_chebyshev per process "
                                       f"per step, {procs} processes at once"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def workload_config(name):
    """The bench line's `config` for a workload: its parameters, one key each."""
    from gpuqt_b200 import workloads as W
    c = W.CONFIGS[name]
    lattice = {"graphene": "honeycomb graphene (4-orbital cell)", "square": "square",
               "cubic": "cubic"}[c["kind"]]
    return {"workload": name, "lattice": lattice,
            "cells": "x".join(str(v) for v in c["cells"]), "sites": W.config_sites(name),
            "z": {"graphene": 3, "square": 4, "cubic": 6}[c["kind"]],
            "pbc": "all in-plane" if c["kind"] != "cubic" else "all",
            "hopping": c["hopping"], "anderson_w": c["anderson"],
            "seed": c.get("seed", c.get("disorder_seed")), "energy_max": c["energy_max"],
            "moments": c["moments"]}


def dos_error(g, m, mu64, mu32):
    e = m.energy
    d64 = g.chebyshev_summation(mu64[0], mu64[1], e, m.energy_max, m.volume)
    d32 = g.chebyshev_summation(mu32[0], mu32[1], e, m.energy_max, m.volume)
    return float(np.max(np.abs(d32 - d64)) / np.max(np.abs(d64)))


def run_ours(args):
    import torch

    import gpuqt_b200 as g
    from gpuqt_b200 import workloads as W

    rank, world, local = dist()
    if world > 1:
        # The forms, batch, cubic and precision sections characterise one GPU (the N = 1
        # run reports them); a run over N replicas measures the scaled loop alone.
        args.no_forms = args.no_batch = args.no_cubic = args.no_precision = True
    hbm_peak, peak_kind = peaks()
    tmp = tempfile.mkdtemp(prefix=f"gqt_bench_{rank}_")
    try:
        src = W.config_dir(tmp, WORKLOAD)
        m = g.Model.load(src)
        n, M = m.n, m.n_moments
        # Replicas: rank r runs the r-th random-phase vector of the model's stream.
        for _ in range(rank):
            m.initial_state()
        phi = m.initial_state()
        H = g.Hamiltonian(m)
        stream = torch.cuda.current_stream()
        g.set_stream(stream.cuda_stream)
        x = g.Vector.from_host(*phi)
        mu = torch.empty(2 * M, dtype=torch.float64, device="cuda")

        # --- plain FP64 moment sets, inputs resident in HBM
        for _ in range(args.warmup):
            g.moments_device(H, x, x, M, mu.data_ptr())
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        g.reset_launch_count()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(local) as clk:
            t0.record(stream)
            for _ in range(args.steps):
                g.moments_device(H, x, x, M, mu.data_ptr())
            t1.record(stream)
            torch.cuda.synchronize()
        launches = g.launch_count()
        barrier(world)
        torch.cuda.synchronize()
        ms = max_over_ranks(t0.elapsed_time(t1), world)
        clocks = clk.summary()
        value = world * n * M * args.steps / (ms / 1e3)
        per_launch_s = t0.elapsed_time(t1) / 1e3 / (args.steps * M)
        coded = H.format == g.FORMAT_CODED
        fmt = "coded" if coded else "ell"
        bpl = fp64_bytes_per_site(coded=coded) * n
        achieved = bpl / per_launch_s / 1e9
        traffic = None
        tp = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tp):
            with open(tp) as f:
                traffic = json.load(f).get(f"k_step_fp64_{fmt}_graphene2m_bytes_per_launch")

        # --- e2e: host phase vector (pinned) -> device, moments -> host, every step
        re_h = torch.from_numpy(np.ascontiguousarray(phi[0])).pin_memory()
        im_h = torch.from_numpy(np.ascontiguousarray(phi[1])).pin_memory()
        for _ in range(2):
            x.upload_ptr(re_h.data_ptr(), im_h.data_ptr())
            g.moments(H, x, x, M)
        barrier(world)
        torch.cuda.synchronize()
        marks = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps + 1)]
        wall0 = time.perf_counter()
        marks[0].record(stream)
        for k in range(args.steps):
            x.upload_ptr(re_h.data_ptr(), im_h.data_ptr())
            marks[2 * k + 1].record(stream)
            mr, mi = g.moments(H, x, x, M)
            marks[2 * k + 2].record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
        e_ms = max_over_ranks(marks[0].elapsed_time(marks[-1]), world)
        up = sum(marks[2 * k].elapsed_time(marks[2 * k + 1]) for k in range(args.steps))
        mo = sum(marks[2 * k + 1].elapsed_time(marks[2 * k + 2]) for k in range(args.steps))
        e2e = {"value": world * n * M * args.steps / (e_ms / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": 2 * n * 8, "d2h_bytes_per_step": M * 16,
               "ms_upload_per_step": up / args.steps, "ms_moments_per_step": mo / args.steps,
               "wall_ms_per_step": wall * 1e3 / args.steps}

        forms = None
        evolution = None
        if not args.no_forms:
            forms, evolution = measure_forms(g, torch, m, H, phi, args, stream, hbm_peak)
        batch = None
        if not args.no_batch:
            del x
            batch = measure_batch(g, torch, tmp, stream, hbm_peak)
        cubic = None
        if not args.no_cubic:
            cubic = measure_cubic(g, torch, tmp, stream, hbm_peak)
        precision = None
        precision_msd = None
        if not args.no_precision:
            from gpuqt_b200 import precision_report
            precision = precision_report.report("graphene4m", 20)
            precision_msd = precision_report.msd_report("graphene2m", 20)
        cpu = None
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline_line(reference_dir(src, os.path.join(tmp, "ref")), n)
            if cpu.get("value") is not None:
                cpu["other_workloads"] = cpu_baseline_configs(tmp)

        if rank == 0:
            line = {
                "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded Anderson lattice, random-phase vectors)",
                "config": dict(workload_config(WORKLOAD),
                               step="one KPM moment set (3000 moments)",
                               vectors_per_gpu=1,
                               form="plain FP64 (reference arithmetic)",
                               operator_format=fmt + (f" ({H.n_codes} distinct entries)"
                                                      if coded else ""),
                               parallelism=f"replicas x{world}",
                               l2="inputs larger than L2 (220 MB touched per Chebyshev "
                                  "step)"),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak,
                             "unit": "GB/s", "frac": achieved / hbm_peak,
                             "traffic": traffic, "peak_kind": peak_kind,
                             "kernel": f"k_step<double2,V=1,Z=3,Exact,kCheb,dot> ({fmt})",
                             "bytes_per_launch": bpl},
                "cpu_baseline": cpu,
                "e2e": e2e,
                "gpu_launches": launches,
                "clocks": clocks,
                "forms": forms,
                "evolution": evolution,
                "batch": batch,
                "cubic256": cubic,
                "precision": precision,
                "precision_msd": precision_msd,
            }
            print(json.dumps(line), flush=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
        barrier(world)
        if world > 1:
            import torch.distributed as td
            td.destroy_process_group()


def measure_forms(g, torch, m, H, phi, args, stream, hbm_peak):
    """FP32-storage forms on the same lattice: 1, 16 and 32 vectors per launch, with the
    DOS error of vector 0 against its FP64 moments; and the Bessel evolution."""
    n, M = m.n, m.n_moments
    out = {}
    ev = lambda: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    x64 = g.Vector.from_host(*phi)
    r64, i64 = g.moments(H, x64, x64, M)
    fp64_rate = None
    coded = H.format == g.FORMAT_CODED
    for V in (1, 16, 32):
        vecs = [phi] + [m.initial_state() for _ in range(V - 1)]
        re = np.stack([v[0] for v in vecs])
        im = np.stack([v[1] for v in vecs])
        X = g.Vector.from_host(re, im, nvec=V, precision=g.FP32)
        mu = torch.empty(2 * M * V, dtype=torch.float64, device="cuda")
        # the vector-block shape (vectors per thread) as the autotuner picks it
        shape = g.autotune_nvec(H, g.FP32, 20, [V])[1] if V >= 4 else None
        for _ in range(2):
            g.moments_device(H, X, X, M, mu.data_ptr())
        reps = max(2, min(args.steps, 5))
        a, b = ev()
        a.record(stream)
        for _ in range(reps):
            g.moments_device(H, X, X, M, mu.data_ptr())
        b.record(stream)
        torch.cuda.synchronize()
        s = a.elapsed_time(b) / 1e3
        rate = V * n * M * reps / s
        bpl = fp32_bytes_per_site_vector(V, coded=coded) * V * n
        ach = bpl / (s / (reps * M)) / 1e9
        r32, i32 = g.moments(H, X, X, M)
        r32, i32 = np.atleast_2d(r32)[0], np.atleast_2d(i32)[0]
        out[f"fp32_v{V}"] = {"site_moments_per_s": rate, "vectors_per_launch": V,
                             "achieved_gbs": ach, "frac": ach / hbm_peak,
                             "bytes_per_site_moment": fp32_bytes_per_site_vector(V, coded=coded),
                             "autotune_rate": shape,
                             "dos_err_vs_fp64": dos_error(g, m, (r64, i64), (r32, i32))}
        if V == 16 and coded:
            # the same form on the plain ELL arrays
            H.set_format(g.FORMAT_ELL)
            g.moments_device(H, X, X, M, mu.data_ptr())
            a, b = ev()
            a.record(stream)
            for _ in range(reps):
                g.moments_device(H, X, X, M, mu.data_ptr())
            b.record(stream)
            torch.cuda.synchronize()
            H.set_format(g.FORMAT_CODED)
            s = a.elapsed_time(b) / 1e3
            ach = fp32_bytes_per_site_vector(V, coded=False) * V * n / (s / (reps * M)) / 1e9
            out["fp32_v16_ell"] = {"site_moments_per_s": V * n * M * reps / s,
                                   "vectors_per_launch": V, "achieved_gbs": ach,
                                   "frac": ach / hbm_peak,
                                   "bytes_per_site_moment":
                                       fp32_bytes_per_site_vector(V, coded=False)}

    # The FP32X form (FP32 storage with a BF16 residual), 16 vectors per launch, from
    # the same 16 FP64 vectors; error of vector 0 against its FP64 moments.
    vecs = [phi] + [m.initial_state() for _ in range(15)]
    X16 = g.Vector.from_host(np.stack([v[0] for v in vecs]), np.stack([v[1] for v in vecs]),
                             nvec=16)
    mu = torch.empty(2 * M * 16, dtype=torch.float64, device="cuda")
    for _ in range(2):
        g.moments_device(H, X16, X16, M, mu.data_ptr(), precision=g.FP32X)
    reps = max(2, min(args.steps, 5))
    a, b = ev()
    a.record(stream)
    for _ in range(reps):
        g.moments_device(H, X16, X16, M, mu.data_ptr(), precision=g.FP32X)
    b.record(stream)
    torch.cuda.synchronize()
    s = a.elapsed_time(b) / 1e3
    bx = fp32x_bytes_per_site_vector(16, coded=coded)
    ach = bx * 16 * n * M * reps / s / 1e9
    mh = mu.view(M, 16, 2).cpu().numpy()
    from gpuqt_b200 import precision_report as P
    out["fp32x_v16"] = {"site_moments_per_s": 16 * n * M * reps / s, "vectors_per_launch": 16,
                        "achieved_gbs": ach, "frac": ach / hbm_peak,
                        "bytes_per_site_moment": bx,
                        "dos_err_vs_fp64": P.compare(g, m, (r64, i64),
                                                     (mh[:, 0, 0].copy(), mh[:, 0, 1].copy()))}
    del X16, mu

    def fp64_rate(fmt):
        # plain FP64 rate from a short timed loop, for the ratios
        H.set_format(fmt)
        mu = torch.empty(2 * M, dtype=torch.float64, device="cuda")
        g.moments_device(H, x64, x64, M, mu.data_ptr())
        a, b = ev()
        a.record(stream)
        for _ in range(3):
            g.moments_device(H, x64, x64, M, mu.data_ptr())
        b.record(stream)
        torch.cuda.synchronize()
        return n * M * 3 / (a.elapsed_time(b) / 1e3)

    default = H.format
    rate64 = fp64_rate(default)
    rate64_ell = fp64_rate(g.FORMAT_ELL) if coded else rate64
    H.set_format(default)
    for k in [k for k in out if k.startswith("fp32")]:
        out[k]["speedup_vs_fp64"] = out[k]["site_moments_per_s"] / rate64
    out["fp32x_v16"]["byte_ceiling_vs_fp64"] = (fp64_bytes_per_site(coded=coded) /
                                                fp32x_bytes_per_site_vector(16, coded=coded))
    out["fp64_v1_site_moments_per_s"] = rate64

    # Symmetric moment sets from half the Chebyshev steps (gqt_moments_doubled): the
    # same moments (moments produced per second), equal to the direct ones up to
    # rounding of the largest moment's order.
    def doubled(X, V):
        mu = torch.empty(2 * M * V, dtype=torch.float64, device="cuda")
        g.moments_doubled_device(H, X, M, mu.data_ptr())
        a, b = ev()
        a.record(stream)
        for _ in range(3):
            g.moments_doubled_device(H, X, M, mu.data_ptr())
        b.record(stream)
        torch.cuda.synchronize()
        return V * n * M * 3 / (a.elapsed_time(b) / 1e3)

    def pair_roofline(rate, bytes_per_step):
        # a pair step yields two moments: steps/s = moments/s / 2
        ach = rate / 2 * bytes_per_step / 1e9
        return {"bytes_per_site_step": bytes_per_step, "achieved_gbs": ach,
                "frac": ach / hbm_peak}

    dr, di = g.moments_doubled(H, x64, M)
    rate64_dbl = doubled(x64, 1)
    out["fp64_doubled"] = dict(
        {"site_moments_per_s": rate64_dbl,
         "max_err_vs_direct": float(np.max(np.hypot(dr - r64, di - i64)) /
                                    np.max(np.hypot(r64, i64))),
         "speedup_vs_fp64": rate64_dbl / rate64},
        **pair_roofline(rate64_dbl, fp64_pair_bytes_per_site_step(coded=coded)))
    vecs = [phi] + [m.initial_state() for _ in range(15)]
    X16 = g.Vector.from_host(np.stack([v[0] for v in vecs]), np.stack([v[1] for v in vecs]),
                             nvec=16, precision=g.FP32)
    r32, i32 = g.moments_doubled(H, X16, M)
    rate32_dbl = doubled(X16, 16)
    out["fp32_v16_doubled"] = dict(
        {"site_moments_per_s": rate32_dbl, "vectors_per_launch": 16,
         "dos_err_vs_fp64": dos_error(g, m, (r64, i64), (r32[0], i32[0])),
         "speedup_vs_fp64": rate32_dbl / rate64},
        **pair_roofline(rate32_dbl, fp32_pair_bytes_per_site_vector_step(16, coded=coded)))
    # GQT_FP32R (the recurrence in FP32, FP64 sums) on the same FP32 vectors: same bytes
    # as the FP32-storage form, direct and symmetric loops.
    mu = torch.empty(2 * M * 16, dtype=torch.float64, device="cuda")
    for _ in range(2):
        g.moments_device(H, X16, X16, M, mu.data_ptr(), precision=g.FP32R)
    a, b = ev()
    a.record(stream)
    for _ in range(3):
        g.moments_device(H, X16, X16, M, mu.data_ptr(), precision=g.FP32R)
    b.record(stream)
    torch.cuda.synchronize()
    rate_r = 16 * n * M * 3 / (a.elapsed_time(b) / 1e3)
    mh = mu.view(M, 16, 2).cpu().numpy()
    br = fp32_bytes_per_site_vector(16, coded=coded)
    ach = br * rate_r / 1e9
    out["fp32r_v16"] = {"site_moments_per_s": rate_r, "vectors_per_launch": 16,
                        "achieved_gbs": ach, "frac": ach / hbm_peak,
                        "bytes_per_site_moment": br,
                        "dos_err_vs_fp64": dos_error(g, m, (r64, i64),
                                                     (mh[:, 0, 0].copy(), mh[:, 0, 1].copy())),
                        "speedup_vs_fp64": rate_r / rate64}
    g.moments_doubled_device(H, X16, M, mu.data_ptr(), precision=g.FP32R)
    a, b = ev()
    a.record(stream)
    for _ in range(3):
        g.moments_doubled_device(H, X16, M, mu.data_ptr(), precision=g.FP32R)
    b.record(stream)
    torch.cuda.synchronize()
    rate_rd = 16 * n * M * 3 / (a.elapsed_time(b) / 1e3)
    mh = mu.view(M, 16, 2).cpu().numpy()
    out["fp32r_v16_doubled"] = dict(
        {"site_moments_per_s": rate_rd, "vectors_per_launch": 16,
         "dos_err_vs_fp64": dos_error(g, m, (r64, i64), (mh[:, 0, 0].copy(),
                                                         mh[:, 0, 1].copy())),
         "speedup_vs_fp64": rate_rd / rate64},
        **pair_roofline(rate_rd, fp32_pair_bytes_per_site_vector_step(16, coded=coded)))
    del X16, mu
    ach = fp64_bytes_per_site(coded=False) * rate64_ell / 1e9
    out["fp64_v1_ell"] = {"site_moments_per_s": rate64_ell, "achieved_gbs": ach,
                          "frac": ach / hbm_peak,
                          "bytes_per_site_moment": fp64_bytes_per_site(coded=False)}
    ach = fp64_bytes_per_site(coded=coded) * rate64 / 1e9
    out["fp64_v1"] = {"site_moments_per_s": rate64, "achieved_gbs": ach,
                      "frac": ach / hbm_peak,
                      "bytes_per_site_moment": fp64_bytes_per_site(coded=coded)}

    # The target ratio, like for like: batched FP32 storage over plain FP64 in the
    # same loop (direct over direct, doubled over doubled), each next to the ratio of
    # the two forms' byte models, which bounds it while both are HBM-bound.
    d32 = out["fp32_v16"]
    ceil_direct = fp64_bytes_per_site(coded=coded) / fp32_bytes_per_site_vector(16, coded=coded)
    ceil_dbl = (fp64_pair_bytes_per_site_step(coded=coded) /
                fp32_pair_bytes_per_site_vector_step(16, coded=coded))
    ratio_direct = d32["site_moments_per_s"] / rate64
    ratio_dbl = rate32_dbl / rate64_dbl
    out["target_ratios"] = {
        "target": "batched FP32 >= 3x plain FP64 site-moments/s, both >= 0.70 of HBM "
                  "roofline, <= 1e-6 error",
        "speedup_direct": ratio_direct, "byte_ceiling_direct": ceil_direct,
        "speedup_doubled": ratio_dbl, "byte_ceiling_doubled": ceil_dbl,
        "speedup_fp32_doubled_over_fp64_direct": rate32_dbl / rate64,
        "frac_fp64_direct": out["fp64_v1"]["frac"], "frac_fp32_v16_direct": d32["frac"],
        "frac_fp64_doubled": out["fp64_doubled"]["frac"],
        "frac_fp32_v16_doubled": out["fp32_v16_doubled"]["frac"],
        "dos_err_fp32_v16": d32["dos_err_vs_fp64"],
        "speedup_fp32x_v16_direct": out["fp32x_v16"]["speedup_vs_fp64"],
        "frac_fp32x_v16_direct": out["fp32x_v16"]["frac"],
        "speedup_fp32r_direct": out["fp32r_v16"]["site_moments_per_s"] / rate64,
        "speedup_fp32r_doubled": out["fp32r_v16_doubled"]["site_moments_per_s"] / rate64_dbl,
        "speedup_fp32r_doubled_over_fp64_direct":
            out["fp32r_v16_doubled"]["site_moments_per_s"] / rate64,
        "frac_fp32r_v16_direct": out["fp32r_v16"]["frac"],
        "frac_fp32r_v16_doubled": out["fp32r_v16_doubled"]["frac"],
        "dos_err_fp32r_v16": out["fp32r_v16"]["dos_err_vs_fp64"],
        "met_like_for_like": bool(max(ratio_direct, ratio_dbl,
                                      out["fp32r_v16"]["site_moments_per_s"] / rate64,
                                      out["fp32r_v16_doubled"]["site_moments_per_s"] /
                                      rate64_dbl) >= 3.0 and
                                  d32["frac"] >= 0.7 and out["fp64_v1"]["frac"] >= 0.7),
        "note": "while both forms are HBM-bound the like-for-like ratio is capped by "
                "the byte models (byte_ceiling_*): FP32 storage keeps four 8-byte vector "
                "streams per site-vector-moment (three in a doubled step) against 75 B "
                "(59 B) for the coded FP64 step"}
    # Bessel evolution of one MSD step (1 fs): evolve and evolvex, FP64.
    dt = m.time_step[0] * m.energy_max
    st = x64.clone()
    g.evolve(H, 1, dt, st)
    g.evolvex(H, 1, dt, st)
    reps = 5
    a, b = ev()
    before = g.launch_count()
    a.record(stream)
    for _ in range(reps):
        g.evolve(H, 1, dt, st)
    b.record(stream)
    # apply and the 0/1 term precede the series
    terms = (g.launch_count() - before) // reps - 2
    c, d = ev()
    c.record(stream)
    for _ in range(reps):
        g.evolvex(H, 1, dt, st)
    d.record(stream)
    torch.cuda.synchronize()
    ms_e, ms_x = a.elapsed_time(b) / reps, c.elapsed_time(d) / reps
    # Per-term algorithmic bytes over the series (the apply and 0/1 terms ride along).
    gb_e = terms * n * cheb2_bytes_per_site(coded=coded) / (ms_e / 1e3) / 1e9
    gb_x = terms * n * cheb2x_bytes_per_site(coded=coded) / (ms_x / 1e3) / 1e9
    evolution = {"dt_scaled": dt, "bessel_terms": terms, "ms_evolve": ms_e,
                 "ms_evolvex": ms_x,
                 "k_cheb2": {"bytes_per_site_term": cheb2_bytes_per_site(coded=coded),
                             "achieved_gbs": gb_e, "frac": gb_e / hbm_peak},
                 "k_cheb2x": {"bytes_per_site_term": cheb2x_bytes_per_site(coded=coded),
                              "achieved_gbs": gb_x, "frac": gb_x / hbm_peak}}
    return out, evolution


def measure_cubic(g, torch, tmp, stream, hbm_peak, vectors=16):
    """The 3D Anderson lattice near its transition (cubic 256^3 = 16,777,216 sites, z = 6,
    t = -1, W = 16.5, seed 13, E_max 15, 4000 moments): plain FP64 (one vector) and FP32
    storage (16 vectors per launch) side by side. One DOS moment set each, timed whole;
    a VAC correlation step (current operator, moment set, two evolutions; the moment
    set's time is the DOS set's) and an MSD step (evolvex, two evolutions, moment set),
    composed from timed parts; the FP32 error against FP64 on the first vector for the
    DOS and for the VAC moment sets of the first two correlation steps."""
    from gpuqt_b200 import precision_report as P
    from gpuqt_b200 import workloads as W
    name = "cubic256"
    m = g.Model.load(W.config_dir(tmp, name))
    H = g.Hamiltonian(m)
    n, M = m.n, m.n_moments
    coded = H.format == g.FORMAT_CODED
    z = 6

    def timed(fn, reps=1, warm=True):
        if warm:
            fn()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    vecs = [m.initial_state() for _ in range(vectors)]
    x64 = g.Vector.from_host(*vecs[0])
    mu64 = torch.empty(2 * M, dtype=torch.float64, device="cuda")
    ms64 = timed(lambda: g.moments_device(H, x64, x64, M, mu64.data_ptr()))
    r64, i64 = g.moments(H, x64, x64, M)
    X = g.Vector.from_host(np.stack([v[0] for v in vecs]), np.stack([v[1] for v in vecs]),
                           nvec=vectors, precision=g.FP32)
    mu32 = torch.empty(2 * M * vectors, dtype=torch.float64, device="cuda")
    # the vector-block shape as the autotuner picks it on this lattice
    g.autotune_nvec(H, g.FP32, 20, [vectors])
    ms32 = timed(lambda: g.moments_device(H, X, X, M, mu32.data_ptr()))
    mu_h = mu32.view(M, vectors, 2).cpu().numpy()
    dos = P.compare(g, m, (r64, i64), (mu_h[:, 0, 0].copy(), mu_h[:, 0, 1].copy()))
    b64 = fp64_bytes_per_site(z=z, coded=coded)
    b32 = fp32_bytes_per_site_vector(vectors, z=z, coded=coded)
    rate64 = n * M / (ms64 / 1e3)
    rate32 = vectors * n * M / (ms32 / 1e3)

    # Parts of the correlation steps (FP64 state; the FP32 form's 16-vector state).
    dt = m.time_step[0] * m.energy_max
    tmp64 = g.Vector(n)
    tmp32 = g.Vector(n, nvec=vectors, precision=g.FP32)
    before = g.launch_count()
    g.evolve(H, 1, dt, x64)
    terms = g.launch_count() - before - 2
    parts = {
        "fp64": {"current": timed(lambda: g.apply_current(H, x64, tmp64), 3),
                 "evolve": timed(lambda: g.evolve(H, 1, dt, x64), 3),
                 "evolvex": timed(lambda: g.evolvex(H, 1, dt, x64), 3)},
        "fp32_v16": {"current": timed(lambda: g.apply_current(H, X, tmp32), 3),
                     "evolve": timed(lambda: g.evolve(H, 1, dt, X), 2),
                     "evolvex": timed(lambda: g.evolvex(H, 1, dt, X), 2)},
    }
    del tmp32

    def form(rate, ms_set, bytes_sm, V, p):
        ach = rate * bytes_sm / 1e9
        vac = p["current"] + ms_set + 2 * p["evolve"]
        msd = p["evolvex"] + 2 * p["evolve"] + ms_set
        return {"vectors_per_launch": V, "dos_site_moments_per_s": rate, "ms_dos_set": ms_set,
                "bytes_per_site_moment": bytes_sm, "achieved_gbs": ach, "frac": ach / hbm_peak,
                "ms_current": p["current"], "ms_evolve": p["evolve"],
                "ms_evolvex": p["evolvex"], "ms_vac_step": vac, "ms_msd_step": msd,
                "vac_step_site_moments_per_s": V * n * M / (vac / 1e3),
                "msd_step_site_moments_per_s": V * n * M / (msd / 1e3)}

    e64 = parts["fp64"]
    gb_e = terms * n * cheb2_bytes_per_site(z=z, coded=coded) / (e64["evolve"] / 1e3) / 1e9
    gb_x = terms * n * cheb2x_bytes_per_site(z=z, coded=coded) / (e64["evolvex"] / 1e3) / 1e9
    out = {
        "config": dict(workload_config(name), vectors=vectors,
                       note="VAC/MSD step times are the timed moment set plus the timed "
                            "current, evolve and evolvex of that form"),
        "fp64": form(rate64, ms64, b64, 1, parts["fp64"]),
        "fp32_v16": form(rate32, ms32, b32, vectors, parts["fp32_v16"]),
        "speedup_dos": rate32 / rate64,
        "byte_ceiling_dos": b64 / b32,
        "evolution_fp64": {"dt_scaled": dt, "bessel_terms": terms,
                           "k_cheb2_frac": gb_e / hbm_peak, "k_cheb2_gbs": gb_e,
                           "k_cheb2x_frac": gb_x / hbm_peak, "k_cheb2x_gbs": gb_x},
        "dos_err_fp32_vs_fp64": dos,
    }
    # GQT_FP32R on the initial FP32 vectors again (the evolution parts above changed X):
    # the DOS moment set, direct and symmetric
    X.upload(np.stack([v[0] for v in vecs]), np.stack([v[1] for v in vecs]))
    msr = timed(lambda: g.moments_device(H, X, X, M, mu32.data_ptr(), precision=g.FP32R))
    mu_h = mu32.view(M, vectors, 2).cpu().numpy()
    rate_r = vectors * n * M / (msr / 1e3)
    msd_r = timed(lambda: g.moments_doubled_device(H, X, M, mu32.data_ptr(),
                                                   precision=g.FP32R))
    rate_rd = vectors * n * M / (msd_r / 1e3)
    ach = rate_r * b32 / 1e9
    bp = fp32_pair_bytes_per_site_vector_step(vectors, z=z, coded=coded)
    out["fp32r_v16"] = {"vectors_per_launch": vectors, "dos_site_moments_per_s": rate_r,
                        "ms_dos_set": msr, "bytes_per_site_moment": b32,
                        "achieved_gbs": ach, "frac": ach / hbm_peak,
                        "dos_err_vs_fp64": P.compare(g, m, (r64, i64),
                                                     (mu_h[:, 0, 0].copy(),
                                                      mu_h[:, 0, 1].copy())),
                        "doubled_site_moments_per_s": rate_rd,
                        "doubled_frac": rate_rd / 2 * bp / 1e9 / hbm_peak,
                        "speedup_dos": rate_r / rate64}
    del X, mu32
    # VAC moment sets of the first two correlation steps, FP32 storage against FP64
    # (vector 0; states evolved in FP64, as the library's FP32 form does).
    a = P.vac_moments(g, m, H, vecs[0], g.FP64, 2)
    b = P.vac_moments(g, m, H, vecs[0], g.FP32, 2)
    per = [P.compare(g, m, a[k], b[k]) for k in range(2)]
    out["vac_err_fp32_vs_fp64"] = {k: max(q[k] for q in per) for k in per[0]}
    out["vac_err_steps"] = 2
    return out


def measure_batch(g, torch, tmp, stream, hbm_peak, vectors=64, moments=2000):
    """The realisation batch: 8 uneven square lattices in one block-diagonal operator,
    `vectors` random-phase vectors each, FP32 storage, vectors per launch chosen by the
    autotuner; one moment set per vector block. Reports the rate over the whole job and
    the DOS error of one vector against its FP64 moments."""
    from gpuqt_b200 import workloads as W
    dirs = W.batch_dirs(os.path.join(tmp, "batch"), moments=moments)
    models = [g.Model.load(d) for d in dirs]
    B = g.Hamiltonian.batch(models)
    best, rates = g.autotune_nvec(B, g.FP32, 20, [4, 8, 16, 32])
    V = best
    tile = B.batch_tile
    # The tile sizes at the chosen vector count, as the autotuner saw them (a short
    # probe each; the autotuner's choice is restored afterwards).
    tile_rates = {}
    Xp = g.Vector(B.n, nvec=V, precision=g.FP32)
    mup = torch.empty(2 * 20 * len(models) * V, dtype=torch.float64, device="cuda")
    for t in (256, 512, 1024):
        B.set_batch_tile(t)
        g.moments_device(B, Xp, Xp, 20, mup.data_ptr())
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(3):
            g.moments_device(B, Xp, Xp, 20, mup.data_ptr())
        b.record(stream)
        torch.cuda.synchronize()
        tile_rates[t] = 3 * V * sum(m.n for m in models) * 20 / (a.elapsed_time(b) / 1e3)
    B.set_batch_tile(tile)
    del Xp, mup
    rng = np.random.default_rng(11)
    sites = sum(m.n for m in models)
    X = g.Vector(B.n, nvec=V, precision=g.FP32)
    mu = torch.empty(2 * moments * len(models) * V, dtype=torch.float64, device="cuda")

    def fill():
        per = []
        for m in models:
            ph = rng.uniform(0.0, 2 * np.pi, size=(V, m.n))
            per.append((np.cos(ph), np.sin(ph)))
        X.upload(*B.scatter(per))
        return per

    per0 = fill()
    g.moments_device(B, X, X, moments, mu.data_ptr())  # warm-up, graph capture
    torch.cuda.synchronize()
    blocks = vectors // V
    total_ms = 0.0
    for k in range(blocks):
        if k:
            fill()  # host generation and upload stay outside the timed kernels
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        g.moments_device(B, X, X, moments, mu.data_ptr())
        b.record(stream)
        torch.cuda.synchronize()
        total_ms += a.elapsed_time(b)
    rate = vectors * sites * moments / (total_ms / 1e3)
    bytes_site_moment = (fp32_bytes_per_site_vector(V, z=4, coded=B.format == g.FORMAT_CODED)
                         * B.n / sites)
    # DOS error of vector 0 of realisation 0 against its FP64 moments
    X.upload(*B.scatter(per0))
    r32, i32 = g.moments(B, X, X, moments)
    m0 = models[0]
    H0 = g.Hamiltonian(m0)
    x0 = g.Vector.from_host(per0[0][0][0], per0[0][1][0])
    r64, i64 = g.moments(H0, x0, x0, moments)
    err = dos_error(g, m0, (r64, i64), (r32[0, 0], i32[0, 0]))
    # The same batch as symmetric moment sets from half the steps (gqt_moments_doubled).
    g.moments_doubled_device(B, X, moments, mu.data_ptr())
    torch.cuda.synchronize()
    dbl_ms = 0.0
    for k in range(blocks):
        if k:
            fill()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        g.moments_doubled_device(B, X, moments, mu.data_ptr())
        b.record(stream)
        torch.cuda.synchronize()
        dbl_ms += a.elapsed_time(b)
    X.upload(*B.scatter(per0))
    q32, j32 = g.moments_doubled(B, X, moments)
    dbl_err = dos_error(g, m0, (r64, i64), (q32[0, 0], j32[0, 0]))
    del X, mu

    # The FP32R form (FP32 recurrence, the staged batch step with each model's windows):
    # 32 vectors per launch direct, 16 for symmetric sets; the same vectors and checks.
    def fp32r(Vr, doubled):
        Xr = g.Vector(B.n, nvec=Vr, precision=g.FP32)
        mur = torch.empty(2 * moments * len(models) * Vr, dtype=torch.float64, device="cuda")
        if doubled:
            run = lambda: g.moments_doubled_device(B, Xr, moments, mur.data_ptr(),
                                                   precision=g.FP32R)
        else:
            run = lambda: g.moments_device(B, Xr, Xr, moments, mur.data_ptr(),
                                           precision=g.FP32R)
        Xr.upload(*B.scatter([(p[0][:Vr], p[1][:Vr]) for p in per0]))
        run()
        torch.cuda.synchronize()
        ms = 0.0
        for k in range(vectors // Vr):
            per = []
            for m in models:
                ph = rng.uniform(0.0, 2 * np.pi, size=(Vr, m.n))
                per.append((np.cos(ph), np.sin(ph)))
            Xr.upload(*B.scatter(per))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            run()
            b.record(stream)
            torch.cuda.synchronize()
            ms += a.elapsed_time(b)
        r = vectors * sites * moments / (ms / 1e3)
        Xr.upload(*B.scatter([(p[0][:Vr], p[1][:Vr]) for p in per0]))
        if doubled:
            qr, qi = g.moments_doubled(B, Xr, moments, precision=g.FP32R)
            bps = fp32_pair_bytes_per_site_vector_step(Vr, z=4) * B.n / sites
            ach = r / 2 * bps / 1e9
        else:
            qr, qi = g.moments(B, Xr, Xr, moments, precision=g.FP32R)
            bps = fp32_bytes_per_site_vector(Vr, z=4) * B.n / sites
            ach = r * bps / 1e9
        stages, slots = B.stage_plan(Vr, g.FP32R, symmetric=doubled)
        return {"site_moments_per_s": r, "vectors_per_launch": Vr, "ms_total": ms,
                "bytes_per_site_moment" if not doubled else "bytes_per_site_step": bps,
                "achieved_gbs": ach, "frac": ach / hbm_peak,
                "dos_err_vs_fp64": dos_error(g, m0, (r64, i64), (qr[0, 0], qi[0, 0])),
                "stages": stages, "window_slots": slots}

    fp32r_direct = None
    if B.format == g.FORMAT_CODED:
        # the vectors per launch as the autotuner picks them for this form
        vr, vr_rates = g.autotune_nvec(B, g.FP32R, 20, [16, 32])
        fp32r_direct = dict(fp32r(vr, False), autotune_rates=vr_rates)
    fp32r_doubled = fp32r(16, True) if B.format == g.FORMAT_CODED else None
    return {"realisations": [[m.n, round(m.energy_max, 4)] for m in models],
            "doubled": {"site_moments_per_s": vectors * sites * moments / (dbl_ms / 1e3),
                        "ms_total": dbl_ms, "dos_err_vs_fp64": dbl_err},
            "sites": sites, "padded_sites": B.n, "vectors": vectors, "moments": moments,
            "operator_format": "coded" if B.format == g.FORMAT_CODED else "ell",
            "autotuned_vectors_per_launch": V, "autotune_rates": rates,
            "autotuned_tile_sites": tile, "tile_rates_at_best_vectors": tile_rates,
            "site_moments_per_s": rate, "ms_total": total_ms,
            "achieved_gbs": rate * bytes_site_moment / 1e9,
            "frac": rate * bytes_site_moment / 1e9 / hbm_peak,
            "dos_err_vs_fp64": err,
            "fp32r": fp32r_direct, "fp32r_doubled": fp32r_doubled}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-forms", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-cubic", action="store_true")
    ap.add_argument("--no-precision", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
