"""A short, fixed run of the KPM moment loop for profilers (ncu) and quick timing.

    python -m gpuqt_b200.profile_case --workload graphene2m --form fp64 --moments 20 --sets 2

Builds the workload's lattice, then runs `sets` moment sets of `moments` moments in
one arithmetic form: fp64 (plain, one vector), fp32v1, or fp32vV (V vectors per
launch, FP32 storage), with the operator in the coded format (the default where the
lattice has one) or in the plain ELL arrays (`--format ell`). With `--doubled` each
set is a symmetric moment set from half the Chebyshev steps (gqt_moments_doubled: the
step kernels in pair mode); the rate counts the moments produced. With `--evolve`
each set is instead one evolve and one evolvex of the workload's first time step
(the Bessel-series kernels k_cheb2 and k_cheb2x), timed separately. Prints one JSON
line with the measured rate.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import tempfile

import numpy as np

from . import workloads as W


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="graphene2m", choices=sorted(W.CONFIGS) + ["batch"])
    ap.add_argument("--form", default="fp64")
    ap.add_argument("--moments", type=int, default=20)
    ap.add_argument("--sets", type=int, default=2)
    ap.add_argument("--format", default="default", choices=["default", "ell", "coded"])
    ap.add_argument("--autotune", action="store_true",
                    help="let the autotuner pick the shape for this vector count first")
    ap.add_argument("--doubled", action="store_true",
                    help="symmetric moment sets from half the steps (pair-mode kernels)")
    ap.add_argument("--evolve", action="store_true",
                    help="time evolve and evolvex of one time step instead of moments")
    ap.add_argument("--loop", type=int, default=0,
                    help="FP64 moment loop: 0 step by step, S >= 2 wavefront windows of S")
    ap.add_argument("--chunk", type=int, default=0,
                    help="sites per chunk of the wavefront loop (0: the default)")
    ap.add_argument("--staging", type=int, default=None,
                    help="staged FP32 step: -1 off, 0 automatic, 1 as many stages as fit, 2..4")
    args = ap.parse_args()

    import torch

    import gpuqt_b200 as g

    mo = re.fullmatch(r"(fp64|fp32r|fp32)(?:v(\d+))?", args.form)
    if not mo:
        raise SystemExit(f"unknown form {args.form}")
    prec = g.FP64 if mo.group(1) == "fp64" else g.FP32  # storage of the vectors
    run_prec = g.FP32R if mo.group(1) == "fp32r" else None  # form of the recurrence
    V = int(mo.group(2) or 1)
    tmp = tempfile.mkdtemp(prefix="gqt_prof_")
    try:
        if args.workload == "batch":
            models = [g.Model.load(d) for d in W.batch_dirs(tmp, moments=args.moments)]
            H = g.Hamiltonian.batch(models)
            rng = np.random.default_rng(1)
            per = []
            for mm in models:
                ph = rng.uniform(0.0, 2 * np.pi, size=(V, mm.n))
                per.append((np.cos(ph), np.sin(ph)))
            X = g.Vector.from_host(*H.scatter(per), nvec=V, precision=prec)
            sites = sum(mm.n for mm in models)
        else:
            m = g.Model.load(W.config_dir(tmp, args.workload))
            H = g.Hamiltonian(m)
            vecs = [m.initial_state() for _ in range(V)]
            X = g.Vector.from_host(np.stack([v[0] for v in vecs]),
                                   np.stack([v[1] for v in vecs]), nvec=V, precision=prec)
            sites = m.n
        if args.format != "default":
            H.set_format(g.FORMAT_ELL if args.format == "ell" else g.FORMAT_CODED)
        if args.loop:
            H.set_loop(args.loop, args.chunk)
        if args.staging is not None:
            H.set_staging(args.staging)
        tuned = None
        if args.autotune:
            tuned = g.autotune_nvec(H, prec, 20, [V])[1]
        R = getattr(H, "n_real", 1)
        mu = torch.empty(2 * args.moments * V * R, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream()
        g.set_stream(stream.cuda_stream)
        if args.evolve:
            if args.workload == "batch":
                raise SystemExit("--evolve needs a single model")
            dt = float(m.time_step[0]) * m.energy_max
            ev = lambda: (torch.cuda.Event(enable_timing=True),
                          torch.cuda.Event(enable_timing=True))
            g.evolve(H, 1, dt, X)
            g.evolvex(H, 1, dt, X)
            before = g.launch_count()
            a, b = ev()
            a.record(stream)
            for _ in range(args.sets):
                g.evolve(H, 1, dt, X)
            b.record(stream)
            terms = (g.launch_count() - before) // args.sets - 2
            c, d = ev()
            c.record(stream)
            for _ in range(args.sets):
                g.evolvex(H, 1, dt, X)
            d.record(stream)
            torch.cuda.synchronize()
            print(json.dumps({"workload": args.workload, "form": args.form, "sites": sites,
                              "format": "coded" if H.format == g.FORMAT_CODED else "ell",
                              "dt_scaled": dt, "bessel_terms": terms, "sets": args.sets,
                              "ms_evolve": a.elapsed_time(b) / args.sets,
                              "ms_evolvex": c.elapsed_time(d) / args.sets}))
            return
        if args.doubled:
            def one():
                g.moments_doubled_device(H, X, args.moments, mu.data_ptr(), precision=run_prec)
        else:
            def one():
                g.moments_device(H, X, X, args.moments, mu.data_ptr(), precision=run_prec)
        one()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.sets):
            one()
        b.record(stream)
        torch.cuda.synchronize()
        s = a.elapsed_time(b) / 1e3
        print(json.dumps({"workload": args.workload, "form": args.form, "sites": sites,
                          "format": "coded" if H.format == g.FORMAT_CODED else "ell",
                          "n_codes": H.n_codes,
                          "moments": args.moments, "sets": args.sets, "autotune": tuned,
                          "doubled": args.doubled, "loop": list(H.loop),
                          "staging": H.staging[0], "stage_windows": H.staging[1],
                          "site_moments_per_s": V * sites * args.moments * args.sets / s}))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    main()
