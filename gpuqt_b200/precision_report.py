"""Error of the FP32-storage form against the FP64 form on the same inputs.

    python -m gpuqt_b200.precision_report --workload graphene4m --vac-steps 20

Runs the DOS moment set and the VAC moment sets (src/sigma.cu:278-327) in the FP64
form and in the FP32-storage form (and, under "fp32x", in the FP32X form: FP32 storage
with a BF16 residual) for the first random-phase vector of the workload and prints
one JSON line with, per quantity: the largest per-moment error relative to the moment
(complex modulus), the largest per-moment error relative to mu_0, and the largest
per-energy error of the damped Chebyshev sum relative to its peak (and relative to the
value, over energies where the value exceeds 1 % of the peak).
"""
from __future__ import annotations

import argparse
import json
import shutil
import tempfile

import numpy as np

from . import workloads as W


def compare(g, model, mu64, mu32) -> dict:
    r64, i64 = mu64
    r32, i32 = mu32
    num = np.hypot(r32 - r64, i32 - i64)
    den = np.hypot(r64, i64)
    d64 = g.chebyshev_summation(r64, i64, model.energy, model.energy_max, model.volume)
    d32 = g.chebyshev_summation(r32, i32, model.energy, model.energy_max, model.volume)
    fin = np.isfinite(d64)
    err = np.abs(d32 - d64)[fin]
    ref = np.abs(d64[fin])
    band = ref > 0.01 * ref.max()
    return {"moment_rel_max": float(np.max(num / np.maximum(den, 1e-300))),
            "moment_rel_mu0_max": float(np.max(num) / abs(r64[0] + 1j * i64[0])),
            "energy_rel_peak_max": float(err.max() / ref.max()),
            "energy_rel_in_band_max": float(np.max(err[band] / ref[band]))}


def vac_moments(g, model, H, phi, precision, steps):
    """VAC moment sets with FP64 states (evolved in FP64) and the recurrence in
    `precision` (the library's FP32 form keeps the states FP64)."""
    left = g.Vector.from_host(*phi)
    right = left.clone()
    lcopy = g.Vector(model.n)
    g.apply_current(H, left, right)
    out = []
    for m in range(steps):
        g.apply_current(H, left, lcopy)
        out.append(g.moments(H, right, lcopy, model.n_moments, precision=precision))
        if m < steps - 1:
            dt = model.time_step[m] * model.energy_max
            g.evolve(H, -1, dt, left)
            g.evolve(H, -1, dt, right)
    return out


def report(workload: str, vac_steps: int, moments: int | None = None,
           fp32x: bool = True) -> dict:
    import gpuqt_b200 as g

    tmp = tempfile.mkdtemp(prefix="gqt_prec_")
    try:
        d = W.config_dir(tmp, workload)
        if moments is not None:
            with open(d + "/para.in") as f:
                lines = [l for l in f if not l.startswith("number_of_moments")]
            lines.append(f"number_of_moments {moments}\n")
            with open(d + "/para.in", "w") as f:
                f.writelines(lines)
        m = g.Model.load(d)
        H = g.Hamiltonian(m)
        phi = m.initial_state()
        out = {"workload": W.CONFIGS[workload]["description"], "sites": m.n,
               "moments": m.n_moments}
        x64 = g.Vector.from_host(*phi)
        x32 = g.Vector.from_host(*phi, precision=g.FP32)
        d64 = g.moments(H, x64, x64, m.n_moments)
        out["dos"] = compare(g, m, d64, g.moments(H, x32, x32, m.n_moments))
        steps = min(vac_steps, m.n_steps) if m.n_steps else vac_steps
        a = vac_moments(g, m, H, phi, g.FP64, steps)
        b = vac_moments(g, m, H, phi, g.FP32, steps)
        per = [compare(g, m, a[k], b[k]) for k in range(steps)]
        out["vac_steps"] = steps
        out["vac"] = {k: max(p[k] for p in per) for k in per[0]}
        if fp32x:
            c = vac_moments(g, m, H, phi, g.FP32X, steps)
            per = [compare(g, m, a[k], c[k]) for k in range(steps)]
            out["fp32x"] = {
                "dos": compare(g, m, d64, g.moments(H, x64, x64, m.n_moments,
                                                    precision=g.FP32X)),
                "vac": {k: max(p[k] for p in per) for k in per[0]}}
        return out
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="graphene4m", choices=sorted(W.CONFIGS))
    ap.add_argument("--vac-steps", type=int, default=20)
    ap.add_argument("--moments", type=int, default=None)
    args = ap.parse_args()
    print(json.dumps(report(args.workload, args.vac_steps, args.moments)))


if __name__ == "__main__":
    main()
