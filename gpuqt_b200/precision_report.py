"""Error of the reduced-precision moment forms against the FP64 form on the same inputs.

    python -m gpuqt_b200.precision_report --workload graphene4m --vac-steps 20
    python -m gpuqt_b200.precision_report --workload graphene2m --msd-steps 20

Runs the DOS moment set and the VAC moment sets (src/sigma.cu:278-327), or the MSD
moment sets (src/sigma.cu:331-391), in the FP64 form and in the FP32-storage form;
under "fp32x" in the FP32X form (FP32 storage with a BF16 residual) and under "fp32r"
in the FP32R form (FP32 vectors and hoppings, the recurrence in FP32). The states are
evolved in FP64 in every case; only the moment recurrence changes form. The run takes
the first random-phase vector of the workload (FP32R, which launches 4, 16 or 32
vectors, runs on 4 copies of it and reports the first). Prints one JSON line with, per
quantity: the largest per-moment error relative to the moment (complex modulus), the
largest per-moment error relative to mu_0, and the largest per-energy error of the
damped Chebyshev sum relative to its peak (and relative to the value, over energies
where the value exceeds 1 % of the peak).
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


def _copies(g, v, copies):
    """An FP64 vector of `copies` identical columns holding v (for the forms that launch
    several vectors at once)."""
    re, im = v.download()
    return g.Vector.from_host(np.tile(re, (copies, 1)), np.tile(im, (copies, 1)),
                              nvec=copies)


def _moments(g, model, H, left, right, precision, copies):
    if copies == 1:
        return g.moments(H, left, right, model.n_moments, precision=precision)
    R = _copies(g, right, copies)
    L = R if left is right else _copies(g, left, copies)
    r, i = g.moments(H, L, R, model.n_moments, precision=precision)
    return r[0].copy(), i[0].copy()


def vac_moments(g, model, H, phi, precision, steps, copies=1):
    """VAC moment sets with FP64 states (evolved in FP64) and the recurrence in
    `precision`."""
    left = g.Vector.from_host(*phi)
    right = left.clone()
    lcopy = g.Vector(model.n)
    g.apply_current(H, left, right)
    out = []
    for m in range(steps):
        g.apply_current(H, left, lcopy)
        out.append(_moments(g, model, H, lcopy, right, precision, copies))
        if m < steps - 1:
            dt = model.time_step[m] * model.energy_max
            g.evolve(H, -1, dt, left)
            g.evolve(H, -1, dt, right)
    return out


def msd_moments(g, model, H, phi, precision, steps, copies=1):
    """MSD moment sets <[X, U] phi|T_m|[X, U] phi> with FP64 states, in the order of
    src/sigma.cu:331-391 (time step m + 1 inside the loop), the recurrence in
    `precision`."""
    state = g.Vector.from_host(*phi)
    state_x = state.clone()
    dt = model.time_step[0] * model.energy_max
    g.evolve(H, 1, dt, state)
    g.evolvex(H, 1, dt, state_x)
    out = []
    for m in range(steps):
        out.append(_moments(g, model, H, state_x, state_x, precision, copies))
        if m < steps - 1:
            dt = model.time_step[m + 1] * model.energy_max
            copy = state.clone()
            g.evolvex(H, 1, dt, copy)
            g.evolve(H, 1, dt, state_x)
            state_x.add(copy)
            g.evolve(H, 1, dt, state)
    return out


def _worst(per):
    return {k: max(p[k] for p in per) for k in per[0]}


def _load(workload, moments):
    import gpuqt_b200 as g

    tmp = tempfile.mkdtemp(prefix="gqt_prec_")
    d = W.config_dir(tmp, workload)
    if moments is not None:
        with open(d + "/para.in") as f:
            lines = [l for l in f if not l.startswith("number_of_moments")]
        lines.append(f"number_of_moments {moments}\n")
        with open(d + "/para.in", "w") as f:
            f.writelines(lines)
    return tmp, g.Model.load(d)


def report(workload: str, vac_steps: int, moments: int | None = None,
           fp32x: bool = True, fp32r: bool = True) -> dict:
    import gpuqt_b200 as g

    tmp, m = _load(workload, moments)
    try:
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
        out["vac_steps"] = steps
        out["vac"] = _worst([compare(g, m, a[k], b[k]) for k in range(steps)])
        if fp32x:
            c = vac_moments(g, m, H, phi, g.FP32X, steps)
            out["fp32x"] = {
                "dos": compare(g, m, d64, g.moments(H, x64, x64, m.n_moments,
                                                    precision=g.FP32X)),
                "vac": _worst([compare(g, m, a[k], c[k]) for k in range(steps)])}
        if fp32r:
            c = vac_moments(g, m, H, phi, g.FP32R, steps, copies=4)
            out["fp32r"] = {
                "dos": compare(g, m, d64, _moments(g, m, H, x64, x64, g.FP32R, 4)),
                "vac": _worst([compare(g, m, a[k], c[k]) for k in range(steps)])}
        return out
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def msd_report(workload: str, msd_steps: int, moments: int | None = None) -> dict:
    """The MSD moment sets of the FP32, FP32X and FP32R forms against FP64, worst over
    the steps, per form."""
    import gpuqt_b200 as g

    tmp, m = _load(workload, moments)
    try:
        H = g.Hamiltonian(m)
        phi = m.initial_state()
        steps = min(msd_steps, m.n_steps) if m.n_steps else msd_steps
        a = msd_moments(g, m, H, phi, g.FP64, steps)
        out = {"workload": W.CONFIGS[workload]["description"], "sites": m.n,
               "moments": m.n_moments, "msd_steps": steps}
        for name, prec, copies in (("fp32", g.FP32, 1), ("fp32x", g.FP32X, 1),
                                   ("fp32r", g.FP32R, 4)):
            b = msd_moments(g, m, H, phi, prec, steps, copies)
            out[name] = _worst([compare(g, m, a[k], b[k]) for k in range(steps)])
        return out
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="graphene4m", choices=sorted(W.CONFIGS))
    ap.add_argument("--vac-steps", type=int, default=20)
    ap.add_argument("--msd-steps", type=int, default=0,
                    help="the MSD report of that many steps instead of DOS and VAC")
    ap.add_argument("--moments", type=int, default=None)
    args = ap.parse_args()
    if args.msd_steps:
        print(json.dumps(msd_report(args.workload, args.msd_steps, args.moments)))
    else:
        print(json.dumps(report(args.workload, args.vac_steps, args.moments)))


if __name__ == "__main__":
    main()
