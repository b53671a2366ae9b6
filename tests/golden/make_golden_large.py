"""Golden fixtures at the benchmark sizes, from the reference's own build.

The small fixtures (make_golden.py) pin every kernel bit for bit on lattices of up to
65,536 sites. This script pins the same results at the sizes of the benchmark
workloads, where the grid-stride loops hand several elements to every thread:

  graphene2m   honeycomb graphene 2,097,152 sites (4-orbital cell x 1024x512), t = -2.7,
               W = 1.0 (seed 3), E_max 8.7: all 3000 DOS moments, and the MSD moment
               sets of 2 Bessel steps of 1 fs (find_msd, src/sigma.cu:331-391)
  graphene4m   the same cell x 1024x1024 = 4,194,304 sites, W = 1.5 (seed 5), E_max 9.0:
               the first 500 DOS moments
  cubic256     cubic 256^3 = 16,777,216 sites, z = 6, W = 16.5 (seed 13), E_max 15:
               the first 200 DOS moments

For each it writes the input directory (tests/golden/inputs/<name>/, a few text files),
runs the reference build (oracle/_ref/ref_driver, `make -C oracle ref`) on a copy
without this library's seed keywords (the seed goes to the driver, which reseeds the
reference's one generator before its Anderson draws; with no vacancies that is the
stream the library's `seed` keyword starts), and stores under tests/golden/ref/<name>/:

  moments.txt   the reference's find_moments_chebyshev moments (%.17g)
  msdmom.npz    graphene2m only: the MSD moment sets, one row per time step
  model.json    n, z, E_max, volume and SHA-256 digests of the reference's ELL arrays
                (neighbour counts, row-major neighbour list, hoppings, xx with entries
                past a row's length zeroed, and the potential)

Needs the reference checkout (GQT_REFERENCE, or a `reference` directory beside this
repository) and a few minutes of CPU; run it here and commit the results:

    python tests/golden/make_golden_large.py [name ...]
"""
from __future__ import annotations

import hashlib
import json
import os
import shutil
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402
from gpuqt_b200 import workloads as W  # noqa: E402

INPUTS = os.path.join(HERE, "inputs")
OUT = os.path.join(HERE, "ref")

# name: (workload, moments, MSD steps of 1 fs or 0)
LARGE = {
    "graphene2m": ("graphene2m", 3000, 2),
    "graphene4m": ("graphene4m", 500, 0),
    "cubic256": ("cubic256", 200, 0),
}


def input_dir(name: str) -> str:
    """Write the input directory of a large fixture (idempotent) and return it."""
    workload, moments, msd = LARGE[name]
    c = dict(W.CONFIGS[workload])
    c.pop("description")
    kind, cells = c.pop("kind"), c.pop("cells")
    c["moments"] = moments
    c["time_step"] = [W.FS] * max(msd, 1)
    c["calculate"] = ("msd",) if msd else ()
    d = os.path.join(INPUTS, name)
    return W.write_input_dir(d, kind, cells, **c)


def seed_of(d: str) -> int:
    with open(os.path.join(d, "para.in")) as f:
        for line in f:
            p = line.split()
            if p and p[0] == "seed":
                return int(p[1])
    raise ValueError("no seed keyword in " + d)


def ell_digests(nn, nl, pot, hr, hi, xx, z: int) -> dict:
    """SHA-256 of each ELL array in the reference's host layout ([i * z + m]), entries
    past a row's length set to zero (their content is not part of the model)."""
    n = nn.size
    mask = np.arange(z)[None, :] < nn[:, None]

    def h(a, dtype):
        a = np.ascontiguousarray(a, dtype=dtype).reshape(n, -1).copy()
        if a.shape[1] == z:
            a[~mask] = 0
        return hashlib.sha256(a.tobytes()).hexdigest()

    return {"neighbor_number": h(nn, np.int32), "neighbor_list": h(nl, np.int32),
            "potential": h(pot, np.float64), "hopping_real": h(hr, np.float64),
            "hopping_imag": h(hi, np.float64), "xx": h(xx, np.float64)}


def ref_copy(d: str, tmp: str) -> str:
    rd = os.path.join(tmp, os.path.basename(d))
    if os.path.isdir(rd):
        shutil.rmtree(rd)
    shutil.copytree(d, rd)
    with open(os.path.join(d, "para.in")) as f:
        lines = [l for l in f if l.split() and l.split()[0] not in
                 ("seed", "disorder_seed", "phase_seed")]
    with open(os.path.join(rd, "para.in"), "w") as f:
        f.writelines(lines)
    return rd


def make(name: str, tmp: str) -> None:
    d = input_dir(name)
    seeds = (seed_of(d), -1)
    rd = ref_copy(d, tmp)
    o = os.path.join(OUT, name)
    os.makedirs(o, exist_ok=True)
    t0 = time.time()
    ell = oracle.ref_ell(rd, os.path.join(tmp, "ell.bin"), seeds=seeds)
    os.remove(os.path.join(tmp, "ell.bin"))
    meta = {"n": ell.n, "z": ell.max_neighbor, "energy_max": ell.energy_max,
            "volume": ell.volume,
            "sha256": ell_digests(ell.neighbor_number, ell.neighbor_list, ell.potential,
                                  ell.hopping_real, ell.hopping_imag, ell.xx,
                                  ell.max_neighbor)}
    del ell
    with open(os.path.join(o, "model.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print(name, "model", f"{time.time() - t0:.0f} s", flush=True)
    t0 = time.time()
    oracle.ref_moments("moments", rd, os.path.join(o, "moments.txt"), seeds=seeds)
    print(name, "moments", f"{time.time() - t0:.0f} s", flush=True)
    if LARGE[name][2]:
        t0 = time.time()
        r, i = oracle.ref_moments("msdmom", rd, os.path.join(tmp, "m.txt"), seeds=seeds)
        M = LARGE[name][1]
        np.savez_compressed(os.path.join(o, "msdmom.npz"), re=r.reshape(-1, M),
                            im=i.reshape(-1, M))
        print(name, "msd moments", f"{time.time() - t0:.0f} s", flush=True)


def main() -> None:
    oracle.build(ref=True)
    names = [a for a in sys.argv[1:] if not a.startswith("-")] or list(LARGE)
    tmp = os.path.join(HERE, "_tmp_large")
    os.makedirs(tmp, exist_ok=True)
    try:
        for name in names:
            make(name, tmp)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    main()
