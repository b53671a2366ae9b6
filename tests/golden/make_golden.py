"""Regenerate the golden fixtures under tests/golden/ from the reference's own build.

Writes small input directories (inputs/<name>/) and runs the reference compiled from
its sources (oracle/_ref: ref_driver and lsqt_cpu, built by `make -C oracle ref`) on
them, storing its raw results at full precision (ref/<name>/). It also copies the
reference's shipped example outputs used as golden vectors (examples/...). Needs the
reference checkout; run it here, commit the results:

    python tests/golden/make_golden.py                  # everything
    python tests/golden/make_golden.py --examples-only  # only the shipped examples
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

REF_EXAMPLES = os.path.join(oracle.REFERENCE_ROOT, "examples")
INPUTS = os.path.join(HERE, "inputs")
OUT = os.path.join(HERE, "ref")

SQUARE = """4
-1 0 0 0 -1 0
1  0 0 0 -1 0
0  1 0 0 -1 0
0 -1 0 0 -1 0
"""
# The 4-orbital rectangular graphene cell of the reference's manual
# (doc/gpuqt.tex:435-456), hopping -2.7 eV.
GRAPHENE_CELL = """1.7321 3 1
4 3
0.866 0    0
0     0.5  0
0     1.5  0
0.866 2    0
3
1  0 0 1 -2.7 0
0  0 0 1 -2.7 0
0 -1 0 3 -2.7 0
3
0  0 0 0 -2.7 0
-1 0 0 0 -2.7 0
0  0 0 2 -2.7 0
3
0 0 0 3 -2.7 0
-1 0 0 3 -2.7 0
0 0 0 1 -2.7 0
3
1  0 0 2 -2.7 0
0  0 0 2 -2.7 0
0 1 0 0 -2.7 0
"""
CUBIC = """6
1 0 0 0 -1 0
-1 0 0 0 -1 0
0 1 0 0 -1 0
0 -1 0 0 -1 0
0 0 1 0 -1 0
0 0 -1 0 -1 0
"""


def energies(lo, hi, n):
    return np.linspace(lo, hi, n)


def write_dir(name, para, lattice=None, energy=None, time_step=None, extra=None):
    d = os.path.join(INPUTS, name)
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "para.in"), "w") as f:
        f.write(para)
    if lattice is not None:
        with open(os.path.join(d, "lattice.in"), "w") as f:
            f.write(lattice)
    with open(os.path.join(d, "energy.in"), "w") as f:
        f.write(f"{len(energy)}\n" + "".join(f"{e:.6f}\n" for e in energy))
    if time_step is not None:
        with open(os.path.join(d, "time_step.in"), "w") as f:
            f.write(f"{len(time_step)}\n" + "".join(f"{t:.6f}\n" for t in time_step))
    for fname, text in (extra or {}).items():
        with open(os.path.join(d, fname), "w") as f:
            f.write(text)
    return d


def general_model_files(n=40, z=5, seed=2024):
    """A seeded random general model: neighbor.in, position.in, potential.in, hopping.in."""
    rng = np.random.default_rng(seed)
    nn = rng.integers(1, z + 1, size=n)
    nb, hop = [], []
    for i in range(n):
        js = rng.choice([j for j in range(n) if j != i], size=nn[i], replace=False)
        nb.append(js)
        hop.append(rng.uniform(-1.5, -0.5, nn[i]) + 1j * rng.uniform(-0.2, 0.2, nn[i]))
    x = np.sort(rng.uniform(0, 30.0, n))
    neighbor = f"{n} {z}\n" + "".join(
        f"{nn[i]} " + " ".join(str(j) for j in nb[i]) + "\n" for i in range(n))
    position = "30.0 900.0\n" + "".join(f"{v:.10f}\n" for v in x)
    potential = "".join(f"{v:.10f}\n" for v in rng.uniform(-0.5, 0.5, n))
    hopping = "complex\n" + "".join(
        "".join(f"{h.real:.10f} {h.imag:.10f}\n" for h in hop[i]) for i in range(n))
    return {"neighbor.in": neighbor, "position.in": position, "potential.in": potential,
            "hopping.in": hopping}


FIXTURES = {
    # name: (para, lattice, energy grid, time steps, extra files, dt for the ops dump)
    "sq16_pbc": ("model 1\nanderson_disorder 2.0\nenergy_max 5.0\nnumber_of_moments 200\n"
                 "calculate_vac\ncalculate_msd\ncalculate_vac0\n",
                 "16 16 1\n1 1 0 0\n1 1 1\n1 4\n0 0 0\n" + SQUARE,
                 energies(-4.9, 4.9, 41), [1.0, 1.0, 1.0], None, 5.0),
    "sq12_open_vac": ("model 1\nanderson_disorder 1.0\nvacancy_disorder 7\nenergy_max 5.2\n"
                      "number_of_moments 150\ncalculate_msd\ncalculate_vac\n",
                      "12 10 1\n1 0 0 0\n1 1 1\n1 4\n0 0 0\n" + SQUARE,
                      energies(-5.0, 5.0, 21), [0.5, 0.7], None, 2.6),
    "graphene_8x4": ("model 1\nanderson_disorder 1.0\nenergy_max 8.7\nnumber_of_moments 300\n"
                     "calculate_msd\ncalculate_vac\n",
                     "8 4 1\n1 1 0 0\n" + GRAPHENE_CELL,
                     energies(-8.5, 8.5, 35), [1.519267, 1.519267, 1.519267], None, 13.2),
    "cubic6": ("model 1\nanderson_disorder 16.5\nenergy_max 15.0\nnumber_of_moments 200\n"
               "calculate_msd\ncalculate_vac\n",
               "6 6 6\n1 1 1 0\n1 1 1\n1 6\n0 0 0\n" + CUBIC,
               energies(-14.0, 14.0, 29), [1.0, 1.0], None, 15.0),
    "chain_z2": ("model 1\nanderson_disorder 3.0\nenergy_max 3.6\nnumber_of_moments 120\n"
                 "number_of_random_vectors 2\ncalculate_msd\n",
                 "300 1 1\n1 0 0 0\n1 1 1\n1 2\n0 0 0\n2\n-1 0 0 0 -1 0\n1 0 0 0 -1 0\n",
                 energies(-3.5, 3.5, 15), [0.3, 0.6, 0.9], None, 3.6),
    "sq20_charge": ("model 1\nanderson_disorder 1.0\ncharged_impurity 10 1.0 1.5\n"
                    "energy_max 6.0\nnumber_of_moments 100\ncalculate_vac\n",
                    "20 20 1\n1 1 0 0\n1 1 1\n1 4\n0 0 0\n" + SQUARE,
                    energies(-5.5, 5.5, 23), [1.0, 1.0], None, 6.0),
    "general40": ("model 0\nenergy_max 9.0\nnumber_of_moments 150\ncalculate_msd\n"
                  "calculate_vac\n",
                  None, energies(-8.0, 8.0, 17), [0.4, 0.4], general_model_files(), 9.0),
    "general_spin": ("model 0\nenergy_max 9.0\nnumber_of_moments 120\ncalculate_spin\n"
                     "calculate_ldos\n",
                     None, energies(-8.0, 8.0, 17), [0.5, 0.5, 0.5],
                     dict(general_model_files(n=48, z=4, seed=77),
                          **{"local_orbitals.in": "3\n0\n7\n21\n"}), 9.0),
    # The CPU-runnable plain FP64 case: 256 x 256 square lattice, t = -1, W = 2,
    # energy scale 5, 1000 moments, VAC with 10 steps of 1.0; disorder seed 1, phase
    # seed 7 (split-seed mode).
    "square256": ("model 1\nanderson_disorder 2.0\nenergy_max 5.0\nnumber_of_moments 1000\n"
                  "calculate_vac\ndisorder_seed 1\nphase_seed 7\n",
                  "256 256 1\n1 1 0 0\n1 1 1\n1 4\n0 0 0\n" + SQUARE,
                  energies(-4.95, 4.95, 199), [1.0] * 10, None, None),
}
SPLIT_SEEDS = {"square256": (1, 7)}
OUT_FILES = ("dos.out", "vac0.out", "vac.out", "msd.out", "S.out", "ldos.out")


def ref_para(para: str) -> str:
    """para.in without this library's seed keywords (the reference rejects them)."""
    return "".join(l + "\n" for l in para.splitlines()
                   if l.split() and l.split()[0] not in ("seed", "disorder_seed", "phase_seed"))


def main() -> None:
    oracle.build(ref=True)
    os.makedirs(OUT, exist_ok=True)
    tmp = os.path.join(HERE, "_tmp")
    for name, (para, lattice, energy, ts, extra, dt) in FIXTURES.items():
        d = write_dir(name, para, lattice, energy, ts, extra)
        # The reference binaries see a copy without the extension keywords.
        rd = os.path.join(tmp, name)
        if os.path.isdir(rd):
            shutil.rmtree(rd)
        shutil.copytree(d, rd)
        with open(os.path.join(rd, "para.in"), "w") as f:
            f.write(ref_para(para))
        seeds = SPLIT_SEEDS.get(name)
        o = os.path.join(OUT, name)
        os.makedirs(o, exist_ok=True)
        ell = oracle.ref_ell(rd, os.path.join(tmp, "ell.bin"), seeds=seeds)
        if ell.n <= 5000:
            np.savez_compressed(os.path.join(o, "ell.npz"), nn=ell.neighbor_number,
                                nl=ell.neighbor_list, pot=ell.potential, hr=ell.hopping_real,
                                hi=ell.hopping_imag, xx=ell.xx,
                                meta=np.array([ell.energy_max, ell.volume]))
        mr, mi = oracle.ref_moments("moments", rd, os.path.join(o, "moments.txt"), seeds=seeds)
        if ts is not None:
            for mode in ("vacmom", "msdmom"):
                if mode == "msdmom" and name == "square256":
                    continue
                r, i = oracle.ref_moments(mode, rd, os.path.join(tmp, "m.txt"), seeds=seeds)
                M = len(mr)
                np.savez_compressed(os.path.join(o, mode + ".npz"), re=r.reshape(-1, M),
                                    im=i.reshape(-1, M))
        if dt is not None:
            ops = oracle.ref_ops(rd, os.path.join(tmp, "ops.bin"), dt, seeds=seeds)
            np.savez_compressed(os.path.join(o, "ops.npz"), dt=np.array([dt]),
                                **{k.replace("+", "_p").replace("-", "_m"): np.stack(v)
                                   for k, v in ops.items()})
        if seeds is None:
            # The reference's own .out files for the full run of this directory.
            for f in OUT_FILES:
                p = os.path.join(rd, f)
                if os.path.exists(p):
                    os.remove(p)
            with open(os.path.join(tmp, "input.txt"), "w") as f:
                f.write(rd + "\n")
            subprocess.run([oracle.REF_LSQT, os.path.join(tmp, "input.txt")], check=True,
                           stdout=subprocess.DEVNULL)
            for f in OUT_FILES:
                p = os.path.join(rd, f)
                if os.path.exists(p):
                    shutil.copy(p, os.path.join(o, f))
        print("fixture", name, "n =", ell.n)

    copy_examples()
    shutil.rmtree(tmp)


def copy_examples() -> None:
    """The reference's shipped example inputs and outputs used as golden vectors."""
    # examples/review/graphene/vacancy: 19.8M sites with 200,000 vacancies; its dos.out
    # holds 10 one-vector rows from unseeded runs (compared statistically).
    src = os.path.join(REF_EXAMPLES, "review", "graphene", "vacancy")
    dst = os.path.join(HERE, "examples", "review_graphene_vacancy")
    os.makedirs(dst, exist_ok=True)
    for f in ("para.in", "lattice.in", "energy.in", "time_step.in", "dos.out"):
        shutil.copy(os.path.join(src, f), os.path.join(dst, f))
    print("example review/graphene/vacancy")
    # Shipped example outputs of the reference (examples/fan2018cpc/lattice/*).
    for ex in ("diffusive", "localized"):
        src = os.path.join(REF_EXAMPLES, "fan2018cpc", "lattice", ex)
        dst = os.path.join(HERE, "examples", "fan2018cpc_" + ex)
        os.makedirs(dst, exist_ok=True)
        for f in ("para.in", "lattice.in", "energy.in", "time_step.in", "dos.out", "vac.out",
                  "msd.out"):
            if os.path.exists(os.path.join(src, f)):
                shutil.copy(os.path.join(src, f), os.path.join(dst, f))
        print("example", ex)


if __name__ == "__main__":
    if "--examples-only" in sys.argv:
        copy_examples()
    else:
        main()
