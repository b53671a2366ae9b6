"""Synthetic lattice inputs in the reference's input format (lattice.in / para.in /
energy.in / time_step.in, src/model_lattice.cu:165-337, src/model.cu:243-384).

Used by bench.py for the benchmark configurations; any directory written here can
also be run by the reference's own binaries (drop the seed keywords, which are this
library's extension).
"""
from __future__ import annotations

import os

import numpy as np

SQUARE = [(-1, 0, 0, 0), (1, 0, 0, 0), (0, 1, 0, 0), (0, -1, 0, 0)]
CUBIC = [(1, 0, 0, 0), (-1, 0, 0, 0), (0, 1, 0, 0), (0, -1, 0, 0), (0, 0, 1, 0),
         (0, 0, -1, 0)]
# The reference manual's 4-orbital rectangular graphene cell (doc/gpuqt.tex:435-456):
# orbital positions and, per orbital, (dx, dy, dz, orbital) of its three neighbours.
GRAPHENE_XYZ = [(0.866, 0.0, 0.0), (0.0, 0.5, 0.0), (0.0, 1.5, 0.0), (0.866, 2.0, 0.0)]
GRAPHENE_HOPS = [
    [(1, 0, 0, 1), (0, 0, 0, 1), (0, -1, 0, 3)],
    [(0, 0, 0, 0), (-1, 0, 0, 0), (0, 0, 0, 2)],
    [(0, 0, 0, 3), (-1, 0, 0, 3), (0, 0, 0, 1)],
    [(1, 0, 0, 2), (0, 0, 0, 2), (0, 1, 0, 0)],
]


def lattice_text(kind: str, cells: tuple[int, int, int], hopping: float = -1.0,
                 pbc: tuple[int, int, int] | None = None, transport: int = 0) -> str:
    nx, ny, nz = cells
    if kind == "graphene":
        pbc = pbc or (1, 1, 0)
        lines = [f"{nx} {ny} {nz}", f"{pbc[0]} {pbc[1]} {pbc[2]} {transport}", "1.7321 3 1",
                 "4 3"]
        lines += [f"{x} {y} {z}" for x, y, z in GRAPHENE_XYZ]
        for hops in GRAPHENE_HOPS:
            lines.append(str(len(hops)))
            lines += [f"{a} {b} {c} {o} {hopping} 0" for a, b, c, o in hops]
    elif kind in ("square", "cubic"):
        hops = SQUARE if kind == "square" else CUBIC
        pbc = pbc or ((1, 1, 0) if kind == "square" else (1, 1, 1))
        lines = [f"{nx} {ny} {nz}", f"{pbc[0]} {pbc[1]} {pbc[2]} {transport}", "1 1 1",
                 f"1 {len(hops)}", "0 0 0", str(len(hops))]
        lines += [f"{a} {b} {c} {o} {hopping} 0" for a, b, c, o in hops]
    else:
        raise ValueError(kind)
    return "\n".join(lines) + "\n"


def write_input_dir(path: str, kind: str, cells, *, hopping: float = -1.0,
                    anderson: float | None = None, energy_max: float = 10.0,
                    moments: int = 1000, energy=None, time_step=None,
                    calculate=("msd",), seed: int | None = None,
                    disorder_seed: int | None = None, phase_seed: int | None = None,
                    random_vectors: int = 1) -> str:
    os.makedirs(path, exist_ok=True)
    para = ["model 1", f"energy_max {energy_max}", f"number_of_moments {moments}",
            f"number_of_random_vectors {random_vectors}"]
    if anderson is not None:
        para.append(f"anderson_disorder {anderson}")
    para += [f"calculate_{c}" for c in calculate]
    for k, v in (("seed", seed), ("disorder_seed", disorder_seed),
                 ("phase_seed", phase_seed)):
        if v is not None:
            para.append(f"{k} {v}")
    with open(os.path.join(path, "para.in"), "w") as f:
        f.write("\n".join(para) + "\n")
    with open(os.path.join(path, "lattice.in"), "w") as f:
        f.write(lattice_text(kind, cells, hopping))
    if energy is None:
        energy = np.linspace(-0.98 * energy_max, 0.98 * energy_max, 201)
    with open(os.path.join(path, "energy.in"), "w") as f:
        f.write(f"{len(energy)}\n" + "".join(f"{e:.6f}\n" for e in energy))
    ts = list(time_step) if time_step is not None else [1.0]
    with open(os.path.join(path, "time_step.in"), "w") as f:
        f.write(f"{len(ts)}\n" + "".join(f"{t:.6f}\n" for t in ts))
    return path


# Benchmark configurations (1 fs = 1.519267 hbar/eV).
FS = 1.519267
CONFIGS = {
    "graphene2m": dict(
        kind="graphene", cells=(1024, 512, 1), hopping=-2.7, anderson=1.0, energy_max=8.7,
        moments=3000, time_step=[FS] * 20, calculate=("msd",), seed=3,
        description="honeycomb graphene, 4-orbital cell x 1024x512 = 2,097,152 sites, z=3, "
                    "t=-2.7 eV, Anderson W=1.0 eV (seed 3), E_max 8.7 eV, 3000 moments, "
                    "MSD steps of 1 fs"),
    "square256": dict(
        kind="square", cells=(256, 256, 1), hopping=-1.0, anderson=2.0, energy_max=5.0,
        moments=1000, time_step=[1.0] * 10, calculate=("vac",), disorder_seed=1,
        phase_seed=7,
        description="square 256x256 = 65,536 sites, z=4, t=-1, W=2 (seed 1), E_max 5, "
                    "1000 moments, phases seed 7"),
    "graphene4m": dict(
        kind="graphene", cells=(1024, 1024, 1), hopping=-2.7, anderson=1.5, energy_max=9.0,
        moments=5000, time_step=[FS] * 20, calculate=("vac",), seed=5,
        description="honeycomb graphene 4,194,304 sites, t=-2.7 eV, W=1.5 eV (seed 5), "
                    "E_max 9.0, 5000 moments"),
    "square1m": dict(
        kind="square", cells=(1024, 1024, 1), hopping=-1.0, anderson=2.0, energy_max=5.2,
        moments=2000, time_step=[1.0], calculate=(), seed=17,
        description="square 1024x1024 = 1,048,576 sites, z=4, t=-1, W=2 (seed 17), E_max 5.2"),
    "cubic_slab": dict(
        kind="cubic", cells=(32, 256, 256), hopping=-1.0, anderson=16.5, energy_max=15.0,
        moments=4000, time_step=[1.0] * 30, calculate=("vac", "msd"), seed=13,
        description="cubic slab 32x256x256 = 2,097,152 sites, z=6, the 65,536-site plane "
                    "stride of 256^3 (a profiling size for it), t=-1, W=16.5 (seed 13), "
                    "E_max 15"),
    "cubic256": dict(
        kind="cubic", cells=(256, 256, 256), hopping=-1.0, anderson=16.5, energy_max=15.0,
        moments=4000, time_step=[1.0] * 30, calculate=("vac", "msd"), seed=13,
        description="cubic 256^3 = 16,777,216 sites, z=6, t=-1, W=16.5 (seed 13), "
                    "E_max 15, 4000 moments"),
}


def config_dir(root: str, name: str) -> str:
    c = dict(CONFIGS[name])
    c.pop("description")
    kind, cells = c.pop("kind"), c.pop("cells")
    return write_input_dir(os.path.join(root, name), kind, cells, **c)


def config_sites(name: str) -> int:
    c = CONFIGS[name]
    per_cell = 4 if c["kind"] == "graphene" else 1
    return per_cell * int(np.prod(c["cells"]))


def batch_realisations(count: int = 8, seed: int = 11):
    """The realisation batch: square lattices L x L with log-uniform L in [128, 2048]
    (L = round(2^u), u ~ U(7, 11)), Anderson W ~ U(0.5, 4), E_max = 4 + W/2 + 0.1,
    hopping -1. Drawn from numpy's MT19937 (RandomState(seed))."""
    rs = np.random.RandomState(seed)
    u = rs.uniform(7.0, 11.0, count)
    w = rs.uniform(0.5, 4.0, count)
    return [dict(L=int(round(2.0 ** x)), W=float(ww), energy_max=4.0 + float(ww) / 2 + 0.1)
            for x, ww in zip(u, w)]


def batch_dirs(root: str, count: int = 8, seed: int = 11, moments: int = 2000):
    """Input directories of the realisation batch (disorder seed seed + 1 + r)."""
    out = []
    for r, c in enumerate(batch_realisations(count, seed)):
        out.append(write_input_dir(os.path.join(root, f"real{r}"), "square", (c["L"], c["L"], 1),
                                   hopping=-1.0, anderson=c["W"], energy_max=c["energy_max"],
                                   moments=moments, calculate=(), disorder_seed=seed + 1 + r))
    return out
