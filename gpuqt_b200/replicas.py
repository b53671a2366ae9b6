"""Replicas across GPUs: one process per GPU, independent random vectors per rank.

The LSQT path shards by independent units: each random-phase vector's DOS / VAC0 /
VAC / MSD rows depend on nothing but the model and that vector. Rank r of W takes
vectors r, r + W, r + 2W, ... of the model's single random stream (vector k is the
k-th draw, as in the reference, which draws them one after another,
src/lsqt.cu:140-150), computes their rows, and rank 0 gathers them and appends the
.out files in the reference's order (per file: vector 0's rows, then vector 1's, ...).
No collective touches the data path; torch.distributed only carries the gather of
the finished rows.

    torchrun --nproc-per-node N -m gpuqt_b200.replicas input_dir [--fp32]
"""
from __future__ import annotations

import os
import sys

import numpy as np

OUT_FILES = ("dos.out", "vac0.out", "vac.out", "msd.out")


def shard(n_items: int, rank: int, world: int) -> list[int]:
    """The items rank `rank` of `world` owns (round-robin)."""
    return list(range(rank, n_items, world))


def draw_phase_vectors(model, wanted: list[int]) -> dict:
    """Vectors 0 .. max(wanted) drawn in order from the model's stream; the wanted ones
    are kept (the others are drawn and discarded, so every rank sees the stream the
    reference would)."""
    out = {}
    if not wanted:
        return out
    keep = set(wanted)
    for k in range(max(wanted) + 1):
        v = model.initial_state()
        if k in keep:
            out[k] = v
    return out


class LibraryCompute:
    """The rows of one random vector through the library's C ABI (the algorithms of
    src/sigma.cu:204-391 over gqt_moments / gqt_evolve / gqt_evolvex)."""

    def __init__(self, precision=None):
        import gpuqt_b200 as g
        self.g = g
        self.precision = g.FP64 if precision is None else precision

    def hamiltonian(self, model):
        return self.g.Hamiltonian(model)

    def _row(self, model, mu):
        return self.g.chebyshev_summation(mu[0], mu[1], model.energy, model.energy_max,
                                          model.volume)

    # States (and their time evolution) stay FP64; the moment recurrence runs in
    # self.precision.
    def _vec(self, model, phi):
        return self.g.Vector.from_host(*phi)

    def _moments(self, H, left, right, model):
        return self.g.moments(H, left, right, model.n_moments, precision=self.precision)

    def dos(self, model, H, phi):
        x = self._vec(model, phi)
        return self._row(model, self._moments(H, x, x, model))

    def vac0(self, model, H, phi):
        g = self.g
        x = self._vec(model, phi)
        v = g.Vector(model.n)
        g.apply_current(H, x, v)
        return self._row(model, self._moments(H, v, v, model))

    def vac(self, model, H, phi):
        g = self.g
        left = self._vec(model, phi)
        right = left.clone()
        lcopy = g.Vector(model.n)
        g.apply_current(H, left, right)
        rows = []
        for m in range(model.n_steps):
            g.apply_current(H, left, lcopy)
            rows.append(self._row(model, self._moments(H, right, lcopy, model)))
            if m < model.n_steps - 1:
                dt = model.time_step[m] * model.energy_max
                g.evolve(H, -1, dt, left)
                g.evolve(H, -1, dt, right)
        return rows

    def msd(self, model, H, phi):
        g = self.g
        state = self._vec(model, phi)
        sx = state.clone()
        copy = g.Vector(model.n)
        dt = model.time_step[0] * model.energy_max
        g.evolve(H, 1, dt, state)
        g.evolvex(H, 1, dt, sx)
        rows = []
        for m in range(model.n_steps):
            rows.append(self._row(model, self._moments(H, sx, sx, model)))
            if m < model.n_steps - 1:
                dt = model.time_step[m + 1] * model.energy_max
                copy.copy_from(state)
                g.evolvex(H, 1, dt, copy)
                g.evolve(H, 1, dt, sx)
                sx.add(copy)
                g.evolve(H, 1, dt, state)
        return rows


def vector_rows(model, H, phi, compute, flags: dict) -> dict:
    """{file: [rows]} of one random vector, for the calculations `flags` enables."""
    rows = {"dos.out": [compute.dos(model, H, phi)]}
    if flags.get("vac0"):
        rows["vac0.out"] = [compute.vac0(model, H, phi)]
    if flags.get("vac"):
        rows["vac.out"] = compute.vac(model, H, phi)
    if flags.get("msd"):
        rows["msd.out"] = compute.msd(model, H, phi)
    return rows


def format_row(row) -> str:
    """One .out row with std::ostream's default formatting (6 significant digits)."""
    return "".join(_fmt(float(x)) + " " for x in row) + "\n"


def _fmt(x: float) -> str:
    if x != x:
        return "-nan" if np.signbit(x) else "nan"
    if x in (float("inf"), float("-inf")):
        return "inf" if x > 0 else "-inf"
    return "%g" % x


def merge_in_order(parts: list[dict], n_vectors: int) -> dict:
    """{file: rows} in the reference's order from the ranks' {vector: {file: rows}}."""
    by_vec = {}
    for p in parts:
        by_vec.update(p)
    missing = [k for k in range(n_vectors) if k not in by_vec]
    if missing:
        raise RuntimeError(f"vectors {missing} were computed by no rank")
    out = {}
    for k in range(n_vectors):
        for f, rows in by_vec[k].items():
            out.setdefault(f, []).extend(rows)
    return out


def run(model, rank: int, world: int, compute, flags: dict, gather) -> dict | None:
    """This rank's share of the random vectors; returns the merged {file: rows} on
    rank 0 (None elsewhere). `gather(obj)` returns the list of every rank's obj on
    rank 0."""
    R = model.n_random_vectors
    mine = shard(R, rank, world)
    H = compute.hamiltonian(model)
    vecs = draw_phase_vectors(model, mine)
    results = {k: vector_rows(model, H, vecs[k], compute, flags) for k in mine}
    parts = gather(results)
    if rank != 0:
        return None
    return merge_in_order(parts, R)


def write_out(input_dir: str, merged: dict) -> None:
    for f, rows in merged.items():
        with open(os.path.join(input_dir, f), "a") as fh:
            for r in rows:
                fh.write(format_row(r))


def _flags_from_para(input_dir: str) -> dict:
    flags = {}
    with open(os.path.join(input_dir, "para.in")) as f:
        for line in f:
            tok = line.split()
            if tok and tok[0].startswith("calculate_"):
                flags[tok[0][len("calculate_"):]] = True
    return flags


def main(argv=None) -> int:
    import datetime

    import torch
    import torch.distributed as td

    import gpuqt_b200 as g

    args = list(sys.argv[1:] if argv is None else argv)
    fp32 = "--fp32" in args
    args = [a for a in args if a != "--fp32"]
    if len(args) != 1:
        print("usage: torchrun --nproc-per-node N -m gpuqt_b200.replicas input_dir [--fp32]")
        return 1
    input_dir = args[0]
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                              device_id=torch.device("cuda", local))

    def gather(obj):
        if world == 1:
            return [obj]
        out = [None] * world if rank == 0 else None
        td.gather_object(obj, out, dst=0)
        return out

    flags = _flags_from_para(input_dir)
    if flags.get("spin") or flags.get("ldos"):
        print("replicas: spin and LDOS runs are not sharded; use lsqt_b200")
        return 1
    model = g.Model.load(input_dir)
    merged = run(model, rank, world, LibraryCompute(g.FP32 if fp32 else g.FP64), flags, gather)
    if rank == 0:
        write_out(input_dir, merged)
    if world > 1:
        td.barrier()
        td.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
