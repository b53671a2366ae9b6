"""The multi-GPU replica path (gpuqt_b200/replicas.py) on CPU: sharding, the random
stream seen by each rank, the gather order, and a world_size-2 gloo run whose merged
.out rows must equal a serial run and the reference's own output. The per-vector
compute is the oracle here (no GPU); on GPUs it is the library."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import gpuqt_b200 as g
import oracle as O
from conftest import REF, fixture_dir
from gpuqt_b200 import replicas as RP


class OracleCompute:
    """The per-vector rows computed by the CPU oracle (test stand-in for the GPU)."""

    def hamiltonian(self, model):
        return O.Model(n=model.n, max_neighbor=model.max_neighbor,
                       energy_max=model.energy_max, volume=model.volume,
                       neighbor_number=model.neighbor_number, neighbor_list=model.neighbor_list,
                       potential=model.potential, hopping_real=model.hopping_real,
                       hopping_imag=model.hopping_imag, xx=model.xx)

    def _row(self, model, mu):
        return O.correlation(model.n_moments, mu[0], mu[1], model.energy, model.energy_max,
                             model.volume)

    def dos(self, model, H, phi):
        return self._row(model, O.find_moments(H, model.n_moments, phi, phi))

    def vac0(self, model, H, phi):
        v = O.apply_current(H, *phi)
        return self._row(model, O.find_moments(H, model.n_moments, v, v))

    def vac(self, model, H, phi):
        mr, mi = O.vac_moments(H, model.n_moments, model.time_step, phi)
        return [self._row(model, (mr[k], mi[k])) for k in range(len(model.time_step))]

    def msd(self, model, H, phi):
        mr, mi = O.msd_moments(H, model.n_moments, model.time_step, phi)
        return [self._row(model, (mr[k], mi[k])) for k in range(len(model.time_step))]


def test_shard_covers_every_item_once():
    for n in (0, 1, 5, 16):
        for w in (1, 2, 3, 8):
            got = sorted(k for r in range(w) for k in RP.shard(n, r, w))
            assert got == list(range(n))


def test_each_rank_sees_the_single_stream():
    d = fixture_dir("chain_z2")
    serial = g.Model.load(d)
    want = [serial.initial_state() for _ in range(5)]
    for rank, world in ((0, 2), (1, 2), (2, 3)):
        m = g.Model.load(d)
        got = RP.draw_phase_vectors(m, RP.shard(5, rank, world))
        for k, v in got.items():
            np.testing.assert_array_equal(v[0], want[k][0])
            np.testing.assert_array_equal(v[1], want[k][1])


def test_merge_order_and_missing_vectors():
    parts = [{1: {"dos.out": ["b"]}, 3: {"dos.out": ["d"]}},
             {0: {"dos.out": ["a"], "msd.out": ["a1", "a2"]}, 2: {"dos.out": ["c"]}}]
    merged = RP.merge_in_order(parts, 4)
    assert merged["dos.out"] == ["a", "b", "c", "d"]
    assert merged["msd.out"] == ["a1", "a2"]
    with pytest.raises(RuntimeError):
        RP.merge_in_order(parts, 5)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, d, out_path):
    import torch.distributed as td
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    td.init_process_group("gloo", rank=rank, world_size=world)

    def gather(obj):
        out = [None] * world if rank == 0 else None
        td.gather_object(obj, out, dst=0)
        return out

    model = g.Model.load(d)
    merged = RP.run(model, rank, world, OracleCompute(), {"msd": True}, gather)
    if rank == 0:
        with open(out_path, "w") as f:
            for name in sorted(merged):
                for row in merged[name]:
                    f.write(name + ": " + RP.format_row(row))
    td.barrier()
    td.destroy_process_group()


def _serial_rows(d):
    model = g.Model.load(d)
    merged = RP.run(model, 0, 1, OracleCompute(), {"msd": True}, lambda o: [o])
    return "".join(name + ": " + RP.format_row(row) for name in sorted(merged)
                   for row in merged[name])


def test_gloo_two_ranks_match_serial_and_reference(tmp_path):
    d = fixture_dir("chain_z2")  # 2 random vectors, MSD with 3 steps
    out = str(tmp_path / "rows.txt")
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, 2, port, d, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    got = open(out).read()
    assert got == _serial_rows(d)
    # The reference's own files for this directory, row for row.
    for name in ("dos.out", "msd.out"):
        ref = open(os.path.join(REF, "chain_z2", name)).read()
        mine = "".join(l[len(name) + 2:] for l in got.splitlines(True) if l.startswith(name))
        assert mine == ref, name
