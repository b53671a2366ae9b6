"""End-to-end runs on the GPU (gqt_lsqt and the lsqt_b200 CLI) against the
reference's .out files: its shipped example outputs (4,000,000 sites) and the
outputs of the reference build on the small fixtures. The .out files carry 6
significant digits; values must agree to that precision (a last-digit difference
is allowed only where the reference's own rerun shows one)."""
from __future__ import annotations

import os
import shutil
import subprocess

import numpy as np
import pytest

import gpuqt_b200 as g
from conftest import EXAMPLES, REF, SMALL_FIXTURES, fixture_dir

pytestmark = pytest.mark.gpu


def _read(path):
    with open(path) as f:
        return [np.array([float(t) for t in l.split()]) for l in f if l.strip()]


def _compare(ours, ref, rel=1e-5):
    a, b = _read(ours), _read(ref)
    assert len(a) == len(b), (ours, len(a), len(b))
    for k, (x, y) in enumerate(zip(a, b)):
        assert x.shape == y.shape
        fin = np.isfinite(y)
        assert np.array_equal(np.isfinite(x), fin)
        scale = np.max(np.abs(y[fin])) if fin.any() else 1.0
        # 6 printed digits: a half unit in the last place, per row scale
        assert np.all(np.abs(x[fin] - y[fin]) <= rel * np.abs(y[fin]) + 1e-12 * scale), k


def _copy_inputs(src, dst):
    os.makedirs(dst, exist_ok=True)
    for f in os.listdir(src):
        if f.endswith(".in"):
            shutil.copy(os.path.join(src, f), dst)


@pytest.mark.parametrize("name", SMALL_FIXTURES)
def test_cli_matches_reference_outputs(tmp_path, name):
    d = tmp_path / name
    _copy_inputs(fixture_dir(name), d)
    (tmp_path / "input.txt").write_text(str(d) + "\n")
    r = subprocess.run([g.CLI_PATH, str(tmp_path / "input.txt")], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    found = 0
    for f in ("dos.out", "vac0.out", "vac.out", "msd.out", "S.out", "ldos.out"):
        ref = os.path.join(REF, name, f)
        if os.path.exists(ref):
            _compare(str(d / f), ref)
            found += 1
    assert found >= 2


@pytest.mark.parametrize("example,outs", [
    ("fan2018cpc_diffusive", ("dos.out", "vac.out", "msd.out")),
    ("fan2018cpc_localized", ("dos.out", "msd.out")),
])
def test_shipped_examples(tmp_path, example, outs):
    d = tmp_path / example
    _copy_inputs(os.path.join(EXAMPLES, example), d)
    g.lsqt(str(d))
    for f in outs:
        _compare(str(d / f), os.path.join(EXAMPLES, example, f))


def test_fp32_run_close_to_fp64(tmp_path):
    a, b = tmp_path / "a", tmp_path / "b"
    _copy_inputs(fixture_dir("graphene_8x4"), a)
    _copy_inputs(fixture_dir("graphene_8x4"), b)
    g.lsqt(str(a), precision=g.FP64)
    g.lsqt(str(b), precision=g.FP32)
    for f in ("dos.out", "vac.out", "msd.out"):
        x, y = _read(str(b / f)), _read(str(a / f))
        for u, v in zip(x, y):
            assert np.max(np.abs(u - v)) <= 1e-5 * np.max(np.abs(v))


def test_replica_launcher_matches_reference(tmp_path):
    """torchrun -m gpuqt_b200.replicas (one rank here) against the reference's files."""
    import socket
    import sys
    name = "chain_z2"
    d = tmp_path / name
    _copy_inputs(fixture_dir(name), d)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
                        "--nproc-per-node=1", "--master-addr=127.0.0.1",
                        f"--master-port={port}", "-m", "gpuqt_b200.replicas", str(d)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    for f in ("dos.out", "msd.out"):
        _compare(str(d / f), os.path.join(REF, name, f))
