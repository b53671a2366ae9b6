"""Host side of checkpoint / resume and the raw moment files, without a GPU: the
para.in keywords, the moment-file reader, and the refusal of damaged or foreign
checkpoints (read before any device work, so these run on the CPU)."""
from __future__ import annotations

import os
import shutil
import struct

import numpy as np
import pytest

import gpuqt_b200 as g
from conftest import fixture_dir


def _fnv1a(data: bytes) -> int:
    h = 1469598103934665603
    for b in data:
        h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def _checkpoint(fingerprint=12345, rng=b"0 1 2 3", good_sum=True) -> bytes:
    body = b"GQTCKPv1" + struct.pack("<Q", fingerprint) + struct.pack("<iii", 0, 0, 1)
    body += struct.pack("<Q", len(rng)) + rng
    body += struct.pack("<I", 1) + struct.pack("<Q", 7) + b"dos.out" + struct.pack("<Q", 0)
    body += struct.pack("<I", 0)
    s = _fnv1a(body) ^ (0 if good_sum else 1)
    return body + struct.pack("<Q", s)


def _dir(tmp_path, extra):
    d = str(tmp_path / "run")
    shutil.copytree(fixture_dir("chain_z2"), d)
    with open(os.path.join(d, "para.in"), "a") as f:
        f.write(extra)
    return d


def test_keywords_parse(tmp_path):
    g.Model.load(_dir(tmp_path, "output_moments\ncheckpoint_every 3\nkpm_doubling\n"
                                "batch_vectors 16\n"))
    bad = str(tmp_path / "bad")
    shutil.copytree(fixture_dir("chain_z2"), bad)
    with open(os.path.join(bad, "para.in"), "a") as f:
        f.write("checkpoint_every 0\n")
    with pytest.raises(g.GqtError) as e:
        g.Model.load(bad)
    assert e.value.status == 4
    bad2 = str(tmp_path / "bad2")
    shutil.copytree(fixture_dir("chain_z2"), bad2)
    with open(os.path.join(bad2, "para.in"), "a") as f:
        f.write("batch_vectors 0\n")
    with pytest.raises(g.GqtError) as e:
        g.Model.load(bad2)
    assert e.value.status == 4


@pytest.mark.parametrize("content,message", [
    (b"not a checkpoint at all", "not a checkpoint"),
    (_checkpoint(good_sum=False), "damaged"),
    (_checkpoint(), "different run"),
    (_checkpoint()[:-9] + _checkpoint()[-8:], "damaged"),
])
def test_damaged_or_foreign_checkpoint_is_refused(tmp_path, content, message):
    d = _dir(tmp_path, "checkpoint_every 1\n")
    with open(os.path.join(d, "lsqt.checkpoint"), "wb") as f:
        f.write(content)
    with pytest.raises(g.GqtError) as e:
        g.lsqt(d)
    assert e.value.status == 4 and message in str(e.value), str(e.value)


def test_moments_reader(tmp_path):
    M = 5
    re = np.arange(3 * M, dtype=np.float64).reshape(3, M)
    im = -re / 7
    rows = np.stack([re, im], axis=-1).astype("<f8").tobytes()
    p = str(tmp_path / "dos_moments.bin")
    with open(p, "wb") as f:
        f.write(b"GQTMOMv1" + struct.pack("<ii", M, 0) + rows)
    r, i = g.read_moments(p)
    np.testing.assert_array_equal(r, re)
    np.testing.assert_array_equal(i, im)
    with open(p, "ab") as f:
        f.write(b"\0" * 8)
    with pytest.raises(ValueError):
        g.read_moments(p)


@pytest.mark.parametrize("extra", ["", "batch_vectors 4\n"])
def test_fp32r_run_needs_groups_of_four(tmp_path, extra):
    """The FP32R moment form launches 4, 16 or 32 vectors: a run without groups, or with
    a vector count (2 here) that leaves a smaller group, is refused before any device
    work."""
    d = _dir(tmp_path, extra)
    with pytest.raises(g.GqtError) as e:
        g.lsqt(d, precision=g.FP32R)
    assert e.value.status == 4 and "FP32R" in str(e.value), str(e.value)
