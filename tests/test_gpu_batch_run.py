"""lsqt() with random vectors in groups (para.in batch_vectors): the groups run
through the multi-vector kernels, and every .out file must hold what the one-vector
run writes — the same rows in the same order, to the 6 printed digits in the FP64 form
(with and without kpm_doubling); in the FP32 moment form within 1e-6 of each row's
peak, the form's precision bar."""
from __future__ import annotations

import os
import shutil

import numpy as np
import pytest

import gpuqt_b200 as g
from conftest import fixture_dir
from test_gpu_golden import _compare, _read

pytestmark = pytest.mark.gpu

OUTS = ("dos.out", "vac0.out", "vac.out", "msd.out", "S.out", "ldos.out")


def _run(tmp_path, name, tag, extra, precision=g.FP64):
    d = str(tmp_path / (name + tag))
    os.makedirs(d)
    for f in os.listdir(fixture_dir(name)):
        if f.endswith(".in"):
            shutil.copy(os.path.join(fixture_dir(name), f), d)
    with open(os.path.join(d, "para.in"), "a") as f:
        f.write(extra)
    assert g.lsqt(d, precision=precision)
    return d


def _close_to_peak(ours, ref, tol):
    """Within tol of each row's peak, plus one unit in the 6th printed digit (a tiny
    deviation can cross a rounding boundary of the printed value)."""
    a, b = _read(ours), _read(ref)
    assert len(a) == len(b)
    for x, y in zip(a, b):
        fin = np.isfinite(y) & (y != 0)
        unit = 10.0 ** (np.floor(np.log10(np.abs(y[fin]))) - 5)
        assert np.all(np.abs(x[fin] - y[fin]) <= tol * np.max(np.abs(y[fin])) + unit)


def _same_outputs(a, b, tol=None):
    found = 0
    for f in OUTS:
        pa, pb = os.path.join(a, f), os.path.join(b, f)
        assert os.path.exists(pa) == os.path.exists(pb), f
        if os.path.exists(pa):
            if tol is None:
                _compare(pb, pa)
            else:
                _close_to_peak(pb, pa, tol)
            found += 1
    return found


@pytest.mark.parametrize("name,vectors", [("sq16_pbc", 5), ("chain_z2", 6)])
def test_groups_write_the_one_vector_outputs(tmp_path, name, vectors):
    extra = f"number_of_random_vectors {vectors}\n"
    a = _run(tmp_path, name, "_seq", extra)
    b = _run(tmp_path, name, "_grp", extra + "batch_vectors 16\n")
    assert _same_outputs(a, b) >= 2
    with open(os.path.join(b, "dos.out")) as f:
        assert sum(1 for l in f if l.strip()) == vectors


def test_groups_with_doubling_and_fp32(tmp_path):
    extra = "number_of_random_vectors 4\n"
    a = _run(tmp_path, "sq16_pbc", "_seq", extra)
    b = _run(tmp_path, "sq16_pbc", "_dbl", extra + "batch_vectors 4\nkpm_doubling\n")
    assert _same_outputs(a, b) >= 4
    c = _run(tmp_path, "sq16_pbc", "_f32", extra + "batch_vectors 4\n", precision=g.FP32)
    assert _same_outputs(a, c, tol=1e-6) >= 4


def test_groups_in_the_fp32r_form(tmp_path):
    """The FP32R moment form (FP32 vectors and hoppings, the recurrence in FP32) on the
    groups: every .out row within 1e-6 of its peak of the FP64 run's, with the direct
    and with the symmetric (kpm_doubling) moment loop."""
    extra = "number_of_random_vectors 4\n"
    a = _run(tmp_path, "sq16_pbc", "_seq", extra)
    b = _run(tmp_path, "sq16_pbc", "_f32r", extra + "batch_vectors 4\n", precision=g.FP32R)
    assert _same_outputs(a, b, tol=1e-6) >= 4
    c = _run(tmp_path, "sq16_pbc", "_f32rd", extra + "batch_vectors 16\nkpm_doubling\n",
             precision=g.FP32R)
    assert _same_outputs(a, c, tol=1e-6) >= 4


def test_groups_refuse_checkpoints(tmp_path):
    d = str(tmp_path / "ck")
    shutil.copytree(fixture_dir("chain_z2"), d)
    with open(os.path.join(d, "para.in"), "a") as f:
        f.write("batch_vectors 4\ncheckpoint_every 2\n")
    with pytest.raises(g.GqtError) as e:
        g.lsqt(d)
    assert e.value.status == 4 and "batch_vectors" in str(e.value)
