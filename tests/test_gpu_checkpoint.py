"""Checkpoint / resume of the lsqt run (gqt_lsqt_run) and the raw moment output
(para.in `output_moments`), on the GPU. A run stopped every few rows and resumed,
with junk appended to an output file after each stop (rows a crashed process wrote
after its last checkpoint), must write the same bytes as an uninterrupted run, and
both must match the reference build's .out files. The raw moments must be the
moments of the .out rows (same rows, same order; damping and summation of them give
the printed values) and, for the first DOS row, the reference's raw moments."""
from __future__ import annotations

import os
import shutil

import numpy as np
import pytest

import gpuqt_b200 as g
from conftest import REF, fixture_dir, ref_moments
from test_gpu_golden import _compare, _read

pytestmark = pytest.mark.gpu

CASES = ["sq16_pbc", "chain_z2", "general_spin"]  # VAC0/VAC/MSD; 2 vectors; spin + LDOS


def _copy(name, dst, extra):
    os.makedirs(dst)
    for f in os.listdir(fixture_dir(name)):
        if f.endswith(".in"):
            shutil.copy(os.path.join(fixture_dir(name), f), dst)
    with open(os.path.join(dst, "para.in"), "a") as f:
        f.write(extra)


def _outputs(d):
    return {f: open(os.path.join(d, f), "rb").read() for f in sorted(os.listdir(d))
            if f.endswith((".out", ".bin"))}


@pytest.mark.parametrize("name", CASES)
def test_resumed_run_writes_the_same_bytes(name, tmp_path):
    a, b = str(tmp_path / "a"), str(tmp_path / "b")
    _copy(name, a, "output_moments\n")
    _copy(name, b, "output_moments\ncheckpoint_every 2\n")
    assert g.lsqt(a)
    assert not os.path.exists(os.path.join(a, "lsqt.checkpoint"))
    stops = 0
    while not g.lsqt(b, max_rows=3):
        stops += 1
        assert os.path.exists(os.path.join(b, "lsqt.checkpoint"))
        with open(os.path.join(b, "dos.out"), "a") as f:
            f.write("1 2 3 partial row\n")
        assert stops < 40
    assert stops >= 2
    assert not os.path.exists(os.path.join(b, "lsqt.checkpoint"))
    out_a, out_b = _outputs(a), _outputs(b)
    assert sorted(out_a) == sorted(out_b)
    for f in out_a:
        assert out_a[f] == out_b[f], f
    found = 0
    for f in ("dos.out", "vac0.out", "vac.out", "msd.out", "S.out", "ldos.out"):
        ref = os.path.join(REF, name, f)
        if os.path.exists(ref):
            _compare(os.path.join(b, f), ref)
            found += 1
    assert found >= 2


def test_raw_moments_are_the_rows_moments(tmp_path):
    name = "sq16_pbc"
    d = str(tmp_path / "m")
    _copy(name, d, "output_moments\n")
    assert g.lsqt(d)
    m = g.Model.load(d)
    for stem in ("dos", "vac0", "vac", "msd"):
        re, im = g.read_moments(os.path.join(d, stem + "_moments.bin"))
        rows = _read(os.path.join(d, stem + ".out"))
        assert re.shape == (len(rows), m.n_moments)
        for k, row in enumerate(rows):
            dos = g.chebyshev_summation(re[k], im[k], m.energy, m.energy_max, m.volume)
            fin = np.isfinite(dos)
            assert np.allclose(dos[fin], row[fin], rtol=1e-5, atol=1e-12 * np.max(np.abs(row[fin])))
    rr, ri = ref_moments(name)
    re, im = g.read_moments(os.path.join(d, "dos_moments.bin"))
    err = np.hypot(re[0] - rr, im[0] - ri) / np.hypot(rr, ri)
    assert float(np.max(err)) <= 1e-12


def test_resume_refuses_changed_run_or_shortened_output(tmp_path):
    d = str(tmp_path / "c")
    _copy("chain_z2", d, "checkpoint_every 1\n")
    assert not g.lsqt(d, max_rows=2)
    with open(os.path.join(d, "para.in")) as f:
        para = f.read()
    with open(os.path.join(d, "para.in"), "w") as f:
        f.write(para.replace("number_of_moments 120", "number_of_moments 110"))
    with pytest.raises(g.GqtError) as e:
        g.lsqt(d)
    assert e.value.status == 4 and "different run" in str(e.value)
    with open(os.path.join(d, "para.in"), "w") as f:
        f.write(para)
    with open(os.path.join(d, "dos.out"), "w") as f:
        f.write("")
    with pytest.raises(g.GqtError) as e:
        g.lsqt(d)
    assert e.value.status == 4 and "shorter" in str(e.value)
