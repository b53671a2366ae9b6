"""The reference's shipped review example examples/review/graphene/vacancy (graphene
with 200,000 vacancies: 19,800,000 sites with ragged rows, 3000 moments) through the
whole lsqt() run, DOS stage. Its shipped dos.out holds 10 rows, each one random vector
of an unseeded run (the rows differ from each other), so a seeded run can only agree
statistically: our row must lie within twice the spread of the shipped rows around
their mean, in the largest and in the root-mean-square deviation."""
from __future__ import annotations

import os
import shutil

import numpy as np
import pytest

import gpuqt_b200 as g
from conftest import EXAMPLES

pytestmark = pytest.mark.gpu


def test_review_graphene_vacancy_dos(tmp_path):
    src = os.path.join(EXAMPLES, "review_graphene_vacancy")
    d = str(tmp_path / "vacancy")
    os.makedirs(d)
    for f in ("lattice.in", "energy.in", "time_step.in"):
        shutil.copy(os.path.join(src, f), d)
    with open(os.path.join(src, "para.in")) as f:
        para = "".join(l for l in f if l.split() and l.split()[0] != "calculate_msd")
    with open(os.path.join(d, "para.in"), "w") as f:
        f.write(para)
    assert g.lsqt(d)
    ours = np.loadtxt(os.path.join(d, "dos.out"))
    shipped = np.loadtxt(os.path.join(src, "dos.out"))
    assert ours.shape == shipped.shape[1:]
    mean = shipped.mean(axis=0)
    peak = np.max(np.abs(mean))
    rows_max = np.max(np.abs(shipped - mean)) / peak
    rows_rms = np.sqrt(np.mean((shipped - mean) ** 2)) / peak
    assert np.all(np.isfinite(ours))
    assert np.max(np.abs(ours - mean)) / peak <= 2 * rows_max
    assert np.sqrt(np.mean((ours - mean) ** 2)) / peak <= 2 * rows_rms
