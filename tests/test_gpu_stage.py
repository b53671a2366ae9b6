"""The staged step of the FP32 moment loops (gqt_ham_set_staging) against the unstaged
step.

Both compute every T_m with the same per-element arithmetic, so the vectors are the
same; the moments are the same per-thread FP64 sums taken over the sites in another
order, equal to 1e-12 of the largest moment. The fixtures cover rows of 3, 4 and 6
entries, ragged rows (vacancies: padding entries of offset 0 and hopping 0), periodic
wraps gathered from global memory (square 256^2: offsets +-255 and +-65280 fall in no
window) or staged (16^2: every offset is frequent), and a last tile that is cut short."""
from __future__ import annotations

import numpy as np
import pytest

import gpuqt_b200 as g
from conftest import fixture_dir
from gpuqt_b200 import workloads as W

pytestmark = pytest.mark.gpu

REL = 1e-12
CASES = ["square256", "graphene_8x4", "cubic6", "sq12_open_vac", "sq16_pbc"]


def _states(m, V, seed=7):
    rng = np.random.default_rng(seed)
    ph = rng.uniform(0.0, 2.0 * np.pi, size=(V, m.n))
    return np.cos(ph) / np.sqrt(m.n), np.sin(ph) / np.sqrt(m.n)


def _rel(a, b):
    scale = float(np.max(np.hypot(b[0], b[1])))
    return float(np.max(np.hypot(a[0] - b[0], a[1] - b[1]))) / scale


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("V", [16, 32])
def test_staged_matches_unstaged(name, V):
    m = g.Model.load(fixture_dir(name))
    H = g.Hamiltonian(m)
    stages, wins = H.staging
    assert stages == 0 and 1 <= len(wins) <= 8
    assert wins[0][0] <= 0 <= wins[0][1]
    X = g.Vector.from_host(*_states(m, V), nvec=V, precision=g.FP32)
    M = 160
    H.set_staging(1)
    assert H.staging[0] == 1
    staged = g.moments(H, X, X, M)
    H.set_staging(-1)
    plain = g.moments(H, X, X, M)
    assert _rel(staged, plain) <= REL
    H.set_staging(0)  # automatic: staged on rows of 6 only
    auto = g.moments(H, X, X, M)
    if m.ell()["max_neighbor"] < 6:
        assert np.array_equal(auto[0], plain[0]) and np.array_equal(auto[1], plain[1])
    else:
        assert _rel(auto, plain) <= REL
    if V <= 16:
        H.set_staging(-1)
        plain_d = g.moments_doubled(H, X, M)
        H.set_staging(0)  # automatic: staged on rows of 6 only
        assert _rel(g.moments_doubled(H, X, M), plain_d) <= REL
        H.set_staging(1)
        assert _rel(g.moments_doubled(H, X, M), plain_d) <= REL
    for s in (2, 3, 4):
        H.set_staging(s)
        assert _rel(g.moments(H, X, X, M), plain) <= REL, s
    # a second run replays the captured loop and gives the same bits
    again = g.moments(H, X, X, M)
    got = g.moments(H, X, X, M)
    assert np.array_equal(again[0], got[0]) and np.array_equal(again[1], got[1])


def test_staging_windows_of_square_lattice():
    """square 256^2: +-1 (with 0) and +-256 are staged; the wraps +-255 and +-65280,
    taken by 256 rows each, are gathered from global memory."""
    m = g.Model.load(fixture_dir("square256"))
    H = g.Hamiltonian(m)
    _, wins = H.staging
    assert wins[0] == (-1, 1)
    assert sorted(wins[1:]) == [(-256, -256), (256, 256)]


def test_staged_left_and_right_apart():
    """A VAC-like moment set: left is the current operator applied to the state."""
    m = g.Model.load(fixture_dir("square256"))
    H = g.Hamiltonian(m)
    V = 16
    X = g.Vector.from_host(*_states(m, V), nvec=V, precision=g.FP32)
    L = g.Vector(m.n, nvec=V, precision=g.FP32)
    g.apply_current(H, X, L)
    H.set_staging(1)
    staged = g.moments(H, L, X, 120)
    H.set_staging(-1)
    assert _rel(staged, g.moments(H, L, X, 120)) <= REL


def test_staging_arguments():
    m = g.Model.load(fixture_dir("sq16_pbc"))
    H = g.Hamiltonian(m)
    for bad in (5, -2):
        with pytest.raises(g.GqtError):
            H.set_staging(bad)
    H.set_staging(1)
    H.set_format(g.FORMAT_ELL)
    V = 16
    X = g.Vector.from_host(*_states(m, V), nvec=V, precision=g.FP32)
    ell = g.moments(H, X, X, 50)  # the ELL arrays are never staged
    H.set_format(g.FORMAT_CODED)
    assert _rel(g.moments(H, X, X, 50), ell) <= REL


def test_stage_plan_leaves_out_windows_that_do_not_fit(tmp_path):
    """cubic 8 x 64 x 64: the periodic wraps along the short axis are taken by 1/8 of the
    entries, so the upload finds more windows than two stages of them fit in shared
    memory. The least used windows are left out (their entries gather from global
    memory) and the step stays staged, with the same moments as the unstaged step."""
    d = W.write_input_dir(str(tmp_path / "cubic"), "cubic", (8, 64, 64), anderson=16.5,
                          energy_max=15.0, moments=120, calculate=(), seed=13)
    m = g.Model.load(d)
    H = g.Hamiltonian(m)
    _, wins = H.staging
    V, M = 16, 120
    for prec in (g.FP32, g.FP32R):
        stages, used = H.stage_plan(V, prec)
        assert stages >= 2 and 1 <= used < len(wins), (prec, stages, used, wins)
        assert H.stage_plan(V, prec, symmetric=True)[0] >= 2
    assert H.stage_plan(V, g.FP64) == (0, 0)
    X = g.Vector.from_host(*_states(m, V), nvec=V, precision=g.FP32)
    staged = {p: g.moments(H, X, X, M, precision=p) for p in (g.FP32, g.FP32R)}
    staged_d = g.moments_doubled(H, X, M, precision=g.FP32R)
    H.set_staging(-1)
    assert H.stage_plan(V, g.FP32R) == (0, 0)
    for p in (g.FP32, g.FP32R):
        assert _rel(staged[p], g.moments(H, X, X, M, precision=p)) <= REL
    assert _rel(staged_d, g.moments_doubled(H, X, M, precision=g.FP32R)) <= REL
