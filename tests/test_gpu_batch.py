"""Realisation batches: several models of different sizes and coordination in one
block-diagonal operator, one launch per Chebyshev step, moments per model. Each
model's moments must equal those of the model run alone."""
from __future__ import annotations

import numpy as np
import pytest

import gpuqt_b200 as g
from conftest import fixture_dir

pytestmark = pytest.mark.gpu

NAMES = ["sq16_pbc", "graphene_8x4", "cubic6", "sq12_open_vac"]


def _models():
    ms = [g.Model.load(fixture_dir(n)) for n in NAMES]
    return ms


def _phases(models, V):
    out = []
    for m in models:
        ph = [m.initial_state() for _ in range(V)]
        out.append((np.stack([p[0] for p in ph]), np.stack([p[1] for p in ph])))
    return out


def _rel(a, b):
    return float(np.max(np.hypot(a[0] - b[0], a[1] - b[1]) / np.hypot(b[0], b[1])))


@pytest.mark.parametrize("V", [1, 4, 16])
def test_batch_fp64_matches_models_alone(V):
    models = _models()
    B = g.Hamiltonian.batch(models)
    assert B.n_real == len(models)
    assert B.n % 256 == 0
    ph = _phases(models, V)
    X = g.Vector.from_host(*B.scatter(ph), nvec=V)
    M = 120
    br, bi = g.moments(B, X, X, M)
    assert br.shape == (len(models), V, M)
    for r, (m, p) in enumerate(zip(models, ph)):
        H = g.Hamiltonian(m)
        x = g.Vector.from_host(p[0], p[1], nvec=V)
        sr, si = g.moments(H, x, x, M)
        sr, si = np.atleast_2d(sr), np.atleast_2d(si)
        # the batch applies (h / E_max) x instead of (h x) / E_max: rounding differs
        assert _rel((br[r], bi[r]), (sr, si)) <= 1e-11, r


@pytest.mark.parametrize("V", [4, 16, 32])
def test_batch_fp32_dos_close_to_fp64(V):
    models = _models()
    B = g.Hamiltonian.batch(models)
    ph = _phases(models, V)
    X64 = g.Vector.from_host(*B.scatter(ph), nvec=V) if V in (1, 4, 16) else None
    X32 = g.Vector.from_host(*B.scatter(ph), nvec=V, precision=g.FP32)
    M = 200
    r32, i32 = g.moments(B, X32, X32, M)
    for r, m in enumerate(models):
        H = g.Hamiltonian(m)
        x = g.Vector.from_host(ph[r][0][0], ph[r][1][0])
        r64, i64 = g.moments(H, x, x, M)
        d64 = g.chebyshev_summation(r64, i64, m.energy, m.energy_max, m.volume)
        d32 = g.chebyshev_summation(r32[r, 0], i32[r, 0], m.energy, m.energy_max, m.volume)
        assert np.max(np.abs(d32 - d64)) <= 1e-6 * np.max(np.abs(d64)), r
    del X64


def test_batch_rejects_evolution():
    B = g.Hamiltonian.batch(_models()[:2])
    x = g.Vector(B.n)
    with pytest.raises(g.GqtError) as e:
        g.evolve(B, 1, 1.0, x)
    assert e.value.status == 6


def test_autotuner_picks_a_candidate():
    B = g.Hamiltonian.batch(_models())
    best, rates = g.autotune_nvec(B, g.FP32, 20, [4, 8, 16, 32])
    assert best in (4, 8, 16, 32)
    assert all(v > 0 for v in rates.values())
    assert rates[best] == max(rates.values())


@pytest.mark.parametrize("tile", [256, 512, 1024])
def test_batch_tile_sizes_give_the_same_moments(tile):
    """Every tile size the step can run with (the autotuner's choice) gives each model
    the moments of the model run alone (to 1e-11, the bound of the batch against single
    runs above: the sums group differently), the deferred window reductions included
    (M = 120 > one window), in the direct and the symmetric (pair) loop."""
    models = _models()
    B = g.Hamiltonian.batch(models)
    assert B.n % 1024 == 0 and B.batch_tile == 256
    B.set_batch_tile(tile)
    assert B.batch_tile == tile
    ph = _phases(models, 4)
    X = g.Vector.from_host(*B.scatter(ph), nvec=4)
    M = 120
    re, im = g.moments(B, X, X, M)
    dr, di = g.moments_doubled(B, X, M)
    for r, m in enumerate(models):
        H = g.Hamiltonian(m)
        for v in (0, 3):
            x = g.Vector.from_host(ph[r][0][v], ph[r][1][v])
            ref = g.moments(H, x, x, M)
            assert _rel((re[r, v], im[r, v]), ref) <= 1e-11
            assert np.max(np.hypot(dr[r, v] - ref[0], di[r, v] - ref[1])) <= (
                1e-11 * np.max(np.hypot(*ref)))
    with pytest.raises(g.GqtError):
        B.set_batch_tile(384)
    single = g.Hamiltonian(models[0])
    assert single.batch_tile == 0
    with pytest.raises(g.GqtError):
        single.set_batch_tile(256)
