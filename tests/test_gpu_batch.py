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


def _pow2_models(tmp_path):
    """Models whose E_max is a power of two: the batch's pre-divided hoppings h / E_max
    equal the single model's h * (1 / E_max) bit for bit, so the FP32R arithmetic is the
    same in both. Square lattices of three sizes (one odd, one with open boundaries and
    vacancy-free ragged rows) and graphene (rows of 3 padded to 4 in the batch)."""
    from gpuqt_b200 import workloads as W
    specs = [("square", (24, 24, 1), -1.0, 2.0, 8.0), ("square", (40, 40, 1), -1.0, 1.0, 8.0),
             ("square", (17, 17, 1), -1.0, 3.0, 8.0), ("graphene", (8, 4, 1), -2.7, 1.0, 16.0)]
    out = []
    for k, (kind, cells, t, w, e) in enumerate(specs):
        d = W.write_input_dir(str(tmp_path / f"m{k}"), kind, cells, hopping=t, anderson=w,
                              energy_max=e, moments=160, calculate=(), seed=20 + k)
        out.append(g.Model.load(d))
    return out


@pytest.mark.parametrize("V", [16, 32])
def test_batch_fp32r_staged_matches_models_alone(tmp_path, V):
    """The staged FP32R batch step (each model's own windows, sums flushed per model)
    against each model run alone in the FP32R form: the same T_m per element, moments
    to FP64 summation order; the symmetric loop as well (16 vectors)."""
    models = _pow2_models(tmp_path)
    B = g.Hamiltonian.batch(models)
    stages, slots = B.stage_plan(V, g.FP32R)
    assert stages >= 2 and slots >= 2, (stages, slots)
    assert B.stage_plan(V, g.FP32) == (0, 0)  # the FP32 form's batch step is not staged
    ph = _phases(models, V)
    X = g.Vector.from_host(*B.scatter(ph), nvec=V, precision=g.FP32)
    M = 160
    br, bi = g.moments(B, X, X, M, precision=g.FP32R)
    dr = di = None
    if V == 16:
        dr, di = g.moments_doubled(B, X, M, precision=g.FP32R)
    for r, (m, p) in enumerate(zip(models, ph)):
        H = g.Hamiltonian(m)
        x = g.Vector.from_host(p[0], p[1], nvec=V, precision=g.FP32)
        sr, si = g.moments(H, x, x, M, precision=g.FP32R)
        scale = float(np.max(np.hypot(sr, si)))
        assert float(np.max(np.hypot(br[r] - sr, bi[r] - si))) <= 1e-12 * scale, r
        if V == 16:
            sr, si = g.moments_doubled(H, x, M, precision=g.FP32R)
            assert float(np.max(np.hypot(dr[r] - sr, di[r] - si))) <= 1e-12 * scale, r


def test_batch_fp32r_dos_close_to_fp64():
    models = _models()
    B = g.Hamiltonian.batch(models)
    V = 16
    ph = _phases(models, V)
    X32 = g.Vector.from_host(*B.scatter(ph), nvec=V, precision=g.FP32)
    M = 200
    r32, i32 = g.moments(B, X32, X32, M, precision=g.FP32R)
    for r, m in enumerate(models):
        H = g.Hamiltonian(m)
        x = g.Vector.from_host(ph[r][0][0], ph[r][1][0])
        r64, i64 = g.moments(H, x, x, M)
        d64 = g.chebyshev_summation(r64, i64, m.energy, m.energy_max, m.volume)
        d32 = g.chebyshev_summation(r32[r, 0], i32[r, 0], m.energy, m.energy_max, m.volume)
        bound = 2e-6 if NAMES[r] == "graphene_8x4" else 1e-6  # few sharp levels
        assert np.max(np.abs(d32 - d64)) <= bound * np.max(np.abs(d64)), r


def test_batch_fp32r_needs_the_staged_step():
    models = _models()[:2]
    B = g.Hamiltonian.batch(models)
    X = g.Vector(B.n, nvec=16, precision=g.FP32)
    B.set_staging(-1)
    with pytest.raises(g.GqtError):
        g.moments(B, X, X, 10, precision=g.FP32R)
    B.set_staging(0)
    X32 = g.Vector(B.n, nvec=32, precision=g.FP32)
    with pytest.raises(g.GqtError):  # symmetric sets: at most 16 vectors per launch
        g.moments_doubled(B, X32, 10, precision=g.FP32R)
    B.set_format(g.FORMAT_ELL)
    with pytest.raises(g.GqtError):
        g.moments(B, X, X, 10, precision=g.FP32R)


def test_batch_fp32r_staged_many_models(tmp_path):
    """32 square lattices (the most a batch takes) of 16^2 to 47^2 sites, each padded to
    1024 sites: a block's tiles fall in many models, with models skipped between them
    (their slots zeroed), and the sums are flushed at every model change. Against each
    model run alone in the FP32R form (E_max a power of two: the same operator)."""
    from gpuqt_b200 import workloads as W
    models = []
    for k in range(32):
        L = 16 + k
        d = W.write_input_dir(str(tmp_path / f"m{k}"), "square", (L, L, 1), hopping=-1.0,
                              anderson=0.5 + 0.1 * k, energy_max=8.0, moments=64,
                              calculate=(), seed=100 + k)
        models.append(g.Model.load(d))
    B = g.Hamiltonian.batch(models)
    V, M = 16, 64
    assert B.stage_plan(V, g.FP32R)[0] >= 2
    ph = _phases(models, V)
    X = g.Vector.from_host(*B.scatter(ph), nvec=V, precision=g.FP32)
    br, bi = g.moments(B, X, X, M, precision=g.FP32R)
    dr, di = g.moments_doubled(B, X, M, precision=g.FP32R)
    for r, (m, p) in enumerate(zip(models, ph)):
        H = g.Hamiltonian(m)
        x = g.Vector.from_host(p[0], p[1], nvec=V, precision=g.FP32)
        sr, si = g.moments(H, x, x, M, precision=g.FP32R)
        scale = float(np.max(np.hypot(sr, si)))
        assert float(np.max(np.hypot(br[r] - sr, bi[r] - si))) <= 1e-12 * scale, r
        sr, si = g.moments_doubled(H, x, M, precision=g.FP32R)
        assert float(np.max(np.hypot(dr[r] - sr, di[r] - si))) <= 1e-12 * scale, r


def test_autotuner_probes_the_fp32r_batch():
    """The autotuner runs the FP32R form on FP32 probe vectors and picks one of the
    candidates it could time; the batch then runs with it."""
    models = _models()
    B = g.Hamiltonian.batch(models)
    best, rates = g.autotune_nvec(B, g.FP32R, 10, [16, 32])
    assert best in (16, 32) and all(rates[v] > 0 for v in (16, 32)), rates
    X = g.Vector(B.n, nvec=best, precision=g.FP32)
    X.upload(*B.scatter(_phases(models, best)))
    r, i = g.moments(B, X, X, 20, precision=g.FP32R)
    assert np.all(np.isfinite(r)) and np.all(np.isfinite(i))
