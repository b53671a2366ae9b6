"""The GQT_FP32R form: FP32 vectors and hoppings, the Chebyshev recurrence in FP32, the
moments summed in FP64 from the stored values.

Its DOS error against the FP64 form is held to 1e-6 of the DOS peak (2e-6 on the
128-site graphene fixture, whose few sharp levels amplify it); the errors at the
benchmark sizes (DOS, VAC and MSD) are asserted in test_gpu_precision.py. Its staged
and unstaged steps (and the two operator formats, and the 4-, 16- and 32-vector
launches) use the same arithmetic, so their moments agree to FP64 summation order
(1e-12 of the largest moment)."""
from __future__ import annotations

import numpy as np
import pytest

import gpuqt_b200 as g
from conftest import fixture_dir
from gpuqt_b200 import workloads as W

pytestmark = pytest.mark.gpu

DOS_BOUND = 1e-6  # of the DOS peak, against FP64
SMALL_BOUND = {"graphene_8x4": 2e-6}
REL = 1e-12


def _states(m, V, seed=3):
    rng = np.random.default_rng(seed)
    ph = rng.uniform(0.0, 2.0 * np.pi, size=(V, m.n))
    return np.cos(ph) / np.sqrt(m.n), np.sin(ph) / np.sqrt(m.n)


def _rel(a, b):
    scale = float(np.max(np.hypot(b[0], b[1])))
    return float(np.max(np.hypot(a[0] - b[0], a[1] - b[1]))) / scale


def _dos_err(m, got, ref):
    worst = 0.0
    for k in range(got[0].shape[0]):
        d1 = g.chebyshev_summation(ref[0][k], ref[1][k], m.energy, m.energy_max, m.volume)
        d2 = g.chebyshev_summation(got[0][k], got[1][k], m.energy, m.energy_max, m.volume)
        worst = max(worst, float(np.max(np.abs(d2 - d1)) / np.max(np.abs(d1))))
    return worst


@pytest.mark.parametrize("name", ["square256", "graphene_8x4", "cubic6", "sq12_open_vac"])
@pytest.mark.parametrize("V", [4, 16, 32])
def test_fp32r_dos_against_fp64(name, V):
    m = g.Model.load(fixture_dir(name))
    H = g.Hamiltonian(m)
    re, im = _states(m, V)
    X32 = g.Vector.from_host(re, im, nvec=V, precision=g.FP32)
    M = m.n_moments
    # the FP64 reference in blocks of 16 vectors (the FP64 form's widest launch)
    parts = []
    nb = min(V, 16)
    for b0 in range(0, V, nb):
        X64 = g.Vector.from_host(re[b0:b0 + nb], im[b0:b0 + nb], nvec=nb)
        parts.append(g.moments(H, X64, X64, M))
    ref = (np.concatenate([p[0] for p in parts]), np.concatenate([p[1] for p in parts]))
    got = g.moments(H, X32, X32, M, precision=g.FP32R)
    bound = SMALL_BOUND.get(name, DOS_BOUND)
    assert _dos_err(m, got, ref) <= bound
    if V == 16:
        # FP64 vectors are rounded to FP32 copies first: the same moments
        conv = g.moments(H, X64, X64, M, precision=g.FP32R)
        assert np.array_equal(conv[0], got[0]) and np.array_equal(conv[1], got[1])
        dbl = g.moments_doubled(H, X32, M, precision=g.FP32R)
        assert _dos_err(m, dbl, ref) <= bound


@pytest.mark.parametrize("name", ["square256", "graphene_8x4", "cubic6", "sq12_open_vac"])
def test_fp32r_staged_unstaged_and_formats_agree(name):
    m = g.Model.load(fixture_dir(name))
    H = g.Hamiltonian(m)
    V = 16
    X = g.Vector.from_host(*_states(m, V), nvec=V, precision=g.FP32)
    M = 200
    staged = g.moments(H, X, X, M, precision=g.FP32R)
    staged_d = g.moments_doubled(H, X, M, precision=g.FP32R)
    H.set_staging(-1)
    assert _rel(g.moments(H, X, X, M, precision=g.FP32R), staged) <= REL
    assert _rel(g.moments_doubled(H, X, M, precision=g.FP32R), staged_d) <= REL
    H.set_format(g.FORMAT_ELL)
    assert _rel(g.moments(H, X, X, M, precision=g.FP32R), staged) <= REL
    assert _rel(g.moments_doubled(H, X, M, precision=g.FP32R), staged_d) <= REL


@pytest.mark.parametrize("name", ["square256", "cubic6", "general40"])
def test_fp32r_four_vectors_match_sixteen(name):
    """The 4-vector launch (unstaged, one thread per site) and the 16-vector launch use
    the same arithmetic per element: the moments of the same vectors agree to FP64
    summation order, in the direct and (Hermitian operators) the symmetric loop."""
    m = g.Model.load(fixture_dir(name))
    H = g.Hamiltonian(m)
    re, im = _states(m, 16)
    X16 = g.Vector.from_host(re, im, nvec=16, precision=g.FP32)
    X4 = g.Vector.from_host(re[:4], im[:4], nvec=4, precision=g.FP32)
    M = 200
    a = g.moments(H, X16, X16, M, precision=g.FP32R)
    b = g.moments(H, X4, X4, M, precision=g.FP32R)
    assert _rel(b, (a[0][:4], a[1][:4])) <= REL
    if name == "general40":  # random hoppings, not Hermitian: no symmetric sets
        return
    a = g.moments_doubled(H, X16, M, precision=g.FP32R)
    b = g.moments_doubled(H, X4, M, precision=g.FP32R)
    assert _rel(b, (a[0][:4], a[1][:4])) <= REL


def test_fp32r_limits():
    m = g.Model.load(fixture_dir("sq16_pbc"))
    H = g.Hamiltonian(m)
    with pytest.raises(g.GqtError):
        g.Vector(m.n, nvec=16, precision=g.FP32R)  # an internal form of the moment loop
    X1 = g.Vector.from_host(*_states(m, 1), nvec=1, precision=g.FP32)
    with pytest.raises(g.GqtError):
        g.moments(H, X1, X1, 10, precision=g.FP32R)  # 4, 16 or 32 vectors
    X32 = g.Vector.from_host(*_states(m, 32), nvec=32, precision=g.FP32)
    with pytest.raises(g.GqtError):
        g.moments_doubled(H, X32, 10, precision=g.FP32R)  # at most 16 for symmetric sets
    # realisation batches: tests/test_gpu_batch.py


def test_fp32r_at_size(tmp_path):
    """Graphene 2,097,152 sites (E_max 8.7, W = 1.0), 16 vectors, all 3000 moments: the
    DOS of the direct and the symmetric loop within 1e-6 of the FP64 DOS peak."""
    m = g.Model.load(W.config_dir(str(tmp_path), "graphene2m"))
    H = g.Hamiltonian(m)
    V = 16
    re, im = _states(m, V)
    X64 = g.Vector.from_host(re, im, nvec=V)
    X32 = g.Vector.from_host(re, im, nvec=V, precision=g.FP32)
    M = m.n_moments
    ref = g.moments(H, X64, X64, M)
    assert _dos_err(m, g.moments(H, X32, X32, M, precision=g.FP32R), ref) <= DOS_BOUND
    assert _dos_err(m, g.moments_doubled(H, X32, M, precision=g.FP32R), ref) <= DOS_BOUND
