"""The FP32X form (FP32 storage with a BF16 residual, GQT_FP32X) of the moment
recurrence against the FP64 form on the same vectors.

FP32X keeps about 32 significant bits per element, so its moments stay within about
1e-9 of FP64 where the FP32-storage form's reach 1e-8 - 1e-7 of mu_0. The tolerances
written here: per moment 1e-9 of the largest moment; DOS and VAC rows 1e-6 relative
pointwise
(|X(E) - X64(E)| / |X64(E)| where |X64(E)| > 1 % of the row's peak) and 1e-8 of the
row's peak."""
from __future__ import annotations

import numpy as np
import pytest

import gpuqt_b200 as g
from conftest import fixture_dir
from gpuqt_b200 import precision_report as P

pytestmark = pytest.mark.gpu


def _check(m, mu64, mu):
    r = P.compare(g, m, mu64, mu)
    # per moment, relative to the largest moment (mu_0 where the spectrum lies inside
    # [-E_max, E_max]; the seeded general model's does not, and its moments grow)
    scale = np.max(np.hypot(mu64[0], mu64[1]))
    err = np.max(np.hypot(mu[0] - mu64[0], mu[1] - mu64[1]))
    assert err <= 1e-9 * scale, (err / scale, r)
    assert r["energy_rel_peak_max"] <= 1e-8, r
    assert r["energy_rel_in_band_max"] <= 1e-6, r
    return r


@pytest.mark.parametrize("name", ["square256", "graphene_8x4", "cubic6", "sq12_open_vac",
                                  "general40"])
def test_fp32x_dos_moments_match_fp64(name):
    m = g.Model.load(fixture_dir(name))
    H = g.Hamiltonian(m)
    x = g.Vector.from_host(*m.initial_state())
    mu64 = g.moments(H, x, x, m.n_moments)
    mu = g.moments(H, x, x, m.n_moments, precision=g.FP32X)
    _check(m, mu64, mu)
    # FP32X is not FP64: the stored vectors carry about 32 bits
    assert np.max(np.abs(mu[0] - mu64[0])) > 0.0


@pytest.mark.parametrize("name,nvec", [("graphene_8x4", 16), ("square256", 4)])
def test_fp32x_vector_blocks_match_fp64_per_vector(name, nvec):
    m = g.Model.load(fixture_dir(name))
    H = g.Hamiltonian(m)
    vecs = [m.initial_state() for _ in range(nvec)]
    X = g.Vector.from_host(np.stack([v[0] for v in vecs]), np.stack([v[1] for v in vecs]),
                           nvec=nvec)
    re, im = g.moments(H, X, X, m.n_moments, precision=g.FP32X)
    for k in (0, nvec - 1):
        x = g.Vector.from_host(*vecs[k])
        _check(m, g.moments(H, x, x, m.n_moments), (re[k], im[k]))


def test_fp32x_vac_moments_match_fp64():
    """VAC moment sets with left != right (current operator, evolved states)."""
    m = g.Model.load(fixture_dir("graphene_8x4"))
    H = g.Hamiltonian(m)
    phi = m.initial_state()
    a = P.vac_moments(g, m, H, phi, g.FP64, len(m.time_step))
    b = P.vac_moments(g, m, H, phi, g.FP32X, len(m.time_step))
    for k in range(len(a)):
        _check(m, a[k], b[k])


@pytest.mark.parametrize("nvec", [1, 16])
def test_fp32x_doubled_matches_fp64(nvec):
    m = g.Model.load(fixture_dir("graphene_8x4"))
    H = g.Hamiltonian(m)
    vecs = [m.initial_state() for _ in range(nvec)]
    X = g.Vector.from_host(np.stack([v[0] for v in vecs]), np.stack([v[1] for v in vecs]),
                           nvec=nvec)
    re, im = g.moments_doubled(H, X, m.n_moments, precision=g.FP32X)
    re, im = np.atleast_2d(re), np.atleast_2d(im)
    x = g.Vector.from_host(*vecs[0])
    mu64 = g.moments(H, x, x, m.n_moments)
    r = P.compare(g, m, mu64, (re[0], im[0]))
    # the doubling identity's subtraction makes the error absolute (of mu_0's order)
    assert r["moment_rel_mu0_max"] <= 1e-9 and r["energy_rel_in_band_max"] <= 1e-6, r


@pytest.mark.slow
def test_fp32x_graphene4m_dos_and_20_vac_steps():
    r = P.report("graphene4m", vac_steps=20, fp32r=False)
    x = r["fp32x"]
    for q in ("dos", "vac"):
        assert x[q]["energy_rel_in_band_max"] <= 1e-6, (q, x[q])
        assert x[q]["energy_rel_peak_max"] <= 1e-8, (q, x[q])


def test_fp32x_is_internal_to_the_moment_loop():
    m = g.Model.load(fixture_dir("sq16_pbc"))
    with pytest.raises(g.GqtError):
        g.Vector(m.n, precision=g.FP32X)
    H = g.Hamiltonian(m)
    # FP32 has an 8-vector form, FP32X does not
    x = g.Vector.from_host(*[np.stack([v] * 8) for v in m.initial_state()], nvec=8,
                           precision=g.FP32)
    with pytest.raises(g.GqtError):  # no 8-vector FP32X launch
        g.moments(H, x, x, m.n_moments, precision=g.FP32X)
    B = g.Hamiltonian.batch([m, g.Model.load(fixture_dir("sq16_pbc"))])
    y = g.Vector(B.n)
    with pytest.raises(g.GqtError):  # one model only
        g.moments(B, y, y, 10, precision=g.FP32X)
