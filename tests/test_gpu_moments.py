"""KPM moments on the GPU against the reference (golden moments of the reference
build): the FP64 form to <= 1e-12 relative in every moment; the FP32-storage form to
<= 1e-6 in the DOS / VAC it produces."""
from __future__ import annotations

import numpy as np
import pytest

import gpuqt_b200 as g
import oracle as O
from conftest import ORACLE_FIXTURES, SMALL_FIXTURES, fixture_dir, ref_moments, ref_npz

pytestmark = pytest.mark.gpu

# Per-moment tolerance of the FP64 form: |mu - mu_ref| / |mu_ref| (complex modulus).
# The Chebyshev vectors are bit-identical to the reference's; the only difference is
# the order of the FP64 sum over sites (compensated here, sequential in the reference).
REL_FP64 = 1e-12


def rel_err(mr, mi, rr, ri):
    num = np.hypot(mr - rr, mi - ri)
    den = np.hypot(rr, ri)
    return float(np.max(num / den))


def _setup(name):
    m = g.Model.load(fixture_dir(name))
    H = g.Hamiltonian(m)
    x = g.Vector.from_host(*m.initial_state())
    return m, H, x


@pytest.mark.parametrize("name", SMALL_FIXTURES + ["square256"])
def test_dos_moments_fp64(name):
    m, H, x = _setup(name)
    rr, ri = ref_moments(name)
    mr, mi = g.moments(H, x, x, len(rr))
    assert rel_err(mr, mi, rr, ri) <= REL_FP64
    # Normalised by the largest moment: the seeded general model's spectrum is not
    # inside [-E_max, E_max], so its moments grow instead of staying near mu_0.
    assert np.max(np.abs(mr - rr)) <= 1e-14 * np.max(np.abs(rr))


@pytest.mark.parametrize("name", ORACLE_FIXTURES + ["sq20_charge", "general40"])
def test_vac_msd_moments_fp64(name):
    """The moment sets of find_vac / find_msd, evolution included."""
    m, H, x = _setup(name)
    M = m.n_moments
    ts = m.time_step
    for which in ("vacmom", "msdmom"):
        ref = ref_npz(name, which)
        if which == "vacmom":
            got = _vac_moments(m, H, x, M, ts)
        else:
            got = _msd_moments(m, H, x, M, ts)
        for k in range(len(ts)):
            assert rel_err(got[k][0], got[k][1], ref["re"][k], ref["im"][k]) <= REL_FP64, (
                which, k)


def _vac_moments(m, H, phi, M, ts):
    left, right, lcopy = phi.clone(), phi.clone(), g.Vector(m.n, precision=phi.precision)
    g.apply_current(H, left, right)
    out = []
    for k in range(len(ts)):
        g.apply_current(H, left, lcopy)
        out.append(g.moments(H, right, lcopy, M))
        if k < len(ts) - 1:
            g.evolve(H, -1, ts[k] * m.energy_max, left)
            g.evolve(H, -1, ts[k] * m.energy_max, right)
    return out


def _msd_moments(m, H, phi, M, ts):
    state, sx, copy = phi.clone(), phi.clone(), g.Vector(m.n, precision=phi.precision)
    g.evolve(H, 1, ts[0] * m.energy_max, state)
    g.evolvex(H, 1, ts[0] * m.energy_max, sx)
    out = []
    for k in range(len(ts)):
        out.append(g.moments(H, sx, sx, M))
        if k < len(ts) - 1:
            dt = ts[k + 1] * m.energy_max
            copy.copy_from(state)
            g.evolvex(H, 1, dt, copy)
            g.evolve(H, 1, dt, sx)
            sx.add(copy)
            g.evolve(H, 1, dt, state)
    return out


def test_square256_vac_fp64():
    m, H, x = _setup("square256")
    ref = ref_npz("square256", "vacmom")
    got = _vac_moments(m, H, x, m.n_moments, m.time_step)
    for k in range(len(m.time_step)):
        assert rel_err(got[k][0], got[k][1], ref["re"][k], ref["im"][k]) <= REL_FP64


def test_moments_are_deterministic():
    m, H, x = _setup("graphene_8x4")
    a = g.moments(H, x, x, 300)
    b = g.moments(H, x, x, 300)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])


def test_single_moment_and_two_stage_api():
    m, H, x = _setup("sq16_pbc")
    rr, ri = ref_moments("sq16_pbc")
    mr, mi = g.moments(H, x, x, 1)
    assert mr.size == 1 and abs(mr[0] - rr[0]) <= 1e-13 * abs(rr[0])
    re, im = g.inner_product(x, x)
    assert abs(re - rr[0]) <= 1e-13 * abs(rr[0])


def test_batched_fp64_matches_single_vectors():
    m = g.Model.load(fixture_dir("graphene_8x4"))
    H = g.Hamiltonian(m)
    V = 4
    phis = [m.initial_state() for _ in range(V)]
    X = g.Vector.from_host(np.stack([p[0] for p in phis]), np.stack([p[1] for p in phis]),
                           nvec=V)
    br, bi = g.moments(H, X, X, 300)
    for k in range(V):
        x = g.Vector.from_host(*phis[k])
        sr, si = g.moments(H, x, x, 300)
        assert rel_err(br[k], bi[k], sr, si) <= 1e-13


def _dos_err(m, mu64, mu32):
    e = m.energy
    d64 = g.chebyshev_summation(mu64[0], mu64[1], e, m.energy_max, m.volume)
    d32 = g.chebyshev_summation(mu32[0], mu32[1], e, m.energy_max, m.volume)
    return float(np.max(np.abs(d32 - d64)) / np.max(np.abs(d64)))


@pytest.mark.parametrize("V", [1, 4, 16])
def test_fp32_form_dos_error(V):
    """FP32 vectors, FP64 operator and sums: DOS within 1e-6 of the FP64 result
    (largest deviation over the energy grid, relative to the DOS peak)."""
    m = g.Model.load(fixture_dir("square256"))
    H = g.Hamiltonian(m)
    phis = [m.initial_state() for _ in range(V)]
    re, im = np.stack([p[0] for p in phis]), np.stack([p[1] for p in phis])
    X64 = g.Vector.from_host(re, im, nvec=V)
    X32 = g.Vector.from_host(re, im, nvec=V, precision=g.FP32)
    M = m.n_moments
    r64, i64 = g.moments(H, X64, X64, M)
    r32, i32 = g.moments(H, X32, X32, M)
    r64, i64, r32, i32 = (np.atleast_2d(a) for a in (r64, i64, r32, i32))
    for k in range(V):
        assert _dos_err(m, (r64[k], i64[k]), (r32[k], i32[k])) <= 1e-6


def test_fp32_form_vac_error():
    m = g.Model.load(fixture_dir("square256"))
    H = g.Hamiltonian(m)
    phi = m.initial_state()
    x64 = g.Vector.from_host(*phi)
    x32 = g.Vector.from_host(*phi, precision=g.FP32)
    steps = m.time_step[:4]
    a = _vac_moments(m, H, x64, m.n_moments, steps)
    b = _vac_moments(m, H, x32, m.n_moments, steps)
    for k in range(len(steps)):
        assert _dos_err(m, a[k], b[k]) <= 1e-6


def test_fp32_evolution_close_to_fp64():
    m = g.Model.load(fixture_dir("graphene_8x4"))
    H = g.Hamiltonian(m)
    phi = m.initial_state()
    a, b = g.Vector.from_host(*phi), g.Vector.from_host(*phi, precision=g.FP32)
    g.evolve(H, 1, 13.2, a)
    g.evolve(H, 1, 13.2, b)
    ar, ai = a.download()
    br, bi = b.download()
    assert np.max(np.hypot(ar - br, ai - bi)) < 1e-6
    g.evolvex(H, -1, 13.2, a)
    g.evolvex(H, -1, 13.2, b)
    ar, ai = a.download()
    br, bi = b.download()
    assert np.max(np.hypot(ar - br, ai - bi)) / np.max(np.hypot(ar, ai)) < 1e-6


def test_moments_form_equals_fp32_vectors():
    """FP64 states with the FP32 recurrence (gqt_moments_form) run exactly the
    computation of FP32 vectors: the conversion rounds as the upload does."""
    m, H, x64 = _setup("graphene_8x4")
    re, im = x64.download()
    x32 = g.Vector.from_host(re, im, precision=g.FP32)
    a = g.moments(H, x64, x64, 300, precision=g.FP32)
    b = g.moments(H, x32, x32, 300)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    y = g.Vector(m.n)
    g.apply_current(H, x64, y)
    a = g.moments(H, y, x64, 300, precision=g.FP32)  # left != right
    y32 = g.Vector(m.n, precision=g.FP32)
    y32.convert_from(y)
    b = g.moments(H, y32, x32, 300)
    np.testing.assert_array_equal(a[0], b[0])


def test_vec_convert_roundtrip():
    rng = np.random.default_rng(4)
    re, im = rng.normal(size=(4, 500)), rng.normal(size=(4, 500))
    a = g.Vector.from_host(re, im, nvec=4)
    b = g.Vector(500, nvec=4, precision=g.FP32)
    b.convert_from(a)
    r32, i32 = b.download()
    np.testing.assert_array_equal(r32, re.astype(np.float32).astype(np.float64))
    c = g.Vector(500, nvec=4)
    c.convert_from(b)
    np.testing.assert_array_equal(c.download()[1], im.astype(np.float32).astype(np.float64))
