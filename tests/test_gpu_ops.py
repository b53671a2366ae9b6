"""Operator kernels on the GPU against the reference: every per-site result of the
FP64 form is bit-identical to the reference's CPU path (golden outputs of the
reference build, and the oracle for single terms)."""
from __future__ import annotations

import numpy as np
import pytest

import gpuqt_b200 as g
import oracle as O
from conftest import SMALL_FIXTURES, fixture_dir, ref_npz

pytestmark = pytest.mark.gpu


def _setup(name):
    m = g.Model.load(fixture_dir(name))
    H = g.Hamiltonian(m)
    phi = m.initial_state()
    return m, H, phi


def _eq(vec: g.Vector, ref2):
    re, im = vec.download()
    np.testing.assert_array_equal(re, ref2[0])
    np.testing.assert_array_equal(im, ref2[1])


@pytest.mark.parametrize("name", SMALL_FIXTURES)
def test_operators_bit_exact(name):
    m, H, phi = _setup(name)
    ops = ref_npz(name, "ops")
    dt = float(ops["dt"][0])
    x = g.Vector.from_host(*phi)
    _eq(x, ops["phi"])
    h1 = g.Vector(m.n)
    g.apply(H, x, h1)
    _eq(h1, ops["H"])
    out = g.Vector(m.n)
    g.apply_commutator(H, x, out)
    _eq(out, ops["commutator"])
    g.apply_current(H, x, out)
    _eq(out, ops["current"])
    g.kernel_polynomial(H, x, h1, out)
    _eq(out, ops["T2"])
    for d, key in ((1, "evolve_p"), (-1, "evolve_m")):
        s = x.clone()
        g.evolve(H, d, dt, s)
        _eq(s, ops[key])
    for d, key in ((1, "evolvex_p"), (-1, "evolvex_m")):
        s = x.clone()
        g.evolvex(H, d, dt, s)
        _eq(s, ops[key])


@pytest.mark.parametrize("name", ["sq12_open_vac", "graphene_8x4", "chain_z2", "general40"])
def test_single_terms_bit_exact(name):
    m, H, phi = _setup(name)
    om = O.Model(n=m.n, max_neighbor=m.max_neighbor, energy_max=m.energy_max, volume=m.volume,
                 neighbor_number=m.neighbor_number, neighbor_list=m.neighbor_list,
                 potential=m.potential, hopping_real=m.hopping_real,
                 hopping_imag=m.hopping_imag, xx=m.xx)
    rng = np.random.default_rng(11)
    vecs = [(rng.normal(size=m.n), rng.normal(size=m.n)) for _ in range(5)]
    d = [g.Vector.from_host(*v) for v in vecs]
    # chebyshev_01
    out = g.Vector(m.n)
    g.chebyshev_01(H, d[0], d[1], out, 0.3, -0.7, -1)
    _eq(out, O.chebyshev_01(m.n, vecs[0], vecs[1], 0.3, -0.7, -1))
    # chebyshev_2, all labels, with s2 aliasing s0 as the algorithms use it
    for label in (1, 2, 3, 4):
        acc = d[2].clone()
        s0 = d[0].clone()
        g.chebyshev_2(H, s0, d[1], s0, acc, 0.125 * label, label)
        t2, o = O.chebyshev_2(om, vecs[0], vecs[1], vecs[2], 0.125 * label, label)
        _eq(s0, t2)
        _eq(acc, o)
    # chebyshev_1x
    g.chebyshev_1x(H, d[3], out, 0.9)
    _eq(out, O.chebyshev_1x(m.n, vecs[3], 0.9))
    # chebyshev_2x, all labels
    for label in (1, 2, 3, 4):
        acc = d[4].clone()
        s2, s2x = g.Vector(m.n), g.Vector(m.n)
        g.chebyshev_2x(H, d[0], d[1], d[2], d[3], s2, s2x, acc, -0.25 * label, label)
        t2, t2x, o = O.chebyshev_2x(om, vecs[0], vecs[1], vecs[2], vecs[3], vecs[4],
                                    -0.25 * label, label)
        _eq(s2, t2)
        _eq(s2x, t2x)
        _eq(acc, o)


def test_vector_ops():
    rng = np.random.default_rng(5)
    n = 1000
    a = (rng.normal(size=n), rng.normal(size=n))
    b = (rng.normal(size=n), rng.normal(size=n))
    va, vb = g.Vector.from_host(*a), g.Vector.from_host(*b)
    va.add(vb)
    _eq(va, (a[0] + b[0], a[1] + b[1]))
    vc = g.Vector(n)
    vc.apply_sz(vb)
    sign = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    _eq(vc, (b[0] * sign, b[1] * sign))
    vc.copy_from(va)
    _eq(vc, (a[0] + b[0], a[1] + b[1]))
    vc.swap(vb)
    _eq(vb, (a[0] + b[0], a[1] + b[1]))
    _eq(vc, b)
    re, im = g.inner_product(vc, va)
    ar, ai = a[0] + b[0], a[1] + b[1]
    assert abs(re - np.sum(b[0] * ar + b[1] * ai)) < 1e-11
    assert abs(im - np.sum(b[1] * ar - b[0] * ai)) < 1e-11


def test_multi_vector_layout_roundtrip():
    rng = np.random.default_rng(9)
    n, V = 300, 4
    re, im = rng.normal(size=(V, n)), rng.normal(size=(V, n))
    for prec in (g.FP64, g.FP32):
        v = g.Vector.from_host(re, im, nvec=V, precision=prec)
        r2, i2 = v.download()
        if prec == g.FP64:
            np.testing.assert_array_equal(r2, re)
        else:
            np.testing.assert_array_equal(r2, re.astype(np.float32).astype(np.float64))
            np.testing.assert_array_equal(i2, im.astype(np.float32).astype(np.float64))


@pytest.mark.parametrize("name", ["graphene_8x4", "cubic6", "sq12_open_vac"])
def test_multi_vector_fp64_matches_single(name):
    m, H, phi = _setup(name)
    rng = np.random.default_rng(1)
    V = 4
    re, im = rng.normal(size=(V, m.n)), rng.normal(size=(V, m.n))
    X = g.Vector.from_host(re, im, nvec=V)
    Y = g.Vector(m.n, nvec=V)
    g.apply(H, X, Y)
    yr, yi = Y.download()
    for k in range(V):
        x = g.Vector.from_host(re[k], im[k])
        y = g.Vector(m.n)
        g.apply(H, x, y)
        r, i = y.download()
        np.testing.assert_array_equal(yr[k], r)
        np.testing.assert_array_equal(yi[k], i)


def test_errors_do_not_crash():
    m, H, phi = _setup("sq16_pbc")
    x = g.Vector.from_host(*phi)
    with pytest.raises(g.GqtError):
        g.apply(H, x, x)                    # output aliases the gathered input
    with pytest.raises(g.GqtError):
        g.chebyshev_2(H, x, x, x, x, 1.0, 5)  # bad label
    with pytest.raises(g.GqtError):
        g.evolve(H, 2, 1.0, x)               # bad direction
    wrong = g.Vector(m.n + 1)
    with pytest.raises(g.GqtError):
        g.apply(H, x, wrong)
    y32 = g.Vector(m.n, precision=g.FP32)
    with pytest.raises(g.GqtError):
        g.chebyshev_1x(H, y32, y32, 1.0)     # single terms take FP64 vectors
    g.sync()


@pytest.mark.parametrize("emax", [8.7, 5.0, 3.0000000000000004, 13.2, 1.0, 0.1, 7.3e5, 2.0 ** -120])
def test_division_by_energy_max_correctly_rounded(emax):
    """The FP64 form's a / E_max (FMA-based, library division at the range edges)
    against IEEE division on the host: a site with no neighbours and potential a,
    applied to x = 1, gives a / E_max. Random significands over the whole exponent
    range, subnormals, zeros of both signs and infinities."""
    rng = np.random.default_rng(int(emax * 1000) % 2**31)
    n = 1 << 20
    a = rng.uniform(1.0, 2.0, n) * np.exp2(rng.integers(-1074, 1024, n).astype(np.float64))
    a[: n // 2] = rng.uniform(-16.0, 16.0, n // 2)  # the operator's own range
    a *= np.where(rng.random(n) < 0.5, -1.0, 1.0)
    a[:8] = [0.0, -0.0, np.inf, -np.inf, 5e-324, -2.2250738585072014e-308, 1.7e308, 1.0]
    H = g.Hamiltonian(n=n, max_neighbor=1, energy_max=emax,
                      neighbor_number=np.zeros(n, np.int32),
                      neighbor_list=np.arange(n, dtype=np.int32), potential=a,
                      hopping_real=np.zeros(n), hopping_imag=np.zeros(n))
    x = g.Vector.from_host(np.ones(n), np.zeros(n))
    y = g.Vector(n)
    g.apply(H, x, y)
    re, _ = y.download()
    with np.errstate(over="ignore", under="ignore"):
        want = a / emax
    np.testing.assert_array_equal(re, want)
    assert np.array_equal(np.signbit(re), np.signbit(want))
