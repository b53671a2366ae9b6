"""Lattices large enough that every thread of the step, operator and evolution kernels
runs several grid-stride iterations (1,048,576 and 2,097,152 sites): the pipelined
loops' hand-over from one element to the next is exercised here, which the small
fixtures (at most one element per thread) never reach. The two operator formats hold
the same numbers, so their per-site results must be bit-identical and their moments
equal to the order of the FP64 sums; the FP32-storage form must stay within 1e-6 of
FP64 in the DOS without being identical to it."""
from __future__ import annotations

import numpy as np
import pytest

import gpuqt_b200 as g
from gpuqt_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["square1m", "graphene2m"])
def lattice(request, tmp_path_factory):
    m = g.Model.load(W.config_dir(str(tmp_path_factory.mktemp(request.param)), request.param))
    return m, g.Hamiltonian(m), m.initial_state()


def _rel(a, b):
    return float(np.max(np.hypot(a[0] - b[0], a[1] - b[1])) / np.max(np.hypot(b[0], b[1])))


def _both(H, fn):
    out = []
    for fmt in (g.FORMAT_ELL, g.FORMAT_CODED):
        H.set_format(fmt)
        out.append(fn())
    H.set_format(g.FORMAT_CODED)
    return out


def test_formats_agree_at_size(lattice):
    m, H, phi = lattice
    assert H.format == g.FORMAT_CODED
    M = 300
    for prec in (g.FP64, g.FP32):
        x = g.Vector.from_host(*phi, precision=prec)
        a, b = _both(H, lambda: g.moments(H, x, x, M))
        assert _rel(a, b) <= 1e-12, prec

    def ops():
        x = g.Vector.from_host(*phi)
        y = g.Vector(m.n)
        g.apply_current(H, x, y)
        s = x.clone()
        g.evolve(H, 1, 5.0, s)
        sx = x.clone()
        g.evolvex(H, -1, 5.0, sx)
        return y.download() + s.download() + sx.download()
    a, b = _both(H, ops)
    for u, w in zip(a, b):
        np.testing.assert_array_equal(u, w)


@pytest.mark.parametrize("V", [1, 16])
def test_fp32_form_at_size(lattice, V):
    m, H, phi = lattice
    M = 400
    vecs = [phi] + [m.initial_state() for _ in range(V - 1)]
    re = np.stack([v[0] for v in vecs])
    im = np.stack([v[1] for v in vecs])
    x64 = g.Vector.from_host(phi[0], phi[1])
    X = g.Vector.from_host(re, im, nvec=V, precision=g.FP32)
    r64, i64 = g.moments(H, x64, x64, M)
    r32, i32 = g.moments(H, X, X, M)
    r32, i32 = np.atleast_2d(r32)[0], np.atleast_2d(i32)[0]
    e = m.energy
    d64 = g.chebyshev_summation(r64, i64, e, m.energy_max, m.volume)
    d32 = g.chebyshev_summation(r32, i32, e, m.energy_max, m.volume)
    err = float(np.max(np.abs(d32 - d64)) / np.max(np.abs(d64)))
    assert np.all(np.isfinite(d64)) and np.all(np.isfinite(d32))
    assert 0.0 < err <= 1e-6, err
