"""Deferred grid stages of the moment loop: the window bookkeeping.

In the moment loop each fused Chebyshev step writes its block partials to one row of
a slab, and one k_slab_combine launch per window of steps turns the rows into
moments. A window holds at most 256 steps and its slab at most 32 MiB of partials
(`max_grid` = 8 blocks per SM x 32 B x the sums per moment), so 16 vectors get
shorter windows than one. The step kernels and their grids do not depend on the
number of moments, so a moment set that ends on a window edge, or one step past it,
must equal the prefix of a longer set (whose windows are cut elsewhere) bit for bit.
The reference's golden moments of square256 (1000 moments, three window edges) are
checked by the FP64 parity tests.
"""
from __future__ import annotations

import numpy as np
import pytest

import gpuqt_b200 as g
from conftest import fixture_dir

pytestmark = pytest.mark.gpu


def _window(sums_per_moment: int) -> int:
    import torch

    sms = torch.cuda.get_device_properties(0).multi_processor_count
    per = sms * 8 * sums_per_moment * 32
    return max(8, min(256, (32 << 20) // per))


def _state(m, nvec, precision):
    phis = [m.initial_state() for _ in range(nvec)]
    if nvec == 1:
        return g.Vector.from_host(*phis[0], precision=precision)
    return g.Vector.from_host(np.stack([p[0] for p in phis]), np.stack([p[1] for p in phis]),
                              nvec=nvec, precision=precision)


@pytest.mark.parametrize("nvec,precision", [(1, g.FP64), (16, g.FP64), (16, g.FP32)])
def test_direct_loop_prefix_is_bit_identical(nvec, precision):
    m = g.Model.load(fixture_dir("square256"))
    H = g.Hamiltonian(m)
    x = _state(m, nvec, precision)
    w = _window(nvec)
    # Steps 2 .. M-1 are deferred: M = w + 2 fills one window exactly, w + 3 spills one
    # step into the next, 2 w + 2 fills two.
    long_r, long_i = g.moments(H, x, x, 2 * w + 40)
    for M in (3, w + 2, w + 3, 2 * w + 2):
        r, i = g.moments(H, x, x, M)
        np.testing.assert_array_equal(r, long_r[..., :M])
        np.testing.assert_array_equal(i, long_i[..., :M])


@pytest.mark.parametrize("nvec", [1, 16])
def test_symmetric_loop_prefix_is_bit_identical(nvec):
    m = g.Model.load(fixture_dir("square256"))
    H = g.Hamiltonian(m)
    x = _state(m, nvec, g.FP64)
    w = _window(2 * nvec)
    # Pair steps 2 .. K are deferred (K = M / 2): K = w + 1 fills one window.
    long_r, long_i = g.moments_doubled(H, x, 2 * (2 * w + 20))
    for M in (4, 2 * (w + 1), 2 * (w + 1) + 1, 2 * (w + 2)):
        r, i = g.moments_doubled(H, x, M)
        np.testing.assert_array_equal(r, long_r[..., :M])
        np.testing.assert_array_equal(i, long_i[..., :M])


def test_deferred_moments_match_direct_inner_products():
    """Moments 2 .. M-1 of the loop (deferred) against T_m built step by step with
    gqt_kernel_polynomial and reduced at once by gqt_inner_product (same FP64 vectors,
    another reduction grid): the 1e-12 relative tolerance of the FP64 parity tests."""
    m = g.Model.load(fixture_dir("square256"))
    H = g.Hamiltonian(m)
    x = _state(m, 1, g.FP64)
    M = _window(1) + 6
    mr, mi = g.moments(H, x, x, M)
    t_prev, t_cur = g.Vector(m.n), g.Vector(m.n)
    t_prev.copy_from(x)
    g.apply(H, x, t_cur)
    nxt = g.Vector(m.n)
    for k in range(2, M):
        g.kernel_polynomial(H, t_prev, t_cur, nxt)
        re, im = g.inner_product(nxt, x)
        want = complex(re, im)
        got = complex(mr[k], mi[k])
        assert abs(got - want) <= 1e-12 * max(abs(want), abs(complex(mr[0], mi[0]))), k
        t_prev, t_cur, nxt = t_cur, nxt, t_prev
