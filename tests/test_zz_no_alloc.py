"""gqt_chebyshev_step_noalloc against the library's allocating entry points.

The no-allocation step is for callers that drive the Chebyshev recurrence
themselves and cannot let the library call cudaMalloc. Examples are a host that has
already given all of HBM to its own pool allocator, and a loop that is being timed or
captured, where cudaMalloc's implicit device synchronisation is not allowed. Its
reduction scratch lives in a static device array shared by all calls, so this test
calls it twice in a row and checks both calls against gqt_apply /
gqt_kernel_polynomial (bit-identical output vector) and gqt_inner_product (moment,
within the 1e-12 relative tolerance of the FP64 parity tests). This file is
collected last so that a run stopping at the first failure has run every other
test first.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import gpuqt_b200 as g
from conftest import fixture_dir

pytestmark = pytest.mark.gpu

REL = 1e-12


def _noalloc(H, mode, t0, t1, out, left, mu):
    g._call("gqt_chebyshev_step_noalloc", H.h, mode, t0.h if t0 is not None else None,
            t1.h, out.h, left.h, ctypes.c_void_p(mu.data_ptr))


def _moment(mu_vec):
    re, im = mu_vec.download()
    return complex(re[0], im[0])


@pytest.mark.parametrize("name", ["square256", "graphene_8x4", "sq12_open_vac"])
def test_noalloc_step_matches_allocating_entry_points(name):
    m = g.Model.load(fixture_dir(name))
    H = g.Hamiltonian(m)
    x = g.Vector.from_host(*m.initial_state())
    h1, ref, out = g.Vector(m.n), g.Vector(m.n), g.Vector(m.n)
    mu = g.Vector(1)  # device slot for one (re, im) moment
    g.apply(H, x, h1)
    g.kernel_polynomial(H, x, h1, ref)
    want_step = complex(*g.inner_product(ref, x))
    want_first = complex(*g.inner_product(h1, x))
    ref_re, ref_im = ref.download()
    h1_re, h1_im = h1.download()
    for call in range(2):  # two calls in a row share the static scratch
        out.zero()
        _noalloc(H, 1, x, h1, out, x, mu)
        got_re, got_im = out.download()
        np.testing.assert_array_equal(got_re, ref_re)
        np.testing.assert_array_equal(got_im, ref_im)
        got = _moment(mu)
        assert abs(got - want_step) <= REL * abs(want_step), (call, got, want_step)

        _noalloc(H, 0, None, x, out, x, mu)
        got_re, got_im = out.download()
        np.testing.assert_array_equal(got_re, h1_re)
        np.testing.assert_array_equal(got_im, h1_im)
        got = _moment(mu)
        assert abs(got - want_first) <= REL * abs(want_first), (call, got, want_first)


def test_noalloc_step_rejects_other_forms():
    m = g.Model.load(fixture_dir("sq16_pbc"))
    H = g.Hamiltonian(m)
    x32 = g.Vector(m.n, precision=g.FP32)
    y32 = g.Vector(m.n, precision=g.FP32)
    mu = g.Vector(1)
    with pytest.raises(g.GqtError) as e:
        _noalloc(H, 1, x32, x32, y32, x32, mu)
    assert e.value.status == 1 and "FP64" in str(e.value)
