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


def _moments(mu_vec):
    re, im = mu_vec.download()
    return re + 1j * im


def _state(m, nvec):
    vecs = [m.initial_state() for _ in range(nvec)]
    return g.Vector.from_host(np.stack([v[0] for v in vecs]), np.stack([v[1] for v in vecs]),
                              nvec=nvec)


def _inner(state, left):
    re, im = g.inner_product(state, left)
    return np.asarray(re) + 1j * np.asarray(im)


def _close(got, want, what):
    got, want = np.atleast_1d(got), np.atleast_1d(want)
    assert np.all(np.abs(got - want) <= REL * np.abs(want)), (what, got, want)


# Rows of 4 (periodic, and open with vacancies), 3 (graphene) and of uneven length
# (general model: the kernel without a row bound), at 1, 4 and 16 vectors per call, in
# the operator's default format (coded where it has one) and on the ELL arrays.
@pytest.mark.parametrize("name,nvec,fmt", [("square256", 1, None), ("graphene_8x4", 1, None),
                                           ("sq12_open_vac", 1, None), ("general40", 1, None),
                                           ("square256", 4, None), ("graphene_8x4", 16, None),
                                           ("general40", 4, None), ("graphene_8x4", 1, "ell")])
def test_noalloc_step_matches_allocating_entry_points(name, nvec, fmt):
    m = g.Model.load(fixture_dir(name))
    H = g.Hamiltonian(m)
    if fmt == "ell":
        H.set_format(g.FORMAT_ELL)
    x = _state(m, nvec)
    h1, ref, out = (g.Vector(m.n, nvec=nvec) for _ in range(3))
    mu = g.Vector(nvec)  # device slots for nvec (re, im) moments
    g.apply(H, x, h1)
    g.kernel_polynomial(H, x, h1, ref)
    want_step = _inner(ref, x)
    want_first = _inner(h1, x)
    ref_re, ref_im = ref.download()
    h1_re, h1_im = h1.download()
    for call in range(2):  # two calls in a row share the static scratch
        out.zero()
        _noalloc(H, 1, x, h1, out, x, mu)
        got_re, got_im = out.download()
        np.testing.assert_array_equal(got_re, ref_re)
        np.testing.assert_array_equal(got_im, ref_im)
        _close(_moments(mu), want_step, ("step", call))

        _noalloc(H, 0, None, x, out, x, mu)
        got_re, got_im = out.download()
        np.testing.assert_array_equal(got_re, h1_re)
        np.testing.assert_array_equal(got_im, h1_im)
        _close(_moments(mu), want_first, ("first step", call))


def test_noalloc_step_rejects_aliased_outputs():
    m = g.Model.load(fixture_dir("sq16_pbc"))
    H = g.Hamiltonian(m)
    x, y = g.Vector.from_host(*m.initial_state()), g.Vector(m.n)
    mu = g.Vector(1)
    for t0, t1, out, left in ((x, y, y, x), (x, x, y, y)):  # out = t1; out = left
        with pytest.raises(g.GqtError) as e:
            _noalloc(H, 1, t0, t1, out, left, mu)
        assert e.value.status == 1 and "alias" in str(e.value)


def test_noalloc_step_rejects_other_forms():
    m = g.Model.load(fixture_dir("sq16_pbc"))
    H = g.Hamiltonian(m)
    x32 = g.Vector(m.n, precision=g.FP32)
    y32 = g.Vector(m.n, precision=g.FP32)
    mu = g.Vector(1)
    with pytest.raises(g.GqtError) as e:
        _noalloc(H, 1, x32, x32, y32, x32, mu)
    assert e.value.status == 1 and "FP64" in str(e.value)
