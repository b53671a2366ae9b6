"""The wavefront moment loop (gqt_ham_set_loop) against the step-by-step loop and the
reference build.

Both loops compute every Chebyshev vector with the same per-site arithmetic, so the
vectors are bit-identical; the moments are the same sums in another fixed order
(per-chunk, per-warp partials combined in chunk order), equal to 1e-12 relative per
moment, and equal to the reference build's to the same bound as the step loop."""
from __future__ import annotations

import numpy as np
import pytest

import gpuqt_b200 as g
from conftest import fixture_dir, ref_moments

pytestmark = pytest.mark.gpu

REL = 1e-12


def _rel(a, b):
    return float(np.max(np.hypot(a[0] - b[0], a[1] - b[1]) / np.hypot(b[0], b[1])))


@pytest.mark.parametrize("window,chunk", [(2, 256), (16, 1024), (64, 512), (7, 2048)])
def test_wave_loop_matches_step_loop_and_reference(window, chunk):
    m = g.Model.load(fixture_dir("square256"))
    H = g.Hamiltonian(m)
    x = g.Vector.from_host(*m.initial_state())
    M = m.n_moments
    step = g.moments(H, x, x, M)
    H.set_loop(window, chunk)
    wave = g.moments(H, x, x, M)
    w, chunks, halo = H.loop
    assert w == window and chunks == 65536 // chunk and 0 <= halo <= chunks // 4
    assert _rel(wave, step) <= REL
    assert _rel(wave, ref_moments("square256")) <= REL
    # a second run replays the captured loop and gives the same bits
    again = g.moments(H, x, x, M)
    assert np.array_equal(again[0], wave[0]) and np.array_equal(again[1], wave[1])
    H.set_loop(0)
    assert np.array_equal(g.moments(H, x, x, M)[0], step[0])


def test_wave_loop_with_left_and_right_apart():
    """A VAC-like moment set: left is the current operator applied to the state."""
    m = g.Model.load(fixture_dir("square256"))
    H = g.Hamiltonian(m)
    x = g.Vector.from_host(*m.initial_state())
    left = g.Vector(m.n)
    g.apply_current(H, x, left)
    step = g.moments(H, left, x, 300)
    H.set_loop(16, 512)
    wave = g.moments(H, left, x, 300)
    assert _rel(wave, step) <= REL


def test_wave_loop_does_not_apply_elsewhere():
    """Forms, vector counts and operators it does not cover run the step loop."""
    m = g.Model.load(fixture_dir("sq16_pbc"))  # 256 sites: too few chunks
    H = g.Hamiltonian(m)
    H.set_loop(16, 256)
    x = g.Vector.from_host(*m.initial_state())
    g.moments(H, x, x, m.n_moments)
    assert H.loop[2] == -2
    with pytest.raises(g.GqtError):
        H.set_loop(1)
    with pytest.raises(g.GqtError):
        H.set_loop(16, 300)


@pytest.mark.slow
def test_wave_loop_at_size_matches_reference_build():
    """Graphene 2,097,152 sites, all 3000 moments, against the reference build (the
    bound of tests/test_reference_at_size.py: 1e-12 relative plus the reference's own
    summation noise)."""
    m = g.Model.load(fixture_dir("graphene2m"))
    H = g.Hamiltonian(m)
    x = g.Vector.from_host(*m.initial_state())
    step = g.moments(H, x, x, m.n_moments)
    H.set_loop(16)
    wave = g.moments(H, x, x, m.n_moments)
    rr, ri = ref_moments("graphene2m")
    floor = 2.0 * float(np.max(np.abs(ri)))
    err = np.hypot(wave[0] - rr, wave[1] - ri)
    assert np.all(err <= REL * np.hypot(rr, ri) + floor)
    assert _rel(wave, step) <= REL
