"""The coded operator format (one byte per ELL entry into a table of the distinct
(j - i, hopping, xx) entries) against the plain ELL format: the same doubles in the
same order, so every result must be bit-identical, in every form."""
from __future__ import annotations

import numpy as np
import pytest

import gpuqt_b200 as g
from conftest import fixture_dir, ref_npz

pytestmark = pytest.mark.gpu

LATTICES = ["sq16_pbc", "sq12_open_vac", "graphene_8x4", "cubic6", "chain_z2", "sq20_charge"]


def _both(name):
    m = g.Model.load(fixture_dir(name))
    H = g.Hamiltonian(m)
    return m, H


@pytest.mark.parametrize("name", LATTICES)
def test_lattices_get_a_coded_form(name):
    m, H = _both(name)
    assert H.format == g.FORMAT_CODED and 0 < H.n_codes <= 256


def _random_ell(n, z, seed):
    rng = np.random.default_rng(seed)
    nl = rng.integers(0, n, size=(n, z)).astype(np.int32)
    return dict(n=n, max_neighbor=z, energy_max=9.0, neighbor_number=np.full(n, z, np.int32),
                neighbor_list=nl.ravel(), potential=rng.uniform(-0.5, 0.5, n),
                hopping_real=rng.uniform(-1.5, -0.5, n * z), hopping_imag=rng.uniform(-.2, .2, n * z),
                xx=rng.uniform(-3, 3, n * z))


def test_many_distinct_entries_stay_ell():
    H = g.Hamiltonian(**_random_ell(400, 3, 5))  # 1200 distinct (j - i, hopping, xx)
    assert H.n_codes == 0 and H.format == g.FORMAT_ELL
    with pytest.raises(g.GqtError):
        H.set_format(g.FORMAT_CODED)
    H.set_format(g.FORMAT_ELL)
    with pytest.raises(g.GqtError):
        H.set_format(7)


def test_small_general_model_coded():
    """A general model with at most 256 distinct entries (general40: 40 sites) is coded
    too, and its results equal the ELL format's."""
    m, H = _both("general40")
    assert H.format == g.FORMAT_CODED
    x = g.Vector.from_host(*m.initial_state())
    res = []
    for fmt in (g.FORMAT_ELL, g.FORMAT_CODED):
        H.set_format(fmt)
        y = g.Vector(m.n)
        g.apply_current(H, x, y)
        res.append(y.download() + g.moments(H, x, y, 100))
    for a, b in zip(*res):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("name", LATTICES)
def test_operators_identical_across_formats(name):
    m, H = _both(name)
    ops = ref_npz(name, "ops")
    dt = float(ops["dt"][0])
    x = g.Vector.from_host(*m.initial_state())
    res = {}
    for fmt in (g.FORMAT_ELL, g.FORMAT_CODED):
        H.set_format(fmt)
        out = []
        for fn in (g.apply, g.apply_commutator, g.apply_current):
            y = g.Vector(m.n)
            fn(H, x, y)
            out.append(y.download())
        for d in (1, -1):
            s = x.clone()
            g.evolve(H, d, dt, s)
            out.append(s.download())
            s = x.clone()
            g.evolvex(H, d, dt, s)
            out.append(s.download())
        out.append(g.moments(H, x, x, 200))
        res[fmt] = out
    for a, b in zip(res[g.FORMAT_ELL], res[g.FORMAT_CODED]):
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])
    # and the coded path is the reference's arithmetic
    np.testing.assert_array_equal(np.stack(res[g.FORMAT_CODED][0]), ops["H"])


@pytest.mark.parametrize("prec,V", [(g.FP32, 16), (g.FP64, 4), (g.FP32, 1)])
def test_batched_forms_identical_across_formats(prec, V):
    m, H = _both("graphene_8x4")
    ph = [m.initial_state() for _ in range(V)]
    X = g.Vector.from_host(np.stack([p[0] for p in ph]), np.stack([p[1] for p in ph]), nvec=V,
                           precision=prec)
    H.set_format(g.FORMAT_ELL)
    a = g.moments(H, X, X, 150)
    H.set_format(g.FORMAT_CODED)
    b = g.moments(H, X, X, 150)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])


def test_batch_identical_across_formats():
    models = [g.Model.load(fixture_dir(n)) for n in ("sq16_pbc", "graphene_8x4", "cubic6")]
    B = g.Hamiltonian.batch(models)
    assert B.format == g.FORMAT_CODED
    ph = []
    for mm in models:
        p = [mm.initial_state() for _ in range(4)]
        ph.append((np.stack([q[0] for q in p]), np.stack([q[1] for q in p])))
    X = g.Vector.from_host(*B.scatter(ph), nvec=4, precision=g.FP32)
    a = g.moments(B, X, X, 120)
    B.set_format(g.FORMAT_ELL)
    b = g.moments(B, X, X, 120)
    np.testing.assert_array_equal(a[0], b[0])
