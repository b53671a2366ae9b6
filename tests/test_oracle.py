"""The oracle (oracle/lsqt_oracle.c) pinned against the reference itself: its shipped
example outputs, the golden fixtures generated by the reference's own build
(tests/golden/make_golden.py) and, where it is built here, the reference build live."""
from __future__ import annotations

import os

import numpy as np
import pytest

import oracle as O
from conftest import EXAMPLES, ORACLE_FIXTURES, fixture_dir, ref_moments, ref_npz


def test_mt19937_known_answer():
    # The C++ standard's check value: the 10000th output of the default-seeded engine.
    g = O.MT19937(5489)
    g.discard(9999)
    assert g.next() == 4123659995


def test_uniform_int_is_top_31_bits():
    a, b = O.MT19937(77), O.MT19937(77)
    for _ in range(1000):
        assert a.uniform_int() == b.next() >> 1


@pytest.mark.parametrize("name", ORACLE_FIXTURES)
def test_lattice_build_bit_exact(name):
    m, _ = O.load_model(fixture_dir(name))
    r = ref_npz(name, "ell")
    assert m.n == r["nn"].size
    np.testing.assert_array_equal(m.neighbor_number, r["nn"])
    z = m.max_neighbor
    mask = np.arange(z)[None, :] < m.neighbor_number[:, None]
    for a, k in ((m.neighbor_list, "nl"), (m.hopping_real, "hr"), (m.hopping_imag, "hi"),
                 (m.xx, "xx")):
        np.testing.assert_array_equal(a.reshape(-1, z)[mask], r[k].reshape(-1, z)[mask])
    np.testing.assert_array_equal(m.potential, r["pot"])
    assert m.volume == r["meta"][1]


@pytest.mark.parametrize("name", ORACLE_FIXTURES)
def test_operators_bit_exact(name):
    m, g = O.load_model(fixture_dir(name))
    phi = O.random_phase_state(g, m.n)
    ops = ref_npz(name, "ops")
    dt = float(ops["dt"][0])
    np.testing.assert_array_equal(np.stack(phi), ops["phi"])
    h = O.apply(m, *phi)
    np.testing.assert_array_equal(np.stack(h), ops["H"])
    np.testing.assert_array_equal(np.stack(O.apply_commutator(m, *phi)), ops["commutator"])
    np.testing.assert_array_equal(np.stack(O.apply_current(m, *phi)), ops["current"])
    np.testing.assert_array_equal(np.stack(O.kernel_polynomial(m, phi, h)), ops["T2"])
    np.testing.assert_array_equal(np.stack(O.evolve(m, 1, dt, phi)), ops["evolve_p"])
    np.testing.assert_array_equal(np.stack(O.evolve(m, -1, dt, phi)), ops["evolve_m"])
    np.testing.assert_array_equal(np.stack(O.evolvex(m, 1, dt, phi)), ops["evolvex_p"])
    np.testing.assert_array_equal(np.stack(O.evolvex(m, -1, dt, phi)), ops["evolvex_m"])


@pytest.mark.parametrize("name", ORACLE_FIXTURES + ["square256"])
def test_moments_bit_exact(name):
    m, g = O.load_model(fixture_dir(name))
    phi = O.random_phase_state(g, m.n)
    rr, ri = ref_moments(name)
    mr, mi = O.find_moments(m, len(rr), phi, phi)
    np.testing.assert_array_equal(mr, rr)
    np.testing.assert_array_equal(mi, ri)


@pytest.mark.parametrize("name", ORACLE_FIXTURES + ["square256"])
def test_vac_msd_moments_bit_exact(name):
    m, g = O.load_model(fixture_dir(name))
    phi = O.random_phase_state(g, m.n)
    p = m.params
    M = p.number_of_moments
    for which, fn in (("vacmom", O.vac_moments), ("msdmom", O.msd_moments)):
        path = os.path.join(os.path.dirname(fixture_dir(name)), "..", "ref", name,
                            which + ".npz")
        if not os.path.exists(path):
            continue
        r = np.load(path)
        mr, mi = fn(m, M, p.time_step, phi)
        np.testing.assert_array_equal(mr, r["re"])
        np.testing.assert_array_equal(mi, r["im"])


def _rows(path):
    with open(path) as f:
        return [l.rstrip("\n") for l in f if l.strip()]


def _fmt(row):
    # std::ostream default formatting (6 significant digits), one trailing space
    return "".join("%g " % x for x in row)


@pytest.mark.parametrize("example,vectors", [("fan2018cpc_diffusive", 1),
                                             ("fan2018cpc_localized", 2)])
def test_shipped_dos_reproduced(example, vectors):
    """The reference's shipped dos.out (4,000,000 sites) reproduced character for
    character: pins the lattice build, the seed-12345678 stream and the DOS path."""
    d = os.path.join(EXAMPLES, example)
    m, g = O.load_model(d)
    p = m.params
    rows = _rows(os.path.join(d, "dos.out"))
    assert len(rows) == vectors
    for k in range(vectors):
        phi = O.random_phase_state(g, m.n)
        mr, mi = O.find_moments(m, p.number_of_moments, phi, phi)
        dos = O.correlation(p.number_of_moments, mr, mi, p.energy, m.energy_max, m.volume)
        assert _fmt(dos) == rows[k]


@pytest.mark.skipif(not O.have_ref(), reason="reference build (oracle/_ref) not present")
def test_split_seed_mode_matches_reference_driver(tmp_path):
    d = fixture_dir("sq16_pbc")
    m, g0 = O.load_model(d, disorder_seed=3)
    r = O.ref_ell(d, str(tmp_path / "ell.bin"), seeds=(3, 9))
    np.testing.assert_array_equal(m.potential, r.potential)
    g = O.MT19937(9)
    phi = O.random_phase_state(g, m.n)
    rr, ri = O.ref_moments("moments", d, str(tmp_path / "m.txt"), seeds=(3, 9))
    mr, mi = O.find_moments(m, len(rr), phi, phi)
    np.testing.assert_array_equal(mr, rr)
