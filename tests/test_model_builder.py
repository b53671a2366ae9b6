"""The library's host model builder (C++, reached through gqt_model_load) against the
reference's own build (golden ELL dumps) and the oracle: bit-exact ELL arrays,
potentials and random phases; the reference's input errors as status codes."""
from __future__ import annotations

import os
import shutil

import numpy as np
import pytest

import gpuqt_b200 as g
import oracle as O
from conftest import ORACLE_FIXTURES, SMALL_FIXTURES, fixture_dir, ref_npz


@pytest.mark.parametrize("name", SMALL_FIXTURES)
def test_ell_matches_reference_build(name):
    m = g.Model.load(fixture_dir(name))
    r = ref_npz(name, "ell")
    assert m.n == r["nn"].size
    np.testing.assert_array_equal(m.neighbor_number, r["nn"])
    z = m.max_neighbor
    mask = np.arange(z)[None, :] < m.neighbor_number[:, None]
    for a, k in ((m.neighbor_list, "nl"), (m.hopping_real, "hr"), (m.hopping_imag, "hi"),
                 (m.xx, "xx")):
        np.testing.assert_array_equal(a.reshape(-1, z)[mask], r[k].reshape(-1, z)[mask])
    np.testing.assert_array_equal(m.potential, r["pot"])
    assert m.energy_max == r["meta"][0] and m.volume == r["meta"][1]


@pytest.mark.parametrize("name", SMALL_FIXTURES)
def test_phases_match_reference_build(name):
    m = g.Model.load(fixture_dir(name))
    phi = m.initial_state()
    np.testing.assert_array_equal(np.stack(phi), ref_npz(name, "ops")["phi"])


def test_square256_split_seeds_match_oracle():
    d = fixture_dir("square256")
    m = g.Model.load(d)
    o, gen = O.load_model(d)
    np.testing.assert_array_equal(m.potential, o.potential)
    np.testing.assert_array_equal(m.neighbor_list, o.neighbor_list)
    phi = m.initial_state()
    ophi = O.random_phase_state(gen, o.n)
    np.testing.assert_array_equal(phi[0], ophi[0])
    np.testing.assert_array_equal(phi[1], ophi[1])


def test_successive_vectors_follow_one_stream():
    d = fixture_dir("chain_z2")
    m = g.Model.load(d)
    o, gen = O.load_model(d)
    for _ in range(3):
        a = m.initial_state()
        b = O.random_phase_state(gen, o.n)
        np.testing.assert_array_equal(a[0], b[0])


def test_local_orbital_state():
    m = g.Model.load(fixture_dir("sq16_pbc"))
    re, im = m.initial_state(5)
    assert re[5] == np.sqrt(256.0) and np.count_nonzero(re) == 1 and not im.any()


def test_energy_and_time_files():
    d = fixture_dir("graphene_8x4")
    m = g.Model.load(d)
    p = O.read_params(d)
    np.testing.assert_array_equal(m.energy, p.energy)
    np.testing.assert_array_equal(m.time_step, p.time_step)
    assert m.n_moments == p.number_of_moments and m.n_steps == len(p.time_step)


def _broken(tmp_path, name, edit):
    d = tmp_path / name
    shutil.copytree(fixture_dir(name), d)
    edit(d)
    return str(d)


@pytest.mark.parametrize("name,edit,needle", [
    ("sq16_pbc", lambda d: (d / "para.in").write_text("model 1\nbogus_keyword 3\n"),
     "Unknown identifier"),
    ("sq16_pbc", lambda d: (d / "para.in").write_text("model 1\nnumber_of_moments 0\n"),
     "moments"),
    ("sq16_pbc", lambda d: (d / "para.in").write_text("model 1\nenergy_max -1\n"),
     "Energy maximum"),
    ("sq16_pbc", lambda d: (d / "para.in").write_text("model 1\ncalculate_spin\n"),
     "spin"),
    ("sq16_pbc", lambda d: (d / "para.in").write_text("model 0\nanderson_disorder 1\n"),
     "General model"),
    ("sq16_pbc", lambda d: (d / "lattice.in").write_text(
        (d / "lattice.in").read_text().replace("16 16 1", "16 0 1", 1)), "cells"),
    ("sq16_pbc", lambda d: (d / "lattice.in").write_text(
        (d / "lattice.in").read_text().replace("1 1 0 0", "0 1 0 0", 1)), "periodic"),
    ("sq16_pbc", lambda d: (d / "energy.in").unlink(), "energy.in"),
    ("sq16_pbc", lambda d: (d / "time_step.in").unlink(), "time_step.in"),
])
def test_input_errors_are_reported(tmp_path, name, edit, needle):
    d = _broken(tmp_path, name, edit)
    with pytest.raises(g.GqtError) as e:
        g.Model.load(d)
    assert e.value.status == 4
    assert needle in str(e.value)


def test_missing_directory(tmp_path):
    with pytest.raises(g.GqtError):
        g.Model.load(str(tmp_path / "nope"))
