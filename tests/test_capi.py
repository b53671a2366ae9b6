"""The C ABI without a GPU: the library loads, exports every entry point that
include/gpuqt.h declares, validates arguments on the host, and its host-side
functions match the oracle."""
from __future__ import annotations

import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import gpuqt_b200 as g
import oracle as O
from conftest import ROOT, fixture_dir


def _declared():
    text = open(os.path.join(ROOT, "include", "gpuqt.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gqt_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", g.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(gqt_[a-z0-9_]+)", out))
    declared = _declared()
    assert len(declared) >= 40
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    lib = g.lib()
    for s in declared:
        assert hasattr(lib, s)


def test_python_binding_covers_the_header():
    assert sorted(g.declared_symbols()) == _declared()


def test_cxx_surface_is_exported():
    out = subprocess.run(["nm", "-DC", "--defined-only", g.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    for sym in ("Model::Model(std::__cxx11::basic_string", "Model::initialize_state(Vector&, int)",
                "Hamiltonian::Hamiltonian(Model&)", "Hamiltonian::apply(Vector&, Vector&)",
                "Hamiltonian::chebyshev_2x(", "Vector::inner_product_1(int, Vector&, Vector&, int)",
                "find_moments_chebyshev(Model&, Hamiltonian&, Vector&, Vector&, Vector&)",
                "find_dos(Model&, Hamiltonian&, Vector&, int)", "evolvex(Model&, int, double",
                "lsqt(std::__cxx11::basic_string"):
        assert sym in out, sym


def test_cli_usage():
    r = subprocess.run([g.CLI_PATH], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stdout


def test_version():
    a, b = ctypes.c_int(), ctypes.c_int()
    assert g.lib().gqt_version(ctypes.byref(a), ctypes.byref(b)) == 0 and a.value == 1


def test_chebyshev_summation_matches_oracle():
    d = fixture_dir("sq16_pbc")
    rng = np.random.default_rng(3)
    M = 200
    mr, mi = rng.normal(size=M) * 10, rng.normal(size=M)
    e = np.linspace(-4.9, 4.9, 41)
    ours = g.chebyshev_summation(mr, mi, e, 5.0, 256.0)
    ref = O.correlation(M, mr, mi, e, 5.0, 256.0)
    np.testing.assert_array_equal(ours, ref)


def _ell(n=4, z=2):
    return dict(n=n, max_neighbor=z, energy_max=3.0,
                neighbor_number=np.full(n, z, np.int32),
                neighbor_list=np.array([(i + 1) % n for i in range(n) for _ in range(z)],
                                       np.int32),
                potential=np.zeros(n), hopping_real=-np.ones(n * z),
                hopping_imag=np.zeros(n * z), xx=np.ones(n * z))


@pytest.mark.parametrize("bad,needle", [
    (dict(neighbor_list=np.array([1, 1, 2, 9, 3, 3, 0, 0], np.int32)), "out of"),
    (dict(neighbor_list=np.array([1, 1, 2, -1, 3, 3, 0, 0], np.int32)), "out of"),
    (dict(neighbor_number=np.array([2, 3, 2, 2], np.int32)), "neighbours"),
    (dict(energy_max=0.0), "energy_max"),
    (dict(n=0), "sites"),
])
def test_hamiltonian_validation_before_upload(bad, needle):
    # These are rejected on the host before any device call, so they fail the same
    # way with or without a GPU.
    ell = _ell()
    ell.update(bad)
    with pytest.raises(g.GqtError) as e:
        g.Hamiltonian(**ell)
    assert needle in str(e.value)


def test_vector_argument_validation():
    with pytest.raises(g.GqtError) as e:
        g.Vector(0)
    assert e.value.status == 1
    with pytest.raises(g.GqtError):
        g.Vector(16, nvec=3)
    with pytest.raises(g.GqtError):
        g.Vector(16, precision=7)
