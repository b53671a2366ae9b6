"""Symmetric moment sets from half the Chebyshev steps (gqt_moments_doubled, para.in
kpm_doubling): mu_2k = 2 <T_k|T_k> - mu_0, mu_{2k-1} = 2 <T_{k-1}|T_k> - mu_1. The
moments equal the reference's direct ones up to rounding, which the subtraction makes
absolute rather than relative: the bar is 1e-12 of the largest moment in the FP64
form (against the reference build's moments, and against the direct loop at size),
and 1e-6 of the DOS peak in the FP32-storage form. The identity needs H = H^+: the two
seeded general-model fixtures draw every hopping independently (not Hermitian), and
the library refuses them."""
from __future__ import annotations

import os
import shutil

import numpy as np
import pytest

import gpuqt_b200 as g
from gpuqt_b200 import workloads as W
from conftest import REF, SMALL_FIXTURES, fixture_dir, ref_moments
from test_gpu_golden import _compare

pytestmark = pytest.mark.gpu

ABS_FP64 = 1e-12


def _err(a, b):
    scale = np.max(np.hypot(b[0], b[1]))
    return float(np.max(np.hypot(a[0] - b[0], a[1] - b[1])) / scale)


HERMITIAN = [n for n in SMALL_FIXTURES if not n.startswith("general")] + ["square256"]


@pytest.mark.parametrize("name", HERMITIAN)
def test_doubled_fp64_against_reference(name):
    m = g.Model.load(fixture_dir(name))
    H = g.Hamiltonian(m)
    x = g.Vector.from_host(*m.initial_state())
    rr, ri = ref_moments(name)
    for M in (len(rr), len(rr) - 1):  # even and odd counts
        got = g.moments_doubled(H, x, M)
        assert got[0].shape == (M,)
        assert _err(got, (rr[:M], ri[:M])) <= ABS_FP64, M
    assert g.moments_doubled(H, x, 1)[0][0] == pytest.approx(rr[0], rel=1e-14)
    r2 = g.moments_doubled(H, x, 2)
    assert abs(r2[0][1] - rr[1]) <= 1e-13 * abs(rr[0])


@pytest.mark.parametrize("workload", ["square1m", "graphene2m"])
def test_doubled_equals_direct_at_size(tmp_path, workload):
    m = g.Model.load(W.config_dir(str(tmp_path), workload))
    H = g.Hamiltonian(m)
    x = g.Vector.from_host(*m.initial_state())
    M = 600
    direct = g.moments(H, x, x, M)
    doubled = g.moments_doubled(H, x, M)
    assert _err(doubled, direct) <= ABS_FP64
    H.set_format(g.FORMAT_ELL)
    assert _err(g.moments_doubled(H, x, M), direct) <= ABS_FP64


@pytest.mark.parametrize("V", [1, 4, 16])
def test_doubled_fp32_form_dos(V):
    m = g.Model.load(fixture_dir("square256"))
    H = g.Hamiltonian(m)
    ph = [m.initial_state() for _ in range(V)]
    re, im = np.stack([p[0] for p in ph]), np.stack([p[1] for p in ph])
    X64 = g.Vector.from_host(re, im, nvec=V)
    X32 = g.Vector.from_host(re, im, nvec=V, precision=g.FP32)
    M = m.n_moments
    a = [np.atleast_2d(t) for t in g.moments(H, X64, X64, M)]
    b = [np.atleast_2d(t) for t in g.moments_doubled(H, X32, M)]
    c = [np.atleast_2d(t) for t in g.moments_doubled(H, X64, M, precision=g.FP32)]
    for k in range(V):
        d64 = g.chebyshev_summation(a[0][k], a[1][k], m.energy, m.energy_max, m.volume)
        for got in (b, c):
            d32 = g.chebyshev_summation(got[0][k], got[1][k], m.energy, m.energy_max, m.volume)
            assert np.max(np.abs(d32 - d64)) <= 1e-6 * np.max(np.abs(d64))


@pytest.mark.parametrize("name", ["general40", "general_spin"])
def test_doubled_refuses_non_hermitian(name):
    m = g.Model.load(fixture_dir(name))
    H = g.Hamiltonian(m)
    x = g.Vector.from_host(*m.initial_state())
    with pytest.raises(g.GqtError) as e:
        g.moments_doubled(H, x, 10)
    assert e.value.status == 6 and "Hermitian" in str(e.value)


def test_doubled_limits():
    m = g.Model.load(fixture_dir("sq16_pbc"))
    H = g.Hamiltonian(m)
    X = g.Vector(m.n, nvec=32, precision=g.FP32)
    with pytest.raises(g.GqtError) as e:
        g.moments_doubled(H, X, 10)
    assert e.value.status == 1


@pytest.mark.parametrize("prec,V", [(g.FP64, 4), (g.FP32, 16), (g.FP32, 32)])
def test_doubled_batch(prec, V):
    """Realisation batches: per-model symmetric moments from half the steps."""
    names = ["sq16_pbc", "graphene_8x4", "cubic6", "sq12_open_vac"]
    models = [g.Model.load(fixture_dir(n)) for n in names]
    B = g.Hamiltonian.batch(models)
    per = []
    for mm in models:
        ph = [mm.initial_state() for _ in range(V)]
        per.append((np.stack([p[0] for p in ph]), np.stack([p[1] for p in ph])))
    X = g.Vector.from_host(*B.scatter(per), nvec=V, precision=prec)
    M = 151
    dr, di = g.moments(B, X, X, M)
    br, bi = g.moments_doubled(B, X, M)
    assert br.shape == (len(models), V, M)
    for r, mm in enumerate(models):
        if prec == g.FP64:
            assert _err((br[r], bi[r]), (dr[r], di[r])) <= ABS_FP64, r
        else:
            for k in range(0, V, 7):
                d1 = g.chebyshev_summation(dr[r, k], di[r, k], mm.energy, mm.energy_max, mm.volume)
                d2 = g.chebyshev_summation(br[r, k], bi[r, k], mm.energy, mm.energy_max, mm.volume)
                assert np.max(np.abs(d2 - d1)) <= 1e-6 * np.max(np.abs(d1)), (r, k)


def _run_dir(tmp_path, name, tag, extra, files=None):
    d = str(tmp_path / (name + tag))
    os.makedirs(d)
    for f in os.listdir(fixture_dir(name)):
        if f.endswith(".in"):
            shutil.copy(os.path.join(fixture_dir(name), f), d)
    with open(os.path.join(d, "para.in"), "a") as f:
        f.write(extra)
    for fname, text in (files or {}).items():
        with open(os.path.join(d, fname), "w") as f:
            f.write(text)
    assert g.lsqt(d)
    return d


@pytest.mark.parametrize("name", ["sq16_pbc", "chain_z2"])
def test_driver_with_doubling_matches_reference_outputs(tmp_path, name):
    d = _run_dir(tmp_path, name, "_dbl", "kpm_doubling\n")
    found = 0
    for f in ("dos.out", "vac0.out", "vac.out", "msd.out"):
        ref = os.path.join(REF, name, f)
        if os.path.exists(ref):
            _compare(os.path.join(d, f), ref)
            found += 1
    assert found >= 2


def test_driver_doubling_ldos(tmp_path):
    files = {"local_orbitals.in": "3\n0\n17\n200\n"}
    a = _run_dir(tmp_path, "sq16_pbc", "_direct", "calculate_ldos\n", files)
    b = _run_dir(tmp_path, "sq16_pbc", "_dbl", "calculate_ldos\nkpm_doubling\n", files)
    for f in ("dos.out", "ldos.out", "vac0.out", "msd.out", "vac.out"):
        _compare(os.path.join(b, f), os.path.join(a, f))
