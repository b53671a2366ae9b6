"""Test infrastructure only: Python access to the CPU oracle and to the reference build.

The oracle (``lsqt_oracle.c``) restates the reference's CPU path in plain C; the
reference build (``_ref/``) is the reference compiled from its own sources with the
driver ``ref_driver.cpp``. Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` leg of ``bench.py`` import this package, and only as the checker:
the product (``gpuqt_b200``) never imports it.

Input directories are parsed here with the reference's rules (src/model.cu:243-384,
src/model_lattice.cu:165-337) into plain arrays for the C builder.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liblsqt_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_DRIVER = os.path.join(REF_DIR, "ref_driver")
REF_LSQT = os.path.join(REF_DIR, "lsqt_cpu")
# The reference checkout: $GQT_REFERENCE, else a `reference` directory beside this
# repository. Only the build of _ref/ reads it; the GPU host never does.
REFERENCE_ROOT = os.environ.get("GQT_REFERENCE") or os.path.join(
    os.path.dirname(os.path.dirname(HERE)), "reference")
REFERENCE_SRC = os.path.join(REFERENCE_ROOT, "src")

_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build(ref: bool | None = None) -> None:
    """Compile the C oracle, and the reference build when its sources are present."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref is None:
        ref = os.path.isdir(REFERENCE_SRC)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_SRC={REFERENCE_SRC}"],
                       check=True)


def have_ref() -> bool:
    return os.path.exists(REF_DRIVER) and os.path.exists(REF_LSQT)


class _MT(ctypes.Structure):
    _fields_ = [("x", ctypes.c_uint32 * 624), ("i", ctypes.c_int)]


class _Lattice(ctypes.Structure):
    _fields_ = [
        ("n_cell", ctypes.c_int * 3),
        ("pbc", ctypes.c_int * 3),
        ("transport_direction", ctypes.c_int),
        ("lattice_constant", ctypes.c_double * 3),
        ("n_orbital", ctypes.c_int),
        ("max_neighbor", ctypes.c_int),
        ("orbital_xyz", _dp),
        ("n_hoppings", _ip),
        ("hop_index", _ip),
        ("hop_value", _dp),
    ]


class _Ham(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int),
        ("max_neighbor", ctypes.c_int),
        ("energy_max", ctypes.c_double),
        ("neighbor_number", _ip),
        ("neighbor_list", _ip),
        ("potential", _dp),
        ("hopping_real", _dp),
        ("hopping_imag", _dp),
        ("xx", _dp),
    ]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(ref=False)
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.orc_mt_next.restype = ctypes.c_uint32
        _lib.orc_uniform_real.restype = ctypes.c_double
        _lib.orc_uniform_real.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        _lib.orc_uniform_int_0_intmax.restype = ctypes.c_int
        _lib.orc_lattice_sites.restype = ctypes.c_long
        _lib.orc_mt_discard.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
        for name in ("orc_evolve", "orc_evolvex"):
            getattr(_lib, name).argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                            _dp, _dp]
        _lib.orc_bessel_cut.argtypes = [ctypes.c_double]
        _lib.orc_chebyshev_01.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_int]
        _lib.orc_chebyshev_1x.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_double]
        _lib.orc_chebyshev_2.argtypes = [ctypes.c_void_p] + [_dp] * 8 + [ctypes.c_double,
                                                                        ctypes.c_int]
        _lib.orc_chebyshev_2x.argtypes = [ctypes.c_void_p] + [_dp] * 14 + [ctypes.c_double,
                                                                          ctypes.c_int]
        _lib.orc_chebyshev_summation.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _dp,
                                                 ctypes.c_double, ctypes.c_double, _dp]
        _lib.orc_add_anderson.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _dp]
    return _lib


def _p(a: np.ndarray, t=_dp):
    return a.ctypes.data_as(t)


# ----------------------------------------------------------------------------- RNG
class MT19937:
    """std::mt19937 with the two distributions the reference draws from."""

    def __init__(self, seed: int):
        self._s = _MT()
        lib().orc_mt_seed(ctypes.byref(self._s), ctypes.c_uint32(seed))

    def next(self) -> int:
        return lib().orc_mt_next(ctypes.byref(self._s))

    def discard(self, count: int) -> None:
        lib().orc_mt_discard(ctypes.byref(self._s), count)

    def uniform(self, a: float, b: float) -> float:
        return lib().orc_uniform_real(ctypes.byref(self._s), a, b)

    def uniform_int(self) -> int:
        return lib().orc_uniform_int_0_intmax(ctypes.byref(self._s))

    @property
    def ref(self):
        return ctypes.byref(self._s)


# ----------------------------------------------------------------------------- inputs
@dataclass
class Params:
    """para.in (src/model.cu:243-310) plus the data files the run needs."""

    use_lattice_model: int = 0
    anderson: float | None = None
    charge: tuple | None = None
    vacancies: int | None = None
    calculate_vac0: bool = False
    calculate_vac: bool = False
    calculate_msd: bool = False
    calculate_spin: bool = False
    calculate_ldos: bool = False
    number_of_random_vectors: int = 1
    number_of_moments: int = 1000
    energy_max: float = 10.0
    seed: int = 12345678
    disorder_seed: int | None = None
    phase_seed: int | None = None
    energy: np.ndarray = field(default_factory=lambda: np.zeros(0))
    time_step: np.ndarray = field(default_factory=lambda: np.zeros(0))


def read_params(d: str) -> Params:
    p = Params()
    with open(os.path.join(d, "para.in")) as f:
        for line in f:
            tok = line.split()
            if not tok:
                continue
            k, v = tok[0], tok[1:]
            if k == "model":
                p.use_lattice_model = int(v[0])
            elif k == "anderson_disorder":
                p.anderson = float(v[0])
            elif k == "charged_impurity":
                p.charge = (int(v[0]), float(v[1]), float(v[2]))
            elif k == "vacancy_disorder":
                p.vacancies = int(v[0])
            elif k in ("calculate_vac0", "calculate_vac", "calculate_msd", "calculate_spin",
                       "calculate_ldos"):
                setattr(p, k, True)
            elif k == "number_of_random_vectors":
                p.number_of_random_vectors = int(v[0])
            elif k == "number_of_moments":
                p.number_of_moments = int(v[0])
            elif k == "energy_max":
                p.energy_max = float(v[0])
            elif k in ("seed", "disorder_seed", "phase_seed"):
                # this library's seed keywords (the reference fixes one stream)
                setattr(p, k, int(v[0]))
            else:
                raise ValueError(f"unknown keyword {k}")
    e = np.loadtxt(os.path.join(d, "energy.in"))
    p.energy = e[1: 1 + int(e[0])].astype(np.float64)
    if p.calculate_vac or p.calculate_msd or p.calculate_spin:
        t = np.loadtxt(os.path.join(d, "time_step.in"))
        p.time_step = np.atleast_1d(t)[1: 1 + int(np.atleast_1d(t)[0])].astype(np.float64)
    return p


@dataclass
class Model:
    """The ELL arrays of a built model, row-major like the reference's CPU build."""

    n: int
    max_neighbor: int
    energy_max: float
    volume: float
    neighbor_number: np.ndarray
    neighbor_list: np.ndarray
    potential: np.ndarray
    hopping_real: np.ndarray
    hopping_imag: np.ndarray
    xx: np.ndarray
    params: Params | None = None
    _keep: list = field(default_factory=list)

    def ham(self) -> _Ham:
        h = _Ham()
        h.n = self.n
        h.max_neighbor = self.max_neighbor
        h.energy_max = self.energy_max
        h.neighbor_number = _p(self.neighbor_number, _ip)
        h.neighbor_list = _p(self.neighbor_list, _ip)
        h.potential = _p(self.potential)
        h.hopping_real = _p(self.hopping_real)
        h.hopping_imag = _p(self.hopping_imag)
        h.xx = _p(self.xx)
        self._keep.append(h)
        return h


def read_lattice(path: str) -> dict:
    """lattice.in, src/model_lattice.cu:176-337 (whitespace-separated tokens)."""
    with open(path) as f:
        tok = f.read().split()
    it = iter(tok)
    nxt = lambda: next(it)  # noqa: E731
    n_cell = [int(nxt()) for _ in range(3)]
    pbc = [int(nxt()) for _ in range(3)]
    td = int(nxt())
    a = [float(nxt()) for _ in range(3)]
    no, z = int(nxt()), int(nxt())
    xyz = np.array([float(nxt()) for _ in range(3 * no)], dtype=np.float64)
    nh = np.zeros(no, dtype=np.int32)
    hidx = np.zeros(no * z * 4, dtype=np.int32)
    hval = np.zeros(no * z * 2, dtype=np.float64)
    for m in range(no):
        nh[m] = int(nxt())
        for i in range(nh[m]):
            k = m * z + i
            hidx[4 * k: 4 * k + 4] = [int(nxt()) for _ in range(4)]
            hval[2 * k] = float(nxt())
            hval[2 * k + 1] = float(nxt())
    return dict(n_cell=n_cell, pbc=pbc, td=td, a=a, no=no, z=z, xyz=xyz, nh=nh, hidx=hidx,
                hval=hval)


def build_lattice(lat: dict) -> dict:
    L = _Lattice()
    for d in range(3):
        L.n_cell[d] = lat["n_cell"][d]
        L.pbc[d] = lat["pbc"][d]
        L.lattice_constant[d] = lat["a"][d]
    L.transport_direction = lat["td"]
    L.n_orbital = lat["no"]
    L.max_neighbor = lat["z"]
    L.orbital_xyz = _p(lat["xyz"])
    L.n_hoppings = _p(lat["nh"], _ip)
    L.hop_index = _p(lat["hidx"], _ip)
    L.hop_value = _p(lat["hval"])
    n = int(lib().orc_lattice_sites(ctypes.byref(L)))
    z = lat["z"]
    out = dict(
        n=n, z=z,
        nn=np.zeros(n, np.int32), nl=np.zeros(n * z, np.int32),
        hr=np.zeros(n * z), hi=np.zeros(n * z), xx=np.zeros(n * z), pot=np.zeros(n),
    )
    vol = ctypes.c_double()
    lib().orc_build_lattice(ctypes.byref(L), _p(out["nn"], _ip), _p(out["nl"], _ip),
                            _p(out["hr"]), _p(out["hi"]), _p(out["xx"]), _p(out["pot"]),
                            ctypes.byref(vol))
    out["volume"] = vol.value
    return out


def load_model(d: str, seed: int | None = None, disorder_seed: int | None = None
               ) -> tuple[Model, MT19937]:
    """Model::Model for lattice inputs (src/model.cu:30-65, src/model_lattice.cu:389-399).

    Returns the model and the generator in the state the reference leaves it in, ready
    for the phase draws. ``disorder_seed`` reseeds the generator before the Anderson
    draws and a para.in ``phase_seed`` reseeds it before the phases (the split-seed
    mode); both default to the para.in keywords."""
    p = read_params(d)
    seed = p.seed if seed is None else seed
    disorder_seed = p.disorder_seed if disorder_seed is None else disorder_seed
    if not p.use_lattice_model:
        raise NotImplementedError("the oracle builds lattice models only")
    if p.charge is not None:
        raise NotImplementedError("charged impurities are not restated in the oracle")
    g = MT19937(seed)
    b = build_lattice(read_lattice(os.path.join(d, "lattice.in")))
    n, z = b["n"], b["z"]
    if p.vacancies is not None:
        n = lib().orc_add_vacancies(g.ref, n, z, p.vacancies, _p(b["nn"], _ip),
                                    _p(b["nl"], _ip), _p(b["hr"]), _p(b["hi"]), _p(b["xx"]))
        for k in ("nl", "hr", "hi", "xx"):
            b[k] = np.ascontiguousarray(b[k][: n * z])
        b["nn"] = np.ascontiguousarray(b["nn"][:n])
        b["pot"] = np.zeros(n)
    if disorder_seed is not None:
        g = MT19937(disorder_seed)
    if p.anderson is not None:
        lib().orc_add_anderson(g.ref, n, p.anderson, _p(b["pot"]))
    m = Model(n=n, max_neighbor=z, energy_max=p.energy_max, volume=b["volume"],
              neighbor_number=b["nn"], neighbor_list=b["nl"], potential=b["pot"],
              hopping_real=b["hr"], hopping_imag=b["hi"], xx=b["xx"], params=p)
    if p.phase_seed is not None:
        g = MT19937(p.phase_seed)
    return m, g


def random_phase_state(g: MT19937, n: int, spin: bool = False):
    re = np.zeros(n)
    im = np.zeros(n)
    lib().orc_random_phase_state(g.ref, n, int(spin), _p(re), _p(im))
    return re, im


# ----------------------------------------------------------------------------- operators
def _vec(n):
    return np.zeros(n), np.zeros(n)


def apply(m: Model, vr, vi):
    o = _vec(m.n)
    lib().orc_apply(ctypes.byref(m.ham()), _p(vr), _p(vi), _p(o[0]), _p(o[1]))
    return o


def apply_commutator(m: Model, vr, vi):
    o = _vec(m.n)
    lib().orc_apply_commutator(ctypes.byref(m.ham()), _p(vr), _p(vi), _p(o[0]), _p(o[1]))
    return o


def apply_current(m: Model, vr, vi):
    o = _vec(m.n)
    lib().orc_apply_current(ctypes.byref(m.ham()), _p(vr), _p(vi), _p(o[0]), _p(o[1]))
    return o


def kernel_polynomial(m: Model, s0, s1):
    o = _vec(m.n)
    lib().orc_kernel_polynomial(ctypes.byref(m.ham()), _p(s0[0]), _p(s0[1]), _p(s1[0]),
                                _p(s1[1]), _p(o[0]), _p(o[1]))
    return o


def chebyshev_01(n, s0, s1, b0, b1, direction):
    o = _vec(n)
    lib().orc_chebyshev_01(n, _p(s0[0]), _p(s0[1]), _p(s1[0]), _p(s1[1]), _p(o[0]), _p(o[1]),
                           b0, b1, direction)
    return o


def chebyshev_2(m: Model, s0, s1, out, bessel, label):
    """Returns (T2, out') without modifying the inputs."""
    s2 = _vec(m.n)
    o = (out[0].copy(), out[1].copy())
    lib().orc_chebyshev_2(ctypes.byref(m.ham()), _p(s0[0]), _p(s0[1]), _p(s1[0]), _p(s1[1]),
                          _p(s2[0]), _p(s2[1]), _p(o[0]), _p(o[1]), bessel, label)
    return s2, o


def chebyshev_1x(n, s1x, b1):
    o = _vec(n)
    lib().orc_chebyshev_1x(n, _p(s1x[0]), _p(s1x[1]), _p(o[0]), _p(o[1]), b1)
    return o


def chebyshev_2x(m: Model, s0, s0x, s1, s1x, out, bessel, label):
    """Returns (T2, T2x, out')."""
    s2, s2x = _vec(m.n), _vec(m.n)
    o = (out[0].copy(), out[1].copy())
    lib().orc_chebyshev_2x(ctypes.byref(m.ham()), _p(s0[0]), _p(s0[1]), _p(s0x[0]),
                           _p(s0x[1]), _p(s1[0]), _p(s1[1]), _p(s1x[0]), _p(s1x[1]),
                           _p(s2[0]), _p(s2[1]), _p(s2x[0]), _p(s2x[1]), _p(o[0]), _p(o[1]),
                           bessel, label)
    return s2, s2x, o


def inner_product(n, state, left):
    re, im = ctypes.c_double(), ctypes.c_double()
    lib().orc_inner_product(n, _p(state[0]), _p(state[1]), _p(left[0]), _p(left[1]),
                            ctypes.byref(re), ctypes.byref(im))
    return re.value, im.value


def find_moments(m: Model, n_moments: int, left, right):
    mr, mi = np.zeros(n_moments), np.zeros(n_moments)
    lib().orc_find_moments(ctypes.byref(m.ham()), n_moments, _p(left[0]), _p(left[1]),
                           _p(right[0]), _p(right[1]), _p(mr), _p(mi))
    return mr, mi


def evolve(m: Model, direction: int, dt_scaled: float, state):
    r, i = state[0].copy(), state[1].copy()
    lib().orc_evolve(ctypes.byref(m.ham()), direction, dt_scaled, _p(r), _p(i))
    return r, i


def evolvex(m: Model, direction: int, dt_scaled: float, state):
    r, i = state[0].copy(), state[1].copy()
    lib().orc_evolvex(ctypes.byref(m.ham()), direction, dt_scaled, _p(r), _p(i))
    return r, i


def bessel_cut(dt_scaled: float) -> int:
    return lib().orc_bessel_cut(dt_scaled)


def vac_moments(m: Model, n_moments: int, time_step: np.ndarray, phi):
    ns = len(time_step)
    mr, mi = np.zeros(ns * n_moments), np.zeros(ns * n_moments)
    ts = np.ascontiguousarray(time_step, dtype=np.float64)
    lib().orc_vac_moments(ctypes.byref(m.ham()), n_moments, ns, _p(ts), _p(phi[0]),
                          _p(phi[1]), _p(mr), _p(mi))
    return mr.reshape(ns, n_moments), mi.reshape(ns, n_moments)


def msd_moments(m: Model, n_moments: int, time_step: np.ndarray, phi):
    ns = len(time_step)
    mr, mi = np.zeros(ns * n_moments), np.zeros(ns * n_moments)
    ts = np.ascontiguousarray(time_step, dtype=np.float64)
    lib().orc_msd_moments(ctypes.byref(m.ham()), n_moments, ns, _p(ts), _p(phi[0]),
                          _p(phi[1]), _p(mr), _p(mi))
    return mr.reshape(ns, n_moments), mi.reshape(ns, n_moments)


def correlation(n_moments: int, mu_re, mu_im, energy, energy_max, volume):
    """apply_damping + perform_chebyshev_summation (src/sigma.cu:76-110)."""
    r = np.ascontiguousarray(mu_re, dtype=np.float64).copy()
    i = np.ascontiguousarray(mu_im, dtype=np.float64).copy()
    lib().orc_apply_damping(n_moments, _p(r), _p(i))
    e = np.ascontiguousarray(energy, dtype=np.float64)
    out = np.zeros(len(e))
    lib().orc_chebyshev_summation(n_moments, _p(r), len(e), _p(e), energy_max, volume,
                                  _p(out))
    return out


# ----------------------------------------------------------------------------- reference build
def ref_run(mode: str, d: str, out: str, *args, seeds: tuple | None = None) -> None:
    cmd = [REF_DRIVER, mode, d, out] + [str(a) for a in args]
    if seeds is not None:
        cmd += [str(seeds[0]), str(seeds[1])]
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)


def ref_ell(d: str, out: str, seeds: tuple | None = None) -> Model:
    ref_run("ell", d, out, seeds=seeds)
    with open(out, "rb") as f:
        n, z = np.frombuffer(f.read(8), np.int32)
        emax, vol = np.frombuffer(f.read(16), np.float64)
        nn = np.frombuffer(f.read(4 * n), np.int32).copy()
        nl = np.frombuffer(f.read(4 * n * z), np.int32).copy()
        pot = np.frombuffer(f.read(8 * n), np.float64).copy()
        hr = np.frombuffer(f.read(8 * n * z), np.float64).copy()
        hi = np.frombuffer(f.read(8 * n * z), np.float64).copy()
        xx = np.frombuffer(f.read(8 * n * z), np.float64).copy()
    return Model(n=int(n), max_neighbor=int(z), energy_max=float(emax), volume=float(vol),
                 neighbor_number=nn, neighbor_list=nl, potential=pot, hopping_real=hr,
                 hopping_imag=hi, xx=xx)


REF_OPS = ("phi", "H", "commutator", "current", "T2", "evolve+", "evolve-", "evolvex+",
           "evolvex-")


def ref_ops(d: str, out: str, dt_scaled: float, seeds: tuple | None = None) -> dict:
    ref_run("ops", d, out, repr(float(dt_scaled)), seeds=seeds)
    raw = np.fromfile(out, np.float64)
    n = raw.size // (2 * len(REF_OPS))
    raw = raw.reshape(len(REF_OPS), 2, n)
    return {k: (raw[j, 0].copy(), raw[j, 1].copy()) for j, k in enumerate(REF_OPS)}


def ref_moments(mode: str, d: str, out: str, seeds: tuple | None = None):
    ref_run(mode, d, out, seeds=seeds)
    a = np.loadtxt(out, dtype=np.float64, ndmin=2)
    return a[:, 0].copy(), a[:, 1].copy()


def rel_err(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.maximum(np.abs(b), 1e-300)
    return float(np.max(np.abs(a - b) / den)) if a.size else 0.0


__all__ = [n for n in dir() if not n.startswith("_")] + ["math"]
