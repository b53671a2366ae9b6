"""gpuqt_b200: Python access to the B200 LSQT library through its C ABI (include/gpuqt.h).

The library (gpuqt_b200/lib/libgpuqt_b200.so) holds the sm_100a kernels and the host
C++ model builder; this module only binds it with ctypes and wraps the handles:

    m = Model.load(input_dir)            # Model::Model (src/model.cu:30-65)
    H = Hamiltonian(m)                   # Hamiltonian::Hamiltonian (src/hamiltonian.cu:124)
    phi = Vector.from_host(*m.initial_state())
    mu = moments(H, phi, phi, m.n_moments)        # find_moments_chebyshev (src/sigma.cu:33)
    evolve(H, +1, dt * m.energy_max, phi)         # evolve (src/sigma.cu:116)

There is no CPU fallback: every compute call runs the library's CUDA kernels and
raises GqtError when the library reports a failure (for example, no GPU present).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libgpuqt_b200.so")
CLI_PATH = os.path.join(HERE, "lib", "lsqt_b200")

FP64 = 0
FP32 = 1
FP32X = 2  # moment recurrence only: FP32 storage with a BF16 residual
FP32R = 3  # moment recurrence only: FP32 vectors, hoppings and recurrence; FP64 sums
FORMAT_ELL = 0    # the reference's ELL arrays
FORMAT_CODED = 1  # one byte per ELL entry into a table of the distinct entries

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p


class GqtError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[gqt status {status}] {message}")
        self.status = status


class EllDesc(ctypes.Structure):
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


# name -> (restype, argtypes); status-returning calls are checked by _call.
_SIGS = {
    "gqt_last_error": (ctypes.c_char_p, []),
    "gqt_version": (ctypes.c_int, [_ip, _ip]),
    "gqt_set_stream": (ctypes.c_int, [_vp]),
    "gqt_get_stream": (_vp, []),
    "gqt_sync": (ctypes.c_int, []),
    "gqt_launch_count": (ctypes.c_uint64, []),
    "gqt_reset_launch_count": (None, []),
    "gqt_ham_create": (ctypes.c_int, [ctypes.POINTER(EllDesc), ctypes.POINTER(_vp)]),
    "gqt_ham_destroy": (ctypes.c_int, [_vp]),
    "gqt_ham_info": (ctypes.c_int, [_vp, _ip, _ip, _ip, _dp]),
    "gqt_ham_set_format": (ctypes.c_int, [_vp, ctypes.c_int]),
    "gqt_ham_format": (ctypes.c_int, [_vp, _ip, _ip]),
    "gqt_ham_set_batch_tile": (ctypes.c_int, [_vp, ctypes.c_int]),
    "gqt_ham_batch_tile": (ctypes.c_int, [_vp, _ip]),
    "gqt_ham_set_loop": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "gqt_ham_loop": (ctypes.c_int, [_vp, _ip, _ip, _ip]),
    "gqt_ham_set_staging": (ctypes.c_int, [_vp, ctypes.c_int]),
    "gqt_ham_staging": (ctypes.c_int, [_vp, _ip, _ip, _ip, _ip]),
    "gqt_ham_stage_plan": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip,
                                          _ip]),
    "gqt_ham_create_batch": (ctypes.c_int, [ctypes.POINTER(EllDesc), ctypes.c_int,
                                            ctypes.POINTER(_vp)]),
    "gqt_ham_realisations": (ctypes.c_int, [_vp, _ip]),
    "gqt_ham_realisation": (ctypes.c_int, [_vp, ctypes.c_int, _ip, _ip, _dp]),
    "gqt_autotune_nvec": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _ip, ctypes.c_int, _ip,
                                         _dp]),
    "gqt_vec_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(_vp)]),
    "gqt_vec_clone": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "gqt_vec_destroy": (ctypes.c_int, [_vp]),
    "gqt_vec_info": (ctypes.c_int, [_vp, _ip, _ip, _ip]),
    "gqt_vec_data": (_vp, [_vp]),
    "gqt_vec_upload": (ctypes.c_int, [_vp, _vp, _vp]),
    "gqt_vec_download": (ctypes.c_int, [_vp, _vp, _vp]),
    "gqt_vec_copy": (ctypes.c_int, [_vp, _vp]),
    "gqt_vec_add": (ctypes.c_int, [_vp, _vp]),
    "gqt_vec_apply_sz": (ctypes.c_int, [_vp, _vp]),
    "gqt_vec_swap": (ctypes.c_int, [_vp, _vp]),
    "gqt_vec_zero": (ctypes.c_int, [_vp]),
    "gqt_apply": (ctypes.c_int, [_vp, _vp, _vp]),
    "gqt_apply_commutator": (ctypes.c_int, [_vp, _vp, _vp]),
    "gqt_apply_current": (ctypes.c_int, [_vp, _vp, _vp]),
    "gqt_kernel_polynomial": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "gqt_chebyshev_01": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_int]),
    "gqt_chebyshev_2": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, ctypes.c_double, ctypes.c_int]),
    "gqt_chebyshev_1x": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double]),
    "gqt_chebyshev_2x": (ctypes.c_int, [_vp] * 8 + [ctypes.c_double, ctypes.c_int]),
    "gqt_inner_product": (ctypes.c_int, [_vp, _vp, _dp, _dp]),
    "gqt_inner_product_into": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int]),
    "gqt_vec_segment_sum": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp]),
    "gqt_moments": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _dp, _dp]),
    "gqt_moments_device": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _vp]),
    "gqt_moments_form": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int, _dp, _dp]),
    "gqt_moments_device_form": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "gqt_vec_convert": (ctypes.c_int, [_vp, _vp]),
    "gqt_moments_doubled": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, _dp, _dp]),
    "gqt_moments_doubled_device": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "gqt_evolve": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, _vp]),
    "gqt_evolvex": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, _vp]),
    "gqt_chebyshev_summation": (ctypes.c_int, [ctypes.c_int, _dp, _dp, ctypes.c_int, _dp,
                                               ctypes.c_double, ctypes.c_double, _dp]),
    "gqt_model_load": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(_vp)]),
    "gqt_model_destroy": (ctypes.c_int, [_vp]),
    "gqt_model_ell": (ctypes.c_int, [_vp, ctypes.POINTER(EllDesc)]),
    "gqt_model_params": (ctypes.c_int, [_vp, _ip, _ip, _ip, _ip, _dp]),
    "gqt_model_energy": (ctypes.c_int, [_vp, _dp]),
    "gqt_model_time_step": (ctypes.c_int, [_vp, _dp]),
    "gqt_model_initial_state": (ctypes.c_int, [_vp, ctypes.c_int, _dp, _dp]),
    "gqt_lsqt": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int]),
    "gqt_lsqt_run": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_longlong, _ip]),
    "gqt_chebyshev_step_noalloc": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, _vp, _vp]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Load the native library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m gpuqt_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def declared_symbols() -> list[str]:
    return sorted(_SIGS)


def _call(name: str, *args) -> None:
    st = getattr(lib(), name)(*args)
    if st != 0:
        msg = lib().gqt_last_error()
        raise GqtError(st, (msg or b"").decode(errors="replace"))


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def set_stream(stream_handle: int | None) -> None:
    """Use a cudaStream_t (e.g. torch.cuda.current_stream().cuda_stream) for this thread."""
    _call("gqt_set_stream", ctypes.c_void_p(stream_handle or 0))


def sync() -> None:
    _call("gqt_sync")


def launch_count() -> int:
    return int(lib().gqt_launch_count())


def reset_launch_count() -> None:
    lib().gqt_reset_launch_count()


# ----------------------------------------------------------------------------- vectors
class Vector:
    """nvec complex vectors of n sites on the device (Vector, src/vector.h:23-47)."""

    def __init__(self, n: int, nvec: int = 1, precision: int = FP64, _handle=None):
        if _handle is None:
            h = _vp()
            _call("gqt_vec_create", n, nvec, precision, ctypes.byref(h))
            _handle = h
        self.h = _handle
        self.n, self.nvec, self.precision = n, nvec, precision

    @classmethod
    def from_host(cls, re, im, nvec: int = 1, precision: int = FP64) -> "Vector":
        re = np.ascontiguousarray(re, dtype=np.float64).reshape(-1)
        im = np.ascontiguousarray(im, dtype=np.float64).reshape(-1)
        v = cls(re.size // nvec, nvec, precision)
        v.upload(re, im)
        return v

    def upload(self, re, im) -> None:
        re = np.ascontiguousarray(re, dtype=np.float64).reshape(-1)
        im = np.ascontiguousarray(im, dtype=np.float64).reshape(-1)
        if re.size != self.n * self.nvec or im.size != self.n * self.nvec:
            raise ValueError("host arrays do not match the vector size")
        _call("gqt_vec_upload", self.h, re.ctypes.data, im.ctypes.data)

    def upload_ptr(self, re_ptr: int, im_ptr: int) -> None:
        """Upload from host addresses (for example pinned tensors)."""
        _call("gqt_vec_upload", self.h, ctypes.c_void_p(re_ptr), ctypes.c_void_p(im_ptr))

    def download(self):
        re = np.empty(self.n * self.nvec)
        im = np.empty(self.n * self.nvec)
        _call("gqt_vec_download", self.h, re.ctypes.data, im.ctypes.data)
        if self.nvec > 1:
            return re.reshape(self.nvec, self.n), im.reshape(self.nvec, self.n)
        return re, im

    def clone(self) -> "Vector":
        h = _vp()
        _call("gqt_vec_clone", self.h, ctypes.byref(h))
        return Vector(self.n, self.nvec, self.precision, _handle=h)

    def copy_from(self, other: "Vector") -> None:
        _call("gqt_vec_copy", self.h, other.h)

    def convert_from(self, other: "Vector") -> None:
        """Copy across forms (FP64 <-> FP32)."""
        _call("gqt_vec_convert", self.h, other.h)

    def add(self, other: "Vector") -> None:
        _call("gqt_vec_add", self.h, other.h)

    def apply_sz(self, other: "Vector") -> None:
        _call("gqt_vec_apply_sz", self.h, other.h)

    def swap(self, other: "Vector") -> None:
        _call("gqt_vec_swap", self.h, other.h)

    def zero(self) -> None:
        _call("gqt_vec_zero", self.h)

    @property
    def data_ptr(self) -> int:
        return int(lib().gqt_vec_data(self.h) or 0)

    def close(self) -> None:
        if self.h is not None and _lib is not None:
            lib().gqt_vec_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ----------------------------------------------------------------------------- model
class Model:
    """A model built by the library's host code from an input directory."""

    def __init__(self, handle):
        self.h = handle
        d = EllDesc()
        _call("gqt_model_ell", self.h, ctypes.byref(d))
        self.n, self.max_neighbor, self.energy_max = d.n, d.max_neighbor, d.energy_max
        n, z = d.n, d.max_neighbor
        self.neighbor_number = np.ctypeslib.as_array(d.neighbor_number, (n,)).copy()
        self.neighbor_list = np.ctypeslib.as_array(d.neighbor_list, (n * z,)).copy()
        self.potential = np.ctypeslib.as_array(d.potential, (n,)).copy()
        self.hopping_real = np.ctypeslib.as_array(d.hopping_real, (n * z,)).copy()
        self.hopping_imag = np.ctypeslib.as_array(d.hopping_imag, (n * z,)).copy()
        self.xx = np.ctypeslib.as_array(d.xx, (n * z,)).copy()
        nm, ne, ns, nr = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        vol = ctypes.c_double()
        _call("gqt_model_params", self.h, ctypes.byref(nm), ctypes.byref(ne), ctypes.byref(ns),
              ctypes.byref(nr), ctypes.byref(vol))
        self.n_moments, self.n_energy, self.n_steps = nm.value, ne.value, ns.value
        self.n_random_vectors, self.volume = nr.value, vol.value
        self.energy = np.zeros(max(self.n_energy, 1))
        _call("gqt_model_energy", self.h, _dptr(self.energy))
        self.energy = self.energy[: self.n_energy]
        self.time_step = np.zeros(max(self.n_steps, 1))
        _call("gqt_model_time_step", self.h, _dptr(self.time_step))
        self.time_step = self.time_step[: self.n_steps]

    @classmethod
    def load(cls, input_dir: str, verbose: bool = False) -> "Model":
        h = _vp()
        _call("gqt_model_load", input_dir.encode(), int(verbose), ctypes.byref(h))
        return cls(h)

    def initial_state(self, orbital: int = -1):
        """The next random-phase vector (orbital < 0) or sqrt(N) e_orbital."""
        re, im = np.zeros(self.n), np.zeros(self.n)
        _call("gqt_model_initial_state", self.h, orbital, _dptr(re), _dptr(im))
        return re, im

    def ell(self) -> dict:
        return dict(n=self.n, max_neighbor=self.max_neighbor, energy_max=self.energy_max,
                    neighbor_number=self.neighbor_number, neighbor_list=self.neighbor_list,
                    potential=self.potential, hopping_real=self.hopping_real,
                    hopping_imag=self.hopping_imag, xx=self.xx)

    def close(self) -> None:
        if self.h is not None and _lib is not None:
            lib().gqt_model_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ----------------------------------------------------------------------------- operator
class Hamiltonian:
    """The ELL operator on the device (Hamiltonian, src/hamiltonian.h:25-54)."""

    def __init__(self, model=None, **ell):
        arrays = model.ell() if model is not None else ell
        n, z = int(arrays["n"]), int(arrays["max_neighbor"])
        self._keep = {
            "nn": np.ascontiguousarray(arrays["neighbor_number"], dtype=np.int32),
            "nl": np.ascontiguousarray(arrays["neighbor_list"], dtype=np.int32),
            "pot": np.ascontiguousarray(arrays["potential"], dtype=np.float64),
            "hr": np.ascontiguousarray(arrays["hopping_real"], dtype=np.float64),
            "hi": np.ascontiguousarray(arrays["hopping_imag"], dtype=np.float64),
        }
        xx = arrays.get("xx")
        if xx is not None:
            self._keep["xx"] = np.ascontiguousarray(xx, dtype=np.float64)
        d = EllDesc()
        d.n, d.max_neighbor, d.energy_max = n, z, float(arrays["energy_max"])
        d.neighbor_number = self._keep["nn"].ctypes.data_as(_ip)
        d.neighbor_list = self._keep["nl"].ctypes.data_as(_ip)
        d.potential = _dptr(self._keep["pot"])
        d.hopping_real = _dptr(self._keep["hr"])
        d.hopping_imag = _dptr(self._keep["hi"])
        d.xx = _dptr(self._keep["xx"]) if "xx" in self._keep else None
        h = _vp()
        _call("gqt_ham_create", ctypes.byref(d), ctypes.byref(h))
        self._adopt(h)

    def _adopt(self, h) -> None:
        self.h = h
        self._keep = None
        n, z, u, e = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        _call("gqt_ham_info", self.h, ctypes.byref(n), ctypes.byref(z), ctypes.byref(u),
              ctypes.byref(e))
        self.n, self.max_neighbor, self.energy_max = n.value, z.value, e.value
        self.uniform_rows = bool(u.value)
        r = ctypes.c_int()
        _call("gqt_ham_realisations", self.h, ctypes.byref(r))
        self.n_real = r.value
        self.realisations = []
        for k in range(self.n_real):
            off, nr, em = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
            _call("gqt_ham_realisation", self.h, k, ctypes.byref(off), ctypes.byref(nr),
                  ctypes.byref(em))
            self.realisations.append((off.value, nr.value, em.value))

    @property
    def format(self) -> int:
        f = ctypes.c_int()
        _call("gqt_ham_format", self.h, ctypes.byref(f), None)
        return f.value

    @property
    def n_codes(self) -> int:
        c = ctypes.c_int()
        _call("gqt_ham_format", self.h, None, ctypes.byref(c))
        return c.value

    @property
    def batch_tile(self) -> int:
        """Sites per tile of a realisation batch's step (0 for a single model)."""
        t = ctypes.c_int()
        _call("gqt_ham_batch_tile", self.h, ctypes.byref(t))
        return t.value

    def set_batch_tile(self, tile_sites: int) -> None:
        _call("gqt_ham_set_batch_tile", self.h, int(tile_sites))

    def set_loop(self, window: int, chunk_sites: int = 0) -> None:
        """Moment loop of the FP64 form: 0 one launch per step, S >= 2 the wavefront
        loop of S steps per launch over chunks of chunk_sites sites (0: 1024)
        (gqt_ham_set_loop)."""
        _call("gqt_ham_set_loop", self.h, int(window), int(chunk_sites))

    @property
    def loop(self) -> tuple[int, int, int]:
        """(window, chunks, halo) of the moment loop (gqt_ham_loop)."""
        w, c, k = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _call("gqt_ham_loop", self.h, ctypes.byref(w), ctypes.byref(c), ctypes.byref(k))
        return w.value, c.value, k.value

    def set_staging(self, stages: int) -> None:
        """Staged step of the FP32 and FP32R moment loops: -1 off; 0 automatic (the
        default: FP32R loops are staged, FP32 loops on rows of six); 1 every loop, as
        many shared-memory stages as fit; 2..4 every loop, that many
        (gqt_ham_set_staging)."""
        _call("gqt_ham_set_staging", self.h, int(stages))

    def stage_plan(self, nvec: int, precision: int, symmetric: bool = False):
        """(stages, windows) the staged step would use in a moment loop of nvec vectors
        in `precision` under the current setting; (0, 0) when it is not staged
        (gqt_ham_stage_plan)."""
        s, w = ctypes.c_int(), ctypes.c_int()
        _call("gqt_ham_stage_plan", self.h, int(nvec), int(precision), int(bool(symmetric)),
              ctypes.byref(s), ctypes.byref(w))
        return s.value, w.value

    @property
    def staging(self) -> tuple[int, list[tuple[int, int]]]:
        """(stages setting, [(lo, hi) neighbour-offset window, ...]) (gqt_ham_staging)."""
        s, nw = ctypes.c_int(), ctypes.c_int()
        lo, hi = (ctypes.c_int * 8)(), (ctypes.c_int * 8)()
        _call("gqt_ham_staging", self.h, ctypes.byref(s), ctypes.byref(nw), lo, hi)
        return s.value, [(lo[w], hi[w]) for w in range(nw.value)]

    def set_format(self, fmt: int) -> None:
        """FORMAT_ELL or FORMAT_CODED (the default when the operator has a coded form)."""
        _call("gqt_ham_set_format", self.h, fmt)

    @classmethod
    def batch(cls, models) -> "Hamiltonian":
        """A realisation batch: independent models as one block-diagonal operator
        (gqt_ham_create_batch); accepts Model objects or ELL dicts."""
        descs = (EllDesc * len(models))()
        keep = []
        for k, mdl in enumerate(models):
            a = mdl.ell() if hasattr(mdl, "ell") else mdl
            arr = {
                "nn": np.ascontiguousarray(a["neighbor_number"], dtype=np.int32),
                "nl": np.ascontiguousarray(a["neighbor_list"], dtype=np.int32),
                "pot": np.ascontiguousarray(a["potential"], dtype=np.float64),
                "hr": np.ascontiguousarray(a["hopping_real"], dtype=np.float64),
                "hi": np.ascontiguousarray(a["hopping_imag"], dtype=np.float64),
            }
            if a.get("xx") is not None:
                arr["xx"] = np.ascontiguousarray(a["xx"], dtype=np.float64)
            keep.append(arr)
            d = descs[k]
            d.n, d.max_neighbor = int(a["n"]), int(a["max_neighbor"])
            d.energy_max = float(a["energy_max"])
            d.neighbor_number = arr["nn"].ctypes.data_as(_ip)
            d.neighbor_list = arr["nl"].ctypes.data_as(_ip)
            d.potential = _dptr(arr["pot"])
            d.hopping_real = _dptr(arr["hr"])
            d.hopping_imag = _dptr(arr["hi"])
            d.xx = _dptr(arr["xx"]) if "xx" in arr else None
        h = _vp()
        _call("gqt_ham_create_batch", descs, len(models), ctypes.byref(h))
        obj = cls.__new__(cls)
        obj._adopt(h)
        return obj

    def scatter(self, per_model: list) -> tuple[np.ndarray, np.ndarray]:
        """Host arrays (nvec * n, vector-major) of a batch vector from per-model
        (re, im) arrays of shape (nvec, n_r); padding sites are zero."""
        nvec = np.atleast_2d(per_model[0][0]).shape[0]
        re = np.zeros((nvec, self.n))
        im = np.zeros((nvec, self.n))
        for (off, nr, _), (r, i) in zip(self.realisations, per_model):
            re[:, off:off + nr] = np.atleast_2d(r)
            im[:, off:off + nr] = np.atleast_2d(i)
        return re, im

    def close(self) -> None:
        if self.h is not None and _lib is not None:
            lib().gqt_ham_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ----------------------------------------------------------------------------- operations
def apply(H: Hamiltonian, x: Vector, out: Vector) -> None:
    _call("gqt_apply", H.h, x.h, out.h)


def apply_commutator(H: Hamiltonian, x: Vector, out: Vector) -> None:
    _call("gqt_apply_commutator", H.h, x.h, out.h)


def apply_current(H: Hamiltonian, x: Vector, out: Vector) -> None:
    _call("gqt_apply_current", H.h, x.h, out.h)


def kernel_polynomial(H: Hamiltonian, s0: Vector, s1: Vector, s2: Vector) -> None:
    _call("gqt_kernel_polynomial", H.h, s0.h, s1.h, s2.h)


def chebyshev_01(H, s0, s1, out, b0: float, b1: float, direction: int) -> None:
    _call("gqt_chebyshev_01", H.h, s0.h, s1.h, out.h, b0, b1, direction)


def chebyshev_2(H, s0, s1, s2, out, bessel: float, label: int) -> None:
    _call("gqt_chebyshev_2", H.h, s0.h, s1.h, s2.h, out.h, bessel, label)


def chebyshev_1x(H, x, out, b1: float) -> None:
    _call("gqt_chebyshev_1x", H.h, x.h, out.h, b1)


def chebyshev_2x(H, s0, s0x, s1, s1x, s2, s2x, out, bessel: float, label: int) -> None:
    _call("gqt_chebyshev_2x", H.h, s0.h, s0x.h, s1.h, s1x.h, s2.h, s2x.h, out.h, bessel, label)


def inner_product(state: Vector, left: Vector):
    re = np.zeros(state.nvec)
    im = np.zeros(state.nvec)
    _call("gqt_inner_product", state.h, left.h, _dptr(re), _dptr(im))
    return (re[0], im[0]) if state.nvec == 1 else (re, im)


def moments(H: Hamiltonian, left: Vector, right: Vector, n_moments: int,
            precision: int | None = None):
    """mu_m = <left|T_m(H/E_max)|right>: shape (n_moments,), (nvec, n_moments), or for a
    realisation batch (n_real, nvec, n_moments). `precision` runs the recurrence in
    another arithmetic form than the vectors' (gqt_moments_form)."""
    R = getattr(H, "n_real", 1)
    re = np.zeros(n_moments * right.nvec * R)
    im = np.zeros(n_moments * right.nvec * R)
    prec = right.precision if precision is None else precision
    _call("gqt_moments_form", H.h, left.h, right.h, n_moments, prec, _dptr(re), _dptr(im))
    if R > 1:
        return re.reshape(R, right.nvec, n_moments), im.reshape(R, right.nvec, n_moments)
    if right.nvec > 1:
        return re.reshape(right.nvec, n_moments), im.reshape(right.nvec, n_moments)
    return re, im


def moments_doubled(H: Hamiltonian, state: Vector, n_moments: int, precision: int | None = None):
    """mu_m = <state|T_m(H/E_max)|state> from n_moments / 2 Chebyshev steps
    (gqt_moments_doubled); shapes as moments()."""
    R = getattr(H, "n_real", 1)
    re = np.zeros(n_moments * state.nvec * R)
    im = np.zeros(n_moments * state.nvec * R)
    prec = state.precision if precision is None else precision
    _call("gqt_moments_doubled", H.h, state.h, n_moments, prec, _dptr(re), _dptr(im))
    if R > 1:
        return re.reshape(R, state.nvec, n_moments), im.reshape(R, state.nvec, n_moments)
    if state.nvec > 1:
        return re.reshape(state.nvec, n_moments), im.reshape(state.nvec, n_moments)
    return re, im


def moments_doubled_device(H: Hamiltonian, state: Vector, n_moments: int, mu_ptr: int,
                           precision: int | None = None) -> None:
    prec = state.precision if precision is None else precision
    _call("gqt_moments_doubled_device", H.h, state.h, n_moments, prec, ctypes.c_void_p(mu_ptr))


def autotune_nvec(H: Hamiltonian, precision: int, n_moments: int, candidates):
    """The vectors-per-launch candidate with the highest measured site-moments/s
    (gqt_autotune_nvec); returns (best, {candidate: rate})."""
    c = np.ascontiguousarray(candidates, dtype=np.int32)
    rates = np.zeros(c.size)
    best = ctypes.c_int()
    _call("gqt_autotune_nvec", H.h, precision, n_moments, c.ctypes.data_as(_ip), c.size,
          ctypes.byref(best), _dptr(rates))
    return best.value, dict(zip(c.tolist(), rates.tolist()))


def moments_device(H: Hamiltonian, left: Vector, right: Vector, n_moments: int,
                   mu_dev_ptr: int, precision: int | None = None) -> None:
    """Moments into device memory (n_moments * nvec double2, moment-major); async.
    `precision` runs the recurrence in another form than the vectors'
    (gqt_moments_device_form)."""
    if precision is None:
        _call("gqt_moments_device", H.h, left.h, right.h, n_moments,
              ctypes.c_void_p(mu_dev_ptr))
    else:
        _call("gqt_moments_device_form", H.h, left.h, right.h, n_moments, precision,
              ctypes.c_void_p(mu_dev_ptr))


def evolve(H: Hamiltonian, direction: int, dt_scaled: float, state: Vector) -> None:
    _call("gqt_evolve", H.h, direction, dt_scaled, state.h)


def evolvex(H: Hamiltonian, direction: int, dt_scaled: float, state: Vector) -> None:
    _call("gqt_evolvex", H.h, direction, dt_scaled, state.h)


def chebyshev_summation(mu_re, mu_im, energy, energy_max: float, volume: float):
    """Jackson damping + Chebyshev sum (src/sigma.cu:76-110) of one moment set."""
    r = np.ascontiguousarray(mu_re, dtype=np.float64).copy()
    i = np.ascontiguousarray(mu_im, dtype=np.float64).copy()
    e = np.ascontiguousarray(energy, dtype=np.float64)
    out = np.zeros(e.size)
    _call("gqt_chebyshev_summation", r.size, _dptr(r), _dptr(i), e.size, _dptr(e),
          float(energy_max), float(volume), _dptr(out))
    return out


def lsqt(input_dir: str, precision: int = FP64, verbose: bool = False,
         max_rows: int = 0) -> bool:
    """The full run of one input directory (lsqt, src/lsqt.cu:135-152). With
    max_rows > 0 the run stops after that many .out rows, leaving a checkpoint that
    the next call resumes (gqt_lsqt_run); returns whether the run is complete."""
    done = ctypes.c_int()
    _call("gqt_lsqt_run", input_dir.encode(), precision, int(verbose), int(max_rows),
          ctypes.byref(done))
    return bool(done.value)


MOMENTS_MAGIC = b"GQTMOMv1"


def read_moments(path: str):
    """Raw moments written with para.in `output_moments`: (re, im), each of shape
    (rows, number_of_moments), one row per .out row in the same order."""
    with open(path, "rb") as f:
        head = f.read(16)
        if len(head) != 16 or head[:8] != MOMENTS_MAGIC:
            raise ValueError(f"{path}: not a moments file")
        m = int(np.frombuffer(head[8:12], dtype="<i4")[0])
        data = np.frombuffer(f.read(), dtype="<f8")
    if m <= 0 or data.size % (2 * m):
        raise ValueError(f"{path}: size is not a whole number of rows")
    rows = data.reshape(-1, m, 2)
    return rows[:, :, 0].copy(), rows[:, :, 1].copy()
