"""Build the native library in-tree: gpuqt_b200/lib/libgpuqt_b200.so and the CLI
gpuqt_b200/lib/lsqt_b200.

CUDA sources are compiled for sm_100a only; host C++ with g++. Objects are rebuilt
when a source or any header under csrc/ or include/ is newer. Run as
``python -m gpuqt_b200.build`` (or through ``__graft_entry__.build()``).
"""
from __future__ import annotations

import os
import shlex
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib")
SO = os.path.join(LIB, "libgpuqt_b200.so")
CLI = os.path.join(LIB, "lsqt_b200")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["gqt_runtime.cu", "gqt_algo.cu", "gqt_forms_fp64.cu", "gqt_forms_fp32.cu",
              "gqt_forms_fp32x.cu",
              "gqt_forms_fp64_coded.cu", "gqt_forms_fp32_coded.cu", "gqt_noalloc.cu",
              "gqt_stage.cu"]
CPP_SOURCES = ["host/model.cpp", "host/vector_ham.cpp", "host/sigma.cpp", "host/lsqt.cpp",
               "host/checkpoint.cpp", "host/batch_run.cpp"]

NVCC_FLAGS = ARCH + ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
                     "-Xptxas", "-v", f"-I{INCLUDE}", f"-I{CSRC}"]
# Extra nvcc flags (e.g. -DGQT_VEC_STREAMS=1 to build a pipeline variant for timing).
NVCC_FLAGS += shlex.split(os.environ.get("GQT_NVCC_FLAGS", ""))
# -ffp-contract=off keeps the host arithmetic (random draws, Chebyshev sums) in the
# reference's rounding: every product and sum rounded on its own.
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-Wall", f"-I{INCLUDE}",
             f"-I{CSRC}", f"-I{CUDA_HOME}/include"]


def _headers() -> list[str]:
    out = []
    for base in (CSRC, INCLUDE):
        for dp, _, files in os.walk(base):
            out += [os.path.join(dp, f) for f in files if f.endswith((".h", ".cuh"))]
    return out


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str], log: str | None = None) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if log is not None:
        with open(log, "w") as f:
            f.write(r.stdout + r.stderr)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))


def build(verbose: bool = False) -> str:
    """Compile what is stale; returns the path of the shared library."""
    if not os.path.exists(NVCC) and not shutil.which("nvcc"):
        raise RuntimeError("nvcc not found: set CUDA_HOME")
    nvcc = NVCC if os.path.exists(NVCC) else shutil.which("nvcc")
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    hdrs = _headers()
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs):
            jobs.append([nvcc] + NVCC_FLAGS + ["-c", s, "-o", o])
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs):
            jobs.append(["g++"] + CXX_FLAGS + ["-c", s, "-o", o])
    main_src = os.path.join(CSRC, "host", "main.cpp")
    main_obj = os.path.join(OBJ, "main.cpp.o")
    if _stale(main_obj, [main_src] + hdrs):
        jobs.append(["g++"] + CXX_FLAGS + ["-c", main_src, "-o", main_obj])

    def one(cmd):
        log = cmd[-1] + ".log"
        if verbose:
            print(" ".join(cmd), flush=True)
        _run(cmd, log)

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        list(ex.map(one, jobs))

    if _stale(SO, objs):
        _run([nvcc] + ARCH + ["-shared", "-cudart", "static", "-o", SO] + objs +
             ["-lpthread", "-ldl", "-lrt"])
    if _stale(CLI, [SO, main_obj]):
        _run(["g++", "-o", CLI, main_obj, f"-L{LIB}", "-lgpuqt_b200",
              "-Wl,-rpath,$ORIGIN"])
    return SO


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
