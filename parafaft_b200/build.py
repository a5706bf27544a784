"""Build the native parts of parafaft_b200 in-tree.

* ``parafaft_b200/lib/libb200fft.so`` — the CUDA transform engine and its C ABI
  (``include/b200fft.h``), compiled for sm_100a only.
* ``parafaft_b200/lib/libparafaft_b200_drivers.so`` — ParaFaFT's own
  ``ParaFaFT_C2C``/``ParaFaFT_R2C`` orchestrators instantiated with
  ``B200Backend<T>`` and ``B200GridBackend<D, T>``, behind a small C ABI used
  by the tests and the benchmark. It does not link cuFFT.
* ``parafaft_b200/lib/libparafaft_cufft_drivers.so`` — the same orchestrators
  on the reference ``CuFFTBackend<T>`` as well (the comparison on the same
  GPU); the only library that links cuFFT.
Both need the ParaFaFT headers at compile time, so they are only (re)built
where those exist; elsewhere the prebuilt libraries are used as they are.

Run as ``python -m parafaft_b200.build [--force]``.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INTEG = PKG / "integration"
LIB = PKG / "lib"
OBJ = PKG / "_build"
INCLUDE = ROOT / "include"

ENGINE_SO = LIB / "libb200fft.so"
DRIVERS_SO = LIB / "libparafaft_b200_drivers.so"
CUFFT_DRIVERS_SO = LIB / "libparafaft_cufft_drivers.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC"] + ARCH

ENGINE_SOURCES = ["api.cu", "fg.cu", "fs_c2c_f32.cu", "fs_c2c_f64.cu",
                  "fs_r2c_f32.cu", "fs_r2c_f64.cu", "fft_tc.cu", "fft_tc5.cu", "fft_tma.cu",
                  "noalloc.cu", "fft_sched.cu", "fs_colpair.cu",
                  "fft_tc5col.cu"]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def reference_root() -> Path | None:
    """ParaFaFT source tree, if present on this machine: $PARAFAFT_ROOT, else a
    ``reference`` checkout beside this repository."""
    env = os.environ.get("PARAFAFT_ROOT")
    for c in ([Path(env)] if env else []) + [ROOT.parent / "reference"]:
        if (c / "parafaft_r2c.hpp").exists():
            return c
    return None


def _newer(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:4]) + " ...")


def build_engine(force: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    LIB.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + [INCLUDE / "b200fft.h"]
    jobs = []
    objs = []
    for src in ENGINE_SOURCES:
        s = CSRC / src
        o = OBJ / (s.stem + ".o")
        objs.append(o)
        if force or _newer(o, [s] + headers):
            jobs.append([_nvcc(), *NVCC_FLAGS, "-I", str(INCLUDE), "-c", str(s), "-o", str(o)])
    if jobs:
        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            list(ex.map(_run, jobs))
    if force or jobs or _newer(ENGINE_SO, objs):
        _run([_nvcc(), *ARCH, "-shared", "-o", str(ENGINE_SO), *map(str, objs)])
    return ENGINE_SO


def build_drivers(force: bool = False) -> Path | None:
    ref = reference_root()
    src = INTEG / "parafaft_drivers.cu"
    if ref is None:
        return DRIVERS_SO if DRIVERS_SO.exists() else None
    deps = [src, INCLUDE / "fft_backend_b200.hpp", INCLUDE / "fft_backend_b200_grid.hpp",
            INCLUDE / "b200fft.h",
            INTEG / "mpi_shim" / "mpi.h", ENGINE_SO]
    common = [_nvcc(), *NVCC_FLAGS, "-I", str(INCLUDE), "-I", str(INTEG / "mpi_shim"),
              "-I", str(ref), "-shared", str(src)]
    jobs = []
    if force or _newer(DRIVERS_SO, deps):
        jobs.append(common + ["-o", str(DRIVERS_SO), "-L", str(LIB), "-lb200fft",
                              "-Xlinker", "-rpath,$ORIGIN"])
    if force or _newer(CUFFT_DRIVERS_SO, deps):
        jobs.append(common + ["-DPFB_WITH_CUFFT", "-o", str(CUFFT_DRIVERS_SO), "-L", str(LIB),
                              "-lb200fft", "-lcufft", "-Xlinker", "-rpath,$ORIGIN"])
    if jobs:
        with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
            list(ex.map(_run, jobs))
    return DRIVERS_SO


def build_all(force: bool = False) -> None:
    build_engine(force)
    build_drivers(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built", ENGINE_SO, DRIVERS_SO if DRIVERS_SO.exists() else "(no drivers)")
