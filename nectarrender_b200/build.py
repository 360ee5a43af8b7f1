"""Builds the native parts of nectarrender_b200 in-tree.

libnectar_b200.so  CUDA kernels (sm_100a) + host code + the C ABI of
                   include/nectar_b200.h
_pathtracer*.so    pybind11 module re-creating the reference's Python API on
                   top of that C ABI

Device code is compiled with --use_fast_math, as the reference's CUDA build
is; host code is compiled without fast-math or FMA contraction, as the
reference's host code is, because object transforms, the camera and the
sample pattern are computed on the host in both.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
INCLUDE = HERE.parent / "include"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-std=c++17", "-lineinfo", "--use_fast_math",
    "-Xcompiler", "-fPIC,-O2", "-Xptxas", "-O3",
    f"-I{CSRC}", f"-I{INCLUDE}",
]
CU_SOURCES = ["capi.cu", "integrator.cu", "wavefront.cu", "bvh_build.cu", "image_ops.cu",
              "static_wave.cu", "viewport.cu", "conv_tc.cu",
              "denoiser.cu", "nrc.cu", "mesh_ingest.cu", "sky_alias.cu"]
CPP_SOURCES = ["host_io.cpp"]
LIB = HERE / "libnectar_b200.so"


def _ext_suffix() -> str:
    return sysconfig.get_config_var("EXT_SUFFIX") or ".so"


MODULE = HERE / f"_pathtracer{_ext_suffix()}"


def _newer(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")
    if os.environ.get("NR_BUILD_VERBOSE"):
        sys.stderr.write(r.stdout + r.stderr)


def _compile(src: str) -> Path:
    s = CSRC / src
    obj = BUILD / (src + ".o")
    if _newer(obj, [s] + _headers()):
        if src.endswith(".cu"):
            extra = ["-Xptxas", "-v"] if os.environ.get("NR_PTXAS_VERBOSE") else []
            _run([NVCC, *NVCC_FLAGS, *extra, "-c", str(s), "-o", str(obj)])
        else:
            _run(["g++", "-O2", "-std=c++17", "-fPIC", f"-I{CSRC}", f"-I{INCLUDE}",
                  "-c", str(s), "-o", str(obj)])
    return obj


def build_library() -> Path:
    BUILD.mkdir(exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(_compile, CU_SOURCES + CPP_SOURCES))
    if _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs),
              f"-L{CUDA_HOME}/lib64", "-lcudart"])
    return LIB


def build_module() -> Path:
    import pybind11
    src = CSRC / "pathtracer_module.cpp"
    if _newer(MODULE, [src, LIB] + _headers()):
        py_inc = sysconfig.get_paths()["include"]
        _run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", str(src),
              f"-I{pybind11.get_include()}", f"-I{py_inc}", f"-I{INCLUDE}",
              f"-L{HERE}", "-lnectar_b200", "-Wl,-rpath,$ORIGIN",
              "-o", str(MODULE)])
    return MODULE


def build_all() -> None:
    build_library()
    build_module()


if __name__ == "__main__":
    build_all()
    print(LIB)
    print(MODULE)
