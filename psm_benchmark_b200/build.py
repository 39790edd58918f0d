"""In-tree build of the native libraries (no JIT cache, no pip install).

    python -m psm_benchmark_b200.build

produces, next to this file:
  libpsm_gen.so  - host-only seeded graph/query generators (g++)
  libpsm_b200.so - sm_100a CUDA kernels + C++ host runtime behind the C ABI
                   declared in include/psm_b200.h (nvcc)
  psm_match      - drop-in command-line driver accepting the reference's
                   SubgraphMatching.out flags (g++, links libpsm_b200.so)

Every CUDA source is compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a). Builds are skipped when the output
is newer than all of its inputs.
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
INCLUDE = ROOT / "include"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("PSM_CXX", "/usr/bin/g++")
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))

GEN_SRCS = [CSRC / "gen" / "gen.cpp"]
CORE_CU = sorted((CSRC / "core").glob("*.cu"))
CORE_CPP = sorted((CSRC / "core").glob("*.cpp"))
CORE_HDR = sorted((CSRC / "core").glob("*.h")) + sorted((CSRC / "core").glob("*.cuh"))
CLI_SRCS = [CSRC / "cli" / "psm_match.cpp"]

GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale(out: Path, inputs) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(Path(p).stat().st_mtime > t for p in inputs)


def _run(cmd):
    print("+", " ".join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def build_gen(force: bool = False) -> Path:
    out = PKG / "libpsm_gen.so"
    deps = GEN_SRCS + [INCLUDE / "psm_gen.h"]
    if force or _stale(out, deps):
        _run([CXX, "-std=c++17", "-O3", "-fPIC", "-shared", "-pthread", f"-I{INCLUDE}",
              *GEN_SRCS, "-o", out])
    return out


def build_core(force: bool = False, verbose_ptxas: bool = False) -> Path:
    out = PKG / "libpsm_b200.so"
    if not CORE_CU and not CORE_CPP:
        return out
    deps = CORE_CU + CORE_CPP + CORE_HDR + [INCLUDE / "psm_b200.h"]
    if not (force or _stale(out, deps)):
        return out
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    objs, cmds = [], []
    for src in CORE_CU:
        obj = objdir / (src.stem + ".cu.o")
        if force or _stale(obj, [src] + CORE_HDR + [INCLUDE / "psm_b200.h"]):
            cmd = [NVCC, *GENCODE, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                   "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC / 'core'}",
                   "-c", src, "-o", obj]
            if verbose_ptxas:
                cmd[1:1] = ["-Xptxas", "-v"]
            cmds.append(cmd)
        objs.append(obj)
    for src in CORE_CPP:
        obj = objdir / (src.stem + ".cpp.o")
        if force or _stale(obj, [src] + CORE_HDR + [INCLUDE / "psm_b200.h"]):
            cmds.append([CXX, "-std=c++17", "-O3", "-fPIC", "-pthread", f"-I{INCLUDE}", f"-I{CSRC / 'core'}",
                         f"-I{CUDA_HOME / 'include'}", "-c", src, "-o", obj])
        objs.append(obj)
    # the translation units are independent: compile them side by side
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as pool:
        for f in [pool.submit(_run, c) for c in cmds]:
            f.result()
    _run([NVCC, *GENCODE, "-shared", "-Xcompiler", "-fPIC", *objs, "-o", out,
          "-lcudart", "-lpthread"])
    return out


def build_cli(force: bool = False) -> Path:
    out = PKG / "psm_match"
    if not all(p.exists() for p in CLI_SRCS):
        return out
    lib = PKG / "libpsm_b200.so"
    if force or _stale(out, CLI_SRCS + [lib, INCLUDE / "psm_b200.h"]):
        _run([CXX, "-std=c++17", "-O2", f"-I{INCLUDE}", *CLI_SRCS, f"-L{PKG}", "-lpsm_b200",
              f"-Wl,-rpath,$ORIGIN", "-o", out])
    return out


def build_all(force: bool = False) -> None:
    build_gen(force)
    build_core(force)
    build_cli(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
