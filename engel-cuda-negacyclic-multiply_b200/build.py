"""Build the sm_100a shared library and the harness-format runner in-tree.

    python build.py            # incremental
    python build.py --clean    # from scratch

Outputs (git-ignored, shipped with the tree):
    lib/libnegacyclic_b200.so   C ABI (include/negacyclic_b200.h) + fherma_init/run/free
    bin/solution                harness runner: reads a case directory, writes out/*/c.bin
    dropin/solve.cu             the whole library as one source file, for a platform project that
                                accepts solve.cu and nothing else (its generated CMakeLists.txt
                                compiles main.cpp + solve.cu with -arch=<arch> -rdc=true -dlto)
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
OBJ = PKG / "_build"
LIB = PKG / "lib" / "libnegacyclic_b200.so"
BIN = PKG / "bin" / "solution"
SOLVE_CU = PKG / "dropin" / "solve.cu"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", f"-I{INCLUDE}", f"-I{CSRC}"]

LIB_SOURCES = ["hostmath.cpp", "k_dec.cu", "k_row.cu", "k_crt.cu", "k_batch.cu", "kernels.cu", "batch.cu",
               "engine.cu", "server.cu", "api.cu", "noalloc.cu", "k_residues.cu", "k_crt_tc.cu", "k_dec_tc.cu",
               "k_w32.cu"]
RUNNER_SOURCES = ["runner.cpp"]


def _headers(src: Path | None = None) -> list[Path]:
    """Headers `src` includes, transitively (quoted includes found in csrc/ or include/)."""
    if src is None:
        return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")))
    seen: set[Path] = set()
    todo = [src]
    while todo:
        f = todo.pop()
        for line in f.read_text(errors="replace").splitlines():
            line = line.strip()
            if not line.startswith("#include \""):
                continue
            name = line.split('"')[1]
            for d in (CSRC, INCLUDE):
                h = d / name
                if h.exists() and h not in seen:
                    seen.add(h)
                    todo.append(h)
    return sorted(seen)


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, verbose: bool) -> Path:
    obj = OBJ / (src.name + ".o")
    if not _stale(obj, [src] + _headers(src)):
        return obj
    cmd = [NVCC, *ARCH, *COMMON, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cu" and verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        (OBJ / (src.name + ".ptxas.txt")).write_text(r.stderr)
    return obj


# One translation unit of every library source, in dependency order.
SOLVE_CU_SOURCES = ["hostmath.cpp", "kernels.cu", "k_dec.cu", "k_row.cu", "k_crt.cu", "k_dec_tc.cu", "k_crt_tc.cu",
                    "k_w32.cu", "k_batch.cu", "k_residues.cu", "batch.cu", "engine.cu", "server.cu", "api.cu", "noalloc.cu"]

SOLVE_CU_HEAD = """\
// solve.cu: the B200 negacyclic product library (c = a*b mod (X^N + 1, q)) as one source file,
// generated from engel-cuda-negacyclic-multiply_b200/csrc by build.py. Do not edit: edit csrc/.
//
// It implements the platform contract fherma_init / fherma_run / fherma_free against the project's
// own fherma.h (the one include left unexpanded), and also carries the library's C ABI.
//
// The platform's CMake project builds it with -arch=<arch> -rdc=true and link-time optimisation
// (-dlto). nvcc 12.9's LTO device link lowers sm_100a code for the plain sm_100 target, which has
// no tcgen05 instructions, so this file leaves the tensor-core kernels out (NC_NO_TCGEN05): the
// residue and CRT stages run on the integer pipes, every other kernel is the library's own, and
// the results are the same bits. libnegacyclic_b200.so (build.py) keeps the tensor-core stages.
#define NC_NO_TCGEN05 1
#pragma nv_diag_suppress 177  // helpers unused once the tensor-core kernels are left out
#pragma nv_diag_suppress 128  // loops a narrow instantiation never enters
"""


def solve_cu_text() -> str:
    """The amalgamation: every source of SOLVE_CU_SOURCES with its quoted includes expanded once,
    `#pragma once` dropped, and `#include "fherma.h"` kept for the project's own copy."""
    seen: set = set()
    out = [SOLVE_CU_HEAD]

    def expand(path: Path) -> None:
        for line in path.read_text().splitlines():
            s = line.strip()
            if s == "#pragma once":
                continue
            if s.startswith("#include \""):
                name = s.split('"')[1]
                if name == "fherma.h":
                    if name not in seen:
                        seen.add(name)
                        out.append('#include "fherma.h"')
                    continue
                for d in (CSRC, INCLUDE):
                    h = d / name
                    if h.exists():
                        if h not in seen:
                            seen.add(h)
                            out.append(f"// ---- {name}")
                            expand(h)
                        break
                else:
                    raise RuntimeError(f"{path.name}: cannot find {name}")
                continue
            out.append(line)

    for src in SOLVE_CU_SOURCES:
        out.append(f"// ==== {src}")
        expand(CSRC / src)
    return "\n".join(out) + "\n"


def write_solve_cu() -> Path:
    text = solve_cu_text()
    if not SOLVE_CU.exists() or SOLVE_CU.read_text() != text:
        SOLVE_CU.parent.mkdir(parents=True, exist_ok=True)
        SOLVE_CU.write_text(text)
    return SOLVE_CU


def build(clean: bool = False, verbose: bool = False) -> Path:
    if clean and OBJ.exists():
        shutil.rmtree(OBJ)
    OBJ.mkdir(parents=True, exist_ok=True)
    LIB.parent.mkdir(parents=True, exist_ok=True)
    BIN.parent.mkdir(parents=True, exist_ok=True)
    sources = [CSRC / s for s in LIB_SOURCES if (CSRC / s).exists()]
    with cf.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), sources))
    if _stale(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    runner = [CSRC / s for s in RUNNER_SOURCES if (CSRC / s).exists()]
    if runner and _stale(BIN, runner + [LIB] + _headers()):
        cmd = ["g++", "-O2", "-std=c++17", f"-I{INCLUDE}", *map(str, runner), "-o", str(BIN),
               f"-L{LIB.parent}", "-lnegacyclic_b200", f"-Wl,-rpath,$ORIGIN/../lib"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"runner link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    write_solve_cu()
    return LIB


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("--verbose", action="store_true", help="keep ptxas register/spill reports in _build/")
    a = ap.parse_args()
    print(build(a.clean, a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
