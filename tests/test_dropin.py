"""The single-file drop-in: dropin/solve.cu, the whole library as the one source file a platform
project takes ("solve.cu, and nothing else", reference README.md:7-9), built by the reference's
generated CMake project unchanged (reference CMakeLists.txt:1-20: main.cpp + solve.cu,
-arch=<FHERMA_CUDA_ARCH> -rdc=true -dlto)."""
from __future__ import annotations

import os
import re
import shutil
import subprocess
from pathlib import Path

import pytest

import build

ROOT = Path(__file__).resolve().parent.parent
REFERENCE = Path(os.environ.get("NC_REFERENCE_DIR", "/root/reference"))
CMAKE_BIN = ROOT / "oracle" / "_ref" / "solve_cu" / "build" / "solution"


def test_solve_cu_is_generated_from_the_current_sources():
    text = build.solve_cu_text()
    path = build.write_solve_cu()
    assert path.read_text() == text


def test_solve_cu_is_self_contained():
    text = build.solve_cu_text()
    quoted = re.findall(r'^\s*#include\s+"([^"]+)"', text, flags=re.M)
    assert quoted == ["fherma.h"], quoted  # the platform's own header, nothing of this repository
    assert "#pragma once" not in text
    for fn in ("fherma_init(const fherma::Point&", "fherma_run(void* state, const fherma::Inputs&",
               "fherma_free(void* state)"):
        assert fn in text, fn
    # the single-file build leaves the tensor-core kernels out (no tcgen05 under -dlto)
    assert text.index("#define NC_NO_TCGEN05 1") < text.index("#define NC_HAS_TCGEN05")


@pytest.mark.skipif(not (REFERENCE / "CMakeLists.txt").exists() or shutil.which("cmake") is None,
                    reason="needs the reference's generated CMake project and cmake")
def test_reference_cmake_project_builds_solve_cu():
    """make -C oracle _ref/solve_cu/build/solution: the reference's CMakeLists.txt, main.cpp and
    fherma.h copied unchanged beside solve.cu, configured with FHERMA_CUDA_ARCH=sm_100a. Rebuilt
    only when solve.cu changed (a full build takes several minutes)."""
    build.write_solve_cu()
    r = subprocess.run(["make", "-C", str(ROOT / "oracle"), f"REF={REFERENCE}", "_ref/solve_cu/build/solution"],
                       capture_output=True, text=True, timeout=1800)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert CMAKE_BIN.exists()
    for name in ("CMakeLists.txt", "main.cpp", "fherma.h"):
        assert (CMAKE_BIN.parent.parent / name).read_bytes() == (REFERENCE / name).read_bytes(), name
    syms = subprocess.run(["nm", "-C", str(CMAKE_BIN)], capture_output=True, text=True).stdout
    for fn in ("fherma_init(fherma::Point const&)", "fherma_run(void*, fherma::Inputs const&)", "fherma_free(void*)"):
        assert fn in syms, fn
