"""The C++ contract entry points (fherma_init / fherma_run / fherma_free, reference fherma.h:45-47)
run as a platform harness runs them, on a B200:

  bin/solution                   this library's harness runner, linked against libnegacyclic_b200.so
  oracle/_ref/dropin_solution    the reference's own main.cpp linked against libnegacyclic_b200.so
  oracle/_ref/solve_cu/build/solution
                                 the reference's generated CMake project, unmodified, with the
                                 single-file dropin/solve.cu as its solve.cu

Each binary runs every golden case directory with two products per process, (a, b) and then
(b, a), so the second fherma_run takes the output vector the state prepared after the first
call; both must have the reference's own SHA-256 digest (products commute). The bench's
N = 65536 workload (seed 20261203, 1% edge values) runs the same way against the oracle.
Matches reference main.cpp:59-86 (init, timed run per case, c.bin per case, free).
"""
from __future__ import annotations

import hashlib
import os
import json
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import cases
import oracle

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
import make_golden  # noqa: E402

pytestmark = pytest.mark.gpu

RECORDS = json.loads((GOLDEN / "reference_outputs.json").read_text())["cases"]
BINARIES = {
    "library_runner": ROOT / "engel-cuda-negacyclic-multiply_b200" / "bin" / "solution",
    "reference_main_cpp": ROOT / "oracle" / "_ref" / "dropin_solution",
    "solve_cu_cmake": ROOT / "oracle" / "_ref" / "solve_cu" / "build" / "solution",
}


def _binary(name: str) -> Path:
    b = BINARIES[name]
    if not b.exists():
        if name == "library_runner":
            pytest.fail(f"{b} is missing: run build.py")
        pytest.skip(f"{b.relative_to(ROOT)} is not built (it needs the reference's sources at build time)")
    return b


def _run(binary: Path, c, tmp: Path) -> list[np.ndarray]:
    cases.write_case_dir(tmp, c.N, c.W, c.L, c.q, [(c.a, c.b), (c.b, c.a)])
    r = subprocess.run([str(binary), str(tmp)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-1000:]
    res = cases.read_results(tmp)
    assert [row["status"] for row in res["cases"]] == ["ok", "ok"], r.stderr[-1000:]
    return [cases.read_output(tmp, i, c.N, c.L) for i in range(2)]


@pytest.mark.parametrize("name", list(BINARIES))
@pytest.mark.parametrize("r", RECORDS, ids=[r["name"] for r in RECORDS])
def test_contract_binary_matches_reference_digest(gpu, name, r, tmp_path):
    binary = _binary(name)
    c = make_golden.build_case(r["N"], r["bits"], r["seed"], r["edge_frac"], r["operands"])
    for i, out in enumerate(_run(binary, c, tmp_path)):
        assert hashlib.sha256(np.ascontiguousarray(out).tobytes()).hexdigest() == r["sha256"], f"call {i}"


@pytest.mark.parametrize("name", list(BINARIES))
def test_contract_binary_on_the_bench_workload(gpu, name, tmp_path):
    binary = _binary(name)
    c = cases.make_case(65536, 868, 20261203, edge_frac=0.01)
    want = oracle.negacyclic(c.N, c.q_limbs, c.a, c.b)
    for i, out in enumerate(_run(binary, c, tmp_path)):
        assert np.array_equal(out, want), f"call {i}: {int((out != want).any(axis=1).sum())} coefficients differ"


def test_host_path_trace(gpu, tmp_path):
    """NC_TRACE=1: one line per fherma_run with the call's phases in order (device clock for the
    transfers and kernels, host clock for staging, enqueueing and the copy-out)."""
    binary = _binary("library_runner")
    c = cases.make_case(16384, 868, 77, edge_frac=0.01)
    cases.write_case_dir(tmp_path, c.N, c.W, c.L, c.q, [(c.a, c.b)] * 3)
    env = dict(os.environ, NC_TRACE="1")
    r = subprocess.run([str(binary), str(tmp_path)], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-1000:]
    lines = [ln for ln in r.stderr.splitlines() if ln.startswith("nc_trace ")]
    assert len(lines) == 3, r.stderr[-1000:]
    for ln in lines:
        f = dict((k, float(v)) for k, v in (x.split("=") for x in ln.split()[1:]))
        assert 0 < f["a_uploaded"] <= f["a_forward"]
        assert f["a_uploaded"] <= f["b_uploaded"] <= f["product"] <= f["downloaded"]
        assert 0 < f["a_staged"] <= f["b_staged"] <= f["enqueued"] <= f["collected"]
    want = oracle.negacyclic(c.N, c.q_limbs, c.a, c.b)
    assert np.array_equal(cases.read_output(tmp_path, 2, c.N, c.L), want)
