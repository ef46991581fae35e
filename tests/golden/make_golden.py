"""Generate tests/golden/reference_outputs.json from the reference's own binaries.

    python tests/golden/make_golden.py [--out DIR]   # on a machine with a B200 (default: tests/golden)

For every seeded case below it writes a case directory in the platform's format, runs the
reference solution built from its unmodified sources (oracle/_ref/solution) or, where that
binary cannot run the case, the minimally patched build (oracle/_ref/solution_patched: kMaxN
65536 and the L = 28 init self-check throw removed), and records the SHA-256 of every output
c.bin, the reference's own per-case status, and (for N <= 64) the full output as hex. Inputs
are regenerated from the seeds by engel-cuda-negacyclic-multiply_b200/cases.py, so the
fixture stays small. The same cases also run through reference main.cpp linked against this
library (oracle/_ref/dropin_solution) and that digest is recorded beside it.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import subprocess
import sys
import tempfile
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "engel-cuda-negacyclic-multiply_b200"))
import cases  # noqa: E402

REF = ROOT / "oracle" / "_ref"

# name, N, bits, seed, edge_frac, operand kind
CASES = [
    ("n64_868", 64, 868, 101, 0.0, "uniform"),
    ("n1024_868_edge", 1024, 868, 102, 0.01, "uniform"),
    ("n1024_868_allmax", 1024, 868, 103, 0.0, "all_q_minus_1"),
    ("n4096_868_edge", 4096, 868, 104, 0.01, "uniform"),
    ("n32768_868_edge", 32768, 868, 105, 0.01, "uniform"),
    ("n65536_868_edge", 65536, 868, 106, 0.01, "uniform"),
    ("n16_434", 16, 434, 107, 0.0, "uniform"),
    ("n1024_434_edge", 1024, 434, 108, 0.01, "uniform"),
    ("n65536_434_edge", 65536, 434, 109, 0.01, "uniform"),
    ("n256_100", 256, 100, 110, 0.0, "uniform"),
    ("n256_600", 256, 600, 111, 0.0, "uniform"),
    ("n256_1000", 256, 1000, 112, 0.0, "uniform"),
    ("n2_868", 2, 868, 113, 0.0, "uniform"),
]


def build_case(N: int, bits: int, seed: int, edge: float, kind: str) -> cases.Case:
    c = cases.make_case(N, bits, seed, edge_frac=edge)
    if kind == "all_q_minus_1":
        top = cases.rows_of_ints([c.q - 1] * N, c.L)
        c.a, c.b = top, top.copy()
    return c


def run_binary(binary: Path, c: cases.Case) -> tuple[str, bytes | None, str]:
    with tempfile.TemporaryDirectory(prefix="golden_") as tmp:
        root = Path(tmp)
        cases.write_case_dir(root, c.N, c.W, c.L, c.q, [(c.a, c.b)])
        r = subprocess.run([str(binary), str(root)], capture_output=True, text=True, timeout=600)
        if r.returncode != 0:
            return "init_failed", None, (r.stderr.strip().splitlines() or ["?"])[-1][:200]
        res = cases.read_results(root)
        status = res["cases"][0]["status"] if res["cases"] else "missing"
        if status != "ok":
            return status, None, ""
        return "ok", (root / "out" / "000000" / "c.bin").read_bytes(), ""


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(Path(__file__).resolve().parent))
    a = ap.parse_args()
    out = Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    records = []
    for name, N, bits, seed, edge, kind in CASES:
        c = build_case(N, bits, seed, edge, kind)
        rec = {"name": name, "N": N, "bits": bits, "seed": seed, "edge_frac": edge, "operands": kind}
        st, data, msg = run_binary(REF / "solution", c)
        rec["unmodified"] = {"status": st, "message": msg}
        if st == "ok":
            rec["binary"] = "solution"
        else:
            st, data, msg = run_binary(REF / "solution_patched", c)
            rec["patched"] = {"status": st, "message": msg}
            rec["binary"] = "solution_patched" if st == "ok" else None
        if data is not None:
            rec["sha256"] = hashlib.sha256(data).hexdigest()
            if N <= 64:
                rec["c_hex"] = data.hex()
        dst, ddata, dmsg = run_binary(REF / "dropin_solution", c)
        rec["dropin"] = {"status": dst, "sha256": hashlib.sha256(ddata).hexdigest() if ddata else None}
        records.append(rec)
        print(json.dumps({k: v for k, v in rec.items() if k != "c_hex"}), flush=True)
    (out / "reference_outputs.json").write_text(json.dumps({"cases": records}, indent=1))
    return 0


if __name__ == "__main__":
    sys.exit(main())
