"""Golden vectors from the reference itself (tests/golden/reference_outputs.json, written by
tests/golden/make_golden.py running the reference's solve.cu + main.cpp on a B200).

The oracle must reproduce every reference output digest (CPU), and so must this library (GPU).
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
import make_golden  # noqa: E402

RECORDS = json.loads((GOLDEN / "reference_outputs.json").read_text())["cases"]
IDS = [r["name"] for r in RECORDS]


def _case(r):
    return make_golden.build_case(r["N"], r["bits"], r["seed"], r["edge_frac"], r["operands"])


def test_fixture_covers_the_contract():
    names = {r["name"] for r in RECORDS}
    assert {"n65536_868_edge", "n1024_868_allmax", "n1024_434_edge", "n2_868"} <= names
    for r in RECORDS:
        assert r["sha256"], r["name"]
        # the reference's main.cpp linked against this library gave the reference's bytes
        assert r["dropin"]["sha256"] == r["sha256"], r["name"]


def test_unmodified_reference_rejects_868_bit_points():
    """Recorded behaviour of the unmodified reference: its L = 28 init self-check throws."""
    for r in RECORDS:
        if r["bits"] == 868 and r["N"] <= 32768:
            assert r["unmodified"]["status"] == "init_failed"
            assert "Barrett reduction does not match division" in r["unmodified"]["message"]
        if r["bits"] != 868 and r["N"] <= 32768:
            assert r["unmodified"]["status"] == "ok"


@pytest.mark.parametrize("r", RECORDS, ids=IDS)
def test_oracle_matches_reference_output(r):
    c = _case(r)
    out = oracle.negacyclic(c.N, c.q_limbs, c.a, c.b)
    assert hashlib.sha256(out.tobytes()).hexdigest() == r["sha256"]
    if "c_hex" in r:
        assert out.tobytes().hex() == r["c_hex"]


@pytest.mark.gpu
@pytest.mark.parametrize("r", RECORDS, ids=IDS)
def test_library_matches_reference_output(gpu, r):
    import negacyclic as nc

    c = _case(r)
    with nc.Plan(c.N, c.q_limbs, W=c.W) as plan:
        out = plan.multiply(c.a, c.b)
    assert hashlib.sha256(np.ascontiguousarray(out).tobytes()).hexdigest() == r["sha256"]
