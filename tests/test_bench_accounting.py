"""The bench's roofline accounting (bench.stage_work): algorithmic IMAD per stage under the plan's
row configuration. The per-stage split moves with the row block; the product total must not."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
import bench  # noqa: E402


def product_imad(k: int, N: int, L: int) -> float:
    logN = N.bit_length() - 1
    return 8 * k * N * (1.5 * logN + 7) + 6 * k * N * L + 4 * L * N


@pytest.mark.parametrize("log_n", range(1, 17))
@pytest.mark.parametrize("k,L", [(29, 28), (15, 14), (48, 32)])
def test_stage_split_sums_to_the_product_for_every_row_block(log_n, k, L):
    N = 1 << log_n
    for log_n2 in range(0, log_n + 1):
        work = bench.stage_work(k, N, L, log_n2)
        assert sum(work) == pytest.approx(product_imad(k, N, L), rel=0, abs=1e-6)
        assert all(w > 0 for w in work)


def test_row_stage_counts_the_row_block_stages():
    # N = 2^16, 868-bit q, row blocks of 2^11: three transforms of 11 stages plus the pointwise product
    k, N, L = 29, 65536, 28
    assert bench.stage_work(k, N, L, 11)[1] == 8 * (3 * k * (N // 2) * 11 + k * N) == 266_076_160
    assert bench.stage_work(k, N, L, 12)[1] == 8 * (3 * k * (N // 2) * 12 + k * N)
    with pytest.raises(ValueError):
        bench.stage_work(k, N, L, 17)
