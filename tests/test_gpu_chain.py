"""Chained products x_0 * x_1 * ... * x_{m-1} mod (X^N + 1, q) in one pass (residues of every
operand, every forward transform and pointwise product in the row stage, one inverse transform,
one CRT) equal the reference's pairwise products chained on the host: the oracle's
negacyclic(negacyclic(x_0, x_1), x_2) ... bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

import cases
import negacyclic as nc
import oracle

pytestmark = pytest.mark.gpu


def chained_oracle(N, q_limbs, xs):
    acc = xs[0]
    for x in xs[1:]:
        acc = oracle.negacyclic(N, q_limbs, acc, x)
    return acc


def operands(N, bits, m, seed, edge_frac=0.02):
    c = cases.make_case(N, bits, seed=seed, edge_frac=edge_frac)
    xs = [c.a, c.b] + [cases.coeffs(c.q, N, c.L, seed * 7 + 3 + f, edge_frac) for f in range(m - 2)]
    return c, xs


@pytest.mark.parametrize("N,bits,m", [(2, 868, 3), (64, 868, 3), (256, 434, 4), (1024, 868, 3),
                                      (4096, 434, 3), (16384, 600, 4), (65536, 868, 3), (65536, 731, 4)])
def test_chain_matches_pairwise_oracle(gpu, N, bits, m):
    c, xs = operands(N, bits, m, seed=31 * N + bits + m)
    want = chained_oracle(N, c.q_limbs, xs)
    with nc.Plan(N, c.q_limbs, W=c.W, factors=m) as plan:
        assert plan.factors == m
        got = plan.multiply_chain(xs)
    assert np.array_equal(got, want)


def test_chain_all_q_minus_one(gpu):
    """Every coefficient at q - 1: the largest integer coefficients the prime bound has to cover."""
    N, bits, m = 4096, 868, 3
    q = cases.gen_prime(bits, 91)
    L = (bits + 31) // 32
    ones = np.tile(cases.limbs_of(q - 1, L), (N, 1))
    with nc.Plan(N, cases.limbs_of(q, L), factors=m) as plan:
        got = plan.multiply_chain([ones] * m)
    assert np.array_equal(got, chained_oracle(N, cases.limbs_of(q, L), [ones] * m))


def test_chain_prime_counts(gpu):
    """The prime count follows (m - 1) log2 N + m bits(q) + 4: three 868-bit operands at N = 65536
    need 43 primes (so the CRT runs on the integer pipes), two need 29."""
    q = cases.limbs_of(cases.gen_prime(868, 92), 28)
    with nc.Plan(65536, q) as two, nc.Plan(65536, q, factors=3) as three:
        assert two.k == 29 and two.crt_engine == nc.CRT_TC_I8
        assert three.k == 43 and three.crt_engine == nc.CRT_IMAD


def test_chain_device_and_plain_products_on_one_plan(gpu):
    """Device operands through nc_multiply_chain_device, then an ordinary product on the same chain
    plan (its larger prime set gives the same canonical output)."""
    import torch

    N, bits, m = 8192, 434, 4
    c, xs = operands(N, bits, m, seed=93)
    want = chained_oracle(N, c.q_limbs, xs)
    with nc.Plan(N, c.q_limbs, factors=m) as plan:
        dev = [torch.from_numpy(x.view(np.int32).copy()).cuda() for x in xs]
        out = torch.empty_like(dev[0])
        stream = torch.cuda.current_stream().cuda_stream
        for _ in range(2):
            out.zero_()
            plan.multiply_chain_device([t.data_ptr() for t in dev], out.data_ptr(), stream)
            torch.cuda.synchronize()
            assert np.array_equal(out.cpu().numpy().view(np.uint32).reshape(N, -1), want)
        pair = plan.multiply(xs[0], xs[1])
        assert np.array_equal(pair, oracle.negacyclic(N, c.q_limbs, xs[0], xs[1]))


def test_chain_operand_count_checked(gpu):
    c, xs = operands(64, 434, 3, seed=94)
    with nc.Plan(64, c.q_limbs, factors=3) as plan:
        with pytest.raises(nc.NegacyclicError):
            plan.multiply_chain(xs[:2])
