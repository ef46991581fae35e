"""Parity of the CUDA path with the oracle, bit for bit, through the C ABI."""
from __future__ import annotations

import numpy as np
import pytest

import cases
import negacyclic as nc
import oracle

pytestmark = pytest.mark.gpu


def run(case: cases.Case) -> np.ndarray:
    with nc.Plan(case.N, case.q_limbs, W=case.W) as plan:
        return plan.multiply(case.a, case.b)


@pytest.mark.parametrize("N", [2, 4, 8, 16, 32, 64, 128, 256])
def test_small_vs_schoolbook(gpu, N):
    c = cases.make_case(N, 868, seed=100 + N)
    want = oracle.schoolbook_py(cases.ints_of_rows(c.a), cases.ints_of_rows(c.b), c.q)
    assert cases.ints_of_rows(run(c)) == want


@pytest.mark.parametrize("N,bits", [
    (512, 868), (1024, 868), (2048, 868), (4096, 868), (8192, 868),
    (16384, 868), (32768, 868), (65536, 868), (1024, 434), (65536, 434),
])
def test_vs_oracle(gpu, N, bits):
    c = cases.make_case(N, bits, seed=N + bits, edge_frac=0.01)
    want = oracle.negacyclic(N, c.q_limbs, c.a, c.b)
    got = run(c)
    bad = np.nonzero((got != want).any(axis=1))[0]
    assert bad.size == 0, f"{bad.size} coefficients differ, first at {bad[:5]}"


@pytest.mark.parametrize("bits", [20, 32, 33, 63, 64, 100, 200, 300, 433, 600, 800, 867, 900, 1000, 1023, 1024])
def test_limb_widths(gpu, bits):
    c = cases.make_case(256, bits, seed=7 * bits)
    assert np.array_equal(run(c), oracle.negacyclic(256, c.q_limbs, c.a, c.b))


@pytest.mark.parametrize("N", [64, 4096, 65536])
def test_edge_operands(gpu, N):
    q = cases.gen_prime(868, 77)
    L = 28
    ql = cases.limbs_of(q, L)
    top = cases.rows_of_ints([q - 1] * N, L)
    zero = np.zeros((N, L), dtype=np.uint32)
    one = np.zeros((N, L), dtype=np.uint32)
    one[0, 0] = 1
    with nc.Plan(N, ql) as plan:
        # the most negative convolution (every coefficient q - 1): sign branch of the CRT
        assert np.array_equal(plan.multiply(top, top), oracle.negacyclic(N, ql, top, top))
        assert not plan.multiply(zero, top).any()
        assert np.array_equal(plan.multiply(one, top), top)
        assert np.array_equal(plan.multiply(top, one), top)


def test_negacyclic_shift_full_size(gpu):
    """a * X^s is a negacyclic rotation of a (size-independent property at N = 65536)."""
    N, L = 65536, 28
    c = cases.make_case(N, 868, seed=31)
    s = 12345
    xs = np.zeros((N, L), dtype=np.uint32)
    xs[s, 0] = 1
    with nc.Plan(N, c.q_limbs) as plan:
        got = cases.ints_of_rows(plan.multiply(c.a, xs))
    a = cases.ints_of_rows(c.a)
    want = [0] * N
    for i, v in enumerate(a):
        j = i + s
        if j < N:
            want[j] = v
        else:
            want[j - N] = (c.q - v) % c.q
    assert got == want


def test_commutative_and_linear_full_size(gpu):
    """a b = b a and a (b1 + b2) = a b1 + a b2 (mod q) at N = 65536."""
    N, L = 65536, 28
    c = cases.make_case(N, 868, seed=41)
    b2 = cases.coeffs(c.q, N, L, seed=4242)
    bsum = cases.rows_of_ints([(x + y) % c.q for x, y in zip(cases.ints_of_rows(c.b), cases.ints_of_rows(b2))], L)
    with nc.Plan(N, c.q_limbs) as plan:
        ab = plan.multiply(c.a, c.b)
        assert np.array_equal(ab, plan.multiply(c.b, c.a))
        ab2 = cases.ints_of_rows(plan.multiply(c.a, b2))
        absum = cases.ints_of_rows(plan.multiply(c.a, bsum))
    abl = cases.ints_of_rows(ab)
    assert absum == [(x + y) % c.q for x, y in zip(abl, ab2)]


def test_device_entry_matches_host_entry(gpu):
    import torch

    c = cases.make_case(16384, 868, seed=5)
    with nc.Plan(c.N, c.q_limbs) as plan:
        host = plan.multiply(c.a, c.b)
        da = torch.from_numpy(c.a.view(np.int32)).to(gpu)
        db = torch.from_numpy(c.b.view(np.int32)).to(gpu)
        dc = torch.empty_like(da)
        stream = torch.cuda.current_stream(gpu)
        plan.multiply_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), stream.cuda_stream)
        stream.synchronize()
        assert np.array_equal(dc.cpu().numpy().view(np.uint32), host)


def test_reference_interface(gpu):
    c = cases.make_case(1024, 868, seed=9)
    point = nc.Point(N=c.N, W=c.W, L=c.L, q=nc.Tensor([c.L], c.q_limbs))
    state = nc.fherma_init(point)
    try:
        out = nc.fherma_run(state, nc.Inputs(nc.Tensor([c.N, c.L], c.a.reshape(-1)),
                                             nc.Tensor([c.N, c.L], c.b.reshape(-1))))
        assert out.c.shape == [c.N, c.L]
        assert np.array_equal(out.c.data.reshape(c.N, c.L), oracle.negacyclic(c.N, c.q_limbs, c.a, c.b))
        with pytest.raises(RuntimeError, match="N\\*L"):
            nc.fherma_run(state, nc.Inputs(nc.Tensor([1], c.a.reshape(-1)[:5]), nc.Tensor([1], c.b.reshape(-1))))
    finally:
        nc.fherma_free(state)
    nc.fherma_free(None)


def test_plans_share_tables_and_repeat(gpu):
    c1 = cases.make_case(4096, 868, seed=1)
    c2 = cases.make_case(1024, 434, seed=2)
    p1 = nc.Plan(c1.N, c1.q_limbs)
    p2 = nc.Plan(c2.N, c2.q_limbs)
    try:
        r1 = p1.multiply(c1.a, c1.b)
        r2 = p2.multiply(c2.a, c2.b)
        assert np.array_equal(p1.multiply(c1.a, c1.b), r1)
        p2.close()
        assert np.array_equal(p1.multiply(c1.a, c1.b), r1)
        assert np.array_equal(r2, oracle.negacyclic(c2.N, c2.q_limbs, c2.a, c2.b))
    finally:
        p1.close()
        p2.close()
