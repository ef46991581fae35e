"""The residue stage of the plan's own products on the tensor cores (k_dec_tc, the default) and on
the integer pipes (k_dec): both give the oracle's product bit for bit, for every operand load width
(L a multiple of 4, even, odd), partial tiles (N < 128), every column-transform length N1 = 1 .. 32
(row configurations), one to three MMA passes (up to 48 primes), the host path and chained
products."""
from __future__ import annotations

import numpy as np
import pytest

import cases
import negacyclic as nc
import oracle

pytestmark = pytest.mark.gpu


def _both_engines(plan, a, b):
    out = {}
    for engine in (nc.RESIDUES_TC_I8, nc.RESIDUES_IMAD):
        plan.residue_engine = engine
        assert plan.residue_engine == engine
        out[engine] = plan.multiply(a, b)
    plan.residue_engine = nc.RESIDUES_TC_I8
    return out


@pytest.mark.parametrize("N,bits", [(2, 868), (8, 100), (64, 600), (128, 434), (256, 868), (1024, 970),
                                    (4096, 31), (16384, 434), (65536, 868), (65536, 600), (8192, 200)])
def test_both_residue_engines_match_the_oracle(gpu, N, bits):
    c = cases.make_case(N, bits, seed=7 * N + bits, edge_frac=0.02)
    want = oracle.negacyclic(N, c.q_limbs, c.a, c.b)
    with nc.Plan(N, c.q_limbs, W=c.W) as plan:
        assert plan.k <= 32 and plan.residue_engine == nc.RESIDUES_TC_I8
        got = _both_engines(plan, c.a, c.b)
    assert np.array_equal(got[nc.RESIDUES_TC_I8], want)
    assert np.array_equal(got[nc.RESIDUES_IMAD], want)


@pytest.mark.parametrize("N,cfg", [(65536, (11, 3, 256)), (65536, (13, 4, 512)), (4096, (7, 3, 256)),
                                   (4096, (12, 4, 256)), (1024, (6, 4, 256)), (32768, (10, 3, 256))])
def test_every_column_length(gpu, N, cfg):
    """N1 = N / 2^log_block from 1 to 32 selects k_dec_tc<log2 N1>."""
    assert cfg in nc.row_variants(N.bit_length() - 1)
    c = cases.make_case(N, 868, seed=N + cfg[0], edge_frac=0.02)
    want = oracle.negacyclic(N, c.q_limbs, c.a, c.b)
    with nc.Plan(N, c.q_limbs, word_bits=64) as plan:
        plan.row_config = cfg
        got = _both_engines(plan, c.a, c.b)
    assert np.array_equal(got[nc.RESIDUES_TC_I8], want)
    assert np.array_equal(got[nc.RESIDUES_IMAD], want)


def test_all_q_minus_one_residues(gpu):
    """Every byte of every operand at its largest: the widest partial sums (< 2^23 each)."""
    N, bits = 2048, 961  # L = 31, k = 32: two MMA passes of 16 primes, odd limb count
    q = cases.gen_prime(bits, 79)
    L = (bits + 31) // 32
    ones = np.tile(cases.limbs_of(q - 1, L), (N, 1))
    with nc.Plan(N, cases.limbs_of(q, L)) as plan:
        assert plan.k == 32
        got = plan.multiply(ones, ones)
    assert np.array_equal(got, oracle.negacyclic(N, cases.limbs_of(q, L), ones, ones))


def test_device_path_and_chain(gpu):
    import torch

    N, bits = 16384, 434
    c = cases.make_case(N, bits, seed=81, edge_frac=0.02)
    d = cases.coeffs(c.q, N, c.L, 82)
    e = cases.coeffs(c.q, N, c.L, 83)
    with nc.Plan(N, c.q_limbs) as plan, nc.Plan(N, c.q_limbs, factors=4) as chain:
        assert chain.k <= 32 and chain.residue_engine == nc.RESIDUES_TC_I8
        dev = [torch.from_numpy(x.view(np.int32).copy()).cuda() for x in (c.a, c.b, d, e)]
        out = torch.empty_like(dev[0])
        plan.multiply_device(dev[0].data_ptr(), dev[1].data_ptr(), out.data_ptr(), 0)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint32).reshape(N, -1),
                              oracle.negacyclic(N, c.q_limbs, c.a, c.b))
        chain.multiply_chain_device([t.data_ptr() for t in dev], out.data_ptr(), 0)
        torch.cuda.synchronize()
        want = c.a
        for x in (c.b, d, e):
            want = oracle.negacyclic(N, c.q_limbs, want, x)
        assert np.array_equal(out.cpu().numpy().view(np.uint32).reshape(N, -1), want)


@pytest.mark.parametrize("N,bits,m", [(256, 1024, 2), (4096, 1000, 2), (16384, 868, 3), (1024, 731, 4)])
def test_beyond_32_primes(gpu, N, bits, m):
    """33 to 48 primes (three MMA passes): wide q and chained products."""
    c = cases.make_case(N, bits, seed=85 + N + bits, edge_frac=0.02)
    xs = [c.a, c.b] + [cases.coeffs(c.q, N, c.L, 86 + f) for f in range(m - 2)]
    want = xs[0]
    for x in xs[1:]:
        want = oracle.negacyclic(N, c.q_limbs, want, x)
    with nc.Plan(N, c.q_limbs, factors=m) as plan:
        assert plan.k > 32 and plan.residue_engine == nc.RESIDUES_TC_I8
        for engine in (nc.RESIDUES_TC_I8, nc.RESIDUES_IMAD):
            plan.residue_engine = engine
            got = plan.multiply_chain(xs) if m > 2 else plan.multiply(xs[0], xs[1])
            assert np.array_equal(got, want), engine


def test_unknown_engine_rejected(gpu):
    c = cases.make_case(64, 434, seed=87)
    with nc.Plan(64, c.q_limbs) as plan:
        with pytest.raises(nc.NegacyclicError) as ei:
            plan.residue_engine = 7
        assert ei.value.code == nc.NC_EINVAL
