"""The 30-bit word engine (u32 residues modulo primes below 2^30) against the oracle, bit for bit:
every ring degree, modulus widths up to the engine's bound, every compiled row configuration,
the host path (grouped upload of b, a in the NTT domain), extreme operands, and the fallback to
the 62-bit engine where the 30-bit one cannot run."""
from __future__ import annotations

import numpy as np
import pytest

import cases
import negacyclic as nc
import oracle

pytestmark = pytest.mark.gpu


def _dev(arr, dev):
    import torch

    return torch.from_numpy(np.ascontiguousarray(arr).view(np.int32)).to(dev)


def _host(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("N,bits", [(2, 100), (8, 127), (64, 300), (256, 868), (1024, 868), (4096, 500),
                                    (8192, 868), (16384, 868), (32768, 868), (65536, 868), (65536, 948),
                                    (2048, 950), (2, 955)])
def test_w32_matches_oracle(gpu, N, bits):
    c = cases.make_case(N, bits, seed=3 * N + bits, edge_frac=0.02)
    want = oracle.negacyclic(N, c.q_limbs, c.a, c.b)
    with nc.Plan(N, c.q_limbs, W=c.W, word_bits=32) as plan:
        assert plan.word_bits == 32
        assert 1 <= plan.plain_primes <= 64
        assert np.array_equal(plan.multiply(c.a, c.b), want)
        plan.word_bits = 64
        assert plan.word_bits == 64 and plan.plain_primes == plan.k
        assert np.array_equal(plan.multiply(c.a, c.b), want)


@pytest.mark.parametrize("log_n", [1, 6, 10, 12, 13, 14, 16])
def test_every_w32_row_variant(gpu, log_n):
    N = 1 << log_n
    c = cases.make_case(N, 868, seed=900 + log_n, edge_frac=0.01)
    want = oracle.negacyclic(N, c.q_limbs, c.a, c.b)
    variants = nc.row_variants(log_n, word_bits=32)
    assert variants
    with nc.Plan(N, c.q_limbs, word_bits=32) as plan:
        for cfg in variants:
            plan.row_config = cfg
            assert plan.row_config == cfg
            assert np.array_equal(plan.multiply(c.a, c.b), want), f"row config {cfg} differs"


def test_w32_device_path_and_repeats(gpu):
    """Device-resident products (no grouped upload), twice on the same buffers."""
    import torch

    c = cases.make_case(65536, 868, seed=4242, edge_frac=0.01)
    want = oracle.negacyclic(c.N, c.q_limbs, c.a, c.b)
    with nc.Plan(c.N, c.q_limbs, word_bits=32) as plan:
        da, db = _dev(c.a, gpu), _dev(c.b, gpu)
        dc = torch.empty_like(da)
        for _ in range(2):
            dc.fill_(-1)
            plan.multiply_device(da.data_ptr(), db.data_ptr(), dc.data_ptr())
            torch.cuda.synchronize()
            assert np.array_equal(_host(dc).reshape(c.N, c.L), want)


def test_w32_extreme_operands(gpu):
    """All coefficients q - 1 (the widest residue sums and the largest CRT values), zeros and ones."""
    for N, bits in [(4096, 868), (65536, 868), (1024, 940)]:
        q = cases.gen_prime(bits, 11)
        L = (bits + 31) // 32
        ql = cases.limbs_of(q, L)
        top = np.tile(cases.limbs_of(q - 1, L), (N, 1))
        zero = np.zeros((N, L), dtype=np.uint32)
        one = zero.copy()
        one[0, 0] = 1
        with nc.Plan(N, ql, word_bits=32) as plan:
            assert np.array_equal(plan.multiply(top, top), oracle.negacyclic(N, ql, top, top))
            assert np.array_equal(plan.multiply(top, zero), zero)
            assert np.array_equal(plan.multiply(top, one), top)


def test_w32_unavailable_falls_back(gpu):
    """A bound beyond 64 primes below 2^30 (q of 1000 bits at N = 65536) keeps the 62-bit engine."""
    c = cases.make_case(65536, 1000, seed=5, edge_frac=0.0)
    with nc.Plan(c.N, c.q_limbs) as plan:
        assert plan.word_bits == 64
        with pytest.raises(nc.NegacyclicError):
            plan.word_bits = 32
        assert np.array_equal(plan.multiply(c.a, c.b), oracle.negacyclic(c.N, c.q_limbs, c.a, c.b))


def test_w32_needs_both_tensor_core_stages(gpu):
    """Selecting an integer-pipe stage runs the 62-bit engine; selecting both tensor-core stages again
    brings the 30-bit engine back."""
    c = cases.make_case(16384, 868, seed=6, edge_frac=0.01)
    want = oracle.negacyclic(c.N, c.q_limbs, c.a, c.b)
    with nc.Plan(c.N, c.q_limbs, word_bits=32) as plan:
        plan.residue_engine = nc.RESIDUES_IMAD
        assert plan.word_bits == 64
        assert np.array_equal(plan.multiply(c.a, c.b), want)
        plan.residue_engine = nc.RESIDUES_TC_I8
        assert plan.word_bits == 32
        assert np.array_equal(plan.multiply(c.a, c.b), want)


def test_w32_autotune_keeps_results_exact(gpu):
    c = cases.make_case(65536, 868, seed=78, edge_frac=0.01)
    with nc.Plan(c.N, c.q_limbs) as plan:
        assert plan.autotune(reps=2) > 0
        assert plan.row_config in nc.row_variants(16, word_bits=plan.word_bits)
        assert np.array_equal(plan.multiply(c.a, c.b), oracle.negacyclic(c.N, c.q_limbs, c.a, c.b))


def test_w32_batches_mix_engines_and_modes(gpu):
    """One batch holding plain products of 30-bit plans (their own residue, row and CRT launches),
    the same products on 62-bit plans, a cached-a product of a 30-bit plan (its NTT-domain operand
    in 30-bit residues, from a forward batch) and a product of N = 2^16 (plain launches), replayed
    from its graph twice."""
    import torch

    specs = [(1024, 868), (4096, 500), (16384, 868), (2048, 950), (65536, 868), (64, 300)]
    with nc.Batch() as fwd, nc.Batch() as batch:
        plans, checks = [], []
        for j, (N, bits) in enumerate(specs):
            c = cases.make_case(N, bits, seed=1300 + j, edge_frac=0.02)
            want = oracle.negacyclic(N, c.q_limbs, c.a, c.b)
            for bits_word in (32, 64):
                p = nc.Plan(N, c.q_limbs, word_bits=bits_word)
                plans.append(p)
                da, db = _dev(c.a, gpu), _dev(c.b, gpu)
                dc = da.new_zeros(da.shape)
                batch.add(p, da.data_ptr(), db.data_ptr(), dc.data_ptr())
                checks.append((dc, want, (N, bits, bits_word), (da, db)))
            if N == 16384:
                p = plans[-2]  # the 30-bit plan: hat_words covers its 30-bit NTT-domain form
                ahat = torch.empty(p.hat_words, dtype=torch.int64, device=gpu)
                da_f = _dev(c.a, gpu)
                fwd.add_forward(p, da_f.data_ptr(), ahat.data_ptr())
                fwd.run(0, True)
                fwd.synchronize()
                db = _dev(c.b, gpu)
                dc = db.new_zeros(db.shape)
                batch.add_cached(p, ahat.data_ptr(), db.data_ptr(), dc.data_ptr())
                checks.append((dc, want, (N, bits, "cached"), (ahat, db, da_f)))
        for _ in range(2):
            for dc, _, _, _ in checks:
                dc.fill_(-1)
            batch.run(0, True)
            batch.synchronize()
            for dc, want, what, _ in checks:
                assert np.array_equal(_host(dc).reshape(want.shape), want), what
        for p in plans:
            p.close()
