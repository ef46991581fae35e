"""The CRT accumulation on the tensor cores (default for <= 32 primes) and on the integer pipes:
both give the oracle's product bit for bit, across ring degrees (partial and full tiles), q widths
and the widest table (L = 31, 32 primes: 144 byte columns)."""
from __future__ import annotations

import numpy as np
import pytest

import cases
import negacyclic as nc
import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,bits", [(2, 868), (64, 868), (128, 434), (256, 868), (1024, 100), (4096, 970),
                                    (16384, 868), (65536, 868), (65536, 434), (8192, 600)])
def test_both_engines_match_the_oracle(gpu, N, bits):
    c = cases.make_case(N, bits, seed=5 * N + bits, edge_frac=0.02)
    want = oracle.negacyclic(N, c.q_limbs, c.a, c.b)
    with nc.Plan(N, c.q_limbs, W=c.W) as plan:
        assert plan.k <= 32
        assert plan.crt_engine == nc.CRT_TC_I8
        tc = plan.multiply(c.a, c.b)
        plan.crt_engine = nc.CRT_IMAD
        imad = plan.multiply(c.a, c.b)
    assert np.array_equal(tc, want)
    assert np.array_equal(imad, want)


def test_all_q_minus_one_operands(gpu):
    """Every v_i near p_i and every byte of the table at its largest: the widest partial sums."""
    N, bits = 4096, 868
    q = cases.gen_prime(bits, 77)
    L = (bits + 31) // 32
    ones = np.tile(cases.limbs_of(q - 1, L), (N, 1))
    with nc.Plan(N, cases.limbs_of(q, L)) as plan:
        got = plan.multiply(ones, ones)
    assert np.array_equal(got, oracle.negacyclic(N, cases.limbs_of(q, L), ones, ones))


def test_tensor_engine_unavailable_beyond_32_primes(gpu):
    q = cases.gen_prime(1024, 78)
    with nc.Plan(256, cases.limbs_of(q, 32)) as plan:
        assert plan.k > 32
        assert plan.crt_engine == nc.CRT_IMAD
        with pytest.raises(nc.NegacyclicError) as ei:
            plan.crt_engine = nc.CRT_TC_I8
        assert ei.value.code == nc.NC_EINVAL


def test_batch_mixes_both_crt_engines(gpu):
    """One batch with tensor-core CRT items (868-bit), integer CRT items (1000-bit: 33 primes) and a
    plan switched to the integer engine: every product matches the oracle."""
    import torch

    specs = [(4096, 868, nc.CRT_TC_I8), (2048, 1000, None), (8192, 868, nc.CRT_IMAD), (1024, 434, nc.CRT_TC_I8)]
    plans, bufs, want = [], [], []
    try:
        for i, (N, bits, engine) in enumerate(specs):
            c = cases.make_case(N, bits, seed=600 + i, edge_frac=0.02)
            p = nc.Plan(N, c.q_limbs, W=c.W)
            if engine is not None:
                p.crt_engine = engine
            else:
                assert p.crt_engine == nc.CRT_IMAD
            plans.append(p)
            x = torch.from_numpy(c.a.view(np.int32).copy()).cuda()
            y = torch.from_numpy(c.b.view(np.int32).copy()).cuda()
            bufs.append((x, y, torch.empty_like(x)))
            want.append(oracle.negacyclic(N, c.q_limbs, c.a, c.b))
        with nc.Batch() as batch:
            for p, (x, y, z) in zip(plans, bufs):
                batch.add(p, x.data_ptr(), y.data_ptr(), z.data_ptr())
            for use_graph in (False, True, True):
                batch.run(0, use_graph)
                batch.synchronize()
                for (_, _, z), w in zip(bufs, want):
                    assert np.array_equal(z.cpu().numpy().view(np.uint32).reshape(w.shape), w)
    finally:
        for p in plans:
            p.close()
