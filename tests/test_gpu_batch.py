"""Row-stage variants and the persistent batched kernel, bit for bit against the oracle."""
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


@pytest.mark.parametrize("log_n", [6, 10, 12, 13, 14, 16])
def test_every_row_variant(gpu, log_n):
    N = 1 << log_n
    c = cases.make_case(N, 868, seed=500 + log_n, edge_frac=0.01)
    want = oracle.negacyclic(N, c.q_limbs, c.a, c.b)
    variants = nc.row_variants(log_n)
    assert variants
    with nc.Plan(N, c.q_limbs, word_bits=64) as plan:
        for cfg in variants:
            plan.row_config = cfg
            assert plan.row_config == cfg
            got = plan.multiply(c.a, c.b)
            assert np.array_equal(got, want), f"row config {cfg} differs"


def test_autotune_keeps_results_exact(gpu):
    c = cases.make_case(16384, 868, seed=77)
    with nc.Plan(c.N, c.q_limbs) as plan:
        ms = plan.autotune(reps=2)
        assert ms > 0
        assert plan.row_config in nc.row_variants(14, word_bits=plan.word_bits)
        assert np.array_equal(plan.multiply(c.a, c.b), oracle.negacyclic(c.N, c.q_limbs, c.a, c.b))
        # later plans of the same (N, L) start from the tuned choice
        with nc.Plan(c.N, c.q_limbs) as p2:
            assert p2.word_bits == plan.word_bits and p2.row_config == plan.row_config


def _run_batch(gpu, specs, use_graph=True, repeat=1):
    """specs: list of (N, bits, seed). Returns (cases, outputs)."""
    plans, cs, bufs = [], [], []
    with nc.Batch() as batch:
        for N, bits, seed in specs:
            c = cases.make_case(N, bits, seed, edge_frac=0.01)
            p = nc.Plan(N, c.q_limbs)
            da, db = _dev(c.a, gpu), _dev(c.b, gpu)
            dc = da.new_zeros(da.shape)
            batch.add(p, da.data_ptr(), db.data_ptr(), dc.data_ptr())
            plans.append(p)
            cs.append(c)
            bufs.append((da, db, dc))
        for _ in range(repeat):
            batch.run(0, use_graph)
            batch.synchronize()
        info = batch.query()
    outs = [_host(b[2]) for b in bufs]
    for p in plans:
        p.close()
    return cs, outs, info


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_uniform(gpu, use_graph):
    specs = [(16384, 868, 600 + i) for i in range(8)]
    cs, outs, info = _run_batch(gpu, specs, use_graph, repeat=2)
    assert info["products"] == 8 and info["ctas"] > 0
    for c, o in zip(cs, outs):
        assert np.array_equal(o, oracle.negacyclic(c.N, c.q_limbs, c.a, c.b))


def test_batch_uneven_mix(gpu):
    import random

    rng = random.Random(5)
    specs = [(1 << rng.randint(1, 16), rng.choice([434, 868, 100, 1000]), 700 + i) for i in range(24)]
    cs, outs, _ = _run_batch(gpu, specs, use_graph=True)
    for c, o in zip(cs, outs):
        assert np.array_equal(o, oracle.negacyclic(c.N, c.q_limbs, c.a, c.b)), (c.N, c.W)


def test_batch_same_result_alone_and_in_mix(gpu):
    spec = (4096, 868, 800)
    (c_alone,), (alone,), _ = _run_batch(gpu, [spec])
    mix = [(1024, 434, 801), spec, (65536, 868, 802), (256, 1000, 803)]
    cs, outs, _ = _run_batch(gpu, mix)
    assert np.array_equal(outs[1], alone)


def test_batch_forward_then_cached(gpu):
    """The NTT-domain form of a, computed once, multiplies several b's exactly."""
    N = 16384
    q = cases.gen_prime(868, 900)
    a = cases.coeffs(q, N, 28, 901)
    bs = [cases.coeffs(q, N, 28, 902 + i) for i in range(3)]
    ql = cases.limbs_of(q, 28)
    import torch

    with nc.Plan(N, ql) as plan, nc.Batch() as fwd, nc.Batch() as use:
        da = _dev(a, gpu)
        ahat = torch.empty(plan.hat_words, dtype=torch.int64, device=gpu)
        fwd.add_forward(plan, da.data_ptr(), ahat.data_ptr())
        fwd.run(0, True)
        fwd.synchronize()
        dbs = [_dev(b, gpu) for b in bs]
        dcs = [x.new_zeros(x.shape) for x in dbs]
        for db, dc in zip(dbs, dcs):
            use.add_cached(plan, ahat.data_ptr(), db.data_ptr(), dc.data_ptr())
        use.run(0, True)
        use.synchronize()
        for b, dc in zip(bs, dcs):
            assert np.array_equal(_host(dc), oracle.negacyclic(N, ql, a, b))


def test_batch_replay_with_new_operands(gpu):
    """A captured graph replays with the same shape and new device pointers."""
    N = 4096
    c1 = cases.make_case(N, 868, seed=950)
    c2 = cases.make_case(N, 868, seed=951, q=c1.q)
    with nc.Plan(N, c1.q_limbs) as plan, nc.Batch() as batch:
        outs = []
        for c in (c1, c2):
            da, db = _dev(c.a, gpu), _dev(c.b, gpu)
            dc = da.new_zeros(da.shape)
            batch.clear()
            batch.add(plan, da.data_ptr(), db.data_ptr(), dc.data_ptr())
            batch.run(0, True)
            batch.synchronize()
            outs.append(_host(dc))
        for c, o in zip((c1, c2), outs):
            assert np.array_equal(o, oracle.negacyclic(N, c.q_limbs, c.a, c.b))


def test_batch_mixes_residue_engines(gpu):
    """One batch with tensor-core residue items (one launch per column length N1: N from 2^6 to
    2^16), products on the integer residue stage (inside the persistent launch), a forward-mode
    item and a cached-a item: every product matches the oracle, in two graph replays."""
    import torch

    specs = [(64, 868, nc.RESIDUES_TC_I8), (8192, 434, nc.RESIDUES_TC_I8), (16384, 868, nc.RESIDUES_IMAD),
             (32768, 600, nc.RESIDUES_TC_I8), (65536, 868, nc.RESIDUES_TC_I8), (4096, 1000, nc.RESIDUES_IMAD),
             (2048, 1024, nc.RESIDUES_TC_I8)]
    plans, bufs, want = [], [], []
    try:
        with nc.Batch() as batch:
            for i, (N, bits, engine) in enumerate(specs):
                c = cases.make_case(N, bits, seed=950 + i, edge_frac=0.02)
                p = nc.Plan(N, c.q_limbs)
                p.residue_engine = engine
                plans.append(p)
                da, db = _dev(c.a, gpu), _dev(c.b, gpu)
                dc = da.new_zeros(da.shape)
                batch.add(p, da.data_ptr(), db.data_ptr(), dc.data_ptr())
                bufs.append((da, db, dc))
                want.append(oracle.negacyclic(N, c.q_limbs, c.a, c.b))
            # a cached-a product whose a_hat comes from a forward item of an earlier batch
            c = cases.make_case(16384, 868, seed=960, edge_frac=0.02)
            p = nc.Plan(16384, c.q_limbs)
            plans.append(p)
            da, db = _dev(c.a, gpu), _dev(c.b, gpu)
            ahat = torch.empty(p.hat_words, dtype=torch.int64, device=gpu)
            with nc.Batch() as fwd:
                fwd.add_forward(p, da.data_ptr(), ahat.data_ptr())
                fwd.run(0, True)
                fwd.synchronize()
            dc = da.new_zeros(da.shape)
            batch.add_cached(p, ahat.data_ptr(), db.data_ptr(), dc.data_ptr())
            bufs.append((da, db, dc))
            want.append(oracle.negacyclic(16384, c.q_limbs, c.a, c.b))
            for _ in range(2):
                for _, _, out in bufs:
                    out.zero_()
                batch.run(0, True)
                batch.synchronize()
                for (_, _, out), w in zip(bufs, want):
                    assert np.array_equal(_host(out), w)
    finally:
        for p in plans:
            p.close()
