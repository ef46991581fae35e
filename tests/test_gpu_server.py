"""The serving loop: continuous batching under an HBM budget, cached NTT-domain operands."""
from __future__ import annotations

import random
import threading
import time

import numpy as np
import pytest

import cases
import negacyclic as nc
import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mix():
    """Plans and operands of an uneven (N, width) mix; two reusable operands per plan."""
    rng = random.Random(11)
    plans = []
    for i, (log_n, bits) in enumerate([(10, 868), (12, 434), (14, 868), (13, 1000), (11, 100)]):
        N = 1 << log_n
        q = cases.gen_prime(bits, 3000 + i)
        L = (bits + 31) // 32
        plans.append((nc.Plan(N, cases.limbs_of(q, L)), q, L, [cases.coeffs(q, N, L, 3100 + 10 * i + j) for j in range(2)]))
    yield plans, rng
    for p, *_ in plans:
        p.close()


def test_poisson_mix_with_cached_operands(gpu, mix):
    plans, rng = mix
    with nc.Server(hbm_budget=1 << 30, staging=1 << 27, max_batch=16, streams=2) as srv:
        ops = {}
        for pi, (p, q, L, reused) in enumerate(plans):
            for j, a in enumerate(reused):
                ops[(pi, j)] = srv.register_operand(p, a)
        jobs = []
        for r in range(60):
            pi = rng.randrange(len(plans))
            p, q, L, reused = plans[pi]
            b = cases.coeffs(q, p.N, L, 5000 + r)
            if rng.random() < 0.3:
                j = rng.randrange(2)
                jobs.append((pi, reused[j], b, ops[(pi, j)]))
            else:
                jobs.append((pi, cases.coeffs(q, p.N, L, 6000 + r), b, -1))
        results = [None] * len(jobs)

        def client(idx):
            for k in idx:
                time.sleep(rng.expovariate(2000.0))  # ~0.5 ms between arrivals per client
                pi, a, b, op = jobs[k]
                p = plans[pi][0]
                rid = srv.submit(p, None if op >= 0 else a, b, operand=op)
                results[k] = srv.wait(rid, p)

        threads = [threading.Thread(target=client, args=(list(range(t, len(jobs), 4)),)) for t in range(4)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        st = srv.stats()
    assert st["completed"] == len(jobs)
    assert st["batches"] >= 1 and st["p99_ms"] >= st["p50_ms"] > 0
    for (pi, a, b, op), (c, ms) in zip(jobs, results):
        p, q, L, _ = plans[pi]
        assert ms > 0
        assert np.array_equal(c, oracle.negacyclic(p.N, cases.limbs_of(q, L), a, b))


def test_same_result_alone_and_in_the_mix(gpu, mix):
    plans, _ = mix
    p, q, L, reused = plans[2]
    b = cases.coeffs(q, p.N, L, 7000)
    alone = p.multiply(reused[0], b)
    with nc.Server(hbm_budget=1 << 30, staging=1 << 27, max_batch=32, streams=3) as srv:
        rids = []
        for i, (pp, qq, LL, rr) in enumerate(plans * 3):
            rids.append((pp, srv.submit(pp, rr[1], cases.coeffs(qq, pp.N, LL, 7100 + i))))
        target = srv.submit(p, reused[0], b)
        more = [(pp, srv.submit(pp, rr[0], rr[1])) for pp, qq, LL, rr in plans]
        got, _ = srv.wait(target, p)
        for pp, rid in rids + more:
            srv.wait(rid, pp)
    assert np.array_equal(got, alone)


def test_admission_waits_for_budget(gpu, mix):
    """A budget that holds about two requests still completes many, never exceeding it."""
    plans, _ = mix
    p, q, L, reused = plans[2]  # N = 2^14, 868-bit: ~11 MB of device memory per request
    per = 3 * p.N * L * 4 + 2 * p.k * p.N * 8
    budget = 2 * per + (1 << 20)
    with nc.Server(hbm_budget=budget, staging=1 << 27, max_batch=8, streams=2) as srv:
        bs = [cases.coeffs(q, p.N, L, 8000 + i) for i in range(10)]
        rids = [srv.submit(p, reused[0], b) for b in bs]
        peak = 0
        while not all(srv.poll(r) for r in rids):
            peak = max(peak, srv.stats()["hbm_in_use"])
            time.sleep(0.0005)
        outs = [srv.wait(r, p)[0] for r in rids]
        assert srv.stats()["batches"] >= 5
    assert peak <= budget
    for b, c in zip(bs, outs):
        assert np.array_equal(c, oracle.negacyclic(p.N, cases.limbs_of(q, L), reused[0], b))


def test_oversized_request_is_rejected(gpu, mix):
    plans, _ = mix
    p, q, L, reused = plans[2]
    with nc.Server(hbm_budget=1 << 20, staging=1 << 27) as srv:
        with pytest.raises(nc.NegacyclicError) as ei:
            srv.submit(p, reused[0], reused[1])
        assert ei.value.code == nc.NC_ENOMEM


def test_high_rate_overlapping_batches(gpu, mix):
    """Eight clients at a high rate, three streams: batches overlap on the device; every result
    exact and no batch gives up a dependency wait."""
    plans, _ = mix
    want = {}
    for pi, (p, q, L, reused) in enumerate(plans):
        want[pi] = p.multiply(reused[0], reused[1])
    # every client submits all 40 requests before it waits, and a result holds its pinned staging
    # until wait(): the 320 requests (~622 MB of staging) must all fit at once
    with nc.Server(hbm_budget=4 << 30, staging=1 << 31, max_batch=32, streams=3) as srv:
        ops = {pi: srv.register_operand(p, reused[0]) for pi, (p, q, L, reused) in enumerate(plans)}
        errors = []

        def client(c):
            r = random.Random(c)
            rids = []
            for i in range(40):
                pi = r.randrange(len(plans))
                p, q, L, reused = plans[pi]
                cached = r.random() < 0.3
                rids.append((pi, srv.submit(p, None if cached else reused[0], reused[1], operand=ops[pi] if cached else -1)))
            for pi, rid in rids:
                c_, _ = srv.wait(rid, plans[pi][0])
                if not np.array_equal(c_, want[pi]):
                    errors.append((c, pi))

        threads = [threading.Thread(target=client, args=(c,)) for c in range(8)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        st = srv.stats()
    assert st["timeouts"] == 0
    assert not errors, errors[:5]
    assert st["completed"] == 320


def test_release_operand_races_submit(gpu, mix):
    """release_operand racing submits that name the operand: each release either is refused with
    NC_EBUSY (a request still uses the operand) or succeeds, after which submits naming it fail
    cleanly with NC_EINVAL; every request that was accepted returns the exact product."""
    plans, _ = mix
    p, q, L, reused = plans[0]  # N = 2^10: short requests, many interleavings
    want = p.multiply(reused[0], reused[1])
    for attempt in range(4):
        with nc.Server(hbm_budget=1 << 28, staging=1 << 26, max_batch=8, streams=2) as srv:
            op = srv.register_operand(p, reused[0])
            accepted, refused, released = [], [], []

            def submitter():
                for _ in range(20):  # 60 requests in all: their staging fits at once
                    try:
                        accepted.append(srv.submit(p, None, reused[1], operand=op))
                    except nc.NegacyclicError as e:
                        refused.append(e.code)
                        return

            def releaser():
                time.sleep(0.0005 * (attempt + 1))
                while True:
                    try:
                        srv.release_operand(op)
                        released.append(True)
                        return
                    except nc.NegacyclicError as e:
                        if e.code != nc.NC_EBUSY:
                            released.append(e.code)
                            return
                        time.sleep(0.0001)

            subs = [threading.Thread(target=submitter) for _ in range(3)]
            rel = threading.Thread(target=releaser)
            for t in subs + [rel]:
                t.start()
            for t in subs + [rel]:
                t.join(timeout=60)
            assert released == [True]
            assert all(code == nc.NC_EINVAL for code in refused), refused
            for rid in accepted:
                c, _ = srv.wait(rid, p)
                assert np.array_equal(c, want)
