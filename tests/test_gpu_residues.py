"""Residue-stage ablation: the integer-pipe engine and the INT8 tensor-core engine both give
x_n mod p_i exactly, for every coefficient and prime, on the same inputs."""
from __future__ import annotations

import numpy as np
import pytest

import cases
import negacyclic as nc

pytestmark = pytest.mark.gpu


def expected_residues(x: np.ndarray, ps: list[int]) -> np.ndarray:
    """x: N x L u32 limbs; returns k x N residues by Python integers."""
    vals = cases.ints_of_rows(x)
    return np.array([[v % p for v in vals] for p in ps], dtype=np.uint64)


def run_engine(plan, x: np.ndarray, engine: int) -> np.ndarray:
    import torch

    dx = torch.from_numpy(x.view(np.int32).copy()).cuda()
    dr = torch.full((plan.k * plan.N,), -1, dtype=torch.int64, device="cuda")
    plan.residues(dx.data_ptr(), dr.data_ptr(), engine)
    torch.cuda.synchronize()
    assert not nc.residues_gave_up()
    return dr.cpu().numpy().view(np.uint64).reshape(plan.k, plan.N)


@pytest.mark.parametrize("N,bits", [(1024, 868), (512, 434), (64, 868), (256, 1000), (128, 100)])
@pytest.mark.parametrize("engine", [nc.RESIDUES_IMAD, nc.RESIDUES_TC_I8])
def test_engine_vs_integers(gpu, N, bits, engine):
    c = cases.make_case(N, bits, seed=3 * N + bits, edge_frac=0.05)
    with nc.Plan(N, c.q_limbs, W=c.W) as plan:
        if engine == nc.RESIDUES_TC_I8 and plan.k > 32:
            pytest.skip("the tensor-core engine takes at most 32 primes")
        got = run_engine(plan, c.a, engine)
        want = expected_residues(c.a, nc.primes(plan.k))
    bad = np.argwhere(got != want)
    assert bad.size == 0, f"{len(bad)} residues differ, first (prime, n) {bad[:4].tolist()}"


def test_engines_agree_on_extreme_limbs(gpu):
    """All-ones limbs maximise every byte product and partial sum of the contraction."""
    q = cases.gen_prime(868, 91)
    L = 28
    N = 4096
    x = cases.coeffs(q, N, L, 92)
    x[::3] = 0xFFFFFFFF  # values above q are fine for a residue
    x[1::7] = 0
    with nc.Plan(N, cases.limbs_of(q, L)) as plan:
        a = run_engine(plan, x, nc.RESIDUES_IMAD)
        b = run_engine(plan, x, nc.RESIDUES_TC_I8)
        spot = expected_residues(x[:256], nc.primes(plan.k))
    assert np.array_equal(a, b)
    assert np.array_equal(a[:, :256], spot)


def test_engines_agree_at_full_size(gpu):
    q = cases.gen_prime(868, 93)
    L = 28
    N = 65536
    x = cases.coeffs(q, N, L, 94, edge_frac=0.01)
    with nc.Plan(N, cases.limbs_of(q, L)) as plan:
        a = run_engine(plan, x, nc.RESIDUES_IMAD)
        b = run_engine(plan, x, nc.RESIDUES_TC_I8)
        rows = np.arange(0, N, 509)
        spot = expected_residues(x[rows], nc.primes(plan.k))
    assert np.array_equal(a, b)
    assert np.array_equal(a[:, rows], spot)


def test_tensor_engine_rejects_too_many_primes(gpu):
    q = cases.gen_prime(1024, 95)
    with nc.Plan(256, cases.limbs_of(q, 32)) as plan:
        assert plan.k > 32
        import torch

        dx = torch.zeros(256 * 32, dtype=torch.int32, device="cuda")
        dr = torch.zeros(plan.k * 256, dtype=torch.int64, device="cuda")
        with pytest.raises(nc.NegacyclicError) as ei:
            plan.residues(dx.data_ptr(), dr.data_ptr(), nc.RESIDUES_TC_I8)
        assert ei.value.code == nc.NC_EINVAL
