"""The allocation-free entry point, through the C ABI.

nc_multiply_device_noalloc serves callers that must not allocate device memory when they call
the library (memory owned by another framework's pool, latency-critical loops, services that
allocate only at start-up). Its residue scratch is a fixed array inside the library instead of
the plan's own, so its results must equal nc_multiply_device's bit for bit, call after call.
This file is collected last on purpose.
"""
from __future__ import annotations

import numpy as np
import pytest

import cases
import negacyclic as nc

pytestmark = pytest.mark.gpu


def _dev(arr, dev):
    import torch

    return torch.from_numpy(np.ascontiguousarray(arr).view(np.int32)).to(dev)


@pytest.mark.parametrize("N,bits", [(4096, 868), (16384, 868), (32768, 434)])
def test_noalloc_matches_plan_scratch_on_two_calls(gpu, N, bits):
    import torch

    q = cases.gen_prime(bits, 4000 + N)
    L = (bits + 31) // 32
    ql = cases.limbs_of(q, L)
    with nc.Plan(N, ql) as plan:
        for call in range(2):  # two calls in a row, different operands each time
            a = cases.coeffs(q, N, L, 4100 + 10 * call + N)
            b = cases.coeffs(q, N, L, 4101 + 10 * call + N)
            da, db = _dev(a, gpu), _dev(b, gpu)
            want, got = torch.zeros_like(da), torch.full_like(da, -1)
            plan.multiply_device(da.data_ptr(), db.data_ptr(), want.data_ptr(), 0)
            plan.multiply_device_noalloc(da.data_ptr(), db.data_ptr(), got.data_ptr(), 0)
            torch.cuda.synchronize()
            assert torch.equal(got, want), f"call {call}: allocation-free product differs"


def test_noalloc_calls_leave_device_memory_unchanged(gpu):
    """No call allocates device memory, the first one on a fresh plan included: the fixed array
    is placed on the device when the first plan there is created, not when the entry point runs."""
    import torch

    N, bits = 8192, 868
    q = cases.gen_prime(bits, 4300)
    L = (bits + 31) // 32
    with nc.Plan(N, cases.limbs_of(q, L)) as plan:
        a = _dev(cases.coeffs(q, N, L, 4301), gpu)
        b = _dev(cases.coeffs(q, N, L, 4302), gpu)
        want, got = torch.zeros_like(a), torch.full_like(a, -1)
        # the plan-scratch path first: it loads the product kernels and allocates its own scratch
        plan.multiply_device(a.data_ptr(), b.data_ptr(), want.data_ptr(), 0)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        for _ in range(2):
            plan.multiply_device_noalloc(a.data_ptr(), b.data_ptr(), got.data_ptr(), 0)
            torch.cuda.synchronize()
            assert torch.cuda.mem_get_info()[0] == free_before, "an allocation-free call changed free device memory"
        assert torch.equal(got, want)


def test_noalloc_rejects_products_beyond_the_static_scratch(gpu):
    import torch

    q = cases.gen_prime(868, 4200)
    with nc.Plan(65536, cases.limbs_of(q, 28)) as plan:  # k * N = 29 * 65536 > 2^19
        buf = torch.zeros(65536 * 28, dtype=torch.int32, device=gpu)
        with pytest.raises(nc.NegacyclicError, match="static scratch limit") as ei:
            plan.multiply_device_noalloc(buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 0)
        assert ei.value.code == nc.NC_EINVAL
