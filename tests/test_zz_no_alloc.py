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


def test_noalloc_rejects_products_beyond_the_static_scratch(gpu):
    import torch

    q = cases.gen_prime(868, 4200)
    with nc.Plan(65536, cases.limbs_of(q, 28)) as plan:  # k * N = 29 * 65536 > 2^19
        buf = torch.zeros(65536 * 28, dtype=torch.int32, device=gpu)
        with pytest.raises(nc.NegacyclicError, match="static scratch limit") as ei:
            plan.multiply_device_noalloc(buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 0)
        assert ei.value.code == nc.NC_EINVAL
