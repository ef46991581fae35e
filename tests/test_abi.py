"""The C ABI library loads, exports every declared symbol and the reference's C++ contract, and
rejects invalid points before touching a GPU. No compute calls here."""
from __future__ import annotations

import re
import subprocess

import pytest

import negacyclic as nc
from conftest import ROOT, has_gpu

HEADER = ROOT / "include" / "negacyclic_b200.h"


def declared_symbols() -> set[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(nc_[a-z0-9_]+)\s*\(", text))


def test_library_loads():
    lib = nc.load()
    assert lib.nc_version() >= 100


def test_every_declared_symbol_is_exported_and_bound():
    lib = nc.load()
    decl = declared_symbols()
    assert decl, "no declarations parsed"
    bound = {name for name, _, _ in nc.C_SYMBOLS}
    assert decl == bound, f"header vs binding mismatch: {decl ^ bound}"
    for name in decl:
        assert hasattr(lib, name), name


def test_reference_contract_symbols_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", "-C", str(nc.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    assert "fherma_init(fherma::Point const&)" in out
    assert "fherma_run(void*, fherma::Inputs const&)" in out
    assert "fherma_free(void*)" in out


@pytest.mark.parametrize("N,L,q,msg", [
    (3, 1, [0xFFFFFFFB], "power of two"),
    (0, 1, [0xFFFFFFFB], "power of two"),
    (1 << 17, 1, [0xFFFFFFFB], "power of two"),
    (8, 0, [], "L must"),
    (8, 33, [1] * 33, "L must"),
    (8, 1, [10], "odd"),
    (8, 2, [7, 0], "top limb"),
])
def test_invalid_points_rejected(N, L, q, msg):
    import numpy as np

    arr = np.array(q if q else [0], dtype=np.uint32)
    lib = nc.load()
    import ctypes

    h = ctypes.c_void_p()
    st = lib.nc_plan_create(N, 0, L, arr.ctypes.data_as(nc._u32p), ctypes.byref(h))
    assert st == nc.NC_EINVAL
    assert msg in lib.nc_last_error().decode()
    assert not h.value


def test_width_must_match_limbs():
    import numpy as np

    q = np.array([0xFFFFFFFB, 1], dtype=np.uint32)
    with pytest.raises(nc.NegacyclicError, match="W must"):
        nc.Plan(8, q, W=100)


def test_null_arguments():
    lib = nc.load()
    assert lib.nc_plan_create(8, 0, 1, None, None) == nc.NC_EINVAL
    assert lib.nc_multiply(None, None, None, None) == nc.NC_EINVAL
    assert lib.nc_plan_destroy(None) == nc.NC_OK


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU failure mode")
def test_valid_point_without_gpu_fails_loudly():
    import numpy as np

    q = np.array([0xFFFFFFFB], dtype=np.uint32)  # 2^32 - 5, prime
    with pytest.raises(nc.NegacyclicError) as ei:
        nc.Plan(8, q)
    assert ei.value.code in (nc.NC_ECUDA, nc.NC_ENOMEM)


def test_prime_set():
    import random

    import cases

    ps = nc.primes(48)
    assert len(ps) == 48 and ps == sorted(ps, reverse=True)
    rng = random.Random(1)
    for p in ps:
        assert p < (1 << 62) and p % (1 << 17) == 1
        assert (1 << 62) - p < (1 << 28)
        assert cases.is_probable_prime(p, 16, rng)


def test_row_variants_listed_without_gpu():
    for log_n in range(1, 17):
        v = nc.row_variants(log_n)
        assert v, log_n
        for blk, radix, threads in v:
            assert 1 <= blk <= min(log_n, 13) and log_n - blk <= 5
            assert radix in (3, 4) and threads in (256, 512)
    assert (12, 4, 256) in nc.row_variants(16)
    assert nc.load().nc_row_variants(17, None, 0) == nc.NC_EINVAL


def test_batch_entry_points_reject_nulls():
    lib = nc.load()
    assert lib.nc_batch_add(None, None, None, None, None) == nc.NC_EINVAL
    assert lib.nc_batch_run(None, None, 1) == nc.NC_EINVAL
    assert lib.nc_batch_destroy(None) == nc.NC_OK
    assert lib.nc_plan_hat_words(None) == 0


@pytest.mark.parametrize("factors,bits,msg", [(1, 64, "factors must"), (5, 64, "factors must"),
                                              (4, 868, "48-prime"), (4, 732, "48-prime")])
def test_chain_plans_rejected_before_any_device_work(factors, bits, msg):
    """A chain plan whose operand count is outside 2..4, or whose coefficient bound
    (m - 1) log2 N + m bits(q) + 4 exceeds the 48 primes (m = 4 at N = 65536 allows 731 bits)."""
    import ctypes

    import cases

    L = (bits + 31) // 32
    q = cases.limbs_of(cases.gen_prime(bits, 95), L)
    h = ctypes.c_void_p()
    st = nc.load().nc_plan_create_chain(65536, 0, L, nc._u32(q), factors, ctypes.byref(h))
    assert st == nc.NC_EINVAL
    assert msg in nc.load().nc_last_error().decode()
    assert not h.value


def test_chain_entry_points_reject_nulls():
    lib = nc.load()
    assert lib.nc_plan_create_chain(8, 0, 1, None, 3, None) == nc.NC_EINVAL
    assert lib.nc_multiply_chain(None, None, None) == nc.NC_EINVAL
    assert lib.nc_multiply_chain_device(None, None, None, None) == nc.NC_EINVAL
    assert lib.nc_plan_factors(None) == nc.NC_EINVAL
