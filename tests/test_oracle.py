"""Pins the CPU oracle: the reference's own known-answer self-checks (solve.cu fherma_init),
its prime rule, and whole products against independent big-integer schoolbooks."""
from __future__ import annotations

import random

import numpy as np
import pytest

import cases
import oracle

M64 = (1 << 64) - 1


@pytest.fixture(scope="module")
def L():
    return oracle.lib()


@pytest.fixture(scope="module")
def q868():
    return cases.gen_prime(868, seed=2024)


# ------------------------------------------------------------------ reference self-checks


def test_kat_mul_mod(L):
    # solve.cu:1151
    assert L.oracle_mul_mod(7, 5, 11) == 2


def test_kat_montgomery(L):
    # solve.cu:1152-1159: 7*5 mod 11 through Montgomery form, R = 2^64
    p = 11
    npr = L.oracle_neg_inv64(p)
    assert (npr * p) & M64 == M64  # -p^-1 * p = -1 mod 2^64
    lift = L.oracle_pow_mod(2, 128, p)
    left = L.oracle_mont_mul(7, lift, p, npr)
    right = L.oracle_mont_mul(5, lift, p, npr)
    assert L.oracle_mont_mul(L.oracle_mont_mul(left, right, p, npr), 1, p, npr) == 2


def test_kat_barrett(L):
    # solve.cu:1160-1161; barrett_mu keeps the low 64 bits of floor(2^96 / p) (solve.cu:239-251)
    mu = L.oracle_barrett_mu96(11)
    assert mu == ((1 << 96) // 11) & M64
    assert L.oracle_barrett_reduce(0, 100, 11, mu) == 1


def test_kat_reciprocal(L):
    # solve.cu:1162-1165: floor(2^64 / 3) = 6148914691236517205, remainder 1
    import ctypes

    rem = ctypes.c_uint64()
    assert L.oracle_div_pow2_64(3, ctypes.byref(rem)) == 6148914691236517205
    assert rem.value == 1


def test_kat_shoup_vs_montgomery(L, q868):
    # solve.cu:1285-1314 on the first prime of the point
    p = oracle.reference_primes(1024, q868.bit_length())[0]
    npr = L.oracle_neg_inv64(p)
    lift = L.oracle_pow_mod(2, 128, p)
    for trial in range(32):
        left = ((trial * 0x9E3779B97F4A7C15) & M64) % p
        right = (((trial + 3) * 0xBF58476D1CE4E5B9) & M64) % p or 1
        sh = L.oracle_shoup_companion(right, p)
        assert sh == (right << 64) // p
        left_m = L.oracle_mont_mul(left, lift, p, npr)
        right_m = L.oracle_mont_mul(right, lift, p, npr)
        assert L.oracle_shoup_mul(left_m, right, sh, p) == L.oracle_mont_mul(left_m, right_m, p, npr)


def test_kat_wide_reduction(L, q868):
    # solve.cu:1370-1376: 128-bit remainders on 24 values; 1359-1368: floor(2^128 / p)
    import ctypes

    p = oracle.reference_primes(1024, q868.bit_length())[0]
    hi, lo = ctypes.c_uint64(), ctypes.c_uint64()
    L.oracle_magic128(p, ctypes.byref(hi), ctypes.byref(lo))
    assert (hi.value << 64 | lo.value) == (1 << 128) // p
    for trial in range(24):
        h = (trial << 36) & M64
        l_ = (trial * 0x9E3779B97F4A7C15) & M64
        assert L.oracle_mod128(h, l_, p) == ((h << 64) | l_) % p


def test_kat_digit_sum(L, q868):
    # solve.cu:1377-1394: sum_l sample_l * (2^(32 l) mod p) vs the residue of the 28-limb sample
    p = oracle.reference_primes(1024, q868.bit_length())[0]
    sample = np.array([(0xFFFFFFFF - 17 * l) & 0xFFFFFFFF for l in range(32)], dtype=np.uint32)
    value = cases.int_of(sample[:28])
    digit = sum(int(sample[l]) * pow(2, 32 * l, p) for l in range(28)) % p
    assert digit == value % p
    assert L.oracle_limbs_mod_u64(sample.ctypes.data_as(oracle._u32p), 28, p) == value % p


def test_kat_mod_q(L, q868):
    # solve.cu:1396-1415: a 34-limb value reduced mod the 868-bit q
    ql = cases.limbs_of(q868, 28)
    slow = np.array([((int(ql[l]) if l < 28 else 0) + l * 97 + 11) & 0xFFFFFFFF for l in range(34)], dtype=np.uint32)
    slow[30] = 0x3FFFF
    value = cases.int_of(slow)
    L.oracle_mod_q(slow.ctypes.data_as(oracle._u32p), 34, ql.ctypes.data_as(oracle._u32p), 28)
    assert cases.int_of(slow) == value % q868


# ------------------------------------------------------------------ prime rule


def _py_reference_primes(N: int, q_bits: int) -> list[int]:
    # restated independently: solve.cu:1174-1204
    log_n = N.bit_length() - 1
    bound = log_n + 2 * q_bits + 4
    step = 2 * N
    cand = (1 << 62) - 1
    cand -= (cand - 1) % step
    prod, out = 1, []
    rng = random.Random(7)
    while cand > step and prod.bit_length() < bound:
        if cases.is_probable_prime(cand, 20, rng):
            out.append(cand)
            prod *= cand
        cand -= step
    return out


@pytest.mark.parametrize("N", [2, 1024, 16384, 65536])
@pytest.mark.parametrize("bits", [434, 868])
def test_reference_prime_rule(N, bits):
    got = oracle.reference_primes(N, bits)
    assert got == _py_reference_primes(N, bits)
    assert len(got) == (29 if bits == 868 else 15)
    for p in got:
        assert p % (2 * N) == 1 and p < (1 << 62)


def test_find_psi(L):
    for N in (2, 64, 4096):
        for p in oracle.reference_primes(N, 100)[:3]:
            psi = L.oracle_find_psi(p, N)
            assert pow(psi, N, p) == p - 1


# ------------------------------------------------------------------ whole products


@pytest.mark.parametrize("N,bits", [(2, 868), (4, 64), (8, 434), (16, 868), (32, 33), (64, 868), (128, 100)])
def test_oracle_vs_python_schoolbook(N, bits):
    c = cases.make_case(N, bits, seed=N * 1000 + bits)
    got = oracle.negacyclic(N, c.q_limbs, c.a, c.b)
    want = oracle.schoolbook_py(cases.ints_of_rows(c.a), cases.ints_of_rows(c.b), c.q)
    assert cases.ints_of_rows(got) == want


def test_oracle_vs_c_schoolbook_1024():
    c = cases.make_case(1024, 868, seed=11, edge_frac=0.01)
    got = oracle.negacyclic(1024, c.q_limbs, c.a, c.b)
    want = oracle.schoolbook_c(1024, c.q_limbs, c.a, c.b)
    assert np.array_equal(got, want)


def test_c_schoolbook_vs_python():
    c = cases.make_case(32, 868, seed=5)
    want = oracle.schoolbook_py(cases.ints_of_rows(c.a), cases.ints_of_rows(c.b), c.q)
    assert cases.ints_of_rows(oracle.schoolbook_c(32, c.q_limbs, c.a, c.b)) == want


def test_oracle_edge_operands():
    N, bits = 256, 868
    q = cases.gen_prime(bits, 99)
    Lq = (bits + 31) // 32
    ql = cases.limbs_of(q, Lq)
    top = cases.rows_of_ints([q - 1] * N, Lq)
    zero = np.zeros((N, Lq), dtype=np.uint32)
    one = cases.rows_of_ints([1] + [0] * (N - 1), Lq)
    # most negative case: every coefficient q - 1
    got = oracle.negacyclic(N, ql, top, top)
    want = oracle.schoolbook_py([q - 1] * N, [q - 1] * N, q)
    assert cases.ints_of_rows(got) == want
    assert not oracle.negacyclic(N, ql, zero, top).any()
    assert np.array_equal(oracle.negacyclic(N, ql, one, top), top)


def test_oracle_spot_checks_large():
    N = 16384
    c = cases.make_case(N, 868, seed=3, edge_frac=0.01)
    got = oracle.negacyclic(N, c.q_limbs, c.a, c.b)
    a, b = cases.ints_of_rows(c.a), cases.ints_of_rows(c.b)
    for k in (0, 1, N // 2, N - 1):
        assert cases.int_of(got[k]) == oracle.coefficient_py(a, b, c.q, k)
