"""Init-time self-checks (nc_self_check; nc_plan_create runs the same ones, plus a device
known-answer product). The reference's fherma_init checks its arithmetic before it returns a
state (solve.cu:1151-1165, 1285-1314, 1370-1415), but its L = 28 Barrett check rejects nearly
every 868-bit q; these must hold for every valid point, and reject invalid ones with a message."""
from __future__ import annotations

import numpy as np
import pytest

import cases
import negacyclic as nc


@pytest.mark.parametrize("bits", [20, 62, 100, 434, 600, 868, 960, 1000, 1024])
@pytest.mark.parametrize("log_n", [1, 4, 10, 14, 16])
def test_self_check_holds_for_valid_points(bits, log_n):
    q = cases.gen_prime(bits, 9000 + bits)
    L = (bits + 31) // 32
    nc.self_check(1 << log_n, cases.limbs_of(q, L), W=bits)


def test_self_check_holds_for_composite_odd_moduli():
    # the CRT and Barrett constants need q odd, not prime
    for q in (3 ** 500, (1 << 867) + 1, (1 << 1023) + (1 << 500) + 1):
        bits = q.bit_length()
        nc.self_check(65536, cases.limbs_of(q, (bits + 31) // 32))


@pytest.mark.parametrize("N,limbs,W,msg", [
    (3, [7], 0, "power of two"),
    (131072, [7], 0, "power of two"),
    (1024, [8], 0, "odd"),
    (1024, [7, 0], 0, "top limb"),
    (1024, [7], 40, "bit width"),
    (1024, [0xffffffff] * 33, 0, "L must be"),
])
def test_self_check_rejects_invalid_points(N, limbs, W, msg):
    with pytest.raises(nc.NegacyclicError, match=msg) as ei:
        nc.self_check(N, np.array(limbs, dtype=np.uint32), W=W)
    assert ei.value.code == nc.NC_EINVAL


def test_thirty_bit_prime_set():
    """The 30-bit engine's primes: 64 distinct primes below 2^30 (above 2^29), 1 mod 2^17, descending;
    the reference's bound picks 59 of them for an 868-bit q at N = 2^16 and all 64 reach 948 bits."""
    ps = nc.primes32(64)
    assert len(ps) == 64 and ps == sorted(ps, reverse=True) and len(set(ps)) == 64
    for p in ps:
        assert (1 << 29) < p < (1 << 30) and (p - 1) % (1 << 17) == 0
        assert all(pow(a, p - 1, p) == 1 for a in (2, 3, 5, 7, 11, 13))

    def needed(log_n, bits):
        prod, k = 1, 0
        while prod.bit_length() < log_n + 2 * bits + 4:
            prod *= ps[k]
            k += 1
        return k

    assert needed(16, 868) == 59
    prod = 1
    for p in ps:
        prod *= p
    assert (prod.bit_length() - 16 - 4) // 2 == 948


def test_mirror_twiddle_identity():
    """The 30-bit row stage stages only forward twiddles: the inverse twiddle of node 2^s + j of the
    merged tree, psi^-bitrev(2^s + j), is the negated forward twiddle of the mirror node
    2^s + (2^s - 1 - j), because psi^N = -1 (psi a primitive 2N-th root, N = 2^16). Checked for
    three of the engine's primes over every node, with psi found independently here."""
    def bitrev16(x):
        return int(format(x, "016b")[::-1], 2)

    rev = np.array([bitrev16(x) for x in range(1 << 16)], dtype=np.int64)
    s_of = np.zeros(1 << 16, dtype=np.int64)
    for s in range(16):
        s_of[1 << s:2 << s] = s
    node = np.arange(1, 1 << 16, dtype=np.int64)
    mirror = (1 << s_of[1:]) + ((1 << s_of[1:]) - 1 - (node - (1 << s_of[1:])))
    for p in nc.primes32(64)[::31]:
        g = next(a for a in range(2, 200) if pow(a, (p - 1) // 2, p) != 1)
        psi = pow(g, (p - 1) >> 17, p)
        assert pow(psi, 1 << 16, p) == p - 1
        # psi^e for every e < 2^17
        powers = np.empty(1 << 17, dtype=np.int64)
        acc = 1
        for e in range(1 << 17):
            powers[e] = acc
            acc = acc * psi % p
        fwd = powers[rev]                       # psi^bitrev(n)
        inv = powers[((1 << 17) - rev) % (1 << 17)]  # psi^-bitrev(n)
        assert np.array_equal(inv[node], (p - fwd[mirror]) % p)
