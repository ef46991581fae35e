/*
 * CPU oracle for the negacyclic product c = a*b mod (X^N + 1, q).
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker: tests/, the smoke test and
 * bench.py's cpu_baseline leg call it to produce the expected answer. The product
 * path (the CUDA library) never links, loads or calls it.
 *
 * It restates, in plain C, the algorithm of the reference solution
 * (engel-cuda-negacyclic-multiply, solve.cu):
 *   - 62-bit NTT primes p = 1 (mod 2N), searched downward from 2^62 and taken
 *     until bitlen(prod p) >= log2 N + 2*bits(q) + 4           (solve.cu:1174-1204)
 *   - a primitive 2N-th root psi found as base^((p-1)/2N) with psi^N = -1,
 *     bases tried from 2 upward                                 (solve.cu:495-502)
 *   - residues of each coefficient: sum_j limb_j * (2^(32j) mod p) (solve.cu:533-570)
 *   - psi-twist, cyclic NTT with omega = psi^2, pointwise product,
 *     inverse NTT, multiply by N^-1 and psi^-i                 (solve.cu:1226-1257, 620-642, 952-1044)
 *   - direct CRT: v_i = r_i * (M/p_i)^-1 mod p_i,
 *     acc = sum v_i * (M/p_i mod q), k = floor(sum v_i / p_i) taken as a
 *     64.64 fixed-point sum, result = acc - k*(M mod q) mod q, and one more
 *     (M mod q) subtracted when the fraction is >= 1/2 (negative coefficient)
 *                                                               (solve.cu:752-836)
 *   - reduction mod q by shift-and-subtract                     (solve.cu:453-466)
 *
 * The arithmetic primitives mirrored by the reference's self-checks in fherma_init
 * (solve.cu:1151-1165, 1285-1314, 1370-1415) are exported so the tests can pin them.
 * Parity of whole products is pinned against a Python big-integer schoolbook and
 * against outputs of the reference solve.cu itself (tests/golden).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

#define OR_MAX_PRIMES 48 /* solve.cu:22 kMaxChannels */
#define OR_WIDE 96       /* limbs of the prime product (48 * 62 bits < 96 * 32) */

/* ---------------------------------------------------------------- 64-bit helpers */

uint64_t oracle_mul_mod(uint64_t a, uint64_t b, uint64_t p) { return (uint64_t)(((u128)a * b) % p); }

uint64_t oracle_pow_mod(uint64_t base, uint64_t e, uint64_t p) {
    uint64_t r = 1 % p;
    base %= p;
    while (e) {
        if (e & 1) r = oracle_mul_mod(r, base, p);
        base = oracle_mul_mod(base, base, p);
        e >>= 1;
    }
    return r;
}

/* -p^-1 mod 2^64 by Newton iteration (solve.cu:253-257 computes p^-1). */
uint64_t oracle_neg_inv64(uint64_t p) {
    uint64_t x = p; /* correct to 3 bits for odd p */
    for (int i = 0; i < 6; ++i) x *= 2 - p * x;
    return 0 - x;
}

/* Montgomery product a*b*2^-64 mod p with two final corrections (solve.cu:134-148). */
uint64_t oracle_mont_mul(uint64_t a, uint64_t b, uint64_t p, uint64_t nprime) {
    u128 t = (u128)a * b;
    uint64_t m = (uint64_t)t * nprime;
    u128 mp = (u128)m * p;
    uint64_t lo = (uint64_t)t + (uint64_t)mp; /* zero by construction; only its carry matters */
    uint64_t r = (uint64_t)(t >> 64) + (uint64_t)(mp >> 64) + (lo < (uint64_t)t ? 1u : 0u);
    if (r >= p) r -= p;
    if (r >= p) r -= p;
    return r;
}

/* Shoup companion floor(w * 2^64 / p). */
uint64_t oracle_shoup_companion(uint64_t w, uint64_t p) { return (uint64_t)(((u128)w << 64) / p); }

/* Shoup product a*w mod p with one correction; valid for p < 2^63 (solve.cu:151-156). */
uint64_t oracle_shoup_mul(uint64_t a, uint64_t w, uint64_t wshoup, uint64_t p) {
    uint64_t qh = (uint64_t)(((u128)a * wshoup) >> 64);
    uint64_t r = a * w - qh * p;
    if (r >= p) r -= p;
    return r;
}

/* floor(2^96 / p) and the Barrett remainder of a 128-bit value (solve.cu:158-195, 239-251). */
uint64_t oracle_barrett_mu96(uint64_t p) { return (uint64_t)((((u128)1) << 96) / p); }

uint64_t oracle_barrett_reduce(uint64_t hi, uint64_t lo, uint64_t p, uint64_t mu) {
    (void)mu; /* the restated reduction is exact division; mu is checked by its own KAT */
    u128 v = ((u128)hi << 64) | lo;
    return (uint64_t)(v % p);
}

/* floor(2^64 / d) and its remainder (solve.cu:1117-1128). */
uint64_t oracle_div_pow2_64(uint64_t d, uint64_t* rem) {
    u128 n = (u128)1 << 64;
    *rem = (uint64_t)(n % d);
    return (uint64_t)(n / d);
}

/* floor(2^128 / p) as hi:lo, used by the fixed-point quotient estimate (solve.cu:1359-1368). */
void oracle_magic128(uint64_t p, uint64_t* hi, uint64_t* lo) {
    /* 2^128 = (2^64 * 2^64); do it as two 64-bit long-division steps. */
    u128 top = (u128)1 << 64; /* 2^64 */
    uint64_t qh = (uint64_t)(top / p);
    uint64_t r = (uint64_t)(top % p);
    u128 next = (u128)r << 64;
    uint64_t ql = (uint64_t)(next / p);
    *hi = qh;
    *lo = ql;
}

/* 128-bit value mod p (solve.cu:77-98 / 200-237 compute the same remainder). */
uint64_t oracle_mod128(uint64_t hi, uint64_t lo, uint64_t p) { return (uint64_t)((((u128)hi << 64) | lo) % p); }

/* Deterministic Miller-Rabin for 64-bit n (same bases as solve.cu:476). */
int oracle_is_prime_u64(uint64_t n) {
    if (n < 2) return 0;
    if ((n & 1) == 0) return n == 2;
    uint64_t d = n - 1;
    int s = 0;
    while ((d & 1) == 0) {
        d >>= 1;
        ++s;
    }
    static const uint64_t bases[] = {2ull, 325ull, 9375ull, 28178ull, 450775ull, 9780504ull, 1795265022ull};
    for (int b = 0; b < 7; ++b) {
        uint64_t a = bases[b] % n;
        if (a == 0) continue;
        uint64_t x = oracle_pow_mod(a, d, n);
        if (x == 1 || x == n - 1) continue;
        int composite = 1;
        for (int r = 1; r < s; ++r) {
            x = oracle_mul_mod(x, x, n);
            if (x == n - 1) {
                composite = 0;
                break;
            }
        }
        if (composite) return 0;
    }
    return 1;
}

/* ---------------------------------------------------------------- multi-limb helpers */

static int top_bit_limbs(const uint32_t* v, int n) {
    for (int i = n - 1; i >= 0; --i)
        if (v[i]) return i * 32 + (31 - __builtin_clz(v[i]));
    return -1;
}

/* acc[0..n) += t[0..tn) * f (f < 2^64); carries propagate to the end of acc. */
static void limbs_addmul_u64(uint32_t* acc, int n, const uint32_t* t, int tn, uint64_t f) {
    uint32_t f0 = (uint32_t)f, f1 = (uint32_t)(f >> 32);
    uint64_t carry = 0;
    for (int i = 0; i < n; ++i) {
        uint64_t ti = i < tn ? t[i] : 0;
        u128 cur = (u128)acc[i] + (u128)ti * f0 + carry;
        acc[i] = (uint32_t)cur;
        carry = (uint64_t)(cur >> 32);
    }
    if (!f1) return;
    carry = 0;
    for (int i = 1; i < n; ++i) {
        uint64_t ti = (i - 1) < tn ? t[i - 1] : 0;
        u128 cur = (u128)acc[i] + (u128)ti * f1 + carry;
        acc[i] = (uint32_t)cur;
        carry = (uint64_t)(cur >> 32);
    }
}

/* r = value mod p for an n-limb value (solve.cu:280-291). */
uint64_t oracle_limbs_mod_u64(const uint32_t* v, int n, uint64_t p) {
    u128 r = 0;
    for (int i = n - 1; i >= 0; --i) r = ((r << 32) | v[i]) % p;
    return (uint64_t)r;
}

/* acc mod q in place by shift-and-subtract over the bit positions (solve.cu:453-466). */
void oracle_mod_q(uint32_t* acc, int n, const uint32_t* q, int ql) {
    int qt = top_bit_limbs(q, ql);
    if (qt < 0) return;
    int at = top_bit_limbs(acc, n);
    for (int shift = at - qt; shift >= 0; --shift) {
        /* compare acc with q << shift */
        int word = shift >> 5, bits = shift & 31;
        int cmp = 0;
        for (int i = n - 1; i >= 0 && cmp == 0; --i) {
            int src = i - word;
            uint32_t s = 0;
            if (src >= 0 && src < ql) s = q[src] << bits;
            if (bits && src - 1 >= 0 && src - 1 < ql) s |= q[src - 1] >> (32 - bits);
            if (acc[i] != s) cmp = acc[i] > s ? 1 : -1;
        }
        if (cmp < 0) continue;
        uint64_t borrow = 0;
        for (int i = 0; i < n; ++i) {
            int src = i - word;
            uint32_t s = 0;
            if (src >= 0 && src < ql) s = q[src] << bits;
            if (bits && src - 1 >= 0 && src - 1 < ql) s |= q[src - 1] >> (32 - bits);
            uint64_t d = (uint64_t)acc[i] - s - borrow;
            acc[i] = (uint32_t)d;
            borrow = (d >> 63) & 1;
        }
    }
}

/* out = (x - y) mod q for x, y in [0, q), L limbs. */
static void sub_mod_q(uint32_t* x, const uint32_t* y, const uint32_t* q, int L) {
    uint64_t borrow = 0;
    for (int i = 0; i < L; ++i) {
        uint64_t d = (uint64_t)x[i] - y[i] - borrow;
        x[i] = (uint32_t)d;
        borrow = (d >> 63) & 1;
    }
    if (borrow) {
        uint64_t carry = 0;
        for (int i = 0; i < L; ++i) {
            uint64_t s = (uint64_t)x[i] + q[i] + carry;
            x[i] = (uint32_t)s;
            carry = s >> 32;
        }
    }
}

/* ---------------------------------------------------------------- planning */

/* The reference's prime rule (solve.cu:1174-1204). Returns the count, or -1 if the
   bound cannot be met within OR_MAX_PRIMES primes. */
int oracle_primes(uint32_t N, int q_bits, uint64_t* out, int max_out) {
    int log_n = 0;
    for (uint32_t v = N; v > 1; v >>= 1) ++log_n;
    const int bound_bits = log_n + 2 * q_bits + 4;
    const uint64_t step = 2ull * N;
    uint64_t cand = (1ull << 62) - 1;
    cand -= (cand - 1) % step;
    uint32_t prod[OR_WIDE];
    memset(prod, 0, sizeof prod);
    prod[0] = 1;
    int count = 0;
    while (cand > step && top_bit_limbs(prod, OR_WIDE) + 1 < bound_bits) {
        if (oracle_is_prime_u64(cand)) {
            if (count >= max_out || count >= OR_MAX_PRIMES) return -1;
            uint32_t next[OR_WIDE];
            memset(next, 0, sizeof next);
            limbs_addmul_u64(next, OR_WIDE, prod, OR_WIDE, cand);
            memcpy(prod, next, sizeof prod);
            out[count++] = cand;
        }
        cand -= step;
    }
    if (top_bit_limbs(prod, OR_WIDE) + 1 < bound_bits) return -1;
    return count;
}

/* psi with psi^N = -1, tried from base 2 upward (solve.cu:495-502). */
uint64_t oracle_find_psi(uint64_t p, uint32_t N) {
    uint64_t e = (p - 1) / (2ull * N);
    for (uint64_t base = 2; base < 10000; ++base) {
        uint64_t psi = oracle_pow_mod(base, e, p);
        if (oracle_pow_mod(psi, N, p) == p - 1) return psi;
    }
    return 0;
}

/* ---------------------------------------------------------------- NTT over one prime */

static uint32_t bitrev(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
}

/* In-place cyclic NTT with root w (order N): bit-reversed load, then radix-2 DIT,
   natural-order output (the reference's forward_ntt shape, solve.cu:1006-1038). */
static void ntt_cyclic(uint64_t* x, uint32_t N, uint64_t w, uint64_t p) {
    int bits = 0;
    for (uint32_t v = N; v > 1; v >>= 1) ++bits;
    for (uint32_t i = 0; i < N; ++i) {
        uint32_t j = bitrev(i, bits);
        if (i < j) {
            uint64_t t = x[i];
            x[i] = x[j];
            x[j] = t;
        }
    }
    for (uint32_t half = 1; half < N; half <<= 1) {
        uint64_t step = oracle_pow_mod(w, N / (2 * half), p);
        uint64_t tw = 1;
        for (uint32_t lane = 0; lane < half; ++lane) {
            uint64_t tws = oracle_shoup_companion(tw, p);
            for (uint32_t start = 0; start < N; start += 2 * half) {
                uint64_t u = x[start + lane];
                uint64_t v = oracle_shoup_mul(x[start + lane + half], tw, tws, p);
                uint64_t s = u + v;
                x[start + lane] = s >= p ? s - p : s;
                x[start + lane + half] = u >= v ? u - v : u + p - v;
            }
            tw = oracle_mul_mod(tw, step, p);
        }
    }
}

/* Negacyclic product of one residue row pair: ra <- ra * rb mod (X^N + 1, p). */
static void negacyclic_row(uint64_t* ra, uint64_t* rb, uint32_t N, uint64_t p) {
    uint64_t psi = oracle_find_psi(p, N);
    uint64_t psi_inv = oracle_pow_mod(psi, p - 2, p);
    uint64_t w = oracle_mul_mod(psi, psi, p);
    uint64_t w_inv = oracle_pow_mod(w, p - 2, p);
    uint64_t n_inv = oracle_pow_mod(N, p - 2, p);
    uint64_t t = 1;
    for (uint32_t i = 0; i < N; ++i) {
        ra[i] = oracle_mul_mod(ra[i], t, p);
        rb[i] = oracle_mul_mod(rb[i], t, p);
        t = oracle_mul_mod(t, psi, p);
    }
    ntt_cyclic(ra, N, w, p);
    ntt_cyclic(rb, N, w, p);
    for (uint32_t i = 0; i < N; ++i) ra[i] = oracle_mul_mod(ra[i], rb[i], p);
    ntt_cyclic(ra, N, w_inv, p);
    t = n_inv;
    for (uint32_t i = 0; i < N; ++i) {
        ra[i] = oracle_mul_mod(ra[i], t, p);
        t = oracle_mul_mod(t, psi_inv, p);
    }
}

/* ---------------------------------------------------------------- whole product */

/* c = a*b mod (X^N + 1, q). a, b, c hold N*L little-endian u32 limbs, coefficient-major
   (coefficient i at [i*L, i*L+L)). Returns 0, or a negative code for an invalid point.
   threads <= 0 uses every available thread. */
int oracle_negacyclic(uint32_t N, uint32_t L, const uint32_t* q, const uint32_t* a, const uint32_t* b,
                      uint32_t* c, int threads) {
    if (N < 2 || (N & (N - 1)) || L == 0 || L > 32) return -1;
    if ((q[0] & 1u) == 0) return -2;
    const int q_bits = top_bit_limbs(q, (int)L) + 1;
    uint64_t primes[OR_MAX_PRIMES];
    const int k = oracle_primes(N, q_bits, primes, OR_MAX_PRIMES);
    if (k <= 0) return -3;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    uint64_t* ra = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)k * N);
    uint64_t* rb = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)k * N);
    if (!ra || !rb) {
        free(ra);
        free(rb);
        return -4;
    }

    /* residues and per-prime negacyclic products */
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < k; ++i) {
        uint64_t p = primes[i];
        uint64_t* xa = ra + (size_t)i * N;
        uint64_t* xb = rb + (size_t)i * N;
        for (uint32_t n = 0; n < N; ++n) {
            xa[n] = oracle_limbs_mod_u64(a + (size_t)n * L, (int)L, p);
            xb[n] = oracle_limbs_mod_u64(b + (size_t)n * L, (int)L, p);
        }
        negacyclic_row(xa, xb, N, p);
    }

    /* CRT tables: M, M/p_i mod q, (M/p_i)^-1 mod p_i, M mod q (solve.cu:1342-1369) */
    uint32_t M[OR_WIDE];
    memset(M, 0, sizeof M);
    M[0] = 1;
    for (int i = 0; i < k; ++i) {
        uint32_t next[OR_WIDE];
        memset(next, 0, sizeof next);
        limbs_addmul_u64(next, OR_WIDE, M, OR_WIDE, primes[i]);
        memcpy(M, next, sizeof M);
    }
    uint32_t* miq = (uint32_t*)calloc((size_t)k * L, sizeof(uint32_t));
    uint64_t y[OR_MAX_PRIMES];
    for (int i = 0; i < k; ++i) {
        uint32_t mi[OR_WIDE];
        memset(mi, 0, sizeof mi);
        mi[0] = 1;
        uint64_t prod_mod = 1;
        for (int j = 0; j < k; ++j) {
            if (j == i) continue;
            uint32_t next[OR_WIDE];
            memset(next, 0, sizeof next);
            limbs_addmul_u64(next, OR_WIDE, mi, OR_WIDE, primes[j]);
            memcpy(mi, next, sizeof mi);
            prod_mod = oracle_mul_mod(prod_mod, primes[j] % primes[i], primes[i]);
        }
        y[i] = oracle_pow_mod(prod_mod, primes[i] - 2, primes[i]);
        oracle_mod_q(mi, OR_WIDE, q, (int)L);
        memcpy(miq + (size_t)i * L, mi, sizeof(uint32_t) * L);
    }
    uint32_t mmq[OR_WIDE];
    memcpy(mmq, M, sizeof M);
    oracle_mod_q(mmq, OR_WIDE, q, (int)L);

    const int W = (int)L + 4; /* sum of k < 2^6 terms of 62+32L bits */
#pragma omp parallel for schedule(static)
    for (int64_t n = 0; n < (int64_t)N; ++n) {
        uint32_t acc[36 + 4];
        memset(acc, 0, sizeof acc);
        u128 frac = 0; /* sum of floor(v_i * 2^64 / p_i): integer part in bits 64.. */
        for (int i = 0; i < k; ++i) {
            uint64_t p = primes[i];
            uint64_t v = oracle_mul_mod(ra[(size_t)i * N + n], y[i], p);
            limbs_addmul_u64(acc, W, miq + (size_t)i * L, (int)L, v);
            frac += (((u128)v) << 64) / p;
        }
        uint64_t whole = (uint64_t)(frac >> 64);
        uint64_t part = (uint64_t)frac;
        oracle_mod_q(acc, W, q, (int)L);
        uint32_t mult[36 + 4];
        memset(mult, 0, sizeof mult);
        limbs_addmul_u64(mult, W, mmq, (int)L, whole);
        oracle_mod_q(mult, W, q, (int)L);
        sub_mod_q(acc, mult, q, (int)L);
        if (part >= (1ull << 63)) sub_mod_q(acc, mmq, q, (int)L);
        memcpy(c + (size_t)n * L, acc, sizeof(uint32_t) * L);
    }
    free(miq);
    free(ra);
    free(rb);
    return 0;
}

/* Plain O(N^2) negacyclic schoolbook over exact integers: both signed partial sums are
   accumulated exactly and reduced mod q once per output coefficient. For small N only; an
   independent check of oracle_negacyclic. */
int oracle_schoolbook(uint32_t N, uint32_t L, const uint32_t* q, const uint32_t* a, const uint32_t* b, uint32_t* c) {
    if (L == 0 || L > 32) return -1;
    const int W = 2 * (int)L + 2; /* N * q^2 < 2^(32 + 64 L) for N < 2^32 */
    uint32_t* acc[2];
    acc[0] = (uint32_t*)malloc(sizeof(uint32_t) * W);
    acc[1] = (uint32_t*)malloc(sizeof(uint32_t) * W);
    for (uint32_t k = 0; k < N; ++k) {
        memset(acc[0], 0, sizeof(uint32_t) * W);
        memset(acc[1], 0, sizeof(uint32_t) * W);
        for (uint32_t i = 0; i < N; ++i) {
            uint32_t j = (k + N - i) % N; /* i + j = k (positive) or k + N (negative) */
            const uint32_t* x = a + (size_t)i * L;
            const uint32_t* z = b + (size_t)j * L;
            uint32_t* dst = acc[i <= k ? 0 : 1];
            for (uint32_t s = 0; s < L; ++s) {
                uint64_t carry = 0;
                const uint64_t xs = x[s];
                for (uint32_t t = 0; t < L; ++t) {
                    uint64_t cur = (uint64_t)dst[s + t] + xs * z[t] + carry;
                    dst[s + t] = (uint32_t)cur;
                    carry = cur >> 32;
                }
                for (int u = (int)(s + L); carry && u < W; ++u) {
                    uint64_t cur = (uint64_t)dst[u] + carry;
                    dst[u] = (uint32_t)cur;
                    carry = cur >> 32;
                }
            }
        }
        oracle_mod_q(acc[0], W, q, (int)L);
        oracle_mod_q(acc[1], W, q, (int)L);
        sub_mod_q(acc[0], acc[1], q, (int)L);
        memcpy(c + (size_t)k * L, acc[0], sizeof(uint32_t) * L);
    }
    free(acc[0]);
    free(acc[1]);
    return 0;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
