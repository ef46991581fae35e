// Host-side precompute for the negacyclic product (see hostmath.h).
#include "hostmath.h"

#include <algorithm>
#include <mutex>
#include <thread>

namespace nc {

using u128 = unsigned __int128;

uint64_t mulmod64(uint64_t a, uint64_t b, uint64_t p) { return uint64_t((u128(a) * b) % p); }

uint64_t powmod64(uint64_t a, uint64_t e, uint64_t p) {
    uint64_t r = 1 % p;
    a %= p;
    while (e) {
        if (e & 1) r = mulmod64(r, a, p);
        a = mulmod64(a, a, p);
        e >>= 1;
    }
    return r;
}

// Deterministic Miller-Rabin for 64-bit integers: the first twelve primes as bases.
bool is_prime64(uint64_t n) {
    if (n < 2) return false;
    static const uint64_t small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    for (uint64_t s : small) {
        if (n % s == 0) return n == s;
    }
    uint64_t d = n - 1;
    int r = 0;
    while ((d & 1) == 0) {
        d >>= 1;
        ++r;
    }
    for (uint64_t a : small) {
        uint64_t x = powmod64(a, d, n);
        if (x == 1 || x == n - 1) continue;
        bool composite = true;
        for (int i = 1; i < r; ++i) {
            x = mulmod64(x, x, n);
            if (x == n - 1) {
                composite = false;
                break;
            }
        }
        if (composite) return false;
    }
    return true;
}

int bit_length(const uint32_t* v, int L) {
    for (int i = L - 1; i >= 0; --i)
        if (v[i]) return i * 32 + 32 - __builtin_clz(v[i]);
    return 0;
}

// ---------------------------------------------------------------------------- big integers

namespace {

using Big = std::vector<uint32_t>;  // little-endian words, no fixed length

void trim(Big& a) {
    while (!a.empty() && a.back() == 0) a.pop_back();
}

int bits_of(const Big& a) { return bit_length(a.data(), int(a.size())); }

Big mul_u64(const Big& a, uint64_t f) {
    Big r(a.size() + 3, 0);
    const uint64_t f0 = uint32_t(f), f1 = f >> 32;
    for (size_t pass = 0; pass < 2; ++pass) {
        const uint64_t fv = pass ? f1 : f0;
        uint64_t carry = 0;
        for (size_t i = 0; i < a.size(); ++i) {
            const u128 cur = u128(r[i + pass]) + u128(a[i]) * fv + carry;
            r[i + pass] = uint32_t(cur);
            carry = uint64_t(cur >> 32);
        }
        for (size_t i = a.size() + pass; carry && i < r.size(); ++i) {
            const uint64_t cur = uint64_t(r[i]) + carry;
            r[i] = uint32_t(cur);
            carry = cur >> 32;
        }
    }
    trim(r);
    return r;
}

// a / d exactly (remainder discarded) and a mod d.
Big div_u64(const Big& a, uint64_t d, uint64_t* rem) {
    Big q(a.size(), 0);
    u128 r = 0;
    for (int i = int(a.size()) - 1; i >= 0; --i) {
        r = (r << 32) | a[i];
        q[i] = uint32_t(r / d);
        r %= d;
    }
    if (rem) *rem = uint64_t(r);
    trim(q);
    return q;
}

int cmp_shifted(const Big& a, const Big& b, int shift) {
    // compare a with b << shift
    const int words = int(std::max(a.size(), b.size() + size_t(shift / 32) + 1));
    for (int i = words - 1; i >= 0; --i) {
        const int w = shift >> 5, s = shift & 31;
        uint32_t bv = 0;
        const int src = i - w;
        if (src >= 0 && src < int(b.size())) bv = b[src] << s;
        if (s && src - 1 >= 0 && src - 1 < int(b.size())) bv |= b[src - 1] >> (32 - s);
        const uint32_t av = i < int(a.size()) ? a[i] : 0;
        if (av != bv) return av > bv ? 1 : -1;
    }
    return 0;
}

void sub_shifted(Big& a, const Big& b, int shift) {
    const int w = shift >> 5, s = shift & 31;
    int64_t borrow = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        uint32_t bv = 0;
        const int src = int(i) - w;
        if (src >= 0 && src < int(b.size())) bv = b[src] << s;
        if (s && src - 1 >= 0 && src - 1 < int(b.size())) bv |= b[src - 1] >> (32 - s);
        const int64_t cur = int64_t(a[i]) - bv - borrow;
        a[i] = uint32_t(cur);
        borrow = cur < 0 ? 1 : 0;
    }
    trim(a);
}

// a mod m and (optionally) floor(a / m), by shift-and-subtract.
Big divmod(Big a, const Big& m, Big* quot) {
    trim(a);
    const int mb = bits_of(m);
    int ab = bits_of(a);
    Big q;
    if (quot) q.assign(a.size() + 1, 0);
    for (int shift = ab - mb; shift >= 0; --shift) {
        if (cmp_shifted(a, m, shift) >= 0) {
            sub_shifted(a, m, shift);
            if (quot) q[shift >> 5] |= 1u << (shift & 31);
        }
    }
    if (quot) {
        trim(q);
        *quot = q;
    }
    return a;
}

Big add_big(const Big& a, const Big& b) {
    Big r(std::max(a.size(), b.size()) + 1, 0);
    uint64_t carry = 0;
    for (size_t i = 0; i + 1 < r.size(); ++i) {
        const uint64_t cur = uint64_t(i < a.size() ? a[i] : 0) + (i < b.size() ? b[i] : 0) + carry;
        r[i] = uint32_t(cur);
        carry = cur >> 32;
    }
    r.back() = uint32_t(carry);
    trim(r);
    return r;
}

Big mul_big(const Big& a, const Big& b) {
    Big r(a.size() + b.size() + 1, 0);
    for (size_t i = 0; i < a.size(); ++i) {
        uint64_t carry = 0;
        for (size_t j = 0; j < b.size(); ++j) {
            const uint64_t cur = uint64_t(r[i + j]) + uint64_t(a[i]) * b[j] + carry;
            r[i + j] = uint32_t(cur);
            carry = cur >> 32;
        }
        for (size_t t = i + b.size(); carry; ++t) {
            const uint64_t cur = uint64_t(r[t]) + carry;
            r[t] = uint32_t(cur);
            carry = cur >> 32;
        }
    }
    trim(r);
    return r;
}

int cmp_big(const Big& a, const Big& b) { return cmp_shifted(a, b, 0); }

Big pow2(int e) {
    Big r(size_t(e / 32 + 1), 0);
    r[e / 32] = 1u << (e % 32);
    return r;
}

uint32_t bitrev(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
}

std::vector<PrimeConst> make_prime_set() {
    std::vector<PrimeConst> out;
    const uint64_t step = 1ull << kRootLog;
    uint64_t cand = (1ull << 62) - step + 1;
    while (int(out.size()) < kMaxPrimes) {
        if (is_prime64(cand)) {
            PrimeConst c{};
            c.p = cand;
            c.m = (1ull << 62) - cand;
            c.g = uint32_t((u128(1) << 93) / cand);
            out.push_back(c);
        }
        cand -= step;
    }
    return out;
}

}  // namespace

const std::vector<PrimeConst>& prime_set() {
    static const std::vector<PrimeConst> set = make_prime_set();
    return set;
}

int primes_needed(int logN, int qbits, int factors) {
    const int bound_bits = (factors - 1) * logN + factors * qbits + 4;
    Big prod{1};
    const auto& ps = prime_set();
    for (int k = 1; k <= kMaxPrimes; ++k) {
        prod = mul_u64(prod, ps[k - 1].p);
        if (bits_of(prod) >= bound_bits) return k;
    }
    return -1;
}

const HostTables& host_tables() {
    static HostTables t;
    static std::once_flag once;
    std::call_once(once, [] {
        t.pc = prime_set();
        t.psi.assign(kMaxPrimes, 0);
        t.pow32.assign(size_t(kMaxPrimes) * kMaxL, 0);
        t.fwd.assign(size_t(kMaxPrimes) * kMaxN * 2, 0);
        t.inv.assign(size_t(kMaxPrimes) * kMaxN * 2, 0);
        auto work = [](int i) {
            const uint64_t p = t.pc[i].p;
            // psi of multiplicative order 2^17: g^((p-1)/2^17) with psi^(2^16) = -1
            uint64_t psi = 0;
            for (uint64_t g = 2; g < 1000000; ++g) {
                const uint64_t c = powmod64(g, (p - 1) >> kRootLog, p);
                if (powmod64(c, 1ull << kMaxLogN, p) == p - 1) {
                    psi = c;
                    break;
                }
            }
            t.psi[i] = psi;
            uint64_t place = 1;
            for (int l = 0; l < kMaxL; ++l) {
                t.pow32[size_t(i) * kMaxL + l] = place;
                place = mulmod64(place, 1ull << 32, p);
            }
            std::vector<uint64_t> pw(kMaxN + 1);
            pw[0] = 1;
            for (int e = 1; e <= kMaxN; ++e) pw[e] = mulmod64(pw[e - 1], psi, p);
            // pw[kMaxN] = -1, so psi^-e = -psi^(kMaxN - e)
            uint64_t* f = t.fwd.data() + size_t(i) * kMaxN * 2;
            uint64_t* g = t.inv.data() + size_t(i) * kMaxN * 2;
            for (uint32_t j = 0; j < uint32_t(kMaxN); ++j) {
                const uint32_t e = bitrev(j, kMaxLogN);
                const uint64_t w = pw[e];
                const uint64_t wi = e == 0 ? 1 : p - pw[kMaxN - e];
                f[2 * j] = w;
                f[2 * j + 1] = uint64_t((u128(w) << 64) / p);
                g[2 * j] = wi;
                g[2 * j + 1] = uint64_t((u128(wi) << 64) / p);
            }
        };
        const int nthreads = std::max(1, std::min<int>(16, int(std::thread::hardware_concurrency())));
        std::vector<std::thread> pool;
        for (int w = 0; w < nthreads; ++w)
            pool.emplace_back([&, w] {
                for (int i = w; i < kMaxPrimes; i += nthreads) work(i);
            });
        for (auto& th : pool) th.join();
    });
    return t;
}

// ---------------------------------------------------------------------------- self-checks

std::string check_arithmetic() {
    // the reference's fherma_init opens with known answers of its modular helpers
    // (solve.cu:1151-1165); these are the same facts for the helpers used here
    if (mulmod64(7, 5, 11) != 2) return "mulmod64(7, 5, 11) != 2";
    if (powmod64(3, 10, 11) != 1) return "powmod64(3, 10, 11) != 1";
    if (uint64_t((u128(1) << 64) / 3) != 6148914691236517205ull || uint64_t((u128(1) << 64) % 3) != 1)
        return "2^64 / 3 division";
    if (!is_prime64(2305843009213693951ull) || is_prime64(2305843009213693953ull)) return "Miller-Rabin on 2^61 - 1";
    const Big q{0xffffffffu, 0xffffffffu, 0xffffffffu, 0x7fffffffu};  // 2^127 - 1
    const Big x = mul_big(q, q);
    Big quo;
    const Big r = divmod(add_big(x, Big{5}), q, &quo);
    if (r != Big{5} || quo != q) return "big-integer (2^127 - 1)^2 + 5 division";
    return std::string();
}

std::string check_prime_set() {
    const auto& ps = prime_set();
    if (int(ps.size()) != kMaxPrimes) return "prime set size";
    for (int i = 0; i < kMaxPrimes; ++i) {
        const PrimeConst& c = ps[size_t(i)];
        if (!is_prime64(c.p)) return "prime " + std::to_string(i) + " is composite";
        if (((c.p - 1) & ((1ull << kRootLog) - 1)) != 0) return "prime " + std::to_string(i) + " is not 1 mod 2^17";
        if (c.m != (1ull << 62) - c.p || c.m >= (1ull << 28)) return "prime " + std::to_string(i) + " is not 2^62 - m";
        if (u128(c.g) * c.p > (u128(1) << 93) || (u128(c.g) + 1) * c.p <= (u128(1) << 93))
            return "prime " + std::to_string(i) + ": g != floor(2^93 / p)";
        if (i > 0 && c.p >= ps[size_t(i) - 1].p) return "prime set not descending";
    }
    return std::string();
}

std::string check_tables(const HostTables& t, int samples) {
    for (int i = 0; i < kMaxPrimes; ++i) {
        const uint64_t p = t.pc[size_t(i)].p;
        const uint64_t psi = t.psi[size_t(i)];
        const std::string at = "prime " + std::to_string(i) + ": ";
        if (powmod64(psi, 1ull << kMaxLogN, p) != p - 1) return at + "psi^(2^16) != -1";
        for (int l = 0; l < kMaxL; ++l)
            if (t.pow32[size_t(i) * kMaxL + size_t(l)] != powmod64(2, 32ull * uint64_t(l), p))
                return at + "2^(32 l) mod p";
        const uint64_t* f = t.fwd.data() + size_t(i) * kMaxN * 2;
        const uint64_t* g = t.inv.data() + size_t(i) * kMaxN * 2;
        for (int s = 0; s < samples; ++s) {
            const uint32_t j = uint32_t((uint64_t(s) * 2654435761u + uint64_t(i)) % uint64_t(kMaxN));
            const uint32_t e = bitrev(j, kMaxLogN);
            if (f[2 * j] != powmod64(psi, e, p)) return at + "twiddle psi^bitrev(j)";
            if (mulmod64(f[2 * j], g[2 * j], p) != 1) return at + "inverse twiddle";
            for (const uint64_t* w : {f + 2 * j, g + 2 * j}) {
                const u128 lhs = u128(w[0]) << 64, qp = u128(w[1]) * p;  // w' = floor(w 2^64 / p)
                if (qp > lhs || lhs - qp >= p) return at + "Shoup companion of a twiddle";
            }
        }
    }
    return std::string();
}

std::string check_qconst(const QConst& c) {
    const int k = int(c.k), L = int(c.L);
    const auto& ps = prime_set();
    if (k < 1 || k > kMaxPrimes || L < 1 || L > kMaxL) return "prime or limb count";
    Big qb(c.q, c.q + L);
    trim(qb);
    if (bits_of(qb) != int(c.qbits)) return "bit length of q";
    Big neg(c.neg_m, c.neg_m + kMqStride);
    trim(neg);
    if (cmp_big(neg, qb) >= 0) return "(-M) mod q is not below q";
    const uint64_t N = 1ull << c.logN;
    for (int i = 0; i < k; ++i) {
        const uint64_t p = ps[size_t(i)].p;
        const std::string at = "prime " + std::to_string(i) + ": ";
        // y_i (M / p_i) N = 1 (mod p_i), with M / p_i mod p_i formed as a product of the other primes
        uint64_t mi = 1;
        for (int j = 0; j < k; ++j)
            if (j != i) mi = mulmod64(mi, ps[size_t(j)].p % p, p);
        if (mulmod64(mulmod64(c.y[i], mi, p), N % p, p) != 1) return at + "y_i (M/p_i) N != 1 mod p_i";
        const u128 lhs = u128(c.y[i]) << 64, qp = u128(c.ys[i]) * p;
        if (qp > lhs || lhs - qp >= p) return at + "Shoup companion of y_i";
        // (M / p_i mod q) p_i + ((-M) mod q) = 0 (mod q)
        Big mq(c.mq + size_t(i) * kMqStride, c.mq + size_t(i) * kMqStride + kMqStride);
        trim(mq);
        if (cmp_big(mq, qb) >= 0) return at + "(M/p_i) mod q is not below q";
        if (!divmod(add_big(mul_u64(mq, p), neg), qb, nullptr).empty()) return at + "(M/p_i mod q) p_i != M mod q";
    }
    // mu = floor(2^(qbits + kBarrettT + 1) / q): mu q <= 2^e < (mu + 1) q
    Big mu(c.mu, c.mu + 4);
    trim(mu);
    const Big e = pow2(int(c.qbits) + kBarrettT + 1);
    if (cmp_big(mul_big(mu, qb), e) > 0 || cmp_big(add_big(mul_big(mu, qb), qb), e) <= 0) return "Barrett constant mu";
    return std::string();
}

void schoolbook_negacyclic(int N, int L, const uint32_t* q, const uint32_t* a, const uint32_t* b, uint32_t* c) {
    Big qb(q, q + L);
    trim(qb);
    for (int k = 0; k < N; ++k) {
        Big pos, neg;
        for (int i = 0; i < N; ++i) {
            const int j = k - i >= 0 ? k - i : k - i + N;
            Big x(a + size_t(i) * L, a + size_t(i) * L + L), y(b + size_t(j) * L, b + size_t(j) * L + L);
            trim(x);
            trim(y);
            if (k - i >= 0)
                pos = add_big(pos, mul_big(x, y));
            else
                neg = add_big(neg, mul_big(x, y));
        }
        pos = divmod(pos, qb, nullptr);
        neg = divmod(neg, qb, nullptr);
        if (cmp_big(pos, neg) < 0) pos = add_big(pos, qb);
        if (!neg.empty()) sub_shifted(pos, neg, 0);
        for (int l = 0; l < L; ++l) c[size_t(k) * L + size_t(l)] = size_t(l) < pos.size() ? pos[size_t(l)] : 0;
    }
}

std::string build_qconst(const uint32_t* q, int L, int logN, QConst* out, int factors) {
    if (L < 1 || L > kMaxL) return "L must be between 1 and 32";
    if (logN < 1 || logN > kMaxLogN) return "N must be a power of two from 2 to 65536";
    if ((q[0] & 1u) == 0) return "q must be odd";
    const int qbits = bit_length(q, L);
    if (qbits <= 32 * (L - 1)) return "the top limb of q must be nonzero";
    if (factors < 2 || factors > kMaxFactors) return "a product has 2 to 4 factors";
    const int k = primes_needed(logN, qbits, factors);
    if (k < 0) return "the coefficient bound does not fit the 48-prime residue budget";
    const auto& ps = prime_set();

    *out = QConst{};
    out->L = uint32_t(L);
    out->LW = uint32_t((L + 1) & ~1);
    out->k = uint32_t(k);
    out->qbits = uint32_t(qbits);
    out->logN = uint32_t(logN);
    Big qb(q, q + L);
    trim(qb);
    for (int l = 0; l < L; ++l) out->q[l] = q[l];

    Big M{1};
    for (int i = 0; i < k; ++i) M = mul_u64(M, ps[i].p);
    const uint64_t N = 1ull << logN;
    for (int i = 0; i < k; ++i) {
        const uint64_t p = ps[i].p;
        uint64_t rem = 0;
        const Big Mi = div_u64(M, p, &rem);
        uint64_t mi_mod_p = 0;
        div_u64(Mi, p, &mi_mod_p);
        // y = (M/p_i)^-1 * N^-1 mod p_i
        const uint64_t inv_mi = powmod64(mi_mod_p, p - 2, p);
        const uint64_t inv_n = powmod64(N % p, p - 2, p);
        const uint64_t y = mulmod64(inv_mi, inv_n, p);
        out->y[i] = y;
        out->ys[i] = uint64_t((u128(y) << 64) / p);
        const Big miq = divmod(Mi, qb, nullptr);
        for (size_t l = 0; l < miq.size() && l < size_t(kMqStride); ++l) out->mq[i * kMqStride + l] = miq[l];
    }
    const Big mmq = divmod(M, qb, nullptr);
    Big neg = qb;
    if (!mmq.empty()) sub_shifted(neg, mmq, 0);
    else neg.clear();  // M = 0 mod q cannot happen for prime q > 2^62, kept for completeness
    if (bits_of(neg) == bits_of(qb) && cmp_shifted(neg, qb, 0) == 0) neg.clear();
    for (size_t l = 0; l < neg.size(); ++l) out->neg_m[l] = neg[l];
    Big mu;
    divmod(pow2(qbits + kBarrettT + 1), qb, &mu);
    if (bits_of(mu) > 96) return "internal: Barrett constant too wide";
    for (size_t l = 0; l < mu.size() && l < 4; ++l) out->mu[l] = mu[l];
    return std::string();
}

// ---------------------------------------------------------------------------- 30-bit engine

namespace {

// The 64 largest primes below 2^30 that are 1 mod 2^17 (all above 2^29.8), descending.
std::vector<PrimeConst32> make_prime_set32() {
    std::vector<PrimeConst32> out;
    const uint64_t step = 1ull << kRootLog;
    for (uint64_t cand = (1ull << 30) - step + 1; int(out.size()) < kMaxPrimes32; cand -= step) {
        if (!is_prime64(cand)) continue;
        uint32_t inv = 1;  // p^-1 mod 2^32 by Newton's iteration (each step doubles the correct bits)
        for (int it = 0; it < 5; ++it) inv *= 2u - uint32_t(cand) * inv;
        PrimeConst32 c{};
        c.p = uint32_t(cand);
        c.pinv = 0u - inv;
        c.bar = uint32_t((1ull << 50) / cand);
        c.quo = uint32_t((1ull << 61) / cand);
        out.push_back(c);
    }
    return out;
}

uint32_t shoup32(uint32_t w, uint32_t p) { return uint32_t((uint64_t(w) << 32) / p); }

}  // namespace

const std::vector<PrimeConst32>& prime_set32() {
    static const std::vector<PrimeConst32> set = make_prime_set32();
    return set;
}

int primes_needed32(int logN, int qbits) {
    const int bound_bits = logN + 2 * qbits + 4;
    Big prod{1};
    const auto& ps = prime_set32();
    for (int k = 1; k <= kMaxPrimes32; ++k) {
        prod = mul_u64(prod, ps[size_t(k) - 1].p);
        if (bits_of(prod) >= bound_bits) return k;
    }
    return -1;
}

const HostTables32& host_tables32() {
    static HostTables32 t;
    static std::once_flag once;
    std::call_once(once, [] {
        t.pc = prime_set32();
        t.psi.assign(kMaxPrimes32, 0);
        t.pow32.assign(size_t(kMaxPrimes32) * kMaxL, 0);
        t.fwd.assign(size_t(kMaxPrimes32) * kMaxN * 2, 0);
        t.inv.assign(size_t(kMaxPrimes32) * kMaxN * 2, 0);
        auto work = [](int i) {
            const uint64_t p = t.pc[size_t(i)].p;
            uint64_t psi = 0;
            for (uint64_t g = 2; g < 1000000; ++g) {
                const uint64_t c = powmod64(g, (p - 1) >> kRootLog, p);
                if (powmod64(c, 1ull << kMaxLogN, p) == p - 1) {
                    psi = c;
                    break;
                }
            }
            t.psi[size_t(i)] = uint32_t(psi);
            uint64_t place = 1;
            for (int l = 0; l < kMaxL; ++l) {
                t.pow32[size_t(i) * kMaxL + size_t(l)] = uint32_t(place);
                place = (place << 32) % p;
            }
            std::vector<uint32_t> pw(kMaxN + 1);
            pw[0] = 1;
            for (int e = 1; e <= kMaxN; ++e) pw[size_t(e)] = uint32_t(uint64_t(pw[size_t(e) - 1]) * psi % p);
            uint32_t* f = t.fwd.data() + size_t(i) * kMaxN * 2;
            uint32_t* g = t.inv.data() + size_t(i) * kMaxN * 2;
            for (uint32_t j = 0; j < uint32_t(kMaxN); ++j) {
                const uint32_t e = bitrev(j, kMaxLogN);
                const uint32_t w = pw[e];
                const uint32_t wi = e == 0 ? 1u : uint32_t(p - pw[size_t(kMaxN) - e]);  // psi^-e = -psi^(N - e)
                f[2 * j] = w;
                f[2 * j + 1] = shoup32(w, uint32_t(p));
                g[2 * j] = wi;
                g[2 * j + 1] = shoup32(wi, uint32_t(p));
            }
        };
        const int nthreads = std::max(1, std::min<int>(16, int(std::thread::hardware_concurrency())));
        std::vector<std::thread> pool;
        for (int w = 0; w < nthreads; ++w)
            pool.emplace_back([&, w] {
                for (int i = w; i < kMaxPrimes32; i += nthreads) work(i);
            });
        for (auto& th : pool) th.join();
    });
    return t;
}

std::string check_prime_set32() {
    const auto& ps = prime_set32();
    if (int(ps.size()) != kMaxPrimes32) return "30-bit prime set size";
    for (int i = 0; i < kMaxPrimes32; ++i) {
        const PrimeConst32& c = ps[size_t(i)];
        const std::string at = "30-bit prime " + std::to_string(i) + ": ";
        if (!is_prime64(c.p)) return at + "composite";
        if (((c.p - 1) & ((1u << kRootLog) - 1)) != 0) return at + "not 1 mod 2^17";
        if (c.p >= (1u << 30) || c.p <= (1u << 29)) return at + "not in (2^29, 2^30)";
        if (uint32_t(c.p * (0u - c.pinv)) != 1u) return at + "pinv is not -p^-1 mod 2^32";
        if (uint64_t(c.bar) != (1ull << 50) / c.p || uint64_t(c.quo) != (1ull << 61) / c.p)
            return at + "reciprocal constants";
        if (i > 0 && c.p >= ps[size_t(i) - 1].p) return "30-bit prime set not descending";
    }
    return std::string();
}

std::string check_tables32(const HostTables32& t, int samples) {
    for (int i = 0; i < kMaxPrimes32; ++i) {
        const uint64_t p = t.pc[size_t(i)].p;
        const uint64_t psi = t.psi[size_t(i)];
        const std::string at = "30-bit prime " + std::to_string(i) + ": ";
        if (powmod64(psi, 1ull << kMaxLogN, p) != p - 1) return at + "psi^(2^16) != -1";
        for (int l = 0; l < kMaxL; ++l)
            if (t.pow32[size_t(i) * kMaxL + size_t(l)] != powmod64(2, 32ull * uint64_t(l), p))
                return at + "2^(32 l) mod p";
        const uint32_t* f = t.fwd.data() + size_t(i) * kMaxN * 2;
        const uint32_t* g = t.inv.data() + size_t(i) * kMaxN * 2;
        for (int s = 0; s < samples; ++s) {
            const uint32_t j = uint32_t((uint64_t(s) * 2654435761u + uint64_t(i)) % uint64_t(kMaxN));
            const uint32_t e = bitrev(j, kMaxLogN);
            if (f[2 * j] != powmod64(psi, e, p)) return at + "twiddle psi^bitrev(j)";
            if (uint64_t(f[2 * j]) * g[2 * j] % p != 1) return at + "inverse twiddle";
            for (const uint32_t* w : {f + 2 * j, g + 2 * j}) {
                const uint64_t lhs = uint64_t(w[0]) << 32, qp = uint64_t(w[1]) * p;  // w' = floor(w 2^32 / p)
                if (w[0] >= p || qp > lhs || lhs - qp >= p) return at + "Shoup companion of a twiddle";
            }
        }
    }
    return std::string();
}

std::string build_qconst32(const uint32_t* q, int L, int logN, QConst32* out) {
    if (L < 1 || L > kMaxL) return "L must be between 1 and 32";
    if (logN < 1 || logN > kMaxLogN) return "N must be a power of two from 2 to 65536";
    if ((q[0] & 1u) == 0) return "q must be odd";
    const int qbits = bit_length(q, L);
    if (qbits <= 32 * (L - 1)) return "the top limb of q must be nonzero";
    const int k = primes_needed32(logN, qbits);
    if (k < 0) return "the coefficient bound does not fit the 64-prime 30-bit residue budget";
    const auto& ps = prime_set32();
    *out = QConst32{};
    out->L = uint32_t(L);
    out->LW = uint32_t((L + 1) & ~1);
    out->k = uint32_t(k);
    out->qbits = uint32_t(qbits);
    out->logN = uint32_t(logN);
    Big qb(q, q + L);
    trim(qb);
    for (int l = 0; l < L; ++l) out->q[l] = q[l];
    Big M{1};
    for (int i = 0; i < k; ++i) M = mul_u64(M, ps[size_t(i)].p);
    const uint64_t N = 1ull << logN;
    for (int i = 0; i < k; ++i) {
        const uint64_t p = ps[size_t(i)].p;
        const Big Mi = div_u64(M, p, nullptr);
        uint64_t mi_mod_p = 0;
        div_u64(Mi, p, &mi_mod_p);
        // y = (M/p_i)^-1 N^-1 2^32 mod p_i: the 2^32 cancels the 2^-32 of the pointwise product
        const uint64_t y = mulmod64(mulmod64(powmod64(mi_mod_p, p - 2, p), powmod64(N % p, p - 2, p), p),
                                    (1ull << 32) % p, p);
        out->y[i] = uint32_t(y);
        out->ys[i] = shoup32(uint32_t(y), uint32_t(p));
        const Big miq = divmod(Mi, qb, nullptr);
        for (size_t l = 0; l < miq.size() && l < size_t(kMqStride); ++l) out->mq[size_t(i) * kMqStride + l] = miq[l];
    }
    const Big mmq = divmod(M, qb, nullptr);
    Big neg = qb;
    if (!mmq.empty()) sub_shifted(neg, mmq, 0);
    else neg.clear();
    if (cmp_big(neg, qb) == 0) neg.clear();
    for (size_t l = 0; l < neg.size(); ++l) out->neg_m[l] = neg[l];
    Big mu;
    divmod(pow2(qbits + kBarrettT + 1), qb, &mu);
    if (bits_of(mu) > 96) return "internal: Barrett constant too wide";
    for (size_t l = 0; l < mu.size() && l < 4; ++l) out->mu[l] = mu[l];
    return std::string();
}

std::string check_qconst32(const QConst32& c) {
    const int k = int(c.k), L = int(c.L);
    const auto& ps = prime_set32();
    if (k < 1 || k > kMaxPrimes32 || L < 1 || L > kMaxL) return "prime or limb count";
    Big qb(c.q, c.q + L);
    trim(qb);
    if (bits_of(qb) != int(c.qbits)) return "bit length of q";
    Big neg(c.neg_m, c.neg_m + kMqStride);
    trim(neg);
    if (cmp_big(neg, qb) >= 0) return "(-M) mod q is not below q";
    const uint64_t N = 1ull << c.logN;
    for (int i = 0; i < k; ++i) {
        const uint64_t p = ps[size_t(i)].p;
        const std::string at = "30-bit prime " + std::to_string(i) + ": ";
        uint64_t mi = 1;
        for (int j = 0; j < k; ++j)
            if (j != i) mi = mulmod64(mi, ps[size_t(j)].p % p, p);
        // y_i (M / p_i) N = 2^32 (mod p_i)
        if (mulmod64(mulmod64(c.y[i], mi, p), N % p, p) != (1ull << 32) % p) return at + "y_i (M/p_i) N != 2^32";
        const uint64_t lhs = uint64_t(c.y[i]) << 32, qp = uint64_t(c.ys[i]) * p;
        if (c.y[i] >= p || qp > lhs || lhs - qp >= p) return at + "Shoup companion of y_i";
        Big mq(c.mq + size_t(i) * kMqStride, c.mq + size_t(i) * kMqStride + kMqStride);
        trim(mq);
        if (cmp_big(mq, qb) >= 0) return at + "(M/p_i) mod q is not below q";
        if (!divmod(add_big(mul_u64(mq, p), neg), qb, nullptr).empty()) return at + "(M/p_i mod q) p_i != M mod q";
    }
    Big mu(c.mu, c.mu + 4);
    trim(mu);
    const Big e = pow2(int(c.qbits) + kBarrettT + 1);
    if (cmp_big(mul_big(mu, qb), e) > 0 || cmp_big(add_big(mul_big(mu, qb), qb), e) <= 0) return "Barrett constant mu";
    return std::string();
}

}  // namespace nc
