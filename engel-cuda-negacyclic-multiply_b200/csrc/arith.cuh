// Device arithmetic for 62-bit primes p = 2^62 - m (m < 2^28) and multi-limb carry chains.
//
// Counterparts in the reference: shoup_mul (solve.cu:151-156), mont_mul (solve.cu:134-148),
// reduce_128 (solve.cu:200-237) and the 34-limb accum_factor (solve.cu:644-660). The forms here
// differ: butterflies keep values lazily reduced (Harvey's [0, 2p) / [0, 4p) ranges, valid
// because p < 2^62), the pointwise product and the residue reduction use the special shape of
// p instead of Montgomery or a 128-bit reciprocal, and limb products run as PTX carry chains.
#pragma once

#include <cstdint>

#include "common.h"

namespace nc {

constexpr uint64_t kMask62 = (1ull << 62) - 1;

__device__ __forceinline__ uint64_t csub(uint64_t x, uint64_t m) { return x >= m ? x - m : x; }

// Programmatic dependent launch. A product kernel launched with it may be scheduled while the
// kernel before it on the stream still runs (once every CTA of that kernel has called
// pdl_trigger(): on entry, or, in kernels that allocate tensor memory, once the CTA holds it), so
// its prologue (tensor-memory allocation, constant tables) overlaps that kernel's last wave.
// pdl_wait() returns once the kernel before has completed and its writes are visible; every read
// or write of data that kernel produces or consumes comes after it. In a kernel launched without
// the attribute, both return at once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// y * w mod p in [0, 2p) for any y < 2^64 and w < p, with wq = floor(w * 2^64 / p).
__device__ __forceinline__ uint64_t shoup_lazy(uint64_t y, uint64_t w, uint64_t wq, uint64_t p) {
    const uint64_t q = __umul64hi(y, wq);
    return y * w - q * p;
}

// Forward Cooley-Tukey butterfly (x, y) -> (x + w y, x - w y); inputs and outputs in [0, 4p).
__device__ __forceinline__ void ct_bfly(uint64_t& x, uint64_t& y, uint64_t w, uint64_t wq, uint64_t p,
                                        uint64_t p2) {
    const uint64_t u = csub(x, p2);
    const uint64_t t = shoup_lazy(y, w, wq, p);
    x = u + t;
    y = u - t + p2;
}

// Inverse Gentleman-Sande butterfly (x, y) -> (x + y, (x - y) w); inputs and outputs in [0, 2p).
__device__ __forceinline__ void gs_bfly(uint64_t& x, uint64_t& y, uint64_t w, uint64_t wq, uint64_t p,
                                        uint64_t p2) {
    const uint64_t s = csub(x + y, p2);
    const uint64_t d = x - y + p2;
    x = s;
    y = shoup_lazy(d, w, wq, p);
}

// Reduce hi:lo (< 2^126) modulo p = 2^62 - m into [0, 2p).
__device__ __forceinline__ uint64_t reduce_special(uint64_t hi, uint64_t lo, uint64_t m) {
    // T = h * 2^62 + l = h * m + l (mod p), h < 2^64
    const uint64_t h = (hi << 2) | (lo >> 62);
    const uint64_t l = lo & kMask62;
    const uint32_t h0 = static_cast<uint32_t>(h), h1 = static_cast<uint32_t>(h >> 32);
    const uint32_t m0 = static_cast<uint32_t>(m);
    const uint64_t p0 = static_cast<uint64_t>(h0) * m0;  // < 2^60
    const uint64_t p1 = static_cast<uint64_t>(h1) * m0;  // < 2^60
    // T' = p0 + p1 * 2^32 + l < 2^93
    uint64_t t_lo = p0 + (p1 << 32);
    uint64_t t_hi = (p1 >> 32) + (t_lo < p0 ? 1u : 0u);
    const uint64_t t2 = t_lo + l;
    t_hi += t2 < l ? 1u : 0u;
    t_lo = t2;
    const uint64_t h2 = (t_hi << 2) | (t_lo >> 62);  // < 2^31
    return static_cast<uint64_t>(static_cast<uint32_t>(h2)) * m0 + (t_lo & kMask62);  // < 2^62 + 2^59
}

// S = (a2:a1:a0) + (b2:b1:b0) * 2^32 (< 2^99, a limb-by-constant sum) reduced mod p into [0, 2p).
__device__ __forceinline__ uint64_t reduce_limb_sum(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t b0, uint32_t b1,
                                                    uint32_t b2, uint64_t m) {
    const uint64_t lo_a = (uint64_t(a1) << 32) | a0;
    const uint64_t lo = lo_a + (uint64_t(b0) << 32);
    const uint64_t hi = uint64_t(a2) + b1 + (uint64_t(b2) << 32) + (lo < lo_a ? 1u : 0u);
    return reduce_special(hi, lo, m);
}

// y * z mod p in [0, 2p) for y < 2^62 and z < 2^64 (pointwise product of two transforms).
__device__ __forceinline__ uint64_t mulmod_special(uint64_t y, uint64_t z, uint64_t m) {
    return reduce_special(__umul64hi(y, z), y * z, m);
}

// 32-bit carry-chain helpers (PTX add/mad with carry flags).
__device__ __forceinline__ void mac_u32x64(uint32_t x, uint32_t c0, uint32_t c1, uint32_t& a0, uint32_t& a1,
                                           uint32_t& a2, uint32_t& b0, uint32_t& b1, uint32_t& b2) {
    // (a2:a1:a0) += x * c0 ; (b2:b1:b0) += x * c1   (the b words sit one limb higher)
    asm("mad.lo.cc.u32 %0, %3, %4, %0;\n\t"
        "madc.hi.cc.u32 %1, %3, %4, %1;\n\t"
        "addc.u32 %2, %2, 0;"
        : "+r"(a0), "+r"(a1), "+r"(a2)
        : "r"(x), "r"(c0));
    asm("mad.lo.cc.u32 %0, %3, %4, %0;\n\t"
        "madc.hi.cc.u32 %1, %3, %4, %1;\n\t"
        "addc.u32 %2, %2, 0;"
        : "+r"(b0), "+r"(b1), "+r"(b2)
        : "r"(x), "r"(c1));
}

}  // namespace nc
