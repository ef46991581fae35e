// Host-side bulk copy of the host path and the server (staging into pinned memory, copy-out).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>
#if defined(__x86_64__)
#include <emmintrin.h>
#endif

namespace nc {

// Copy with non-temporal stores (plain memcpy when dst is not 16-byte aligned). They skip the
// read-for-ownership of the destination and leave no dirty lines in the CPU caches for a DMA to
// snoop: measured on the B200 host, staging into pinned memory went from about 40 to 64-90 GB/s
// over 8 threads and the overlapping H2D copies from about 34 to 45 GB/s; the copy-out of the
// product into the caller's buffer gained a little too.
inline void stage_copy(char* dst, const char* src, size_t n) {
#if defined(__x86_64__)
    if ((reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
        size_t i = 0;
        for (; i + 64 <= n; i += 64) {
            const __m128i x0 = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + i));
            const __m128i x1 = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + i + 16));
            const __m128i x2 = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + i + 32));
            const __m128i x3 = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + i + 48));
            _mm_stream_si128(reinterpret_cast<__m128i*>(dst + i), x0);
            _mm_stream_si128(reinterpret_cast<__m128i*>(dst + i + 16), x1);
            _mm_stream_si128(reinterpret_cast<__m128i*>(dst + i + 32), x2);
            _mm_stream_si128(reinterpret_cast<__m128i*>(dst + i + 48), x3);
        }
        if (i < n) std::memcpy(dst + i, src + i, n - i);
        _mm_sfence();  // the stores are visible before this thread reports its part done
        return;
    }
#endif
    std::memcpy(dst, src, n);
}

}  // namespace nc
