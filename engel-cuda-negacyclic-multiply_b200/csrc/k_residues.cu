// The residue stage on its own, by two engines, for an ablation of the decomposition:
//
//   r[i * N + n] = x_n mod p_i   (canonical, natural order, prime-major; x_n = N x L u32 limbs)
//
// Engine IMAD: the product path's own residue arithmetic (dec_residues: limb times 2^(32 l) mod
// p_i as 32x64-bit carry chains on the integer pipes, 256 coefficients per CTA).
//
// Engine TC_I8: the same sums as an exact INT8 contraction on the fifth-generation tensor cores.
// With x_n = sum_b x_{n,b} 2^(8 b) over its 4 L bytes and w_{i,b} = 2^(8 b) mod p_i split into
// bytes w_{i,b,c} (c < 8),
//
//   x_n = sum_c 2^(8 c) S[n][i,c]  (mod p_i),   S[n][i,c] = sum_b x_{n,b} w_{i,b,c},
//
// and S is a u8 x u8 matrix product (128 coefficients x 128 bytes of K x 8 columns per prime)
// that one CTA issues as four tcgen05.mma kind::i8 (K = 32 each) with its s32 accumulator in
// tensor memory; every S < 128 * 255^2 < 2^23, so the contraction is exact. The epilogue reads
// the eight partial sums of each prime back with tcgen05.ld, forms sum_c 2^(8 c) S_c (< 2^80)
// and reduces it mod p_i. Limits: k <= 32 (8 k accumulator columns <= 256), L <= 32.
//
// Neither engine is on the product path; nc_residues exists to time one against the other on
// the same inputs and to check that they agree bit for bit.
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "handles.h"
#include "hostmath.h"
#include "kernel_registry.h"
#include "negacyclic_b200.h"
#include "crt_tc.cuh"
#include "stages.cuh"

namespace nc {
namespace {

// ------------------------------------------------------------------------------------------
// engine IMAD

template <int LW>
__global__ void __launch_bounds__(kThreads, 2) k_residues_imad(ProductDesc d, Tables t, const uint32_t* x,
                                                              uint64_t* r) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int N = 1 << d.logN;
    const int T = N < kTile ? N : kTile;
    const int L = int(d.L), k = int(d.k);
    const int j0 = int(blockIdx.x) * T;
    uint32_t* s_in = reinterpret_cast<uint32_t*>(smem);
    uint64_t* s_res = reinterpret_cast<uint64_t*>(smem);
    uint64_t* s_pow = reinterpret_cast<uint64_t*>(smem + dec_main_bytes(k));
    uint64_t* s_p = s_pow + size_t(k) * kMaxL;
    load_tile(x, N, L, j0, T, 1, s_in);
    for (int w = threadIdx.x; w < k * kMaxL; w += blockDim.x) s_pow[w] = __ldg(t.pow32 + w);
    for (int w = threadIdx.x; w < k; w += blockDim.x) s_p[w] = __ldg(t.primes + w);
    __syncthreads();
    dec_residues<LW>(s_in, L, k, T, s_pow, s_res);
    __syncthreads();
    for (int w = threadIdx.x; w < k * T; w += blockDim.x) {
        const int i = w / T, j = w - i * T;
        r[size_t(i) * N + j0 + j] = csub(s_res[size_t(i) * T + j], s_p[i]);
    }
}

void* imad_kernel(int LW) {
    switch (LW) {
#define NC_RES(n) \
    case n: return reinterpret_cast<void*>(&k_residues_imad<n>);
        NC_LW_CASES(NC_RES)
#undef NC_RES
        default: return nullptr;
    }
}

// ------------------------------------------------------------------------------------------
// engine TC_I8

constexpr int kTcRows = 128;        // coefficients per CTA: the MMA's M
constexpr int kTcKBytes = 128;      // K in bytes: 4 L <= 128, zero padded
constexpr int kTcMaxGroups = 32;    // primes per CTA (8 accumulator columns each): N <= 256
constexpr int kTcGroupBytes = 1024; // one prime's weights in shared memory: 8 K chunks x 8 rows x 16 B
constexpr uint32_t kTcSpinLimit = 1u << 22;
constexpr size_t kTcSmemMax = size_t(96) << 10;  // >= operands (49 KB) and >= 228 KB / 3 + 1

struct TcArgs {
    const uint32_t* x;     // N x L limbs
    uint64_t* r;           // k x N residues
    const uint4* w;        // weight table, kTcGroupBytes per prime
    const uint64_t* primes;
    uint32_t* status;      // [0] = 1 once a wait gave up
    int N, L, k, groups;   // groups = k rounded up to even (the MMA's N = 8 groups, a multiple of 16)
    uint32_t tmem_cols;    // power of two >= 8 groups
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor of a K-major operand without swizzling (crt_tc.cuh).
using crt_tc_detail::kmajor_desc;

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t it = 0; it < kTcSpinLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void add128(uint64_t& lo, uint64_t& hi, uint64_t add_lo, uint64_t add_hi) {
    const uint64_t s = lo + add_lo;
    hi += add_hi + (s < lo ? 1u : 0u);
    lo = s;
}

// One CTA: 128 coefficients, 4 warps. Shared memory: A (limb bytes) as [row group 16][K chunk 8]
// [8 rows][16 B], B (weight bytes) as [prime][K chunk 8][8 byte planes][16 B], the MMA's mbarrier
// and the tensor-memory address slot.
__global__ void __launch_bounds__(128) k_residues_tc(TcArgs a) {
#if NC_HAS_TCGEN05
    extern __shared__ __align__(16) uint8_t tc_smem[];  // core matrices need 16-byte alignment
    uint8_t* sA = tc_smem;
    uint8_t* sB = tc_smem + kTcRows * kTcKBytes;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sB + size_t(a.groups) * kTcGroupBytes);
    uint32_t* s_taddr = reinterpret_cast<uint32_t*>(bar + 1);
    const int tid = int(threadIdx.x), warp = tid >> 5, lane = tid & 31;
    const int m0 = int(blockIdx.x) * kTcRows;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(s_taddr)),
                     "r"(a.tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // A: chunk q = (row group, K chunk, row); a warp covers 8 rows x 4 chunks, so its 16-byte
    // shared stores fall on distinct banks within each 128-byte wavefront.
    for (int q = tid; q < kTcRows * (kTcKBytes / 16); q += 128) {
        const int rlo = q & 7, kc = (q >> 3) & 7, rg = q >> 6;
        const int m = m0 + rg * 8 + rlo;
        const int l0 = kc * 4;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (m < a.N && l0 < a.L) {
            const uint32_t* src = a.x + size_t(m) * size_t(a.L) + l0;
            if ((a.L & 3) == 0) {
                v = __ldg(reinterpret_cast<const uint4*>(src));
            } else {
                v.x = __ldg(src);
                v.y = l0 + 1 < a.L ? __ldg(src + 1) : 0u;
                v.z = l0 + 2 < a.L ? __ldg(src + 2) : 0u;
                v.w = l0 + 3 < a.L ? __ldg(src + 3) : 0u;
            }
        }
        *reinterpret_cast<uint4*>(sA + rg * 1024 + kc * 128 + rlo * 16) = v;
    }
    // B: the first `groups` primes' weights, already in shared-memory order
    for (int q = tid; q < a.groups * (kTcGroupBytes / 16); q += 128) reinterpret_cast<uint4*>(sB)[q] = __ldg(a.w + q);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic-proxy stores -> MMA reads
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t taddr = *s_taddr;

    if (tid == 0) {
        // kind::i8 instruction descriptor: D s32 (bits 4-5 = 2), A and B u8 and K-major (0),
        // N >> 3 in bits 17-22, M >> 4 in bits 24-28
        const uint32_t idesc = (2u << 4) | (uint32_t(a.groups) << 17) | (uint32_t(kTcRows >> 4) << 24);
        const uint32_t a0 = smem_addr(sA), b0 = smem_addr(sB);
#pragma unroll
        for (int s = 0; s < kTcKBytes / 32; ++s) {
            const uint64_t da = kmajor_desc(a0 + uint32_t(s) * 256u, 128u, 1024u);
            const uint64_t db = kmajor_desc(b0 + uint32_t(s) * 256u, 128u, 1024u);
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(taddr),
                "l"(da), "l"(db), "r"(idesc), "r"(s));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(bar))
                     : "memory");
    }
    const bool ok = mbar_wait(smem_addr(bar), 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (__all_sync(0xffffffffu, ok)) {
        const int m = m0 + warp * 32 + lane;
        const uint32_t lane_base = taddr + (uint32_t(warp * 32) << 16);
        for (int i = 0; i < a.k; ++i) {
            uint32_t s[8];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                : "=r"(s[0]), "=r"(s[1]), "=r"(s[2]), "=r"(s[3]), "=r"(s[4]), "=r"(s[5]), "=r"(s[6]), "=r"(s[7])
                : "r"(lane_base + uint32_t(8 * i)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            // V = sum_c S_c 2^(8 c) < 2^80: bytes 0..5 fit below 2^64, bytes 6 and 7 straddle it
            uint64_t lo = uint64_t(s[0]) + (uint64_t(s[1]) << 8) + (uint64_t(s[2]) << 16) + (uint64_t(s[3]) << 24) +
                          (uint64_t(s[4]) << 32) + (uint64_t(s[5]) << 40);
            uint64_t hi = 0;
            add128(lo, hi, uint64_t(s[6]) << 48, uint64_t(s[6]) >> 16);
            add128(lo, hi, uint64_t(s[7]) << 56, uint64_t(s[7]) >> 8);
            const uint64_t p = __ldg(a.primes + i);
            const uint64_t res = csub(reduce_special(hi, lo, (uint64_t(1) << 62) - p), p);
            if (m < a.N) a.r[size_t(i) * size_t(a.N) + m] = res;
        }
    } else if (lane == 0) {
        atomicExch(a.status, 1u);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(a.tmem_cols) : "memory");
#endif
}

// Per device: the weight table (kMaxPrimes x kTcGroupBytes) and the status word.
struct TcDevice {
    uint4* w = nullptr;
    uint32_t* status = nullptr;
};
std::mutex g_tc_mu;
std::map<int, TcDevice> g_tc;

TcDevice tc_device(int device) {
    std::lock_guard<std::mutex> lock(g_tc_mu);
    auto it = g_tc.find(device);
    if (it != g_tc.end()) return it->second;
    // byte c of 2^(8 b) mod p_i at [i][b / 16][c][b % 16]
    const std::vector<PrimeConst>& ps = prime_set();
    std::vector<uint8_t> host(size_t(kMaxPrimes) * kTcGroupBytes, 0);
    for (int i = 0; i < kMaxPrimes; ++i) {
        const uint64_t p = ps[size_t(i)].p;
        uint64_t w = 1;
        for (int b = 0; b < kTcKBytes; ++b) {
            for (int c = 0; c < 8; ++c)
                host[size_t(i) * kTcGroupBytes + size_t(b / 16) * 128 + size_t(c) * 16 + size_t(b % 16)] =
                    uint8_t(w >> (8 * c));
            w = uint64_t((unsigned __int128)w * 256u % p);
        }
    }
    TcDevice d;
    check(cudaMalloc(&d.w, host.size()), "tensor-core weight table");
    const cudaError_t e = cudaMalloc(&d.status, 16);
    if (e != cudaSuccess) {
        cudaFree(d.w);
        check(e, "tensor-core status word");
    }
    cudaStream_t s = nullptr;
    check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
    cudaError_t c = cudaMemcpyAsync(d.w, host.data(), host.size(), cudaMemcpyHostToDevice, s);
    if (c == cudaSuccess) c = cudaMemsetAsync(d.status, 0, 16, s);
    if (c == cudaSuccess) c = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    check(c, "tensor-core weight upload");
    g_tc[device] = d;
    return d;
}

void residues(const Plan* p, const uint32_t* d_x, uint64_t* d_r, int engine, cudaStream_t stream) {
    if (!p) throw Error(kEInval, "null plan");
    if (!d_x || !d_r) throw Error(kEInval, "null device buffer");
    if ((reinterpret_cast<uintptr_t>(d_x) & 15) != 0 || (reinterpret_cast<uintptr_t>(d_r) & 7) != 0)
        throw Error(kEInval, "x must be 16-byte aligned and r 8-byte aligned");
    int device = -1;
    check(cudaGetDevice(&device), "cudaGetDevice");
    if (device != p->device) throw Error(kEInval, "the plan's device is not the current device");
    const ProductDesc d = p->desc(d_x, d_x, nullptr);
    if (engine == NC_RESIDUES_IMAD) {
        void* fn = imad_kernel(int(d.LW));
        if (!fn) throw Error(kEInval, "no residue kernel for this limb count");
        const int T = p->N < kTile ? p->N : kTile;
        const Tables t = p->tables->view();
        const uint32_t* x = d_x;
        uint64_t* r = d_r;
        ProductDesc dd = d;
        Tables tt = t;
        void* args[] = {&dd, &tt, &x, &r};
        check(cudaLaunchKernel(fn, dim3(unsigned(p->N / T)), dim3(kThreads), args, dec_smem_bytes(p->k), stream),
              "residue launch");
        return;
    }
    if (engine != NC_RESIDUES_TC_I8) throw Error(kEInval, "unknown residue engine");
    if (p->k > kTcMaxGroups) throw Error(kEInval, "the tensor-core engine takes at most 32 primes (q up to ~960 bits)");
    if (!p->tables->tensor_cores) throw Error(kEInval, "the tensor-core engine needs a compute capability 10.0 device");
    const TcDevice dev = tc_device(device);
    TcArgs a{};
    a.x = d_x;
    a.r = d_r;
    a.w = dev.w;
    a.primes = p->tables->view().primes;
    a.status = dev.status;
    a.N = p->N;
    a.L = p->L;
    a.k = p->k;
    a.groups = (p->k + 1) & ~1;
    uint32_t cols = 32;
    while (cols < uint32_t(8 * a.groups)) cols <<= 1;
    a.tmem_cols = cols;
    // Shared memory: operands, mbarrier and address slot; raised so that no more CTAs share an SM
    // than its 512 tensor-memory columns hold (a further CTA would wait inside tcgen05.alloc).
    const int per_sm = int(512 / cols);
    size_t smem = size_t(kTcRows) * kTcKBytes + size_t(a.groups) * kTcGroupBytes + 16;
    const size_t floor_bytes = size_t(233472) / size_t(per_sm + 1) + 1;
    if (smem < floor_bytes) smem = floor_bytes;
    if (smem > kTcSmemMax) throw Error(kEInval, "internal: tensor-core shared memory above its limit");
    void* args[] = {&a};
    check(cudaLaunchKernel(reinterpret_cast<void*>(&k_residues_tc), dim3(unsigned((p->N + kTcRows - 1) / kTcRows)),
                           dim3(128), args, smem, stream),
          "tensor-core residue launch");
}

int residue_status(int* gave_up) {
    int device = -1;
    check(cudaGetDevice(&device), "cudaGetDevice");
    uint32_t v = 0;
    {
        std::lock_guard<std::mutex> lock(g_tc_mu);
        auto it = g_tc.find(device);
        if (it != g_tc.end()) {
            check(cudaMemcpy(&v, it->second.status, 4, cudaMemcpyDeviceToHost), "status read");
            if (v != 0) check(cudaMemset(it->second.status, 0, 4), "status reset");
        }
    }
    if (gave_up) *gave_up = v != 0;
    return NC_OK;
}

}  // namespace

cudaError_t prepare_residues(const PrimeConst* pc, const uint64_t* pow32) {
    cudaError_t e = upload_prime_constants(pc, pow32);
    for (int lw = 2; lw <= kMaxL && e == cudaSuccess; lw += 2)
        e = cudaFuncSetAttribute(imad_kernel(lw), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(dec_smem_bytes(kMaxPrimes)));
    if (e == cudaSuccess)  // room for the operands and for the occupancy-limiting floor (two CTAs per SM)
        e = cudaFuncSetAttribute(reinterpret_cast<void*>(&k_residues_tc), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(kTcSmemMax));
    return e;
}

}  // namespace nc

namespace {
template <class F>
int residue_guard(F&& f) {
    try {
        f();
        nc::set_last_error("");
        return NC_OK;
    } catch (const nc::Error& e) {
        nc::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        nc::set_last_error(e.what());
        return NC_EINVAL;
    }
}
}  // namespace

extern "C" int nc_residues(const nc_plan* plan, const uint32_t* d_x, uint64_t* d_r, int engine, void* stream) {
    return residue_guard([&] {
        if (!plan) throw nc::Error(nc::kEInval, "null plan");
        nc::residues(plan->p, d_x, d_r, engine, static_cast<cudaStream_t>(stream));
    });
}

extern "C" int nc_residues_status(int* gave_up) {
    return residue_guard([&] { nc::residue_status(gave_up); });
}
