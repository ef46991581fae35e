// nc_multiply_device_noalloc: the device-resident product for callers that must not allocate
// device memory when they call it.
//
// Who needs it: code whose device memory is owned by another framework's pool allocator (which
// forbids cudaMalloc behind its back), latency-critical loops where cudaMalloc's implicit
// device-wide synchronisation is unacceptable, and services that allocate only at start-up and
// never again. nc_multiply_device already allocates nothing per call, but it needs the plan's
// own residue scratch (2 * k * N u64, 30 MB at N = 65536), allocated by nc_plan_create; this
// variant instead takes its residue scratch from one fixed array compiled into the library.
//
// The array: kStaticResidueWords u64 (8 MiB) of file-scope __device__ memory. Every GPU that
// loads this library holds it until the process exits. One product needs 2 * k * N words, so the
// limit is k * N <= 2^19: N <= 16384 at an 868-bit q (k = 29), N <= 32768 at a 434-bit q
// (k = 15). Larger products are rejected with NC_EINVAL.
//
// Sharing: every call, from every plan and every stream, uses the same array and it keeps the
// last call's contents. Nothing in it needs to start at zero (each stage writes every residue
// before the next stage reads it), but calls that overlap on the GPU race on it: order them on
// one stream or synchronise between them.
//
// Set-up: host code cannot use the array's name as a device address. When the library first
// sets a device up (the first plan created on it uploads the device tables, with that device
// current), prepare_noalloc looks the array's address up with cudaGetSymbolAddress, checks the
// result and keeps it. That lookup is also what loads this file's module, and with it the array,
// onto the device under CUDA's lazy module loading: so the allocation happens at plan creation,
// and a call of the entry point never allocates or loads anything, not even its first.
#include <cuda_runtime.h>

#include <map>
#include <mutex>

#include "handles.h"
#include "kernels.h"
#include "negacyclic_b200.h"

namespace nc {
namespace {

constexpr size_t kStaticResidueWords = size_t(1) << 20;  // two operands of k * N <= 2^19 residues

__device__ __align__(256) uint64_t g_static_residues[kStaticResidueWords];

std::mutex g_addr_mu;
std::map<int, uint64_t*> g_addr;  // device -> device address of g_static_residues

uint64_t* static_residues(int device) {
    std::lock_guard<std::mutex> lock(g_addr_mu);
    auto it = g_addr.find(device);
    if (it == g_addr.end())
        throw Error(kEInval, "the allocation-free scratch was not set up on this device (create a plan on it first)");
    return it->second;
}

void multiply_noalloc(const Plan* p, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, cudaStream_t stream) {
    if (!p) throw Error(kEInval, "null plan");
    if (!d_a || !d_b || !d_c) throw Error(kEInval, "null device buffer");
    if (((reinterpret_cast<uintptr_t>(d_a) | reinterpret_cast<uintptr_t>(d_b) | reinterpret_cast<uintptr_t>(d_c)) &
         15) != 0)
        throw Error(kEInval, "device buffers must be 16-byte aligned");
    const size_t words = size_t(p->k) * size_t(p->N);
    if (2 * words > kStaticResidueWords)
        throw Error(kEInval, "k * N = " + std::to_string(words) +
                                 " residues exceeds the static scratch limit of 524288 (k * N <= 2^19: N <= 16384 "
                                 "at an 868-bit q); use nc_multiply_device");
    int device = -1;
    check(cudaGetDevice(&device), "cudaGetDevice");
    if (device != p->device) throw Error(kEInval, "the plan's device is not the current device");
    uint64_t* scratch = static_residues(device);
    ProductDesc d = p->desc(d_a, d_b, d_c);
    d.ra = scratch;
    d.rb = scratch + words;
    check(launch_product(d, p->tables->view(), p->cfg, stream), "kernel launch");
}

}  // namespace

cudaError_t prepare_noalloc(int device) {
    std::lock_guard<std::mutex> lock(g_addr_mu);
    if (g_addr.count(device)) return cudaSuccess;
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_residues);
    if (e != cudaSuccess) return e;
    g_addr[device] = static_cast<uint64_t*>(ptr);
    return cudaSuccess;
}

}  // namespace nc

extern "C" int nc_multiply_device_noalloc(const nc_plan* plan, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c,
                                          void* stream) {
    try {
        if (!plan) throw nc::Error(nc::kEInval, "null plan");
        nc::multiply_noalloc(plan->p, d_a, d_b, d_c, static_cast<cudaStream_t>(stream));
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
