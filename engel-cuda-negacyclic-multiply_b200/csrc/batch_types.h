// Plain-old-data shared by the persistent kernel and its host side.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "common.h"

namespace nc {

enum : uint32_t { kItemDec = 0, kItemRow = 1, kItemCrt = 2 };

// Row items of the persistent launch: radix 8 on the launch's 256-thread CTAs, row blocks of at
// most 2^11 residues (one block per CTA at 2^11). Radix 16 on blocks of 2^12 took ~60% longer per
// row at N = 2^16 and needs twice the registers for its sixteen values.
constexpr int kBatchRowLogE = 3;
constexpr int kBatchRowLogMax = 11;
inline RowConfig batch_row_config(int logN) {
    RowConfig c{};
    c.logN2 = logN < kBatchRowLogMax ? logN : kBatchRowLogMax;
    c.logE = kBatchRowLogE;
    c.threads = kThreads;
    return c;
}

// One product of a batch with the item counts its dependents wait for.
struct BatchProduct {
    ProductDesc d;
    uint32_t n_dec;          // residue items of this product
    uint32_t n_row;          // row items
    uint32_t tiles;          // residue tiles per operand
    uint32_t first_operand;  // 1 when a is given in the NTT domain (only b is decomposed)
    uint32_t tiles_tc;       // 128-coefficient tiles per operand (residues on the tensor cores)
    uint32_t pad;
};

struct BatchArgs {
    const BatchProduct* products;
    const uint2* items;  // x = stage << 28 | product, y = index inside the stage (residue and row items)
    int n_items;
    uint32_t* counters;  // per product: residue items done, row items done
    uint32_t* head;      // next queue position
    uint32_t* error;     // [0] nonzero once a wait gave up; [1..3] what it waited for
    Tables tables;
};

// The launches of a batch outside the persistent one, one CTA per item: CRT (x = product, y =
// 256-coefficient tile) and tensor-core residues (x = product, y = operand * tiles_tc + tile).
struct BatchCrtArgs {
    const BatchProduct* products;
    const uint2* items;
    int n_items;
    Tables tables;
};

}  // namespace nc
