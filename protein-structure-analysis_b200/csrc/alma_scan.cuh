// Device-wide exclusive prefix sums (three-pass: per-block scan, scan of the
// block totals, add-back).  Used for cell starts and neighbor-row pointers.
#pragma once
#include "alma_block_scan.cuh"
#include "alma_common.cuh"

namespace alma {

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

template <typename T>
__global__ void scan_tiles_kernel(const T *__restrict__ in, int64_t *__restrict__ out, int64_t *__restrict__ tile_sums,
                                  int64_t n) {
    __shared__ int64_t sm[33];
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    int64_t v[SCAN_ITEMS], s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        v[k] = (base + k < n) ? (int64_t)in[base + k] : 0;
        s += v[k];
    }
    int64_t ex;
    const int64_t tot = block_exclusive_scan(s, ex, sm);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        if (base + k < n) out[base + k] = ex;
        ex += v[k];
    }
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

// Single block: exclusive scan of the tile totals in place, total to *grand.
__global__ void scan_tile_sums_kernel(int64_t *__restrict__ sums, int64_t nt, int64_t *__restrict__ grand) {
    __shared__ int64_t sm[33];
    int64_t carry = 0;
    for (int64_t b = 0; b < nt; b += SCAN_THREADS) {
        const int64_t k = b + threadIdx.x;
        const int64_t v = k < nt ? sums[k] : 0;
        int64_t ex;
        const int64_t tot = block_exclusive_scan(v, ex, sm);
        if (k < nt) sums[k] = ex + carry;
        carry += tot;
    }
    if (threadIdx.x == 0) *grand = carry;
}

__global__ void scan_add_kernel(int64_t *__restrict__ out, const int64_t *__restrict__ tile_sums, int64_t n) {
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
    const int64_t add = tile_sums[blockIdx.x];
    for (int k = threadIdx.x; k < SCAN_TILE; k += SCAN_THREADS) {
        const int64_t idx = base + k;
        if (idx < n) out[idx] += add;
    }
}

inline int64_t scan_num_tiles(int64_t n) { return (n + SCAN_TILE - 1) / SCAN_TILE; }

// out[0..n) = exclusive prefix of in; out[n] = total.  tile_sums: scratch of
// scan_num_tiles(n) int64.
template <typename T>
inline void exclusive_scan(const T *in, int64_t *out, int64_t n, int64_t *tile_sums, cudaStream_t st) {
    const int64_t nt = scan_num_tiles(n) > 0 ? scan_num_tiles(n) : 1;
    scan_tiles_kernel<T><<<(unsigned)nt, SCAN_THREADS, 0, st>>>(in, out, tile_sums, n);
    scan_tile_sums_kernel<<<1, SCAN_THREADS, 0, st>>>(tile_sums, nt, out + n);
    scan_add_kernel<<<(unsigned)nt, SCAN_THREADS, 0, st>>>(out, tile_sums, n);
}

}  // namespace alma
