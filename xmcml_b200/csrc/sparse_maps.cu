// Sparse read-back of the detector trajectory maps.
//
// LaunchOMP's OutputInfo carries one grid-sized u64 counter map per detector
// (base/xmcml/xmcmlLauncher/launcher_omp.cpp:10-58, filled by UpdateDetectorTrajectory,
// base/xmcml/xmcml/mcml_kernel.cpp:794-810); most of their cells stay zero (a detector's photons cross
// the planes of a cone under it). Instead of copying every map, the device lists the non-zero cells
// of all maps as (cell, count) pairs grouped by map: a count pass per block of 4,096 cells, an
// exclusive scan of the block counts (CUB), and a write pass that puts each block's non-zero cells at
// its offset. The host then adds the pairs into the caller's maps.
#include <cub/cub.cuh>

#include "xmc_internal.h"

namespace xmc {
namespace {

constexpr int kNzThreads = 256;
constexpr int kNzPerThread = 16;
constexpr int kNzCells = kNzThreads * kNzPerThread;  // cells per block

// Non-zero cells of one block of 4,096 cells: launch block b is block b % blocks_per_map of map
// b / blocks_per_map (a 1-D grid, so the number of maps is not bound by the grid's y extent); thread t
// reads cells t, t + 256, ...
__global__ void __launch_bounds__(kNzThreads) nz_count_kernel(const unsigned long long* __restrict__ maps,
                                                              unsigned long long cells, unsigned blocks_per_map,
                                                              unsigned long long* __restrict__ counts) {
    using BlockReduce = cub::BlockReduce<unsigned, kNzThreads>;
    __shared__ typename BlockReduce::TempStorage tmp;
    const unsigned map = blockIdx.x / blocks_per_map, blk = blockIdx.x % blocks_per_map;
    const unsigned long long base = (unsigned long long)blk * kNzCells;
    const unsigned long long* m = maps + (unsigned long long)map * cells;
    unsigned cnt = 0;
#pragma unroll
    for (int j = 0; j < kNzPerThread; ++j) {
        const unsigned long long cell = base + (unsigned long long)j * kNzThreads + threadIdx.x;
        if (cell < cells && m[cell]) ++cnt;
    }
    const unsigned total = BlockReduce(tmp).Sum(cnt);
    if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

// The same cells again: each thread writes its non-zero cells at the block's offset plus the count of
// the lower threads' non-zero cells.
__global__ void __launch_bounds__(kNzThreads) nz_write_kernel(const unsigned long long* __restrict__ maps,
                                                              unsigned long long cells, unsigned blocks_per_map,
                                                              const unsigned long long* __restrict__ offsets,
                                                              unsigned* __restrict__ idx,
                                                              unsigned long long* __restrict__ val) {
    using BlockScan = cub::BlockScan<unsigned, kNzThreads>;
    __shared__ typename BlockScan::TempStorage tmp;
    const unsigned map = blockIdx.x / blocks_per_map, blk = blockIdx.x % blocks_per_map;
    const unsigned long long base = (unsigned long long)blk * kNzCells;
    const unsigned long long* m = maps + (unsigned long long)map * cells;
    unsigned long long v[kNzPerThread];
    unsigned cnt = 0;
#pragma unroll
    for (int j = 0; j < kNzPerThread; ++j) {
        const unsigned long long cell = base + (unsigned long long)j * kNzThreads + threadIdx.x;
        v[j] = cell < cells ? m[cell] : 0ull;
        cnt += v[j] != 0ull;
    }
    unsigned before = 0;
    BlockScan(tmp).ExclusiveSum(cnt, before);
    unsigned long long o = offsets[blockIdx.x] + before;
#pragma unroll
    for (int j = 0; j < kNzPerThread; ++j) {
        if (v[j]) {
            idx[o] = (unsigned)(base + (unsigned long long)j * kNzThreads + threadIdx.x);
            val[o] = v[j];
            ++o;
        }
    }
}

}  // namespace

unsigned sparse_blocks_per_map(size_t cells) { return (unsigned)((cells + kNzCells - 1) / kNzCells); }

cudaError_t sparse_maps_count(const unsigned long long* maps, size_t cells, int n_maps, unsigned long long* counts,
                              unsigned long long* offsets, void** scan_tmp, size_t* scan_tmp_bytes, cudaStream_t st) {
    const unsigned bpm = sparse_blocks_per_map(cells);
    const size_t n = (size_t)bpm * n_maps;
    if (n == 0) return cudaSuccess;
    if (n > 0x7fffffffu) return cudaErrorInvalidValue;  // the 1-D grid's limit (beyond any map memory)
    nz_count_kernel<<<(unsigned)n, kNzThreads, 0, st>>>(maps, cells, bpm, counts);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    size_t need = 0;
    e = cub::DeviceScan::ExclusiveSum(nullptr, need, counts, offsets, (int)n, st);
    if (e != cudaSuccess) return e;
    if (need > *scan_tmp_bytes) {
        if (*scan_tmp) cudaFree(*scan_tmp);
        *scan_tmp = nullptr;
        *scan_tmp_bytes = 0;
        e = cudaMalloc(scan_tmp, need);
        if (e != cudaSuccess) return e;
        *scan_tmp_bytes = need;
    }
    return cub::DeviceScan::ExclusiveSum(*scan_tmp, need, counts, offsets, (int)n, st);
}

cudaError_t sparse_maps_write(const unsigned long long* maps, size_t cells, int n_maps, const unsigned long long* offsets,
                              unsigned* idx, unsigned long long* val, cudaStream_t st) {
    const unsigned bpm = sparse_blocks_per_map(cells);
    const size_t n = (size_t)bpm * n_maps;
    if (n == 0) return cudaSuccess;
    if (n > 0x7fffffffu) return cudaErrorInvalidValue;
    nz_write_kernel<<<(unsigned)n, kNzThreads, 0, st>>>(maps, cells, bpm, offsets, idx, val);
    return cudaGetLastError();
}

}  // namespace xmc
