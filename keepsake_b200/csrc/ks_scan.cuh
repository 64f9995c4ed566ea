// Exclusive prefix sum of uint32 arrays on the device (block scan + recursive scan of block sums).
#pragma once
#include "ks_internal.h"

namespace ksb
{

constexpr int kScanBlock = 1024;

__global__ void scan_block_kernel(const uint32_t *in, uint32_t n_in, uint32_t *out, uint32_t n_out,
                                  uint32_t *block_sums)
{
    __shared__ uint32_t warp_sums[32];
    uint32_t i = blockIdx.x * kScanBlock + threadIdx.x;
    uint32_t v = i < n_in ? in[i] : 0u;
    uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o)
            x += y;
    }
    if (lane == 31)
        warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t s = warp_sums[lane];
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= (uint32_t)o)
                s += y;
        }
        warp_sums[lane] = s;
    }
    __syncthreads();
    uint32_t base = warp ? warp_sums[warp - 1] : 0u;
    if (i < n_out)
        out[i] = base + x - v;
    if (threadIdx.x == kScanBlock - 1 && block_sums)
        block_sums[blockIdx.x] = base + x;
}

__global__ void scan_add_kernel(uint32_t *out, uint32_t n, const uint32_t *block_offsets)
{
    uint32_t i = blockIdx.x * kScanBlock + threadIdx.x;
    if (i < n)
        out[i] += block_offsets[blockIdx.x];
}

// Scratch for exclusive_scan: one level of block sums per recursion step.
struct ScanScratch
{
    DevBuf<uint32_t> levels[4];
    DevBuf<uint32_t> level_out[4];
};

// out[i] = sum(in[0..i)), for i in [0, n]: out must hold n + 1 entries (out[n] = total).
inline cudaError_t exclusive_scan(const uint32_t *in, uint32_t *out, uint32_t n, ScanScratch &s, cudaStream_t st,
                                  int depth = 0)
{
    if (n == 0) {
        return cudaMemsetAsync(out, 0, sizeof(uint32_t), st);
    }
    // scan n + 1 values so that out[n] holds the total; in[n] is treated as 0
    uint32_t m = n + 1;
    uint32_t blocks = (m + kScanBlock - 1) / kScanBlock;
    if (depth >= 4)
        return cudaErrorInvalidValue;
    if (s.levels[depth].count < blocks) {
        cudaError_t e = s.levels[depth].alloc(blocks);
        if (e != cudaSuccess)
            return e;
        e = s.level_out[depth].alloc(blocks + 1);
        if (e != cudaSuccess)
            return e;
    }
    scan_block_kernel<<<blocks, kScanBlock, 0, st>>>(in, n, out, m, s.levels[depth].ptr);
    if (blocks > 1) {
        cudaError_t e = exclusive_scan(s.levels[depth].ptr, s.level_out[depth].ptr, blocks, s, st, depth + 1);
        if (e != cudaSuccess)
            return e;
        scan_add_kernel<<<blocks, kScanBlock, 0, st>>>(out, m, s.level_out[depth].ptr);
    }
    return cudaGetLastError();
}

} // namespace ksb
