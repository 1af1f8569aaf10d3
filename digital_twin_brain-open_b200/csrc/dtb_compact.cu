// Standalone spike compaction: a spike bitmap on the device (bit i of word i/32 =
// neuron i) becomes the ascending list of spiking neuron indices plus its length.
// This is the compaction stage of the reference's sending path
// (src/stage/spike.cpp:244-762: expand+reduce, segmented reduce, scans, scan and
// select) as one deterministic operator: three short kernels over 4096-neuron
// tiles -- per-tile popcounts, one exclusive scan over the tiles, and an ordered
// write of each tile's set bits.  Its scratch is one count per tile.
#include <algorithm>

#include "dtb_compact.h"
#include "dtb_engine.h"

namespace dtb {

// Per-tile popcounts: CTA t counts the set bits of words [128 t, 128 t + 128).
__global__ void __launch_bounds__(kCompactWordsPerTile)
compact_count_kernel(const uint32_t* __restrict__ bits, uint32_t n, uint32_t* __restrict__ tile_counts) {
    const uint32_t w = blockIdx.x * kCompactWordsPerTile + threadIdx.x;
    const uint32_t n_words = (n + 31) / 32;
    uint32_t x = 0;
    if (w < n_words) {
        x = __ldg(bits + w);
        if (w == n_words - 1 && (n & 31u)) x &= (1u << (n & 31u)) - 1u;
    }
    uint32_t c = __reduce_add_sync(0xffffffffu, static_cast<uint32_t>(__popc(x)));
    __shared__ uint32_t s[kCompactWordsPerTile / 32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int i = 0; i < kCompactWordsPerTile / 32; ++i) t += s[i];
        tile_counts[blockIdx.x] = t;
    }
}

// Exclusive scan of the tile counts in place (one CTA); the total goes to *count.
__global__ void __launch_bounds__(1024)
compact_scan_kernel(uint32_t* __restrict__ tile_counts, uint32_t n_tiles, uint32_t* __restrict__ count) {
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t base = 0; base < n_tiles; base += 1024) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < n_tiles ? tile_counts[i] : 0u;
        uint32_t incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = s_warp[lane];
            uint32_t wi = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += y;
            }
            s_warp[lane] = wi - w;
        }
        __syncthreads();
        const uint32_t carry = s_carry;
        if (i < n_tiles) tile_counts[i] = carry + s_warp[warp] + incl - v;
        __syncthreads();
        if (threadIdx.x == 1023) s_carry = carry + s_warp[31] + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) *count = s_carry;
}

// Ordered write: each tile writes the indices of its set bits, ascending, at its offset.
__global__ void __launch_bounds__(kCompactWordsPerTile)
compact_write_kernel(const uint32_t* __restrict__ bits, uint32_t n, const uint32_t* __restrict__ tile_offsets,
                     uint32_t* __restrict__ idx) {
    const uint32_t w = blockIdx.x * kCompactWordsPerTile + threadIdx.x;
    const uint32_t n_words = (n + 31) / 32;
    uint32_t x = 0;
    if (w < n_words) {
        x = __ldg(bits + w);
        if (w == n_words - 1 && (n & 31u)) x &= (1u << (n & 31u)) - 1u;
    }
    const uint32_t c = __popc(x);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    __shared__ uint32_t s_warp[kCompactWordsPerTile / 32];
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int i = 0; i < kCompactWordsPerTile / 32; ++i) { const uint32_t v = s_warp[i]; s_warp[i] = t; t += v; }
    }
    __syncthreads();
    uint32_t pos = __ldg(tile_offsets + blockIdx.x) + s_warp[warp] + incl - c;
    while (x) {
        const int b = __ffs(x) - 1;
        idx[pos++] = w * 32 + static_cast<uint32_t>(b);
        x &= x - 1;
    }
}

cudaError_t compact_launch(const uint32_t* bits, uint32_t n, uint32_t* idx, uint32_t* count, uint32_t* tile_scratch,
                           cudaStream_t s) {
    const uint32_t tiles = compact_tiles(n);
    if (tiles == 0) {
        return cudaMemsetAsync(count, 0, sizeof(uint32_t), s);
    }
    compact_count_kernel<<<tiles, kCompactWordsPerTile, 0, s>>>(bits, n, tile_scratch);
    compact_scan_kernel<<<1, 1024, 0, s>>>(tile_scratch, tiles, count);
    compact_write_kernel<<<tiles, kCompactWordsPerTile, 0, s>>>(bits, n, tile_scratch, idx);
    return cudaGetLastError();
}

}  // namespace dtb

extern "C" int32_t dtb_compact_spikes(const uint32_t* d_bits, uint32_t n_neurons, uint32_t* d_indices,
                                      uint32_t* d_count, void* stream) {
    if (!d_count || (n_neurons && (!d_bits || !d_indices))) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    if (n_neurons > dtb::kCompactMaxNeurons)
        return dtb::fail(DTB_INVALID_PARAMETER, "dtb_compact_spikes: n_neurons " + std::to_string(n_neurons) +
                                                    " exceeds the limit of " + std::to_string(dtb::kCompactMaxNeurons));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint32_t tiles = dtb::compact_tiles(n_neurons);
    uint32_t* scratch = nullptr;
    if (tiles) DTB_CU(cudaMallocAsync(reinterpret_cast<void**>(&scratch), sizeof(uint32_t) * tiles, s));
    const cudaError_t e = dtb::compact_launch(d_bits, n_neurons, d_indices, d_count, scratch, s);
    if (scratch) cudaFreeAsync(scratch, s);
    if (e != cudaSuccess) return dtb::cuda_fail(e, "dtb_compact_spikes");
    return DTB_OK;
}
