// Spike compaction operator shared by the C-ABI entry points.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace dtb {

constexpr int kCompactWordsPerTile = 128;                  // 4096 neurons per tile
constexpr uint32_t kCompactTileNeurons = kCompactWordsPerTile * 32;
// Largest bitmap the operator takes: the last tile boundary below 2^32, so the tile
// count, the word count (n + 31) / 32 and every neuron index stay in 32 bits.
constexpr uint32_t kCompactMaxNeurons = 0xFFFFFFFFu / kCompactTileNeurons * kCompactTileNeurons;

inline uint32_t compact_tiles(uint32_t n) {
    return static_cast<uint32_t>((static_cast<uint64_t>(n) + kCompactTileNeurons - 1) / kCompactTileNeurons);
}

// Count, scan and write; `tile_scratch` holds compact_tiles(n) words.
cudaError_t compact_launch(const uint32_t* bits, uint32_t n, uint32_t* idx, uint32_t* count, uint32_t* tile_scratch,
                           cudaStream_t s);

}  // namespace dtb
