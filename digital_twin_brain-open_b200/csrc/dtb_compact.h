// Spike compaction operator shared by the C-ABI entry points.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace dtb {

constexpr int kCompactWordsPerTile = 128;                  // 4096 neurons per tile
constexpr uint32_t kCompactTileNeurons = kCompactWordsPerTile * 32;

inline uint32_t compact_tiles(uint32_t n) {
    return (n + kCompactTileNeurons - 1) / kCompactTileNeurons;
}

// Count, scan and write; `tile_scratch` holds compact_tiles(n) words.
cudaError_t compact_launch(const uint32_t* bits, uint32_t n, uint32_t* idx, uint32_t* count, uint32_t* tile_scratch,
                           cudaStream_t s);

}  // namespace dtb
