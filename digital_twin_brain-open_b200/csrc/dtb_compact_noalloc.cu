// Spike compaction that allocates nothing.
//
// Some callers of this library cannot allocate device memory at the point where
// they need a compaction:
// * a long-running serving or data-assimilation loop whose device-memory budget is
//   fixed when it starts, so that its admission decisions stay valid;
// * a runtime that embeds the engine and owns all device memory through its own
//   pool, and forbids allocations from libraries.
// For them, dtb_compact_spikes_noalloc runs the same kernels as dtb_compact_spikes
// but takes its scratch -- one count per 4096 neurons -- from a fixed array that is
// compiled into this library, instead of allocating it per call.
//
// Limits and sharing, which a caller must respect:
// * the array holds kNoAllocMaxTiles counts, so n_neurons may be at most
//   kNoAllocMaxNeurons = 2^26 (67,108,864); larger inputs are rejected with
//   DTB_INVALID_PARAMETER before anything is launched;
// * it is a file-scope __device__ array: every GPU that loads the library holds
//   its 64 KiB until the process exits;
// * every call uses the same array and leaves its contents behind.  Each count is
//   written before it is read, so nothing has to be cleared between calls, but two
//   calls whose kernels overlap on the GPU (unordered streams, or host threads that
//   do not order their calls) race on it and produce wrong lists: order them;
// * the first call on each device looks up the array's device address, with that
//   device current, and keeps it for the life of the process; make that first call
//   before any stream capture.  The kept address assumes the device's primary
//   context is never reset: after a cudaDeviceReset the old address is stale, so
//   the library must not be called again in that process.
#include <mutex>

#include "dtb_compact.h"
#include "dtb_engine.h"

namespace dtb {

constexpr uint32_t kNoAllocMaxTiles = 16384;                                 // 64 KiB of counts
constexpr uint32_t kNoAllocMaxNeurons = kNoAllocMaxTiles * kCompactTileNeurons;  // 2^26
constexpr int kNoAllocMaxDevices = 64;

// The scratch.  In host code this name is only a stand-in for the symbol, not a
// device address; the address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) uint32_t g_noalloc_tile_counts[kNoAllocMaxTiles];

namespace {
std::mutex g_noalloc_mu;
uint32_t* g_noalloc_ptr[kNoAllocMaxDevices] = {};
}  // namespace

// Device address of the scratch on the current device (looked up once per device).
static int noalloc_scratch(uint32_t** out) {
    int dev = 0;
    DTB_CU(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(DTB_UNSUPPORTED, "device index beyond the scratch table");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_tile_counts);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_tile_counts)");
        g_noalloc_ptr[dev] = static_cast<uint32_t*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return DTB_OK;
}

}  // namespace dtb

extern "C" int32_t dtb_compact_spikes_noalloc(const uint32_t* d_bits, uint32_t n_neurons, uint32_t* d_indices,
                                              uint32_t* d_count, void* stream) {
    if (!d_count || (n_neurons && (!d_bits || !d_indices))) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    if (n_neurons > dtb::kNoAllocMaxNeurons)
        return dtb::fail(DTB_INVALID_PARAMETER, "dtb_compact_spikes_noalloc: n_neurons " + std::to_string(n_neurons) +
                                                    " exceeds the fixed scratch limit of " +
                                                    std::to_string(dtb::kNoAllocMaxNeurons) +
                                                    " neurons; use dtb_compact_spikes");
    uint32_t* scratch = nullptr;
    const int st = dtb::noalloc_scratch(&scratch);
    if (st != DTB_OK) return st;
    const cudaError_t e = dtb::compact_launch(d_bits, n_neurons, d_indices, d_count, scratch,
                                              static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return dtb::cuda_fail(e, "dtb_compact_spikes_noalloc");
    return DTB_OK;
}
