// Host-side launch interface of the per-step kernels and the device network builder.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "dtb_device.cuh"

namespace dtb {

// One launch group: a batch of networks advanced together.
struct LaunchBatch {
    const NetView* nets;          // device array [n_nets]
    const uint32_t* lif_prefix;   // device [n_nets + 1] cumulative LIF tiles (1024 neurons)
    const uint32_t* tile_net;     // device [lif tiles] network of every LIF tile (batches), or null
    const uint32_t* pull_prefix;  // device [n_nets + 1] cumulative pull tiles (256 neurons)
    const uint32_t* vbase;        // device [n_nets + 1] cumulative padded neuron counts
    uint32_t n_nets;
    uint32_t lif_tiles_total;
    uint32_t pull_tiles_total;
    uint32_t push_ctas;
    uint32_t lif_ctas;            // persistent grid of the LIF kernel
    uint32_t lif_chunk;           // consecutive tiles a LIF CTA steps before striding (0 or 1: one)
    const uint32_t* win_prefix;   // device [n_nets + 1] cumulative local-push windows
    uint32_t windows_total;
    uint32_t* local_scratch;      // device [2 * windows_total + 3]: rows per window, unit prefix, unit counter, ticket
    uint32_t sm_count;
    cudaStream_t aux;             // second stream of the concurrent local push (fork/join by events)
    cudaEvent_t ev_fork, ev_join;
    SpikeList spikes;
};

cudaError_t launch_lif(const LaunchBatch& b, int jmode, uint32_t flags, int prop_mode, cudaStream_t s);
// Push kernel variants chosen by the autotuner.
enum PushKind : int { PUSH_REG = 0, PUSH_TMA = 1, PUSH_LOCAL = 2 };
struct PushCfg {
    int kind;    // PUSH_REG: register-staged loads, param = synapses in flight per lane (4, 8, 16)
                 // PUSH_TMA: bulk-copy staged rows, param = synapses per stage (256, 512)
                 // PUSH_LOCAL: own-population synapses summed per window in shared memory,
                 //   the rest register-staged (param = synapses in flight per lane, 8)
    int param;
    int lpr = 32;  // PUSH_REG: lanes per row (32, 16, 8; sub-warp rows use 8 in flight per lane)
};

// Every variant the autotuner times.
constexpr int kPushCandidates = 12;
constexpr int kLocalConcurrent = 2008;   // PUSH_LOCAL param: cross-population part on a second stream
constexpr int kLocalConcurrent2 = 2016;  // ... with two push CTAs per SM beside a 512-thread window CTA
constexpr int kLocalConcurrentHalf = 3008;  // ... as 2008 with half-warp rows in the window kernel (short spans)
extern const PushCfg kPushCands[kPushCandidates];
// Sets kernel attributes and returns the persistent grid (max resident CTAs).
// `acc` is the AccMode of the launch (float, exact or fixed-point accumulators).
cudaError_t push_prepare(int acc, int weight_type, const PushCfg& cfg, int sm_count, uint32_t* ctas);
cudaError_t launch_push(const LaunchBatch& b, int acc, int weight_type, const PushCfg& cfg, uint32_t ctas,
                        cudaStream_t s);
// Kernels launch_push issues beyond the first (the local variant's prep and window passes).
inline uint32_t push_extra_launches(const LaunchBatch& b, int acc, const PushCfg& cfg) {
    return (cfg.kind == PUSH_LOCAL && acc != ACC_EXACT && b.windows_total) ? 2u : 0u;   // concurrent form: same count
}
cudaError_t launch_pull(const LaunchBatch& b, int gather, int weight_type, uint32_t flags, int prop_mode, cudaStream_t s);
cudaError_t launch_fold_finish(const LaunchBatch& b, int acc, cudaStream_t s);
// Per-population sums of the end-of-step synaptic currents (after the push of
// the step; with exact or fixed accumulators J still lacks the step's sums).
cudaError_t launch_stat_isyn(const LaunchBatch& b, int acc, int sm_count, cudaStream_t s);
cudaError_t launch_gather_finish(const LaunchBatch& b, int weight_type, cudaStream_t s);

// Population-local push tables (rows must be sorted by postsynaptic neuron;
// *unsorted is set otherwise).  Pass 1 (woff == nullptr): per-neuron own-
// population in-degree into own_cnt, per-population max |w| (float bits) into
// maxw_bits; pass 2: own_seg and woff from pop_loc.
cudaError_t build_local_offsets(const unsigned long long* out_ptr, const uint32_t* out_col, const void* out_w, int wt,
                                const uint32_t* pop_off, uint32_t n_pops, uint32_t n, const uint4* pop_loc,
                                uint32_t* own_cnt, uint32_t* maxw_bits, uint2* own_seg, uint32_t* woff,
                                uint32_t* unsorted, cudaStream_t s);

// ---- device network generator (dtb_generate.cu)
struct GenSpec {
    uint32_t n, n_pops, in_degree, dyadic;
    unsigned long long seed;
    const uint32_t* pop_off;          // device [n_pops + 1]
    const uint32_t* pop_exc;          // device [n_pops]
    const unsigned long long* cdf;    // device [n_pops * n_pops]
};

// Builds the requested CSRs on the device.  out_* / in_* may be null when not
// wanted.  Temporary device memory is allocated and released inside.
cudaError_t build_structured(const GenSpec& g, int weight_type,
                             unsigned long long* out_ptr, uint32_t* out_col, void* out_w,
                             unsigned long long* in_ptr, uint32_t* in_col, void* in_w,
                             uint32_t* out_deg, cudaStream_t s);

// Host mirror of one generated edge (used by the host builder for small networks
// and by the tests through the oracle).
void host_gen_edge(uint32_t n_pops, const uint32_t* pop_off, const uint32_t* pop_exc,
                   const unsigned long long* cdf, unsigned long long seed, uint32_t dyadic,
                   uint32_t post, uint32_t pop_of_post, uint32_t k,
                   uint32_t* pre, uint32_t* kind, float* w0, float* w1);

}  // namespace dtb
