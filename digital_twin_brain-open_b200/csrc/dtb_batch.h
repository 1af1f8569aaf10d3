// The batched form: several engines advanced by one launch of each per-step kernel.
#pragma once

#include <map>
#include <vector>

#include "dtb_engine.h"

namespace dtb {

class Batch {
public:
    ~Batch();
    int create(Engine* const* engines, uint32_t n);
    int set_members(Engine* const* engines, uint32_t n);
    int run(const dtb_run_request& rq, dtb_run_output* outs);
    int refresh_views();

    std::vector<Engine*> m;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, tev[2] = {nullptr, nullptr};
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int sm_count = 148;
    uint32_t wtype = W_F32;
    NetView* d_views = nullptr;
    uint32_t* d_prefix = nullptr;     // [lif n+1][pull n+1][vbase n+1][local windows n+1]
    uint32_t* list = nullptr;
    uint32_t* list_count = nullptr;
    uint32_t* list_ticket = nullptr;
    uint32_t cap_members = 0;         // capacity of d_views / d_prefix
    uint64_t cap_neurons = 0;         // capacity of the spike list
    uint32_t* local_scratch = nullptr;
    uint32_t* tile_net = nullptr;     // network of every LIF tile
    uint32_t cap_tiles = 0;
    uint32_t cap_windows = 0;         // capacity of local_scratch (windows)
    LaunchBatch lb{};
    PushCfg push_cfg{PUSH_REG, 8, 32};
    uint32_t push_ctas = 0;
    bool push_tuned[3] = {false, false, false};
    bool autotune = true;
    // tuned variant per size class (bit length of the batch's padded neuron count), so a
    // serving batch whose membership changes keeps a variant fit for its current size
    std::map<uint32_t, PushCfg> tuned_by_size[3];
    uint32_t size_class = 0;
    TuneResult tune;                      // samples of the size class being tuned
    uint32_t tune_class = ~0u;            // that class (size class << 2 | accumulator mode)
    bool use_graph = true;
    cudaGraphExec_t graph = nullptr;
    uint64_t graph_key[9] = {};
    uint64_t seen_key[9] = {};        // shape of the last chunks launched eagerly, and how often in a row
    uint32_t seen_count = 0;
    uint32_t graph_launches = 0;
};

}  // namespace dtb
