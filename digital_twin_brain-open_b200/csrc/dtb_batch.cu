// Batched form: many independent networks (data-assimilation ensemble members,
// served requests) advanced by ONE launch of each per-step kernel.
//
// The reference batches an ensemble by packing its members into one network as
// disjoint population ranges (data_assimilation/DA_voxel.py:47-52, 264-268).  Here
// the members stay separate engines -- each with its own state, CSR, clock, noise
// stream and statistics -- and a batch launch walks all of them: CTA -> (member,
// tile) through a prefix over the members' tiles, one shared spike list whose
// entries carry a virtual neuron id (member base + neuron).  Uneven members cost
// nothing extra: tiles and spiking rows are distributed over the whole GPU.
//
// A window of steps of a push mode is captured once into a CUDA graph (2 kernel
// nodes per step, 5 with the population-local push) and replayed per window; the
// push variant is chosen by the same on-line autotuner as a single engine's, on
// the batch's own spike list.
#include <algorithm>
#include <cstring>

#include "dtb_batch.h"

namespace dtb {

// Consecutive LIF tiles per CTA in a batch of several members (lif_kernel): a member
// switch costs a chain of dependent loads that miss the L1, paid once per chunk.
// Measured on the 64-member ensemble (batched device time of 6 windows): chunks of
// 4 / 8 / 16 tiles -> 4.34 / 4.60 / 4.81 s; one tile per chunk ran ~7 % slower than four.
constexpr uint32_t kBatchLifChunk = 4;

Batch::~Batch() {
    if (stream) cudaStreamSynchronize(stream);
    if (graph) cudaGraphExecDestroy(graph);
    for (void* p : {static_cast<void*>(d_views), static_cast<void*>(d_prefix), static_cast<void*>(list),
                    static_cast<void*>(list_count), static_cast<void*>(list_ticket), static_cast<void*>(local_scratch),
                    static_cast<void*>(tile_net)})
        if (p) cudaFree(p);
    for (cudaEvent_t e : {ev0, ev1, tev[0], tev[1], ev_fork, ev_join})
        if (e) cudaEventDestroy(e);
    if (aux) cudaStreamDestroy(aux);
    if (stream) cudaStreamDestroy(stream);
}

int Batch::create(Engine* const* engines, uint32_t n) {
    DTB_CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    DTB_CU(cudaEventCreate(&ev0));
    DTB_CU(cudaEventCreate(&ev1));
    DTB_CU(cudaEventCreate(&tev[0]));
    DTB_CU(cudaEventCreate(&tev[1]));
    DTB_CU(cudaStreamCreateWithFlags(&aux, cudaStreamNonBlocking));
    DTB_CU(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    DTB_CU(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    return set_members(engines, n);
}

// (Re)define the members.  Device tables grow when needed and are reused
// otherwise, so a serving loop can change membership between slices cheaply;
// a captured graph is dropped because it holds the old tables' sizes.
int Batch::set_members(Engine* const* engines, uint32_t n) {
    if (n == 0) return fail(DTB_INVALID_PARAMETER, "empty batch");
    for (uint32_t i = 0; i < n; ++i) {
        if (!engines[i]) return fail(DTB_INVALID_PARAMETER, "NULL engine in batch");
        for (uint32_t j = 0; j < i; ++j)
            if (engines[j] == engines[i]) return fail(DTB_INVALID_PARAMETER, "an engine appears twice in the batch");
        if (engines[i]->wtype != engines[0]->wtype) return fail(DTB_UNSUPPORTED, "batch members must share the weight type");
        if (engines[i]->device != engines[0]->device) return fail(DTB_UNSUPPORTED, "batch members must share the device");
    }
    if (!m.empty() && engines[0]->wtype != wtype) push_tuned[0] = push_tuned[1] = push_tuned[2] = false;
    m.assign(engines, engines + n);
    wtype = m[0]->wtype;
    sm_count = m[0]->sm_count;
    std::vector<uint32_t> pre(4 * (n + 1), 0);
    uint64_t total = 0;
    for (uint32_t i = 0; i < n; ++i) {
        pre[i + 1] = pre[i] + m[i]->n_pad / kLifTile;
        pre[(n + 1) + i + 1] = pre[(n + 1) + i] + m[i]->n_pad / kPullTile;
        total += m[i]->n_pad;
        if (total >= 0xFFFFFFFFull) return fail(DTB_UNSUPPORTED, "a batch holds at most 2^32 neurons");
        pre[2 * (n + 1) + i + 1] = static_cast<uint32_t>(total);
        pre[3 * (n + 1) + i + 1] = pre[3 * (n + 1) + i] + m[i]->n_windows;
    }
    DTB_CU(cudaStreamSynchronize(stream));
    if (n > cap_members) {
        if (d_views) cudaFree(d_views);
        if (d_prefix) cudaFree(d_prefix);
        d_views = nullptr;
        d_prefix = nullptr;
        DTB_CU(cudaMalloc(reinterpret_cast<void**>(&d_views), sizeof(NetView) * n));
        DTB_CU(cudaMalloc(reinterpret_cast<void**>(&d_prefix), sizeof(uint32_t) * pre.size()));
        cap_members = n;
    }
    if (total > cap_neurons) {
        if (list) cudaFree(list);
        list = nullptr;
        DTB_CU(cudaMalloc(reinterpret_cast<void**>(&list), sizeof(uint32_t) * total));
        cap_neurons = total;
    }
    const uint32_t windows = pre[3 * (n + 1) + n];
    std::vector<uint32_t> tnet(pre[n]);
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t t = pre[i]; t < pre[i + 1]; ++t) tnet[t] = i;
    if (pre[n] > cap_tiles) {
        if (tile_net) cudaFree(tile_net);
        tile_net = nullptr;
        DTB_CU(cudaMalloc(reinterpret_cast<void**>(&tile_net), sizeof(uint32_t) * std::max<uint32_t>(pre[n], 1u)));
        cap_tiles = pre[n];
    }
    if (pre[n]) DTB_CU(cudaMemcpyAsync(tile_net, tnet.data(), sizeof(uint32_t) * pre[n], cudaMemcpyHostToDevice, stream));
    if (windows > cap_windows) {
        if (local_scratch) cudaFree(local_scratch);
        local_scratch = nullptr;
        DTB_CU(cudaMalloc(reinterpret_cast<void**>(&local_scratch), sizeof(uint32_t) * (2ull * windows + 3)));
        cap_windows = windows;
    }
    // the prep kernel's block ticket sits after this membership's tables: start it at zero
    if (local_scratch) DTB_CU(cudaMemsetAsync(local_scratch, 0, sizeof(uint32_t) * (2ull * cap_windows + 3), stream));
    if (!list_count) {
        DTB_CU(cudaMalloc(reinterpret_cast<void**>(&list_count), sizeof(uint32_t)));
        DTB_CU(cudaMalloc(reinterpret_cast<void**>(&list_ticket), sizeof(uint32_t)));
    }
    DTB_CU(cudaMemsetAsync(list_count, 0, sizeof(uint32_t), stream));
    DTB_CU(cudaMemsetAsync(list_ticket, 0, sizeof(uint32_t), stream));
    DTB_CU(cudaMemcpyAsync(d_prefix, pre.data(), sizeof(uint32_t) * pre.size(), cudaMemcpyHostToDevice, stream));
    lb.nets = d_views;
    lb.lif_prefix = d_prefix;
    lb.pull_prefix = d_prefix + (n + 1);
    lb.vbase = d_prefix + 2 * (n + 1);
    lb.n_nets = n;
    lb.lif_tiles_total = pre[n];
    lb.pull_tiles_total = pre[(n + 1) + n];
    lb.push_ctas = static_cast<uint32_t>(sm_count) * 8u;
    lb.lif_ctas = static_cast<uint32_t>(sm_count) * m[0]->lif_ctas_per_sm;
    lb.lif_chunk = n > 1 ? kBatchLifChunk : 1u;
    lb.spikes = SpikeList{list, list_count, list_ticket, static_cast<uint32_t>(total)};
    lb.tile_net = tile_net;
    lb.win_prefix = d_prefix + 3 * (n + 1);
    lb.windows_total = windows;
    lb.local_scratch = local_scratch;
    lb.sm_count = static_cast<uint32_t>(sm_count);
    lb.aux = aux;
    lb.ev_fork = ev_fork;
    lb.ev_join = ev_join;
    if (graph) {
        cudaGraphExecDestroy(graph);
        graph = nullptr;
    }
    std::memset(graph_key, 0, sizeof(graph_key));
    std::memset(seen_key, 0, sizeof(seen_key));
    seen_count = 0;
    DTB_CU(cudaStreamSynchronize(stream));
    return DTB_OK;
}

int Batch::refresh_views() {
    std::vector<NetView> v(m.size());
    for (size_t i = 0; i < m.size(); ++i) v[i] = m[i]->view;
    DTB_CU(cudaMemcpyAsync(d_views, v.data(), sizeof(NetView) * v.size(), cudaMemcpyHostToDevice, stream));
    DTB_CU(cudaStreamSynchronize(stream));
    return DTB_OK;
}

int Batch::run(const dtb_run_request& rq, dtb_run_output* outs) {
    if (rq.iters == 0) return fail(DTB_INVALID_PARAMETER, "iter must be positive");
    if (rq.prop_mode > DTB_PROP_OR || rq.syn_mode > DTB_SYN_PUSH_FIXED) return fail(DTB_INVALID_PARAMETER, "unknown mode");
    if (rq.t_steps > 1) return fail(DTB_UNSUPPORTED, "substeps (t_steps > 1) run through dtb_run, one engine at a time");
    const bool freq = (rq.flags & DTB_RUN_FREQ) != 0;
    const bool vmean = (rq.flags & DTB_RUN_VMEAN) != 0;
    const bool record = (rq.flags & DTB_RUN_RECORD_SPIKES) != 0;
    const int acc = acc_of(rq.syn_mode);
    const bool pull = rq.syn_mode == DTB_SYN_PULL;
    const bool samples = (rq.flags & (DTB_RUN_SAMPLE_SPIKE | DTB_RUN_SAMPLE_V | DTB_RUN_SAMPLE_IOU)) != 0;
    const bool imean = (rq.flags & DTB_RUN_IMEAN) != 0, rimean = (rq.flags & DTB_RUN_RECEPTOR_IMEAN) != 0;
    const bool sisyn = (rq.flags & DTB_RUN_SAMPLE_ISYN) != 0;
    if ((imean || rimean || sisyn) && rq.syn_mode == DTB_SYN_PULL)
        return fail(DTB_UNSUPPORTED, "synaptic-current outputs need a push mode (the pull kernel completes J one step later)");
    const bool isyn_any = imean || rimean || sisyn;
    bool injected = false;
    for (size_t i = 0; i < m.size(); ++i) {
        Engine& e = *m[i];
        if (!pull && !e.has_push) return fail(DTB_UNSUPPORTED, "a member has no out-degree CSR");
        if (pull && !e.has_pull) return fail(DTB_UNSUPPORTED, "a member has no in-degree CSR");
        if (acc == ACC_FIXED && e.fix_shift == 0)
            return fail(DTB_UNSUPPORTED, "a member's weights do not allow the fixed-point push");
        if ((freq && !outs[i].freqs) || (vmean && !outs[i].vmeans) || (record && !outs[i].spike_bits) ||
            (imean && !outs[i].imeans) || (rimean && !outs[i].receptor_imeans) ||
            (sisyn && !e.sample_order.empty() && !outs[i].sample_isyn))
            return fail(DTB_INVALID_PARAMETER, "requested output buffer is NULL");
        const bool inj = e.noise_src == DTB_NOISE_INJECTED;
        if (i > 0 && inj != injected) return fail(DTB_UNSUPPORTED, "batch members must share the noise source");
        injected = inj;
        if (inj && (e.steps - e.inj_first) + rq.iters > e.inj_rows)
            return fail(DTB_INVALID_PARAMETER, "a member has not enough injected noise rows");
        if (inj && rq.prop_mode != DTB_PROP_THRESHOLD && !e.inj_u)
            return fail(DTB_INVALID_PARAMETER, "noise train needs injected uniforms");
        DTB_CU(cudaStreamSynchronize(e.stream));
    }
    uint32_t cap = std::min<uint32_t>(rq.iters, 4096u);
    for (Engine* e : m) {
        if (record) cap = std::min<uint32_t>(cap, std::max<uint32_t>(1u, static_cast<uint32_t>((512ull << 20) / (4ull * e->n_words))));
    }
    for (Engine* e : m) {
        if (acc == ACC_EXACT) DTB_TRY(e->ensure_dj());
        if (acc == ACC_FIXED) DTB_TRY(e->ensure_djf());
        DTB_TRY(e->ensure_hist(cap, record, samples));
        if (isyn_any) DTB_TRY(e->ensure_isum(cap, sisyn));
    }
    DTB_TRY(refresh_views());
    uint32_t kflags = 0;
    if (rq.flags & DTB_RUN_USE_OU) kflags |= kFlagUseOU;
    if (freq || vmean) kflags |= kFlagStats;
    if (record) kflags |= kFlagRecord;
    if (!pull) kflags |= kFlagList;
    if (injected) kflags |= kFlagInjected;
    if (samples) kflags |= kFlagSample;
    if (isyn_any) kflags |= kFlagIsyn;
    const int pm = static_cast<int>(rq.prop_mode);
    const int wt = static_cast<int>(wtype);
    uint64_t tune_at = ~0ull;
    if (!pull) {
        if (autotune) {
            uint64_t total = 0;
            for (Engine* e : m) total += e->n_pad;
            size_class = 64u - static_cast<uint32_t>(__builtin_clzll(total | 1ull));
            const auto it = tuned_by_size[acc].find(size_class);
            push_tuned[acc] = it != tuned_by_size[acc].end();
            if (push_tuned[acc]) push_cfg = it->second;
        }
        DTB_CU(push_prepare(acc, wt, push_cfg, sm_count, &push_ctas));
        if (autotune && !push_tuned[acc]) {
            const uint64_t settle = 300;
            const uint64_t st = m[0]->steps;
            tune_at = st >= settle ? 1 : (settle - st < rq.iters ? settle - st : ~0ull);
        }
    }
    for (Engine* e : m) set_u64_kernel<<<1, 1, 0, stream>>>(e->events, 0ull);
    DTB_CU(cudaGetLastError());
    uint32_t launches = static_cast<uint32_t>(m.size());
    double ms_total = 0.0;
    uint32_t done = 0;
    while (done < rq.iters) {
        const uint32_t rows = std::min(cap, rq.iters - done);
        for (Engine* e : m) {
            set_u64_kernel<<<1, 1, 0, stream>>>(&e->clock->run_base, e->steps);
            if (freq || vmean) {
                DTB_CU(cudaMemsetAsync(e->hist_cnt, 0, sizeof(int) * rows * e->P, stream));
                DTB_CU(cudaMemsetAsync(e->hist_vsum, 0, sizeof(long long) * rows * e->P, stream));
            }
            if (isyn_any) DTB_CU(cudaMemsetAsync(e->hist_isum, 0, sizeof(long long) * rows * e->P * 5, stream));
            ++launches;
        }
        DTB_CU(cudaEventRecord(ev0, stream));
        // Graph-replayed window: a push mode with no tuning pending inside it.  A chunk that
        // starts a run folds nothing into J on its first step, and the last chunk of an
        // exact or fixed run ends by folding the sums into J, so both are in the key.
        const bool last_chunk = done + rows == rq.iters;
        const bool graphable = use_graph && !pull && !(tune_at >= done && tune_at < done + rows);
        bool replay = false;
        if (graphable) {
            const uint64_t key[9] = {rows, kflags, static_cast<uint64_t>(pm),
                                     static_cast<uint64_t>(push_cfg.kind) * 100000 + push_cfg.param * 100 + push_cfg.lpr,
                                     push_ctas, rq.syn_mode, done == 0, last_chunk, 1};
            if (graph && std::memcmp(key, graph_key, sizeof(key)) == 0) {
                replay = true;
            } else {
                // the same shape twice in a row under this membership before it is captured:
                // a serving batch whose membership changes every slice keeps launching eagerly
                if (std::memcmp(key, seen_key, sizeof(key)) != 0) {
                    std::memcpy(seen_key, key, sizeof(key));
                    seen_count = 0;
                }
                if (++seen_count >= 3) {
                    if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
                    cudaGraph_t g = nullptr;
                    DTB_CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
                    cudaError_t ce = cudaSuccess;
                    for (uint32_t s = 0; s < rows && ce == cudaSuccess; ++s) {
                        ce = launch_lif(lb, jmode_of(rq.syn_mode, done + s == 0), kflags, pm, stream);
                        if (ce == cudaSuccess) ce = launch_push(lb, acc, wt, push_cfg, push_ctas, stream);
                        if (ce == cudaSuccess && isyn_any) ce = launch_stat_isyn(lb, acc, sm_count, stream);
                    }
                    if (ce == cudaSuccess && last_chunk && acc != ACC_FLOAT) ce = launch_fold_finish(lb, acc, stream);
                    const cudaError_t ee = cudaStreamEndCapture(stream, &g);
                    if (ce != cudaSuccess) { if (g) cudaGraphDestroy(g); return cuda_fail(ce, "graph capture"); }
                    if (ee != cudaSuccess) return cuda_fail(ee, "cudaStreamEndCapture");
                    const cudaError_t ie = cudaGraphInstantiate(&graph, g, 0);
                    cudaGraphDestroy(g);
                    if (ie != cudaSuccess) { graph = nullptr; return cuda_fail(ie, "cudaGraphInstantiate"); }
                    std::memcpy(graph_key, key, sizeof(key));
                    replay = true;
                }
            }
        }
        if (replay) {
            DTB_CU(cudaGraphLaunch(graph, stream));
            ++graph_launches;
            launches += (2 + push_extra_launches(lb, acc, push_cfg) + (isyn_any ? 1u : 0u)) * rows +
                        (last_chunk && acc != ACC_FLOAT ? 1u : 0u);
        } else {
            for (uint32_t s = 0; s < rows; ++s) {
                const bool first = (done + s) == 0;
                if (pull) {
                    DTB_CU(launch_pull(lb, first ? 0 : 1, wt, kflags, pm, stream));
                    ++launches;
                    continue;
                }
                DTB_CU(launch_lif(lb, jmode_of(rq.syn_mode, first), kflags, pm, stream));
                if (tune_at == done + s) {
                    std::vector<NetView> v(m.size());
                    for (size_t i = 0; i < m.size(); ++i) v[i] = m[i]->view;
                    if (tune_class != (size_class << 2 | static_cast<uint32_t>(acc))) {
                        tune.reset();       // samples of another membership size or mode do not carry over
                        tune.observe = 0;   // a batch serves requests: tune on the first busy steps
                        tune.want = 2;
                        tune_class = size_class << 2 | static_cast<uint32_t>(acc);
                    }
                    DTB_TRY(tune_push_views(lb, v, acc, wt, sm_count, stream, tev, tune));
                    if (tune.tuned) {
                        push_cfg = tune.best;
                        push_tuned[acc] = true;
                        tuned_by_size[acc][size_class] = push_cfg;
                        tune.reset();
                        DTB_CU(push_prepare(acc, wt, push_cfg, sm_count, &push_ctas));
                    } else {
                        tune_at = tune.next_step(tune_at);
                    }
                }
                DTB_CU(launch_push(lb, acc, wt, push_cfg, push_ctas, stream));
                launches += 2 + push_extra_launches(lb, acc, push_cfg);
                if (isyn_any) {
                    DTB_CU(launch_stat_isyn(lb, acc, sm_count, stream));
                    ++launches;
                }
            }
            if (last_chunk) {
                if (acc != ACC_FLOAT && !pull) { DTB_CU(launch_fold_finish(lb, acc, stream)); ++launches; }
                if (pull) { DTB_CU(launch_gather_finish(lb, wt, stream)); ++launches; }
            }
        }
        DTB_CU(cudaEventRecord(ev1, stream));
        DTB_CU(cudaEventSynchronize(ev1));
        float ms = 0.f;
        DTB_CU(cudaEventElapsedTime(&ms, ev0, ev1));
        ms_total += ms;
        for (size_t i = 0; i < m.size(); ++i) {
            Engine& e = *m[i];
            for (uint32_t s = 0; s < rows; ++s) {
                volatile float tt = e.t + e.dt;
                e.t = tt;
            }
            e.steps += rows;
            DTB_TRY(e.finish_hist(rows, done, outs[i], freq, vmean, record));
            if (samples && !e.sample_order.empty()) DTB_TRY(e.finish_samples(rows, done, outs[i]));
            if (isyn_any) DTB_TRY(e.finish_isum(rows, done, outs[i], imean, rimean, sisyn && !e.sample_order.empty()));
        }
        done += rows;
    }
    for (size_t i = 0; i < m.size(); ++i) {
        Engine& e = *m[i];
        Clock ck;
        unsigned long long ev = 0;
        DTB_CU(cudaMemcpyAsync(&ck, e.clock, sizeof(Clock), cudaMemcpyDeviceToHost, stream));
        DTB_CU(cudaMemcpyAsync(&ev, e.events, sizeof(ev), cudaMemcpyDeviceToHost, stream));
        DTB_CU(cudaStreamSynchronize(stream));
        outs[i].events = ev;
        outs[i].device_ms = ms_total;
        outs[i].launches = launches;
        for (int k = 0; k < 4; ++k) outs[i].kernel_ms[k] = 0.0;
        if (ck.n != e.steps) return fail(DTB_DEVICE_FAULT, "device clock out of step with the host (member " + std::to_string(i) + ")");
        if (ck.err) return fail(DTB_DEVICE_FAULT, "kernel check failed in member " + std::to_string(i) + ", bits " + std::to_string(ck.err));
    }
    return DTB_OK;
}

}  // namespace dtb

using dtb::Batch;
using dtb::Engine;

extern "C" {

int32_t dtb_batch_create(void* const* engines, uint32_t n, void** batch) {
    if (!engines || !batch) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    *batch = nullptr;
    try {
        auto* b = new Batch();
        const int s = b->create(reinterpret_cast<Engine* const*>(engines), n);
        if (s != DTB_OK) { delete b; return s; }
        *batch = b;
        return DTB_OK;
    } catch (const std::bad_alloc&) {
        return dtb::fail(DTB_OUT_OF_MEMORY, "host allocation failed");
    }
}

int32_t dtb_batch_destroy(void* batch) {
    if (!batch) return dtb::fail(DTB_INVALID_PARAMETER, "NULL batch");
    delete static_cast<Batch*>(batch);
    return DTB_OK;
}

int32_t dtb_batch_run(void* batch, const dtb_run_request* req, dtb_run_output* outs) {
    if (!batch || !req || !outs) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    try {
        return static_cast<Batch*>(batch)->run(*req, outs);
    } catch (const std::bad_alloc&) {
        return dtb::fail(DTB_OUT_OF_MEMORY, "host allocation failed");
    }
}

int32_t dtb_batch_set_graph(void* batch, int32_t enable) {
    if (!batch) return dtb::fail(DTB_INVALID_PARAMETER, "NULL batch");
    static_cast<Batch*>(batch)->use_graph = enable != 0;
    return DTB_OK;
}

int32_t dtb_batch_set_push_variant(void* batch, int32_t kind, int32_t param) {
    if (!batch) return dtb::fail(DTB_INVALID_PARAMETER, "NULL batch");
    Batch* b = static_cast<Batch*>(batch);
    if (kind < 0) {
        b->autotune = true;
        for (int a = 0; a < 3; ++a) {
            b->push_tuned[a] = false;
            b->tuned_by_size[a].clear();
        }
        b->tune.reset();
        return DTB_OK;
    }
    dtb::PushCfg cfg;
    if (!dtb::push_cfg_from_abi(kind, param, cfg)) return dtb::fail(DTB_INVALID_PARAMETER, "unknown push variant");
    b->push_cfg = cfg;
    b->autotune = false;
    return DTB_OK;
}

int32_t dtb_batch_info(void* batch, uint32_t* n_members, uint32_t* graph_launches, int32_t* push_kind,
                       int32_t* push_param) {
    if (!batch) return dtb::fail(DTB_INVALID_PARAMETER, "NULL batch");
    const Batch* b = static_cast<const Batch*>(batch);
    if (n_members) *n_members = static_cast<uint32_t>(b->m.size());
    if (graph_launches) *graph_launches = b->graph_launches;
    if (push_kind) *push_kind = b->push_cfg.kind;
    if (push_param) *push_param = b->push_cfg.lpr != 32 ? 1000 + b->push_cfg.lpr : b->push_cfg.param;
    return DTB_OK;
}

}  // extern "C"
