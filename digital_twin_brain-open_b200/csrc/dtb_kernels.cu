// Per-step kernels of the engine.
//
//   lif_kernel<JM>        fused OU + LIF + threshold + receptor decay + spike
//                         compaction + per-population statistics, 4 neurons/thread
//                         with 128-bit loads (replaces the reference's OU, membrane,
//                         spike, compaction, J-decay, synaptic-current and stat kernels:
//                         src/stage/extern_stimuli.cpp:39-112, membrane_voltage.cpp:114-235,
//                         spike.cpp:42-68, 244-762, presynaptic_voltage.cpp:46-120,
//                         synaptic_current.cpp:7-71, stat_result.cpp:161-327)
//   push_kernel<ACC,WT>   out-degree CSR propagation of the compacted spikes: one warp per
//                         spiking row, 4 synapses in flight per lane, one vector reduction
//                         (or two 64-bit fixed-point atomics) per synapse
//                         (src/stage/presynaptic_voltage.cpp:122-225)
//   lif_pull_kernel<G,WT> deterministic in-degree gather fused into the LIF step: one warp
//                         gathers 32 neurons, then each lane steps one neuron
//   fold_finish_kernel / gather_finish_kernel: bring J back to "complete" at the end of a run
//
// A launch covers a batch of networks (one for the plain path).  CTA -> network is
// a binary search over the batch's tile prefix; every network keeps its own clock,
// and the last CTA of a network to finish (ticket counter) advances that clock.
#include <algorithm>
#include <atomic>

#include "dtb_device.cuh"
#include "dtb_kernels.h"

namespace dtb {

constexpr int kStatSlots = 32;
constexpr int kPushThreads = 256;
constexpr int kTmaWarps = 4;
constexpr uint32_t kWaitLimit = 1u << 22;   // mbarrier polls before a wait is declared failed

// Fire-and-forget reductions (no returned value, so no scoreboard wait).
__device__ __forceinline__ void red_add_u64(unsigned long long* addr, unsigned long long v) {
    asm volatile("red.global.add.u64 [%0], %1;" :: "l"(addr), "l"(v) : "memory");
}

// The accumulators (J, or dJf in fixed-point mode: 80 MB at 5M neurons) are
// reduced into with an L2 evict_last policy, so the CSR stream of the push
// (gigabytes in a burst step, loaded evict_first by ld.global.cs) does not push
// them out of L2.  Without it the scattered reductions of the cross-population
// push missed L2 and wrote about 15 bytes of DRAM back per event.
__device__ __forceinline__ unsigned long long l2_policy_keep() {
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ void red_add_f32x2_keep(float2* addr, float2 v, unsigned long long pol) {
    asm volatile("red.global.add.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" :: "l"(addr), "f"(v.x), "f"(v.y), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void red_add_f32x4_keep(float4* addr, float4 v, unsigned long long pol) {
    asm volatile("red.global.add.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;"
                 :: "l"(addr), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w), "l"(pol) : "memory");
}
__device__ __forceinline__ void red_add_u64_keep(unsigned long long* addr, unsigned long long v, unsigned long long pol) {
    asm volatile("red.global.add.L2::cache_hint.u64 [%0], %1, %2;" :: "l"(addr), "l"(v), "l"(pol) : "memory");
}

__device__ inline uint32_t find_net(const uint32_t* __restrict__ prefix, uint32_t n_nets, uint32_t x) {
    uint32_t lo = 0, hi = n_nets - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= x) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ inline void load_netview(NetView& dst, const NetView* __restrict__ src) {
    const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
    uint32_t* d = reinterpret_cast<uint32_t*>(&dst);
    for (int w = threadIdx.x; w < static_cast<int>(sizeof(NetView) / 4); w += blockDim.x) d[w] = s[w];
}

__device__ inline long long warp_sum_ll(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ inline unsigned long long warp_sum_ull(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Neuron slots of a LIF tile: thread `slot` of the tile's CTA steps neurons
// tile_first + slot + kLifThreads * k (k = 0..3), so each step of k touches 32
// consecutive neurons per warp.  One Philox4x32-10 block per (slot, step) gives
// the four draws of the slot's neurons: counter (tile_first / 4 + slot, step,
// stream); draw k belongs to neuron tile_first + slot + kLifThreads * k.
constexpr uint32_t kSlotsPerTile = kLifThreads;
static_assert(kLifTile == 4 * kLifThreads, "a LIF thread steps four neurons");

// Normal draws (OU) and uniforms (noise train) for the four neurons of a slot.
// Substep k of ts draws from its own streams: injected row (n - inj_base - 1) ts + k,
// Philox stream word XOR k << 20 (k = 0 is the plain step's stream).
__device__ inline void draw_noise(const NetView& nv, uint32_t tile_first, uint32_t slot, unsigned long long n,
                                  unsigned long long inj_base, bool injected, bool need_u, float z[4], float u[4],
                                  uint32_t& err, uint32_t sub = 0, uint32_t ts = 1) {
    if (injected) {
        const unsigned long long row = (n - inj_base - 1) * ts + sub;
        if (row < nv.inj_rows && nv.inj_z != nullptr) {
            const float* zr = nv.inj_z + row * nv.n_pad + tile_first + slot;
#pragma unroll
            for (int k = 0; k < 4; ++k) z[k] = __ldcs(zr + kSlotsPerTile * k);
            if (need_u) {
                if (nv.inj_u != nullptr) {
                    const float* ur = nv.inj_u + row * nv.n_pad + tile_first + slot;
#pragma unroll
                    for (int k = 0; k < 4; ++k) u[k] = __ldcs(ur + kSlotsPerTile * k);
                } else {
                    u[0] = u[1] = u[2] = u[3] = 1.0f;
                    err |= kErrNoiseExhausted;
                }
            }
        } else {
            z[0] = z[1] = z[2] = z[3] = 0.0f;
            u[0] = u[1] = u[2] = u[3] = 1.0f;
            err |= kErrNoiseExhausted;
        }
    } else {
        const uint32_t k0 = static_cast<uint32_t>(nv.seed), k1 = static_cast<uint32_t>(nv.seed >> 32);
        const uint32_t ctr = (tile_first >> 2) + slot;
        const U4 r = philox4x32_10(U4{ctr, static_cast<uint32_t>(n), static_cast<uint32_t>(n >> 32), kStreamOU ^ (sub << 20)}, k0, k1);
        box_muller(r.x, r.y, z[0], z[1]);
        box_muller(r.z, r.w, z[2], z[3]);
        if (need_u) {
            const U4 q = philox4x32_10(U4{ctr, static_cast<uint32_t>(n), static_cast<uint32_t>(n >> 32), kStreamNoise ^ (sub << 20)}, k0, k1);
            u[0] = u01(q.x); u[1] = u01(q.y); u[2] = u01(q.z); u[3] = u01(q.w);
        }
    }
}

__device__ inline void draw_noise1(const NetView& nv, uint32_t i, unsigned long long n, unsigned long long inj_base,
                                   bool injected, bool need_u, float& z, float& u, uint32_t& err) {
    // one neuron: same streams as draw_noise (draw k of its slot)
    if (injected) {
        const unsigned long long row = n - inj_base - 1;
        if (row < nv.inj_rows && nv.inj_z != nullptr) {
            z = __ldcs(nv.inj_z + row * nv.n_pad + i);
            if (need_u) {
                if (nv.inj_u != nullptr) u = __ldcs(nv.inj_u + row * nv.n_pad + i);
                else { u = 1.0f; err |= kErrNoiseExhausted; }
            }
        } else {
            z = 0.0f; u = 1.0f; err |= kErrNoiseExhausted;
        }
    } else {
        const uint32_t k0 = static_cast<uint32_t>(nv.seed), k1 = static_cast<uint32_t>(nv.seed >> 32);
        const uint32_t w = i % kLifTile, k = w / kSlotsPerTile;
        const uint32_t ctr = ((i - w) >> 2) + w % kSlotsPerTile;
        const U4 r = philox4x32_10(U4{ctr, static_cast<uint32_t>(n), static_cast<uint32_t>(n >> 32), kStreamOU}, k0, k1);
        float z4[4];
        box_muller(r.x, r.y, z4[0], z4[1]);
        box_muller(r.z, r.w, z4[2], z4[3]);
        z = z4[k];
        if (need_u) {
            const U4 q = philox4x32_10(U4{ctr, static_cast<uint32_t>(n), static_cast<uint32_t>(n >> 32), kStreamNoise}, k0, k1);
            const uint32_t qq[4] = {q.x, q.y, q.z, q.w};
            u = u01(qq[k]);
        }
    }
}

__device__ inline bool propagated(int prop_mode, bool active, float u, float rate) {
    if (prop_mode == PROP_THRESHOLD) return active;
    const bool noise = u < rate;
    return prop_mode == PROP_NOISE ? noise : (noise || active);
}

__device__ inline bool excluded(const NetView& nv, uint32_t i) {
    return nv.stat_excl != nullptr && ((__ldg(nv.stat_excl + (i >> 5)) >> (i & 31)) & 1u);
}

// Shared per-CTA statistics accumulator: population slots relative to the
// CTA's first population; populations beyond the window go straight to global.
struct StatAcc {
    int* cnt;
    long long* vs;
    uint32_t p0;
};

__device__ inline void stat_add(const NetView& nv, const StatAcc& sa, long long row, uint32_t p, int c, long long v) {
    const uint32_t slot = p - sa.p0;
    if (slot < static_cast<uint32_t>(kStatSlots)) {
        if (c) atomicAdd(sa.cnt + slot, c);
        atomicAdd(reinterpret_cast<unsigned long long*>(sa.vs + slot), static_cast<unsigned long long>(v));
    } else {
        const size_t o = static_cast<size_t>(row) * nv.n_pops + p;
        if (c) atomicAdd(nv.hist_cnt + o, c);
        atomicAdd(reinterpret_cast<unsigned long long*>(nv.hist_vsum + o), static_cast<unsigned long long>(v));
    }
}

// Warp-collective: lanes holding (pop, count, V sum) with `has` add their sums per
// distinct pop, one shared-slot (or global) update per pop.
__device__ inline void warp_stat_segments(const NetView& nv, const StatAcc& sa, long long row, uint32_t pop, bool has,
                                          int cnt, long long vs, uint32_t lane) {
    uint32_t rem = __ballot_sync(0xffffffffu, has);
    while (rem) {
        const uint32_t leader = static_cast<uint32_t>(__ffs(rem) - 1);
        const uint32_t pk = __shfl_sync(0xffffffffu, pop, leader);
        const bool in = ((rem >> lane) & 1u) && pop == pk;
        const int c = __reduce_add_sync(0xffffffffu, static_cast<unsigned>(in ? cnt : 0));
        const long long v = warp_sum_ll(in ? vs : 0ll);
        if (lane == leader) stat_add(nv, sa, row, pk, c, v);
        rem &= ~__ballot_sync(0xffffffffu, in);
    }
}

__device__ inline long long v_fix(float v) {
    return __float2ll_rn(__fmul_rn(v, static_cast<float>(kVsumScale)));
}

__device__ inline void advance_clock(const NetView& nv, uint32_t tiles, float t, unsigned long long n, uint32_t err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        if (err) atomicOr(&nv.clock->err, err);
        __threadfence();
        const uint32_t k = atomicAdd(nv.ticket, 1u);
        if (k == tiles - 1) {
            nv.clock->t = t;
            nv.clock->n = n;
            *nv.ticket = 0u;
            __threadfence();
        }
    }
}

// mbarrier and bulk-copy helpers (cp.async.bulk, no multicast).
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    uint64_t g;
    asm volatile("cvta.to.global.u64 %0, %1;" : "=l"(g) : "l"(src));
    asm volatile("cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_addr(dst)), "l"(g), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                 : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity) : "memory");
    return ok != 0;
}
// Bounded wait on one mbarrier phase; false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (uint32_t it = 0; it < kWaitLimit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// ---------------------------------------------------------------------------
// Fused LIF step (push and exact-push modes): a persistent grid walks the
// batch's 1024-neuron tiles.  A tile's state (V, i_ou, t_last: 4 KiB each; J:
// 16 KiB) moves by bulk copies (cp.async.bulk, no multicast) through a
// two-stage ring in shared memory: the copies of the next tile are in flight
// while the CTA steps the current one, each thread steps its quad of neurons
// one neuron at a time in the stage, and the finished tile leaves by bulk
// stores.  One CTA barrier per tile, before the finished stage is stored: the
// refill of a stage needs only its store to have read it (thread 0 waits for
// that), and the statistics slots alternate by tile parity, so no warp waits for
// the others at the top of a tile (measured: LIF 0.0866 -> 0.0802 ms per step at
// 5M against a second barrier there).  Spike-list slots are taken per warp; the
// device clock's ticket is taken once per CTA and network.
// Every mbarrier wait is bounded; a wait that runs out raises kErrTimeout (the
// host turns it into DTB_DEVICE_FAULT) after one more bounded wait.
// ---------------------------------------------------------------------------
constexpr uint32_t kLifStageFloats = 3 * kLifTile + 4 * kLifTile;   // V | i_ou | t_last | J (float4)
constexpr size_t kLifSmem = static_cast<size_t>(kLifStages) * kLifStageFloats * sizeof(float);

__device__ __forceinline__ void bulk_store(void* gdst, const void* ssrc, uint32_t bytes) {
    uint64_t g;
    asm volatile("cvta.to.global.u64 %0, %1;" : "=l"(g) : "l"(gdst));
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
                 :: "l"(g), "r"(smem_addr(ssrc)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// thread 0: issue the copies of tile `gt` into stage `stg`
// Network of a batch tile: one load from the tile table when the batch has one.
__device__ __forceinline__ uint32_t tile_to_net(const uint32_t* __restrict__ tile_net, const uint32_t* __restrict__ tile_prefix,
                                                uint32_t n_nets, uint32_t gt) {
    if (n_nets <= 1) return 0u;
    return tile_net ? __ldg(tile_net + gt) : find_net(tile_prefix, n_nets, gt);
}

__device__ __forceinline__ void lif_prefetch(const NetView* __restrict__ nets, const uint32_t* __restrict__ tile_prefix,
                                             const uint32_t* __restrict__ tile_net, uint32_t n_nets, uint32_t gt,
                                             float* stage, uint64_t* bar) {
    const uint32_t net = tile_to_net(tile_net, tile_prefix, n_nets, gt);
    const NetView* nv = nets + net;
    const size_t first = static_cast<size_t>(gt - __ldg(tile_prefix + net)) * kLifTile;
    mbar_expect_tx(bar, static_cast<uint32_t>(kLifStageFloats * sizeof(float)));
    bulk_load(stage, nv->V + first, kLifTile * sizeof(float), bar);
    bulk_load(stage + kLifTile, nv->iou + first, kLifTile * sizeof(float), bar);
    bulk_load(stage + 2 * kLifTile, nv->tlast + first, kLifTile * sizeof(float), bar);
    bulk_load(stage + 3 * kLifTile, nv->J + first, kLifTile * sizeof(float4), bar);
}

// thread 0: the CTA finished `cnt` tiles of `nv`; the last CTA of the network advances its clock
__device__ __forceinline__ void lif_ticket(const NetView& nv, uint32_t cnt, float t, unsigned long long n) {
    __threadfence();
    const uint32_t k = atomicAdd(nv.ticket, cnt);
    if (k + cnt == nv.lif_tiles) {
        nv.clock->t = t;
        nv.clock->n = n;
        *nv.ticket = 0u;
        __threadfence();
    }
}

// A CTA steps chunks of `chunk` consecutive tiles, chunks strided by the grid:
// tile gt is followed by gt + 1 inside its chunk, else by the CTA's next chunk.
// Chunks of several tiles keep a batch CTA on one member for several tiles, so the
// member's view, clock and parameters are fetched once per chunk, not per tile.
__device__ __forceinline__ uint32_t lif_next_tile(uint32_t gt, uint32_t chunk, uint32_t total_tiles) {
    if (gt % chunk + 1 < chunk && gt + 1 < total_tiles) return gt + 1;
    return (gt / chunk + gridDim.x) * chunk;
}

template <int JM>
__global__ void __launch_bounds__(kLifThreads, kLifCtasPerSm)
lif_kernel(const NetView* __restrict__ nets, const uint32_t* __restrict__ tile_prefix,
           const uint32_t* __restrict__ vbase, uint32_t n_nets, uint32_t total_tiles, SpikeList sl, uint32_t flags,
           int prop_mode, const uint32_t* __restrict__ tile_net, uint32_t chunk) {
    extern __shared__ __align__(128) float lsm[];
    __shared__ __align__(8) uint64_t s_bar[kLifStages];
    // population slots of the statistics, by tile parity: tile `it` adds into set it & 1,
    // which its flush (after barrier B) empties while the next tile fills the other set
    __shared__ int s_cnt[2][kStatSlots];
    __shared__ long long s_vs[2][kStatSlots];

    const int tid = threadIdx.x, lane = tid & 31;
    uint32_t cur_net = 0xFFFFFFFFu;
    const bool use_ou = (flags & kFlagUseOU) != 0;
    const bool need_u = prop_mode != PROP_THRESHOLD;
    const bool injected = (flags & kFlagInjected) != 0;
    // substep k of ts: spikes OR into the step's bitmap and list (a neuron enters the list
    // once), counts are of neurons newly spiking, V statistics and samples come from the
    // last substep, and the clock's step count advances after it (dist_simulator.cpp:2085-2112)
    const uint32_t sub = (flags >> kSubShift) & 0xFFu;
    const uint32_t ts = max(1u, (flags >> kTsShift) & 0xFFu);
    const bool last_sub = sub + 1 >= ts;
    uint32_t late = 0;                 // a bulk-copy wait ran out
    uint32_t done_here = 0;            // tiles of cur_net this CTA finished (thread 0's ticket)
    float t_last_tile = 0.f;
    unsigned long long n_last_tile = 0;
    // finished (network, tiles) pairs, handed in when the CTA ends; a full table is handed in early
    constexpr int kTicketSlots = 48;
    __shared__ uint32_t s_tk_net[kTicketSlots], s_tk_cnt[kTicketSlots];
    __shared__ float s_tk_t[kTicketSlots];
    __shared__ unsigned long long s_tk_n[kTicketSlots];
    uint32_t n_tk = 0;                 // thread 0's count of table entries
    if (tid < 2 * kStatSlots) { s_cnt[tid / kStatSlots][tid % kStatSlots] = 0; s_vs[tid / kStatSlots][tid % kStatSlots] = 0; }
    if (tid == 0) {
        for (int s = 0; s < kLifStages; ++s) mbar_init(&s_bar[s], 1);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    // thread 0: the next tile to prefetch; the first kLifStages - 1 tiles go in now
    uint32_t pre = blockIdx.x * chunk;
    if (tid == 0) {
        for (int s = 0; s + 1 < kLifStages && pre < total_tiles; ++s) {
            lif_prefetch(nets, tile_prefix, tile_net, n_nets, pre, lsm + s * kLifStageFloats, &s_bar[s]);
            pre = lif_next_tile(pre, chunk, total_tiles);
        }
    }
    __syncthreads();

    uint32_t it = 0;
    for (uint32_t gt = blockIdx.x * chunk; gt < total_tiles; gt = lif_next_tile(gt, chunk, total_tiles), ++it) {
        const uint32_t net = tile_to_net(tile_net, tile_prefix, n_nets, gt);
        const uint32_t stg = it % kLifStages;
        if (net != cur_net) {
            // hand in the previous network's tiles (views are read through the
            // read-only cache, so switching needs no barrier)
            if (tid == 0 && done_here) {
                if (n_tk == kTicketSlots) {
                    for (uint32_t q = 0; q < n_tk; ++q) lif_ticket(nets[s_tk_net[q]], s_tk_cnt[q], s_tk_t[q], s_tk_n[q]);
                    n_tk = 0;
                }
                s_tk_net[n_tk] = cur_net;
                s_tk_cnt[n_tk] = done_here;
                s_tk_t[n_tk] = t_last_tile;
                s_tk_n[n_tk] = n_last_tile;
                ++n_tk;
            }
            done_here = 0;
            cur_net = net;
        }
        // every thread is past barrier B of the previous tile, so its stage has been read and
        // its store issued: once that store has read the stage, refill it with the tile
        // kLifStages - 1 ahead (the other warps wait for their tile on its mbarrier)
        if (tid == 0 && pre < total_tiles) {
            const uint32_t sn = (it + kLifStages - 1) % kLifStages;
            bulk_wait_read();
            lif_prefetch(nets, tile_prefix, tile_net, n_nets, pre, lsm + sn * kLifStageFloats, &s_bar[sn]);
            pre = lif_next_tile(pre, chunk, total_tiles);
        }
        const NetView& nv = nets[net];
        const uint32_t tile = gt - __ldg(tile_prefix + net);
        const uint32_t tile_first = tile * kLifTile;
        const uint32_t i0 = tile_first + tid;             // this thread: neurons i0 + kSlotsPerTile * k
        const float t_prev = nv.clock->t;
        const unsigned long long n_prev = nv.clock->n;
        const unsigned long long run_base = nv.clock->run_base;
        const unsigned long long inj_base = nv.clock->inj_base;
        const uint32_t p_tile = __ldg(nv.tile_pop + tile);
        const unsigned long long n = n_prev + 1;
        const float t = __fadd_rn(t_prev, nv.dt);
        const uint32_t parity = static_cast<uint32_t>(n & 1ull);
        uint32_t err = 0;
        const long long row = static_cast<long long>(n - run_base - 1);
        bool stats = (flags & kFlagStats) != 0;
        bool record = (flags & kFlagRecord) != 0 && nv.rec_bits != nullptr;
        if ((stats || record) && (row < 0 || row >= static_cast<long long>(nv.hist_cap))) {
            stats = false; record = false; err |= kErrHistOverflow;
        }
        const bool sample = (flags & kFlagSample) && nv.n_samples && row >= 0 && row < static_cast<long long>(nv.hist_cap) &&
                            last_sub;
        StatAcc sa{s_cnt[it & 1u], s_vs[it & 1u], p_tile};
        float z[4], u[4] = {1.f, 1.f, 1.f, 1.f};
        draw_noise(nv, tile_first, tid, n, inj_base, injected, need_u, z, u, err, sub, ts);
        // propagated spikes of this step's earlier substeps, one word per k of this warp
        uint32_t old_w[4] = {0u, 0u, 0u, 0u};
        if (sub) {
            const uint32_t* bits = parity ? nv.bits1 : nv.bits0;
            const uint32_t word0 = (tile_first >> 5) + (tid >> 5);
#pragma unroll
            for (int k = 0; k < 4; ++k) old_w[k] = bits[word0 + (kSlotsPerTile / 32) * k];
        }
        const uint32_t phase = (it / kLifStages) & 1u;
        if (!mbar_wait_bounded(&s_bar[stg], phase)) {
            late = 1;
            mbar_wait_bounded(&s_bar[stg], phase);
        }
        if (late) err |= kErrTimeout;
        // stage accesses: each step of k reads and writes 32 consecutive neurons
        // per warp, so every shared-memory access is free of bank conflicts
        float* st = lsm + stg * kLifStageFloats;
        float* sV = st + tid;
        float* sI = st + kLifTile + tid;
        float* sT = st + 2 * kLifTile + tid;
        float4* sJ = reinterpret_cast<float4*>(st + 3 * kLifTile) + tid;

        uint32_t nib_prop = 0, nib_act = 0;
        uint32_t ev = 0;                   // out-degrees of this thread's (at most four) spiking neurons
        uint32_t p = p_tile;
        const uint32_t i_first = min(i0, nv.n - 1);
        while (p + 1 < nv.n_pops && __ldg(nv.pop_off + p + 1) <= i_first) ++p;
        const uint32_t p_first = p;
        bool uniform = true;
        int cnt_acc = 0, cnt_nxt = 0;          // neurons of p_first, and of p_first + 1
        long long vs_acc = 0, vs_nxt = 0;
        PopParams pp;
        load_pop_params(nv, p, i_first, pp);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t i = i0 + kSlotsPerTile * k;
            if (i >= nv.n) { uniform = false; continue; }
            if (p + 1 < nv.n_pops && __ldg(nv.pop_off + p + 1) <= i) {
                while (p + 1 < nv.n_pops && __ldg(nv.pop_off + p + 1) <= i) ++p;
                uniform = false;
                if (!nv.per_neuron) load_pop_params(nv, p, i, pp);
            }
            if (nv.per_neuron && k > 0) load_pop_params(nv, p, i, pp);
            const int ks = kSlotsPerTile * k;
            const float4 Jk = sJ[ks];
            NeuronIn in;
            in.V = sV[ks];
            in.iou = sI[ks];
            in.tlast = sT[ks];
            if constexpr (JM == J_FOLD) {
                longlong2* dq = reinterpret_cast<longlong2*>(nv.dJ + static_cast<size_t>(i) * 4);
                const longlong2 d01 = dq[0], d23 = dq[1];
                in.J[0] = decay_add(Jk.x, pp.decay[0], fix_to_float(d01.x));
                in.J[1] = decay_add(Jk.y, pp.decay[1], fix_to_float(d01.y));
                in.J[2] = decay_add(Jk.z, pp.decay[2], fix_to_float(d23.x));
                in.J[3] = decay_add(Jk.w, pp.decay[3], fix_to_float(d23.y));
                dq[0] = make_longlong2(0, 0);
                dq[1] = make_longlong2(0, 0);
            } else if constexpr (JM == J_FIXF) {
                ulonglong2* dq = reinterpret_cast<ulonglong2*>(nv.dJf) + i;
                const ulonglong2 d = *dq;
                in.J[0] = decay_add(Jk.x, pp.decay[0], fixed_field(d.x, 0, nv.fix_unscale));
                in.J[1] = decay_add(Jk.y, pp.decay[1], fixed_field(d.x, 1, nv.fix_unscale));
                in.J[2] = decay_add(Jk.z, pp.decay[2], fixed_field(d.y, 0, nv.fix_unscale));
                in.J[3] = decay_add(Jk.w, pp.decay[3], fixed_field(d.y, 1, nv.fix_unscale));
                *dq = make_ulonglong2(0ull, 0ull);
            } else {
                in.J[0] = Jk.x; in.J[1] = Jk.y; in.J[2] = Jk.z; in.J[3] = Jk.w;
            }
            const NeuronOut o = lif_update(pp, in, t, z[k], use_ou);
            sV[ks] = o.V;
            sI[ks] = o.iou;
            sT[ks] = o.tlast;
            if constexpr (JM == J_DIRECT) {
                sJ[ks] = make_float4(__fmul_rn(in.J[0], pp.decay[0]), __fmul_rn(in.J[1], pp.decay[1]),
                                     __fmul_rn(in.J[2], pp.decay[2]), __fmul_rn(in.J[3], pp.decay[3]));
            } else if constexpr (JM == J_FOLD || JM == J_FIXF) {
                sJ[ks] = make_float4(in.J[0], in.J[1], in.J[2], in.J[3]);
            }
            const bool sp = propagated(prop_mode, o.active, u[k], pp.noise_rate);
            const bool seen = (old_w[k] >> lane) & 1u;     // spiked in an earlier substep of this step
            nib_prop |= static_cast<uint32_t>(sp) << k;
            nib_act |= static_cast<uint32_t>(o.active) << k;
            if (sp && !seen) ev += __ldg(nv.out_deg + i);
            // sampled neurons (stat_samples_kernel, src/stage/stat_result.cpp:393-431)
            if (sample) {
                const uint32_t sbw = __ldg(nv.sample_bits + (i >> 5)), sh = i & 31u;
                if ((sbw >> sh) & 1u) {
                    const size_t so = static_cast<size_t>(row) * nv.n_samples + __ldg(nv.sample_pre + (i >> 5)) +
                                      __popc(sbw & ((1u << sh) - 1u));
                    nv.hist_sspk[so] = static_cast<uint8_t>(o.active || seen);
                    nv.hist_sv[so] = o.V;
                    nv.hist_siou[so] = o.iou;
                }
            }
            if (stats) {
                if (excluded(nv, i)) { uniform = false; continue; }
                const int fresh = o.active && !seen;
                const long long vq = last_sub ? v_fix(o.V) : 0ll;
                if (p == p_first) {
                    cnt_acc += fresh;
                    vs_acc += vq;
                } else if (p == p_first + 1) {
                    cnt_nxt += fresh;
                    vs_nxt += vq;
                } else {                      // a population narrower than a thread's span
                    stat_add(nv, sa, row, p, fresh, vq);
                }
            }
        }

        // ---- spike bitmaps and list: step k of a warp covers one 32-neuron word
        //      (propagated: parity buffer and one slot range per warp in the list;
        //      threshold: history row)
        {
            uint32_t* bits = parity ? nv.bits1 : nv.bits0;
            const uint32_t word0 = (tile_first >> 5) + (tid >> 5);
            uint32_t wprop[4], wtotal = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint32_t all = __ballot_sync(0xffffffffu, (nib_prop >> k) & 1u);
                wprop[k] = all & ~old_w[k];                     // new to the step's list
                wtotal += __popc(wprop[k]);
                const uint32_t wact = __ballot_sync(0xffffffffu, (nib_act >> k) & 1u);
                if (lane == 0) {
                    const uint32_t word = word0 + (kSlotsPerTile / 32) * k;
                    bits[word] = all | old_w[k];
                    if (record) {
                        uint32_t* rw = nv.rec_bits + static_cast<size_t>(row) * nv.n_words + word;
                        *rw = sub ? (*rw | wact) : wact;
                    }
                }
            }
            if ((flags & kFlagList) && wtotal) {
                uint32_t base = 0;
                if (lane == 0) base = atomicAdd(sl.count, wtotal);
                base = __shfl_sync(0xffffffffu, base, 0);
                const uint32_t below = (1u << lane) - 1u;
                const uint32_t vb = __ldg(vbase + net) + i0;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if ((nib_prop >> k) & 1u) sl.list[base + __popc(wprop[k] & below)] = vb + kSlotsPerTile * k;
                    base += __popc(wprop[k]);
                }
            }
        }
        // ---- population statistics: one sum per warp when the warp's neurons share a
        //      population, else one per (warp, population) by a segmented reduction
        if (stats) {
            const uint32_t pl = __shfl_sync(0xffffffffu, p_first, 0);
            const bool wuni = __all_sync(0xffffffffu, uniform && p_first == pl);
            if (wuni) {
                const int c = __reduce_add_sync(0xffffffffu, static_cast<unsigned>(cnt_acc));
                const long long v = warp_sum_ll(vs_acc);
                if (lane == 0) stat_add(nv, sa, row, pl, c, v);
            } else {
                warp_stat_segments(nv, sa, row, p_first, i0 < nv.n, cnt_acc, vs_acc, lane);
                warp_stat_segments(nv, sa, row, p_first + 1, cnt_nxt != 0 || vs_nxt != 0, cnt_nxt, vs_nxt, lane);
            }
        }
        const unsigned long long wev = warp_sum_ull(ev);
        if (lane == 0 && wev) atomicAdd(nv.events, wev);

        // barrier B: the stage holds the finished tile; store it, flush statistics
        __syncthreads();
        if (tid == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            bulk_store(nv.V + tile_first, st, kLifTile * sizeof(float));
            bulk_store(nv.iou + tile_first, st + kLifTile, kLifTile * sizeof(float));
            bulk_store(nv.tlast + tile_first, st + 2 * kLifTile, kLifTile * sizeof(float));
            if constexpr (JM != J_ASIS) bulk_store(nv.J + tile_first, st + 3 * kLifTile, kLifTile * sizeof(float4));
            bulk_commit();
        }
        if (stats && tid < kStatSlots) {
            const int c = s_cnt[it & 1u][tid];
            const long long v = s_vs[it & 1u][tid];
            if (c || v) {
                const size_t o = static_cast<size_t>(row) * nv.n_pops + (p_tile + tid);
                if (c) atomicAdd(nv.hist_cnt + o, c);
                atomicAdd(reinterpret_cast<unsigned long long*>(nv.hist_vsum + o), static_cast<unsigned long long>(v));
                s_cnt[it & 1u][tid] = 0;
                s_vs[it & 1u][tid] = 0;
            }
        }
        err = __reduce_or_sync(0xffffffffu, err);
        if (lane == 0 && err) atomicOr(&nv.clock->err, err);
        if (tid == 0) {
            t_last_tile = t;
            n_last_tile = last_sub ? n : n_prev;
            ++done_here;
        }
    }
    // the CTA's last stores complete before its tiles count towards the clock
    if (tid == 0) {
        bulk_wait_all();
        for (uint32_t q = 0; q < n_tk; ++q) lif_ticket(nets[s_tk_net[q]], s_tk_cnt[q], s_tk_t[q], s_tk_n[q]);
        if (done_here) lif_ticket(nets[cur_net], done_here, t_last_tile, n_last_tile);
    }
}

// Prefetch into L2 the 128-byte lines of a CSR span (targets and weight pairs),
// one line per lane: no registers stay live and nothing waits for the data.
template <int WT, int LANES = 32>
__device__ __forceinline__ void prefetch_span_l2(const uint32_t* col, const void* wts, unsigned long long e0,
                                                 uint32_t len, uint32_t lane) {
    if (len == 0) return;
    constexpr uint32_t kWB = WT == W_F32 ? 8 : (WT == W_U8 ? 2 : 4);
    const uintptr_t c0 = reinterpret_cast<uintptr_t>(col + e0) & ~uintptr_t(127);
    const uintptr_t c1 = reinterpret_cast<uintptr_t>(col + e0 + len);
    const uintptr_t w0 = (reinterpret_cast<uintptr_t>(wts) + e0 * kWB) & ~uintptr_t(127);
    const uintptr_t w1 = reinterpret_cast<uintptr_t>(wts) + (e0 + len) * kWB;
    const uint32_t nc = static_cast<uint32_t>((c1 - c0 + 127) >> 7), nw = static_cast<uint32_t>((w1 - w0 + 127) >> 7);
    for (uint32_t k = lane; k < nc + nw; k += LANES) {
        const uintptr_t a = k < nc ? c0 + (static_cast<uintptr_t>(k) << 7) : w0 + (static_cast<uintptr_t>(k - nc) << 7);
        asm volatile("prefetch.global.L2 [%0];" :: "l"(a));
    }
}

// ---------------------------------------------------------------------------
// Push propagation: one warp per spiking row of the out-degree CSR
// ---------------------------------------------------------------------------
template <int ACC, int WT, int kPushUnroll, int LPR, int LOCAL>
__device__ __forceinline__ void push_rows(const NetView* __restrict__ nets, const uint32_t* __restrict__ vbase, uint32_t n_nets,
                                          SpikeList sl) {
    // LPR lanes per row: 32 (a warp per row) or 16 / 8 (2 / 4 rows per warp, for short rows).
    // LOCAL: the own-population span of a row (own_seg) is left to push_local_kernel.
    constexpr uint32_t kGroups = 32 / LPR;
    const uint32_t count = *sl.count;
    const uint32_t lane = (threadIdx.x & 31u) % LPR;
    const uint32_t gw = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * kGroups + (threadIdx.x & 31u) / LPR;
    const uint32_t nw = ((gridDim.x * blockDim.x) >> 5) * kGroups;
    const unsigned long long* ptr = nets[0].out_ptr;
    const uint32_t* col = nets[0].out_col;
    const void* wts = nets[0].out_w;
    float4* J = nets[0].J;
    long long* dJ = nets[0].dJ;
    unsigned long long* dJf = nets[0].dJf;
    float fscale = nets[0].fix_scale;
    const uint2* own = LOCAL ? nets[0].own_seg : nullptr;
    const unsigned long long keep = l2_policy_keep();
    uint32_t vb = 0;
    for (uint32_t r = gw; r < count; r += nw) {
        const uint32_t v = __ldg(sl.list + r);
        if (n_nets > 1) {
            const uint32_t k = find_net(vbase, n_nets, v);
            vb = __ldg(vbase + k);
            ptr = nets[k].out_ptr;
            col = nets[k].out_col;
            wts = nets[k].out_w;
            J = nets[k].J;
            dJ = nets[k].dJ;
            dJf = nets[k].dJf;
            fscale = nets[k].fix_scale;
            if constexpr (LOCAL) own = nets[k].own_seg;
        }
        const uint32_t j = v - vb;
        const unsigned long long beg = __ldg(ptr + j), end = __ldg(ptr + j + 1);
        // virtual positions [0, len): [0, len1) -> beg + x, [len1, len) -> beg2 + (x - len1)
        unsigned long long len1 = end - beg, beg2 = end;
        if constexpr (LOCAL) {
            if (own) {
                const uint2 o = __ldg(own + j);
                len1 = o.x;
                beg2 = beg + o.y;
            }
        }
        const unsigned long long len = len1 + (end - beg2);
        for (unsigned long long x = lane; x < len; x += static_cast<unsigned long long>(LPR) * kPushUnroll) {
            uint32_t c[kPushUnroll];
            float2 w[kPushUnroll];
#pragma unroll
            for (int q = 0; q < kPushUnroll; ++q) {
                const unsigned long long xq = x + static_cast<unsigned long long>(LPR) * q;
                if (xq < len) {
                    const unsigned long long idx = LOCAL ? (xq < len1 ? beg + xq : beg2 + (xq - len1)) : beg + xq;
                    c[q] = __ldcs(col + idx);
                    w[q] = load_weight<WT>(wts, idx);
                }
            }
#pragma unroll
            for (int q = 0; q < kPushUnroll; ++q) {
                const unsigned long long xq = x + static_cast<unsigned long long>(LPR) * q;
                if (xq < len) {
                    const uint32_t target = c[q] & kIndexMask;
                    const uint32_t kind = c[q] >> 31;
                    if constexpr (ACC == ACC_FLOAT) {
                        red_add_f32x2_keep(reinterpret_cast<float2*>(J + target) + kind, w[q], keep);
                    } else if constexpr (ACC == ACC_FIXED) {
                        red_add_u64_keep(dJf + 2ull * target + kind, pack_fixed(w[q], fscale), keep);
                    } else {
                        unsigned long long* d = reinterpret_cast<unsigned long long*>(dJ) + static_cast<size_t>(target) * 4 + 2 * kind;
                        red_add_u64(d, static_cast<unsigned long long>(float_to_fix(w[q].x)));
                        red_add_u64(d + 1, static_cast<unsigned long long>(float_to_fix(w[q].y)));
                    }
                }
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(sl.ticket, 1u) == gridDim.x - 1) {
            *sl.count = 0u;
            *sl.ticket = 0u;
            __threadfence();
        }
    }
}

template <int ACC, int WT, int kPushUnroll, int LPR, int LOCAL = 0>
__global__ void __launch_bounds__(kPushThreads)
push_kernel(const NetView* __restrict__ nets, const uint32_t* __restrict__ vbase, uint32_t n_nets, SpikeList sl) {
    push_rows<ACC, WT, kPushUnroll, LPR, LOCAL>(nets, vbase, n_nets, sl);
}

// The cross-population part held to 64 registers (4 CTAs of 256 threads) for local:2016: two
// CTAs of it and the 512-thread window kernel (64 registers) fill exactly the SM's 65,536
// registers, so the two kernels really share every SM; at the 80 registers the compiler picks
// otherwise, a window CTA cannot start on an SM until the cross-population CTAs there have
// finished.  local:2008 keeps that 80-register form: held to 64 it also shared its SMs but ran
// 2 % slower on burst steps and no faster over whole runs of the regional network.
template <int ACC, int WT>
__global__ void __launch_bounds__(kPushThreads, 4)
push_kernel_cross64(const NetView* __restrict__ nets, const uint32_t* __restrict__ vbase, uint32_t n_nets, SpikeList sl) {
    push_rows<ACC, WT, 8, 32, 1>(nets, vbase, n_nets, sl);
}

// ---------------------------------------------------------------------------
// Population-local push, phase B.  Each population with local windows is cut
// into windows of at most kLocalWin neurons; a row's synapses into one window
// are a contiguous span (rows are sorted by postsynaptic neuron) between two
// woff boundaries.  The work of a step is split into units of up to
// kLocalUnitRows spiking rows of one window's population:
//
//   local_prep_kernel    spiking rows of each window's population (bitmap popcount);
//                        its last block turns them into the units' exclusive prefix
//                        and resets the unit counter
//   push_local_kernel    persistent, one 1024-thread CTA per SM: takes units from an
//                        atomic counter, finds the unit's rows by a block-wide prefix
//                        over the population's bitmap, sums their window spans into
//                        shared memory, and flushes the window to J with coalesced
//                        red.global.add.v4.f32 when it moves to another window.
//
// A bursting population becomes many units spread over every SM, so the step is
// balanced whatever the activity pattern; the L2 sees one 16-byte reduction per
// touched neuron per flush instead of one per synapse.
//
// The window sums are 32-bit fixed point: w is rounded to a multiple of 2^-s and
// added with red.shared.add.u32 (native, fire-and-forget; a shared-memory float
// atomic is a compare-and-swap loop whose latency stalls the warp).  s is chosen
// per population when the tables are built so that max|w| x (largest own-
// population in-degree) x 2^s + in-degree < 2^31: no sum can overflow, whatever
// spikes.  The regional network gets s = 21 (resolution 4.8e-7, below the
// rounding of float atomics onto J of order 10).
// ---------------------------------------------------------------------------
constexpr int kLocalThreads = 1024;
constexpr int kLocalThreadsShared = 768;   // window kernel beside a cross-population CTA on the same SM
constexpr int kLocalThreadsShared2 = 512;  // ... beside two
constexpr int kLocalUnroll = 8;
constexpr uint32_t kLocalUnitRows = 1024;   // spiking rows per work unit (measured: 256 / 512 / 1024 rows -> push 0.596 / 0.561 / 0.548 ms at 5M)
constexpr size_t kLocalSmem = 4ull * kLocalWin * sizeof(int) + kLocalUnitRows * (2 * sizeof(uint32_t) + sizeof(unsigned long long));

__device__ __forceinline__ void red_add_shared_u32(const void* p, uint32_t v) {
    asm volatile("red.shared.add.u32 [%0], %1;" :: "r"(static_cast<uint32_t>(__cvta_generic_to_shared(p))), "r"(v) : "memory");
}

// Spiking-row bitmap word wi of the population [p_lo, p_hi), bits outside masked off.
__device__ __forceinline__ uint32_t pop_word(const uint32_t* bits, uint32_t wi, uint32_t p_lo, uint32_t p_hi) {
    uint32_t m = bits[wi];
    const uint32_t b0 = wi << 5;
    if (b0 < p_lo) m &= ~0u << (p_lo - b0);
    if (p_hi - b0 < 32u) m &= (1u << (p_hi - b0)) - 1u;
    return m;
}

// Exclusive prefix of v over the block (blockDim.x a multiple of 32); *total = sum.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* s_warp, uint32_t* total) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= static_cast<uint32_t>(o)) incl += y;
    }
    __syncthreads();
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t x = lane < nw ? s_warp[lane] : 0u;
        uint32_t xi = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, xi, o);
            if (lane >= static_cast<uint32_t>(o)) xi += y;
        }
        if (lane < nw) s_warp[lane] = xi - x;
        if (lane == 31) s_warp[32] = xi;
    }
    __syncthreads();
    *total = s_warp[32];
    return s_warp[warp] + incl - v;
}

struct LocalWindow {
    const NetView* nv;
    uint32_t a, lo, hi, k, ka1, p_lo, p_hi;
    unsigned long long rb_k;
    float scale, unscale;
};

__device__ __forceinline__ void load_window(const NetView* __restrict__ nets, const uint32_t* __restrict__ win_prefix,
                                            uint32_t n_nets, uint32_t gwin, LocalWindow& W) {
    const uint32_t net = n_nets > 1 ? find_net(win_prefix, n_nets, gwin) : 0u;
    W.nv = nets + net;
    const uint4 wt = W.nv->win_tab[gwin - __ldg(win_prefix + net)];
    W.a = wt.x;
    W.lo = wt.y;
    W.hi = wt.z;
    W.k = wt.w & 0xFFFFu;
    const int sh = static_cast<int>(wt.w >> 16);     // fixed-point exponent s, 16..60
    W.scale = __int_as_float((127 + sh) << 23);      // 2^s
    W.unscale = __int_as_float((127 - sh) << 23);    // 2^-s
    const uint4 pl = W.nv->pop_loc[W.a];
    W.ka1 = pl.x + 1u;
    W.rb_k = (static_cast<unsigned long long>(pl.z) | (static_cast<unsigned long long>(pl.w) << 32)) + W.k;
    W.p_lo = __ldg(W.nv->pop_off + W.a);
    W.p_hi = __ldg(W.nv->pop_off + W.a + 1);
}

// scratch: [windows] spiking rows of each window's population, [windows + 1]
// unit prefix, [1] unit counter, [1] block ticket.  One block per window counts
// its population's spiking rows; the last block to finish (ticket) turns the
// counts into the unit prefix and resets the counter, so the window kernel that
// follows needs one launch before it instead of a count and a scan.
__global__ void __launch_bounds__(256)
local_prep_kernel(const NetView* __restrict__ nets, const uint32_t* __restrict__ win_prefix, uint32_t n_nets,
                  uint32_t windows, uint32_t* scratch) {
    __shared__ uint32_t s_warp[33];
    __shared__ uint32_t s_last;
    LocalWindow W;
    load_window(nets, win_prefix, n_nets, blockIdx.x, W);
    const uint32_t* bits = (W.nv->clock->n & 1ull) ? W.nv->bits1 : W.nv->bits0;
    uint32_t c = 0;
    for (uint32_t wi = (W.p_lo >> 5) + threadIdx.x; wi < ((W.p_hi + 31) >> 5); wi += blockDim.x)
        c += __popc(pop_word(bits, wi, W.p_lo, W.p_hi));
    uint32_t total;
    block_exclusive_scan(c, s_warp, &total);
    uint32_t* ticket = scratch + 2 * windows + 2;
    if (threadIdx.x == 0) {
        scratch[blockIdx.x] = total;
        __threadfence();
        s_last = atomicAdd(ticket, 1u) == windows - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    uint32_t* upre = scratch + windows;
    uint32_t carry = 0;
    for (uint32_t base = 0; base < windows; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t u = i < windows ? (__ldcg(scratch + i) + kLocalUnitRows - 1) / kLocalUnitRows : 0u;
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan(u, s_warp, &tot);
        if (i < windows) upre[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) {
        upre[windows] = carry;
        upre[windows + 1] = 0u;      // the unit counter
        *ticket = 0u;
    }
}

// Add the window's fixed-point sums to J (coalesced 16-byte reductions of the
// touched neurons) and clear them.  FIX: the sums are already in the network's
// fixed-mode units and go to dJf as two packed 64-bit integer reductions, so the
// result does not depend on which CTA flushes first.
template <bool FIX>
__device__ __forceinline__ void local_flush(const LocalWindow& W, int* acc) {
    __syncthreads();
    float4* J = W.nv->J + W.lo;
    unsigned long long* dJf = FIX ? W.nv->dJf + 2ull * W.lo : nullptr;
    const uint32_t width = W.hi - W.lo;
    const unsigned long long keep = l2_policy_keep();
    for (uint32_t i = threadIdx.x; i < width; i += blockDim.x) {
        const int4 v = make_int4(acc[i], acc[kLocalWin + i], acc[2 * kLocalWin + i], acc[3 * kLocalWin + i]);
        if (v.x | v.y | v.z | v.w) {
            if constexpr (FIX) {
                const unsigned long long u0 = static_cast<uint32_t>(v.x), u1 = static_cast<uint32_t>(v.y);
                const unsigned long long u2 = static_cast<uint32_t>(v.z), u3 = static_cast<uint32_t>(v.w);
                if (u0 | u1) red_add_u64_keep(dJf + 2ull * i, (u1 << 32) | u0, keep);
                if (u2 | u3) red_add_u64_keep(dJf + 2ull * i + 1, (u3 << 32) | u2, keep);
            } else {
                red_add_f32x4_keep(J + i, make_float4(__fmul_rn(__int2float_rn(v.x), W.unscale), __fmul_rn(__int2float_rn(v.y), W.unscale),
                                                 __fmul_rn(__int2float_rn(v.z), W.unscale), __fmul_rn(__int2float_rn(v.w), W.unscale)),
                                   keep);
            }
            acc[i] = 0;
            acc[kLocalWin + i] = 0;
            acc[2 * kLocalWin + i] = 0;
            acc[3 * kLocalWin + i] = 0;
        }
    }
    __syncthreads();
}

// launch bound of the full CTA for every NT: 64 registers, so the 768-thread form leaves a
// 256-thread push CTA room on the SM
template <int WT, int NT, int RL = 32, bool FIX = false>
__global__ void __launch_bounds__(kLocalThreads, 1)
push_local_kernel(const NetView* __restrict__ nets, const uint32_t* __restrict__ win_prefix, uint32_t n_nets,
                  uint32_t windows, uint32_t* scratch) {
    // plane c of kLocalWin 32-bit sums: random targets spread over all 32 banks
    extern __shared__ int acc[];
    uint32_t* s_rows = reinterpret_cast<uint32_t*>(acc + 4 * kLocalWin);
    uint32_t* s_len = s_rows + kLocalUnitRows;
    unsigned long long* s_start = reinterpret_cast<unsigned long long*>(s_len + kLocalUnitRows);
    __shared__ uint32_t s_warp[33];
    __shared__ uint32_t s_unit;
    const uint32_t* rows_of = scratch;
    const uint32_t* upre = scratch + windows;
    uint32_t* counter = scratch + 2 * windows + 1;
    const uint32_t total_units = upre[windows];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (uint32_t i = threadIdx.x; i < 4 * kLocalWin; i += NT) acc[i] = 0;
    LocalWindow W{};
    uint32_t cur = 0xFFFFFFFFu;
    for (;;) {
        if (threadIdx.x == 0) s_unit = atomicAdd(counter, 1u);
        __syncthreads();
        const uint32_t u = s_unit;
        if (u >= total_units) break;
        // the unit's window: the last w with upre[w] <= u (windows without units repeat a value)
        uint32_t lo_w = 0, hi_w = windows - 1;
        while (lo_w < hi_w) {
            const uint32_t mid = (lo_w + hi_w + 1) >> 1;
            if (upre[mid] <= u) lo_w = mid; else hi_w = mid - 1;
        }
        const uint32_t gw = lo_w;
        if (gw != cur) {
            if (cur != 0xFFFFFFFFu) local_flush<FIX>(W, acc);
            load_window(nets, win_prefix, n_nets, gw, W);
            if constexpr (FIX) W.scale = W.nv->fix_scale;   // sums in the network's fixed-mode units
            cur = gw;
        }
        const uint32_t r_lo = (u - upre[gw]) * kLocalUnitRows;
        const uint32_t r_hi = min(r_lo + kLocalUnitRows, rows_of[gw]);
        // rows with population rank in [r_lo, r_hi): block prefix over the bitmap
        const uint32_t* bits = (W.nv->clock->n & 1ull) ? W.nv->bits1 : W.nv->bits0;
        const uint32_t w_lo = W.p_lo >> 5, w_hi = (W.p_hi + 31) >> 5;
        const uint32_t per = (w_hi - w_lo + NT - 1) / NT;
        const uint32_t my_lo = min(w_lo + threadIdx.x * per, w_hi), my_hi = min(my_lo + per, w_hi);
        uint32_t c = 0;
        for (uint32_t wi = my_lo; wi < my_hi; ++wi) c += __popc(pop_word(bits, wi, W.p_lo, W.p_hi));
        uint32_t total;
        uint32_t rank = block_exclusive_scan(c, s_warp, &total);
        for (uint32_t wi = my_lo; wi < my_hi && rank < r_hi; ++wi) {
            uint32_t m = pop_word(bits, wi, W.p_lo, W.p_hi);
            if (rank + __popc(m) <= r_lo) { rank += __popc(m); continue; }
            while (m && rank < r_hi) {
                const uint32_t j = (wi << 5) + static_cast<uint32_t>(__ffs(m) - 1);
                m &= m - 1u;
                if (rank >= r_lo) s_rows[rank - r_lo] = j;
                ++rank;
            }
        }
        __syncthreads();
        const uint32_t nrows = r_hi - r_lo;
        // span of every row of the unit: [out_ptr[j] + woff[k], out_ptr[j] + woff[k + 1])
        const NetView& nv = *W.nv;
        for (uint32_t r = threadIdx.x; r < nrows; r += NT) {
            const uint32_t j = s_rows[r];
            const uint32_t* wo = nv.woff + W.rb_k + static_cast<unsigned long long>(j - W.p_lo) * W.ka1;
            const uint32_t s0 = __ldg(wo), s1 = __ldg(wo + 1);
            s_start[r] = __ldg(nv.out_ptr + j) + s0;
            s_len[r] = s1 - s0;
        }
        __syncthreads();
        const uint32_t* col = nv.out_col;
        const void* wts = nv.out_w;
        // RL lanes per row: 32 (a warp per row) or 16 (two rows per warp, for short spans)
        constexpr uint32_t kRows = 32 / RL;
        const uint32_t sl = lane % RL;
        const uint32_t rstride = (NT / 32) * kRows;
        for (uint32_t r = warp * kRows + lane / RL; r < nrows; r += rstride) {
            const unsigned long long e0 = s_start[r], e1 = e0 + s_len[r];
            // the next row of these lanes: pull its span into L2 while this row is summed
            // (measured: one row ahead beats two; prefetching in the scattered push made it slower)
            if (r + rstride < nrows)
                prefetch_span_l2<WT, RL>(col, wts, s_start[r + rstride], s_len[r + rstride], sl);
            for (unsigned long long e = e0 + sl; e < e1; e += static_cast<unsigned long long>(RL) * kLocalUnroll) {
                uint32_t cc[kLocalUnroll];
                float2 w[kLocalUnroll];
#pragma unroll
                for (int q = 0; q < kLocalUnroll; ++q) {
                    const unsigned long long idx = e + static_cast<unsigned long long>(RL) * q;
                    if (idx < e1) {
                        cc[q] = __ldcs(col + idx);
                        w[q] = load_weight<WT>(wts, idx);
                    }
                }
#pragma unroll
                for (int q = 0; q < kLocalUnroll; ++q) {
                    if (e + static_cast<unsigned long long>(RL) * q < e1) {
                        const int* d = acc + (cc[q] >> 31) * (2u * kLocalWin) + ((cc[q] & kIndexMask) - W.lo);
                        if constexpr (FIX) {
                            red_add_shared_u32(d, __float2uint_rn(__fmul_rn(w[q].x, W.scale)));
                            red_add_shared_u32(d + kLocalWin, __float2uint_rn(__fmul_rn(w[q].y, W.scale)));
                        } else {
                            red_add_shared_u32(d, static_cast<uint32_t>(__float2int_rn(__fmul_rn(w[q].x, W.scale))));
                            red_add_shared_u32(d + kLocalWin, static_cast<uint32_t>(__float2int_rn(__fmul_rn(w[q].y, W.scale))));
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
    if (cur != 0xFFFFFFFFu) local_flush<FIX>(W, acc);
}

__device__ inline uint32_t row_lower_bound(const uint32_t* __restrict__ col, unsigned long long beg,
                                           unsigned long long end, uint32_t target) {
    unsigned long long lo = beg, hi = end;
    while (lo < hi) {
        const unsigned long long mid = (lo + hi) >> 1;
        if ((__ldg(col + mid) & kIndexMask) < target) lo = mid + 1; else hi = mid;
    }
    return static_cast<uint32_t>(lo - beg);
}

// One warp per row.  Pass 1 (woff == nullptr): sortedness of every row, and per
// own-population synapse its target's count (own_cnt) and its population's
// largest |w| (maxw_bits, float bits of a non-negative value: ordered as
// integers).  Pass 2: own_seg and the window boundaries of every row whose
// population has local windows.
template <int WT>
__global__ void local_offsets_kernel(const unsigned long long* __restrict__ out_ptr, const uint32_t* __restrict__ col,
                                     const void* __restrict__ wts, const uint32_t* __restrict__ pop_off, uint32_t n_pops,
                                     uint32_t n, const uint4* __restrict__ pop_loc, uint32_t* own_cnt, uint32_t* maxw_bits,
                                     uint2* own_seg, uint32_t* woff, uint32_t* unsorted) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < n; j += nw) {
        const uint32_t a = find_pop(pop_off, n_pops, j);
        const unsigned long long beg = out_ptr[j], end = out_ptr[j + 1];
        const uint32_t p_lo = __ldg(pop_off + a), p_hi = __ldg(pop_off + a + 1);
        if (woff == nullptr) {
            bool bad = false;
            for (unsigned long long e = beg + lane; e + 1 < end; e += 32)
                bad |= (__ldg(col + e) & kIndexMask) > (__ldg(col + e + 1) & kIndexMask);
            if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(unsorted, 1u);
            const uint32_t s = row_lower_bound(col, beg, end, p_lo), t = row_lower_bound(col, beg, end, p_hi);
            float mx = 0.f;
            for (unsigned long long e = beg + s + lane; e < beg + t; e += 32) {
                atomicAdd(own_cnt + (__ldg(col + e) & kIndexMask), 1u);
                const float2 w = load_weight<WT>(wts, e);
                mx = fmaxf(mx, fmaxf(fabsf(w.x), fabsf(w.y)));
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            if (lane == 0 && mx > 0.f) atomicMax(maxw_bits + a, __float_as_uint(mx));
        } else {
            const uint4 pl = pop_loc[a];
            if (pl.x == 0) {
                if (lane == 0) own_seg[j] = make_uint2(0u, 0u);
                continue;
            }
            const unsigned long long rb = static_cast<unsigned long long>(pl.z) | (static_cast<unsigned long long>(pl.w) << 32);
            uint32_t* wo = woff + rb + static_cast<unsigned long long>(j - p_lo) * (pl.x + 1u);
            for (uint32_t k = lane; k <= pl.x; k += 32) {
                const uint32_t bnd = k == pl.x ? p_hi : static_cast<uint32_t>(min(static_cast<unsigned long long>(p_lo) + static_cast<unsigned long long>(k) * pl.y,
                                                                                   static_cast<unsigned long long>(p_hi)));
                wo[k] = row_lower_bound(col, beg, end, bnd);
            }
            if (lane == 0) own_seg[j] = make_uint2(row_lower_bound(col, beg, end, p_lo), row_lower_bound(col, beg, end, p_hi));
        }
    }
}

// ---------------------------------------------------------------------------
// Push propagation with TMA-staged row fetches.  Every warp owns a two-stage
// ring in shared memory; lane 0 issues bulk copies (cp.async.bulk, no
// multicast) of the next row chunk -- postsynaptic ids and weight pairs -- while
// the warp turns the current chunk into vector reductions.  Copies start on the
// 16-byte boundary at or below the chunk and end on the one at or above it (the
// CSR arrays carry 64 bytes of tail padding), and the consumer skips the slack.
// Every mbarrier wait is bounded: on timeout the kernel raises an error bit,
// waits (bounded) for its other copy in flight, and stops.
// ---------------------------------------------------------------------------
template <int WT> struct WBytes { static constexpr int v = 4; };
template <> struct WBytes<W_F32> { static constexpr int v = 8; };
template <> struct WBytes<W_U8> { static constexpr int v = 2; };

template <int WT, int CH>
struct TmaLayout {
    static constexpr int WB = WBytes<WT>::v;
    static constexpr int COLB = CH * 4 + 32;
    static constexpr int WTB = CH * WB + 32;
    static constexpr int STAGE = (COLB + WTB + 127) / 128 * 128;
    static constexpr int SMEM = kTmaWarps * 2 * STAGE + kTmaWarps * 2 * 8;
};

template <int WT>
__device__ __forceinline__ float2 smem_weight(const unsigned char* base, uint32_t e) {
    if constexpr (WT == W_F32) {
        return reinterpret_cast<const float2*>(base)[e];
    } else if constexpr (WT == W_BF16) {
        return __bfloat1622float2(reinterpret_cast<const __nv_bfloat162*>(base)[e]);
    } else if constexpr (WT == W_F16) {
        return __half22float2(reinterpret_cast<const __half2*>(base)[e]);
    } else {
        const uchar2 u = reinterpret_cast<const uchar2*>(base)[e];
        return make_float2(static_cast<float>(u.x) / 255.f, static_cast<float>(u.y) / 255.f);
    }
}

template <int ACC, int WT, int CH>
__global__ void __launch_bounds__(kTmaWarps * 32)
push_tma_kernel(const NetView* __restrict__ nets, const uint32_t* __restrict__ vbase, uint32_t n_nets, SpikeList sl) {
    using L = TmaLayout<WT, CH>;
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* ring = smem + warp * 2 * L::STAGE;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kTmaWarps * 2 * L::STAGE) + warp * 2;
    if (lane == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncwarp();
    const uint32_t count = *sl.count;
    const uint32_t nw = gridDim.x * kTmaWarps;
    const unsigned long long keep = l2_policy_keep();
    // producer cursor (lane-uniform): list index, remaining range of the row, its network
    uint32_t pr = blockIdx.x * kTmaWarps + warp;
    unsigned long long pc = 0, pe = 0;
    uint32_t pnet = 0;
    auto next_row = [&]() -> bool {
        while (pr < count) {
            const uint32_t v = __ldg(sl.list + pr);
            pnet = n_nets > 1 ? find_net(vbase, n_nets, v) : 0u;
            const uint32_t j = v - __ldg(vbase + pnet);
            const unsigned long long* ptr = nets[pnet].out_ptr;
            pc = __ldg(ptr + j);
            pe = __ldg(ptr + j + 1);
            if (pc < pe) return true;
            pr += nw;
        }
        return false;
    };
    bool have = next_row();
    uint32_t s_cnt[2] = {0, 0}, s_oc[2] = {0, 0}, s_ow[2] = {0, 0}, s_net[2] = {0, 0};
    bool s_full[2] = {false, false};
    uint32_t phase[2] = {0, 0};
    auto issue = [&](int stg) {
        const unsigned long long e0 = pc, e1 = min(pe, pc + static_cast<unsigned long long>(CH));
        const unsigned long long c0 = (e0 * 4) & ~15ull, c1 = (e1 * 4 + 15) & ~15ull;
        const unsigned long long w0 = (e0 * L::WB) & ~15ull, w1 = (e1 * L::WB + 15) & ~15ull;
        unsigned char* stage = ring + stg * L::STAGE;
        if (lane == 0) {
            const unsigned char* colb = reinterpret_cast<const unsigned char*>(nets[pnet].out_col);
            const unsigned char* wb = reinterpret_cast<const unsigned char*>(nets[pnet].out_w);
            mbar_expect_tx(&bars[stg], static_cast<uint32_t>((c1 - c0) + (w1 - w0)));
            bulk_load(stage, colb + c0, static_cast<uint32_t>(c1 - c0), &bars[stg]);
            bulk_load(stage + L::COLB, wb + w0, static_cast<uint32_t>(w1 - w0), &bars[stg]);
        }
        s_cnt[stg] = static_cast<uint32_t>(e1 - e0);
        s_oc[stg] = static_cast<uint32_t>((e0 * 4 - c0) / 4);
        s_ow[stg] = static_cast<uint32_t>((e0 * L::WB - w0) / L::WB);
        s_net[stg] = pnet;
        s_full[stg] = true;
        pc = e1;
        if (pc >= pe) {
            pr += nw;
            have = next_row();
        }
    };
    if (have) issue(0);
    int st = 0;
    bool failed = false;
    while (s_full[st]) {
        if (have) issue(st ^ 1);
        if (!mbar_wait_bounded(&bars[st], phase[st])) {
            failed = true;
            break;
        }
        phase[st] ^= 1;
        const unsigned char* stage = ring + st * L::STAGE;
        const uint32_t* scol = reinterpret_cast<const uint32_t*>(stage) + s_oc[st];
        const unsigned char* sw = stage + L::COLB;
        const uint32_t cnt = s_cnt[st], ow = s_ow[st];
        float4* J = nets[s_net[st]].J;
        long long* dJ = nets[s_net[st]].dJ;
        unsigned long long* dJf = nets[s_net[st]].dJf;
        const float fscale = nets[s_net[st]].fix_scale;
#pragma unroll 4
        for (uint32_t e = lane; e < cnt; e += 32) {
            const uint32_t c = scol[e];
            const float2 w = smem_weight<WT>(sw, ow + e);
            const uint32_t target = c & kIndexMask, kind = c >> 31;
            if constexpr (ACC == ACC_FLOAT) {
                red_add_f32x2_keep(reinterpret_cast<float2*>(J + target) + kind, w, keep);
            } else if constexpr (ACC == ACC_FIXED) {
                red_add_u64_keep(dJf + 2ull * target + kind, pack_fixed(w, fscale), keep);
            } else {
                unsigned long long* d = reinterpret_cast<unsigned long long*>(dJ) + static_cast<size_t>(target) * 4 + 2 * kind;
                red_add_u64(d, static_cast<unsigned long long>(float_to_fix(w.x)));
                red_add_u64(d + 1, static_cast<unsigned long long>(float_to_fix(w.y)));
            }
        }
        __syncwarp();
        s_full[st] = false;
        st ^= 1;
    }
    if (failed) {
        if (lane == 0) atomicOr(&nets[0].clock->err, kErrTimeout);
        // let the other copy in flight land before the CTA's shared memory is released
        if (s_full[st ^ 1]) mbar_wait_bounded(&bars[st ^ 1], phase[st ^ 1]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(sl.ticket, 1u) == gridDim.x - 1) {
            *sl.count = 0u;
            *sl.ticket = 0u;
            __threadfence();
        }
    }
}

// ---------------------------------------------------------------------------
// Deterministic in-degree gather of 32 neurons by one warp: lane k returns the
// exact fixed-point input of neuron base + k (sum over in-edges whose source
// spiked in `prev_bits`).
// ---------------------------------------------------------------------------
template <int WT>
__device__ inline void gather32(const NetView& nv, uint32_t base, const uint32_t* __restrict__ prev_bits,
                                int lane, long long acc_out[4]) {
    acc_out[0] = acc_out[1] = acc_out[2] = acc_out[3] = 0;
    const uint32_t last = min(base + 32u, nv.n);
    for (uint32_t j = base; j < last; ++j) {
        const unsigned long long beg = __ldg(nv.in_ptr + j), end = __ldg(nv.in_ptr + j + 1);
        long long a0 = 0, a1 = 0, a2 = 0, a3 = 0;
        for (unsigned long long e = beg + lane; e < end; e += 128) {
            uint32_t c[4];
            uint32_t hit = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const unsigned long long idx = e + 32ull * q;
                c[q] = idx < end ? __ldcs(nv.in_col + idx) : 0u;
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const unsigned long long idx = e + 32ull * q;
                if (idx < end) {
                    const uint32_t src = c[q] & kIndexMask;
                    hit |= ((__ldg(prev_bits + (src >> 5)) >> (src & 31u)) & 1u) << q;
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if ((hit >> q) & 1u) {
                    const float2 w = load_weight<WT>(nv.in_w, e + 32ull * q);
                    const long long f0 = float_to_fix(w.x), f1 = float_to_fix(w.y);
                    if (c[q] >> 31) { a2 += f0; a3 += f1; } else { a0 += f0; a1 += f1; }
                }
            }
        }
        a0 = warp_sum_ll(a0);
        a1 = warp_sum_ll(a1);
        a2 = warp_sum_ll(a2);
        a3 = warp_sum_ll(a3);
        if (static_cast<uint32_t>(lane) == j - base) {
            acc_out[0] = a0; acc_out[1] = a1; acc_out[2] = a2; acc_out[3] = a3;
        }
    }
}

// Pull-fused LIF step: GATHER=1 folds last step's spikes into J first; GATHER=0
// (first step of a run) takes J as complete.
template <int GATHER, int WT>
__global__ void __launch_bounds__(kPullThreads)
lif_pull_kernel(const NetView* __restrict__ nets, const uint32_t* __restrict__ tile_prefix, uint32_t n_nets,
                uint32_t flags, int prop_mode) {
    __shared__ NetView s_nv;
    __shared__ uint32_t s_net, s_tile, s_p0;
    __shared__ unsigned long long s_events;
    __shared__ int s_cnt[kStatSlots];
    __shared__ long long s_vs[kStatSlots];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        const uint32_t k = n_nets > 1 ? find_net(tile_prefix, n_nets, blockIdx.x) : 0u;
        s_net = k;
        s_tile = blockIdx.x - __ldg(tile_prefix + k);
        s_events = 0ull;
    }
    if (tid < kStatSlots) { s_cnt[tid] = 0; s_vs[tid] = 0; }
    __syncthreads();
    load_netview(s_nv, nets + s_net);
    __syncthreads();
    const NetView& nv = s_nv;
    const float t_prev = nv.clock->t;
    const unsigned long long n_prev = nv.clock->n;
    const unsigned long long run_base = nv.clock->run_base;
    const unsigned long long inj_base = nv.clock->inj_base;
    const unsigned long long n = n_prev + 1;
    const float t = __fadd_rn(t_prev, nv.dt);
    const uint32_t parity = static_cast<uint32_t>(n & 1ull);
    const uint32_t tile_first = s_tile * kPullTile;
    const uint32_t base = tile_first + warp * 32;
    const uint32_t i = base + lane;
    uint32_t err = 0;
    const long long row = static_cast<long long>(n - run_base - 1);
    bool stats = (flags & kFlagStats) != 0;
    bool record = (flags & kFlagRecord) != 0 && nv.rec_bits != nullptr;
    if ((stats || record) && (row < 0 || row >= static_cast<long long>(nv.hist_cap))) {
        stats = false; record = false; err |= kErrHistOverflow;
    }
    if (tid == 0) s_p0 = find_pop(nv.pop_off, nv.n_pops, min(tile_first, nv.n - 1));
    __syncthreads();
    StatAcc sa{s_cnt, s_vs, s_p0};

    long long acc[4] = {0, 0, 0, 0};
    if constexpr (GATHER) {
        const uint32_t* prev = parity ? nv.bits0 : nv.bits1;
        gather32<WT>(nv, base, prev, lane, acc);
    }
    const bool valid = i < nv.n;
    bool active = false, sp = false;
    float vnew = 0.f;
    uint32_t p = 0;
    if (valid) {
        p = find_pop(nv.pop_off, nv.n_pops, i);
        PopParams pp;
        load_pop_params(nv, p, i, pp);
        float4 Jv = nv.J[i];
        float* Jc = reinterpret_cast<float*>(&Jv);
        NeuronIn in;
        in.V = nv.V[i];
        in.iou = nv.iou[i];
        in.tlast = nv.tlast[i];
#pragma unroll
        for (int c = 0; c < 4; ++c) in.J[c] = GATHER ? decay_add(Jc[c], pp.decay[c], fix_to_float(acc[c])) : Jc[c];
        float z, u = 1.f;
        draw_noise1(nv, i, n, inj_base, (flags & kFlagInjected) != 0, prop_mode != PROP_THRESHOLD, z, u, err);
        const NeuronOut o = lif_update(pp, in, t, z, (flags & kFlagUseOU) != 0);
        nv.V[i] = o.V;
        nv.iou[i] = o.iou;
        nv.tlast[i] = o.tlast;
        if constexpr (GATHER) nv.J[i] = make_float4(in.J[0], in.J[1], in.J[2], in.J[3]);
        active = o.active;
        vnew = o.V;
        sp = propagated(prop_mode, o.active, u, pp.noise_rate);
    }
    const uint32_t wprop = __ballot_sync(0xffffffffu, sp);
    const uint32_t wact = __ballot_sync(0xffffffffu, active);
    if ((flags & kFlagSample) && nv.n_samples && valid && row >= 0 && row < static_cast<long long>(nv.hist_cap)) {
        const uint32_t sbw = __ldg(nv.sample_bits + (i >> 5));
        if ((sbw >> (i & 31u)) & 1u) {
            const uint32_t slot = __ldg(nv.sample_pre + (i >> 5)) + __popc(sbw & ((1u << (i & 31u)) - 1u));
            const size_t o = static_cast<size_t>(row) * nv.n_samples + slot;
            nv.hist_sspk[o] = active ? 1 : 0;
            nv.hist_sv[o] = vnew;
            nv.hist_siou[o] = nv.iou[i];
        }
    }
    if (lane == 0) {
        uint32_t* bits = parity ? nv.bits1 : nv.bits0;
        bits[base >> 5] = wprop;
        if (record) nv.rec_bits[static_cast<size_t>(row) * nv.n_words + (base >> 5)] = wact;
    }
    const unsigned long long ev = warp_sum_ull(sp ? static_cast<unsigned long long>(__ldg(nv.out_deg + i)) : 0ull);
    if (lane == 0 && ev) atomicAdd(&s_events, ev);
    if (stats) {
        const bool inc = valid && !excluded(nv, i);
        const uint32_t pl = __shfl_sync(0xffffffffu, p, 0);
        const bool wuni = __all_sync(0xffffffffu, !valid || (inc && p == pl)) && __any_sync(0xffffffffu, valid);
        const int c = inc && active ? 1 : 0;
        const long long v = inc ? v_fix(vnew) : 0;
        if (wuni) {
            const int cs = __reduce_add_sync(0xffffffffu, static_cast<unsigned>(c));
            const long long vs = warp_sum_ll(v);
            if (lane == 0) stat_add(nv, sa, row, pl, cs, vs);
        } else if (inc) {
            stat_add(nv, sa, row, p, c, v);
        }
    }
    __syncthreads();
    if (tid == 0 && s_events) atomicAdd(nv.events, s_events);
    if (stats && tid < kStatSlots) {
        const int c = s_cnt[tid];
        const long long v = s_vs[tid];
        if (c || v) {
            const size_t o = static_cast<size_t>(row) * nv.n_pops + (s_p0 + tid);
            if (c) atomicAdd(nv.hist_cnt + o, c);
            atomicAdd(reinterpret_cast<unsigned long long*>(nv.hist_vsum + o), static_cast<unsigned long long>(v));
        }
    }
    advance_clock(nv, nv.n_pad / kPullTile, t, n, err);
}

// End of an exact- or fixed-push run: J <- J*decay + dJ (or dJf), the sums <- 0
// (J becomes complete).
template <int ACC>
__global__ void __launch_bounds__(kLifThreads)
fold_finish_kernel(const NetView* __restrict__ nets, const uint32_t* __restrict__ tile_prefix, uint32_t n_nets) {
    const uint32_t k = n_nets > 1 ? find_net(tile_prefix, n_nets, blockIdx.x) : 0u;
    const NetView& nv = nets[k];
    const uint32_t tile = blockIdx.x - __ldg(tile_prefix + k);
    const uint32_t i0 = tile * kLifTile + threadIdx.x * 4;
    const uint32_t n = nv.n;
    uint32_t p = find_pop(nv.pop_off, nv.n_pops, min(i0, n - 1));
    for (int q = 0; q < 4; ++q) {
        const uint32_t i = i0 + q;
        if (i >= n) break;
        while (p + 1 < nv.n_pops && __ldg(nv.pop_off + p + 1) <= i) ++p;
        PopParams pp;
        load_pop_params(nv, p, i, pp);
        float4 Jv = nv.J[i];
        float* Jc = reinterpret_cast<float*>(&Jv);
        if constexpr (ACC == ACC_FIXED) {
            unsigned long long* d = nv.dJf + 2ull * i;
#pragma unroll
            for (int c = 0; c < 4; ++c) Jc[c] = decay_add(Jc[c], pp.decay[c], fixed_field(d[c >> 1], c & 1, nv.fix_unscale));
            d[0] = 0ull;
            d[1] = 0ull;
        } else {
            long long* d = nv.dJ + static_cast<size_t>(i) * 4;
#pragma unroll
            for (int c = 0; c < 4; ++c) { Jc[c] = decay_add(Jc[c], pp.decay[c], fix_to_float(d[c])); d[c] = 0; }
        }
        nv.J[i] = Jv;
    }
}

// End of a pull run: J <- J*decay + gather(last step's spikes).
template <int WT>
__global__ void __launch_bounds__(kPullThreads)
gather_finish_kernel(const NetView* __restrict__ nets, const uint32_t* __restrict__ tile_prefix, uint32_t n_nets) {
    const uint32_t k = n_nets > 1 ? find_net(tile_prefix, n_nets, blockIdx.x) : 0u;
    const NetView& nv = nets[k];
    const uint32_t tile = blockIdx.x - __ldg(tile_prefix + k);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t base = tile * kPullTile + warp * 32;
    const unsigned long long n = nv.clock->n;
    const uint32_t* last = (n & 1ull) ? nv.bits1 : nv.bits0;
    long long acc[4];
    gather32<WT>(nv, base, last, lane, acc);
    const uint32_t i = base + lane;
    if (i < nv.n) {
        const uint32_t p = find_pop(nv.pop_off, nv.n_pops, i);
        PopParams pp;
        load_pop_params(nv, p, i, pp);
        float4 Jv = nv.J[i];
        float* Jc = reinterpret_cast<float*>(&Jv);
#pragma unroll
        for (int c = 0; c < 4; ++c) Jc[c] = decay_add(Jc[c], pp.decay[c], fix_to_float(acc[c]));
        nv.J[i] = Jv;
    }
}

// ---------------------------------------------------------------------------
// End-of-step synaptic currents per population: output_imean and
// output_receptor_imeas (stat_result.cpp:269-380; block_new.py:152-156, the
// mean_psc of every population).  Runs after the step's push, when J is
// complete: I_u = g_u (V_u - V) J_u and I_syn = ((I_0 + I_1) + I_2) + I_3 in
// the LIF step's operation order, V after the step.  Sums are fixed point
// (2^24, like the V sums) so batches and reruns agree bit for bit; neurons
// excluded from statistics are skipped.
// ---------------------------------------------------------------------------
template <int JM>
__global__ void __launch_bounds__(256)
stat_isyn_kernel(const NetView* __restrict__ nets, const uint32_t* __restrict__ tile_prefix, uint32_t n_nets,
                 uint32_t total_tiles) {
    __shared__ unsigned long long s_is[kStatSlots][5];
    const uint32_t tid = threadIdx.x, lane = tid & 31u;
    for (uint32_t gt = blockIdx.x; gt < total_tiles; gt += gridDim.x) {
        const uint32_t net = n_nets > 1 ? find_net(tile_prefix, n_nets, gt) : 0u;
        const NetView& nv = nets[net];
        const long long row = static_cast<long long>(nv.clock->n - nv.clock->run_base) - 1;
        if (nv.hist_isum == nullptr || row < 0 || row >= static_cast<long long>(nv.isum_cap)) continue;
        const bool sampled = nv.hist_sisyn != nullptr && nv.n_samples != 0;
        for (uint32_t q = tid; q < kStatSlots * 5; q += blockDim.x) (&s_is[0][0])[q] = 0ull;
        __syncthreads();
        const uint32_t tile = gt - __ldg(tile_prefix + net);
        const uint32_t p_tile = __ldg(nv.tile_pop + tile);
        const uint32_t i0 = tile * kLifTile + tid * 4;
        uint32_t p = p_tile;
        const uint32_t i_first = min(i0, nv.n - 1);
        while (p + 1 < nv.n_pops && __ldg(nv.pop_off + p + 1) <= i_first) ++p;
        const uint32_t p_first = p;
        PopParams pp;
        load_pop_params(nv, p, i_first, pp);
        long long acc[5] = {0, 0, 0, 0, 0};
        bool uniform = true;
        for (int k = 0; k < 4; ++k) {
            const uint32_t i = i0 + k;
            if (i >= nv.n) { uniform = false; continue; }
            if (p + 1 < nv.n_pops && __ldg(nv.pop_off + p + 1) <= i) {
                while (p + 1 < nv.n_pops && __ldg(nv.pop_off + p + 1) <= i) ++p;
                if (!nv.per_neuron) load_pop_params(nv, p, i, pp);
            }
            if (nv.per_neuron && k > 0) load_pop_params(nv, p, i, pp);
            if (excluded(nv, i)) { uniform = false; continue; }
            const float V = nv.V[i];
            const float4 Jv = nv.J[i];
            float J[4] = {Jv.x, Jv.y, Jv.z, Jv.w};
            if constexpr (JM == J_FOLD) {
                const long long* d = nv.dJ + static_cast<size_t>(i) * 4;
#pragma unroll
                for (int c = 0; c < 4; ++c) J[c] = decay_add(J[c], pp.decay[c], fix_to_float(d[c]));
            } else if constexpr (JM == J_FIXF) {
                const unsigned long long* d = nv.dJf + 2ull * i;
#pragma unroll
                for (int c = 0; c < 4; ++c) J[c] = decay_add(J[c], pp.decay[c], fixed_field(d[c >> 1], c & 1, nv.fix_unscale));
            }
            float I[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) I[c] = __fmul_rn(__fmul_rn(pp.g[c], __fsub_rn(pp.Vu[c], V)), J[c]);
            const float isyn = __fadd_rn(__fadd_rn(__fadd_rn(I[0], I[1]), I[2]), I[3]);
            if (sampled) {
                const uint32_t sw = __ldg(nv.sample_bits + (i >> 5)), sb = 1u << (i & 31);
                if (sw & sb)
                    nv.hist_sisyn[static_cast<size_t>(row) * nv.n_samples + __ldg(nv.sample_pre + (i >> 5)) + __popc(sw & (sb - 1u))] = isyn;
            }
            long long q[5] = {v_fix(isyn), v_fix(I[0]), v_fix(I[1]), v_fix(I[2]), v_fix(I[3])};
            if (p == p_first) {
#pragma unroll
                for (int c = 0; c < 5; ++c) acc[c] += q[c];
            } else {
                uniform = false;
                const uint32_t slot = p - p_tile;
#pragma unroll
                for (int c = 0; c < 5; ++c) {
                    if (slot < static_cast<uint32_t>(kStatSlots)) atomicAdd(&s_is[slot][c], static_cast<unsigned long long>(q[c]));
                    else atomicAdd(reinterpret_cast<unsigned long long*>(nv.hist_isum) + (static_cast<size_t>(row) * nv.n_pops + p) * 5 + c,
                                   static_cast<unsigned long long>(q[c]));
                }
            }
        }
        const uint32_t pl = __shfl_sync(0xffffffffu, p_first, 0);
        const bool wuni = __all_sync(0xffffffffu, uniform && p_first == pl);
        if (wuni) {
#pragma unroll
            for (int c = 0; c < 5; ++c) acc[c] = warp_sum_ll(acc[c]);
        }
        if ((wuni && lane == 0) || (!wuni && i0 < nv.n)) {
            const uint32_t slot = (wuni ? pl : p_first) - p_tile;
            const uint32_t pp_ = wuni ? pl : p_first;
#pragma unroll
            for (int c = 0; c < 5; ++c) {
                if (!acc[c]) continue;
                if (slot < static_cast<uint32_t>(kStatSlots)) atomicAdd(&s_is[slot][c], static_cast<unsigned long long>(acc[c]));
                else atomicAdd(reinterpret_cast<unsigned long long*>(nv.hist_isum) + (static_cast<size_t>(row) * nv.n_pops + pp_) * 5 + c,
                               static_cast<unsigned long long>(acc[c]));
            }
        }
        __syncthreads();
        for (uint32_t q = tid; q < kStatSlots * 5; q += blockDim.x) {
            const uint32_t slot = q / 5, c = q % 5;
            const unsigned long long v = s_is[slot][c];
            if (v && p_tile + slot < nv.n_pops)
                atomicAdd(reinterpret_cast<unsigned long long*>(nv.hist_isum) + (static_cast<size_t>(row) * nv.n_pops + p_tile + slot) * 5 + c, v);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Host-side launchers
// ---------------------------------------------------------------------------
cudaError_t launch_lif(const LaunchBatch& b, int jmode, uint32_t flags, int prop_mode, cudaStream_t s) {
    if (b.lif_tiles_total == 0) return cudaSuccess;
    // dynamic shared memory above 48 KiB needs an opt-in per kernel and device
    static std::atomic<uint32_t> attr_set{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint32_t bit = 1u << (dev & 31);
    if (!(attr_set.load() & bit)) {
        for (auto fn : {lif_kernel<J_DIRECT>, lif_kernel<J_FOLD>, lif_kernel<J_ASIS>, lif_kernel<J_FIXF>}) {
            e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kLifSmem));
            if (e != cudaSuccess) return e;
        }
        attr_set.fetch_or(bit);
    }
    const uint32_t T = b.lif_tiles_total;
    const uint32_t chunk = std::max(1u, b.lif_chunk);
    const dim3 grid(std::min((T + chunk - 1) / chunk, b.lif_ctas)), block(kLifThreads);
    switch (jmode) {
        case J_DIRECT: lif_kernel<J_DIRECT><<<grid, block, kLifSmem, s>>>(b.nets, b.lif_prefix, b.vbase, b.n_nets, T, b.spikes, flags, prop_mode, b.tile_net, chunk); break;
        case J_FOLD: lif_kernel<J_FOLD><<<grid, block, kLifSmem, s>>>(b.nets, b.lif_prefix, b.vbase, b.n_nets, T, b.spikes, flags, prop_mode, b.tile_net, chunk); break;
        case J_FIXF: lif_kernel<J_FIXF><<<grid, block, kLifSmem, s>>>(b.nets, b.lif_prefix, b.vbase, b.n_nets, T, b.spikes, flags, prop_mode, b.tile_net, chunk); break;
        default: lif_kernel<J_ASIS><<<grid, block, kLifSmem, s>>>(b.nets, b.lif_prefix, b.vbase, b.n_nets, T, b.spikes, flags, prop_mode, b.tile_net, chunk); break;
    }
    return cudaGetLastError();
}

template <int ACC, int WT>
static cudaError_t push_launch_wt(const LaunchBatch& b, const PushCfg& cfg, uint32_t ctas, cudaStream_t s) {
    constexpr bool FIX = ACC == ACC_FIXED;
    if (cfg.kind == PUSH_LOCAL && ACC != ACC_EXACT &&
        (cfg.param == kLocalConcurrent || cfg.param == kLocalConcurrent2 || cfg.param == kLocalConcurrentHalf) &&
        b.aux && b.windows_total) {
        // cross-population spans on the auxiliary stream, one (two) 256-thread CTA(s) per SM, next
        // to the window kernel's 768 (512)-thread CTA: L2 reductions and shared-memory sums overlap
        const bool two = cfg.param == kLocalConcurrent2;
        cudaError_t e = cudaEventRecord(b.ev_fork, s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b.aux, b.ev_fork, 0);
        if (e != cudaSuccess) return e;
        if (two)
            push_kernel_cross64<ACC, WT><<<b.sm_count * 2u, kPushThreads, 0, b.aux>>>(b.nets, b.vbase, b.n_nets, b.spikes);
        else
            push_kernel<ACC, WT, 8, 32, 1><<<b.sm_count, kPushThreads, 0, b.aux>>>(b.nets, b.vbase, b.n_nets, b.spikes);
        e = cudaEventRecord(b.ev_join, b.aux);
        if (e != cudaSuccess) return e;
        local_prep_kernel<<<b.windows_total, 256, 0, s>>>(b.nets, b.win_prefix, b.n_nets, b.windows_total, b.local_scratch);
        if (two)
            push_local_kernel<WT, kLocalThreadsShared2, 32, FIX><<<b.sm_count, kLocalThreadsShared2, kLocalSmem, s>>>(
                b.nets, b.win_prefix, b.n_nets, b.windows_total, b.local_scratch);
        else if (cfg.param == kLocalConcurrentHalf)
            push_local_kernel<WT, kLocalThreadsShared, 16, FIX><<<b.sm_count, kLocalThreadsShared, kLocalSmem, s>>>(
                b.nets, b.win_prefix, b.n_nets, b.windows_total, b.local_scratch);
        else
            push_local_kernel<WT, kLocalThreadsShared, 32, FIX><<<b.sm_count, kLocalThreadsShared, kLocalSmem, s>>>(
                b.nets, b.win_prefix, b.n_nets, b.windows_total, b.local_scratch);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, b.ev_join, 0);
        return e;
    }
    if (cfg.kind == PUSH_LOCAL && ACC != ACC_EXACT) {
        const dim3 grid(ctas), block(kPushThreads);
        if (cfg.lpr == 16)
            push_kernel<ACC, WT, 8, 16, 1><<<grid, block, 0, s>>>(b.nets, b.vbase, b.n_nets, b.spikes);
        else
            push_kernel<ACC, WT, 8, 32, 1><<<grid, block, 0, s>>>(b.nets, b.vbase, b.n_nets, b.spikes);
        if (b.windows_total) {
            local_prep_kernel<<<b.windows_total, 256, 0, s>>>(b.nets, b.win_prefix, b.n_nets, b.windows_total, b.local_scratch);
            push_local_kernel<WT, kLocalThreads, 32, FIX><<<b.sm_count, kLocalThreads, kLocalSmem, s>>>(
                b.nets, b.win_prefix, b.n_nets, b.windows_total, b.local_scratch);
        }
    } else if (cfg.kind == PUSH_REG || cfg.kind == PUSH_LOCAL) {
        const dim3 grid(ctas), block(kPushThreads);
        if (cfg.lpr == 16) {
            push_kernel<ACC, WT, 8, 16><<<grid, block, 0, s>>>(b.nets, b.vbase, b.n_nets, b.spikes);
        } else if (cfg.lpr == 8) {
            push_kernel<ACC, WT, 8, 8><<<grid, block, 0, s>>>(b.nets, b.vbase, b.n_nets, b.spikes);
        } else {
            switch (cfg.param) {
                case 4: push_kernel<ACC, WT, 4, 32><<<grid, block, 0, s>>>(b.nets, b.vbase, b.n_nets, b.spikes); break;
                case 16: push_kernel<ACC, WT, 16, 32><<<grid, block, 0, s>>>(b.nets, b.vbase, b.n_nets, b.spikes); break;
                default: push_kernel<ACC, WT, 8, 32><<<grid, block, 0, s>>>(b.nets, b.vbase, b.n_nets, b.spikes); break;
            }
        }
    } else {
        const dim3 grid(ctas), block(kTmaWarps * 32);
        if (cfg.param == 256) {
            using L = TmaLayout<WT, 256>;
            push_tma_kernel<ACC, WT, 256><<<grid, block, L::SMEM, s>>>(b.nets, b.vbase, b.n_nets, b.spikes);
        } else {
            using L = TmaLayout<WT, 512>;
            push_tma_kernel<ACC, WT, 512><<<grid, block, L::SMEM, s>>>(b.nets, b.vbase, b.n_nets, b.spikes);
        }
    }
    return cudaGetLastError();
}

template <int ACC, int WT>
static cudaError_t push_prepare_wt(const PushCfg& cfg, int sm_count, uint32_t* ctas) {
    int per_sm = 0;
    cudaError_t e = cudaSuccess;
    if (cfg.kind == PUSH_LOCAL && ACC != ACC_EXACT) {
        constexpr bool FIX = ACC == ACC_FIXED;
        for (auto fn : {push_local_kernel<WT, kLocalThreads, 32, FIX>, push_local_kernel<WT, kLocalThreadsShared, 32, FIX>,
                        push_local_kernel<WT, kLocalThreadsShared2, 32, FIX>, push_local_kernel<WT, kLocalThreadsShared, 16, FIX>})
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kLocalSmem));
        // the cross-population CTAs land on an SM first: ask for the largest shared-memory
        // carve-out so a window CTA (229 KB) can join them there
        for (auto fn : {push_kernel<ACC, WT, 8, 32, 1>, push_kernel<ACC, WT, 8, 16, 1>, push_kernel_cross64<ACC, WT>})
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         static_cast<int>(cudaSharedmemCarveoutMaxShared));
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cfg.lpr == 16 ? push_kernel<ACC, WT, 8, 16, 1> : push_kernel<ACC, WT, 8, 32, 1>,
                                                              kPushThreads, 0);
    } else if (cfg.kind == PUSH_REG || cfg.kind == PUSH_LOCAL) {
        if (cfg.lpr == 16) {
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, push_kernel<ACC, WT, 8, 16>, kPushThreads, 0);
        } else if (cfg.lpr == 8) {
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, push_kernel<ACC, WT, 8, 8>, kPushThreads, 0);
        } else {
            switch (cfg.param) {
                case 4: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, push_kernel<ACC, WT, 4, 32>, kPushThreads, 0); break;
                case 16: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, push_kernel<ACC, WT, 16, 32>, kPushThreads, 0); break;
                default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, push_kernel<ACC, WT, 8, 32>, kPushThreads, 0); break;
            }
        }
    } else if (cfg.param == 256) {
        using L = TmaLayout<WT, 256>;
        e = cudaFuncSetAttribute(push_tma_kernel<ACC, WT, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::SMEM);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, push_tma_kernel<ACC, WT, 256>, kTmaWarps * 32, L::SMEM);
    } else {
        using L = TmaLayout<WT, 512>;
        e = cudaFuncSetAttribute(push_tma_kernel<ACC, WT, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::SMEM);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, push_tma_kernel<ACC, WT, 512>, kTmaWarps * 32, L::SMEM);
    }
    if (e != cudaSuccess) return e;
    *ctas = static_cast<uint32_t>(std::max(1, per_sm) * sm_count);
    return cudaSuccess;
}

template <int ACC>
static cudaError_t push_launch_acc(const LaunchBatch& b, int wt, const PushCfg& cfg, uint32_t ctas, cudaStream_t s) {
    switch (wt) {
        case W_F32: return push_launch_wt<ACC, W_F32>(b, cfg, ctas, s);
        case W_BF16: return push_launch_wt<ACC, W_BF16>(b, cfg, ctas, s);
        case W_F16: return push_launch_wt<ACC, W_F16>(b, cfg, ctas, s);
        default: return push_launch_wt<ACC, W_U8>(b, cfg, ctas, s);
    }
}

const PushCfg kPushCands[kPushCandidates] = {{PUSH_REG, 4, 32}, {PUSH_REG, 8, 32}, {PUSH_REG, 16, 32},
                                             {PUSH_REG, 8, 16}, {PUSH_REG, 8, 8},
                                             {PUSH_TMA, 256, 32}, {PUSH_TMA, 512, 32},
                                             {PUSH_LOCAL, 8, 32}, {PUSH_LOCAL, 8, 16},
                                             {PUSH_LOCAL, kLocalConcurrent, 32}, {PUSH_LOCAL, kLocalConcurrent2, 32},
                                             {PUSH_LOCAL, kLocalConcurrentHalf, 32}};

template <int ACC>
static cudaError_t push_prepare_acc(int wt, const PushCfg& cfg, int sm_count, uint32_t* ctas) {
    switch (wt) {
        case W_F32: return push_prepare_wt<ACC, W_F32>(cfg, sm_count, ctas);
        case W_BF16: return push_prepare_wt<ACC, W_BF16>(cfg, sm_count, ctas);
        case W_F16: return push_prepare_wt<ACC, W_F16>(cfg, sm_count, ctas);
        default: return push_prepare_wt<ACC, W_U8>(cfg, sm_count, ctas);
    }
}

cudaError_t push_prepare(int acc, int wt, const PushCfg& cfg, int sm_count, uint32_t* ctas) {
    switch (acc) {
        case ACC_EXACT: return push_prepare_acc<ACC_EXACT>(wt, cfg, sm_count, ctas);
        case ACC_FIXED: return push_prepare_acc<ACC_FIXED>(wt, cfg, sm_count, ctas);
        default: return push_prepare_acc<ACC_FLOAT>(wt, cfg, sm_count, ctas);
    }
}

cudaError_t launch_push(const LaunchBatch& b, int acc, int wt, const PushCfg& cfg, uint32_t ctas, cudaStream_t s) {
    switch (acc) {
        case ACC_EXACT: return push_launch_acc<ACC_EXACT>(b, wt, cfg, ctas, s);
        case ACC_FIXED: return push_launch_acc<ACC_FIXED>(b, wt, cfg, ctas, s);
        default: return push_launch_acc<ACC_FLOAT>(b, wt, cfg, ctas, s);
    }
}

cudaError_t build_local_offsets(const unsigned long long* out_ptr, const uint32_t* out_col, const void* out_w, int wt,
                                const uint32_t* pop_off, uint32_t n_pops, uint32_t n, const uint4* pop_loc,
                                uint32_t* own_cnt, uint32_t* maxw_bits, uint2* own_seg, uint32_t* woff,
                                uint32_t* unsorted, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const uint32_t blocks = std::min<uint32_t>((n + 7) / 8, 148u * 64u);
    switch (wt) {
        case W_F32: local_offsets_kernel<W_F32><<<blocks, 256, 0, s>>>(out_ptr, out_col, out_w, pop_off, n_pops, n, pop_loc, own_cnt, maxw_bits, own_seg, woff, unsorted); break;
        case W_BF16: local_offsets_kernel<W_BF16><<<blocks, 256, 0, s>>>(out_ptr, out_col, out_w, pop_off, n_pops, n, pop_loc, own_cnt, maxw_bits, own_seg, woff, unsorted); break;
        case W_F16: local_offsets_kernel<W_F16><<<blocks, 256, 0, s>>>(out_ptr, out_col, out_w, pop_off, n_pops, n, pop_loc, own_cnt, maxw_bits, own_seg, woff, unsorted); break;
        default: local_offsets_kernel<W_U8><<<blocks, 256, 0, s>>>(out_ptr, out_col, out_w, pop_off, n_pops, n, pop_loc, own_cnt, maxw_bits, own_seg, woff, unsorted); break;
    }
    return cudaGetLastError();
}

template <int G>
static void pull_dispatch(const LaunchBatch& b, int wt, uint32_t flags, int prop_mode, cudaStream_t s) {
    const dim3 grid(b.pull_tiles_total), block(kPullThreads);
    switch (wt) {
        case W_F32: lif_pull_kernel<G, W_F32><<<grid, block, 0, s>>>(b.nets, b.pull_prefix, b.n_nets, flags, prop_mode); break;
        case W_BF16: lif_pull_kernel<G, W_BF16><<<grid, block, 0, s>>>(b.nets, b.pull_prefix, b.n_nets, flags, prop_mode); break;
        case W_F16: lif_pull_kernel<G, W_F16><<<grid, block, 0, s>>>(b.nets, b.pull_prefix, b.n_nets, flags, prop_mode); break;
        default: lif_pull_kernel<G, W_U8><<<grid, block, 0, s>>>(b.nets, b.pull_prefix, b.n_nets, flags, prop_mode); break;
    }
}

cudaError_t launch_pull(const LaunchBatch& b, int gather, int wt, uint32_t flags, int prop_mode, cudaStream_t s) {
    if (b.pull_tiles_total == 0) return cudaSuccess;
    if (gather) pull_dispatch<1>(b, wt, flags, prop_mode, s); else pull_dispatch<0>(b, wt, flags, prop_mode, s);
    return cudaGetLastError();
}

cudaError_t launch_stat_isyn(const LaunchBatch& b, int acc, int sm_count, cudaStream_t s) {
    if (b.lif_tiles_total == 0) return cudaSuccess;
    const dim3 grid(std::min<uint32_t>(b.lif_tiles_total, static_cast<uint32_t>(sm_count) * 8u)), block(256);
    if (acc == ACC_EXACT) stat_isyn_kernel<J_FOLD><<<grid, block, 0, s>>>(b.nets, b.lif_prefix, b.n_nets, b.lif_tiles_total);
    else if (acc == ACC_FIXED) stat_isyn_kernel<J_FIXF><<<grid, block, 0, s>>>(b.nets, b.lif_prefix, b.n_nets, b.lif_tiles_total);
    else stat_isyn_kernel<J_DIRECT><<<grid, block, 0, s>>>(b.nets, b.lif_prefix, b.n_nets, b.lif_tiles_total);
    return cudaGetLastError();
}

cudaError_t launch_fold_finish(const LaunchBatch& b, int acc, cudaStream_t s) {
    if (b.lif_tiles_total == 0) return cudaSuccess;
    if (acc == ACC_FIXED)
        fold_finish_kernel<ACC_FIXED><<<b.lif_tiles_total, kLifThreads, 0, s>>>(b.nets, b.lif_prefix, b.n_nets);
    else
        fold_finish_kernel<ACC_EXACT><<<b.lif_tiles_total, kLifThreads, 0, s>>>(b.nets, b.lif_prefix, b.n_nets);
    return cudaGetLastError();
}

cudaError_t launch_gather_finish(const LaunchBatch& b, int wt, cudaStream_t s) {
    if (b.pull_tiles_total == 0) return cudaSuccess;
    const dim3 grid(b.pull_tiles_total), block(kPullThreads);
    switch (wt) {
        case W_F32: gather_finish_kernel<W_F32><<<grid, block, 0, s>>>(b.nets, b.pull_prefix, b.n_nets); break;
        case W_BF16: gather_finish_kernel<W_BF16><<<grid, block, 0, s>>>(b.nets, b.pull_prefix, b.n_nets); break;
        case W_F16: gather_finish_kernel<W_F16><<<grid, block, 0, s>>>(b.nets, b.pull_prefix, b.n_nets); break;
        default: gather_finish_kernel<W_U8><<<grid, block, 0, s>>>(b.nets, b.pull_prefix, b.n_nets); break;
    }
    return cudaGetLastError();
}

}  // namespace dtb
