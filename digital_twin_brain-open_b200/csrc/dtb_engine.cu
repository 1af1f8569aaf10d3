// Engine: ownership of one network's device memory, ingest, the run loop and the
// property surface.  The run loop is the reference's per-iteration body
// (tools/dist_simulator.cpp:2072-2315) with the MPI exchange replaced by in-HBM
// delivery and every per-step host synchronisation removed.
#include "dtb_engine.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>

namespace dtb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

int fail(int status, const std::string& msg) {
    g_last_error = msg;
    return status;
}

int cuda_fail(cudaError_t e, const char* what) {
    cudaGetLastError();
    const int st = (e == cudaErrorMemoryAllocation) ? DTB_OUT_OF_MEMORY
                 : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? DTB_NO_DEVICE : DTB_CUDA_ERROR;
    return fail(st, std::string(what) + ": " + cudaGetErrorString(e));
}

__global__ void set_u64_kernel(unsigned long long* p, unsigned long long v) { *p = v; }
__global__ void set_u32_kernel(uint32_t* p, uint32_t v) { *p = v; }

static constexpr size_t kCsrPadWords = 16;   // 64 bytes after every CSR array
static constexpr size_t kCsrPadBytes = 64;
__global__ void set_clock_kernel(Clock* c, float t, unsigned long long n) {
    c->t = t;
    c->n = n;
    c->err = 0u;
}
__global__ void fill_range_kernel(float* p, uint32_t begin, uint32_t end, float v) {
    for (uint32_t i = begin + blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x) p[i] = v;
}

static uint32_t round_up(uint32_t x, uint32_t m) { return (x + m - 1) / m * m; }

Engine::~Engine() {
    if (stream) cudaStreamSynchronize(stream);
    if (graph) cudaGraphExecDestroy(graph);
    for (void* p : allocs) cudaFree(p);
    if (h_cnt) cudaFreeHost(h_cnt);
    if (h_vsum) cudaFreeHost(h_vsum);
    if (h_isum) cudaFreeHost(h_isum);
    for (cudaEvent_t e : tev) cudaEventDestroy(e);
    if (tune_ev[0]) cudaEventDestroy(tune_ev[0]);
    if (tune_ev[1]) cudaEventDestroy(tune_ev[1]);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (aux) cudaStreamDestroy(aux);
    if (stream) cudaStreamDestroy(stream);
}

void Engine::dfree(void* p) {
    if (!p) return;
    auto it = std::find(allocs.begin(), allocs.end(), p);
    if (it != allocs.end()) allocs.erase(it);
    cudaFree(p);
}

int Engine::weight_bytes() const {
    switch (wtype) {
        case W_F32: return 8;
        case W_BF16: case W_F16: return 4;
        default: return 2;
    }
}

int Engine::init_common(const dtb_options& opt, uint32_t n_neurons) {
    if (!(opt.dt > 0.0f) || !std::isfinite(opt.dt)) return fail(DTB_INVALID_PARAMETER, "dt must be positive");
    if (opt.weight_type > DTB_W_U8) return fail(DTB_UNSUPPORTED, "device weight type must be F32, BF16, F16 or U8");
    if (n_neurons == 0) return fail(DTB_INVALID_NETWORK, "network has no neurons");
    if (n_neurons >= 0x7FFFFFFFu - kPad) return fail(DTB_UNSUPPORTED, "more than 2^31 neurons");
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) {
        cudaGetLastError();
        return fail(DTB_NO_DEVICE, "no CUDA device");
    }
    DTB_CU(cudaGetDevice(&device));
    DTB_CU(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device));
    DTB_CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    DTB_CU(cudaStreamCreateWithFlags(&aux, cudaStreamNonBlocking));
    DTB_CU(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    DTB_CU(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    DTB_CU(cudaEventCreate(&ev0));
    DTB_CU(cudaEventCreate(&ev1));
    dt = opt.dt;
    wtype = opt.weight_type;
    seed = opt.seed;
    n = n_neurons;
    n_pad = round_up(n, kPad);
    n_words = n_pad / 32;
    return DTB_OK;
}

int Engine::setup_populations_from_property(const float* prop) {
    // Populations are runs of equal column-3 values (src/configuration.cpp:1902-1930).
    pop_ids.clear();
    pop_off.clear();
    for (uint32_t i = 0; i < n; ++i) {
        const float v = prop[static_cast<size_t>(i) * 22 + 3];
        if (i == 0 || v != prop[static_cast<size_t>(i - 1) * 22 + 3]) {
            if (!(v >= 0.0f) || v > 4294967040.0f) return fail(DTB_INVALID_NETWORK, "population id must be a non-negative integer");
            pop_ids.push_back(static_cast<uint32_t>(v));
            pop_off.push_back(i);
        }
    }
    pop_off.push_back(n);
    P = static_cast<uint32_t>(pop_ids.size());
    return DTB_OK;
}

int Engine::upload_params() {
    ++params_version;
    std::vector<PopParams> pp(P);
    for (uint32_t p = 0; p < P; ++p) pp[p] = derive(pop_raw[p], dt);
    DTB_CU(cudaMemcpyAsync(pop_dev, pp.data(), sizeof(PopParams) * P, cudaMemcpyHostToDevice, stream));
    if (per_neuron) {
        if (!np_dev) DTB_TRY(dalloc(np_dev, static_cast<size_t>(kParamFloats) * n_pad));
        std::vector<float> soa(static_cast<size_t>(kParamFloats) * n_pad, 0.0f);
        for (uint32_t i = 0; i < n; ++i) {
            const PopParams d = derive(neuron_raw[i], dt);
            const float* f = reinterpret_cast<const float*>(&d);
            for (int k = 0; k < kParamFloats; ++k) soa[static_cast<size_t>(k) * n_pad + i] = f[k];
        }
        DTB_CU(cudaMemcpyAsync(np_dev, soa.data(), soa.size() * sizeof(float), cudaMemcpyHostToDevice, stream));
        DTB_CU(cudaStreamSynchronize(stream));
    } else {
        DTB_CU(cudaStreamSynchronize(stream));
    }
    return refresh_view();
}

int Engine::init_state() {
    // block_new.py:57-62: V = (V_th + V_reset) / 2, t_last = -T_ref, J = 0, i_bg = OU mean
    std::vector<float> v(n_pad, 0.0f), tl(n_pad, 0.0f), io(n_pad, 0.0f);
    for (uint32_t p = 0; p < P; ++p) {
        for (uint32_t i = pop_off[p]; i < pop_off[p + 1]; ++i) {
            const RawParams& r = per_neuron ? neuron_raw[i] : pop_raw[p];
            volatile float s = r.V_th + r.V_reset;
            v[i] = s / 2.0f;
            tl[i] = -r.T_ref;
            io[i] = r.ou_mean;
        }
    }
    DTB_CU(cudaMemcpyAsync(V, v.data(), sizeof(float) * n_pad, cudaMemcpyHostToDevice, stream));
    DTB_CU(cudaMemcpyAsync(tlast, tl.data(), sizeof(float) * n_pad, cudaMemcpyHostToDevice, stream));
    DTB_CU(cudaMemcpyAsync(iou, io.data(), sizeof(float) * n_pad, cudaMemcpyHostToDevice, stream));
    DTB_CU(cudaMemsetAsync(J, 0, sizeof(float4) * n_pad, stream));
    DTB_CU(cudaMemsetAsync(bits0, 0, sizeof(uint32_t) * n_words, stream));
    DTB_CU(cudaMemsetAsync(bits1, 0, sizeof(uint32_t) * n_words, stream));
    set_clock_kernel<<<1, 1, 0, stream>>>(clock, 0.0f, 0ull);
    DTB_CU(cudaGetLastError());
    DTB_CU(cudaStreamSynchronize(stream));
    steps = 0;
    t = 0.0f;
    return DTB_OK;
}

int Engine::refresh_view() {
    NetView v{};
    v.n = n;
    v.n_pad = n_pad;
    v.n_words = n_words;
    v.n_pops = P;
    v.dt = dt;
    v.per_neuron = per_neuron ? 1u : 0u;
    if (view_ts > 1) {
        // a t_steps run: every kernel steps by dt / t_steps with constants derived for it
        volatile float dts = dt / static_cast<float>(view_ts);
        v.dt = dts;
    }
    v.weight_type = wtype;
    v.hist_cap = hist_cap;
    v.V = V;
    v.iou = iou;
    v.tlast = tlast;
    v.J = J;
    v.dJ = dJ;
    v.pop = view_ts > 1 ? pop_sub_dev : pop_dev;
    v.pop_off = pop_off_dev;
    v.np_params = view_ts > 1 ? np_sub_dev : np_dev;
    v.out_ptr = out_ptr;
    v.out_col = out_col;
    v.out_w = out_w;
    v.out_deg = out_deg;
    v.in_ptr = in_ptr;
    v.in_col = in_col;
    v.in_w = in_w;
    v.bits0 = bits0;
    v.bits1 = bits1;
    v.rec_bits = rec_bits;
    v.stat_excl = excl;
    v.clock = clock;
    v.seed = seed;
    v.inj_z = inj_z;
    v.inj_u = inj_u;
    v.inj_rows = inj_rows;
    v.hist_cnt = hist_cnt;
    v.hist_vsum = hist_vsum;
    v.hist_isum = hist_isum;
    v.isum_cap = isum_cap;
    v.events = events;
    v.ticket = ticket;
    v.lif_tiles = n_pad / kLifTile;
    v.tile_pop = tile_pop;
    v.n_samples = n_samples;
    v.sample_bits = sample_bits;
    v.sample_pre = sample_pre;
    v.hist_sspk = hist_sspk;
    v.hist_sv = hist_sv;
    v.hist_siou = hist_siou;
    v.hist_sisyn = hist_sisyn;
    v.own_seg = own_seg;
    v.woff = woff;
    v.pop_loc = pop_loc;
    v.win_tab = win_tab;
    v.n_windows = n_windows;
    v.dJf = dJf;
    v.fix_shift = fix_shift;
    v.fix_scale = fix_shift ? static_cast<float>(std::ldexp(1.0, static_cast<int>(fix_shift))) : 0.0f;
    v.fix_unscale = fix_shift ? static_cast<float>(std::ldexp(1.0, -static_cast<int>(fix_shift))) : 0.0f;
    view = v;
    DTB_CU(cudaMemcpyAsync(view_dev, &view, sizeof(NetView), cudaMemcpyHostToDevice, stream));
    DTB_CU(cudaStreamSynchronize(stream));
    return DTB_OK;
}

LaunchBatch Engine::single_batch() const {
    LaunchBatch b{};
    b.nets = view_dev;
    b.lif_prefix = prefix_dev;
    b.pull_prefix = prefix_dev + 2;
    b.vbase = prefix_dev + 4;
    b.n_nets = 1;
    b.lif_tiles_total = n_pad / kLifTile;
    b.pull_tiles_total = n_pad / kPullTile;
    b.push_ctas = static_cast<uint32_t>(sm_count) * 8u;
    b.lif_ctas = static_cast<uint32_t>(sm_count) * lif_ctas_per_sm;
    b.lif_chunk = 1;
    b.spikes = SpikeList{list, list_count, list_ticket, n_pad};
    b.win_prefix = prefix_dev + 6;
    b.windows_total = n_windows;
    b.local_scratch = local_scratch;
    b.sm_count = static_cast<uint32_t>(sm_count);
    b.aux = aux;
    b.ev_fork = ev_fork;
    b.ev_join = ev_join;
    return b;
}

// (kind, param) of dtb_set_push_variant -> one of the tuner's candidates;
// param 1000 + lanes per row selects sub-warp rows.
bool push_cfg_from_abi(int kind, int param, PushCfg& cfg) {
    cfg = PushCfg{kind, param, 32};
    if ((kind == PUSH_REG || kind == PUSH_LOCAL) && param >= 1000 && param < 2000) {
        cfg.param = 8;
        cfg.lpr = param - 1000;
    }
    for (const PushCfg& c : kPushCands)
        if (c.kind == cfg.kind && c.param == cfg.param && c.lpr == cfg.lpr) return true;
    return false;
}

int acc_of(uint32_t syn_mode) {
    return syn_mode == DTB_SYN_PUSH_EXACT ? ACC_EXACT : syn_mode == DTB_SYN_PUSH_FIXED ? ACC_FIXED : ACC_FLOAT;
}

int jmode_of(uint32_t syn_mode, bool first) {
    switch (syn_mode) {
        case DTB_SYN_PUSH_EXACT: return first ? J_ASIS : J_FOLD;
        case DTB_SYN_PUSH_FIXED: return first ? J_ASIS : J_FIXF;
        default: return J_DIRECT;
    }
}

uint32_t fixed_shift_for(uint64_t max_in_degree, double max_w, bool negative) {
    if (negative || !(max_w >= 0.0) || !std::isfinite(max_w)) return 0;
    // device weight types round the input (bf16/f16 by up to 2^-8 relative): bound with margin
    const double w = std::max(max_w, 1e-30) * (1.0 + 1.0 / 128.0);
    for (int sh = 32; sh >= 12; --sh)
        if (static_cast<double>(max_in_degree) * (w * std::ldexp(1.0, sh) + 0.5) < 4294967295.0) return static_cast<uint32_t>(sh);
    return 0;
}

// Population-local push tables.  A population gets k = ceil(size / kLocalWin)
// windows when its rows carry, on average, at least kLocalMinSpan own-population
// synapses per window and its window sums fit 32-bit fixed point at a
// resolution of 2^-kLocalMinShift or finer; other populations stay with the
// scattered push.
constexpr double kLocalMinSpan = 32.0;
constexpr int kLocalMinShift = 16;
constexpr int kLocalMaxShift = 60;

int Engine::build_local_tables() {
    if (!has_push || n == 0) return DTB_OK;
    // pass 1: sortedness, own-population in-degree per neuron, max |w| per population
    uint32_t* d_tmp = nullptr;
    const size_t tmp_words = static_cast<size_t>(n) + P + 1;
    DTB_CU(cudaMalloc(reinterpret_cast<void**>(&d_tmp), sizeof(uint32_t) * tmp_words));
    std::vector<uint32_t> cnt(n), maxw(P);
    uint32_t unsorted = 0;
    auto pass1 = [&]() -> int {
        DTB_CU(cudaMemsetAsync(d_tmp, 0, sizeof(uint32_t) * tmp_words, stream));
        DTB_CU(build_local_offsets(out_ptr, out_col, out_w, static_cast<int>(wtype), pop_off_dev, P, n, nullptr, d_tmp,
                                   d_tmp + n, nullptr, nullptr, d_tmp + n + P, stream));
        DTB_CU(cudaMemcpyAsync(cnt.data(), d_tmp, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, stream));
        DTB_CU(cudaMemcpyAsync(maxw.data(), d_tmp + n, sizeof(uint32_t) * P, cudaMemcpyDeviceToHost, stream));
        DTB_CU(cudaMemcpyAsync(&unsorted, d_tmp + n + P, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        DTB_CU(cudaStreamSynchronize(stream));
        return DTB_OK;
    };
    const int st = pass1();
    cudaFree(d_tmp);
    if (st != DTB_OK) return st;
    if (unsorted) return DTB_OK;
    std::vector<uint4> loc(P, make_uint4(0, 0, 0, 0));
    std::vector<uint4> wins;
    unsigned long long rb = 0;
    for (uint32_t a = 0; a < P; ++a) {
        const uint32_t size = pop_off[a + 1] - pop_off[a];
        if (size == 0) continue;
        uint64_t total = 0;
        uint32_t deg = 0;
        for (uint32_t i = pop_off[a]; i < pop_off[a + 1]; ++i) {
            total += cnt[i];
            deg = std::max(deg, cnt[i]);
        }
        const uint32_t k = (size + kLocalWin - 1) / kLocalWin;
        if (static_cast<double>(total) / size / k < kLocalMinSpan) continue;
        // largest s with max|w| * deg * 2^s + deg < 2^31 (each rounded weight adds at most 1/2)
        float mw;
        std::memcpy(&mw, &maxw[a], sizeof(float));
        const double room = 2147483647.0 - deg;
        int sh = kLocalMaxShift;
        if (mw > 0.f) sh = std::min(kLocalMaxShift, static_cast<int>(std::floor(std::log2(room / (static_cast<double>(mw) * deg)))));
        while (sh >= kLocalMinShift && static_cast<double>(mw) * deg * std::ldexp(1.0, sh) >= room) --sh;
        if (sh < kLocalMinShift) continue;
        const uint32_t width = (size + k - 1) / k;
        loc[a] = make_uint4(k, width, static_cast<uint32_t>(rb), static_cast<uint32_t>(rb >> 32));
        for (uint32_t w = 0; w < k; ++w) {
            const uint32_t lo = std::min<uint64_t>(pop_off[a] + static_cast<uint64_t>(w) * width, pop_off[a + 1]);
            const uint32_t hi = w + 1 == k ? pop_off[a + 1] : std::min<uint64_t>(lo + static_cast<uint64_t>(width), pop_off[a + 1]);
            wins.push_back(make_uint4(a, lo, hi, w | (static_cast<uint32_t>(sh) << 16)));
        }
        rb += static_cast<unsigned long long>(size) * (k + 1);
    }
    if (wins.empty()) return DTB_OK;
    DTB_TRY(dalloc(own_seg, n, false));
    DTB_TRY(dalloc(woff, rb, false));
    DTB_TRY(dalloc(pop_loc, P, false));
    DTB_TRY(dalloc(win_tab, wins.size(), false));
    DTB_TRY(dalloc(local_scratch, 2 * wins.size() + 3));
    DTB_CU(cudaMemcpyAsync(pop_loc, loc.data(), sizeof(uint4) * P, cudaMemcpyHostToDevice, stream));
    DTB_CU(cudaMemcpyAsync(win_tab, wins.data(), sizeof(uint4) * wins.size(), cudaMemcpyHostToDevice, stream));
    DTB_CU(build_local_offsets(out_ptr, out_col, out_w, static_cast<int>(wtype), pop_off_dev, P, n, pop_loc, nullptr,
                               nullptr, own_seg, woff, nullptr, stream));
    n_windows = static_cast<uint32_t>(wins.size());
    const uint32_t wp[2] = {0u, n_windows};
    DTB_CU(cudaMemcpyAsync(prefix_dev + 6, wp, sizeof(wp), cudaMemcpyHostToDevice, stream));
    DTB_CU(cudaStreamSynchronize(stream));
    return DTB_OK;
}

// Allocations every network needs, independent of its connectivity.
static int alloc_core(Engine& e) {
    DTB_TRY(e.dalloc(e.V, e.n_pad));
    DTB_TRY(e.dalloc(e.iou, e.n_pad));
    DTB_TRY(e.dalloc(e.tlast, e.n_pad));
    DTB_TRY(e.dalloc(e.J, e.n_pad));
    DTB_TRY(e.dalloc(e.pop_dev, e.P));
    DTB_TRY(e.dalloc(e.pop_off_dev, e.P + 1));
    DTB_TRY(e.dalloc(e.out_deg, e.n_pad));
    DTB_TRY(e.dalloc(e.bits0, e.n_words));
    DTB_TRY(e.dalloc(e.bits1, e.n_words));
    DTB_TRY(e.dalloc(e.clock, 1));
    DTB_TRY(e.dalloc(e.events, 1));
    DTB_TRY(e.dalloc(e.ticket, 1));
    DTB_TRY(e.dalloc(e.view_dev, 1));
    DTB_TRY(e.dalloc(e.prefix_dev, 8));
    DTB_TRY(e.dalloc(e.list, e.n_pad, false));
    DTB_TRY(e.dalloc(e.list_count, 1));
    DTB_TRY(e.dalloc(e.list_ticket, 1));
    {
        // population of the first neuron of every 1024-neuron LIF tile
        const uint32_t tiles = e.n_pad / kLifTile;
        std::vector<uint32_t> tp(tiles);
        uint32_t p = 0;
        for (uint32_t t = 0; t < tiles; ++t) {
            const uint32_t i = std::min(t * static_cast<uint32_t>(kLifTile), e.n - 1);
            while (p + 1 < e.P && e.pop_off[p + 1] <= i) ++p;
            tp[t] = p;
        }
        DTB_TRY(e.dalloc(e.tile_pop, tiles));
        DTB_CU(cudaMemcpyAsync(e.tile_pop, tp.data(), sizeof(uint32_t) * tiles, cudaMemcpyHostToDevice, e.stream));
    }
    const uint32_t pre[6] = {0u, e.n_pad / kLifTile, 0u, e.n_pad / kPullTile, 0u, e.n_pad};
    DTB_CU(cudaMemcpyAsync(e.prefix_dev, pre, sizeof(pre), cudaMemcpyHostToDevice, e.stream));
    DTB_CU(cudaMemcpyAsync(e.pop_off_dev, e.pop_off.data(), sizeof(uint32_t) * (e.P + 1), cudaMemcpyHostToDevice, e.stream));
    DTB_CU(cudaStreamSynchronize(e.stream));
    e.ou_set.assign(e.P, 0);
    return DTB_OK;
}

// Convert one input weight pair to float32.
static void weight_to_f32(const void* w, uint32_t type, uint64_t e, float& a, float& b) {
    switch (type) {
        case DTB_W_F32: { const float* f = static_cast<const float*>(w) + 2 * e; a = f[0]; b = f[1]; break; }
        case DTB_W_F64: { const double* f = static_cast<const double*>(w) + 2 * e; a = static_cast<float>(f[0]); b = static_cast<float>(f[1]); break; }
        case DTB_W_F16: { const __half* f = static_cast<const __half*>(w) + 2 * e; a = __half2float(f[0]); b = __half2float(f[1]); break; }
        case DTB_W_BF16: { const __nv_bfloat16* f = static_cast<const __nv_bfloat16*>(w) + 2 * e; a = __bfloat162float(f[0]); b = __bfloat162float(f[1]); break; }
        default: { const uint8_t* f = static_cast<const uint8_t*>(w) + 2 * e; a = static_cast<float>(f[0]) / 255.f; b = static_cast<float>(f[1]) / 255.f; break; }
    }
}

// Write weight pair e of the input in the device encoding at slot `dst_index`.
static void encode_weight(const void* w, uint32_t in_type, uint64_t e, uint32_t dev_type, uint8_t* dst, uint64_t dst_index) {
    if (dev_type == W_U8 && in_type == DTB_W_U8) {
        std::memcpy(dst + 2 * dst_index, static_cast<const uint8_t*>(w) + 2 * e, 2);
        return;
    }
    if (dev_type == W_F16 && in_type == DTB_W_F16) {
        std::memcpy(dst + 4 * dst_index, static_cast<const uint8_t*>(w) + 4 * e, 4);
        return;
    }
    float a, b;
    weight_to_f32(w, in_type, e, a, b);
    switch (dev_type) {
        case W_F32: { float* f = reinterpret_cast<float*>(dst) + 2 * dst_index; f[0] = a; f[1] = b; break; }
        case W_BF16: { __nv_bfloat16* f = reinterpret_cast<__nv_bfloat16*>(dst) + 2 * dst_index; f[0] = __float2bfloat16_rn(a); f[1] = __float2bfloat16_rn(b); break; }
        case W_F16: { __half* f = reinterpret_cast<__half*>(dst) + 2 * dst_index; f[0] = __float2half_rn(a); f[1] = __float2half_rn(b); break; }
        default: {
            uint8_t* f = dst + 2 * dst_index;
            f[0] = static_cast<uint8_t>(std::lrint(std::min(std::max(a, 0.f), 1.f) * 255.f));
            f[1] = static_cast<uint8_t>(std::lrint(std::min(std::max(b, 0.f), 1.f) * 255.f));
            break;
        }
    }
}

int Engine::upload_csr_host(const uint32_t* pre, const uint32_t* post, const uint8_t* kind_in, const void* w,
                            uint32_t in_type, bool build_push, bool build_pull) {
    const int wb = weight_bytes();
    std::vector<uint64_t> ptr, perm;
    std::vector<uint32_t> deg(n_pad, 0);
    for (uint64_t e = 0; e < n_edges; ++e) deg[pre[e]]++;
    DTB_CU(cudaMemcpyAsync(out_deg, deg.data(), sizeof(uint32_t) * n_pad, cudaMemcpyHostToDevice, stream));
    DTB_CU(cudaStreamSynchronize(stream));
    auto build = [&](const uint32_t* key, const uint32_t* other, unsigned long long*& d_ptr, uint32_t*& d_col, void*& d_w) -> int {
        counting_sort(key, n_edges, n, ptr, perm);
        std::vector<uint32_t> col(n_edges);
        std::vector<uint8_t> wt(static_cast<size_t>(n_edges) * wb);
        for (uint64_t q = 0; q < n_edges; ++q) {
            const uint64_t e = perm[q];
            col[q] = other[e] | ((kind_in[e] != 0 ? 1u : 0u) << 31);
            encode_weight(w, in_type, e, wtype, wt.data(), q);
        }
        DTB_TRY(dalloc(d_ptr, static_cast<size_t>(n) + 1, false));
        DTB_TRY(dalloc(d_col, n_edges + kCsrPadWords));
        uint8_t* wdev = nullptr;
        DTB_TRY(dalloc(wdev, static_cast<size_t>(n_edges) * wb + kCsrPadBytes));
        d_w = wdev;
        DTB_CU(cudaMemcpyAsync(d_ptr, ptr.data(), sizeof(uint64_t) * (n + 1), cudaMemcpyHostToDevice, stream));
        DTB_CU(cudaMemcpyAsync(d_col, col.data(), sizeof(uint32_t) * n_edges, cudaMemcpyHostToDevice, stream));
        DTB_CU(cudaMemcpyAsync(wdev, wt.data(), wt.size(), cudaMemcpyHostToDevice, stream));
        DTB_CU(cudaStreamSynchronize(stream));
        return DTB_OK;
    };
    if (build_push) {
        DTB_TRY(build(pre, post, out_ptr, out_col, out_w));
        has_push = true;
    }
    if (build_pull) {
        DTB_TRY(build(post, pre, in_ptr, in_col, in_w));
        has_pull = true;
    }
    return DTB_OK;
}

int Engine::create_from_arrays(const dtb_network_arrays& a, const dtb_options& opt) {
    if (!a.property) return fail(DTB_INVALID_PARAMETER, "property is NULL");
    if (a.n_edges && (!a.input_neuron_idx || !a.output_neuron_idx || !a.input_channel_offset || !a.weight))
        return fail(DTB_INVALID_PARAMETER, "edge arrays missing");
    if (a.weight_type > DTB_W_F64) return fail(DTB_UNSUPPORTED, "unknown input weight type");
    if (!opt.build_push && !opt.build_pull) return fail(DTB_INVALID_PARAMETER, "neither push nor pull CSR requested");
    DTB_TRY(init_common(opt, a.n_neurons));
    n_edges = a.n_edges;
    for (uint64_t e = 0; e < n_edges; ++e) {
        if (a.input_neuron_idx[e] >= n || a.output_neuron_idx[e] >= n)
            return fail(DTB_INVALID_NETWORK, "edge " + std::to_string(e) + " references a neuron outside the block");
        if (a.input_block_idx && a.input_block_idx[e] != 0)
            return fail(DTB_UNSUPPORTED, "edges from other blocks (input_block_idx != 0): one network per GPU");
    }
    DTB_TRY(setup_populations_from_property(a.property));
    // per-population parameters; per-neuron mode if any population is not uniform
    pop_raw.resize(P);
    for (uint32_t p = 0; p < P; ++p) {
        const float* row0 = a.property + static_cast<size_t>(pop_off[p]) * 22;
        pop_raw[p] = raw_from_property(row0, opt.ou_mean, opt.ou_sigma, opt.ou_tau);
        for (uint32_t i = pop_off[p] + 1; i < pop_off[p + 1] && !per_neuron; ++i)
            if (!same_params(row0, a.property + static_cast<size_t>(i) * 22)) per_neuron = true;
    }
    if (per_neuron) {
        neuron_raw.resize(n);
        for (uint32_t i = 0; i < n; ++i)
            neuron_raw[i] = raw_from_property(a.property + static_cast<size_t>(i) * 22, opt.ou_mean, opt.ou_sigma, opt.ou_tau);
    }
    DTB_TRY(alloc_core(*this));
    // statistics exclusion (column 1, blocked_in_stat)
    excl_count.assign(P, 0);
    std::vector<uint32_t> ex(n_words, 0);
    bool any_ex = false;
    for (uint32_t p = 0; p < P; ++p)
        for (uint32_t i = pop_off[p]; i < pop_off[p + 1]; ++i)
            if (a.property[static_cast<size_t>(i) * 22 + 1] != 0.0f) {
                ex[i >> 5] |= 1u << (i & 31);
                excl_count[p]++;
                any_ex = true;
            }
    if (any_ex) {
        DTB_TRY(dalloc(excl, n_words));
        DTB_CU(cudaMemcpyAsync(excl, ex.data(), sizeof(uint32_t) * n_words, cudaMemcpyHostToDevice, stream));
    }
    {
        // fixed-mode scale: largest in-degree and weight of the network
        std::vector<uint32_t> indeg(n, 0);
        double max_w = 0.0;
        bool negative = false;
        for (uint64_t e = 0; e < n_edges; ++e) {
            ++indeg[a.output_neuron_idx[e]];
            float w0, w1;
            weight_to_f32(a.weight, a.weight_type, e, w0, w1);
            negative |= (w0 < 0.0f) || (w1 < 0.0f) || !std::isfinite(w0) || !std::isfinite(w1);
            max_w = std::max(max_w, static_cast<double>(std::max(w0, w1)));
        }
        const uint32_t deg = n ? *std::max_element(indeg.begin(), indeg.end()) : 0u;
        fix_shift = fixed_shift_for(deg, max_w, negative);
    }
    DTB_TRY(upload_csr_host(a.input_neuron_idx, a.output_neuron_idx, a.input_channel_offset, a.weight, a.weight_type,
                            opt.build_push != 0, opt.build_pull != 0));
    DTB_TRY(upload_params());
    DTB_TRY(init_state());
    DTB_TRY(build_local_tables());
    return refresh_view();
}

int Engine::create_structured(const dtb_structured_spec& s, const dtb_options& opt) {
    if (s.n_pops == 0 || !s.pop_sizes || !s.pop_exc || !s.src_cdf || !s.pop_property)
        return fail(DTB_INVALID_PARAMETER, "structured spec incomplete");
    if (s.in_degree == 0) return fail(DTB_INVALID_PARAMETER, "in_degree must be positive");
    if (!opt.build_push && !opt.build_pull) return fail(DTB_INVALID_PARAMETER, "neither push nor pull CSR requested");
    uint64_t total = 0;
    for (uint32_t b = 0; b < s.n_pops; ++b) {
        if (s.pop_sizes[b] < 2) return fail(DTB_INVALID_PARAMETER, "every population needs at least 2 neurons");
        if (s.pop_exc[b] > s.pop_sizes[b]) return fail(DTB_INVALID_PARAMETER, "pop_exc larger than the population");
        total += s.pop_sizes[b];
        const uint64_t* row = s.src_cdf + static_cast<size_t>(b) * s.n_pops;
        if (row[s.n_pops - 1] != (1ull << 32)) return fail(DTB_INVALID_PARAMETER, "src_cdf rows must end at 2^32");
        for (uint32_t c = 1; c < s.n_pops; ++c)
            if (row[c] < row[c - 1]) return fail(DTB_INVALID_PARAMETER, "src_cdf rows must be non-decreasing");
    }
    if (total >= 0x7FFFFFFFull - kPad) return fail(DTB_UNSUPPORTED, "more than 2^31 neurons");
    DTB_TRY(init_common(opt, static_cast<uint32_t>(total)));
    n_edges = static_cast<uint64_t>(n) * s.in_degree;
    fix_shift = fixed_shift_for(s.in_degree, 1.0, false);   // generated weights lie in [0, 1)
    P = s.n_pops;
    pop_ids.resize(P);
    pop_off.resize(P + 1);
    pop_raw.resize(P);
    pop_off[0] = 0;
    for (uint32_t b = 0; b < P; ++b) {
        pop_ids[b] = s.pop_id_base + b;
        pop_off[b + 1] = pop_off[b] + s.pop_sizes[b];
        pop_raw[b] = raw_from_property(s.pop_property + static_cast<size_t>(b) * 22, opt.ou_mean, opt.ou_sigma, opt.ou_tau);
    }
    excl_count.assign(P, 0);
    DTB_TRY(alloc_core(*this));
    // device tables for the generator
    uint32_t* d_exc = nullptr;
    unsigned long long* d_cdf = nullptr;
    DTB_TRY(dalloc(d_exc, P));
    DTB_TRY(dalloc(d_cdf, static_cast<size_t>(P) * P));
    DTB_CU(cudaMemcpyAsync(d_exc, s.pop_exc, sizeof(uint32_t) * P, cudaMemcpyHostToDevice, stream));
    DTB_CU(cudaMemcpyAsync(d_cdf, s.src_cdf, sizeof(uint64_t) * P * P, cudaMemcpyHostToDevice, stream));
    const int wb = weight_bytes();
    if (opt.build_push) {
        DTB_TRY(dalloc(out_ptr, static_cast<size_t>(n) + 1, false));
        DTB_TRY(dalloc(out_col, n_edges + kCsrPadWords, false));
        uint8_t* w = nullptr;
        DTB_TRY(dalloc(w, static_cast<size_t>(n_edges) * wb + kCsrPadBytes, false));
        out_w = w;
        has_push = true;
    }
    if (opt.build_pull) {
        DTB_TRY(dalloc(in_ptr, static_cast<size_t>(n) + 1, false));
        DTB_TRY(dalloc(in_col, n_edges + kCsrPadWords, false));
        uint8_t* w = nullptr;
        DTB_TRY(dalloc(w, static_cast<size_t>(n_edges) * wb + kCsrPadBytes, false));
        in_w = w;
        has_pull = true;
    }
    GenSpec g{};
    g.n = n;
    g.n_pops = P;
    g.in_degree = s.in_degree;
    g.dyadic = s.dyadic_weights;
    g.seed = s.seed;
    g.pop_off = pop_off_dev;
    g.pop_exc = d_exc;
    g.cdf = d_cdf;
    const cudaError_t ge = build_structured(g, static_cast<int>(wtype), out_ptr, out_col, out_w, in_ptr, in_col, in_w, out_deg, stream);
    if (ge == cudaErrorUnknown) return fail(DTB_DEVICE_FAULT, "device CSR build: placement check failed");
    if (ge != cudaSuccess) return cuda_fail(ge, "build_structured");
    dfree(d_exc);
    dfree(d_cdf);
    dev_bytes -= sizeof(uint32_t) * P + sizeof(unsigned long long) * P * P;
    DTB_TRY(upload_params());
    DTB_TRY(init_state());
    DTB_TRY(build_local_tables());
    return refresh_view();
}

int Engine::create_from_npz(const std::string& path, const dtb_options& opt) {
    std::vector<std::string> names = {"property", "input_block_idx", "input_neuron_idx", "output_neuron_idx",
                                      "input_channel_offset", "weight", "src_timestamp"};
    std::vector<NpyArray> arr;
    std::vector<bool> found;
    const std::string err = npz_load(path, names, arr, found);
    if (!err.empty()) return fail(DTB_IO_ERROR, err);
    if (found[6]) return fail(DTB_UNSUPPORTED, "input (spike replay) blocks are not supported");
    for (int k : {0, 2, 3, 4, 5})
        if (!found[k]) return fail(DTB_IO_ERROR, "npz member missing: " + names[k]);
    for (const auto& a : arr)
        if (a.fortran) return fail(DTB_UNSUPPORTED, "Fortran-ordered arrays");
    const NpyArray& prop = arr[0];
    if (prop.dtype != "<f4" || prop.shape.size() != 2 || prop.shape[1] != 22)
        return fail(DTB_INVALID_NETWORK, "property must be float32 [N, 22]");
    const uint64_t S = arr[2].count();
    if (arr[2].dtype != "<u4" || arr[3].dtype != "<u4" || arr[3].count() != S)
        return fail(DTB_INVALID_NETWORK, "input/output_neuron_idx must be uint32 [S]");
    if (arr[4].word() != 1 || arr[4].count() != S) return fail(DTB_INVALID_NETWORK, "input_channel_offset must be uint8 [S]");
    const NpyArray& w = arr[5];
    if (w.shape.size() != 2 || w.shape[0] != S || w.shape[1] != 2) return fail(DTB_INVALID_NETWORK, "weight must be [S, 2]");
    uint32_t wt;
    if (w.dtype == "<f4") wt = DTB_W_F32;
    else if (w.dtype == "<f8") wt = DTB_W_F64;
    else if (w.dtype == "<f2") wt = DTB_W_F16;
    else if (w.dtype == "|u1" || w.dtype == "|i1") wt = DTB_W_U8;   // bytes read as unsigned, value / 255
    else return fail(DTB_UNSUPPORTED, "weight dtype " + w.dtype);
    // The reference takes the weight type from the directory in the path
    // (src/configuration.cpp:1411-1435: "/double", "/single", "/half", "/int8" or "/uint8",
    // the first of them found from the end wins in that order of tests); the file's own
    // dtype must agree.  A path with none of them is taken by its dtype (the reference
    // refuses it as an unknown block type).
    const struct { const char* dir; uint32_t type; } rule[] = {
        {"/double", DTB_W_F64}, {"/single", DTB_W_F32}, {"/half", DTB_W_F16}, {"/int8", DTB_W_U8}, {"/uint8", DTB_W_U8}};
    for (const auto& r : rule) {
        if (path.rfind(r.dir) == std::string::npos) continue;
        if (r.type != wt)
            return fail(DTB_INVALID_NETWORK, "weight dtype " + w.dtype + " does not match the directory " + r.dir +
                                                 " of " + path);
        break;
    }
    std::vector<int16_t> blk;
    if (found[1]) {
        const NpyArray& b = arr[1];
        if (b.count() != S || b.word() != 2) return fail(DTB_INVALID_NETWORK, "input_block_idx must be int16/uint16 [S]");
        blk.resize(S);
        std::memcpy(blk.data(), b.data.data(), S * 2);
    }
    dtb_network_arrays a{};
    a.n_neurons = static_cast<uint32_t>(prop.shape[0]);
    a.property = reinterpret_cast<const float*>(prop.data.data());
    a.n_edges = S;
    a.input_block_idx = found[1] ? blk.data() : nullptr;
    a.input_neuron_idx = reinterpret_cast<const uint32_t*>(arr[2].data.data());
    a.output_neuron_idx = reinterpret_cast<const uint32_t*>(arr[3].data.data());
    a.input_channel_offset = arr[4].data.data();
    a.weight = w.data.data();
    a.weight_type = wt;
    return create_from_arrays(a, opt);
}

int Engine::ensure_dj() {
    if (dJ) return DTB_OK;
    DTB_TRY(dalloc(dJ, static_cast<size_t>(n_pad) * 4));
    DTB_CU(cudaStreamSynchronize(stream));
    return refresh_view();
}

// Constants for substeps of dt / ts (the reference derives OU, decay and membrane factors
// from delta_t / t_steps: src/block.cpp:304, 317, 668, 1275), derived again whenever the
// properties changed since; ts = 1 returns the view to the plain constants.
int Engine::use_substep_params(uint32_t ts) {
    const uint32_t want = ts > 1 ? ts : 1u;
    if (want > 1 && (sub_ts != want || sub_version != params_version)) {
        volatile float dts = dt / static_cast<float>(want);
        const float d = dts;
        if (!pop_sub_dev) DTB_TRY(dalloc(pop_sub_dev, P));
        std::vector<PopParams> pp(P);
        for (uint32_t p = 0; p < P; ++p) pp[p] = derive(pop_raw[p], d);
        DTB_CU(cudaMemcpyAsync(pop_sub_dev, pp.data(), sizeof(PopParams) * P, cudaMemcpyHostToDevice, stream));
        if (per_neuron) {
            if (!np_sub_dev) DTB_TRY(dalloc(np_sub_dev, static_cast<size_t>(kParamFloats) * n_pad));
            std::vector<float> soa(static_cast<size_t>(kParamFloats) * n_pad, 0.0f);
            for (uint32_t i = 0; i < n; ++i) {
                const PopParams q = derive(neuron_raw[i], d);
                const float* f = reinterpret_cast<const float*>(&q);
                for (int k = 0; k < kParamFloats; ++k) soa[static_cast<size_t>(k) * n_pad + i] = f[k];
            }
            DTB_CU(cudaMemcpyAsync(np_sub_dev, soa.data(), soa.size() * sizeof(float), cudaMemcpyHostToDevice, stream));
        }
        DTB_CU(cudaStreamSynchronize(stream));
        sub_ts = want;
        sub_version = params_version;
    }
    if (view_ts == want) return DTB_OK;
    view_ts = want;
    return refresh_view();
}

int Engine::ensure_djf() {
    if (dJf) return DTB_OK;
    DTB_TRY(dalloc(dJf, static_cast<size_t>(n_pad) * 2));
    DTB_CU(cudaStreamSynchronize(stream));
    return refresh_view();
}

int Engine::ensure_hist(uint32_t rows, bool record, bool samples) {
    bool changed = false;
    if (samples && n_samples && sample_cap < std::max(rows, hist_cap)) {
        dfree(hist_sspk);
        dfree(hist_sv);
        dfree(hist_siou);
        hist_sspk = nullptr;
        hist_sv = hist_siou = nullptr;
        const uint32_t r = std::max(rows, hist_cap);
        DTB_TRY(dalloc(hist_sspk, static_cast<size_t>(r) * n_samples));
        DTB_TRY(dalloc(hist_sv, static_cast<size_t>(r) * n_samples));
        DTB_TRY(dalloc(hist_siou, static_cast<size_t>(r) * n_samples));
        sample_cap = r;
        changed = true;
    }
    if (rows > hist_cap) {
        dfree(hist_cnt);
        dfree(hist_vsum);
        hist_cnt = nullptr;
        hist_vsum = nullptr;
        DTB_TRY(dalloc(hist_cnt, static_cast<size_t>(rows) * P));
        DTB_TRY(dalloc(hist_vsum, static_cast<size_t>(rows) * P));
        hist_cap = rows;
        changed = true;
        if (h_cnt) cudaFreeHost(h_cnt);
        if (h_vsum) cudaFreeHost(h_vsum);
        h_cnt = nullptr;
        h_vsum = nullptr;
        DTB_CU(cudaMallocHost(&h_cnt, sizeof(int) * rows * P));
        DTB_CU(cudaMallocHost(&h_vsum, sizeof(long long) * rows * P));
        h_cap = rows;
    }
    if (record && rec_cap < hist_cap) {
        dfree(rec_bits);
        rec_bits = nullptr;
        DTB_TRY(dalloc(rec_bits, static_cast<size_t>(hist_cap) * n_words));
        rec_cap = hist_cap;
        changed = true;
    }
    if (changed) return refresh_view();
    return DTB_OK;
}

// Device and pinned host buffers of the synaptic-current sums.
int Engine::ensure_isum(uint32_t rows, bool sample) {
    bool changed = false;
    if (rows > isum_cap) {
        dfree(hist_isum);
        hist_isum = nullptr;
        DTB_TRY(dalloc(hist_isum, static_cast<size_t>(rows) * P * 5));
        if (h_isum) cudaFreeHost(h_isum);
        h_isum = nullptr;
        DTB_CU(cudaMallocHost(&h_isum, sizeof(long long) * rows * P * 5));
        isum_cap = rows;
        changed = true;
    }
    if (sample && n_samples && sisyn_cap < isum_cap) {
        dfree(hist_sisyn);
        hist_sisyn = nullptr;
        DTB_TRY(dalloc(hist_sisyn, static_cast<size_t>(isum_cap) * n_samples));
        sisyn_cap = isum_cap;
        changed = true;
    }
    return changed ? refresh_view() : DTB_OK;
}

// Means of the chunk's synaptic-current sums into the caller's buffers.
int Engine::finish_isum(uint32_t rows, uint32_t out_row0, const dtb_run_output& out, bool imean, bool receptor,
                        bool sample) {
    std::vector<float> si;
    if (sample && n_samples) {
        si.resize(static_cast<size_t>(rows) * n_samples);
        DTB_CU(cudaMemcpyAsync(si.data(), hist_sisyn, si.size() * sizeof(float), cudaMemcpyDeviceToHost, stream));
    }
    if (imean || receptor)
        DTB_CU(cudaMemcpyAsync(h_isum, hist_isum, sizeof(long long) * rows * P * 5, cudaMemcpyDeviceToHost, stream));
    DTB_CU(cudaStreamSynchronize(stream));
    if (!si.empty()) {
        const size_t K = sample_order.size();
        for (uint32_t r = 0; r < rows; ++r)
            for (size_t k = 0; k < K; ++k)
                out.sample_isyn[static_cast<size_t>(out_row0 + r) * K + k] = si[static_cast<size_t>(r) * n_samples + sample_order[k]];
    }
    for (uint32_t r = 0; r < rows && (imean || receptor); ++r) {
        for (uint32_t p = 0; p < P; ++p) {
            const uint32_t cnt = pop_off[p + 1] - pop_off[p] - excl_count[p];
            const long long* q = h_isum + (static_cast<size_t>(r) * P + p) * 5;
            auto mean = [&](long long v) {
                return cnt ? static_cast<float>(static_cast<double>(v) / kVsumScale / static_cast<double>(cnt)) : 0.0f;
            };
            const size_t row = static_cast<size_t>(out_row0 + r);
            if (imean) out.imeans[row * P + p] = mean(q[0]);
            if (receptor)
                for (int c = 0; c < 4; ++c) out.receptor_imeans[(row * 4 + c) * P + p] = mean(q[1 + c]);
        }
    }
    return DTB_OK;
}

int Engine::begin_run_chunk(uint64_t run_base, uint32_t rows, bool stats) {
    set_u64_kernel<<<1, 1, 0, stream>>>(&clock->run_base, run_base);
    DTB_CU(cudaGetLastError());
    if (stats) {
        DTB_CU(cudaMemsetAsync(hist_cnt, 0, sizeof(int) * rows * P, stream));
        DTB_CU(cudaMemsetAsync(hist_vsum, 0, sizeof(long long) * rows * P, stream));
    }
    return DTB_OK;
}

int Engine::finish_samples(uint32_t rows, uint32_t out_row0, const dtb_run_output& out) {
    const size_t S = n_samples, K = sample_order.size();
    if (!S) return DTB_OK;
    std::vector<uint8_t> spk(static_cast<size_t>(rows) * S);
    std::vector<float> v(static_cast<size_t>(rows) * S), io(static_cast<size_t>(rows) * S);
    if (out.sample_spike) DTB_CU(cudaMemcpyAsync(spk.data(), hist_sspk, spk.size(), cudaMemcpyDeviceToHost, stream));
    if (out.sample_v) DTB_CU(cudaMemcpyAsync(v.data(), hist_sv, v.size() * 4, cudaMemcpyDeviceToHost, stream));
    if (out.sample_iou) DTB_CU(cudaMemcpyAsync(io.data(), hist_siou, io.size() * 4, cudaMemcpyDeviceToHost, stream));
    DTB_CU(cudaStreamSynchronize(stream));
    for (uint32_t r = 0; r < rows; ++r) {
        const size_t dst = static_cast<size_t>(out_row0 + r) * K, src = static_cast<size_t>(r) * S;
        for (size_t k = 0; k < K; ++k) {
            const size_t o = src + sample_order[k];
            if (out.sample_spike) out.sample_spike[dst + k] = spk[o];
            if (out.sample_v) out.sample_v[dst + k] = v[o];
            if (out.sample_iou) out.sample_iou[dst + k] = io[o];
        }
    }
    return DTB_OK;
}

int Engine::finish_hist(uint32_t rows, uint32_t out_row0, const dtb_run_output& out, bool freq, bool vmean, bool record) {
    if (freq || vmean) {
        DTB_CU(cudaMemcpyAsync(h_cnt, hist_cnt, sizeof(int) * rows * P, cudaMemcpyDeviceToHost, stream));
        DTB_CU(cudaMemcpyAsync(h_vsum, hist_vsum, sizeof(long long) * rows * P, cudaMemcpyDeviceToHost, stream));
    }
    if (record) {
        const size_t out_words = (n + 31) / 32;
        DTB_CU(cudaMemcpy2DAsync(out.spike_bits + static_cast<size_t>(out_row0) * out_words, out_words * 4, rec_bits,
                                 static_cast<size_t>(n_words) * 4, out_words * 4, rows, cudaMemcpyDeviceToHost, stream));
    }
    DTB_CU(cudaStreamSynchronize(stream));
    for (uint32_t r = 0; r < rows && (freq || vmean); ++r) {
        for (uint32_t p = 0; p < P; ++p) {
            const size_t src = static_cast<size_t>(r) * P + p;
            const size_t dst = static_cast<size_t>(out_row0 + r) * P + p;
            if (freq) out.freqs[dst] = h_cnt[src];
            if (vmean) {
                const uint32_t cnt = pop_off[p + 1] - pop_off[p] - excl_count[p];
                out.vmeans[dst] = cnt ? static_cast<float>(static_cast<double>(h_vsum[src]) / kVsumScale / static_cast<double>(cnt)) : 0.0f;
            }
        }
    }
    return DTB_OK;
}

int Engine::run(const dtb_run_request& rq, dtb_run_output& out) {
    if (rq.iters == 0) return fail(DTB_INVALID_PARAMETER, "iter must be positive");
    if (rq.prop_mode > DTB_PROP_OR) return fail(DTB_INVALID_PARAMETER, "unknown prop_mode");
    if (rq.syn_mode > DTB_SYN_PUSH_FIXED) return fail(DTB_INVALID_PARAMETER, "unknown syn_mode");
    const bool pull = rq.syn_mode == DTB_SYN_PULL;
    if (!pull && !has_push) return fail(DTB_UNSUPPORTED, "network was built without the out-degree CSR");
    if (pull && !has_pull) return fail(DTB_UNSUPPORTED, "network was built without the in-degree CSR");
    if (rq.syn_mode == DTB_SYN_PUSH_FIXED && fix_shift == 0)
        return fail(DTB_UNSUPPORTED, "fixed-point push needs non-negative weights whose in-degree sums fit 32 bits");
    const bool freq = (rq.flags & DTB_RUN_FREQ) != 0;
    const bool vmean = (rq.flags & DTB_RUN_VMEAN) != 0;
    const bool record = (rq.flags & DTB_RUN_RECORD_SPIKES) != 0;
    if ((freq && !out.freqs) || (vmean && !out.vmeans) || (record && !out.spike_bits))
        return fail(DTB_INVALID_PARAMETER, "requested output buffer is NULL");
    const bool samples = (rq.flags & (DTB_RUN_SAMPLE_SPIKE | DTB_RUN_SAMPLE_V | DTB_RUN_SAMPLE_IOU)) != 0;
    const bool sisyn = (rq.flags & DTB_RUN_SAMPLE_ISYN) != 0;
    if ((samples || sisyn) && sample_order.empty())
        return fail(DTB_UNSET_SAMPLE_FAILURE, "sample outputs requested but no samples are set");
    if (sisyn && !out.sample_isyn) return fail(DTB_INVALID_PARAMETER, "requested sample buffer is NULL");
    if (((rq.flags & DTB_RUN_SAMPLE_SPIKE) && !out.sample_spike) || ((rq.flags & DTB_RUN_SAMPLE_V) && !out.sample_v) ||
        ((rq.flags & DTB_RUN_SAMPLE_IOU) && !out.sample_iou))
        return fail(DTB_INVALID_PARAMETER, "requested sample buffer is NULL");
    if ((rq.flags & DTB_RUN_SAMPLE_IOU) && !(rq.flags & DTB_RUN_USE_OU))
        return fail(DTB_INVALID_PARAMETER, "sample_iou needs use_ou_background");
    const bool imean = (rq.flags & DTB_RUN_IMEAN) != 0, rimean = (rq.flags & DTB_RUN_RECEPTOR_IMEAN) != 0;
    if ((imean && !out.imeans) || (rimean && !out.receptor_imeans))
        return fail(DTB_INVALID_PARAMETER, "requested imean buffer is NULL");
    if ((imean || rimean || sisyn) && pull)
        return fail(DTB_UNSUPPORTED, "synaptic-current outputs need a push mode (the pull kernel completes J one step later)");
    const bool isyn_any = imean || rimean || sisyn;
    const uint32_t ts = std::max(1u, rq.t_steps);
    if (ts > 1) {
        // the reference's Run validation (dist_simulator.cpp:3225-3234) and this engine's limits
        if (ts > 255) return fail(DTB_INVALID_PARAMETER, "t_steps must be at most 255");
        if (!(rq.flags & DTB_RUN_USE_OU)) return fail(DTB_INVALID_PARAMETER, "t_steps > 1 needs use_ou_background");
        if (pull) return fail(DTB_UNSUPPORTED, "substeps need a push mode");
        if (rq.prop_mode != DTB_PROP_THRESHOLD) return fail(DTB_UNSUPPORTED, "substeps propagate threshold spikes only");
    }
    const bool injected = noise_src == DTB_NOISE_INJECTED;
    if (injected) {
        // rows are consumed t_steps per step (every step since dtb_set_noise at this t_steps)
        const uint64_t used = (steps - inj_first) * ts;
        if (used + static_cast<uint64_t>(rq.iters) * ts > inj_rows)
            return fail(DTB_INVALID_PARAMETER, "not enough injected noise rows for this run");
        if (rq.prop_mode != DTB_PROP_THRESHOLD && !inj_u) return fail(DTB_INVALID_PARAMETER, "noise train needs injected uniforms");
    }
    DTB_TRY(use_substep_params(ts));
    struct PlainView {
        Engine* e;
        bool on;
        ~PlainView() { if (on) e->use_substep_params(1); }
    } restore{this, ts > 1};
    const int acc = acc_of(rq.syn_mode);
    if (acc == ACC_EXACT) DTB_TRY(ensure_dj());
    if (acc == ACC_FIXED) DTB_TRY(ensure_djf());
    uint32_t cap = std::min<uint32_t>(rq.iters, 4096u);
    if (record) cap = std::min<uint32_t>(cap, std::max<uint32_t>(1u, static_cast<uint32_t>((512ull << 20) / (4ull * n_words))));
    DTB_TRY(ensure_hist(cap, record, samples));
    if (isyn_any) DTB_TRY(ensure_isum(cap, sisyn));
    uint32_t kflags = 0;
    if (samples) kflags |= kFlagSample;
    if (rq.flags & DTB_RUN_USE_OU) kflags |= kFlagUseOU;
    if (freq || vmean) kflags |= kFlagStats;
    if (record) kflags |= kFlagRecord;
    if (!pull) kflags |= kFlagList;
    if (injected) kflags |= kFlagInjected;
    const LaunchBatch b = single_batch();
    const int pm = static_cast<int>(rq.prop_mode);
    const int wt = static_cast<int>(wtype);
    const bool time_k = (rq.flags & DTB_RUN_TIME_KERNELS) != 0;
    uint64_t tune_at = ~0ull;   // run-relative step at which the push variants are timed
    if (!pull) {
        DTB_CU(push_prepare(acc, wt, push_cfg, sm_count, &push_ctas));
        if (autotune && !push_tuned[acc] && ts == 1) {
            // time the variants on a live spike list, once the network has left its quiet start
            const uint64_t settle = 300;
            tune_at = steps >= settle ? 1 : (settle - steps < rq.iters ? settle - steps : ~0ull);
        }
    }
    set_u64_kernel<<<1, 1, 0, stream>>>(events, 0ull);
    DTB_CU(cudaGetLastError());
    uint32_t launches = 1;
    double ms_total = 0.0;
    double kms[4] = {0.0, 0.0, 0.0, 0.0};
    uint32_t done = 0;
    while (done < rq.iters) {
        const uint32_t rows = std::min(cap, rq.iters - done);
        const bool last_chunk = done + rows == rq.iters;
        DTB_TRY(begin_run_chunk(steps, rows, freq || vmean));
        if (isyn_any) DTB_CU(cudaMemsetAsync(hist_isum, 0, sizeof(long long) * rows * P * 5, stream));
        ++launches;
        std::vector<std::pair<int, size_t>> timed;   // (kernel class, event pair index)
        if (time_k) DTB_TRY(ensure_timing_events(6 * static_cast<size_t>(rows) + 4));   // 2 events x (3 launches per step + 1)
        uint32_t chunk_launches = 0;
        auto timed_launch = [&](int cls, auto&& fn) -> int {
            if (time_k) DTB_CU(cudaEventRecord(tev[2 * timed.size()], stream));
            DTB_CU(fn());
            if (time_k) {
                DTB_CU(cudaEventRecord(tev[2 * timed.size() + 1], stream));
                timed.emplace_back(cls, timed.size());
            }
            ++chunk_launches;
            return DTB_OK;
        };
        // the chunk's launches; `tuning` false while a graph is being captured
        auto issue = [&](bool tuning) -> int {
            for (uint32_t s = 0; s < rows; ++s) {
                const bool first = (done + s) == 0;
                if (pull) {
                    DTB_TRY(timed_launch(2, [&] { return launch_pull(b, first ? 0 : 1, wt, kflags, pm, stream); }));
                    continue;
                }
                for (uint32_t k = 0; k < ts; ++k) {
                    // substeps after the first fold nothing new: J decays with no input
                    const int jm = jmode_of(rq.syn_mode, first && k == 0);
                    const int jmk = k == 0 ? jm : (jm == J_ASIS ? jmode_of(rq.syn_mode, false) : jm);
                    const uint32_t f = ts > 1 ? (kflags | substep_flags(k, ts)) : kflags;
                    DTB_TRY(timed_launch(0, [&] { return launch_lif(b, jmk, f, pm, stream); }));
                }
                if (tuning && tune_at == done + s) {
                    DTB_TRY(tune_push(b, acc));
                    if (!push_tuned[acc]) tune_at = tune_acc[acc].next_step(tune_at);
                }
                DTB_TRY(timed_launch(1, [&] { return launch_push(b, acc, wt, push_cfg, push_ctas, stream); }));
                chunk_launches += push_extra_launches(b, acc, push_cfg);
                if (isyn_any) DTB_TRY(timed_launch(3, [&] { return launch_stat_isyn(b, acc, sm_count, stream); }));
            }
            if (last_chunk && (acc == ACC_EXACT || acc == ACC_FIXED) && !pull)
                DTB_TRY(timed_launch(3, [&] { return launch_fold_finish(b, acc, stream); }));
            if (last_chunk && pull) DTB_TRY(timed_launch(3, [&] { return launch_gather_finish(b, wt, stream); }));
            return DTB_OK;
        };
        DTB_CU(cudaEventRecord(ev0, stream));
        bool eager_graphable = false;
        // a push chunk with no tuning pending and no per-kernel timing: replay its graph once its
        // shape has been seen before (the kernels read every per-run value from device memory)
        const bool graphable = use_graph && !pull && !time_k && !(tune_at >= done && tune_at < done + rows);
        const uint64_t key[10] = {rows, kflags, static_cast<uint64_t>(pm), rq.syn_mode,
                                  static_cast<uint64_t>(push_cfg.kind) * 100000 + push_cfg.param * 100 + push_cfg.lpr,
                                  push_ctas, done == 0, last_chunk, isyn_any, ts};
        if (graphable && graph && std::memcmp(key, graph_key, sizeof(key)) == 0) {
            DTB_CU(cudaGraphLaunch(graph, stream));
            ++graph_launches;
            // launches of the replayed chunk, counted as the eager path does
            chunk_launches = rows * (ts + 1u + push_extra_launches(b, acc, push_cfg) + (isyn_any ? 1u : 0u)) +
                             (last_chunk && acc != ACC_FLOAT ? 1u : 0u);
        } else if (graphable && std::memcmp(key, seen_key, sizeof(key)) == 0 && ++seen_count >= 2 &&
                   seen_ms_per_step < kGraphMaxMsPerStep) {
            if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
            cudaGraph_t g = nullptr;
            DTB_CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            const int st = issue(false);
            const cudaError_t ee = cudaStreamEndCapture(stream, &g);
            if (st != DTB_OK) { if (g) cudaGraphDestroy(g); return st; }
            if (ee != cudaSuccess) return cuda_fail(ee, "cudaStreamEndCapture");
            const cudaError_t ie = cudaGraphInstantiate(&graph, g, 0);
            cudaGraphDestroy(g);
            if (ie != cudaSuccess) { graph = nullptr; return cuda_fail(ie, "cudaGraphInstantiate"); }
            std::memcpy(graph_key, key, sizeof(key));
            DTB_CU(cudaGraphLaunch(graph, stream));
            ++graph_launches;
        } else {
            if (graphable && std::memcmp(key, seen_key, sizeof(key)) != 0) {
                std::memcpy(seen_key, key, sizeof(key));
                seen_count = 0;
            }
            eager_graphable = graphable;
            DTB_TRY(issue(true));
        }
        launches += chunk_launches;
        DTB_CU(cudaEventRecord(ev1, stream));
        DTB_CU(cudaEventSynchronize(ev1));
        float ms = 0.f;
        DTB_CU(cudaEventElapsedTime(&ms, ev0, ev1));
        ms_total += ms;
        if (eager_graphable) seen_ms_per_step = ms / static_cast<float>(rows);
        for (const auto& tp : timed) {
            float km = 0.f;
            DTB_CU(cudaEventElapsedTime(&km, tev[2 * tp.second], tev[2 * tp.second + 1]));
            kms[tp.first] += km;
        }
        for (uint32_t s = 0; s < rows * ts; ++s) {
            volatile float tt = t + view.dt;    // dt, or dt / t_steps per substep
            t = tt;
        }
        steps += rows;
        DTB_TRY(finish_hist(rows, done, out, freq, vmean, record));
        if (samples) DTB_TRY(finish_samples(rows, done, out));
        if (isyn_any) DTB_TRY(finish_isum(rows, done, out, imean, rimean, sisyn));
        done += rows;
    }
    for (int k = 0; k < 4; ++k) out.kernel_ms[k] = kms[k];
    out.launches = launches;
    Clock ck;
    unsigned long long ev = 0;
    DTB_CU(cudaMemcpyAsync(&ck, clock, sizeof(Clock), cudaMemcpyDeviceToHost, stream));
    DTB_CU(cudaMemcpyAsync(&ev, events, sizeof(ev), cudaMemcpyDeviceToHost, stream));
    DTB_CU(cudaStreamSynchronize(stream));
    out.events = ev;
    out.device_ms = ms_total;
    if (ck.n != steps) return fail(DTB_DEVICE_FAULT, "device clock out of step with the host");
    if (ck.err) {
        set_clock_kernel<<<1, 1, 0, stream>>>(clock, ck.t, ck.n);
        cudaStreamSynchronize(stream);
        return fail(DTB_DEVICE_FAULT, "kernel check failed, error bits " + std::to_string(ck.err));
    }
    return DTB_OK;
}

// The variant to keep: the fastest mean, except that variants within kTuneTie of it
// count as tied (a few sampled steps do not resolve smaller differences) and the tie
// goes to the concurrent population-local push, then to list order.  On the regional
// 5M network local:8 and local:2008 come within 1-3 % of each other on the sampled
// bursts, while over whole runs local:2008 is 6.6 % faster (push 0.548 vs 0.585 ms).
constexpr float kTuneTie = 0.02f;
static void pick_best(TuneResult& res) {
    if (res.report.empty()) { res.best_ms = 0.0f; return; }
    float fastest = 1e30f;
    for (const TuneEntry& t : res.report) fastest = std::min(fastest, t.ms);
    const TuneEntry* pick = nullptr;
    for (const TuneEntry& t : res.report) {
        if (t.ms > fastest * (1.0f + kTuneTie)) continue;
        const bool preferred = t.cfg.kind == PUSH_LOCAL && t.cfg.param == kLocalConcurrent;
        if (!pick || (preferred && !(pick->cfg.kind == PUSH_LOCAL && pick->cfg.param == kLocalConcurrent))) pick = &t;
    }
    res.best = pick->cfg;
    res.best_ms = pick->ms;
}

// Time every push variant on the spike list the LIF kernel just wrote, into
// scratch accumulators so the simulation state is untouched, and return the
// fastest.  `views` are the host copies of the launch's networks.
int tune_push_views(const LaunchBatch& b, const std::vector<NetView>& views, int acc, int wtype, int sm_count,
                    cudaStream_t stream, cudaEvent_t ev[2], TuneResult& res) {
    uint32_t count = 0;
    DTB_CU(cudaMemcpyAsync(&count, b.spikes.count, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    DTB_CU(cudaStreamSynchronize(stream));
    uint64_t total_n = 0;
    for (const NetView& v : views) total_n += v.n_pad;
    res.sampled = false;
    ++res.observed;
    res.peak = std::max(res.peak, count);
    if (res.observed <= res.observe || count < res.peak / 2 || count < std::max<uint64_t>(64u, total_n / 500u)) {
        if (res.observed >= res.observe + kTuneGiveUp) {
            // settle: the best of the samples so far, or the default variant
            res.tuned = true;
            pick_best(res);
        }
        return DTB_OK;
    }
    res.sampled = true;
    const size_t per = acc == ACC_EXACT ? sizeof(long long) * 4 : acc == ACC_FIXED ? sizeof(unsigned long long) * 2 : sizeof(float4);
    void* scratch = nullptr;
    NetView* tview = nullptr;
    DTB_CU(cudaMalloc(&scratch, per * total_n));
    if (cudaMalloc(reinterpret_cast<void**>(&tview), sizeof(NetView) * views.size()) != cudaSuccess) {
        cudaFree(scratch);
        return cuda_fail(cudaErrorMemoryAllocation, "tune_push");
    }
    std::vector<NetView> tv(views);
    size_t off = 0;
    for (NetView& v : tv) {
        char* base = static_cast<char*>(scratch) + off * per;
        if (acc == ACC_EXACT) v.dJ = reinterpret_cast<long long*>(base);
        else if (acc == ACC_FIXED) v.dJf = reinterpret_cast<unsigned long long*>(base);
        else v.J = reinterpret_cast<float4*>(base);
        off += v.n_pad;
    }
    std::vector<TuneEntry> step;
    auto body = [&]() -> int {
        DTB_CU(cudaMemcpyAsync(tview, tv.data(), sizeof(NetView) * tv.size(), cudaMemcpyHostToDevice, stream));
        DTB_CU(cudaMemsetAsync(scratch, 0, per * total_n, stream));
        LaunchBatch tb = b;
        tb.nets = tview;
        for (const PushCfg& c : kPushCands) {
            if (c.kind == PUSH_LOCAL && (acc == ACC_EXACT || b.windows_total == 0)) continue;
            uint32_t ctas = 0;
            DTB_CU(push_prepare(acc, wtype, c, sm_count, &ctas));
            float ms_min = 1e30f;
            for (int rep = 0; rep < 3; ++rep) {
                set_u32_kernel<<<1, 1, 0, stream>>>(b.spikes.count, count);
                DTB_CU(cudaEventRecord(ev[0], stream));
                DTB_CU(launch_push(tb, acc, wtype, c, ctas, stream));
                DTB_CU(cudaEventRecord(ev[1], stream));
                DTB_CU(cudaEventSynchronize(ev[1]));
                float ms = 0.f;
                DTB_CU(cudaEventElapsedTime(&ms, ev[0], ev[1]));
                ms_min = std::min(ms_min, ms);
            }
            step.push_back({c, ms_min});
        }
        set_u32_kernel<<<1, 1, 0, stream>>>(b.spikes.count, count);
        DTB_CU(cudaGetLastError());
        return DTB_OK;
    };
    const int st = body();
    cudaStreamSynchronize(stream);
    cudaFree(scratch);
    cudaFree(tview);
    if (st != DTB_OK) return st;
    // running mean per variant over the samples
    if (res.report.size() != step.size()) {
        res.report = step;
        res.samples = 1;
    } else {
        ++res.samples;
        for (size_t k = 0; k < step.size(); ++k)
            res.report[k].ms += (step[k].ms - res.report[k].ms) / static_cast<float>(res.samples);
    }
    if (res.samples < res.want) return DTB_OK;
    res.tuned = true;
    pick_best(res);
    return DTB_OK;
}

int Engine::tune_push(const LaunchBatch& b, int acc) {
    if (!tune_ev[0]) {
        DTB_CU(cudaEventCreate(&tune_ev[0]));
        DTB_CU(cudaEventCreate(&tune_ev[1]));
    }
    TuneResult& res = tune_acc[acc];
    DTB_TRY(tune_push_views(b, {view}, acc, static_cast<int>(wtype), sm_count, stream, tune_ev, res));
    if (!res.tuned) return DTB_OK;
    push_cfg = res.best;
    push_tuned[acc] = true;
    tuned_ms = res.best_ms;
    tune_report = res.report;
    DTB_CU(push_prepare(acc, static_cast<int>(wtype), push_cfg, sm_count, &push_ctas));
    return DTB_OK;
}

int Engine::ensure_timing_events(size_t count) {
    while (tev.size() < count) {
        cudaEvent_t e;
        DTB_CU(cudaEventCreate(&e));
        tev.push_back(e);
    }
    return DTB_OK;
}

int Engine::info(dtb_engine_info& inf) const {
    inf.n_neurons = n;
    inf.n_pops = P;
    inf.n_edges = n_edges;
    inf.device_bytes = dev_bytes;
    inf.step = steps;
    inf.t = t;
    inf.weight_type = wtype;
    inf.has_push = has_push;
    inf.has_pull = has_pull;
    inf.per_neuron_params = per_neuron;
    inf.push_kind = static_cast<uint32_t>(push_cfg.kind);
    inf.push_param = static_cast<uint32_t>(push_cfg.lpr != 32 ? 1000 + push_cfg.lpr : push_cfg.param);
    inf.push_tuned_ms = tuned_ms;
    inf.local_windows = n_windows;
    inf.fixed_shift = fix_shift;
    inf.graph_launches = graph_launches;
    return DTB_OK;
}

int Engine::populations(uint32_t* ids, uint32_t* counts) const {
    for (uint32_t p = 0; p < P; ++p) {
        if (ids) ids[p] = pop_ids[p];
        if (counts) counts[p] = pop_off[p + 1] - pop_off[p];
    }
    return DTB_OK;
}

static void to_per_neuron(Engine& e) {
    if (e.per_neuron) return;
    e.neuron_raw.resize(e.n);
    for (uint32_t p = 0; p < e.P; ++p)
        for (uint32_t i = e.pop_off[p]; i < e.pop_off[p + 1]; ++i) e.neuron_raw[i] = e.pop_raw[p];
    e.per_neuron = true;
}

int Engine::update_props(uint32_t cnt, const uint32_t* nid, const uint32_t* pid, const float* val) {
    if (cnt == 0) return DTB_OK;
    if (!nid || !pid || !val) return fail(DTB_INVALID_PARAMETER, "NULL array");
    to_per_neuron(*this);
    for (uint32_t k = 0; k < cnt; ++k) {
        if (nid[k] >= n) continue;   // the reference ignores out-of-range neurons (property.cpp:72)
        float* f = nullptr;
        if (!raw_field(neuron_raw[nid[k]], pid[k], &f)) continue;
        *f = val[k];
    }
    return upload_params();
}

int Engine::update_prop_cols(uint32_t cnt, const uint32_t* pid, const uint32_t* pop, const float* val, int assign) {
    if (cnt == 0) return DTB_OK;
    if (!pid || !pop || !val) return fail(DTB_INVALID_PARAMETER, "NULL array");
    for (uint32_t k = 0; k < cnt; ++k) {
        for (uint32_t p = 0; p < P; ++p) {
            if (pop_ids[p] != pop[k]) continue;
            float* f = nullptr;
            if (!raw_field(pop_raw[p], pid[k], &f)) continue;
            *f = assign ? val[k] : *f * val[k];
            if (per_neuron) {
                for (uint32_t i = pop_off[p]; i < pop_off[p + 1]; ++i) {
                    float* g = nullptr;
                    raw_field(neuron_raw[i], pid[k], &g);
                    *g = assign ? val[k] : *g * val[k];
                }
            }
        }
    }
    return upload_params();
}

// Gamma(alpha, 1) by Marsaglia & Tsang (2000), "A simple method for generating
// gamma variables", with the alpha < 1 boost U^(1/alpha) * Gamma(alpha + 1).
static double sample_gamma(double alpha, std::mt19937_64& rng) {
    std::uniform_real_distribution<double> uni(0.0, 1.0);
    std::normal_distribution<double> nrm(0.0, 1.0);
    if (alpha <= 0.0) return 0.0;
    double scale = 1.0;
    if (alpha < 1.0) {
        scale = std::pow(1.0 - uni(rng), 1.0 / alpha);
        alpha += 1.0;
    }
    const double d = alpha - 1.0 / 3.0, c = 1.0 / std::sqrt(9.0 * d);
    for (;;) {
        double x, v;
        do { x = nrm(rng); v = 1.0 + c * x; } while (v <= 0.0);
        v = v * v * v;
        const double u = 1.0 - uni(rng);
        const double xx = x * x;
        if (u < 1.0 - 0.0331 * xx * xx) return scale * d * v;
        if (std::log(u) < 0.5 * xx + d * (1.0 - v + std::log(v))) return scale * d * v;
    }
}

int Engine::update_gamma(uint32_t cnt, const uint32_t* pid, const uint32_t* pop, const float* alpha, const float* beta) {
    if (cnt == 0) return DTB_OK;
    if (!pid || !pop || !alpha || !beta) return fail(DTB_INVALID_PARAMETER, "NULL array");
    for (uint32_t k = 0; k < cnt; ++k)
        if (!(alpha[k] >= 0.0f) || !(beta[k] > 0.0f)) return fail(DTB_INVALID_PARAMETER, "gamma needs alpha >= 0 and beta > 0");
    to_per_neuron(*this);
    std::mt19937_64 rng(seed ^ (0x9E3779B97F4A7C15ull * (++gamma_calls)));
    for (uint32_t k = 0; k < cnt; ++k) {
        for (uint32_t p = 0; p < P; ++p) {
            if (pop_ids[p] != pop[k]) continue;
            for (uint32_t i = pop_off[p]; i < pop_off[p + 1]; ++i) {
                float* f = nullptr;
                if (!raw_field(neuron_raw[i], pid[k], &f)) break;
                *f = static_cast<float>(sample_gamma(alpha[k], rng) / beta[k]);
            }
        }
    }
    return upload_params();
}

int Engine::read_property(uint32_t prop_id, float* dst) const {
    if (!dst) return fail(DTB_INVALID_PARAMETER, "NULL destination");
    if (prop_id >= DTB_N_PROPS) return fail(DTB_INVALID_PARAMETER, "unknown property id");
    for (uint32_t p = 0; p < P; ++p) {
        for (uint32_t i = pop_off[p]; i < pop_off[p + 1]; ++i) {
            RawParams r = per_neuron ? neuron_raw[i] : pop_raw[p];
            float* f = nullptr;
            raw_field(r, prop_id, &f);
            dst[i] = *f;
        }
    }
    return DTB_OK;
}

int Engine::set_ou(uint32_t cnt, const uint32_t* pop, const float* mean, const float* sigma, const float* tau) {
    if (cnt == 0) return DTB_OK;
    if (!pop || !mean || !sigma || !tau) return fail(DTB_INVALID_PARAMETER, "NULL array");
    for (uint32_t k = 0; k < cnt; ++k)
        if (!(tau[k] > 0.0f) || !(sigma[k] >= 0.0f)) return fail(DTB_INVALID_PARAMETER, "OU needs tau > 0 and sigma >= 0");
    for (uint32_t k = 0; k < cnt; ++k) {
        for (uint32_t p = 0; p < P; ++p) {
            if (pop_ids[p] != pop[k]) continue;
            pop_raw[p].ou_mean = mean[k];
            pop_raw[p].ou_sigma = sigma[k];
            pop_raw[p].ou_tau = tau[k];
            if (per_neuron)
                for (uint32_t i = pop_off[p]; i < pop_off[p + 1]; ++i) {
                    neuron_raw[i].ou_mean = mean[k];
                    neuron_raw[i].ou_sigma = sigma[k];
                    neuron_raw[i].ou_tau = tau[k];
                }
            if (!ou_set[p]) {
                // first configuration resets the population's OU current to its mean (src/block.cpp:244-266)
                fill_range_kernel<<<64, 256, 0, stream>>>(iou, pop_off[p], pop_off[p + 1], mean[k]);
                DTB_CU(cudaGetLastError());
                ou_set[p] = 1;
            }
        }
    }
    return upload_params();
}

// Updatesample (dist_simulator.cpp:3635): the neurons whose spike, V and OU
// current every step reports.  Duplicates are merged; outputs follow the order
// of first appearance in `idx`.
int Engine::set_samples(uint32_t count, const uint32_t* idx) {
    if (count && !idx) return fail(DTB_INVALID_PARAMETER, "NULL sample list");
    std::vector<uint32_t> bits(n_words, 0);
    for (uint32_t k = 0; k < count; ++k) {
        if (idx[k] >= n) return fail(DTB_INVALID_PARAMETER, "sample index outside the network");
        bits[idx[k] >> 5] |= 1u << (idx[k] & 31u);
    }
    std::vector<uint32_t> pre(n_words, 0);
    uint32_t total = 0;
    for (uint32_t w = 0; w < n_words; ++w) {
        pre[w] = total;
        total += static_cast<uint32_t>(__builtin_popcount(bits[w]));
    }
    // slot of each listed neuron (slots are ascending neuron order)
    sample_order.assign(count, 0);
    for (uint32_t k = 0; k < count; ++k) {
        const uint32_t i = idx[k], w = i >> 5, b = i & 31u;
        sample_order[k] = pre[w] + static_cast<uint32_t>(__builtin_popcount(bits[w] & ((1u << b) - 1u)));
    }
    if (!sample_bits) {
        DTB_TRY(dalloc(sample_bits, n_words));
        DTB_TRY(dalloc(sample_pre, n_words));
    }
    DTB_CU(cudaMemcpyAsync(sample_bits, bits.data(), sizeof(uint32_t) * n_words, cudaMemcpyHostToDevice, stream));
    DTB_CU(cudaMemcpyAsync(sample_pre, pre.data(), sizeof(uint32_t) * n_words, cudaMemcpyHostToDevice, stream));
    DTB_CU(cudaStreamSynchronize(stream));
    if (total != n_samples) {
        dfree(hist_sspk);
        dfree(hist_sv);
        dfree(hist_siou);
        dfree(hist_sisyn);
        hist_sspk = nullptr;
        hist_sv = hist_siou = hist_sisyn = nullptr;
        sample_cap = 0;
        sisyn_cap = 0;
    }
    n_samples = total;
    return refresh_view();
}

int Engine::set_noise(uint32_t source, uint32_t rows, const float* z, const float* u) {
    if (source > DTB_NOISE_INJECTED) return fail(DTB_INVALID_PARAMETER, "unknown noise source");
    dfree(inj_z);
    dfree(inj_u);
    inj_z = inj_u = nullptr;
    inj_rows = 0;
    noise_src = static_cast<int>(source);
    if (source == DTB_NOISE_INJECTED) {
        if (rows == 0 || !z) return fail(DTB_INVALID_PARAMETER, "injected noise needs rows and z");
        DTB_TRY(dalloc(inj_z, static_cast<size_t>(rows) * n_pad));
        DTB_CU(cudaMemcpy2DAsync(inj_z, sizeof(float) * n_pad, z, sizeof(float) * n, sizeof(float) * n, rows,
                                 cudaMemcpyHostToDevice, stream));
        if (u) {
            DTB_TRY(dalloc(inj_u, static_cast<size_t>(rows) * n_pad));
            DTB_CU(cudaMemcpy2DAsync(inj_u, sizeof(float) * n_pad, u, sizeof(float) * n, sizeof(float) * n, rows,
                                     cudaMemcpyHostToDevice, stream));
        }
        inj_rows = rows;
        inj_first = steps;
        set_u64_kernel<<<1, 1, 0, stream>>>(&clock->inj_base, steps);
        DTB_CU(cudaGetLastError());
    }
    DTB_CU(cudaStreamSynchronize(stream));
    return refresh_view();
}

int Engine::read_state(int which, void* dst) {
    if (!dst) return fail(DTB_INVALID_PARAMETER, "NULL destination");
    switch (which) {
        case DTB_STATE_V: DTB_CU(cudaMemcpyAsync(dst, V, sizeof(float) * n, cudaMemcpyDeviceToHost, stream)); break;
        case DTB_STATE_J: DTB_CU(cudaMemcpyAsync(dst, J, sizeof(float4) * n, cudaMemcpyDeviceToHost, stream)); break;
        case DTB_STATE_I_OU: DTB_CU(cudaMemcpyAsync(dst, iou, sizeof(float) * n, cudaMemcpyDeviceToHost, stream)); break;
        case DTB_STATE_T_LAST: DTB_CU(cudaMemcpyAsync(dst, tlast, sizeof(float) * n, cudaMemcpyDeviceToHost, stream)); break;
        default: return fail(DTB_INVALID_PARAMETER, "unknown state id");
    }
    DTB_CU(cudaStreamSynchronize(stream));
    return DTB_OK;
}

int Engine::write_state(int which, const void* src) {
    if (!src) return fail(DTB_INVALID_PARAMETER, "NULL source");
    switch (which) {
        case DTB_STATE_V: DTB_CU(cudaMemcpyAsync(V, src, sizeof(float) * n, cudaMemcpyHostToDevice, stream)); break;
        case DTB_STATE_J: DTB_CU(cudaMemcpyAsync(J, src, sizeof(float4) * n, cudaMemcpyHostToDevice, stream)); break;
        case DTB_STATE_I_OU: DTB_CU(cudaMemcpyAsync(iou, src, sizeof(float) * n, cudaMemcpyHostToDevice, stream)); break;
        case DTB_STATE_T_LAST: DTB_CU(cudaMemcpyAsync(tlast, src, sizeof(float) * n, cudaMemcpyHostToDevice, stream)); break;
        default: return fail(DTB_INVALID_PARAMETER, "unknown state id");
    }
    DTB_CU(cudaStreamSynchronize(stream));
    return DTB_OK;
}

int Engine::read_out_csr(uint32_t* n_rows, uint64_t* n_edges_out, uint32_t* rows, uint64_t* row_ptr, uint32_t* post,
                         uint8_t* kind, float* weight) {
    if (!has_push) return fail(DTB_UNSUPPORTED, "network was built without the out-degree CSR");
    std::vector<unsigned long long> ptr(static_cast<size_t>(n) + 1);
    DTB_CU(cudaMemcpyAsync(ptr.data(), out_ptr, sizeof(unsigned long long) * (n + 1), cudaMemcpyDeviceToHost, stream));
    DTB_CU(cudaStreamSynchronize(stream));
    uint32_t nr = 0;
    for (uint32_t j = 0; j < n; ++j) {
        if (ptr[j + 1] > ptr[j]) {
            if (rows) rows[nr] = j;
            if (row_ptr) row_ptr[nr] = ptr[j];
            ++nr;
        }
    }
    if (row_ptr) row_ptr[nr] = ptr[n];
    *n_rows = nr;
    *n_edges_out = n_edges;
    if (post || kind) {
        std::vector<uint32_t> col(n_edges);
        DTB_CU(cudaMemcpyAsync(col.data(), out_col, sizeof(uint32_t) * n_edges, cudaMemcpyDeviceToHost, stream));
        DTB_CU(cudaStreamSynchronize(stream));
        for (uint64_t e = 0; e < n_edges; ++e) {
            if (post) post[e] = col[e] & kIndexMask;
            if (kind) kind[e] = static_cast<uint8_t>(col[e] >> 31);
        }
    }
    if (weight) {
        const int wb = weight_bytes();
        std::vector<uint8_t> w(static_cast<size_t>(n_edges) * wb);
        DTB_CU(cudaMemcpyAsync(w.data(), out_w, w.size(), cudaMemcpyDeviceToHost, stream));
        DTB_CU(cudaStreamSynchronize(stream));
        const uint32_t as_in = wtype == W_F32 ? DTB_W_F32 : wtype == W_BF16 ? DTB_W_BF16 : wtype == W_F16 ? DTB_W_F16 : DTB_W_U8;
        for (uint64_t e = 0; e < n_edges; ++e) weight_to_f32(w.data(), as_in, e, weight[2 * e], weight[2 * e + 1]);
    }
    return DTB_OK;
}

// State blob: header, V, i_ou, t_last, J, both spike-bit buffers.
struct BlobHeader {
    uint64_t magic, n, n_words, steps;
    float t;
    uint32_t pad;
};
static constexpr uint64_t kBlobMagic = 0x44544242'53544154ull;

uint64_t Engine::state_size() const {
    return sizeof(BlobHeader) + sizeof(float) * 3ull * n + sizeof(float4) * static_cast<uint64_t>(n) + 8ull * n_words;
}

int Engine::save_state(void* blob, uint64_t bytes) {
    if (!blob || bytes < state_size()) return fail(DTB_INVALID_PARAMETER, "state blob too small");
    uint8_t* p = static_cast<uint8_t*>(blob);
    BlobHeader h{kBlobMagic, n, n_words, steps, t, 0};
    std::memcpy(p, &h, sizeof(h));
    p += sizeof(h);
    DTB_CU(cudaMemcpyAsync(p, V, sizeof(float) * n, cudaMemcpyDeviceToHost, stream)); p += sizeof(float) * n;
    DTB_CU(cudaMemcpyAsync(p, iou, sizeof(float) * n, cudaMemcpyDeviceToHost, stream)); p += sizeof(float) * n;
    DTB_CU(cudaMemcpyAsync(p, tlast, sizeof(float) * n, cudaMemcpyDeviceToHost, stream)); p += sizeof(float) * n;
    DTB_CU(cudaMemcpyAsync(p, J, sizeof(float4) * n, cudaMemcpyDeviceToHost, stream)); p += sizeof(float4) * n;
    DTB_CU(cudaMemcpyAsync(p, bits0, 4ull * n_words, cudaMemcpyDeviceToHost, stream)); p += 4ull * n_words;
    DTB_CU(cudaMemcpyAsync(p, bits1, 4ull * n_words, cudaMemcpyDeviceToHost, stream));
    DTB_CU(cudaStreamSynchronize(stream));
    return DTB_OK;
}

int Engine::load_state(const void* blob, uint64_t bytes) {
    if (!blob || bytes < state_size()) return fail(DTB_INVALID_PARAMETER, "state blob too small");
    const uint8_t* p = static_cast<const uint8_t*>(blob);
    BlobHeader h;
    std::memcpy(&h, p, sizeof(h));
    if (h.magic != kBlobMagic || h.n != n || h.n_words != n_words) return fail(DTB_INVALID_PARAMETER, "state blob is for another network");
    p += sizeof(h);
    DTB_CU(cudaMemcpyAsync(V, p, sizeof(float) * n, cudaMemcpyHostToDevice, stream)); p += sizeof(float) * n;
    DTB_CU(cudaMemcpyAsync(iou, p, sizeof(float) * n, cudaMemcpyHostToDevice, stream)); p += sizeof(float) * n;
    DTB_CU(cudaMemcpyAsync(tlast, p, sizeof(float) * n, cudaMemcpyHostToDevice, stream)); p += sizeof(float) * n;
    DTB_CU(cudaMemcpyAsync(J, p, sizeof(float4) * n, cudaMemcpyHostToDevice, stream)); p += sizeof(float4) * n;
    DTB_CU(cudaMemcpyAsync(bits0, p, 4ull * n_words, cudaMemcpyHostToDevice, stream)); p += 4ull * n_words;
    DTB_CU(cudaMemcpyAsync(bits1, p, 4ull * n_words, cudaMemcpyHostToDevice, stream));
    if (dJ) DTB_CU(cudaMemsetAsync(dJ, 0, sizeof(long long) * 4 * n_pad, stream));
    if (dJf) DTB_CU(cudaMemsetAsync(dJf, 0, sizeof(unsigned long long) * 2 * n_pad, stream));
    set_clock_kernel<<<1, 1, 0, stream>>>(clock, h.t, h.steps);
    DTB_CU(cudaGetLastError());
    DTB_CU(cudaStreamSynchronize(stream));
    steps = h.steps;
    t = h.t;
    return DTB_OK;
}

}  // namespace dtb

// ===========================================================================
// C-ABI
// ===========================================================================
using dtb::Engine;

namespace {

template <class F>
int32_t guarded(F&& f) {
    try {
        return static_cast<int32_t>(f());
    } catch (const std::bad_alloc&) {
        return dtb::fail(DTB_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& e) {
        return dtb::fail(DTB_INVALID_PARAMETER, e.what());
    }
}

Engine* as_engine(void* p) { return static_cast<Engine*>(p); }

}  // namespace

extern "C" {

int32_t dtb_abi_version(void) { return DTB_ABI_VERSION; }

int32_t dtb_engine_version(void) { return 1 * 1000 + 0 * 100 + 0; }

const char* dtb_status_string(int32_t s) {
    switch (s) {
        case DTB_OK: return "SNN_OK";
        case DTB_INVALID_PARAMETER: return "SNN_INVALID_PARAMETER";
        case DTB_UNSET_SAMPLE_FAILURE: return "SNN_UNSET_SAMPLE_FAILURE";
        case DTB_UNSUPPORTED: return "SNN_UNSUPPORTED";
        case DTB_NOT_ENABLE_METRIC: return "SNN_NOT_ENABLE_METRIC";
        case DTB_INVALID_NETWORK: return "SNN_INVALID_NETWORK";
        case DTB_OUT_OF_MEMORY: return "DTB_OUT_OF_MEMORY";
        case DTB_CUDA_ERROR: return "DTB_CUDA_ERROR";
        case DTB_DEVICE_FAULT: return "DTB_DEVICE_FAULT";
        case DTB_IO_ERROR: return "DTB_IO_ERROR";
        case DTB_NO_DEVICE: return "DTB_NO_DEVICE";
        default: return "DTB_UNKNOWN_STATUS";
    }
}

const char* dtb_last_error(void) { return dtb::last_error(); }

void dtb_default_options(dtb_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->dt = 0.1f;
    o->weight_type = DTB_W_F32;
    o->seed = 0;
    o->build_push = 1;
    o->build_pull = 0;
    o->ou_mean = 0.6f;
    o->ou_sigma = 0.2f;
    o->ou_tau = 10.0f;
}

int32_t dtb_create(const dtb_network_arrays* net, const dtb_options* opt, void** engine) {
    if (!net || !opt || !engine) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    *engine = nullptr;
    return guarded([&]() -> int {
        auto* e = new Engine();
        const int s = e->create_from_arrays(*net, *opt);
        if (s != DTB_OK) { delete e; return s; }
        *engine = e;
        return DTB_OK;
    });
}

int32_t dtb_create_structured(const dtb_structured_spec* spec, const dtb_options* opt, void** engine) {
    if (!spec || !opt || !engine) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    *engine = nullptr;
    return guarded([&]() -> int {
        auto* e = new Engine();
        const int s = e->create_structured(*spec, *opt);
        if (s != DTB_OK) { delete e; return s; }
        *engine = e;
        return DTB_OK;
    });
}

int32_t dtb_create_from_npz(const char* path, const dtb_options* opt, void** engine) {
    if (!path || !opt || !engine) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    if (!*path) return dtb::fail(DTB_INVALID_PARAMETER, "empty file path");
    *engine = nullptr;
    return guarded([&]() -> int {
        auto* e = new Engine();
        const int s = e->create_from_npz(path, *opt);
        if (s != DTB_OK) { delete e; return s; }
        *engine = e;
        return DTB_OK;
    });
}

int32_t dtb_destroy(void* engine) {
    if (!engine) return dtb::fail(DTB_INVALID_PARAMETER, "NULL engine");
    delete as_engine(engine);
    return DTB_OK;
}

int32_t dtb_info(void* engine, dtb_engine_info* info) {
    if (!engine || !info) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    return as_engine(engine)->info(*info);
}

int32_t dtb_set_push_variant(void* engine, int32_t kind, int32_t param) {
    if (!engine) return dtb::fail(DTB_INVALID_PARAMETER, "NULL engine");
    Engine* e = as_engine(engine);
    if (kind < 0) {
        e->autotune = true;
        for (int a = 0; a < 3; ++a) {
            e->push_tuned[a] = false;
            e->tune_acc[a].reset();
        }
        return DTB_OK;
    }
    dtb::PushCfg cfg;
    if (!dtb::push_cfg_from_abi(kind, param, cfg)) return dtb::fail(DTB_INVALID_PARAMETER, "unknown push variant");
    e->push_cfg = cfg;
    e->autotune = false;
    return DTB_OK;
}

int32_t dtb_set_graph(void* engine, int32_t enable) {
    if (!engine) return dtb::fail(DTB_INVALID_PARAMETER, "NULL engine");
    Engine* e = as_engine(engine);
    e->use_graph = enable != 0;
    if (!e->use_graph && e->graph) {
        cudaGraphExecDestroy(e->graph);
        e->graph = nullptr;
    }
    std::memset(e->graph_key, 0, sizeof(e->graph_key));
    std::memset(e->seen_key, 0, sizeof(e->seen_key));
    return DTB_OK;
}

int32_t dtb_tuning_report(void* engine, uint32_t* n, int32_t* kinds, int32_t* params, float* ms) {
    if (!engine || !n) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    Engine* e = as_engine(engine);
    const uint32_t cap = *n;
    *n = static_cast<uint32_t>(e->tune_report.size());
    for (uint32_t i = 0; i < *n && i < cap; ++i) {
        const dtb::PushCfg& c = e->tune_report[i].cfg;
        if (kinds) kinds[i] = c.kind;
        if (params) params[i] = c.lpr != 32 ? 1000 + c.lpr : c.param;
        if (ms) ms[i] = e->tune_report[i].ms;
    }
    return DTB_OK;
}

int32_t dtb_get_stream(void* engine, void** stream) {
    if (!engine || !stream) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    *stream = as_engine(engine)->stream;
    return DTB_OK;
}

int32_t dtb_populations(void* engine, uint32_t* ids, uint32_t* counts) {
    if (!engine) return dtb::fail(DTB_INVALID_PARAMETER, "NULL engine");
    return as_engine(engine)->populations(ids, counts);
}

int32_t dtb_update_props(void* engine, uint32_t n, const uint32_t* nid, const uint32_t* pid, const float* val) {
    if (!engine) return dtb::fail(DTB_INVALID_PARAMETER, "NULL engine");
    return guarded([&] { return as_engine(engine)->update_props(n, nid, pid, val); });
}

int32_t dtb_update_prop_cols(void* engine, uint32_t n, const uint32_t* pid, const uint32_t* pop, const float* val, int32_t assign) {
    if (!engine) return dtb::fail(DTB_INVALID_PARAMETER, "NULL engine");
    return guarded([&] { return as_engine(engine)->update_prop_cols(n, pid, pop, val, assign); });
}

int32_t dtb_update_gamma(void* engine, uint32_t n, const uint32_t* pid, const uint32_t* pop, const float* alpha, const float* beta) {
    if (!engine) return dtb::fail(DTB_INVALID_PARAMETER, "NULL engine");
    return guarded([&] { return as_engine(engine)->update_gamma(n, pid, pop, alpha, beta); });
}

int32_t dtb_read_property(void* engine, uint32_t prop_id, float* values) {
    if (!engine) return dtb::fail(DTB_INVALID_PARAMETER, "NULL engine");
    return guarded([&] { return as_engine(engine)->read_property(prop_id, values); });
}

int32_t dtb_set_ou(void* engine, uint32_t n, const uint32_t* pop, const float* mean, const float* sigma, const float* tau) {
    if (!engine) return dtb::fail(DTB_INVALID_PARAMETER, "NULL engine");
    return guarded([&] { return as_engine(engine)->set_ou(n, pop, mean, sigma, tau); });
}

int32_t dtb_set_samples(void* engine, uint32_t n, const uint32_t* neuron_ids) {
    if (!engine) return dtb::fail(DTB_INVALID_PARAMETER, "NULL engine");
    return guarded([&] { return as_engine(engine)->set_samples(n, neuron_ids); });
}

int32_t dtb_set_noise(void* engine, uint32_t source, uint32_t steps, const float* z, const float* u) {
    if (!engine) return dtb::fail(DTB_INVALID_PARAMETER, "NULL engine");
    return guarded([&] { return as_engine(engine)->set_noise(source, steps, z, u); });
}

int32_t dtb_run(void* engine, const dtb_run_request* req, dtb_run_output* out) {
    if (!engine || !req || !out) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    return guarded([&] { return as_engine(engine)->run(*req, *out); });
}

int32_t dtb_read_state(void* engine, int32_t which, void* dst) {
    if (!engine) return dtb::fail(DTB_INVALID_PARAMETER, "NULL engine");
    return as_engine(engine)->read_state(which, dst);
}

int32_t dtb_write_state(void* engine, int32_t which, const void* src) {
    if (!engine) return dtb::fail(DTB_INVALID_PARAMETER, "NULL engine");
    return as_engine(engine)->write_state(which, src);
}

int32_t dtb_read_out_csr(void* engine, uint32_t* n_rows, uint64_t* n_edges, uint32_t* rows, uint64_t* row_ptr,
                         uint32_t* post, uint8_t* kind, float* weight) {
    if (!engine || !n_rows || !n_edges) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    return guarded([&] { return as_engine(engine)->read_out_csr(n_rows, n_edges, rows, row_ptr, post, kind, weight); });
}

int32_t dtb_build_out_csr_host(uint32_t n_neurons, uint64_t n_edges, const uint32_t* pre, const uint32_t* post,
                               const uint8_t* kind, uint32_t* n_rows, uint32_t* rows, uint64_t* row_ptr,
                               uint32_t* post_out, uint8_t* kind_out, uint64_t* perm) {
    if (!n_rows || (n_edges && (!pre || !post || !kind))) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    return guarded([&]() -> int {
        for (uint64_t e = 0; e < n_edges; ++e)
            if (pre[e] >= n_neurons || post[e] >= n_neurons) return dtb::fail(DTB_INVALID_NETWORK, "edge index out of range");
        std::vector<uint64_t> ptr, p;
        dtb::counting_sort(pre, n_edges, n_neurons, ptr, p);
        uint32_t nr = 0;
        for (uint32_t j = 0; j < n_neurons; ++j) {
            if (ptr[j + 1] > ptr[j]) {
                if (rows) rows[nr] = j;
                if (row_ptr) row_ptr[nr] = ptr[j];
                ++nr;
            }
        }
        if (row_ptr) row_ptr[nr] = n_edges;
        *n_rows = nr;
        for (uint64_t q = 0; q < n_edges; ++q) {
            if (post_out) post_out[q] = post[p[q]];
            if (kind_out) kind_out[q] = kind[p[q]] != 0 ? 1 : 0;
            if (perm) perm[q] = p[q];
        }
        return DTB_OK;
    });
}

int32_t dtb_state_size(void* engine, uint64_t* bytes) {
    if (!engine || !bytes) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    *bytes = as_engine(engine)->state_size();
    return DTB_OK;
}

int32_t dtb_save_state(void* engine, void* blob, uint64_t bytes) {
    if (!engine) return dtb::fail(DTB_INVALID_PARAMETER, "NULL engine");
    return as_engine(engine)->save_state(blob, bytes);
}

int32_t dtb_load_state(void* engine, const void* blob, uint64_t bytes) {
    if (!engine) return dtb::fail(DTB_INVALID_PARAMETER, "NULL engine");
    return as_engine(engine)->load_state(blob, bytes);
}

}  // extern "C"
