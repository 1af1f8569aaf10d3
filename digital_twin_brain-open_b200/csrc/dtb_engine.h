// The engine object behind the C-ABI: one network resident in one GPU's HBM.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "dtb_b200.h"
#include "dtb_device.cuh"
#include "dtb_host.h"
#include "dtb_kernels.h"

namespace dtb {

void set_error(const std::string& msg);
const char* last_error();        // message of the last failure on the calling thread
int fail(int status, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define DTB_CU(x) do { cudaError_t e__ = (x); if (e__ != cudaSuccess) return ::dtb::cuda_fail(e__, #x); } while (0)
#define DTB_TRY(x) do { int s__ = (x); if (s__ != DTB_OK) return s__; } while (0)

struct TuneEntry { PushCfg cfg; float ms; };
// Push-variant tuning state.  The tuner reads the spike count of every step for
// `observe` steps to learn the network's peak activity, then times every variant on
// `want` live spike lists of at least half that peak, kTuneStride or more steps apart;
// `best` is the variant with the smallest mean.  Bursting networks spend most of
// their push time in their bursts, which a fixed sampling step can miss.  A step that
// does not qualify is retried at the next step for kTuneEager reads, then every
// kTuneStride steps; after kTuneGiveUp reads the tuner settles for the samples it has
// (or the default variant) so a quiet network stops paying for the reads.
constexpr uint32_t kTuneObserve = 50;     // plain engine; a batch uses 0 (latency-sensitive)
constexpr uint32_t kTuneSamples = 4;      // plain engine; a batch uses 2
constexpr uint64_t kTuneStride = 47;
constexpr uint32_t kTuneEager = 200;
constexpr uint32_t kTuneGiveUp = 400;
struct TuneResult {
    uint32_t observe = kTuneObserve, want = kTuneSamples;
    bool tuned = false;
    bool sampled = false;            // the last call timed the variants
    PushCfg best{PUSH_REG, 8, 32};
    float best_ms = 0.0f;            // mean per sampled step of the best variant
    uint32_t samples = 0;
    uint32_t observed = 0;           // steps whose spike count was read
    uint32_t peak = 0;               // largest spike count seen
    std::vector<TuneEntry> report;   // per variant: mean time per sampled step
    void reset() { tuned = sampled = false; samples = observed = peak = 0; report.clear(); }
    // run-relative step of the next call after one at step `s`
    uint64_t next_step(uint64_t s) const {
        return s + ((sampled || observed >= observe + kTuneEager) ? kTuneStride : 1);
    }
};
bool push_cfg_from_abi(int kind, int param, PushCfg& cfg);
__global__ void set_u64_kernel(unsigned long long* p, unsigned long long v);
__global__ void set_u32_kernel(uint32_t* p, uint32_t v);
// Reads the live spike count and, when the step qualifies as a sample (TuneResult),
// times every push variant on it and adds the times to `res`.  A list of fewer than
// 0.2 % of the neurons never qualifies.
int tune_push_views(const LaunchBatch& b, const std::vector<NetView>& views, int acc, int wtype, int sm_count,
                    cudaStream_t stream, cudaEvent_t ev[2], TuneResult& res);
// AccMode of a push syn_mode, and the LIF kernel's J mode for a step of that mode
// (the first step of a run takes J as complete).
int acc_of(uint32_t syn_mode);
int jmode_of(uint32_t syn_mode, bool first);
// Largest fixed-point exponent s <= 32 with in_degree x (max_w x 2^s + 1/2) < 2^32,
// so no packed 32-bit field of DTB_SYN_PUSH_FIXED can carry; 0 (mode unavailable)
// for negative weights or when s would fall below 12.
uint32_t fixed_shift_for(uint64_t max_in_degree, double max_w, bool negative);

class Engine {
public:
    ~Engine();

    int init_common(const dtb_options& opt, uint32_t n);
    int create_from_arrays(const dtb_network_arrays& a, const dtb_options& opt);
    int create_structured(const dtb_structured_spec& s, const dtb_options& opt);
    int create_from_npz(const std::string& path, const dtb_options& opt);

    int run(const dtb_run_request& rq, dtb_run_output& out);
    int info(dtb_engine_info& info) const;
    int populations(uint32_t* ids, uint32_t* counts) const;
    int update_props(uint32_t n, const uint32_t* nid, const uint32_t* pid, const float* val);
    int update_prop_cols(uint32_t n, const uint32_t* pid, const uint32_t* pop, const float* val, int assign);
    int update_gamma(uint32_t n, const uint32_t* pid, const uint32_t* pop, const float* alpha, const float* beta);
    int set_ou(uint32_t n, const uint32_t* pop, const float* mean, const float* sigma, const float* tau);
    int read_property(uint32_t prop_id, float* dst) const;
    int set_noise(uint32_t source, uint32_t steps, const float* z, const float* u);
    int set_samples(uint32_t count, const uint32_t* idx);
    int read_state(int which, void* dst);
    int write_state(int which, const void* src);
    int read_out_csr(uint32_t* n_rows, uint64_t* n_edges, uint32_t* rows, uint64_t* row_ptr, uint32_t* post,
                     uint8_t* kind, float* weight);
    uint64_t state_size() const;
    int save_state(void* blob, uint64_t bytes);
    int load_state(const void* blob, uint64_t bytes);

    // ---- pieces shared with the batch / serving layers
    LaunchBatch single_batch() const;
    int refresh_view();
    int ensure_dj();
    int ensure_djf();
    int use_substep_params(uint32_t ts);   // point the view at the dt / ts constants (ts 1: the plain ones)
    int ensure_hist(uint32_t rows, bool record, bool samples = false);
    int begin_run_chunk(uint64_t run_base, uint32_t rows, bool stats);
    int finish_hist(uint32_t rows, uint32_t out_row0, const dtb_run_output& out, bool freq, bool vmean, bool record);
    int finish_samples(uint32_t rows, uint32_t out_row0, const dtb_run_output& out);
    int ensure_isum(uint32_t rows, bool sample);
    int finish_isum(uint32_t rows, uint32_t out_row0, const dtb_run_output& out, bool imean, bool receptor, bool sample);

    // identity
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaStream_t aux = nullptr;                            // second stream of the concurrent local push
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    float dt = 0.1f;
    uint32_t wtype = W_F32;
    uint64_t seed = 0;
    uint32_t n = 0, n_pad = 0, n_words = 0, P = 0;
    uint64_t n_edges = 0;
    bool has_push = false, has_pull = false;
    int sm_count = 148;

    // populations and parameters (host copies)
    std::vector<uint32_t> pop_ids, pop_off, excl_count;
    std::vector<RawParams> pop_raw;
    std::vector<RawParams> neuron_raw;  // only in per-neuron mode
    bool per_neuron = false;
    std::vector<uint8_t> ou_set;
    uint64_t gamma_calls = 0;

    // host mirror of the clock
    uint64_t steps = 0;
    float t = 0.0f;
    int noise_src = DTB_NOISE_PHILOX;
    uint64_t inj_rows = 0, inj_first = 0;

    // device memory
    std::vector<void*> allocs;
    uint64_t dev_bytes = 0;
    float* V = nullptr;
    float* iou = nullptr;
    float* tlast = nullptr;
    float4* J = nullptr;
    long long* dJ = nullptr;
    unsigned long long* dJf = nullptr;   // fixed-mode sums, allocated on first use
    uint32_t fix_shift = 0;              // fixed_shift_for() of the network (0: mode unavailable)
    PopParams* pop_dev = nullptr;
    PopParams* pop_sub_dev = nullptr;    // constants for substeps of dt / sub_ts (t_steps runs)
    float* np_sub_dev = nullptr;         // the same per neuron (per-neuron mode)
    uint32_t sub_ts = 0;                 // substeps the *_sub tables were derived for (0: none)
    uint32_t view_ts = 1;                // substeps the device view steps by (1 outside t_steps runs)
    uint64_t params_version = 0, sub_version = ~0ull;   // property changes since creation
    uint32_t* pop_off_dev = nullptr;
    float* np_dev = nullptr;
    unsigned long long* out_ptr = nullptr;
    uint32_t* out_col = nullptr;
    void* out_w = nullptr;
    unsigned long long* in_ptr = nullptr;
    uint32_t* in_col = nullptr;
    void* in_w = nullptr;
    uint32_t* out_deg = nullptr;
    uint32_t* bits0 = nullptr;
    uint32_t* bits1 = nullptr;
    uint32_t* excl = nullptr;
    Clock* clock = nullptr;
    unsigned long long* events = nullptr;
    uint32_t* ticket = nullptr;
    int* hist_cnt = nullptr;
    long long* hist_vsum = nullptr;
    long long* hist_isum = nullptr;      // [isum_cap * P * 5] synaptic-current sums (imean outputs)
    uint32_t isum_cap = 0;
    long long* h_isum = nullptr;
    uint32_t* rec_bits = nullptr;
    uint32_t hist_cap = 0, rec_cap = 0;
    uint32_t n_samples = 0, sample_cap = 0;
    uint32_t* sample_bits = nullptr;
    uint32_t* sample_pre = nullptr;
    uint8_t* hist_sspk = nullptr;
    float* hist_sv = nullptr;
    float* hist_siou = nullptr;
    float* hist_sisyn = nullptr;         // [isum_cap * sample_cap slots] sampled end-of-step I_syn
    uint32_t sisyn_cap = 0;
    std::vector<uint32_t> sample_order;   // sample slot -> position in the caller's list
    float* inj_z = nullptr;
    float* inj_u = nullptr;
    NetView* view_dev = nullptr;
    uint32_t* prefix_dev = nullptr;   // [lif 2][pull 2][vbase 2][local windows 2]
    uint32_t* list = nullptr;
    uint32_t* list_count = nullptr;
    uint32_t* list_ticket = nullptr;
    uint32_t* tile_pop = nullptr;
    uint32_t lif_ctas_per_sm = kLifCtasPerSm;
    // population-local push tables (built when every out-degree row is sorted)
    uint2* own_seg = nullptr;
    uint32_t* woff = nullptr;
    uint4* pop_loc = nullptr;
    uint4* win_tab = nullptr;
    uint32_t n_windows = 0;
    uint32_t* local_scratch = nullptr;   // [2 * n_windows + 3] per-step unit bookkeeping (zeroed)
    int build_local_tables();

    // push kernel variant (autotuned on the first active run)
    PushCfg push_cfg{PUSH_REG, 8, 32};
    uint32_t push_ctas = 0;
    bool autotune = true;
    bool push_tuned[3] = {false, false, false};
    TuneResult tune_acc[3];               // samples gathered so far (float, exact and fixed push)
    float tuned_ms = 0.0f;
    std::vector<TuneEntry> tune_report;
    int tune_push(const LaunchBatch& b, int acc);
    // Window graphs of the plain path: a chunk of push-mode steps is launched eagerly
    // the first two times its shape is seen in a row, captured into a CUDA graph the
    // third time and replayed from then on (one graph kept per engine) -- but only when
    // the eager chunk was launch-bound, under kGraphMaxMsPerStep of device time per
    // step.  Replay saves a few microseconds of launch work per step; capturing a
    // 500-step window costs about 70 ms, as much as 100 steps of the 5M-neuron network,
    // where replay gains about 1 %, so such networks stay eager.
    static constexpr float kGraphMaxMsPerStep = 0.2f;
    bool use_graph = true;
    cudaGraphExec_t graph = nullptr;
    uint64_t graph_key[10] = {};
    uint64_t seen_key[10] = {};
    uint32_t seen_count = 0;
    float seen_ms_per_step = 0.0f;        // device time per step of the last eager chunk of seen_key
    uint32_t graph_launches = 0;
    cudaEvent_t tune_ev[2] = {nullptr, nullptr};
    NetView view{};

    // pinned staging for the statistics
    int* h_cnt = nullptr;
    long long* h_vsum = nullptr;
    size_t h_cap = 0;

    template <class T> int dalloc(T*& p, size_t count, bool zero = true) {
        void* q = nullptr;
        const size_t bytes = count * sizeof(T) > 0 ? count * sizeof(T) : 16;
        DTB_CU(cudaMalloc(&q, bytes));
        allocs.push_back(q);
        dev_bytes += bytes;
        if (zero) DTB_CU(cudaMemsetAsync(q, 0, bytes, stream));
        p = static_cast<T*>(q);
        return DTB_OK;
    }
    void dfree(void* p);

private:
    int setup_populations_from_property(const float* prop);
    int upload_params();
    int init_state();
    int upload_csr_host(const uint32_t* pre, const uint32_t* post, const uint8_t* kind_in, const void* w, uint32_t in_type,
                        bool build_push, bool build_pull);
    int weight_bytes() const;
    int ensure_timing_events(size_t count);
    std::vector<cudaEvent_t> tev;
};

}  // namespace dtb
