/*
 * dtb_b200.h -- C-ABI of the B200 engine for the Digital Twin Brain per-timestep
 * hot path: LIF membrane update with four receptor conductances (AMPA, NMDA,
 * GABAa, GABAb), refractory clamp and Ornstein-Uhlenbeck background current;
 * spike detection and compaction; CSR spike propagation into per-receptor
 * accumulators.
 *
 * This library replaces the reference's block engine, the C++ class
 * dtb::BrainBlock<T,T2> (include/block.hpp:21-889) and its stage launchers
 * (include/stage.hpp:45-422), behind the service surface of protos/snn.proto.
 * Every entry point takes plain pointers and sizes; host buffers are copied in
 * or filled; device memory is owned by the engine.  Every call returns a
 * dtb_status (the snn.proto SnnStatus codes, extended with engine codes) and
 * never aborts the process: the reference kills its process on any internal
 * error (MPICHECK / HIP_CHECK, tools/dist_simulator.cpp:63-70,
 * include/common.hpp:83).
 *
 * Threading: calls on one engine must be serialised by the caller; distinct
 * engines may be used from different threads.  All engines of a process use
 * the CUDA device that was current when they were created.
 */
#ifndef DTB_B200_H
#define DTB_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DTB_ABI_VERSION 2

/* Status codes.  0-5 are snn.proto's SnnStatus (protos/snn.proto:44-51). */
typedef enum dtb_status {
    DTB_OK = 0,
    DTB_INVALID_PARAMETER = 1,
    DTB_UNSET_SAMPLE_FAILURE = 2,
    DTB_UNSUPPORTED = 3,
    DTB_NOT_ENABLE_METRIC = 4,
    DTB_INVALID_NETWORK = 5,
    DTB_OUT_OF_MEMORY = 16,   /* device or pinned-host allocation failed      */
    DTB_CUDA_ERROR = 17,      /* a CUDA call failed; see dtb_last_error()     */
    DTB_DEVICE_FAULT = 18,    /* a kernel reported an in-kernel check failure */
    DTB_IO_ERROR = 19,        /* file missing, short or malformed             */
    DTB_NO_DEVICE = 20
} dtb_status;

/* Synaptic weight storage (reference: DataType, include/weights.hpp:14-21,
 * chosen there by a directory-name substring, src/configuration.cpp:1411-1435). */
typedef enum dtb_weight_type {
    DTB_W_F32 = 0,
    DTB_W_BF16 = 1,   /* bf16 pair, accumulated in fp32 (no reference counterpart) */
    DTB_W_F16 = 2,    /* reference "half"                                          */
    DTB_W_U8 = 3,     /* reference "int8"/"uint8": value / 255                      */
    DTB_W_F64 = 4     /* reference "double": narrowed to fp32 on upload             */
} dtb_weight_type;

/* What drives the receptor accumulators each step. */
typedef enum dtb_prop_mode {
    DTB_PROP_THRESHOLD = 0, /* threshold spikes (models/block_new.py:147, debug_mode=False) */
    DTB_PROP_NOISE = 1,     /* noise train u < noise_rate replaces them (block_new.py:143-146) */
    DTB_PROP_OR = 2         /* noise OR threshold (src/stage/spike.cpp:42-68)                 */
} dtb_prop_mode;

/* How spikes reach the accumulators. */
typedef enum dtb_syn_mode {
    DTB_SYN_PUSH = 0,        /* out-degree CSR, fp32 vector reductions into J (fastest)       */
    DTB_SYN_PUSH_EXACT = 1,  /* out-degree CSR, 64-bit fixed-point atomics: deterministic     */
    DTB_SYN_PULL = 2,        /* in-degree CSR gather fused into the LIF step: deterministic   */
    DTB_SYN_PUSH_FIXED = 3   /* out-degree CSR, each step's input summed as two unsigned      */
                             /* 32-bit fixed-point fields packed in one 64-bit reduction per  */
                             /* synapse (units of 2^-fixed_shift, chosen at creation from the */
                             /* largest in-degree and weight so no field can carry): the float*/
                             /* push's kernels with integer reductions, deterministic (a run  */
                             /* gives the same bits alone, batched or served), bit-exact      */
                             /* against the oracle whenever every weight is a multiple of     */
                             /* 2^-fixed_shift.  Needs                                        */
                             /* non-negative weights (dtb_engine_info.fixed_shift != 0)       */
} dtb_syn_mode;

/* Source of the OU normal draws and the noise-train uniforms. */
typedef enum dtb_noise_source {
    DTB_NOISE_PHILOX = 0,    /* counter-based Philox4x32-10 keyed by (seed, step, neuron)     */
    DTB_NOISE_INJECTED = 1   /* host-supplied draws, e.g. a replay of the reference's stream  */
} dtb_noise_source;

/* Property ids: snn.proto PropType (protos/snn.proto:94-115). */
typedef enum dtb_prop_id {
    DTB_EXT_STIMULI_I = 0, DTB_MEMBRANE_C = 1, DTB_REF_T = 2, DTB_LEAKAGE_G = 3,
    DTB_LEAKAGE_V = 4, DTB_THRESHOLD_V = 5, DTB_RESET_V = 6,
    DTB_CONDUCT_G_AMPA = 7, DTB_CONDUCT_G_NMDA = 8, DTB_CONDUCT_G_GABAa = 9, DTB_CONDUCT_G_GABAb = 10,
    DTB_MEMBRANE_V_AMPA = 11, DTB_MEMBRANE_V_NMDA = 12, DTB_MEMBRANE_V_GABAa = 13, DTB_MEMBRANE_V_GABAb = 14,
    DTB_TAO_AMPA = 15, DTB_TAO_NMDA = 16, DTB_TAO_GABAa = 17, DTB_TAO_GABAb = 18,
    DTB_NOISE_RATE = 19,
    DTB_N_PROPS = 20
} dtb_prop_id;

/* Options fixed at creation. */
typedef struct dtb_options {
    float dt;                 /* ms; InitRequest.delta_t (snn.proto:27-37)                 */
    uint32_t weight_type;     /* dtb_weight_type of the device copy                        */
    uint64_t seed;            /* Philox key                                                */
    uint32_t build_push;      /* build the out-degree CSR (push modes)                     */
    uint32_t build_pull;      /* build the in-degree CSR (pull mode)                       */
    float ou_mean, ou_sigma, ou_tau; /* initial OU parameters of every population          */
    uint32_t reserved[8];
} dtb_options;

/* A block in the reference's npz key set (src/configuration.cpp:1094-1098,
 * 1508-1517, 1789).  Edges may come in any order; rows keep the input order
 * of each presynaptic neuron (the reference's stable sort,
 * src/configuration.cpp:227-249, 1079-1392). */
typedef struct dtb_network_arrays {
    uint32_t n_neurons;
    const float* property;            /* [n_neurons * 22] row-major float32          */
    uint64_t n_edges;
    const int16_t* input_block_idx;   /* [n_edges] relative block id, or NULL (all 0) */
    const uint32_t* input_neuron_idx; /* [n_edges] presynaptic neuron                */
    const uint32_t* output_neuron_idx;/* [n_edges] postsynaptic neuron               */
    const uint8_t* input_channel_offset; /* [n_edges] 0: AMPA/NMDA, nonzero: GABAa/GABAb */
    const void* weight;               /* [n_edges * 2] of weight_type                */
    uint32_t weight_type;             /* dtb_weight_type of `weight`                 */
} dtb_network_arrays;

/* A regional network generated on the device (counter-based, reproducible). */
typedef struct dtb_structured_spec {
    uint32_t n_pops;
    const uint32_t* pop_sizes;   /* [n_pops], contiguous populations in id order            */
    const uint32_t* pop_exc;     /* [n_pops], first pop_exc[b] neurons of b are excitatory    */
    const uint64_t* src_cdf;     /* [n_pops*n_pops], row a: source-population CDF x 2^32      */
    const float* pop_property;   /* [n_pops*22] property row of each population (column 3,
                                    the population id, is ignored)                            */
    uint32_t pop_id_base;        /* id of population 0                                       */
    uint32_t in_degree;          /* edges per postsynaptic neuron                            */
    uint64_t seed;               /* Philox key of the edge stream                            */
    uint32_t dyadic_weights;     /* weights quantised to multiples of 1/256                  */
} dtb_structured_spec;

typedef struct dtb_engine_info {
    uint32_t n_neurons;
    uint32_t n_pops;
    uint64_t n_edges;
    uint64_t device_bytes;       /* bytes held on the device                                 */
    uint64_t step;               /* steps simulated so far                                   */
    float t;                     /* simulated time, ms (float32, advanced by t += dt)        */
    uint32_t weight_type;
    uint32_t has_push, has_pull;
    uint32_t per_neuron_params;  /* 1 once any parameter differs within a population        */
    uint32_t push_kind;          /* push kernel in use: 0 register-staged, 1 TMA-staged rows,  */
                                 /* 2 population-local windows + register-staged remainder     */
    uint32_t push_param;         /* synapses in flight per lane (0, 2) or per stage (1)       */
    float push_tuned_ms;         /* push time of the chosen variant when it was tuned, ms     */
    uint32_t local_windows;      /* population-local push windows (0: variant 2 = variant 0)  */
    uint32_t fixed_shift;        /* DTB_SYN_PUSH_FIXED units 2^-fixed_shift (0: unavailable)   */
    uint32_t graph_launches;     /* window graphs replayed by dtb_run so far                   */
} dtb_engine_info;

/* RunRequest (snn.proto:63-77) flags. */
#define DTB_RUN_USE_OU        (1u << 0)  /* use_ou_background                                 */
#define DTB_RUN_FREQ          (1u << 1)  /* output_freq: per-population spike counts          */
#define DTB_RUN_VMEAN         (1u << 2)  /* output_vmean                                      */
#define DTB_RUN_RECORD_SPIKES (1u << 3)  /* copy every step's threshold-spike bitmap out      */
#define DTB_RUN_TIME_KERNELS  (1u << 4)  /* time every kernel launch with CUDA events          */
#define DTB_RUN_SAMPLE_SPIKE  (1u << 5)  /* output_sample_spike: spikes of the sampled neurons */
#define DTB_RUN_SAMPLE_V      (1u << 6)  /* output_sample_vmemb                                 */
#define DTB_RUN_SAMPLE_IOU    (1u << 7)  /* output_sample_iou (needs DTB_RUN_USE_OU)            */
#define DTB_RUN_IMEAN         (1u << 8)  /* output_imean: per-population mean I_syn (push modes) */
#define DTB_RUN_RECEPTOR_IMEAN (1u << 9) /* output_receptor_imeas: mean I_u per receptor        */
#define DTB_RUN_SAMPLE_ISYN   (1u << 10) /* output_sample_isynaptic: end-of-step I_syn (push)   */

typedef struct dtb_run_request {
    uint32_t iters;      /* RunRequest.iter; > 0                                                */
    uint32_t flags;      /* DTB_RUN_*                                                            */
    uint32_t prop_mode;  /* dtb_prop_mode                                                        */
    uint32_t syn_mode;   /* dtb_syn_mode                                                         */
    uint32_t t_steps;    /* RunRequest.t_steps: substeps per step (0 or 1: none; at most 255).
                            Each step then runs t_steps substeps of dt / t_steps -- OU, membrane
                            update and threshold, receptor decay with no input between them --
                            spikes OR-ed over the substeps and propagated once after the last
                            (tools/dist_simulator.cpp:2085-2112, src/block.cpp:729-737, 875-888);
                            outputs stay per step: counts are of neurons that spiked in any
                            substep, V means and samples are taken after the last substep.
                            Needs DTB_RUN_USE_OU, threshold propagation and a push mode, as the
                            reference's Run validation requires OU (dist_simulator.cpp:3225-3234) */
    uint32_t reserved[3];
} dtb_run_request;

typedef struct dtb_run_output {
    int32_t* freqs;         /* [iters * n_pops] spike counts (freq_char is derived on the host) */
    float* vmeans;          /* [iters * n_pops]                                                 */
    uint32_t* spike_bits;   /* [iters * ceil(n_neurons/32)] threshold spikes, bit i = neuron i  */
    uint64_t events;        /* out: synaptic events delivered (sum over steps of out-degrees of
                               the propagated spikes)                                          */
    double device_ms;       /* out: device time of the run, CUDA events on the engine stream    */
    double kernel_ms[4];    /* out, with DTB_RUN_TIME_KERNELS: summed device time of the LIF,
                               push, pull and end-of-run kernels                               */
    uint32_t launches;      /* out: kernels launched by this run                               */
    uint32_t reserved;
    uint8_t* sample_spike;  /* [iters * n_samples] in the order given to dtb_set_samples          */
    float* sample_v;        /* [iters * n_samples]                                               */
    float* sample_iou;      /* [iters * n_samples]                                               */
    float* imeans;          /* [iters * n_pops] mean I_syn at the end of each step (DTB_RUN_IMEAN)  */
    float* receptor_imeans; /* [iters * 4 * n_pops] mean I_AMPA, I_NMDA, I_GABAa, I_GABAb per step,
                               receptor-major within a step (DTB_RUN_RECEPTOR_IMEAN)            */
    float* sample_isyn;     /* [iters * n_samples] end-of-step I_syn of the sampled neurons        */
} dtb_run_output;

/* --- version and errors ------------------------------------------------- */
int32_t dtb_abi_version(void);
/* GetVersion (snn.proto:6): major*1000 + minor*100 + patch (include/version.hpp:3-5). */
int32_t dtb_engine_version(void);
const char* dtb_status_string(int32_t status);
/* Message of the last failure on the calling thread (empty if none). */
const char* dtb_last_error(void);

/* --- lifetime ----------------------------------------------------------- */
/* Replaces BrainBlock construction + init_connection_table_gpu +
 * init_config_params_gpu + init_all_stages_gpu (src/block.cpp:19-179). */
void dtb_default_options(dtb_options* opt);
int32_t dtb_create(const dtb_network_arrays* net, const dtb_options* opt, void** engine);
/* Generate a regional network on the device (no reference counterpart: the
 * reference reads networks from npz files written by python/make_block.py). */
int32_t dtb_create_structured(const dtb_structured_spec* spec, const dtb_options* opt, void** engine);
/* InitRequest path: load block_<i>.npz (src/configuration.cpp:1394, 1778). */
int32_t dtb_create_from_npz(const char* path, const dtb_options* opt, void** engine);
int32_t dtb_destroy(void* engine);
int32_t dtb_info(void* engine, dtb_engine_info* info);
/* Push kernel variant: kind 0 (register-staged, param 4/8/16 synapses in flight
 * per lane, or 1000 + lanes per row 16/8 for sub-warp rows), 1 (TMA bulk-copy
 * staged rows, param 256/512 synapses per stage) or 2 (population-local: each
 * row's own-population synapses are summed per window of its population in
 * shared memory, the rest as kind 0; param 8 or 1016, or 2008 / 2016 / 3008 for
 * the forms that run the rest on a second stream beside the window kernel; float
 * push mode only, the exact mode runs kind 0 instead);
 * kind < 0 re-enables the autotuner.  From step 300 it reads the spike count of
 * every step for 50 steps, then times every variant on the live spike lists of
 * four steps with at least half the peak count seen (and 0.2 % of the neurons),
 * 47 or more steps apart, and keeps the variant with the smallest mean; it gives
 * up (keeping the best so far, or kind 0 param 8) after 400 reads of quiet steps. */
int32_t dtb_set_push_variant(void* engine, int32_t kind, int32_t param);
/* Window graphs of dtb_run (no reference counterpart): with enable != 0 (the
 * default) a chunk of push-mode steps is launched kernel by kernel the first two
 * times its shape (steps, flags, modes, push variant) is seen in a row, captured
 * into a CUDA graph the third time and replayed from then on -- when the eager
 * chunk took under 0.2 ms of device time per step (launch-bound networks; larger
 * ones stay eager, where a capture would cost more than replay saves).  Results
 * are the same bits either way.  enable = 0 launches every chunk kernel by kernel. */
int32_t dtb_set_graph(void* engine, int32_t enable);
/* The autotuner's last measurement: on entry *n is the capacity of the arrays,
 * on return the number of variants timed (kind, param, push time in ms). */
int32_t dtb_tuning_report(void* engine, uint32_t* n, int32_t* kinds, int32_t* params, float* ms);
/* The CUDA stream (cudaStream_t) every kernel and copy of this engine runs on,
 * so a caller can order its own work and CUDA events against the engine. */
int32_t dtb_get_stream(void* engine, void** stream);

/* InitResponse.subblk_info (snn.proto:39-61): population ids and sizes. */
int32_t dtb_populations(void* engine, uint32_t* ids, uint32_t* counts);

/* --- property surface (snn.proto Update* RPCs) ------------------------------- */
/* Updateprop: per-neuron set (src/stage/property.cpp:57-160). */
int32_t dtb_update_props(void* engine, uint32_t n, const uint32_t* neuron_ids,
                         const uint32_t* prop_ids, const float* values);
/* Updatehyperpara: per-population multiply (assign=0) or assign (assign=1)
 * (src/stage/property.cpp:185-438). Unknown population ids are ignored. */
int32_t dtb_update_prop_cols(void* engine, uint32_t n, const uint32_t* prop_ids,
                             const uint32_t* pop_ids, const float* values, int32_t assign);
/* Updategamma: per-neuron value = Gamma(alpha, 1) / beta within each listed
 * population (src/stage/property.cpp:494-651). */
int32_t dtb_update_gamma(void* engine, uint32_t n, const uint32_t* prop_ids,
                         const uint32_t* pop_ids, const float* alpha, const float* beta);
/* The current value of one property (dtb_prop_id) for every neuron [n_neurons], as
 * creation and the Update* calls left it (REF_T in ms).  No reference counterpart:
 * the reference keeps the properties on the device and offers no read. */
int32_t dtb_read_property(void* engine, uint32_t prop_id, float* values);
/* Updateoubackgroundparam: per-population OU mean, sigma, tau
 * (src/block.cpp:222-281). A population's OU current is reset to its mean the
 * first time it is configured, as the reference does. */
int32_t dtb_set_ou(void* engine, uint32_t n, const uint32_t* pop_ids, const float* mean,
                   const float* sigma, const float* tau);

/* Updatesample (tools/dist_simulator.cpp:3635; stat_samples_kernel,
 * src/stage/stat_result.cpp:393-431): neurons whose spike, membrane potential
 * and OU current each step reports through the DTB_RUN_SAMPLE_* outputs.
 * Requesting sample outputs with no samples set returns DTB_UNSET_SAMPLE_FAILURE,
 * as the reference's Run validation does (dist_simulator.cpp:3225-3234). */
int32_t dtb_set_samples(void* engine, uint32_t n, const uint32_t* neuron_ids);

/* Noise source for subsequent steps.  DTB_NOISE_INJECTED takes `steps` rows of
 * n_neurons normal draws `z` and (optionally) uniforms `u`, consumed one row per
 * step from the next step on. */
int32_t dtb_set_noise(void* engine, uint32_t source, uint32_t steps, const float* z, const float* u);

/* --- stepping ------------------------------------------------------------ */
/* Run: the per-iteration loop of tools/dist_simulator.cpp:2072-2315 with
 * in-HBM spike delivery; outputs land in caller-owned host buffers. */
int32_t dtb_run(void* engine, const dtb_run_request* req, dtb_run_output* out);

/* --- batched form ---------------------------------------------------------- */
/* A batch advances several engines (ensemble members, served requests) with one
 * launch of each per-step kernel; a window of float-push steps is captured once
 * into a CUDA graph and replayed.  No reference counterpart as an API: the
 * reference packs an ensemble into one network (data_assimilation/DA_voxel.py:47-52).
 * Members keep their own state, clock, noise stream and outputs; they must share
 * the weight type, the device and the noise source.  The engines must outlive the
 * batch; they stay usable on their own between batch runs. */
int32_t dtb_batch_create(void* const* engines, uint32_t n, void** batch);
int32_t dtb_batch_destroy(void* batch);
/* Run every member `req->iters` steps; outs[i] receives member i's outputs. */
int32_t dtb_batch_run(void* batch, const dtb_run_request* req, dtb_run_output* outs);
/* enable != 0: capture float-push windows into a CUDA graph (default). */
int32_t dtb_batch_set_graph(void* batch, int32_t enable);
/* The batch's push variant, as dtb_set_push_variant (kind < 0: autotune). */
int32_t dtb_batch_set_push_variant(void* batch, int32_t kind, int32_t param);
int32_t dtb_batch_info(void* batch, uint32_t* n_members, uint32_t* graph_launches, int32_t* push_kind,
                       int32_t* push_param);

/* --- serving form -----------------------------------------------------------
 * No reference counterpart: the reference serves one network per process group,
 * one Run RPC at a time (dist_simulator.cpp:3217-3451).  A server holds a pool of
 * networks under an HBM cap and replays a trace of simulate-window requests in
 * real time, either with continuous batching or one request at a time. */
#define DTB_SERVE_BATCHED    0u  /* continuous batching over slices of slice_steps  */
#define DTB_SERVE_SEQUENTIAL 1u  /* arrival order, one request at a time (dtb_run)   */

typedef struct dtb_server_options {
    uint64_t hbm_cap_bytes;  /* device memory of resident networks; idle ones beyond it are evicted to host */
    uint32_t slice_steps;    /* steps per continuous-batching slice                               */
    uint32_t max_batch;      /* most requests in flight together                                  */
    uint32_t syn_mode;       /* DTB_SYN_* of every run                                            */
    uint32_t flags;          /* DTB_RUN_USE_OU etc.; DTB_RUN_FREQ is always on                    */
    uint32_t autotune;       /* 1: each engine and the batch autotune their push variant (the batch
                                once per size class of its membership, on two busy steps)       */
    uint32_t reserved[3];
} dtb_server_options;

/* One request: Updateoubackgroundparam (optional) followed by Run(iter=iters)
 * on one network, with RunResponse.freq of every step as the output. */
typedef struct dtb_request {
    uint32_t net;            /* id from dtb_server_add_*                                     */
    uint32_t iters;          /* steps to simulate                                            */
    double arrival_s;        /* seconds after the replay starts; non-decreasing over a trace */
    const float* ou_mean;    /* [P] per population, or NULL to keep the current parameters   */
    const float* ou_sigma;   /* [P]                                                          */
    const float* ou_tau;     /* [P]                                                          */
    int32_t* freqs;          /* [iters * P] per-step population spike counts, or NULL        */
    double start_s;          /* out: first step issued (seconds after the replay starts)     */
    double finish_s;         /* out: last step finished                                      */
    uint64_t events;         /* out: synaptic events delivered                               */
    int32_t status;          /* out: DTB_OK once served                                      */
    uint32_t reserved;
} dtb_request;

typedef struct dtb_server_stats {
    uint32_t n_nets;
    uint32_t resident;           /* networks in HBM                         */
    uint64_t resident_bytes;
    uint64_t evictions;          /* networks moved to the host              */
    uint64_t restores;           /* networks rebuilt from the host          */
    uint64_t slices;             /* batched slices (or runs, sequentially)  */
    uint64_t batch_members_sum;  /* sum over slices of requests in flight   */
} dtb_server_stats;

void dtb_server_default_options(dtb_server_options* opt);
int32_t dtb_server_create(const dtb_server_options* opt, void** server);
int32_t dtb_server_destroy(void* server);
/* Add a network (built resident; idle networks are evicted if the cap requires). */
int32_t dtb_server_add_structured(void* server, const dtb_structured_spec* spec, const dtb_options* opt,
                                  uint32_t* net_id);
int32_t dtb_server_add_npz(void* server, const char* path, const dtb_options* opt, uint32_t* net_id);
/* Serve the n requests (sorted by arrival) under `policy`; fills their outputs. */
int32_t dtb_server_play(void* server, uint32_t n, dtb_request* reqs, uint32_t policy);
int32_t dtb_server_info(void* server, dtb_server_stats* info);

/* Online serving: requests that are not known in advance, the gRPC Run path.
 * dtb_server_start starts a scheduler thread on the calling thread's device with
 * `policy`: DTB_SERVE_BATCHED admits submitted requests in arrival order as slots
 * (max_batch) and device memory free up, between slices of slice_steps steps of the
 * requests already in flight, which advance together; DTB_SERVE_SEQUENTIAL runs
 * one request at a time.  A network is admitted while the resident networks stay
 * within hbm_cap_bytes and the device has its bytes free (cudaMemGetInfo, plus
 * 1 GiB for a rebuild); idle networks are evicted to the host otherwise.
 * dtb_server_submit may be called from any thread: it copies the OU arrays, stamps
 * arrival_s (seconds since start) and returns a ticket; `req` and its freqs buffer
 * stay the caller's and must remain valid until the request is reported done.
 * dtb_server_poll waits up to wait_ms for the ticket; *done = 1 once start_s,
 * finish_s, events, freqs and status are filled in (the ticket is then retired).
 * dtb_server_stop finishes every submitted request, then ends the thread; networks
 * are added only while the scheduler is stopped, and dtb_server_play is refused
 * while it runs.  A scheduler failure ends it: every unfinished request carries
 * the status, and polls return it. */
int32_t dtb_server_start(void* server, uint32_t policy);
int32_t dtb_server_submit(void* server, dtb_request* req, uint64_t* ticket);
int32_t dtb_server_poll(void* server, uint64_t ticket, uint32_t wait_ms, int32_t* done);
int32_t dtb_server_stop(void* server);

/* --- BOLD signal (data assimilation) ----------------------------------------
 * models/bold_model_pytorch.py:61-96, driven per simulated step by
 * data_assimilation/DA_voxel.py:314-331.  Parameters are doubles, as the
 * reference's Python floats are. */
typedef struct dtb_bold_params {
    double epsilon, tao_s, tao_f, tao_0, alpha, E_0, V_0;
    double delta_t;          /* s per step (BOLD.__init__ default 1e-3) */
} dtb_bold_params;
void dtb_bold_default_params(dtb_bold_params* p);   /* DA_voxel.py:470-476 */
/* Advance n voxels by `steps` steps of BOLD.run: u [steps * n] voxel activity,
 * state [4 * n] = s, q, v, f_in (in/out; BOLD.run starts from 0, 0, 1, 1),
 * out [steps * n] the BOLD signal of every step or NULL.  Device pointers,
 * enqueued on `stream` (NULL: the default stream). */
int32_t dtb_bold_run(const dtb_bold_params* p, uint32_t n, uint32_t steps, const float* u, float* state,
                     float* out, void* stream);

/* Ensemble Kalman update DA_voxel.filter (data_assimilation/DA_voxel.py:289-307):
 * w_hat [E * V * S] float32 (member-major, then voxel, then state; S = hp_num + 6,
 * the BOLD signal last), bold_y [V] the observed BOLD, noise [E * V] the
 * standard-normal draws the reference takes from torch.normal (scaled by
 * sqrt(bold_sigma) inside), rate as in filter(); w_out [E * V * S].  Device
 * pointers on `stream`; accumulation in double, one rounding to float32. */
int32_t dtb_da_filter(uint32_t ensembles, uint32_t voxels, uint32_t states, const float* w_hat, const float* bold_y,
                      const float* noise, double bold_sigma, double rate, float* w_out, void* stream);

/* --- state access (tests, checkpoint, serving eviction) ------------------ */
#define DTB_STATE_V      0  /* float [n]                                       */
#define DTB_STATE_J      1  /* float [n*4] (AMPA, NMDA, GABAa, GABAb per neuron) */
#define DTB_STATE_I_OU   2  /* float [n]                                       */
#define DTB_STATE_T_LAST 3  /* float [n] time of the last threshold spike      */
int32_t dtb_read_state(void* engine, int32_t which, void* host_dst);
int32_t dtb_write_state(void* engine, int32_t which, const void* host_src);

/* The out-degree CSR as the reference's builder lays it out
 * (src/configuration.cpp:1079-1392): rows are presynaptic neurons with at least
 * one synapse, in ascending order (`rows`), row_ptr over them, and per synapse
 * the postsynaptic neuron, the receptor pair (0 or 1) and the weight pair as
 * float32.  Pass NULL for arrays not wanted; *n_rows / *n_edges are always set. */
int32_t dtb_read_out_csr(void* engine, uint32_t* n_rows, uint64_t* n_edges, uint32_t* rows,
                         uint64_t* row_ptr, uint32_t* post, uint8_t* kind, float* weight);

/* The same out-degree CSR built on the host from edge arrays, with no device
 * involved (src/configuration.cpp:1079-1392 semantics: a stable sort of the
 * synapses by presynaptic neuron).  Outputs: *n_rows, rows [n_neurons],
 * row_ptr [n_neurons + 1] (first *n_rows + 1 used), post_out, kind_out (0/1)
 * and perm (input index of each CSR slot), each [n_edges]. */
int32_t dtb_build_out_csr_host(uint32_t n_neurons, uint64_t n_edges, const uint32_t* pre, const uint32_t* post,
                               const uint8_t* kind, uint32_t* n_rows, uint32_t* rows, uint64_t* row_ptr,
                               uint32_t* post_out, uint8_t* kind_out, uint64_t* perm);

/* Spike compaction (the sending-side compaction of src/stage/spike.cpp:244-762
 * as one operator): turns the device spike bitmap `d_bits` (bit i of word i/32
 * is neuron i; ceil(n/32) words) into the ascending list of spiking neurons
 * `d_indices` (room for n entries) and its length `*d_count`, all in device
 * memory, ordered on `stream` (a cudaStream_t, NULL = default stream).
 * Deterministic.  Scratch: one word per 4096 neurons, allocated and released
 * on `stream` by each call.  n_neurons <= 4,294,963,200 (the last 4096-neuron
 * tile boundary below 2^32); larger values return DTB_INVALID_PARAMETER before
 * anything runs. */
int32_t dtb_compact_spikes(const uint32_t* d_bits, uint32_t n_neurons, uint32_t* d_indices, uint32_t* d_count,
                           void* stream);

/* The same compaction for callers that cannot allocate device memory at the point
 * of the call: a serving or data-assimilation loop whose device-memory budget is
 * fixed when it starts (so that its admission decisions stay valid), or a runtime
 * that embeds the engine, owns all device memory through its own pool and forbids
 * libraries to allocate.  No counterpart in the reference.  It allocates
 * nothing: its scratch is a fixed 64 KiB array inside the library, so
 * n_neurons <= 2^26 (larger inputs return DTB_INVALID_PARAMETER before anything
 * runs).  All calls share that array, which keeps the last call's counts (each is
 * written before it is read, so nothing needs clearing): calls whose kernels
 * overlap on the GPU race and must be ordered.  The first call on each device
 * looks the array's address up (with that device current) and keeps it for the
 * life of the process; make that first call before any stream capture.  The kept
 * address assumes the device's primary context is never reset: after a
 * cudaDeviceReset the library must not be called again in that process. */
int32_t dtb_compact_spikes_noalloc(const uint32_t* d_bits, uint32_t n_neurons, uint32_t* d_indices,
                                   uint32_t* d_count, void* stream);

/* Serving eviction: the whole dynamic state (V, J, I_ou, t_last, clock and the
 * last step's spikes) as one blob.  dtb_state_size gives its size. */
int32_t dtb_state_size(void* engine, uint64_t* bytes);
int32_t dtb_save_state(void* engine, void* host_blob, uint64_t bytes);
int32_t dtb_load_state(void* engine, const void* host_blob, uint64_t bytes);

#ifdef __cplusplus
}
#endif

#endif /* DTB_B200_H */
