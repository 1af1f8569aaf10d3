// Device-side data layout and arithmetic shared by every kernel of the engine.
//
// Layout in HBM of one network (all arrays padded to n_pad = round_up(n, 1024)):
//   V[n_pad], i_ou[n_pad], t_last[n_pad]         float32 SoA, read with 128-bit loads
//   J[n_pad]                                      float4 (AMPA, NMDA, GABAa, GABAb)
//   dJ[n_pad*4]                                   int64 fixed point (scale 2^32), exact mode only
//   dJf[n_pad*2]                                  two u32 fixed-point sums (scale 2^s) per u64, fixed mode only
//   bits[2][n_words]                              propagated spikes, double-buffered by step parity
//   out_ptr[n+1] u64, out_col[S] u32, out_w[S]    out-degree CSR (push); col = post | kind << 31
//   in_ptr[n+1]  u64, in_col[S]  u32, in_w[S]     in-degree CSR (pull);  col = pre  | kind << 31
//   out_deg[n] u32                                out-degree per neuron (event accounting)
//   pop[P] PopParams, pop_off[P+1]               per-population derived constants
// The receptor pair of a synapse is chosen by its kind bit: 0 -> (AMPA, NMDA) = J.xy,
// 1 -> (GABAa, GABAb) = J.zw, as the reference's 1-bit connkind does
// (src/stage/presynaptic_voltage.cpp:150, 178-187).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace dtb {

constexpr int kLifThreads = 256;
constexpr int kLifTile = 1024;          // neurons per LIF CTA: 256 threads x 4 neurons
// Depth of the LIF kernel's bulk-copy ring (tiles in flight = stages - 1) and the CTAs
// that fit on an SM with it (28 KiB of shared memory per stage).
#ifndef DTB_LIF_STAGES
#define DTB_LIF_STAGES 2
#endif
constexpr int kLifStages = DTB_LIF_STAGES;
constexpr int kLifCtasPerSm = kLifStages <= 2 ? 3 : (kLifStages == 3 ? 2 : 1);
constexpr int kPullThreads = 256;
constexpr int kPullTile = 256;          // neurons per pull CTA: 8 warps x 32 neurons
constexpr int kPad = 1024;              // every per-neuron array is padded to a multiple of this
constexpr uint32_t kLocalWin = 13312;   // neurons per local-push window: 4 receptor planes of 32-bit sums, 208 KiB
constexpr uint32_t kKindBit = 0x80000000u;
constexpr uint32_t kIndexMask = 0x7fffffffu;
constexpr float kFixScale = 4294967296.0f;          // 2^32: fixed-point unit of dJ
constexpr float kFixInv = 2.3283064365386963e-10f;  // 2^-32
constexpr double kVsumScale = 16777216.0;           // 2^24: fixed-point unit of the V sums

// Philox streams (third counter word).
constexpr uint32_t kStreamOU = 0x0D0E0001u;
constexpr uint32_t kStreamNoise = 0x0D0E0002u;
constexpr uint32_t kStreamEdges = 0x5EED0001u;
constexpr uint32_t kStreamGamma = 0x0D0E0003u;

// Error bits a kernel may raise in Clock::err (read back by the host after a run).
constexpr uint32_t kErrHistOverflow = 1u;
constexpr uint32_t kErrNoiseExhausted = 2u;
constexpr uint32_t kErrIndex = 4u;
constexpr uint32_t kErrTimeout = 8u;      // a bounded wait gave up

// J_DIRECT: J complete on entry, J*decay written back, the float push adds into J;
// J_FOLD: J + exact 64-bit sums (dJ) folded on entry; J_ASIS: J complete, unchanged;
// J_FIXF: J + packed 32-bit fixed-point sums (dJf) folded on entry.
enum JMode : int { J_DIRECT = 0, J_FOLD = 1, J_ASIS = 2, J_FIXF = 3 };
// Accumulator of a push launch: float reductions into J, exact 64-bit sums into dJ,
// or packed 32-bit fixed-point sums into dJf.
enum AccMode : int { ACC_FLOAT = 0, ACC_EXACT = 1, ACC_FIXED = 2 };
enum WType : int { W_F32 = 0, W_BF16 = 1, W_F16 = 2, W_U8 = 3 };
enum PropMode : int { PROP_THRESHOLD = 0, PROP_NOISE = 1, PROP_OR = 2 };

// Run flags seen by the kernels.
constexpr uint32_t kFlagUseOU = 1u;
constexpr uint32_t kFlagStats = 2u;
constexpr uint32_t kFlagRecord = 4u;
constexpr uint32_t kFlagList = 8u;       // write the spike list for the push kernel
constexpr uint32_t kFlagInjected = 16u;
constexpr uint32_t kFlagSample = 32u;     // record the sampled neurons
constexpr uint32_t kFlagIsyn = 64u;       // synaptic-current statistics after the push (host-side marker)
// Substeps (RunRequest.t_steps > 1, tools/dist_simulator.cpp:2085-2112): a LIF launch
// may be substep `k` of `ts` of one step; both ride in the flags word.  The device
// clock's step count advances after the last substep only, its time after every one.
constexpr uint32_t kSubShift = 16u;       // bits 16-23: substep index k
constexpr uint32_t kTsShift = 24u;        // bits 24-31: substeps per step (0 = 1)
__host__ __device__ inline uint32_t substep_flags(uint32_t k, uint32_t ts) { return (k << kSubShift) | (ts << kTsShift); }

// Derived per-population constants (host computes them once per property change).
struct __align__(16) PopParams {
    float dtC;        // fl(fl(1/C) * dt): block_new.py:109 evaluates dt / C as reciprocal(C) * dt
    float neg_gL;     // -g_L
    float V_L, V_th, V_reset, T_ref, I_ext, noise_rate;
    float g[4], Vu[4], decay[4];   // decay = fl(exp(fl(reciprocal(tau) * -dt)))
    float ou_mean, ou_f1, ou_f2s;  // f1 = 1 - exp(-dt/tau_i); f2s = fl(sqrt(1 - exp(-2dt/tau_i)) * sigma)
    float pad;
};
static_assert(sizeof(PopParams) == 96, "PopParams layout");
constexpr int kParamFloats = 24;

struct Clock {
    float t;                       // simulated time after step n (float32, t += dt)
    uint32_t err;                  // error bits raised by kernels
    unsigned long long n;          // steps done
    unsigned long long run_base;   // n at the start of the current run (history row 0)
    unsigned long long inj_base;   // n before the first injected-noise row
};

// Device-visible description of one network.  A launch covers a batch of these.
struct NetView {
    uint32_t n, n_pad, n_words, n_pops;
    float dt;
    uint32_t per_neuron;           // 1: parameters from np_params SoA, else from pop[]
    uint32_t weight_type;
    uint32_t hist_cap;
    float* V;
    float* iou;
    float* tlast;
    float4* J;
    long long* dJ;                 // [n_pad * 4], exact mode
    const PopParams* pop;
    const uint32_t* pop_off;       // [n_pops + 1]
    const float* np_params;        // [kParamFloats][n_pad] SoA of PopParams fields
    const unsigned long long* out_ptr;
    const uint32_t* out_col;
    const void* out_w;
    const uint32_t* out_deg;
    const unsigned long long* in_ptr;
    const uint32_t* in_col;
    const void* in_w;
    uint32_t* bits0;
    uint32_t* bits1;
    uint32_t* rec_bits;            // [hist_cap * n_words] threshold spikes per step
    const uint32_t* stat_excl;     // bitmap of neurons excluded from statistics, or null
    Clock* clock;
    unsigned long long seed;
    const float* inj_z;            // [inj_rows * n_pad]
    const float* inj_u;
    unsigned long long inj_rows;
    int* hist_cnt;                 // [hist_cap * n_pops]
    long long* hist_vsum;          // [hist_cap * n_pops] fixed point, scale 2^24
    long long* hist_isum;          // [isum_cap * n_pops * 5] I_syn, I_AMPA, I_NMDA, I_GABAa, I_GABAb sums, scale 2^24
    uint32_t isum_cap;
    unsigned long long* events;    // cumulative synaptic events
    uint32_t* ticket;              // last-tile counter of the per-step kernels
    const uint32_t* tile_pop;      // [lif_tiles] population of each LIF tile's first neuron
    uint32_t lif_tiles;
    uint32_t n_samples;            // sampled neurons (set_samples)
    const uint32_t* sample_bits;   // [n_words] bitmap of sampled neurons
    const uint32_t* sample_pre;    // [n_words] samples in the words before each word
    uint8_t* hist_sspk;            // [hist_cap * n_samples] spike of each sampled neuron
    float* hist_sv;                // [hist_cap * n_samples] V after the step
    float* hist_siou;              // [hist_cap * n_samples] OU current after the step
    float* hist_sisyn;             // [isum_cap * n_samples] I_syn at the end of the step
    // Population-local push (rows sorted by postsynaptic neuron).  A population
    // with local windows is cut into pop_loc[a].x windows of pop_loc[a].y neurons;
    // row j keeps, for each boundary k of its own population's windows, the offset
    // inside the row of the first synapse at or past that boundary.
    const uint2* own_seg;          // [n] own-population synapses of row j: [beg + x, beg + y); {0,0} = none local
    const uint32_t* woff;          // row j of population a: woff[rb(a) + (j - pop_off[a]) * (k_a + 1) + k]
    const uint4* pop_loc;          // [n_pops] {k_a, window width, rb(a) low word, rb(a) high word}
    const uint4* win_tab;          // [n_windows] {population, first neuron, end neuron, window index | s << 16}
    uint32_t n_windows;
    // Fixed-point push (DTB_SYN_PUSH_FIXED): one step's input to neuron i as two
    // pairs of unsigned 32-bit sums in units of 2^-fix_shift, receptor pair k in
    // dJf[2 i + k] = (sum of w.y) << 32 | (sum of w.x).  fix_shift is chosen at
    // creation so no field can carry (every weight >= 0, in-degree x max w x
    // 2^fix_shift < 2^32); 0 when the network does not allow the mode.
    unsigned long long* dJf;       // [n_pad * 2]
    uint32_t fix_shift;
    float fix_scale, fix_unscale;  // 2^fix_shift, 2^-fix_shift
};

// Batch-wide spike list written by the LIF kernel and consumed by the push kernel.
struct SpikeList {
    uint32_t* list;                // virtual neuron ids: vbase[net] + neuron
    uint32_t* count;
    uint32_t* ticket;              // last-CTA counter of the push kernel
    uint32_t capacity;
};

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11): a 10-round counter-based generator.  Each round maps the
// counter through two 32x32->64 multiplications by the published multipliers
// and XORs in the key, which is bumped by the published Weyl constants.
// ---------------------------------------------------------------------------
struct U4 { uint32_t x, y, z, w; };

__host__ __device__ inline void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
    const uint64_t p = static_cast<uint64_t>(a) * static_cast<uint64_t>(b);
    hi = static_cast<uint32_t>(p >> 32);
    lo = static_cast<uint32_t>(p);
}

__host__ __device__ inline U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(M0, c.x, hi0, lo0);
        mulhilo32(M1, c.z, hi1, lo1);
        U4 o;
        o.x = hi1 ^ c.y ^ k0;
        o.y = lo1;
        o.z = hi0 ^ c.w ^ k1;
        o.w = lo0;
        c = o;
        k0 += W0;
        k1 += W1;
    }
    return c;
}

__host__ __device__ inline uint32_t mulhi_u32(uint32_t r, uint32_t m) {
    return static_cast<uint32_t>((static_cast<uint64_t>(r) * m) >> 32);
}

__device__ inline float u01_open(uint32_t r) {     // (0, 1]
    return (static_cast<float>(r >> 8) + 1.0f) * (1.0f / 16777216.0f);
}
__device__ inline float u01(uint32_t r) {          // [0, 1)
    return static_cast<float>(r >> 8) * (1.0f / 16777216.0f);
}

// Box-Muller: two independent N(0,1) draws from two uniforms, on the SFU's
// approximate log2 / rsqrt / sin / cos (the Philox draws are held to statistical
// bars, never to bits; measured 2 % faster LIF than the IEEE-rounded functions).
__device__ inline void box_muller(uint32_t a, uint32_t b, float& z0, float& z1) {
    const float x = -2.0f * __logf(u01_open(a));
    const float rad = x > 0.0f ? x * rsqrtf(x) : 0.0f;
    float s, c;
    __sincosf(6.28318530717958647692f * u01(b), &s, &c);
    z0 = rad * c;
    z1 = rad * s;
}

// ---------------------------------------------------------------------------
// Weight decoding: every device weight type is widened to a float2 pair.
// ---------------------------------------------------------------------------
template <int WT> struct WeightT;
template <> struct WeightT<W_F32> { using T = float2; };
template <> struct WeightT<W_BF16> { using T = __nv_bfloat162; };
template <> struct WeightT<W_F16> { using T = __half2; };
template <> struct WeightT<W_U8> { using T = uchar2; };

template <int WT>
__device__ inline float2 load_weight(const void* base, unsigned long long e) {
    using T = typename WeightT<WT>::T;
    const T* p = reinterpret_cast<const T*>(base) + e;
    if constexpr (WT == W_F32) {
        return __ldcs(p);
    } else if constexpr (WT == W_BF16) {
        const unsigned int raw = __ldcs(reinterpret_cast<const unsigned int*>(p));
        __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(&raw);
        return __bfloat1622float2(v);
    } else if constexpr (WT == W_F16) {
        const unsigned int raw = __ldcs(reinterpret_cast<const unsigned int*>(p));
        __half2 v = *reinterpret_cast<const __half2*>(&raw);
        return __half22float2(v);
    } else {
        const unsigned short raw = __ldcs(reinterpret_cast<const unsigned short*>(p));
        // the reference's uint8 weights are value / 255 (presynaptic_voltage.cpp:169-174)
        return make_float2(static_cast<float>(raw & 0xFFu) / 255.f, static_cast<float>(raw >> 8) / 255.f);
    }
}

// ---------------------------------------------------------------------------
// The per-neuron LIF step, in block_new's float32 op order (models/block_new.py).
// Every operation is an explicitly rounded intrinsic so nothing is contracted
// into an FMA: the result is bit-identical to the CPU oracle.
// ---------------------------------------------------------------------------
struct NeuronIn {
    float V, iou, tlast;
    float J[4];     // complete receptor state of the previous step
};

struct NeuronOut {
    float V, iou, tlast;
    bool active;
};

// I_syn = ((I0 + I1) + I2) + I3, I_u = (g_u * (V_u - V)) * J_u  (block_new.py:86-90)
__device__ inline float synaptic_current(const PopParams& p, float V, const float J[4]) {
    float I[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) I[c] = __fmul_rn(__fmul_rn(p.g[c], __fsub_rn(p.Vu[c], V)), J[c]);
    return __fadd_rn(__fadd_rn(__fadd_rn(I[0], I[1]), I[2]), I[3]);
}

__device__ inline NeuronOut lif_update(const PopParams& p, const NeuronIn& in, float t, float z, bool use_ou) {
    NeuronOut o;
    const float isyn = synaptic_current(p, in.V, in.J);
    // OU background (block_new.py:92-96): i += f1 * (mu - i) + f2s * z
    float i = in.iou;
    if (use_ou) {
        const float drift = __fmul_rn(p.ou_f1, __fsub_rn(p.ou_mean, i));
        const float diff = __fmul_rn(p.ou_f2s, z);
        i = __fadd_rn(i, __fadd_rn(drift, diff));
    }
    o.iou = i;
    // Euler step (block_new.py:104-117)
    const float main_part = __fmul_rn(p.neg_gL, __fsub_rn(in.V, p.V_L));
    float cd = __fadd_rn(__fadd_rn(main_part, isyn), p.I_ext);
    if (use_ou) cd = __fadd_rn(cd, i);
    const float v_normal = __fadd_rn(in.V, __fmul_rn(p.dtC, cd));
    const bool not_sat = t >= __fadd_rn(in.tlast, p.T_ref);
    const float v = not_sat ? v_normal : p.V_reset;
    o.active = v >= p.V_th;
    o.V = fminf(v, p.V_th);
    o.tlast = o.active ? t : in.tlast;   // update_t_ik_last (block_new.py:119-120)
    return o;
}

// J <- J * decay + dJ (block_new.py:74-76), both roundings explicit.
__device__ inline float decay_add(float j, float d, float add) {
    return __fadd_rn(__fmul_rn(j, d), add);
}

__device__ inline float fix_to_float(long long x) {
    return __fmul_rn(__ll2float_rn(x), kFixInv);
}

__device__ inline long long float_to_fix(float w) {
    return __float2ll_rn(__fmul_rn(w, kFixScale));
}

// Fixed-mode pieces: a weight pair as one packed u64 addend, and a 32-bit field
// back to float (u is rounded to float32 once; the power-of-two scale is exact).
__device__ inline unsigned long long pack_fixed(float2 w, float scale) {
    const unsigned long long lo = __float2uint_rn(__fmul_rn(w.x, scale));
    const unsigned long long hi = __float2uint_rn(__fmul_rn(w.y, scale));
    return (hi << 32) | lo;
}
__device__ inline float fixed_field(unsigned long long packed, int hi, float unscale) {
    return __fmul_rn(__uint2float_rn(static_cast<uint32_t>(hi ? packed >> 32 : packed)), unscale);
}

// Population of neuron i: largest p with pop_off[p] <= i.
__device__ inline uint32_t find_pop(const uint32_t* __restrict__ off, uint32_t n_pops, uint32_t i) {
    uint32_t lo = 0, hi = n_pops - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(off + mid) <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ inline void load_pop_params(const NetView& nv, uint32_t p, uint32_t i, PopParams& out) {
    if (!nv.per_neuron) {
        const float4* src = reinterpret_cast<const float4*>(nv.pop + p);
        float4* dst = reinterpret_cast<float4*>(&out);
#pragma unroll
        for (int k = 0; k < 6; ++k) dst[k] = __ldg(src + k);
    } else {
        float* dst = reinterpret_cast<float*>(&out);
#pragma unroll
        for (int k = 0; k < kParamFloats; ++k) dst[k] = __ldg(nv.np_params + static_cast<size_t>(k) * nv.n_pad + i);
    }
}

}  // namespace dtb
