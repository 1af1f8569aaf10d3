/*
 * CPU oracle of the DTB per-timestep hot path, in C -- TEST INFRASTRUCTURE ONLY.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
 * as the checker and as the timed CPU port; the product never does.
 *
 * It restates the reference's CPU model models/block_new.py:
 *   run                   block_new.py:122-158
 *   update_i_background   block_new.py:92-96
 *   update_Vi             block_new.py:104-117
 *   update_J_ui / bmm     block_new.py:71-84   (W.s over ALL synapses every step,
 *                                               the cost structure of torch.sparse.mm)
 *   update_I_syn          block_new.py:86-90
 *   update_t_ik_last      block_new.py:119-120
 * in the same float32 operation order as oracle/lif_oracle.py (which is pinned
 * to block_new's own output).  W.s is accumulated in double per postsynaptic
 * neuron in in-edge order and rounded once, exactly like numpy.bincount.
 * Build with -ffp-contract=off so no multiply-add is fused.
 *
 * It also replays the engine's regional-network edge stream (Philox4x32-10,
 * Salmon et al. SC'11) so large sample networks can be built on the host fast.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    int32_t n;
    const int64_t* in_ptr;    /* [n+1] in-edge CSR by postsynaptic neuron      */
    const uint32_t* in_pre;   /* [S] presynaptic neuron                         */
    const uint8_t* in_kind;   /* [S] 0: AMPA/NMDA, 1: GABAa/GABAb               */
    const float* w0;          /* [S]                                            */
    const float* w1;          /* [S]                                            */
    /* per-neuron derived constants (see lif_oracle.LifOracle) */
    const float* dtC;
    const float* neg_gL;
    const float* V_L;
    const float* V_th;
    const float* V_reset;
    const float* T_ref;
    const float* I_ext;
    const float* noise_rate;
    const float* g;           /* [4*n] channel-major */
    const float* Vu;          /* [4*n] */
    const float* decay;       /* [4*n] */
    const float* ou_mean;
    const float* ou_f1;
    const float* ou_f2s;
    /* state (updated in place) */
    float* V;
    float* i_bg;
    float* t_last;
    float* J;                 /* [4*n] channel-major */
    float* I_syn;
    float* t;                 /* scalar */
    /* scratch */
    uint8_t* active;
    uint8_t* prop;
} oracle_net;

static float fadd(float a, float b) { return a + b; }
static float fmul(float a, float b) { return a * b; }
static float fsub(float a, float b) { return a - b; }

/* `steps` steps; z [steps*n] normal draws, u [steps*n] uniforms or NULL;
 * prop_mode 0/1/2 as in lif_oracle.  Threshold spikes go to spikes_out
 * [steps*n] and per-step spike counts to counts_out [steps] when non-NULL.
 * Returns the synaptic events delivered (in-edges whose source propagated). */
int64_t oracle_run(oracle_net* s, int32_t steps, float dt, const float* z, const float* u, int prop_mode,
                   uint8_t* spikes_out, int64_t* counts_out) {
    const int32_t n = s->n;
    int64_t events = 0;
    for (int32_t st = 0; st < steps; ++st) {
        const float* zs = z + (int64_t)st * n;
        const float* us = u ? u + (int64_t)st * n : NULL;
        const float t = fadd(*s->t, dt);
        *s->t = t;
        int64_t cnt = 0;
#pragma omp parallel for schedule(static) reduction(+ : cnt)
        for (int32_t i = 0; i < n; ++i) {
            const float ib = fadd(s->i_bg[i], fadd(fmul(s->ou_f1[i], fsub(s->ou_mean[i], s->i_bg[i])),
                                                   fmul(s->ou_f2s[i], zs[i])));
            s->i_bg[i] = ib;
            const float main_part = fmul(s->neg_gL[i], fsub(s->V[i], s->V_L[i]));
            const float cd = fadd(fadd(fadd(main_part, s->I_syn[i]), s->I_ext[i]), ib);
            const float vn = fadd(s->V[i], fmul(s->dtC[i], cd));
            const int not_sat = t >= fadd(s->t_last[i], s->T_ref[i]);
            const float v = not_sat ? vn : s->V_reset[i];
            const uint8_t a = v >= s->V_th[i];
            s->V[i] = v < s->V_th[i] ? v : s->V_th[i];
            s->active[i] = a;
            uint8_t p = a;
            if (prop_mode != 0) {
                const uint8_t noise = us[i] < s->noise_rate[i];
                p = prop_mode == 1 ? noise : (uint8_t)(noise | a);
            }
            s->prop[i] = p;
            cnt += a;
        }
        int64_t ev = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : ev)
        for (int32_t i = 0; i < n; ++i) {
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
            for (int64_t e = s->in_ptr[i]; e < s->in_ptr[i + 1]; ++e) {
                if (s->prop[s->in_pre[e]]) {
                    const int c = s->in_kind[e] ? 2 : 0;
                    acc[c] += (double)s->w0[e];
                    acc[c + 1] += (double)s->w1[e];
                    ++ev;
                }
            }
            float I[4];
            for (int c = 0; c < 4; ++c) {
                const int64_t k = (int64_t)c * n + i;
                const float j = fadd(fmul(s->J[k], s->decay[k]), (float)acc[c]);
                s->J[k] = j;
                I[c] = fmul(fmul(s->g[k], fsub(s->Vu[k], s->V[i])), j);
            }
            s->I_syn[i] = fadd(fadd(fadd(I[0], I[1]), I[2]), I[3]);
            if (s->active[i]) s->t_last[i] = t;
        }
        events += ev;
        if (spikes_out) memcpy(spikes_out + (int64_t)st * n, s->active, (size_t)n);
        if (counts_out) counts_out[st] = cnt;
    }
    return events;
}

/* ---- event-driven twin for long statistical runs ------------------------
 * The same step as oracle_run, but W.s is gathered from the out-edge rows of the
 * propagating neurons only (O(events) instead of O(S) per step), so 10,000-step
 * runs of in-degree-1000 networks finish in seconds.  Each postsynaptic sum is
 * still accumulated in double and rounded once; for weights that are multiples
 * of 2^-24 below 1 (every generator here) a double sum of up to 2^29 of them is
 * exact in any order, so the result is bit-identical to oracle_run's.  Threads
 * own disjoint postsynaptic ranges (rows ascend by target), so no two write the
 * same accumulator.  Population spike counts and the pooled inter-spike-interval
 * moments are kept on the fly from absolute step `warm` on. */
typedef struct {
    const int64_t* out_ptr;   /* [n+1] out-edge CSR by presynaptic neuron        */
    const uint32_t* out_post; /* [S] postsynaptic neuron, ascending within a row  */
    const uint8_t* out_kind;  /* [S] 0: AMPA/NMDA, 1: GABAa/GABAb                 */
    const float* ow0;         /* [S]                                             */
    const float* ow1;         /* [S]                                             */
    const int32_t* pop_of;    /* [n] population index, 0..n_pops-1                */
    int32_t n_pops;
    int64_t step0;            /* absolute index of this call's first step          */
    int64_t warm;             /* statistics from this absolute step on              */
    int64_t* pop_spikes;      /* [n_pops] threshold spikes since `warm`             */
    int64_t* last_spike;      /* [n] absolute step of the last threshold spike, -1  */
    double* isi;              /* [3] count, sum, sum of squares of ISIs (in steps)  */
    double* acc;              /* scratch [4*n], zero between calls                 */
    uint32_t* list;           /* scratch [n]                                       */
} oracle_events;

static int64_t lower_post(const uint32_t* post, int64_t b, int64_t e, uint32_t x) {
    while (b < e) {
        const int64_t m = b + (e - b) / 2;
        if (post[m] < x) b = m + 1; else e = m;
    }
    return b;
}

int64_t oracle_run_events(oracle_net* s, oracle_events* ev, int32_t steps, float dt, const float* z, const float* u,
                          int prop_mode, int64_t* counts_out) {
    const int32_t n = s->n, P = ev->n_pops;
    int64_t events = 0;
    for (int32_t st = 0; st < steps; ++st) {
        const int64_t abs_step = ev->step0 + st;
        const int stat = abs_step >= ev->warm;
        const float* zs = z + (int64_t)st * n;
        const float* us = u ? u + (int64_t)st * n : NULL;
        const float t = fadd(*s->t, dt);
        *s->t = t;
        int64_t cnt = 0;
        double ic = 0.0, is = 0.0, iq = 0.0;
        int64_t* ps = ev->pop_spikes;
#pragma omp parallel for schedule(static) reduction(+ : cnt, ic, is, iq) reduction(+ : ps[:P])
        for (int32_t i = 0; i < n; ++i) {
            const float ib = fadd(s->i_bg[i], fadd(fmul(s->ou_f1[i], fsub(s->ou_mean[i], s->i_bg[i])),
                                                   fmul(s->ou_f2s[i], zs[i])));
            s->i_bg[i] = ib;
            const float main_part = fmul(s->neg_gL[i], fsub(s->V[i], s->V_L[i]));
            const float cd = fadd(fadd(fadd(main_part, s->I_syn[i]), s->I_ext[i]), ib);
            const float vn = fadd(s->V[i], fmul(s->dtC[i], cd));
            const int not_sat = t >= fadd(s->t_last[i], s->T_ref[i]);
            const float v = not_sat ? vn : s->V_reset[i];
            const uint8_t a = v >= s->V_th[i];
            s->V[i] = v < s->V_th[i] ? v : s->V_th[i];
            s->active[i] = a;
            uint8_t p = a;
            if (prop_mode != 0) {
                const uint8_t noise = us[i] < s->noise_rate[i];
                p = prop_mode == 1 ? noise : (uint8_t)(noise | a);
            }
            s->prop[i] = p;
            cnt += a;
            if (a && stat) {
                ps[ev->pop_of[i]] += 1;
                const int64_t prev = ev->last_spike[i];
                if (prev >= ev->warm) {
                    const double d = (double)(abs_step - prev);
                    ic += 1.0;
                    is += d;
                    iq += d * d;
                }
            }
            if (a) ev->last_spike[i] = abs_step;
        }
        ev->isi[0] += ic;
        ev->isi[1] += is;
        ev->isi[2] += iq;
        int32_t m = 0;
        int64_t ev_step = 0;
        for (int32_t i = 0; i < n; ++i)
            if (s->prop[i]) {
                ev->list[m++] = (uint32_t)i;
                ev_step += ev->out_ptr[i + 1] - ev->out_ptr[i];
            }
#pragma omp parallel
        {
#ifdef _OPENMP
            const int64_t nth = omp_get_num_threads(), tid = omp_get_thread_num();
#else
            const int64_t nth = 1, tid = 0;
#endif
            const uint32_t lo = (uint32_t)((int64_t)n * tid / nth), hi = (uint32_t)((int64_t)n * (tid + 1) / nth);
            double* acc = ev->acc;
            for (int32_t k = 0; k < m; ++k) {
                const uint32_t j = ev->list[k];
                const int64_t e1 = ev->out_ptr[j + 1];
                for (int64_t e = lower_post(ev->out_post, ev->out_ptr[j], e1, lo); e < e1 && ev->out_post[e] < hi; ++e) {
                    const int64_t c = ev->out_kind[e] ? 2 : 0;
                    const uint32_t q = ev->out_post[e];
                    acc[c * n + q] += (double)ev->ow0[e];
                    acc[(c + 1) * n + q] += (double)ev->ow1[e];
                }
            }
            for (uint32_t i = lo; i < hi; ++i) {
                float I[4];
                for (int c = 0; c < 4; ++c) {
                    const int64_t k = (int64_t)c * n + i;
                    const float j = fadd(fmul(s->J[k], s->decay[k]), (float)acc[k]);
                    acc[k] = 0.0;
                    s->J[k] = j;
                    I[c] = fmul(fmul(s->g[k], fsub(s->Vu[k], s->V[i])), j);
                }
                s->I_syn[i] = fadd(fadd(fadd(I[0], I[1]), I[2]), I[3]);
                if (s->active[i]) s->t_last[i] = t;
            }
        }
        events += ev_step;
        if (counts_out) counts_out[st] = cnt;
    }
    ev->step0 += steps;
    return events;
}

/* ---- FP64 restatement ---------------------------------------------------
 * The same step in double precision throughout (constants derived in double by
 * lif_oracle.LifOracle(dtype=float64); weights widened exactly; the normal draws
 * widened from the float32 stream every run shares).  This is block_new under
 * torch.set_default_dtype(torch.float64), the reference for precision
 * statements about float32 and bf16 runs. */
typedef struct {
    int32_t n;
    const int64_t* in_ptr;
    const uint32_t* in_pre;
    const uint8_t* in_kind;
    const double* w0;
    const double* w1;
    const double* dtC;
    const double* neg_gL;
    const double* V_L;
    const double* V_th;
    const double* V_reset;
    const double* T_ref;
    const double* I_ext;
    const double* g;          /* [4*n] channel-major */
    const double* Vu;
    const double* decay;
    const double* ou_mean;
    const double* ou_f1;
    const double* ou_f2s;
    double* V;
    double* i_bg;
    double* t_last;
    double* J;
    double* I_syn;
    double* t;
    uint8_t* active;
} oracle_net64;

/* Threshold propagation only.  V_out [steps*n_v] receives V of the first n_v
 * neurons after every step when non-NULL.  clock32 != 0 rounds the clock to
 * float32 after every `t += dt` (block_new's float32 time) and keeps everything
 * else in double: it isolates the part of a float32 run's difference that the
 * refractory test `t >= t_last + T_ref` makes. */
int64_t oracle_run_f64(oracle_net64* s, int32_t steps, double dt, const float* z, uint8_t* spikes_out,
                       int64_t* counts_out, float* V_out, int32_t n_v, int32_t clock32) {
    const int32_t n = s->n;
    int64_t events = 0;
    for (int32_t st = 0; st < steps; ++st) {
        const float* zs = z + (int64_t)st * n;
        const double t = clock32 ? (double)(float)(*s->t + dt) : *s->t + dt;
        *s->t = t;
        int64_t cnt = 0;
#pragma omp parallel for schedule(static) reduction(+ : cnt)
        for (int32_t i = 0; i < n; ++i) {
            const double ib = s->i_bg[i] + (s->ou_f1[i] * (s->ou_mean[i] - s->i_bg[i]) + s->ou_f2s[i] * (double)zs[i]);
            s->i_bg[i] = ib;
            const double cd = ((s->neg_gL[i] * (s->V[i] - s->V_L[i]) + s->I_syn[i]) + s->I_ext[i]) + ib;
            const double vn = s->V[i] + s->dtC[i] * cd;
            const double v = t >= s->t_last[i] + s->T_ref[i] ? vn : s->V_reset[i];
            const uint8_t a = v >= s->V_th[i];
            s->V[i] = v < s->V_th[i] ? v : s->V_th[i];
            s->active[i] = a;
            cnt += a;
        }
        int64_t ev = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : ev)
        for (int32_t i = 0; i < n; ++i) {
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
            for (int64_t e = s->in_ptr[i]; e < s->in_ptr[i + 1]; ++e) {
                if (s->active[s->in_pre[e]]) {
                    const int c = s->in_kind[e] ? 2 : 0;
                    acc[c] += s->w0[e];
                    acc[c + 1] += s->w1[e];
                    ++ev;
                }
            }
            double I = 0.0;
            for (int c = 0; c < 4; ++c) {
                const int64_t k = (int64_t)c * n + i;
                const double j = s->J[k] * s->decay[k] + acc[c];
                s->J[k] = j;
                I += s->g[k] * (s->Vu[k] - s->V[i]) * j;
            }
            s->I_syn[i] = I;
            if (s->active[i]) s->t_last[i] = t;
        }
        events += ev;
        if (spikes_out) memcpy(spikes_out + (int64_t)st * n, s->active, (size_t)n);
        if (counts_out) counts_out[st] = cnt;
        if (V_out)
            for (int32_t i = 0; i < n_v; ++i) V_out[(int64_t)st * n_v + i] = (float)s->V[i];
    }
    return events;
}

/* ---- Philox4x32-10 and the regional-network edge stream ---------------- */
static void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t o0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        const uint32_t o1 = (uint32_t)p1;
        const uint32_t o2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        const uint32_t o3 = (uint32_t)p0;
        c[0] = o0; c[1] = o1; c[2] = o2; c[3] = o3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

/* Edges (post, k) for k < in_degree of every post, post-major, written to
 * pre/kind/w0/w1 at index post*in_degree + k. */
void oracle_structured_edges(int32_t n_pops, const uint32_t* pop_off, const uint32_t* pop_exc, const uint64_t* cdf,
                             uint64_t seed, int32_t dyadic, uint32_t in_degree, uint32_t* pre, uint8_t* kind,
                             float* w0, float* w1) {
    const uint32_t n = pop_off[n_pops];
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t post = 0; post < (int64_t)n; ++post) {
        int32_t lo = 0, hi = n_pops - 1;
        while (lo < hi) {
            const int32_t mid = (lo + hi + 1) >> 1;
            if (pop_off[mid] <= (uint32_t)post) lo = mid; else hi = mid - 1;
        }
        const int32_t a = lo;
        const uint64_t* row = cdf + (int64_t)a * n_pops;
        for (uint32_t k = 0; k < in_degree; ++k) {
            uint32_t c[4] = {(uint32_t)post, k, 0x5EED0001u, 0u};
            philox(c, (uint32_t)seed, (uint32_t)(seed >> 32));
            int32_t b0 = 0, b1 = n_pops - 1;
            while (b0 < b1) {
                const int32_t mid = (b0 + b1) >> 1;
                if ((uint64_t)c[0] < row[mid]) b1 = mid; else b0 = mid + 1;
            }
            const int32_t b = b0;
            const uint32_t off = pop_off[b], size = pop_off[b + 1] - off;
            uint32_t j;
            if (b == a) {
                j = off + (uint32_t)(((uint64_t)c[1] * (size - 1)) >> 32);
                if (j >= (uint32_t)post) ++j;
            } else {
                j = off + (uint32_t)(((uint64_t)c[1] * size) >> 32);
            }
            const int64_t e = post * (int64_t)in_degree + k;
            pre[e] = j;
            kind[e] = (j - off) >= pop_exc[b];
            if (dyadic) {
                w0[e] = (float)(c[2] >> 24) * (1.0f / 256.0f);
                w1[e] = (float)(c[3] >> 24) * (1.0f / 256.0f);
            } else {
                w0[e] = (float)(c[2] >> 8) * (1.0f / 16777216.0f);
                w1[e] = (float)(c[3] >> 8) * (1.0f / 16777216.0f);
            }
        }
    }
}

int32_t oracle_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
