// Balloon-Windkessel BOLD model for data assimilation: the step after the hot
// path in DA_voxel.py (voxel activity -> BOLD signal, data_assimilation/DA_voxel.py:314-331).
//
// The reference advances models/bold_model_pytorch.py:61-96 (BOLD.run) once
// per simulated step as ~20 separate tensor operations.  Here one thread owns
// one voxel's state (s, q, v, f_in) in registers for a whole window of steps:
// one launch per window, the activity streamed in and the signal streamed out
// with coalesced loads and stores.  Arithmetic follows BOLD.run in float32 and
// in its order: q, v, f_in, s are advanced in place in that order (q reads the
// old v and f_in, f_in the old s, the output the new q and v); divisions by
// parameters are correctly rounded divisions; x ** y is powf.  Parameters are
// Python floats in the reference, so every parameter expression is evaluated
// in double on the host and rounded to float32 once.
#include <cmath>

#include "dtb_engine.h"

namespace dtb {

struct BoldConst {
    float eps, tao_s, tao_f, tao_0, e0, v0, dt;
    float one_m_e0, div_alpha, div_alpha_m1, seven_e0, e0_term;
};

__global__ void __launch_bounds__(128)
bold_kernel(BoldConst c, uint32_t n, uint32_t steps, const float* __restrict__ u, float* __restrict__ state,
            float* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float s = state[i], q = state[n + i], v = state[2 * n + i], f = state[3 * n + i];
    for (uint32_t k = 0; k < steps; ++k) {
        const float uk = __ldcs(u + static_cast<size_t>(k) * n + i);
        // d_s = epsilon * u - s / tao_s - (f_in - 1) / tao_f
        const float d_s = __fsub_rn(__fsub_rn(__fmul_rn(c.eps, uk), __fdiv_rn(s, c.tao_s)),
                                    __fdiv_rn(__fsub_rn(f, 1.0f), c.tao_f));
        // q_part = 1 - (1 - E_0) ** (1 / f_in) where f_in > 0, else 1
        const float q_part = f > 0.0f ? __fsub_rn(1.0f, powf(c.one_m_e0, __fdiv_rn(1.0f, f))) : 1.0f;
        const float dq = __fdiv_rn(__fsub_rn(__fdiv_rn(__fmul_rn(f, q_part), c.e0), __fmul_rn(q, powf(v, c.div_alpha_m1))),
                                   c.tao_0);
        q = __fadd_rn(q, __fmul_rn(dq, c.dt));
        const float dv = __fdiv_rn(__fsub_rn(f, powf(v, c.div_alpha)), c.tao_0);
        v = __fadd_rn(v, __fmul_rn(dv, c.dt));
        f = __fadd_rn(f, __fmul_rn(s, c.dt));
        f = f > 0.0f ? f : 0.0f;
        s = __fadd_rn(s, __fmul_rn(d_s, c.dt));
        if (out) {
            // V_0 * (7 E_0 (1 - q) + 2 (1 - q / v) + (2 E_0 - 0.2) (1 - v))
            const float a = __fmul_rn(c.seven_e0, __fsub_rn(1.0f, q));
            const float b = __fmul_rn(2.0f, __fsub_rn(1.0f, __fdiv_rn(q, v)));
            const float d = __fmul_rn(c.e0_term, __fsub_rn(1.0f, v));
            out[static_cast<size_t>(k) * n + i] = __fmul_rn(c.v0, __fadd_rn(__fadd_rn(a, b), d));
        }
    }
    state[i] = s;
    state[n + i] = q;
    state[2 * n + i] = v;
    state[3 * n + i] = f;
}

}  // namespace dtb

extern "C" {

void dtb_bold_default_params(dtb_bold_params* p) {
    if (!p) return;
    // data_assimilation/DA_voxel.py:470-476
    *p = dtb_bold_params{200.0, 0.8, 0.4, 1.0, 0.2, 0.8, 0.02, 1e-3};
}

int32_t dtb_bold_run(const dtb_bold_params* p, uint32_t n, uint32_t steps, const float* u, float* state, float* out,
                     void* stream) {
    if (!p || (n && (!u || !state))) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    if (!(p->alpha > 0.0) || !(p->tao_s != 0.0) || !(p->tao_f != 0.0) || !(p->tao_0 != 0.0) || !(p->E_0 != 0.0))
        return dtb::fail(DTB_INVALID_PARAMETER, "BOLD parameters: alpha > 0 and nonzero time constants and E_0");
    if (n == 0 || steps == 0) return DTB_OK;
    const double div_alpha = 1.0 / p->alpha;
    const dtb::BoldConst c{static_cast<float>(p->epsilon), static_cast<float>(p->tao_s), static_cast<float>(p->tao_f),
                           static_cast<float>(p->tao_0), static_cast<float>(p->E_0), static_cast<float>(p->V_0),
                           static_cast<float>(p->delta_t), static_cast<float>(1.0 - p->E_0),
                           static_cast<float>(div_alpha), static_cast<float>(div_alpha - 1.0),
                           static_cast<float>(7.0 * p->E_0), static_cast<float>(2.0 * p->E_0 - 0.2)};
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    dtb::bold_kernel<<<(n + 127) / 128, 128, 0, s>>>(c, n, steps, u, state, out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return dtb::cuda_fail(e, "bold_kernel");
    return DTB_OK;
}

}  // extern "C"
