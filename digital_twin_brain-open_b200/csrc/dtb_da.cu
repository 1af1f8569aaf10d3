// Ensemble Kalman update of data assimilation: DA_voxel.filter
// (data_assimilation/DA_voxel.py:289-307), the step that follows the BOLD
// model in each assimilation window.
//
// w_hat [E][V][S] holds, per ensemble member and voxel, the assimilated
// hyper-parameters, the hemodynamic state and, last, the BOLD signal.  With
// d = w_hat - mean_e(w_hat), c_v = sum_e d[e,v,S-1]^2 / (E-1) + sigma,
// T[e,v] = d[e,v,S-1] / c_v / (E-1) and the innovation
// I[e,v] = y[v] + sqrt(sigma) n[e,v] - w_hat[e,v,S-1]:
//   w = w_hat + rate * I[e,v] * sum_e' T[e',v] d[e',v,s]
//             + (1 - rate) * sum_e' G[e,e'] d[e',v,s],   G = I T^T / V.
// Three kernels: per-voxel statistics (one warp per voxel), the E x E gain G,
// and the update (one thread per output).  Everything accumulates in double and
// is rounded once, so the result is the float32 rounding of the exact update
// (the reference's float32 reductions and GEMMs agree to ~1e-7 relative).
#include "dtb_engine.h"

namespace dtb {

__global__ void __launch_bounds__(256)
da_stats_kernel(uint32_t E, uint32_t V, uint32_t S, const float* __restrict__ w, const float* __restrict__ y,
                const float* __restrict__ noise, double sigma, double* __restrict__ mean, double* __restrict__ temp,
                double* __restrict__ innov, double* __restrict__ colsum) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const double sq = sqrt(sigma);
    for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < V; v += nw) {
        for (uint32_t s = 0; s < S; ++s) {
            double acc = 0.0;
            for (uint32_t e = lane; e < E; e += 32) acc += w[(static_cast<size_t>(e) * V + v) * S + s];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) mean[static_cast<size_t>(v) * S + s] = acc / E;
        }
        __syncwarp();
        const double ml = mean[static_cast<size_t>(v) * S + S - 1];
        double cx = 0.0;
        for (uint32_t e = lane; e < E; e += 32) {
            const double d = w[(static_cast<size_t>(e) * V + v) * S + S - 1] - ml;
            cx += d * d;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cx += __shfl_xor_sync(0xffffffffu, cx, o);
        const double cxx = cx / (E - 1) + sigma;
        for (uint32_t e = lane; e < E; e += 32) {
            const double last = w[(static_cast<size_t>(e) * V + v) * S + S - 1];
            temp[static_cast<size_t>(e) * V + v] = (last - ml) / cxx / (E - 1);
            innov[static_cast<size_t>(e) * V + v] = static_cast<double>(y[v]) + sq * noise[static_cast<size_t>(e) * V + v] - last;
        }
        __syncwarp();
        for (uint32_t s = 0; s < S; ++s) {
            const double m = mean[static_cast<size_t>(v) * S + s];
            double acc = 0.0;
            for (uint32_t e = lane; e < E; e += 32)
                acc += temp[static_cast<size_t>(e) * V + v] * (w[(static_cast<size_t>(e) * V + v) * S + s] - m);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) colsum[static_cast<size_t>(v) * S + s] = acc;
        }
    }
}

// G[e][f] = sum_v I[e,v] T[f,v] / V: one warp per (e, f).
__global__ void __launch_bounds__(256)
da_gain_kernel(uint32_t E, uint32_t V, const double* __restrict__ innov, const double* __restrict__ temp,
               double* __restrict__ gain) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < E * E; k += nw) {
        const uint32_t e = k / E, f = k % E;
        double acc = 0.0;
        for (uint32_t v = lane; v < V; v += 32) acc += innov[static_cast<size_t>(e) * V + v] * temp[static_cast<size_t>(f) * V + v];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) gain[k] = acc / V;
    }
}

__global__ void __launch_bounds__(256)
da_update_kernel(uint32_t E, uint32_t V, uint32_t S, const float* __restrict__ w, const double* __restrict__ mean,
                 const double* __restrict__ innov, const double* __restrict__ colsum, const double* __restrict__ gain,
                 double rate, float* __restrict__ out) {
    const size_t total = static_cast<size_t>(E) * V * S;
    for (size_t k = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; k < total; k += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const uint32_t s = static_cast<uint32_t>(k % S);
        const uint32_t v = static_cast<uint32_t>((k / S) % V);
        const uint32_t e = static_cast<uint32_t>(k / (static_cast<size_t>(S) * V));
        const size_t col = static_cast<size_t>(v) * S + s;
        const double m = mean[col];
        double acc = 0.0;
        for (uint32_t f = 0; f < E; ++f) acc += gain[static_cast<size_t>(e) * E + f] * (w[static_cast<size_t>(f) * V * S + col] - m);
        const double x = static_cast<double>(w[k]) + rate * innov[static_cast<size_t>(e) * V + v] * colsum[col] + (1.0 - rate) * acc;
        out[k] = static_cast<float>(x);
    }
}

}  // namespace dtb

extern "C" int32_t dtb_da_filter(uint32_t ensembles, uint32_t voxels, uint32_t states, const float* w_hat,
                                 const float* bold_y, const float* noise, double bold_sigma, double rate, float* w_out,
                                 void* stream) {
    if (!w_hat || !bold_y || !noise || !w_out) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    if (ensembles < 2 || voxels == 0 || states == 0) return dtb::fail(DTB_INVALID_PARAMETER, "need >= 2 members, voxels and states");
    if (!(bold_sigma >= 0.0)) return dtb::fail(DTB_INVALID_PARAMETER, "bold_sigma must be >= 0");
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t E = ensembles, V = voxels, S = states;
    double* buf = nullptr;
    const size_t n_mean = V * S, n_ev = E * V;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&buf), sizeof(double) * (2 * n_mean + 2 * n_ev + E * E), s);
    if (e != cudaSuccess) return dtb::cuda_fail(e, "dtb_da_filter scratch");
    double* mean = buf;
    double* colsum = mean + n_mean;
    double* temp = colsum + n_mean;
    double* innov = temp + n_ev;
    double* gain = innov + n_ev;
    const uint32_t warps_v = static_cast<uint32_t>(std::min<size_t>((V + 7) / 8, 4096));
    dtb::da_stats_kernel<<<warps_v, 256, 0, s>>>(ensembles, voxels, states, w_hat, bold_y, noise, bold_sigma, mean, temp, innov, colsum);
    dtb::da_gain_kernel<<<static_cast<uint32_t>(std::min<size_t>((E * E + 7) / 8, 4096)), 256, 0, s>>>(ensembles, voxels, innov, temp, gain);
    dtb::da_update_kernel<<<static_cast<uint32_t>(std::min<size_t>((E * V * S + 255) / 256, 65535)), 256, 0, s>>>(
        ensembles, voxels, states, w_hat, mean, innov, colsum, gain, rate, w_out);
    e = cudaGetLastError();
    cudaFreeAsync(buf, s);
    if (e != cudaSuccess) return dtb::cuda_fail(e, "dtb_da_filter");
    return DTB_OK;
}
