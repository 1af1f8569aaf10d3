// Device generator and CSR builder for regional networks.
//
// Edge (post, k), k < in_degree, is a pure function of (seed, post, k): one
// Philox4x32-10 block with counter (post, k, kStreamEdges, 0) gives
//   x -> source population b (inverse CDF over the row of the post's population),
//   y -> source neuron inside b (multiply-high; self-loops skipped),
//   z, w -> the weight pair, uniform in [0, 1) with 24 random bits (or 8 when dyadic).
// The kind bit (GABA pair) is set when the source is in the inhibitory tail of b.
//
// The in-degree CSR (pull) is the generation order itself.  The out-degree CSR
// (push) must hold, for each presynaptic neuron, its synapses in input order --
// the reference's stable sort by presynaptic neuron (src/configuration.cpp:227-249,
// 1079-1392; thrust::stable_sort_by_key there).  It is built by
//   1. an out-degree histogram and exclusive scan -> row offsets (64-bit: a 5e9-synapse
//      network overflows the reference's 32-bit rowptrs);
//   2. chunks of consecutive postsynaptic neurons, each key-sorted by presynaptic
//      neuron with a stable radix sort (CUB); because chunks are taken in input order,
//      appending each chunk's run of a row after the previous chunk's keeps every
//      row in input order;
//   3. a placement pass that regenerates each edge and writes it at
//      row_cursor[pre] + rank within the chunk's run (coalesced: runs are contiguous).
#include <cub/cub.cuh>

#include "dtb_kernels.h"

namespace dtb {

__host__ __device__ inline void gen_edge(uint32_t n_pops, const uint32_t* pop_off, const uint32_t* pop_exc,
                                         const unsigned long long* cdf, unsigned long long seed, uint32_t dyadic,
                                         uint32_t post, uint32_t a, uint32_t k,
                                         uint32_t& pre, uint32_t& kind, float& w0, float& w1) {
    const U4 r = philox4x32_10(U4{post, k, kStreamEdges, 0u}, static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
    const unsigned long long* row = cdf + static_cast<size_t>(a) * n_pops;
    uint32_t lo = 0, hi = n_pops - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (static_cast<unsigned long long>(r.x) < row[mid]) hi = mid; else lo = mid + 1;
    }
    const uint32_t b = lo;
    const uint32_t off = pop_off[b];
    const uint32_t size = pop_off[b + 1] - off;
    uint32_t j;
    if (b == a) {
        j = off + mulhi_u32(r.y, size - 1);
        if (j >= post) ++j;
    } else {
        j = off + mulhi_u32(r.y, size);
    }
    pre = j;
    kind = (j - off) >= pop_exc[b] ? 1u : 0u;
    if (dyadic) {
        w0 = static_cast<float>(r.z >> 24) * (1.0f / 256.0f);
        w1 = static_cast<float>(r.w >> 24) * (1.0f / 256.0f);
    } else {
        w0 = static_cast<float>(r.z >> 8) * (1.0f / 16777216.0f);
        w1 = static_cast<float>(r.w >> 8) * (1.0f / 16777216.0f);
    }
}

__device__ inline uint32_t pop_of(const uint32_t* __restrict__ off, uint32_t n_pops, uint32_t i) {
    uint32_t lo = 0, hi = n_pops - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (off[mid] <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <int WT>
__device__ inline void store_weight(void* base, unsigned long long e, float w0, float w1) {
    if constexpr (WT == W_F32) {
        reinterpret_cast<float2*>(base)[e] = make_float2(w0, w1);
    } else if constexpr (WT == W_BF16) {
        reinterpret_cast<__nv_bfloat162*>(base)[e] = __floats2bfloat162_rn(w0, w1);
    } else if constexpr (WT == W_F16) {
        reinterpret_cast<__half2*>(base)[e] = __floats2half2_rn(w0, w1);
    } else {
        const unsigned lo = static_cast<unsigned>(rintf(fminf(fmaxf(w0, 0.f), 1.f) * 255.f));
        const unsigned hi = static_cast<unsigned>(rintf(fminf(fmaxf(w1, 0.f), 1.f) * 255.f));
        reinterpret_cast<uchar2*>(base)[e] = make_uchar2(static_cast<unsigned char>(lo), static_cast<unsigned char>(hi));
    }
}

// Pass 1: out-degree histogram; optionally write the in-degree CSR (warp per post).
template <int WT>
__global__ void gen_in_and_count(GenSpec g, uint32_t* __restrict__ deg, uint32_t* __restrict__ in_col, void* __restrict__ in_w) {
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned long long warp = (static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const unsigned long long nwarps = (static_cast<unsigned long long>(gridDim.x) * blockDim.x) >> 5;
    for (unsigned long long post = warp; post < g.n; post += nwarps) {
        const uint32_t a = pop_of(g.pop_off, g.n_pops, static_cast<uint32_t>(post));
        for (uint32_t k = lane; k < g.in_degree; k += 32) {
            uint32_t pre, kind;
            float w0, w1;
            gen_edge(g.n_pops, g.pop_off, g.pop_exc, g.cdf, g.seed, g.dyadic, static_cast<uint32_t>(post), a, k, pre, kind, w0, w1);
            atomicAdd(deg + pre, 1u);
            if (in_col != nullptr) {
                const unsigned long long e = post * g.in_degree + k;
                in_col[e] = pre | (kind << 31);
                store_weight<WT>(in_w, e, w0, w1);
            }
        }
    }
}

__global__ void fill_in_ptr(unsigned long long* __restrict__ in_ptr, uint32_t n, uint32_t k) {
    for (unsigned long long i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x)
        in_ptr[i] = i * k;
}

__global__ void widen_u32(const uint32_t* __restrict__ src, unsigned long long* __restrict__ dst, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[i];
}

// Pass 2a: keys (presynaptic neuron) and values (local edge index) of one chunk.
__global__ void gen_chunk_keys(GenSpec g, uint32_t post0, uint32_t posts, uint32_t* __restrict__ keys,
                               uint32_t* __restrict__ vals, uint32_t* __restrict__ cnt) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t q = warp; q < posts; q += nwarps) {
        const uint32_t post = post0 + q;
        const uint32_t a = pop_of(g.pop_off, g.n_pops, post);
        for (uint32_t k = lane; k < g.in_degree; k += 32) {
            uint32_t pre, kind;
            float w0, w1;
            gen_edge(g.n_pops, g.pop_off, g.pop_exc, g.cdf, g.seed, g.dyadic, post, a, k, pre, kind, w0, w1);
            const uint32_t e = q * g.in_degree + k;
            keys[e] = pre;
            vals[e] = e;
            atomicAdd(cnt + pre, 1u);
        }
    }
}

// Pass 2c: place the sorted chunk into the out-degree CSR.
template <int WT>
__global__ void place_chunk(GenSpec g, uint32_t post0, uint32_t m, const uint32_t* __restrict__ keys,
                           const uint32_t* __restrict__ vals, const uint32_t* __restrict__ start,
                           const unsigned long long* __restrict__ cursor, uint32_t* __restrict__ out_col,
                           void* __restrict__ out_w, uint32_t* __restrict__ err) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) {
        const uint32_t j = keys[q];
        const uint32_t e = vals[q];
        const uint32_t post = post0 + e / g.in_degree;
        const uint32_t k = e % g.in_degree;
        const uint32_t a = pop_of(g.pop_off, g.n_pops, post);
        uint32_t pre, kind;
        float w0, w1;
        gen_edge(g.n_pops, g.pop_off, g.pop_exc, g.cdf, g.seed, g.dyadic, post, a, k, pre, kind, w0, w1);
        if (pre != j) { atomicOr(err, 1u); continue; }
        const unsigned long long dest = cursor[j] + (q - start[j]);
        out_col[dest] = post | (kind << 31);
        store_weight<WT>(out_w, dest, w0, w1);
    }
}

__global__ void advance_cursor(unsigned long long* __restrict__ cursor, const uint32_t* __restrict__ cnt, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) cursor[i] += cnt[i];
}

namespace {

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes ? bytes : 16); }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

#define GEN_TRY(x) do { cudaError_t e__ = (x); if (e__ != cudaSuccess) return e__; } while (0)

template <int WT>
cudaError_t build_impl(const GenSpec& g, unsigned long long* out_ptr, uint32_t* out_col, void* out_w,
                       unsigned long long* in_ptr, uint32_t* in_col, void* in_w, uint32_t* out_deg, cudaStream_t s) {
    const uint32_t n = g.n;
    const int threads = 256;
    const unsigned long long total_edges = static_cast<unsigned long long>(n) * g.in_degree;
    // out-degree histogram (+ in-degree CSR)
    GEN_TRY(cudaMemsetAsync(out_deg, 0, sizeof(uint32_t) * n, s));
    {
        const unsigned long long warps = n;
        const unsigned long long blocks = std::min<unsigned long long>((warps * 32 + threads - 1) / threads, 1u << 20);
        gen_in_and_count<WT><<<static_cast<unsigned>(blocks), threads, 0, s>>>(g, out_deg, in_col, in_w);
        GEN_TRY(cudaGetLastError());
    }
    if (in_ptr != nullptr) {
        fill_in_ptr<<<1024, 256, 0, s>>>(in_ptr, n, g.in_degree);
        GEN_TRY(cudaGetLastError());
    }
    if (out_ptr == nullptr) return cudaStreamSynchronize(s);

    // row offsets
    DevBuf wide, scan_tmp;
    GEN_TRY(wide.alloc(sizeof(unsigned long long) * (n + 1)));
    widen_u32<<<1024, 256, 0, s>>>(out_deg, wide.as<unsigned long long>(), n);
    GEN_TRY(cudaGetLastError());
    size_t tmp_bytes = 0;
    GEN_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, wide.as<unsigned long long>(), out_ptr, n, s));
    GEN_TRY(scan_tmp.alloc(tmp_bytes));
    GEN_TRY(cub::DeviceScan::ExclusiveSum(scan_tmp.p, tmp_bytes, wide.as<unsigned long long>(), out_ptr, n, s));
    GEN_TRY(cudaMemcpyAsync(out_ptr + n, &total_edges, sizeof(total_edges), cudaMemcpyHostToDevice, s));
    GEN_TRY(cudaStreamSynchronize(s));

    // chunked stable sort + placement
    const unsigned long long max_chunk_edges = 1ull << 28;
    uint32_t posts_per_chunk = static_cast<uint32_t>(std::max<unsigned long long>(1, max_chunk_edges / g.in_degree));
    posts_per_chunk = std::min(posts_per_chunk, n);
    const uint32_t m_max = posts_per_chunk * g.in_degree;
    DevBuf keys, vals, keys2, vals2, cnt, start, cursor, sort_tmp, start_tmp, err;
    GEN_TRY(keys.alloc(sizeof(uint32_t) * m_max));
    GEN_TRY(vals.alloc(sizeof(uint32_t) * m_max));
    GEN_TRY(keys2.alloc(sizeof(uint32_t) * m_max));
    GEN_TRY(vals2.alloc(sizeof(uint32_t) * m_max));
    GEN_TRY(cnt.alloc(sizeof(uint32_t) * n));
    GEN_TRY(start.alloc(sizeof(uint32_t) * n));
    GEN_TRY(cursor.alloc(sizeof(unsigned long long) * n));
    GEN_TRY(err.alloc(sizeof(uint32_t)));
    GEN_TRY(cudaMemsetAsync(err.p, 0, sizeof(uint32_t), s));
    GEN_TRY(cudaMemcpyAsync(cursor.p, out_ptr, sizeof(unsigned long long) * n, cudaMemcpyDeviceToDevice, s));
    int end_bit = 1;
    while (end_bit < 32 && (1ull << end_bit) < n) ++end_bit;
    size_t sort_bytes = 0, start_bytes = 0;
    {
        cub::DoubleBuffer<uint32_t> dk(keys.as<uint32_t>(), keys2.as<uint32_t>()), dv(vals.as<uint32_t>(), vals2.as<uint32_t>());
        GEN_TRY(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, dk, dv, static_cast<int>(m_max), 0, end_bit, s));
        GEN_TRY(cub::DeviceScan::ExclusiveSum(nullptr, start_bytes, cnt.as<uint32_t>(), start.as<uint32_t>(), n, s));
    }
    GEN_TRY(sort_tmp.alloc(sort_bytes));
    GEN_TRY(start_tmp.alloc(start_bytes));
    for (uint32_t post0 = 0; post0 < n; post0 += posts_per_chunk) {
        const uint32_t posts = std::min(posts_per_chunk, n - post0);
        const uint32_t m = posts * g.in_degree;
        GEN_TRY(cudaMemsetAsync(cnt.p, 0, sizeof(uint32_t) * n, s));
        {
            const unsigned blocks = std::min<unsigned>((posts * 32u + threads - 1) / threads, 1u << 20);
            gen_chunk_keys<<<blocks, threads, 0, s>>>(g, post0, posts, keys.as<uint32_t>(), vals.as<uint32_t>(), cnt.as<uint32_t>());
            GEN_TRY(cudaGetLastError());
        }
        cub::DoubleBuffer<uint32_t> dk(keys.as<uint32_t>(), keys2.as<uint32_t>()), dv(vals.as<uint32_t>(), vals2.as<uint32_t>());
        GEN_TRY(cub::DeviceRadixSort::SortPairs(sort_tmp.p, sort_bytes, dk, dv, static_cast<int>(m), 0, end_bit, s));
        GEN_TRY(cub::DeviceScan::ExclusiveSum(start_tmp.p, start_bytes, cnt.as<uint32_t>(), start.as<uint32_t>(), n, s));
        {
            const unsigned blocks = std::min<unsigned>((m + threads - 1) / threads, 1u << 20);
            switch (WT) {
                default:
                    place_chunk<WT><<<blocks, threads, 0, s>>>(g, post0, m, dk.Current(), dv.Current(), start.as<uint32_t>(),
                                                              cursor.as<unsigned long long>(), out_col, out_w, err.as<uint32_t>());
            }
            GEN_TRY(cudaGetLastError());
        }
        advance_cursor<<<1024, 256, 0, s>>>(cursor.as<unsigned long long>(), cnt.as<uint32_t>(), n);
        GEN_TRY(cudaGetLastError());
    }
    uint32_t h_err = 0;
    GEN_TRY(cudaMemcpyAsync(&h_err, err.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    GEN_TRY(cudaStreamSynchronize(s));
    if (h_err) return cudaErrorUnknown;
    return cudaSuccess;
}

}  // namespace

cudaError_t build_structured(const GenSpec& g, int weight_type, unsigned long long* out_ptr, uint32_t* out_col, void* out_w,
                             unsigned long long* in_ptr, uint32_t* in_col, void* in_w, uint32_t* out_deg, cudaStream_t s) {
    switch (weight_type) {
        case W_F32: return build_impl<W_F32>(g, out_ptr, out_col, out_w, in_ptr, in_col, in_w, out_deg, s);
        case W_BF16: return build_impl<W_BF16>(g, out_ptr, out_col, out_w, in_ptr, in_col, in_w, out_deg, s);
        case W_F16: return build_impl<W_F16>(g, out_ptr, out_col, out_w, in_ptr, in_col, in_w, out_deg, s);
        default: return build_impl<W_U8>(g, out_ptr, out_col, out_w, in_ptr, in_col, in_w, out_deg, s);
    }
}

void host_gen_edge(uint32_t n_pops, const uint32_t* pop_off, const uint32_t* pop_exc, const unsigned long long* cdf,
                   unsigned long long seed, uint32_t dyadic, uint32_t post, uint32_t pop_of_post, uint32_t k,
                   uint32_t* pre, uint32_t* kind, float* w0, float* w1) {
    gen_edge(n_pops, pop_off, pop_exc, cdf, seed, dyadic, post, pop_of_post, k, *pre, *kind, *w0, *w1);
}

}  // namespace dtb
