// Host-side pieces of the engine that need no GPU: parameter derivation, the
// population table, the host CSR builder and the npz reader.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "dtb_device.cuh"

namespace dtb {

// Raw neuron parameters: the property columns of the reference
// (python/make_block.py:426-464) plus the OU parameters.
struct RawParams {
    float noise_rate, I_ext, C, T_ref, g_L, V_L, V_th, V_reset;
    float g[4], Vu[4], tau[4];
    float ou_mean, ou_sigma, ou_tau;
};

RawParams raw_from_property(const float* row, float ou_mean, float ou_sigma, float ou_tau);
bool same_params(const float* a, const float* b);   // property rows equal except column 3 (population)

// Derived constants in block_new's float32 evaluation order (see PopParams).
PopParams derive(const RawParams& r, float dt);

// snn.proto PropType -> raw field; returns false for unknown ids.
bool raw_field(RawParams& r, uint32_t prop_id, float** field);

// Stable CSR (counting sort): rows indexed by `key` (0..n_rows-1) keep the input
// order of their entries.  Returns row offsets [n_rows + 1] and the permutation.
void counting_sort(const uint32_t* key, uint64_t n_items, uint32_t n_rows,
                   std::vector<uint64_t>& row_ptr, std::vector<uint64_t>& perm);

// Minimal npz reader: numpy .npy members of a zip archive, stored or deflated
// (zip64 aware).
struct NpyArray {
    std::string dtype;            // numpy descr, e.g. "<f4", "|u1"
    std::vector<uint64_t> shape;
    std::vector<uint8_t> data;
    bool fortran = false;
    uint64_t count() const { uint64_t c = 1; for (auto s : shape) c *= s; return c; }
    size_t word() const;
};

// Returns an empty string on success, else the reason.
std::string npz_load(const std::string& path, const std::vector<std::string>& names,
                     std::vector<NpyArray>& out, std::vector<bool>& found);

}  // namespace dtb
