// Host-side helpers: parameter derivation, stable counting sort, npz reader.
#include "dtb_host.h"

#include <zlib.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>

namespace dtb {

RawParams raw_from_property(const float* row, float ou_mean, float ou_sigma, float ou_tau) {
    RawParams r;
    r.noise_rate = row[0];
    r.I_ext = row[2];
    r.C = row[4];
    r.T_ref = row[5];
    r.g_L = row[6];
    r.V_L = row[7];
    r.V_th = row[8];
    r.V_reset = row[9];
    for (int c = 0; c < 4; ++c) {
        r.g[c] = row[10 + c];
        r.Vu[c] = row[14 + c];
        r.tau[c] = row[18 + c];
    }
    r.ou_mean = ou_mean;
    r.ou_sigma = ou_sigma;
    r.ou_tau = ou_tau;
    return r;
}

bool same_params(const float* a, const float* b) {
    for (int c = 0; c < 22; ++c) {
        if (c == 3) continue;
        if (std::memcmp(a + c, b + c, sizeof(float)) != 0) return false;
    }
    return true;
}

// float32 arithmetic with the rounding of each step explicit (volatile stops the
// compiler from keeping wider intermediates or contracting).
static float f32_mul(float a, float b) { volatile float r = a * b; return r; }
static float f32_sub(float a, float b) { volatile float r = a - b; return r; }
static float f32_div(float a, float b) { volatile float r = a / b; return r; }

PopParams derive(const RawParams& r, float dt) {
    PopParams p;
    std::memset(&p, 0, sizeof(p));
    // dt / C evaluated as reciprocal(C) * dt (torch __rtruediv__), block_new.py:109
    p.dtC = f32_mul(f32_div(1.0f, r.C), dt);
    p.neg_gL = -r.g_L;
    p.V_L = r.V_L;
    p.V_th = r.V_th;
    p.V_reset = r.V_reset;
    p.T_ref = r.T_ref;
    p.I_ext = r.I_ext;
    p.noise_rate = r.noise_rate;
    const float neg_dt = -dt;
    const float neg_2dt = static_cast<float>(-2.0 * static_cast<double>(dt));
    for (int c = 0; c < 4; ++c) {
        p.g[c] = r.g[c];
        p.Vu[c] = r.Vu[c];
        // exp(-dt / tau) = exp(reciprocal(tau) * -dt), block_new.py:74; exp in double, rounded once
        const float x = f32_mul(f32_div(1.0f, r.tau[c]), neg_dt);
        p.decay[c] = static_cast<float>(std::exp(static_cast<double>(x)));
    }
    // OU factors, block_new.py:93-95
    const float rt = f32_div(1.0f, r.ou_tau);
    const float e1 = static_cast<float>(std::exp(static_cast<double>(f32_mul(rt, neg_dt))));
    const float e2 = static_cast<float>(std::exp(static_cast<double>(f32_mul(rt, neg_2dt))));
    p.ou_f1 = f32_sub(1.0f, e1);
    const float f2 = static_cast<float>(std::sqrt(static_cast<double>(f32_sub(1.0f, e2))));
    p.ou_f2s = f32_mul(f2, r.ou_sigma);
    p.ou_mean = r.ou_mean;
    return p;
}

bool raw_field(RawParams& r, uint32_t prop_id, float** field) {
    switch (prop_id) {
        case 0: *field = &r.I_ext; return true;
        case 1: *field = &r.C; return true;
        case 2: *field = &r.T_ref; return true;
        case 3: *field = &r.g_L; return true;
        case 4: *field = &r.V_L; return true;
        case 5: *field = &r.V_th; return true;
        case 6: *field = &r.V_reset; return true;
        case 7: case 8: case 9: case 10: *field = &r.g[prop_id - 7]; return true;
        case 11: case 12: case 13: case 14: *field = &r.Vu[prop_id - 11]; return true;
        case 15: case 16: case 17: case 18: *field = &r.tau[prop_id - 15]; return true;
        case 19: *field = &r.noise_rate; return true;
        default: return false;
    }
}

void counting_sort(const uint32_t* key, uint64_t n_items, uint32_t n_rows,
                   std::vector<uint64_t>& row_ptr, std::vector<uint64_t>& perm) {
    row_ptr.assign(static_cast<size_t>(n_rows) + 1, 0);
    for (uint64_t e = 0; e < n_items; ++e) row_ptr[key[e] + 1]++;
    for (uint32_t r = 0; r < n_rows; ++r) row_ptr[r + 1] += row_ptr[r];
    std::vector<uint64_t> cursor(row_ptr.begin(), row_ptr.end() - 1);
    perm.resize(n_items);
    for (uint64_t e = 0; e < n_items; ++e) perm[cursor[key[e]]++] = e;
}

// ---------------------------------------------------------------------------
// npz: a zip archive of .npy files (numpy.savez / savez_compressed).
// ---------------------------------------------------------------------------
size_t NpyArray::word() const {
    if (dtype.size() < 3) return 0;
    return static_cast<size_t>(std::atoi(dtype.c_str() + 2));
}

namespace {

uint16_t rd16(const uint8_t* p) { return static_cast<uint16_t>(p[0] | (p[1] << 8)); }
uint32_t rd32(const uint8_t* p) { return static_cast<uint32_t>(p[0]) | (static_cast<uint32_t>(p[1]) << 8) |
                                         (static_cast<uint32_t>(p[2]) << 16) | (static_cast<uint32_t>(p[3]) << 24); }
uint64_t rd64(const uint8_t* p) { return static_cast<uint64_t>(rd32(p)) | (static_cast<uint64_t>(rd32(p + 4)) << 32); }

std::string parse_npy(const std::vector<uint8_t>& buf, NpyArray& out) {
    if (buf.size() < 10 || std::memcmp(buf.data(), "\x93NUMPY", 6) != 0) return "not an npy member";
    const int major = buf[6];
    size_t hlen, hoff;
    if (major == 1) { hlen = rd16(buf.data() + 8); hoff = 10; }
    else { if (buf.size() < 12) return "short npy header"; hlen = rd32(buf.data() + 8); hoff = 12; }
    if (hoff + hlen > buf.size()) return "short npy header";
    const std::string h(reinterpret_cast<const char*>(buf.data() + hoff), hlen);
    auto find_val = [&](const char* key) -> std::string {
        const size_t k = h.find(key);
        if (k == std::string::npos) return "";
        size_t c = h.find(':', k);
        if (c == std::string::npos) return "";
        ++c;
        while (c < h.size() && h[c] == ' ') ++c;
        return h.substr(c);
    };
    std::string d = find_val("'descr'");
    if (d.empty() || d[0] != '\'') return "npy descr missing";
    out.dtype = d.substr(1, d.find('\'', 1) - 1);
    const std::string fo = find_val("'fortran_order'");
    out.fortran = fo.rfind("True", 0) == 0;
    std::string s = find_val("'shape'");
    if (s.empty() || s[0] != '(') return "npy shape missing";
    out.shape.clear();
    size_t i = 1;
    while (i < s.size() && s[i] != ')') {
        while (i < s.size() && (s[i] == ' ' || s[i] == ',')) ++i;
        if (i < s.size() && s[i] != ')') {
            char* end = nullptr;
            out.shape.push_back(std::strtoull(s.c_str() + i, &end, 10));
            i = static_cast<size_t>(end - s.c_str());
        }
    }
    const size_t data_off = hoff + hlen;
    const uint64_t need = out.count() * out.word();
    if (buf.size() - data_off < need) return "npy data truncated";
    out.data.assign(buf.begin() + static_cast<long>(data_off), buf.begin() + static_cast<long>(data_off + need));
    return "";
}

}  // namespace

std::string npz_load(const std::string& path, const std::vector<std::string>& names,
                     std::vector<NpyArray>& out, std::vector<bool>& found) {
    out.assign(names.size(), NpyArray());
    found.assign(names.size(), false);
    std::ifstream f(path, std::ios::binary);
    if (!f) return "cannot open " + path;
    f.seekg(0, std::ios::end);
    const uint64_t fsize = static_cast<uint64_t>(f.tellg());
    // end of central directory (last 64 KB + 22 bytes)
    const uint64_t tail = std::min<uint64_t>(fsize, 65557);
    std::vector<uint8_t> t(tail);
    f.seekg(static_cast<std::streamoff>(fsize - tail));
    f.read(reinterpret_cast<char*>(t.data()), static_cast<std::streamsize>(tail));
    long eocd = -1;
    for (long i = static_cast<long>(tail) - 22; i >= 0; --i)
        if (rd32(t.data() + i) == 0x06054b50u) { eocd = i; break; }
    if (eocd < 0) return "not a zip archive: " + path;
    uint64_t n_entries = rd16(t.data() + eocd + 10);
    uint64_t cd_size = rd32(t.data() + eocd + 12);
    uint64_t cd_off = rd32(t.data() + eocd + 16);
    if (cd_off == 0xFFFFFFFFu || n_entries == 0xFFFFu) {
        // zip64 end of central directory locator precedes the EOCD
        const long loc = eocd - 20;
        if (loc < 0 || rd32(t.data() + loc) != 0x07064b50u) return "zip64 locator missing";
        const uint64_t z64 = rd64(t.data() + loc + 8);
        std::vector<uint8_t> zr(56);
        f.seekg(static_cast<std::streamoff>(z64));
        f.read(reinterpret_cast<char*>(zr.data()), 56);
        if (rd32(zr.data()) != 0x06064b50u) return "zip64 record missing";
        n_entries = rd64(zr.data() + 32);
        cd_size = rd64(zr.data() + 40);
        cd_off = rd64(zr.data() + 48);
    }
    std::vector<uint8_t> cd(cd_size);
    f.seekg(static_cast<std::streamoff>(cd_off));
    f.read(reinterpret_cast<char*>(cd.data()), static_cast<std::streamsize>(cd_size));
    if (!f) return "short central directory";
    size_t p = 0;
    for (uint64_t e = 0; e < n_entries; ++e) {
        if (p + 46 > cd.size() || rd32(cd.data() + p) != 0x02014b50u) return "bad central directory";
        const uint16_t method = rd16(cd.data() + p + 10);
        uint64_t csize = rd32(cd.data() + p + 20);
        uint64_t usize = rd32(cd.data() + p + 24);
        const uint16_t nlen = rd16(cd.data() + p + 28), xlen = rd16(cd.data() + p + 30), clen = rd16(cd.data() + p + 32);
        uint64_t loff = rd32(cd.data() + p + 42);
        std::string name(reinterpret_cast<const char*>(cd.data() + p + 46), nlen);
        // zip64 extended information
        size_t x = p + 46 + nlen;
        const size_t xend = x + xlen;
        while (x + 4 <= xend) {
            const uint16_t id = rd16(cd.data() + x), sz = rd16(cd.data() + x + 2);
            if (id == 0x0001) {
                size_t q = x + 4;
                if (usize == 0xFFFFFFFFu) { usize = rd64(cd.data() + q); q += 8; }
                if (csize == 0xFFFFFFFFu) { csize = rd64(cd.data() + q); q += 8; }
                if (loff == 0xFFFFFFFFu) { loff = rd64(cd.data() + q); q += 8; }
            }
            x += 4 + sz;
        }
        p = xend + clen;
        if (name.size() > 4 && name.compare(name.size() - 4, 4, ".npy") == 0) name = name.substr(0, name.size() - 4);
        size_t which = names.size();
        for (size_t k = 0; k < names.size(); ++k) if (names[k] == name) which = k;
        if (which == names.size()) continue;
        uint8_t lh[30];
        f.seekg(static_cast<std::streamoff>(loff));
        f.read(reinterpret_cast<char*>(lh), 30);
        if (!f || rd32(lh) != 0x04034b50u) return "bad local header for " + name;
        const uint64_t data_off = loff + 30 + rd16(lh + 26) + rd16(lh + 28);
        std::vector<uint8_t> comp(csize);
        f.seekg(static_cast<std::streamoff>(data_off));
        f.read(reinterpret_cast<char*>(comp.data()), static_cast<std::streamsize>(csize));
        if (!f) return "truncated member " + name;
        std::vector<uint8_t> raw;
        if (method == 0) {
            raw.swap(comp);
        } else if (method == 8) {
            raw.resize(usize);
            z_stream zs;
            std::memset(&zs, 0, sizeof(zs));
            if (inflateInit2(&zs, -MAX_WBITS) != Z_OK) return "zlib init failed";
            uint64_t in_done = 0, out_done = 0;
            int rc = Z_OK;
            while (rc != Z_STREAM_END) {
                const uInt chunk_in = static_cast<uInt>(std::min<uint64_t>(csize - in_done, 1u << 30));
                const uInt chunk_out = static_cast<uInt>(std::min<uint64_t>(usize - out_done, 1u << 30));
                zs.next_in = comp.data() + in_done;
                zs.avail_in = chunk_in;
                zs.next_out = raw.data() + out_done;
                zs.avail_out = chunk_out;
                rc = inflate(&zs, Z_NO_FLUSH);
                in_done += chunk_in - zs.avail_in;
                out_done += chunk_out - zs.avail_out;
                if (rc != Z_OK && rc != Z_STREAM_END) { inflateEnd(&zs); return "inflate failed for " + name; }
                if (rc == Z_OK && zs.avail_in == chunk_in && zs.avail_out == chunk_out) { inflateEnd(&zs); return "inflate stalled for " + name; }
            }
            inflateEnd(&zs);
            if (out_done != usize) return "inflated size mismatch for " + name;
        } else {
            return "unsupported zip method for " + name;
        }
        const std::string err = parse_npy(raw, out[which]);
        if (!err.empty()) return err + " (" + name + ")";
        found[which] = true;
    }
    return "";
}

}  // namespace dtb
