// EM-format volume I/O on the host (IOfun/tom_emread.m:153-176,
// IOfun/tom_emwrite.m:94-150): a 512-byte header — magic[4] (byte 0: 6 = PC
// little endian, 0/3/5 = big endian; byte 3: data type 1 byte, 2 int16, 4 int32,
// 5 float, 9 double), int32 dims[3], char comment[80], int32 parameter[40],
// char fill[256] — followed by the data, x fastest.  Reads convert to float
// (the matching path's type); writes produce PC-order float files.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.h"

namespace {

bool big_endian_file(unsigned char m0) { return m0 == 0 || m0 == 3 || m0 == 5; }

template <typename T> T swap_bytes(T v) {
    unsigned char b[sizeof(T)];
    std::memcpy(b, &v, sizeof(T));
    for (size_t i = 0; i < sizeof(T) / 2; ++i) std::swap(b[i], b[sizeof(T) - 1 - i]);
    std::memcpy(&v, b, sizeof(T));
    return v;
}

struct EmHeader {
    unsigned char magic[4];
    int32_t dims[3];
};

int read_header(FILE* f, EmHeader* h, bool* be) {
    unsigned char raw[512];
    if (std::fread(raw, 1, 512, f) != 512) return TOMGPU_ERR_ARG;
    std::memcpy(h->magic, raw, 4);
    *be = big_endian_file(h->magic[0]);
    for (int d = 0; d < 3; ++d) {
        int32_t v;
        std::memcpy(&v, raw + 4 + 4 * d, 4);
        h->dims[d] = *be ? swap_bytes(v) : v;
    }
    return TOMGPU_OK;
}

size_t type_size(unsigned char t) {
    switch (t) {
        case 1: return 1;
        case 2: return 2;
        case 4: return 4;
        case 5: return 4;
        case 9: return 8;
        default: return 0;
    }
}

}  // namespace

extern "C" {

int tomgpu_em_read(const char* path, int dims[3], float* out, size_t capacity) {
    using tg::fail;
    if (!path || !dims) return fail(nullptr, TOMGPU_ERR_ARG, "null path or dims");
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(nullptr, TOMGPU_ERR_ARG, std::string("cannot open ") + path);
    EmHeader h;
    bool be = false;
    int rc = read_header(f, &h, &be);
    if (rc) {
        std::fclose(f);
        return fail(nullptr, rc, std::string("short EM header in ") + path);
    }
    for (int d = 0; d < 3; ++d) dims[d] = h.dims[d];
    const size_t ts = type_size(h.magic[3]);
    if (!ts || h.dims[0] <= 0 || h.dims[1] <= 0 || h.dims[2] <= 0) {
        std::fclose(f);
        return fail(nullptr, TOMGPU_ERR_UNSUPPORTED, "unsupported EM data type or size");
    }
    const size_t n = (size_t)h.dims[0] * h.dims[1] * h.dims[2];
    if (!out) {  // size query
        std::fclose(f);
        return TOMGPU_OK;
    }
    if (capacity < n) {
        std::fclose(f);
        return fail(nullptr, TOMGPU_ERR_ARG, "output buffer smaller than the volume");
    }
    std::vector<unsigned char> buf(1 << 22);
    size_t done = 0;
    while (done < n) {
        const size_t chunk = std::min(n - done, buf.size() / ts);
        if (std::fread(buf.data(), ts, chunk, f) != chunk) {
            std::fclose(f);
            return fail(nullptr, TOMGPU_ERR_ARG, "EM data shorter than its header says");
        }
        for (size_t i = 0; i < chunk; ++i) {
            const unsigned char* p = buf.data() + i * ts;
            float v = 0;
            switch (h.magic[3]) {
                case 1: v = (float)*p; break;  // MATLAB 'char': unsigned byte
                case 2: { int16_t x; std::memcpy(&x, p, 2); v = (float)(be ? swap_bytes(x) : x); break; }
                case 4: { int32_t x; std::memcpy(&x, p, 4); v = (float)(be ? swap_bytes(x) : x); break; }
                case 5: { float x; std::memcpy(&x, p, 4); v = be ? swap_bytes(x) : x; break; }
                case 9: { double x; std::memcpy(&x, p, 8); v = (float)(be ? swap_bytes(x) : x); break; }
            }
            out[done + i] = v;
        }
        done += chunk;
    }
    std::fclose(f);
    return TOMGPU_OK;
}

int tomgpu_em_write(const char* path, const float* data, const int dims[3], const char* comment) {
    using tg::fail;
    if (!path || !data || !dims || dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0)
        return fail(nullptr, TOMGPU_ERR_ARG, "null pointer or bad dims");
    unsigned char hdr[512];
    std::memset(hdr, 0, sizeof hdr);
    hdr[0] = 6;  // PC, little endian
    hdr[1] = 0;
    hdr[2] = 0;
    hdr[3] = 5;  // float
    for (int d = 0; d < 3; ++d) {
        const int32_t v = dims[d];
        std::memcpy(hdr + 4 + 4 * d, &v, 4);
    }
    if (comment) std::strncpy(reinterpret_cast<char*>(hdr + 16), comment, 80);
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(nullptr, TOMGPU_ERR_ARG, std::string("cannot create ") + path);
    const size_t n = (size_t)dims[0] * dims[1] * dims[2];
    const bool ok = std::fwrite(hdr, 1, 512, f) == 512 && std::fwrite(data, sizeof(float), n, f) == n;
    const bool closed = std::fclose(f) == 0;
    if (!ok || !closed) return fail(nullptr, TOMGPU_ERR_ARG, std::string("write failed: ") + path);
    return TOMGPU_OK;
}

}  // extern "C"
