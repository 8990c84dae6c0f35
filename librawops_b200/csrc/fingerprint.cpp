// Source ingest: the canonical content fingerprint of a RAW or raster source
// (SourceFingerprint.cpp:65-101) and a RAW upload overlapped with it.
//
// The fingerprint is SHA-256 (FIPS 180-4, restated below) over the
// reference's byte stream: a version tag with its terminating NUL, the
// metadata little-endian (width, height as u32; pattern and CFA phases as u8;
// the active area as four u32; the four black then four white levels as u16),
// then the active area's samples row by row, little-endian u16.  A raster
// source hashes its own tag, width, height, working space and every float's
// bits.  SHA-256 is one serial chain of compressions, so it runs on a host
// core; re_image_create_fingerprinted streams the sensor plane to the device
// through two pinned staging buffers while that core hashes the same rows, so
// the upload costs no time beyond the hash.
#include <algorithm>
#include <array>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "rawengine_b200.h"

namespace re {
void set_last_error(const std::string& msg);
re_status image_adopt_device(re_raw_metadata* meta, uint16_t* device_samples, size_t count, re_image** out);
}  // namespace re

namespace {

// ---------------------------------------------------------------- SHA-256

// FIPS 180-4 section 4.2.2: the first 32 bits of the fractional parts of the
// cube roots of the first 64 primes.
constexpr uint32_t kK[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};

class Sha256 {
public:
    void update(const void* data, size_t n) {
        const auto* p = static_cast<const uint8_t*>(data);
        bytes_ += n;
        if (fill_) {
            const size_t take = std::min(n, 64 - fill_);
            std::memcpy(block_ + fill_, p, take);
            fill_ += take;
            p += take;
            n -= take;
            if (fill_ == 64) {
                compress(block_);
                fill_ = 0;
            }
        }
        for (; n >= 64; p += 64, n -= 64) compress(p);
        if (n) {
            std::memcpy(block_, p, n);
            fill_ = n;
        }
    }
    std::array<uint8_t, 32> finish() {
        const uint64_t bits = bytes_ * 8;
        const uint8_t one = 0x80, zero = 0;
        update(&one, 1);
        while (fill_ != 56) update(&zero, 1);
        uint8_t len[8];
        for (int i = 0; i < 8; ++i) len[i] = (uint8_t)(bits >> (56 - 8 * i));
        update(len, 8);
        std::array<uint8_t, 32> out{};
        for (int i = 0; i < 8; ++i)
            for (int b = 0; b < 4; ++b) out[4 * i + b] = (uint8_t)(h_[i] >> (24 - 8 * b));
        return out;
    }

private:
    static uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
    void compress(const uint8_t* m) {
        uint32_t w[64];
        for (int t = 0; t < 16; ++t)
            w[t] = (uint32_t)m[4 * t] << 24 | (uint32_t)m[4 * t + 1] << 16 | (uint32_t)m[4 * t + 2] << 8 | m[4 * t + 3];
        for (int t = 16; t < 64; ++t) {
            const uint32_t s0 = rotr(w[t - 15], 7) ^ rotr(w[t - 15], 18) ^ (w[t - 15] >> 3);
            const uint32_t s1 = rotr(w[t - 2], 17) ^ rotr(w[t - 2], 19) ^ (w[t - 2] >> 10);
            w[t] = w[t - 16] + s0 + w[t - 7] + s1;
        }
        uint32_t a = h_[0], b = h_[1], c = h_[2], d = h_[3], e = h_[4], f = h_[5], g = h_[6], h = h_[7];
        for (int t = 0; t < 64; ++t) {
            const uint32_t t1 = h + (rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25)) + ((e & f) ^ (~e & g)) + kK[t] + w[t];
            const uint32_t t2 = (rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
            h = g;
            g = f;
            f = e;
            e = d + t1;
            d = c;
            c = b;
            b = a;
            a = t1 + t2;
        }
        h_[0] += a; h_[1] += b; h_[2] += c; h_[3] += d;
        h_[4] += e; h_[5] += f; h_[6] += g; h_[7] += h;
    }
    // FIPS 180-4 section 5.3.3: the first 32 bits of the fractional parts of
    // the square roots of the first 8 primes.
    uint32_t h_[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a, 0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
    uint8_t block_[64];
    size_t fill_ = 0;
    uint64_t bytes_ = 0;
};

void u8(Sha256& h, uint8_t v) { h.update(&v, 1); }
void u16(Sha256& h, uint16_t v) {
    const uint8_t b[2] = {(uint8_t)v, (uint8_t)(v >> 8)};
    h.update(b, 2);
}
void u32(Sha256& h, uint32_t v) {
    const uint8_t b[4] = {(uint8_t)v, (uint8_t)(v >> 8), (uint8_t)(v >> 16), (uint8_t)(v >> 24)};
    h.update(b, 4);
}
void tag(Sha256& h, const char* name) { h.update(name, std::strlen(name) + 1); }

// Little-endian u16 samples (the host is little-endian: the bytes are hashed as they lie).
void u16_row(Sha256& h, const uint16_t* s, size_t n) {
    static_assert(sizeof(uint16_t) == 2, "u16");
    const uint16_t probe = 1;
    if (*reinterpret_cast<const uint8_t*>(&probe) == 1) {
        h.update(s, n * 2);
        return;
    }
    for (size_t i = 0; i < n; ++i) u16(h, s[i]);
}

void raw_header(Sha256& h, const re_raw_metadata& m) {
    tag(h, "librawops.source.raw.u16.v1");
    u32(h, m.width);
    u32(h, m.height);
    u8(h, (uint8_t)m.pattern);
    u8(h, (uint8_t)m.cfa_phase_x);
    u8(h, (uint8_t)m.cfa_phase_y);
    u32(h, m.active_area.x);
    u32(h, m.active_area.y);
    u32(h, m.active_area.width);
    u32(h, m.active_area.height);
    for (int i = 0; i < 4; ++i) u16(h, m.black_levels[i]);
    for (int i = 0; i < 4; ++i) u16(h, m.white_levels[i]);
}

re_status fp_fail(re_status s, const std::string& msg) {
    re::set_last_error(msg);
    return s;
}

}  // namespace

extern "C" {

// SourceFingerprint.cpp:65-84 (metadata normalized and validated first, as RawImage does).
re_status re_fingerprint_raw(re_raw_metadata* meta, const uint16_t* samples, size_t count, uint8_t digest[32]) {
    if (!meta || !digest || (!samples && count)) return fp_fail(RE_INVALID_ARGUMENT, "null fingerprint arguments");
    re_status s = re_raw_metadata_normalize(meta, count);
    if (s) return s;
    Sha256 h;
    raw_header(h, *meta);
    const re_rect a = meta->active_area;
    for (uint32_t y = a.y; y < a.y + a.height; ++y)
        u16_row(h, samples + (size_t)y * meta->row_stride_samples + a.x, a.width);
    const auto d = h.finish();
    std::memcpy(digest, d.data(), 32);
    return RE_OK;
}

// SourceFingerprint.cpp:86-101
re_status re_fingerprint_raster(uint32_t width, uint32_t height, size_t row_stride_pixels, uint32_t working_space,
                                const float* pixels, uint8_t digest[32]) {
    if (!width || !height || working_space > 1 || !pixels || !digest)
        return fp_fail(RE_INVALID_ARGUMENT, "invalid raster fingerprint arguments");
    if (!row_stride_pixels) row_stride_pixels = width;
    if (row_stride_pixels < width) return fp_fail(RE_INVALID_ARGUMENT, "raster row stride is below its width");
    Sha256 h;
    tag(h, "librawops.source.raster.f32.v1");
    u32(h, width);
    u32(h, height);
    u8(h, (uint8_t)working_space);
    for (uint32_t y = 0; y < height; ++y) {
        const float* row = pixels + (size_t)y * row_stride_pixels * 3;
        for (size_t i = 0; i < (size_t)width * 3; ++i) {
            uint32_t bits;
            std::memcpy(&bits, row + i, 4);
            u32(h, bits);
        }
    }
    const auto d = h.finish();
    std::memcpy(digest, d.data(), 32);
    return RE_OK;
}

// re_image_create with the upload overlapped with the fingerprint: rows are
// staged into two pinned buffers and copied asynchronously while the same
// rows are hashed.
re_status re_image_create_fingerprinted(re_raw_metadata* meta, const uint16_t* samples, size_t count,
                                        re_image** out, uint8_t digest[32]) {
    if (!meta || !out || !digest || (!samples && count))
        return fp_fail(RE_INVALID_ARGUMENT, "null image arguments");
    re_status s = re_raw_metadata_normalize(meta, count);
    if (s) return s;
    const size_t stride = meta->row_stride_samples;
    constexpr size_t kChunkBytes = 8u << 20;
    const size_t rows_per_chunk = std::max<size_t>(1, kChunkBytes / (stride * 2));
    uint16_t* dev = nullptr;
    uint16_t* pinned[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    cudaStream_t stream = nullptr;
    auto cleanup = [&]() {
        if (stream) cudaStreamSynchronize(stream);
        for (int i = 0; i < 2; ++i) {
            if (done[i]) cudaEventDestroy(done[i]);
            if (pinned[i]) cudaFreeHost(pinned[i]);
        }
        if (stream) cudaStreamDestroy(stream);
    };
    auto cuda_err = [&](cudaError_t e, const char* where) {
        cleanup();
        if (dev) cudaFree(dev);
        return fp_fail(RE_CUDA_ERROR, std::string(where) + ": " + cudaGetErrorString(e));
    };
    cudaError_t e = cudaMalloc(&dev, count * sizeof(uint16_t));
    if (e != cudaSuccess) return cuda_err(e, "image upload");
    e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_err(e, "image upload");
    for (int i = 0; i < 2; ++i) {
        if ((e = cudaMallocHost(&pinned[i], rows_per_chunk * stride * 2)) != cudaSuccess) return cuda_err(e, "image upload");
        if ((e = cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming)) != cudaSuccess)
            return cuda_err(e, "image upload");
    }
    Sha256 h;
    raw_header(h, *meta);
    const re_rect a = meta->active_area;
    int k = 0;
    for (size_t y0 = 0; y0 < meta->height; y0 += rows_per_chunk, k ^= 1) {
        const size_t rows = std::min<size_t>(rows_per_chunk, meta->height - y0);
        if ((e = cudaEventSynchronize(done[k])) != cudaSuccess) return cuda_err(e, "image upload");
        std::memcpy(pinned[k], samples + y0 * stride, rows * stride * 2);
        e = cudaMemcpyAsync(dev + y0 * stride, pinned[k], rows * stride * 2, cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = cudaEventRecord(done[k], stream);
        if (e != cudaSuccess) return cuda_err(e, "image upload");
        for (size_t y = std::max<size_t>(y0, a.y); y < std::min<size_t>(y0 + rows, (size_t)a.y + a.height); ++y)
            u16_row(h, samples + y * stride + a.x, a.width);
    }
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return cuda_err(e, "image upload");
    cleanup();
    const auto d = h.finish();
    std::memcpy(digest, d.data(), 32);
    s = re::image_adopt_device(meta, dev, count, out);
    if (s) cudaFree(dev);
    return s;
}

}  // extern "C"
