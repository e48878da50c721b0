// Seeded synthetic searches for the batched-search microbenchmark: random per-(layer, cell) costs 1-16, about
// 15 % of cells blocked in clustered value-noise blobs, a uniform via cost, one free source and one free target.
// Everything is a pure function of a 64-bit seed through an integer hash, so pcbroute_b200/synth.py regenerates
// the same arrays bit for bit on the host.
#include <algorithm>
#include <cstdint>
#include <thread>
#include <vector>

#include "pcbg_internal.h"

namespace pcbg {
namespace {

__host__ __device__ inline uint64_t mix64(uint64_t z) {
    z ^= z >> 30;
    z *= 0xBF58476D1CE4E5B9ull;
    z ^= z >> 27;
    z *= 0x94D049BB133111EBull;
    z ^= z >> 31;
    return z;
}

__host__ __device__ inline uint64_t hash4(uint64_t seed, uint64_t tag, uint64_t a, uint64_t b) {
    uint64_t x = mix64(seed ^ (tag * 0xD1B54A32D192ED03ull));
    x = mix64(x + a);
    return mix64(x + b);
}

// one octave of value noise at lattice spacing 2^sh, scaled to [0, 255 * 256]
__host__ __device__ inline int64_t octave(uint64_t seed, uint64_t tag, int l, int i, int j, int sh) {
    const int S = 1 << sh, ax = i >> sh, fx = i & (S - 1), by = j >> sh, fy = j & (S - 1);
    auto v = [&](int a, int b) -> int64_t {
        return int64_t(hash4(seed, tag, (uint64_t(l) << 32) | uint64_t(a), uint64_t(b)) >> 56);
    };
    const int64_t v00 = v(ax, by), v10 = v(ax + 1, by), v01 = v(ax, by + 1), v11 = v(ax + 1, by + 1);
    return ((v00 * (S - fx) + v10 * fx) * (S - fy) + (v01 * (S - fx) + v11 * fx) * fy) << (2 * (4 - sh));
}

constexpr int64_t BLOCK_T = 128000;  // about the 85th percentile of 2 * octave(16) + octave(4)

__host__ __device__ inline bool blocked(uint64_t seed, int l, int i, int j) {
    return 2 * octave(seed, 2, l, i, j, 4) + octave(seed, 3, l, i, j, 2) >= BLOCK_T;
}

__global__ void synth_kernel(uint64_t seed, int rw, int rh, int nl, int pitch, int hpad, float via, float* cf, uint8_t* fl,
                             float* vcf) {
    const size_t plane = size_t(hpad) * pitch, total = plane * nl;
    for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < total; q += size_t(gridDim.x) * blockDim.x) {
        const int l = int(q / plane);
        const size_t rem = q % plane;
        const int j = int(rem / pitch), i = int(rem % pitch);
        if (j >= rh || i >= rw) {
            cf[q] = 1e30f;
            fl[q] = 0;
            if (l == 0 && vcf) vcf[rem] = 1e30f;
            continue;
        }
        const bool b = blocked(seed, l, i, j);
        const uint64_t h = hash4(seed, 1, uint64_t(l), uint64_t(j) * rw + i);
        cf[q] = b ? 1e30f : float(1 + int((h >> 32) % 16));
        fl[q] = b ? 0 : 1;
        if (l == 0 && vcf) vcf[rem] = via;
    }
}

__global__ void pick_kernel(uint64_t seed, int rw, int rh, int nl, int pitch, int hpad, uint8_t* fl, int64_t* st) {
    const uint64_t N = uint64_t(rw) * rh * nl, RN = uint64_t(rw) * rh;
    int64_t src = -1, tgt = -1;
    for (int k = 0; k < 64 && src < 0; ++k) {
        const uint64_t c = hash4(seed, 4, uint64_t(k), 0) % N;
        const int l = int(c / RN), j = int((c % RN) / rw), i = int(c % rw);
        if (!blocked(seed, l, i, j)) src = int64_t(c);
    }
    for (int k = 0; k < 64 && tgt < 0; ++k) {
        const uint64_t c = hash4(seed, 5, uint64_t(k), 0) % N;
        const int l = int(c / RN), j = int((c % RN) / rw), i = int(c % rw);
        if (!blocked(seed, l, i, j) && int64_t(c) != src) tgt = int64_t(c);
    }
    if (tgt >= 0) {
        const int l = int(tgt / int64_t(RN)), j = int((tgt % int64_t(RN)) / rw), i = int(tgt % rw);
        fl[(size_t(l) * hpad + j) * pitch + i] |= 2;
    }
    st[0] = src;
    st[1] = tgt;
}

}  // namespace
}  // namespace pcbg

extern "C" int pcbg_synth_search_host(uint64_t seed, int32_t rw, int32_t rh, int32_t nl, float via, float* cf,
                                      uint8_t* flags, float* vcf, int64_t* src_tgt, int32_t threads) {
    using namespace pcbg;
    if (nl < 1 || nl > MAX_LAYERS || rw < 1 || rh < 1) return PCBG_ERR_FAIL;
    const size_t RN = size_t(rw) * rh;
    auto rows = [&](int t, int nt) {
        for (int row = t; row < rh * nl; row += nt) {
            const int l = row / rh, j = row % rh;
            for (int i = 0; i < rw; ++i) {
                const size_t q = size_t(l) * RN + size_t(j) * rw + i;
                const bool b = blocked(seed, l, i, j);
                const uint64_t h = hash4(seed, 1, uint64_t(l), uint64_t(j) * rw + i);
                cf[q] = b ? 1e30f : float(1 + int((h >> 32) % 16));
                flags[q] = b ? 0 : 1;
                if (l == 0 && vcf) vcf[size_t(j) * rw + i] = via;
            }
        }
    };
    const int nt = std::max(1, std::min(threads, rh * nl));
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(rows, t, nt);
    rows(0, nt);
    for (auto& x : th) x.join();
    const uint64_t N = RN * nl;
    int64_t src = -1, tgt = -1;
    for (int k = 0; k < 64 && src < 0; ++k) {
        const uint64_t c = hash4(seed, 4, uint64_t(k), 0) % N;
        if (!blocked(seed, int(c / RN), int(c % rw), int((c % RN) / rw))) src = int64_t(c);
    }
    for (int k = 0; k < 64 && tgt < 0; ++k) {
        const uint64_t c = hash4(seed, 5, uint64_t(k), 0) % N;
        if (!blocked(seed, int(c / RN), int(c % rw), int((c % RN) / rw)) && int64_t(c) != src) tgt = int64_t(c);
    }
    if (tgt >= 0) flags[tgt] |= 2;
    src_tgt[0] = src;
    src_tgt[1] = tgt;
    return 0;
}

extern "C" int pcbg_synth_search(uint64_t seed, int32_t rw, int32_t rh, int32_t nl, int32_t pitch, int32_t hpad, float via,
                                 float* cf, uint8_t* flags, float* vcf, int64_t* src_tgt, void* stream) {
    if (nl < 1 || nl > pcbg::MAX_LAYERS || rw < 1 || rh < 1 || pitch < rw || hpad < rh) return PCBG_ERR_FAIL;
    cudaStream_t S = static_cast<cudaStream_t>(stream);
    const size_t total = size_t(hpad) * pitch * nl;
    const unsigned blocks = unsigned(std::min<size_t>((total + 255) / 256, 148 * 32));
    pcbg::synth_kernel<<<blocks, 256, 0, S>>>(seed, rw, rh, nl, pitch, hpad, via, cf, flags, vcf);
    pcbg::pick_kernel<<<1, 1, 0, S>>>(seed, rw, rh, nl, pitch, hpad, flags, src_tgt);
    return cudaGetLastError() == cudaSuccess ? 0 : PCBG_ERR_FAIL;
}
