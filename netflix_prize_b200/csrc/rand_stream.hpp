// Seeded host-side random streams that reproduce the reference's parameter
// init (src/tx.rs:461,606-630 via rand_array2, src/lib.rs:64-67) and per-epoch
// user shuffle (get_users, src/lib.rs:486-494), so a model created from a
// seed starts from the reference's exact initial state and visits users in
// the reference's order.
//
// The reference draws these from crates pinned in its Cargo.lock: rand 0.9.2
// (StdRng = ChaCha12, SliceRandom::shuffle), rand_core 0.9.3
// (seed_from_u64), rand_distr 0.5.1 (Normal). What is implemented here is the
// published algorithm behind each:
//  - seed expansion: PCG32 (XSH-RR) stepped over the u64 seed, one 32-bit
//    output per key word;
//  - keystream: ChaCha (Bernstein) with 12 rounds, 64-bit block counter from
//    0, zero nonce; generated four blocks at a time; consumed as a stream of
//    little-endian u32 words, a u64 being two consecutive words (low first);
//  - Normal(0, s) in f32: s * f32(z), z an f64 standard normal from the
//    Marsaglia-Tsang 256-layer ziggurat (symmetric form: one u64 per try,
//    low byte = layer, top 52 bits = uniform in [-1, 1); wedge test with an
//    extra 53-bit uniform; tail by Marsaglia's exponential method with two
//    open-interval uniforms);
//  - shuffle: forward Fisher-Yates (position i swaps with uniform [0, i]),
//    drawing several positions from one u32 as digits of a mixed-radix
//    number (i+1)(i+2)..., each u32 bounded with a widening multiply plus one
//    extra word for the low-half correction (Canon's method).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace tsvd {

class ChaCha12Stream {
  public:
    explicit ChaCha12Stream(uint64_t seed) {
        uint64_t s = seed;
        for (int w = 0; w < 8; ++w) {
            s = s * 6364136223846793005ull + 11634580027462260723ull;
            uint32_t x = (uint32_t)(((s >> 18) ^ s) >> 27);
            uint32_t r = (uint32_t)(s >> 59) & 31u;
            key_[w] = r ? (x >> r) | (x << (32 - r)) : x;
        }
    }
    inline uint32_t u32() {
        if (at_ == kWords) generate();
        return words_[at_++];
    }
    inline uint64_t u64() {
        uint64_t lo = u32();
        return lo | ((uint64_t)u32() << 32);
    }
    // The 256-bit ChaCha key the seed expands to (for device-side generation
    // of the same keystream).
    const uint32_t* key() const { return key_; }

  private:
    static constexpr int kBlocks = 4, kWords = 16 * kBlocks;
    static inline uint32_t rl(uint32_t v, int n) { return (v << n) | (v >> (32 - n)); }
    void generate() {
        for (int b = 0; b < kBlocks; ++b) {
            uint32_t init[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u,
                                 key_[0], key_[1], key_[2], key_[3], key_[4], key_[5], key_[6], key_[7],
                                 (uint32_t)block_, (uint32_t)(block_ >> 32), 0u, 0u};
            uint32_t s[16];
            std::memcpy(s, init, sizeof(s));
#define TSVD_QR(a, b2, c, d)                     \
    s[a] += s[b2]; s[d] = rl(s[d] ^ s[a], 16);    \
    s[c] += s[d];  s[b2] = rl(s[b2] ^ s[c], 12);  \
    s[a] += s[b2]; s[d] = rl(s[d] ^ s[a], 8);     \
    s[c] += s[d];  s[b2] = rl(s[b2] ^ s[c], 7);
            for (int round = 0; round < 6; ++round) {
                TSVD_QR(0, 4, 8, 12) TSVD_QR(1, 5, 9, 13) TSVD_QR(2, 6, 10, 14) TSVD_QR(3, 7, 11, 15)
                TSVD_QR(0, 5, 10, 15) TSVD_QR(1, 6, 11, 12) TSVD_QR(2, 7, 8, 13) TSVD_QR(3, 4, 9, 14)
            }
#undef TSVD_QR
            for (int k = 0; k < 16; ++k) words_[16 * b + k] = s[k] + init[k];
            ++block_;
        }
        at_ = 0;
    }
    uint32_t key_[8];
    uint64_t block_ = 0;
    uint32_t words_[kWords];
    int at_ = kWords;
};

struct ZigTables {
    double x[257], f[257];
    static constexpr double kR = 3.654152885361008796;
    static constexpr double kV = 0.00492867323399;
    ZigTables() {
        x[0] = kV / std::exp(-kR * kR / 2.0);
        x[1] = kR;
        for (int k = 2; k < 256; ++k)
            x[k] = std::sqrt(-2.0 * std::log(kV / x[k - 1] + std::exp(-x[k - 1] * x[k - 1] / 2.0)));
        x[256] = 0.0;
        for (int k = 0; k < 257; ++k) f[k] = std::exp(-x[k] * x[k] / 2.0);
    }
};

inline const ZigTables& zig() {
    static const ZigTables t;
    return t;
}

inline double bits_to_unit(uint64_t mantissa52, int exponent) {
    uint64_t b = mantissa52 | ((uint64_t)(1023 + exponent) << 52);
    double d;
    std::memcpy(&d, &b, 8);
    return d;
}

inline double std_normal(ChaCha12Stream& g) {
    const ZigTables& t = zig();
    while (true) {
        const uint64_t w = g.u64();
        const int layer = (int)(w & 0xff);
        const double u = bits_to_unit(w >> 12, 1) - 3.0;
        const double x = u * t.x[layer];
        if (std::fabs(x) < t.x[layer + 1]) return x;
        if (layer == 0) {
            double a = 1.0, b = 0.0;
            do {
                a = std::log(bits_to_unit(g.u64() >> 12, 0) - (1.0 - 1.1102230246251565e-16)) / ZigTables::kR;
                b = std::log(bits_to_unit(g.u64() >> 12, 0) - (1.0 - 1.1102230246251565e-16));
            } while (-2.0 * b < a * a);
            return u < 0.0 ? a - ZigTables::kR : ZigTables::kR - a;
        }
        const double v = (double)(g.u64() >> 11) * (1.0 / 9007199254740992.0);
        if (t.f[layer + 1] + (t.f[layer] - t.f[layer + 1]) * v < std::exp(-x * x / 2.0)) return x;
    }
}

// rand_array2(rows, cols, rng, sigma) in row-major order into a padded
// destination (row stride `stride` floats; padding left untouched).
inline void fill_normal_rows(ChaCha12Stream& g, float sigma, size_t rows, size_t cols, float* dst, size_t stride) {
    for (size_t r = 0; r < rows; ++r) {
        float* row = dst + r * stride;
        for (size_t c = 0; c < cols; ++c) {
            float z = (float)std_normal(g);
            row[c] = 0.0f + sigma * z;
        }
    }
}

inline uint32_t bounded_u32(ChaCha12Stream& g, uint32_t range) {
    const uint64_t m = (uint64_t)g.u32() * range;
    uint32_t hi = (uint32_t)(m >> 32);
    const uint32_t lo = (uint32_t)m;
    if (lo > 0u - range) {
        const uint32_t extra = (uint32_t)(((uint64_t)g.u32() * range) >> 32);
        hi += ((uint64_t)lo + extra) >> 32 ? 1u : 0u;
    }
    return hi;
}

// get_users(n, shuffle, seed, epoch)
inline std::vector<uint32_t> user_order(size_t n, bool shuffle, uint64_t seed, uint64_t epoch) {
    std::vector<uint32_t> v(n);
    for (size_t k = 0; k < n; ++k) v[k] = (uint32_t)k;
    if (!shuffle || n <= 1) return v;
    ChaCha12Stream g(seed ^ (epoch * 0x9E3779B97F4A7C15ull));
    uint32_t digits = 0, left = 1, radix = 0;
    for (size_t i = 0; i < n; ++i) {
        const uint32_t next = radix + 1;
        if (left == 0) {
            uint64_t prod = next;
            uint32_t k = next + 1;
            while (prod * k <= 0xffffffffull) prod *= k++;
            digits = bounded_u32(g, (uint32_t)prod);
            left = k - next;
        }
        --left;
        uint32_t j;
        if (left == 0) {
            j = digits;
        } else {
            j = digits % next;
            digits /= next;
        }
        radix = next;
        std::swap(v[i], v[j]);
    }
    return v;
}

}  // namespace tsvd
