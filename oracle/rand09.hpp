// TEST INFRASTRUCTURE ONLY -- part of the CPU oracle. Nothing in the product
// path (the CUDA library or its host bindings) includes or links this file.
//
// Restatement of the random streams the reference's tsvdx4 path draws from.
// The reference takes them from third-party crates that are pinned in its
// Cargo.lock but not vendored in the repository:
//   rand        0.9.2  (Cargo.lock:1134-1135)  StdRng, SliceRandom::shuffle
//   rand_chacha 0.9.0  (Cargo.lock:1144-1145)  StdRng's ChaCha12 core
//   rand_core   0.9.3  (Cargo.lock:1160-1161)  SeedableRng::seed_from_u64
//   rand_distr  0.5.1  (Cargo.lock:1169-1170)  Normal<f32>
// Call sites: src/tx.rs:461,606-630 (parameter init), src/lib.rs:486-494
// (per-epoch user shuffle), src/lib.rs:64-67 (rand_array2 -> Normal).
//
// Each piece below is written from the published algorithm it implements:
//  * seed expansion: PCG32 (O'Neill 2014, XSH-RR output) run over the u64
//    seed, one 32-bit output per 4 seed bytes;
//  * ChaCha with 12 rounds (Bernstein 2008), 64-bit block counter starting at
//    0, stream id 0, key = the 32 seed bytes; the generator emits the
//    keystream as consecutive little-endian u32 words and a u64 draw takes two
//    consecutive words, the earlier one as the low half;
//  * standard normal: the 256-layer ziggurat of Marsaglia & Tsang (2000) in
//    Doornik's symmetric form (one u64 per attempt: low 8 bits pick the layer,
//    the top 52 bits a uniform in [-1, 1)), tails by Marsaglia's 1964 method;
//    tables are built here from the published construction;
//  * shuffle: Durstenfeld's forward Fisher-Yates, element i swapping with a
//    uniform index in [0, i], several indices drawn from one u32 by treating
//    it as a mixed-radix number over (i+1)(i+2)...;
//  * bounded u32: Lemire's widening multiply with Canon's one-extra-word
//    correction for the low half.
// The tiny-fixture RMSE tests of the reference (tests/regressors_test.rs:75-93
// and :157-175) pin all of this end to end.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <utility>
#include <vector>

namespace oracle {

inline uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }
inline uint32_t rotr32(uint32_t x, uint32_t r) {
    r &= 31u;
    return r == 0 ? x : (x >> r) | (x << (32 - r));
}

// One ChaCha block: 16 state words in, 16 keystream words out.
inline void chacha_block(const uint32_t in[16], uint32_t out[16], int rounds) {
    uint32_t x[16];
    std::memcpy(x, in, sizeof(x));
    auto qr = [&](int a, int b, int c, int d) {
        x[a] += x[b]; x[d] ^= x[a]; x[d] = rotl32(x[d], 16);
        x[c] += x[d]; x[b] ^= x[c]; x[b] = rotl32(x[b], 12);
        x[a] += x[b]; x[d] ^= x[a]; x[d] = rotl32(x[d], 8);
        x[c] += x[d]; x[b] ^= x[c]; x[b] = rotl32(x[b], 7);
    };
    for (int r = 0; r < rounds; r += 2) {
        qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15);
        qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14);
    }
    for (int i = 0; i < 16; ++i) out[i] = x[i] + in[i];
}

// rand's StdRng: ChaCha12 keyed by the seed, read as a word stream.
class StdRng {
  public:
    static StdRng seed_from_u64(uint64_t state) {
        StdRng g;
        for (int w = 0; w < 8; ++w) {
            state = state * 6364136223846793005ull + 11634580027462260723ull;
            uint32_t xorshifted = (uint32_t)(((state >> 18) ^ state) >> 27);
            uint32_t rot = (uint32_t)(state >> 59);
            g.key_[w] = rotr32(xorshifted, rot);
        }
        return g;
    }
    uint32_t next_u32() {
        if (pos_ >= 16) refill();
        return buf_[pos_++];
    }
    uint64_t next_u64() {
        uint64_t lo = next_u32();
        uint64_t hi = next_u32();
        return lo | (hi << 32);
    }
    // StandardUniform f64: top 53 bits scaled to [0, 1).
    double uniform_f64() { return (double)(next_u64() >> 11) * (1.0 / 9007199254740992.0); }
    // Open01 f64: 52 random mantissa bits in [1, 2), shifted into (0, 1).
    double open01_f64() {
        uint64_t bits = (next_u64() >> 12) | (uint64_t(1023) << 52);
        double v;
        std::memcpy(&v, &bits, 8);
        return v - (1.0 - 1.1102230246251565e-16);
    }
    // Uniform integer in [0, range); range > 0.
    uint32_t below(uint32_t range) {
        uint64_t m = (uint64_t)next_u32() * range;
        uint32_t hi = (uint32_t)(m >> 32), lo = (uint32_t)m;
        if (lo > (uint32_t)(0u - range)) {
            uint32_t hi2 = (uint32_t)(((uint64_t)next_u32() * range) >> 32);
            if ((uint64_t)lo + hi2 > 0xffffffffull) hi += 1;
        }
        return hi;
    }

  private:
    void refill() {
        uint32_t st[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u};
        for (int i = 0; i < 8; ++i) st[4 + i] = key_[i];
        st[12] = (uint32_t)ctr_;
        st[13] = (uint32_t)(ctr_ >> 32);
        st[14] = 0;
        st[15] = 0;
        chacha_block(st, buf_, 12);
        ++ctr_;
        pos_ = 0;
    }
    uint32_t key_[8] = {};
    uint64_t ctr_ = 0;
    uint32_t buf_[16] = {};
    int pos_ = 16;
};

// Ziggurat layer tables for exp(-x^2/2): 256 layers of equal area V, base
// layer including the tail beyond R.
struct ZigguratNormal {
    static constexpr double R = 3.654152885361008796;
    static constexpr double V = 0.00492867323399;
    double x[257];
    double f[257];
    ZigguratNormal() {
        auto pdf = [](double t) { return std::exp(-t * t / 2.0); };
        x[0] = V / pdf(R);
        x[1] = R;
        for (int i = 2; i < 256; ++i) x[i] = std::sqrt(-2.0 * std::log(V / x[i - 1] + pdf(x[i - 1])));
        x[256] = 0.0;
        for (int i = 0; i < 257; ++i) f[i] = pdf(x[i]);
    }
    static const ZigguratNormal& get() {
        static const ZigguratNormal t;
        return t;
    }
};

inline double standard_normal_f64(StdRng& rng) {
    const ZigguratNormal& z = ZigguratNormal::get();
    for (;;) {
        uint64_t bits = rng.next_u64();
        int i = (int)(bits & 0xff);
        uint64_t mbits = (bits >> 12) | (uint64_t(1024) << 52);  // [2, 4)
        double u;
        std::memcpy(&u, &mbits, 8);
        u -= 3.0;  // [-1, 1)
        double xv = u * z.x[i];
        if (std::fabs(xv) < z.x[i + 1]) return xv;
        if (i == 0) {
            // Tail beyond R (Marsaglia 1964).
            double tx = 1.0, ty = 0.0;
            while (-2.0 * ty < tx * tx) {
                double a = rng.open01_f64();
                double b = rng.open01_f64();
                tx = std::log(a) / ZigguratNormal::R;
                ty = std::log(b);
            }
            return u < 0.0 ? tx - ZigguratNormal::R : ZigguratNormal::R - tx;
        }
        if (z.f[i + 1] + (z.f[i] - z.f[i + 1]) * rng.uniform_f64() < std::exp(-xv * xv / 2.0)) return xv;
    }
}

// Normal(0, sigma) in f32: an f64 standard normal rounded to f32, scaled.
inline float normal_f32(StdRng& rng, float sigma) {
    float z = (float)standard_normal_f64(rng);
    return 0.0f + sigma * z;
}

// Largest product m(m+1)...(m+c-1) that fits in u32, and its length c.
inline std::pair<uint32_t, uint32_t> dice_bound(uint32_t m) {
    uint64_t prod = m;
    uint32_t cur = m + 1;
    while (prod * cur <= 0xffffffffull) {
        prod *= cur;
        ++cur;
    }
    return {(uint32_t)prod, cur - m};
}

template <class T>
void shuffle(std::vector<T>& v, StdRng& rng) {
    if (v.size() <= 1) return;
    uint32_t n = 0, chunk = 0, left = 1;  // the first index is always 0
    for (size_t i = 0; i < v.size(); ++i) {
        uint32_t next_n = n + 1;
        uint32_t next_left;
        if (left == 0) {
            auto bc = dice_bound(next_n);
            chunk = rng.below(bc.first);
            next_left = bc.second - 1;
        } else {
            next_left = left - 1;
        }
        uint32_t idx;
        if (next_left == 0) {
            idx = chunk;
        } else {
            idx = chunk % next_n;
            chunk /= next_n;
        }
        left = next_left;
        n = next_n;
        std::swap(v[i], v[idx]);
    }
}

}  // namespace oracle
