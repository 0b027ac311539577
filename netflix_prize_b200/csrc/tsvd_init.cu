// Seeded parameter init on the device: the same values that
// fill_normal_rows (rand_stream.hpp) draws on the host for
// rand_array2 (src/lib.rs:64-67) as TxModel::new calls it
// (src/tx.rs:606-630): one ChaCha12 stream, standard normals from the
// 256-layer ziggurat, table after table, row-major.
//
// Word q of the stream (a u64) is u32 words 2q and 2q+1 of the keystream,
// i.e. words of ChaCha block q / 8. A draw that starts at word q reads one
// word when the ziggurat accepts on its first test (about 99% of draws) and
// two or more otherwise, so the words that start draws form a chain. The
// length a draw would have if it started at q depends on the stream alone, so
// it is computed for every word at once (k_sample_lengths). The host then
// walks only the words whose length exceeds one, in stream order, and marks
// the words that such a draw swallows; every other word starts a draw. A scan
// over 8-word blocks numbers the starts, and k_write_tables writes
// sigma * f32(z) for draw k into the table slot k maps to.
//
// Arithmetic mirrors the host draw operation for operation (explicit _rn
// intrinsics where a fused multiply-add would change a rounding). exp and
// log are the device's; they differ from the host's by at most an ulp or
// two, which can change a wedge or tail comparison only when the compared
// values agree to that ulp.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

#include <algorithm>
#include <vector>

#include "rand_stream.hpp"
#include "tsvd_model.hpp"

namespace tsvd {
namespace {

constexpr unsigned kInitBlock = 256;
constexpr unsigned kInitGrid = 148 * 16;
constexpr uint32_t kMaxWordsPerDraw = 255;  // lengths are stored in one byte
constexpr uint64_t kMaxSegmentWords = 1ull << 30;
constexpr double kZigR = ZigTables::kR;
constexpr int kMaxTables = 5;

struct Key {
    uint32_t k[8];
};

struct Tables {
    float* dst[kMaxTables];
    uint64_t start[kMaxTables + 1];  // first draw number of each table; start[n] = total
    uint64_t rows[kMaxTables];
    uint32_t cols[kMaxTables], stride[kMaxTables];
    float sigma[kMaxTables];
    int n;
};

__device__ __forceinline__ uint32_t rotl32(uint32_t v, int n) { return __funnelshift_l(v, v, n); }

__device__ __forceinline__ void chacha12_block(const Key& key, uint64_t blk, uint32_t out[16]) {
    const uint32_t init[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key.k[0], key.k[1],
                               key.k[2],    key.k[3],    key.k[4],    key.k[5],    key.k[6], key.k[7],
                               (uint32_t)blk, (uint32_t)(blk >> 32), 0u, 0u};
    uint32_t x[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = init[i];
#define TSVD_DQR(a, b, c, d)                      \
    x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 16); \
    x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 12); \
    x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 8);  \
    x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 7);
#pragma unroll
    for (int r = 0; r < 6; ++r) {
        TSVD_DQR(0, 4, 8, 12) TSVD_DQR(1, 5, 9, 13) TSVD_DQR(2, 6, 10, 14) TSVD_DQR(3, 7, 11, 15)
        TSVD_DQR(0, 5, 10, 15) TSVD_DQR(1, 6, 11, 12) TSVD_DQR(2, 7, 8, 13) TSVD_DQR(3, 4, 9, 14)
    }
#undef TSVD_DQR
#pragma unroll
    for (int i = 0; i < 16; ++i) out[i] = x[i] + init[i];
}

__device__ __forceinline__ double unit_bits(uint64_t mantissa52, int exponent) {
    return __longlong_as_double((long long)(mantissa52 | ((uint64_t)(1023 + exponent) << 52)));
}

// First ziggurat test for the word w: true (and z) when it accepts.
__device__ __forceinline__ bool fast_normal(uint64_t w, const double* __restrict__ X, double& z) {
    const int layer = (int)(w & 0xff);
    const double u = __dsub_rn(unit_bits(w >> 12, 1), 3.0);
    z = __dmul_rn(u, __ldg(X + layer));
    return fabs(z) < __ldg(X + layer + 1);
}

// Words of the stream on demand (one cached block), for the rare long draws.
struct Cursor {
    Key key;
    uint64_t blk;
    uint32_t w[16];
    __device__ uint64_t word(uint64_t q) {
        const uint64_t b = q >> 3;
        if (b != blk) {
            chacha12_block(key, b, w);
            blk = b;
        }
        const int j = (int)(q & 7) * 2;
        return (uint64_t)w[j] | ((uint64_t)w[j + 1] << 32);
    }
};

// The full draw that starts at word q; *len = words read, or 0 when the draw
// needs more than kMaxWordsPerDraw words (reported as an error).
__device__ __noinline__ double normal_from(Key key, uint64_t q, const double* __restrict__ X,
                                           const double* __restrict__ Fz, uint32_t* len) {
    Cursor c;
    c.key = key;
    c.blk = ~0ull;
    uint64_t pos = q;
    while (pos - q < kMaxWordsPerDraw) {
        const uint64_t w = c.word(pos++);
        const int layer = (int)(w & 0xff);
        const double u = __dsub_rn(unit_bits(w >> 12, 1), 3.0);
        const double x = __dmul_rn(u, __ldg(X + layer));
        if (fabs(x) < __ldg(X + layer + 1)) {
            *len = (uint32_t)(pos - q);
            return x;
        }
        if (layer == 0) {
            // tail beyond R: Marsaglia's exponential method
            while (pos - q + 2 <= kMaxWordsPerDraw) {
                const double ua = __dsub_rn(unit_bits(c.word(pos++) >> 12, 0), 1.0 - 1.1102230246251565e-16);
                const double ub = __dsub_rn(unit_bits(c.word(pos++) >> 12, 0), 1.0 - 1.1102230246251565e-16);
                const double a = __ddiv_rn(log(ua), kZigR);
                const double b = log(ub);
                if (!(__dmul_rn(-2.0, b) < __dmul_rn(a, a))) {
                    *len = (uint32_t)(pos - q);
                    return u < 0.0 ? __dsub_rn(a, kZigR) : __dsub_rn(kZigR, a);
                }
            }
            break;
        }
        const double v = __dmul_rn((double)(c.word(pos++) >> 11), 1.0 / 9007199254740992.0);
        const double f1 = __ldg(Fz + layer + 1), f0 = __ldg(Fz + layer);
        const double lhs = __dadd_rn(f1, __dmul_rn(__dsub_rn(f0, f1), v));
        if (lhs < exp(__ddiv_rn(__dmul_rn(-x, x), 2.0))) {
            *len = (uint32_t)(pos - q);
            return x;
        }
    }
    *len = 0;
    return 0.0;
}

// len[q - seg0] = words the draw starting at word q reads (1..255).
__global__ void __launch_bounds__(kInitBlock) k_sample_lengths(Key key, uint64_t seg0, uint64_t nblk,
                                                               const double* __restrict__ X,
                                                               const double* __restrict__ Fz,
                                                               uint64_t* __restrict__ len8, uint32_t* err) {
    for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nblk; b += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t w[16];
        chacha12_block(key, (seg0 >> 3) + b, w);
        uint64_t packed = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            double z;
            uint32_t n = 1;
            if (!fast_normal((uint64_t)w[2 * j] | ((uint64_t)w[2 * j + 1] << 32), X, z)) {
                normal_from(key, seg0 + 8 * b + j, X, Fz, &n);
                if (n == 0) {
                    atomicOr(err, 1u);
                    n = 1;
                }
            }
            packed |= (uint64_t)n << (8 * j);
        }
        len8[b] = packed;
    }
}

struct LongDraw {
    const uint8_t* len;
    __device__ __forceinline__ bool operator()(uint32_t q) const { return len[q] != 1; }
};

struct IsLong {
    __device__ __forceinline__ uint32_t operator()(uint8_t n) const { return n != 1; }
};

__global__ void k_gather_lengths(const uint32_t* __restrict__ pos, uint64_t n, const uint8_t* __restrict__ len,
                                 uint8_t* __restrict__ out) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
        out[k] = len[pos[k]];
}

// Words in [lo, hi) were read by an earlier draw: they start nothing.
__global__ void k_mark_swallowed(const uint32_t* __restrict__ lo, const uint32_t* __restrict__ hi, uint64_t n,
                                 uint8_t* __restrict__ len) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
        for (uint32_t q = lo[k]; q < hi[k]; ++q) len[q] = 0;
}

__global__ void k_block_starts(const uint64_t* __restrict__ len8, uint64_t nblk, uint32_t* __restrict__ cnt) {
    for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nblk; b += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t v = len8[b];
        uint32_t c = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) c += ((v >> (8 * j)) & 0xff) != 0;
        cnt[b] = c;
    }
}

__global__ void __launch_bounds__(kInitBlock) k_write_tables(Key key, uint64_t seg0, uint64_t nblk,
                                                             const uint64_t* __restrict__ len8,
                                                             const uint32_t* __restrict__ incl, uint64_t base,
                                                             Tables t, const double* __restrict__ X,
                                                             const double* __restrict__ Fz) {
    const uint64_t total = t.start[t.n];
    for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nblk; b += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t lens = len8[b];
        uint64_t k = base + (b ? incl[b - 1] : 0u);
        if (lens == 0 || k >= total) continue;
        // the table slot of draw k (empty tables are stepped over)
        int ti = 0;
        while (ti + 1 < t.n && k >= t.start[ti + 1]) ++ti;
        const uint64_t off = k - t.start[ti];
        uint64_t r = off / t.cols[ti];
        uint32_t c = (uint32_t)(off - r * t.cols[ti]);
        uint32_t w[16];
        chacha12_block(key, (seg0 >> 3) + b, w);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint32_t n = (uint32_t)((lens >> (8 * j)) & 0xff);
            if (n == 0 || k >= total) continue;
            double z;
            if (n == 1) {
                fast_normal((uint64_t)w[2 * j] | ((uint64_t)w[2 * j + 1] << 32), X, z);
            } else {
                uint32_t unused;
                z = normal_from(key, seg0 + 8 * b + j, X, Fz, &unused);
            }
            t.dst[ti][r * t.stride[ti] + c] = __fadd_rn(0.0f, __fmul_rn(t.sigma[ti], (float)z));
            ++k;
            if (++c == t.cols[ti]) {
                c = 0;
                if (++r == t.rows[ti]) {
                    r = 0;
                    do ++ti;
                    while (ti < t.n && t.rows[ti] == 0);
                }
            }
        }
    }
}

}  // namespace

void device_normal_tables(const NormalTable* tables, int n_tables, uint64_t seed, cudaStream_t st) {
    if (n_tables < 1 || n_tables > kMaxTables) throw Error(TSVD_ERR_INVALID, "device_normal_tables: 1..5 tables");
    Tables t{};
    t.n = n_tables;
    uint64_t total = 0;
    for (int i = 0; i < n_tables; ++i) {
        const NormalTable& d = tables[i];
        if (d.cols == 0 || d.stride < d.cols) throw Error(TSVD_ERR_INVALID, "device_normal_tables: bad table shape");
        t.dst[i] = d.dst;
        t.start[i] = total;
        t.rows[i] = d.rows;
        t.cols[i] = d.cols;
        t.stride[i] = d.stride;
        t.sigma[i] = d.sigma;
        if (d.stride != d.cols && d.rows)
            TSVD_CUDA(cudaMemsetAsync(d.dst, 0, d.rows * d.stride * sizeof(float), st));
        total += d.rows * d.cols;
    }
    t.start[n_tables] = total;
    if (total == 0) return;

    ChaCha12Stream g(seed);
    Key key;
    for (int i = 0; i < 8; ++i) key.k[i] = g.key()[i];
    const ZigTables& zt = zig();
    DevMem zig_d, err_d;
    zig_d.alloc(2 * 257 * sizeof(double));
    TSVD_CUDA(cudaMemcpyAsync(zig_d.p, zt.x, 257 * sizeof(double), cudaMemcpyHostToDevice, st));
    TSVD_CUDA(cudaMemcpyAsync(zig_d.as<double>() + 257, zt.f, 257 * sizeof(double), cudaMemcpyHostToDevice, st));
    const double* X = zig_d.as<double>();
    const double* Fz = X + 257;
    err_d.alloc(4);
    TSVD_CUDA(cudaMemsetAsync(err_d.p, 0, 4, st));

    DevMem len, cnt, incl, pos, nsel, plen, cub_tmp, rlo, rhi;
    nsel.alloc(16);
    uint64_t base = 0;     // draws numbered so far
    uint64_t seg0 = 0;     // first word of the segment
    uint64_t covered = 0;  // first word not read by the draws started so far
    std::vector<uint32_t> h_pos, lo, hi;
    std::vector<uint8_t> h_len;
    while (base < total) {
        // about 1.3% extra words per draw; a short segment just continues
        uint64_t want = (total - base) + (total - base) / 40 + 4096;
        want = std::min<uint64_t>((want + 7) & ~7ull, kMaxSegmentWords);
        const uint64_t nblk = want / 8;
        if (len.bytes < want) len.alloc(want);
        if (cnt.bytes < nblk * 4) cnt.alloc(nblk * 4);
        if (incl.bytes < nblk * 4) incl.alloc(nblk * 4);
        k_sample_lengths<<<kInitGrid, kInitBlock, 0, st>>>(key, seg0, nblk, X, Fz, len.as<uint64_t>(),
                                                          err_d.as<uint32_t>());
        TSVD_CUDA(cudaGetLastError());
        // words whose draw is longer than one word, in stream order: count,
        // size the list, then select
        thrust::counting_iterator<uint32_t> it(0);
        thrust::transform_iterator<IsLong, const uint8_t*, uint32_t> longs(len.as<uint8_t>(), IsLong{});
        size_t need = 0;
        TSVD_CUDA(cub::DeviceReduce::Sum(nullptr, need, longs, nsel.as<uint32_t>(), (int)want, st));
        if (cub_tmp.bytes < need) cub_tmp.alloc(need);
        size_t have = cub_tmp.bytes;
        TSVD_CUDA(cub::DeviceReduce::Sum(cub_tmp.p, have, longs, nsel.as<uint32_t>(), (int)want, st));
        uint32_t hdr[2] = {0, 0};  // {long draws, error flag}
        TSVD_CUDA(cudaMemcpyAsync(&hdr[0], nsel.p, 4, cudaMemcpyDeviceToHost, st));
        TSVD_CUDA(cudaMemcpyAsync(&hdr[1], err_d.p, 4, cudaMemcpyDeviceToHost, st));
        TSVD_CUDA(cudaStreamSynchronize(st));
        if (hdr[1]) throw Error(TSVD_ERR_INVALID, "normal init: a ziggurat draw needed more than 255 words");
        const uint32_t n_long = hdr[0];
        if (pos.bytes < (size_t)n_long * 4) pos.alloc((size_t)n_long * 4);
        LongDraw pred{len.as<uint8_t>()};
        need = 0;
        TSVD_CUDA(cub::DeviceSelect::If(nullptr, need, it, pos.as<uint32_t>(), nsel.as<int>() + 2, (int)want, pred, st));
        if (cub_tmp.bytes < need) cub_tmp.alloc(need);
        have = cub_tmp.bytes;
        TSVD_CUDA(cub::DeviceSelect::If(cub_tmp.p, have, it, pos.as<uint32_t>(), nsel.as<int>() + 2, (int)want, pred,
                                        st));
        h_pos.resize(n_long);
        h_len.resize(n_long);
        if (n_long) {
            if (plen.bytes < n_long) plen.alloc(n_long);
            k_gather_lengths<<<kInitGrid, kInitBlock, 0, st>>>(pos.as<uint32_t>(), n_long, len.as<uint8_t>(),
                                                              plen.as<uint8_t>());
            TSVD_CUDA(cudaGetLastError());
            TSVD_CUDA(cudaMemcpyAsync(h_pos.data(), pos.p, (size_t)n_long * 4, cudaMemcpyDeviceToHost, st));
            TSVD_CUDA(cudaMemcpyAsync(h_len.data(), plen.p, n_long, cudaMemcpyDeviceToHost, st));
            TSVD_CUDA(cudaStreamSynchronize(st));
        }
        // walk the long draws in order: a word starts a draw unless an earlier
        // draw read it
        lo.clear();
        hi.clear();
        if (covered > seg0) {
            lo.push_back(0);
            hi.push_back((uint32_t)std::min<uint64_t>(covered - seg0, want));
        }
        for (uint32_t k = 0; k < n_long; ++k) {
            const uint64_t q = seg0 + h_pos[k];
            if (q < covered) continue;
            covered = q + h_len[k];
            const uint64_t e = std::min<uint64_t>(covered - seg0, want);
            if (h_pos[k] + 1 < e) {
                lo.push_back(h_pos[k] + 1);
                hi.push_back((uint32_t)e);
            }
        }
        covered = std::max<uint64_t>(covered, seg0 + want);
        if (!lo.empty()) {
            if (rlo.bytes < lo.size() * 4) {
                rlo.alloc(lo.size() * 4);
                rhi.alloc(lo.size() * 4);
            }
            TSVD_CUDA(cudaMemcpyAsync(rlo.p, lo.data(), lo.size() * 4, cudaMemcpyHostToDevice, st));
            TSVD_CUDA(cudaMemcpyAsync(rhi.p, hi.data(), hi.size() * 4, cudaMemcpyHostToDevice, st));
            k_mark_swallowed<<<ceil_div(lo.size(), kInitBlock), kInitBlock, 0, st>>>(
                rlo.as<uint32_t>(), rhi.as<uint32_t>(), lo.size(), len.as<uint8_t>());
            TSVD_CUDA(cudaGetLastError());
        }
        k_block_starts<<<kInitGrid, kInitBlock, 0, st>>>(len.as<uint64_t>(), nblk, cnt.as<uint32_t>());
        TSVD_CUDA(cudaGetLastError());
        need = 0;
        TSVD_CUDA(cub::DeviceScan::InclusiveSum(nullptr, need, cnt.as<uint32_t>(), incl.as<uint32_t>(), (int)nblk, st));
        if (cub_tmp.bytes < need) cub_tmp.alloc(need);
        have = cub_tmp.bytes;
        TSVD_CUDA(cub::DeviceScan::InclusiveSum(cub_tmp.p, have, cnt.as<uint32_t>(), incl.as<uint32_t>(), (int)nblk,
                                                st));
        k_write_tables<<<kInitGrid, kInitBlock, 0, st>>>(key, seg0, nblk, len.as<uint64_t>(), incl.as<uint32_t>(),
                                                        base, t, X, Fz);
        TSVD_CUDA(cudaGetLastError());
        uint32_t starts = 0;
        TSVD_CUDA(cudaMemcpyAsync(&starts, incl.as<uint32_t>() + (nblk - 1), 4, cudaMemcpyDeviceToHost, st));
        TSVD_CUDA(cudaStreamSynchronize(st));
        base += starts;
        seg0 += want;
    }
}

}  // namespace tsvd
