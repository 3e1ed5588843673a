// Device-side PRNG stream and samplers.
//
// The reference's Blake2xbPRNG (src/randomgen.cpp:188-198) emits the concatenation
// of 4096-byte BLAKE2Xb outputs keyed by the 64-byte seed with the 8-byte
// little-endian counter 0, 1, 2, ... as message. That makes the stream counter
// based: byte p lives in refill p / 4096, output block (p % 4096) / 64, and every
// 64-byte block is one BLAKE2b compression of the refill's root hash. prng_fill
// computes any byte range in parallel (one thread per 64-byte block; BLAKE2b as in
// RFC 7693, BLAKE2X parameters per the BLAKE2X specification).
//
// A PRNG is a device-resident PrngState {seed, offset}: samplers read the offset,
// consume bytes and advance it, so data-dependent consumption (rejection sampling)
// needs no host round trip. The samplers reproduce the reference's consumption
// exactly (src/utils/rlwe.cpp:21-150): ternary draws 32-bit words through
// libstdc++'s uniform_int_distribution<uint64_t>(0, 2), which rejects only a zero
// word; CBD takes 6 bytes per coefficient; uniform takes L*N 64-bit words, then
// replaces each rejected word, in order, by the next acceptable word of the stream.
#include <cstring>
#include <random>

#include "context.hpp"
#include "prng.hpp"
#include "trace.cuh"

namespace tb {

unsigned grid_for(uint64_t work, int threads);

namespace {

__constant__ uint64_t c_iv[8] = {0x6a09e667f3bcc908ULL, 0xbb67ae8584caa73bULL, 0x3c6ef372fe94f82bULL,
                                 0xa54ff53a5f1d36f1ULL, 0x510e527fade682d1ULL, 0x9b05688c2b3e6c1fULL,
                                 0x1f83d9abfb41bd6bULL, 0x5be0cd19137e2179ULL};
__constant__ uint8_t c_sigma[12][16] = {
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}, {14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3},
    {11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4}, {7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8},
    {9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13}, {2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9},
    {12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11}, {13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10},
    {6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5}, {10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0},
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}, {14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3}};

__device__ __forceinline__ uint64_t rotr(uint64_t x, int c) { return (x >> c) | (x << (64 - c)); }

__device__ void b2_compress(uint64_t h[8], const uint64_t m[16], uint64_t t, bool last) {
    uint64_t v[16];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        v[i] = h[i];
        v[i + 8] = c_iv[i];
    }
    v[12] ^= t;
    if (last) v[14] = ~v[14];
#define G(a, b, c, d, x, y)                  \
    v[a] = v[a] + v[b] + (x);                \
    v[d] = rotr(v[d] ^ v[a], 32);            \
    v[c] = v[c] + v[d];                      \
    v[b] = rotr(v[b] ^ v[c], 24);            \
    v[a] = v[a] + v[b] + (y);                \
    v[d] = rotr(v[d] ^ v[a], 16);            \
    v[c] = v[c] + v[d];                      \
    v[b] = rotr(v[b] ^ v[c], 63);
#pragma unroll 1
    for (int r = 0; r < 12; r++) {
        const uint8_t *s = c_sigma[r];
        G(0, 4, 8, 12, m[s[0]], m[s[1]]);
        G(1, 5, 9, 13, m[s[2]], m[s[3]]);
        G(2, 6, 10, 14, m[s[4]], m[s[5]]);
        G(3, 7, 11, 15, m[s[6]], m[s[7]]);
        G(0, 5, 10, 15, m[s[8]], m[s[9]]);
        G(1, 6, 11, 12, m[s[10]], m[s[11]]);
        G(2, 7, 8, 13, m[s[12]], m[s[13]]);
        G(3, 4, 9, 14, m[s[14]], m[s[15]]);
    }
#undef G
#pragma unroll
    for (int i = 0; i < 8; i++) h[i] ^= v[i] ^ v[i + 8];
}

// 64-byte block `sb` of the stream of `seed`.
__device__ void stream_block(const uint64_t *seed, uint64_t sb, uint64_t out[8]) {
    const uint64_t counter = sb >> 6;
    const uint32_t blk = (uint32_t)(sb & 63);
    const uint64_t xof = 4096;
    uint64_t h[8], m[16];
#pragma unroll
    for (int i = 0; i < 8; i++) h[i] = c_iv[i];
    // root: digest 64, key 64, fanout 1, depth 1, leaf 0; node offset 0, xof length 4096
    h[0] ^= 64ull | (64ull << 8) | (1ull << 16) | (1ull << 24);
    h[1] ^= xof << 32;
#pragma unroll
    for (int i = 0; i < 16; i++) m[i] = i < 8 ? seed[i] : 0;
    b2_compress(h, m, 128, false);
#pragma unroll
    for (int i = 0; i < 16; i++) m[i] = 0;
    m[0] = counter;
    b2_compress(h, m, 136, true);
    // output node: digest 64, leaf length 64, node offset blk, xof 4096, inner length 64
#pragma unroll
    for (int i = 0; i < 8; i++) out[i] = c_iv[i];
    out[0] ^= 64ull | (64ull << 32);
    out[1] ^= (uint64_t)blk | (xof << 32);
    out[2] ^= 64ull << 8;
#pragma unroll
    for (int i = 0; i < 16; i++) m[i] = i < 8 ? h[i] : 0;
    b2_compress(out, m, 64, true);
}

// buf[k] = stream[st->offset + k] for k < nbytes, for each of `count` states.
__global__ void prng_fill_kernel(const PrngState *__restrict__ st, uint8_t *__restrict__ buf, uint64_t nbytes,
                                 uint64_t bstride) {
    const PrngState &s = st[blockIdx.y];
    const uint64_t off = s.offset;
    const uint64_t first = off >> 6, last = (off + nbytes + 63) >> 6;
    uint8_t *b = buf + blockIdx.y * bstride;
    for (uint64_t sb = first + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; sb < last;
         sb += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t w[8];
        stream_block(s.seed, sb, w);
        const uint64_t lo = sb << 6;
        const uint8_t *bytes = reinterpret_cast<const uint8_t *>(w);
        if (lo >= off && lo + 64 <= off + nbytes) {
            uint64_t *dst = reinterpret_cast<uint64_t *>(b + (lo - off));
            if (((lo - off) & 7) == 0) {
#pragma unroll
                for (int i = 0; i < 8; i++) dst[i] = w[i];
                continue;
            }
        }
        for (int k = 0; k < 64; k++) {
            const uint64_t p = lo + k;
            if (p >= off && p < off + nbytes) b[p - off] = bytes[k];
        }
    }
}

// Ternary sampling; a zero word would be rejected by the distribution, which the
// fix-up pass then handles sequentially (probability 2^-32 per word).
__global__ void ternary_kernel(const uint8_t *__restrict__ buf, uint64_t bstride, uint32_t n,
                               const Mod *__restrict__ mods, int L, uint64_t *__restrict__ out, uint64_t ostride,
                               PrngState *st) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint8_t *b = buf + blockIdx.y * bstride;
    uint64_t *o = out + blockIdx.y * ostride;
    const uint32_t w = reinterpret_cast<const uint32_t *>(b)[i];
    if (w == 0) atomicOr(&st[blockIdx.y].flag, 1u);
    const uint64_t r = ((uint64_t)w * 3u) >> 32;
    for (int j = 0; j < L; j++) o[(size_t)j * n + i] = r == 0 ? mods[j].value - 1 : r - 1;
}

__global__ void ternary_fixup_kernel(const uint8_t *__restrict__ buf, uint64_t bstride, uint64_t avail_words,
                                     uint32_t n, const Mod *__restrict__ mods, int L, uint64_t *__restrict__ out,
                                     uint64_t ostride, PrngState *st) {
    PrngState &s = st[blockIdx.x];
    if (threadIdx.x != 0) return;
    if (!(s.flag & 1)) {
        s.offset += 4ull * n;
        return;
    }
    const uint32_t *w = reinterpret_cast<const uint32_t *>(buf + blockIdx.x * bstride);
    uint64_t *o = out + blockIdx.x * ostride;
    uint64_t p = 0;
    for (uint32_t i = 0; i < n; i++) {
        uint32_t x;
        do {
            if (p >= avail_words) {
                s.flag = 2;  // stream window exhausted: reported by prng_check
                return;
            }
            x = w[p++];
        } while (x == 0);
        const uint64_t r = ((uint64_t)x * 3u) >> 32;
        for (int j = 0; j < L; j++) o[(size_t)j * n + i] = r == 0 ? mods[j].value - 1 : r - 1;
    }
    s.offset += 4 * p;
    s.flag = 0;
}

// Centered binomial, 6 bytes per coefficient (src/utils/rlwe.cpp:89-104).
__global__ void cbd_kernel(const uint8_t *__restrict__ buf, uint64_t bstride, uint32_t n,
                           const Mod *__restrict__ mods, int L, uint64_t *__restrict__ out, uint64_t ostride) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint8_t *x = buf + blockIdx.y * bstride + 6ull * i;
    uint64_t *o = out + blockIdx.y * ostride;
    const int v = __popc(x[0]) + __popc(x[1]) + __popc(x[2] & 0x1f) - __popc(x[3]) - __popc(x[4]) -
                  __popc(x[5] & 0x1f);
    for (int j = 0; j < L; j++) o[(size_t)j * n + i] = v < 0 ? mods[j].value - (uint64_t)(-v) : (uint64_t)v;
}

__global__ void advance_kernel(PrngState *st, uint64_t bytes) { st[blockIdx.x].offset += bytes; }

constexpr uint64_t REJECTED = ~0ull;

// Uniform mod q_j: word (j, i) is accepted below max_multiple_j (src/utils/rlwe.cpp:126-149).
__global__ void uniform_kernel(const uint8_t *__restrict__ buf, uint64_t bstride, uint32_t n,
                               const Mod *__restrict__ mods, const uint64_t *__restrict__ maxmult, int L,
                               uint64_t *__restrict__ out, uint64_t ostride, PrngState *st) {
    const uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (idx >= (uint64_t)L * n) return;
    const int j = (int)(idx / n);
    const uint64_t w = reinterpret_cast<const uint64_t *>(buf + blockIdx.y * bstride)[idx];
    uint64_t *o = out + blockIdx.y * ostride;
    if (w >= maxmult[j]) {
        o[idx] = REJECTED;
        atomicOr(&st[blockIdx.y].flag, 1u);
    } else {
        o[idx] = reduce64(w, mods[j]);
    }
}

// One warp per state: rejected positions in (limb, coefficient) order take the next
// acceptable words after the first L*N.
__global__ void uniform_fixup_kernel(const uint8_t *__restrict__ buf, uint64_t bstride, uint64_t avail_words,
                                     uint32_t n, const Mod *__restrict__ mods, const uint64_t *__restrict__ maxmult,
                                     int L, uint64_t *__restrict__ out, uint64_t ostride, PrngState *st) {
    PrngState &s = st[blockIdx.x];
    const int lane = threadIdx.x;
    const uint64_t total = (uint64_t)L * n;
    if (!(s.flag & 1)) {
        if (lane == 0) s.offset += 8 * total;
        return;
    }
    const uint64_t *w = reinterpret_cast<const uint64_t *>(buf + blockIdx.x * bstride);
    uint64_t *o = out + blockIdx.x * ostride;
    uint64_t p = total;
    for (int j = 0; j < L; j++) {
        const Mod m = mods[j];
        const uint64_t mm = maxmult[j];
        for (uint32_t i0 = 0; i0 < n; i0 += 32) {
            const uint32_t i = i0 + lane;
            unsigned rej = __ballot_sync(0xffffffffu, i < n && o[(uint64_t)j * n + i] == REJECTED);
            while (rej) {
                const int k = __ffs(rej) - 1;
                rej &= rej - 1;
                uint64_t val = 0;
                bool found = false;
                while (!found) {
                    if (p + lane >= avail_words && p >= avail_words) {
                        if (lane == 0) s.flag = 2;
                        return;
                    }
                    const uint64_t x = p + lane < avail_words ? w[p + lane] : REJECTED;
                    const unsigned acc = __ballot_sync(0xffffffffu, p + lane < avail_words && x < mm);
                    if (acc) {
                        const int f = __ffs(acc) - 1;
                        val = __shfl_sync(0xffffffffu, x, f);
                        p += f + 1;
                        found = true;
                    } else {
                        p += 32;
                    }
                }
                if (lane == 0) o[(uint64_t)j * n + i0 + k] = reduce64(val, m);
            }
        }
    }
    __syncwarp();
    if (lane == 0) {
        s.offset += 8 * p;
        s.flag = 0;
    }
}

}  // namespace

// Samples `count` polynomials over table moduli [first, first + L) from `count`
// device PRNG states into out (polynomial b at out + b*ostride, [L][N]).
int sample_poly(const Context &c, int kind, PrngState *st, int count, int first, int L, uint64_t *out,
                uint64_t ostride, cudaStream_t s) {
    if (count <= 0) return TB_OK;
    const uint32_t n = c.n;
    if (!ostride) ostride = (uint64_t)L * n;
    uint64_t nbytes;
    if (kind == SAMPLE_TERNARY) nbytes = 4ull * n + 256;
    else if (kind == SAMPLE_CBD) nbytes = 6ull * n;
    else nbytes = 8ull * ((uint64_t)L * n + (uint64_t)L * n / 4 + 1024);
    const uint64_t bstride = (nbytes + 255) & ~255ull;
    uint8_t *buf = nullptr;
    cudaError_t e = cudaMallocAsync(&buf, bstride * count, s);
    if (e != cudaSuccess) return status_from(e);
    const Mod *mods = c.d_mods + first;
    {
        TraceScope ts("prng_fill", s);
        dim3 g((unsigned)std::min<uint64_t>((nbytes / 64 + 1 + 127) / 128, 1024), count);
        prng_fill_kernel<<<g, 128, 0, s>>>(st, buf, nbytes, bstride);
    }
    TraceScope ts("sample", s);
    if (kind == SAMPLE_TERNARY) {
        dim3 g((n + 255) / 256, count);
        ternary_kernel<<<g, 256, 0, s>>>(buf, bstride, n, mods, L, out, ostride, st);
        ternary_fixup_kernel<<<count, 32, 0, s>>>(buf, bstride, nbytes / 4, n, mods, L, out, ostride, st);
    } else if (kind == SAMPLE_CBD) {
        dim3 g((n + 255) / 256, count);
        cbd_kernel<<<g, 256, 0, s>>>(buf, bstride, n, mods, L, out, ostride);
        advance_kernel<<<count, 1, 0, s>>>(st, 6ull * n);
    } else {
        // max_multiple_j = 2^64 - 1 - ((2^64 - 1) mod q_j) - 1
        uint64_t *mm = nullptr;
        e = cudaMallocAsync(&mm, 8 * L, s);
        if (e != cudaSuccess) {
            cudaFreeAsync(buf, s);
            return status_from(e);
        }
        std::vector<uint64_t> h(L);
        for (int j = 0; j < L; j++) {
            const uint64_t q = c.table_moduli[first + j];
            h[j] = ~0ull - (~0ull % q) - 1;
        }
        e = cudaMemcpyAsync(mm, h.data(), 8 * L, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // h is a stack buffer
        if (e != cudaSuccess) {
            cudaFreeAsync(buf, s);
            cudaFreeAsync(mm, s);
            return status_from(e);
        }
        dim3 g((unsigned)(((uint64_t)L * n + 255) / 256), count);
        uniform_kernel<<<g, 256, 0, s>>>(buf, bstride, n, mods, mm, L, out, ostride, st);
        uniform_fixup_kernel<<<count, 32, 0, s>>>(buf, bstride, nbytes / 8, n, mods, mm, L, out, ostride, st);
        cudaFreeAsync(mm, s);
    }
    e = cudaGetLastError();
    cudaFreeAsync(buf, s);
    return e == cudaSuccess ? TB_OK : status_from(e);
}

// Raw stream bytes of one state (advances it).
int prng_bytes(PrngState *st, uint64_t nbytes, uint8_t *out, cudaStream_t s) {
    prng_fill_kernel<<<dim3((unsigned)std::max<uint64_t>(1, (nbytes / 64 + 128) / 128), 1), 128, 0, s>>>(st, out,
                                                                                                      nbytes, 0);
    advance_kernel<<<1, 1, 0, s>>>(st, nbytes);
    return status_from(cudaGetLastError());
}

// Fresh states: a seeded factory gives every PRNG the same seed and offset 0
// (src/randomgen.h:412-427); without a seed each state gets random bytes.
int prng_init(PrngState *st, int count, const uint64_t *seed8, cudaStream_t s) {
    std::vector<PrngState> h(count);
    std::random_device rd;
    for (auto &x : h) {
        for (int i = 0; i < 8; i++)
            x.seed[i] = seed8 ? seed8[i] : ((uint64_t)rd() << 32 | rd());
        x.offset = 0;
        x.flag = 0;
        x.pad = 0;
    }
    cudaError_t e = cudaMemcpyAsync(st, h.data(), sizeof(PrngState) * count, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return status_from(e);
}

}  // namespace tb
