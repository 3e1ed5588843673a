// BLAKE2b (RFC 7693), unkeyed, for parameter-set identifiers: the reference's
// HashFunction::hash (src/utils/hash.h:20-33) is a 32-byte BLAKE2b digest of the
// parameter words, and the identifiers must equal the reference's so that
// serialized objects and golden tests agree.
#include <cstdint>
#include <cstring>

#include "hash.hpp"

namespace troyn {
namespace {

constexpr uint64_t IV[8] = {0x6a09e667f3bcc908ULL, 0xbb67ae8584caa73bULL, 0x3c6ef372fe94f82bULL,
                            0xa54ff53a5f1d36f1ULL, 0x510e527fade682d1ULL, 0x9b05688c2b3e6c1fULL,
                            0x1f83d9abfb41bd6bULL, 0x5be0cd19137e2179ULL};

constexpr uint8_t SIGMA[12][16] = {
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}, {14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3},
    {11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4}, {7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8},
    {9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13}, {2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9},
    {12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11}, {13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10},
    {6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5}, {10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0},
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}, {14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3}};

inline uint64_t rotr(uint64_t x, int r) { return (x >> r) | (x << (64 - r)); }

struct State {
    uint64_t h[8];
    uint64_t t = 0;  // bytes hashed (inputs here are far below 2^64 bytes)
    uint8_t buf[128];
};

void compress(State &s, const uint8_t *block, bool last) {
    uint64_t m[16], v[16];
    for (int i = 0; i < 16; i++) std::memcpy(&m[i], block + 8 * i, 8);  // little-endian host
    for (int i = 0; i < 8; i++) {
        v[i] = s.h[i];
        v[i + 8] = IV[i];
    }
    v[12] ^= s.t;
    if (last) v[14] = ~v[14];
    auto g = [&](int a, int b, int c, int d, uint64_t x, uint64_t y) {
        v[a] = v[a] + v[b] + x;
        v[d] = rotr(v[d] ^ v[a], 32);
        v[c] = v[c] + v[d];
        v[b] = rotr(v[b] ^ v[c], 24);
        v[a] = v[a] + v[b] + y;
        v[d] = rotr(v[d] ^ v[a], 16);
        v[c] = v[c] + v[d];
        v[b] = rotr(v[b] ^ v[c], 63);
    };
    for (int r = 0; r < 12; r++) {
        const uint8_t *z = SIGMA[r];
        g(0, 4, 8, 12, m[z[0]], m[z[1]]);
        g(1, 5, 9, 13, m[z[2]], m[z[3]]);
        g(2, 6, 10, 14, m[z[4]], m[z[5]]);
        g(3, 7, 11, 15, m[z[6]], m[z[7]]);
        g(0, 5, 10, 15, m[z[8]], m[z[9]]);
        g(1, 6, 11, 12, m[z[10]], m[z[11]]);
        g(2, 7, 8, 13, m[z[12]], m[z[13]]);
        g(3, 4, 9, 14, m[z[14]], m[z[15]]);
    }
    for (int i = 0; i < 8; i++) s.h[i] ^= v[i] ^ v[i + 8];
}

}  // namespace

void blake2b(const void *in, size_t inlen, void *out, size_t outlen) {
    State s;
    for (int i = 0; i < 8; i++) s.h[i] = IV[i];
    s.h[0] ^= 0x01010000ULL ^ (uint64_t)outlen;  // depth 1, fanout 1, no key
    const uint8_t *p = static_cast<const uint8_t *>(in);
    while (inlen > 128) {
        s.t += 128;
        compress(s, p, false);
        p += 128;
        inlen -= 128;
    }
    std::memset(s.buf, 0, sizeof(s.buf));
    std::memcpy(s.buf, p, inlen);
    s.t += inlen;
    compress(s, s.buf, true);
    std::memcpy(out, s.h, outlen);
}

}  // namespace troyn
