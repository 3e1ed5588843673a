// Device PRNG state and sampler entry points (prng.cu).
#pragma once

#include <cstdint>

#include "context.hpp"

namespace tb {

// One UniformRandomGenerator: its seed and the stream position already consumed.
// flag is scratch for the samplers' rejection fix-ups (2 = stream window exhausted).
struct PrngState {
    uint64_t seed[8];
    uint64_t offset;
    uint32_t flag;
    uint32_t pad;
};

enum { SAMPLE_TERNARY = 0, SAMPLE_CBD = 1, SAMPLE_UNIFORM = 2 };

int prng_init(PrngState *st, int count, const uint64_t *seed8, cudaStream_t s);
int sample_poly(const Context &c, int kind, PrngState *st, int count, int first, int L, uint64_t *out,
                uint64_t ostride, cudaStream_t s);
int prng_bytes(PrngState *st, uint64_t nbytes, uint8_t *out, cudaStream_t s);

}  // namespace tb
