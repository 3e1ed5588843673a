#pragma once
#include <cstddef>

namespace troyn {
// Unkeyed BLAKE2b digest of outlen (1..64) bytes.
void blake2b(const void *in, size_t inlen, void *out, size_t outlen);
}  // namespace troyn
