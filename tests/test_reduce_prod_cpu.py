"""The one-product Barrett reduction of the CKKS tensor product (reduce_prod in
seal-cuda_b200/csrc/common.cuh), restated with 64-bit wrap-around on the CPU: for moduli
of every bit length 2 .. 61 and values below 2^(2n+1) (products of two residues and
sums of two), the remainder before the two conditional subtractions stays in [0, 3q)
and the result is x mod q. This pins the bound the kernel's comment states."""
import random

M64 = (1 << 64) - 1


def reduce_prod(x, q):
    hi, lo = x >> 64, x & M64
    ratio = (1 << 128) // q
    r_hi, r_lo = ratio >> 64, ratio & M64
    s = q.bit_length() - 2
    t = ((lo >> s) | (hi << (64 - s))) & M64 if s else lo
    mu = ((r_hi << s) | (r_lo >> (64 - s))) & M64 if s else r_hi
    assert mu == (1 << (64 + s)) // q and mu < (1 << 63)
    r = (lo - ((t * mu) >> 64) * q) & M64
    assert 0 <= r < 3 * q, (q, x, r)
    for c in (2 * q, q):
        r = min(r, (r - c) & M64)
    return r


def test_reduce_prod_bound_and_value():
    rng = random.Random(2026)
    for n in range(2, 62):
        for _ in range(6):
            q = rng.randrange((1 << (n - 1)) | 1, 1 << n, 2) if n > 2 else 3
            top = 1 << (2 * n + 1)
            cases = [0, 1, q - 1, q, (q - 1) ** 2, 2 * (q - 1) ** 2, top - 1, top - q]
            cases += [rng.randrange(top) for _ in range(200)]
            cases += [rng.randrange(q) * rng.randrange(q) for _ in range(100)]
            for x in cases:
                if x < top:
                    assert reduce_prod(x, q) == x % q, (n, q, x)
