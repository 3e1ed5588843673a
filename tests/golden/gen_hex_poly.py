"""Generates hex_poly.json: how the reference parses and prints hexadecimal plaintext
polynomials (Plaintext(hex_poly) and to_string, src/plaintext.cpp:91-215).

    make -C oracle ref && python tests/golden/gen_hex_poly.py

Calls oracle/_ref/libtroyref.so (the reference's own CPU sources) through ctypes
only: the reference's string code is run in a process without numpy loaded, where
it crashed in this container's Python otherwise.
"""
import ctypes
import json
import os
import random

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle", "_ref", "libtroyref.so")

CASES = ["7FFx^3 + 1x^1 + 3", "0", "", "1", "00Ax^2 + 0", "FFFFFFFFFFFFFFFFx^5", "1x^1", "3 + 1x^1",
         "1x^2 +", "1x^2 + ", "x^2", "1x^ + 1", "12345678901234567x^1", "1x^3 + 2x^3", "1x^2+1",
         "abcx^2 + Fx^1", "1x^10 + 0x^3", "0x^4 + 0"]


def main():
    lib = ctypes.CDLL(LIB)
    lib.ref_plain_hex.restype = ctypes.c_int
    lib.ref_plain_hex.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_char_p,
                                  ctypes.c_size_t]
    rng = random.Random(12)
    cases = list(CASES)
    for _ in range(6):
        coeffs = [rng.getrandbits(62) for _ in range(12)]
        for i in rng.sample(range(12), 4):
            coeffs[i] = 0
        terms = [f"{v:X}" + (f"x^{i}" if i else "") for i, v in reversed(list(enumerate(coeffs))) if v]
        cases.append(" + ".join(terms))
    out = []
    for text in cases:
        buf = (ctypes.c_uint64 * 4096)()
        s = ctypes.create_string_buffer(1 << 16)
        k = lib.ref_plain_hex(text.encode(), buf, 4096, s, len(s))
        if k < 0:
            out.append({"text": text, "accepted": False})
        else:
            out.append({"text": text, "accepted": True, "coeffs": [str(buf[i]) for i in range(k)],
                        "printed": s.value.decode()})
    with open(os.path.join(HERE, "hex_poly.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
