"""Generates the golden fixtures in this directory from the reference itself.

    make -C oracle ref && python tests/golden/gen_golden.py

Runs the reference's own CPU implementation (oracle/_ref/libtroyref.so, compiled
from the reference sources by oracle/Makefile) on seeded inputs and stores:

* ``sessions_n64.npz``: full words of seeded BFV / BGV / CKKS sessions at N=64
  (secret, public, relinearization and Galois keys; encryption, multiply,
  relinearize, rotate, rescale or mod-switch, decrypted slots);
* ``bfv_n4096.json``: SHA-256 of every array of the same chain at the BFV
  single-op configuration (N=4096, {36, 36, 37}, t = 65537) plus the decrypted slots
  checksum;
* ``rns_n64.npz``: inputs and outputs of every RNS-tool operation at N=64;
* ``kat.json``: the known-answer values of the reference's NTT unit tests
  (test/utils/ntt.cpp:52-99) and prime/root tables at small sizes.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from oracle import Oracle, RefSession  # noqa: E402

SEED = np.arange(101, 109, dtype=np.uint64)


def session_arrays(scheme, n, bits, t, slots_seed=7, step=1):
    r = Oracle("ref")
    moduli = r.coeff_modulus_create(n, bits)
    if t is None:
        t = r.plain_modulus_batching(n, 20)
    s = RefSession(scheme, n, moduli, t, SEED)
    logn = n.bit_length() - 1
    elt = r.galois_elt_from_step(logn, step)
    out = {"moduli": np.array(moduli, np.uint64), "t": np.array([t], np.uint64),
           "sk": s.secret_key(), "pk": s.public_key(), "rlk": s.relin_key(), "gk": s.galois_key(elt),
           "elt": np.array([elt], np.uint64)}
    rng = np.random.default_rng(slots_seed)
    if scheme in (1, 3):
        a = rng.integers(0, t, n, dtype=np.uint64)
        b = rng.integers(0, t, n, dtype=np.uint64)
        ia, ib = s.encrypt_slots(a), s.encrypt_slots(b)
        im = s.multiply(ia, ib)
        ir = s.relinearize(im)
        io = s.rotate_rows(ir, step)
        isw = s.mod_switch(io)
        out.update(a=a, b=b, enc_a=s.ct(ia)["data"], enc_b=s.ct(ib)["data"], mul=s.ct(im)["data"],
                   relin=s.ct(ir)["data"], rot=s.ct(io)["data"], modswitch=s.ct(isw)["data"],
                   correction=np.array([s.ct(io)["correction"]], np.uint64), dec=s.decrypt_slots(io),
                   plain_a=s.encode_slots(a))
    else:
        v = rng.uniform(-1, 1, n // 2) + 1j * rng.uniform(-1, 1, n // 2)
        w = rng.uniform(-1, 1, n // 2) + 1j * rng.uniform(-1, 1, n // 2)
        scale = 2.0 ** 30
        ia, ib = s.encrypt_ckks(v, scale), s.encrypt_ckks(w, scale)
        im = s.multiply(ia, ib)
        ir = s.relinearize(im)
        isc = s.rescale(ir)
        io = s.rotate_vector(isc, step)
        out.update(v=v, w=w, scale=np.array([scale]), plain_v=s.encode_ckks(v, scale),
                   enc_a=s.ct(ia)["data"], enc_b=s.ct(ib)["data"], mul=s.ct(im)["data"],
                   relin=s.ct(ir)["data"], rescale=s.ct(isc)["data"], rot=s.ct(io)["data"],
                   rot_scale=np.array([s.ct(io)["scale"]]), dec=s.decrypt_ckks(io, n // 2))
    s.close()
    return out


def main():
    r = Oracle("ref")
    # seeded sessions at N=64
    sess = {}
    for name, (scheme, bits, t) in {"bfv": (1, [40, 40, 40, 40], None), "bgv": (3, [40, 40, 41, 41], None),
                                     "ckks": (2, [60, 40, 40, 60], 0)}.items():
        for k, v in session_arrays(scheme, 64, bits, t).items():
            sess[f"{name}_{k}"] = v
    np.savez_compressed(os.path.join(HERE, "sessions_n64.npz"), **sess)

    # BFV single-op configuration: hashes
    arrs = session_arrays(1, 4096, [36, 36, 37], 65537)
    js = {k: hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest() for k, v in arrs.items()}
    js["moduli"] = [int(x) for x in arrs["moduli"]]
    with open(os.path.join(HERE, "bfv_n4096.json"), "w") as f:
        json.dump(js, f, indent=1, sort_keys=True)

    # RNS-tool operations at N=64
    rng = np.random.default_rng(3)
    rns = {}
    for tag, bits, t in (("bfv", [40, 40, 40, 40], None), ("ckks", [60, 40, 40, 60], 0)):
        q = r.coeff_modulus_create(64, bits)
        if t is None:
            t = r.plain_modulus_batching(64, 20)
        msk, gamma, bsk = r.rns_bases(64, q, t)
        xq = np.stack([rng.integers(0, m, 64, dtype=np.uint64) for m in q])
        xbm = np.stack([rng.integers(0, m, 64, dtype=np.uint64) for m in bsk + [1 << 32]])
        B = len(bsk)
        rns[f"{tag}_q"] = np.array(q, np.uint64)
        rns[f"{tag}_t"] = np.array([t], np.uint64)
        rns[f"{tag}_bsk"] = np.array(bsk, np.uint64)
        rns[f"{tag}_xq"] = xq
        rns[f"{tag}_xbm"] = xbm
        ops = [("fastbconv_mtilde", xq, B + 1), ("sm_mrq", xbm, B), ("fast_floor", np.concatenate([xq, xbm[:B]]), B),
               ("fastbconv_sk", xbm[:B], len(q)), ("div_round_last", xq, len(q)), ("div_round_last_ntt", xq, len(q))]
        if t:
            ops += [("decrypt_scale_round", xq, 1), ("mod_t_div_last", xq, len(q)), ("decrypt_mod_t", xq, 1)]
        for name, data, ol in ops:
            rns[f"{tag}_{name}"] = r.rns_op(name, 64, q, t, data, ol)
    np.savez_compressed(os.path.join(HERE, "rns_n64.npz"), **rns)

    # known answers of the reference's own NTT unit tests (test/utils/ntt.cpp:52-99)
    kat = {"ntt_q": 0xffffffffffc0001,
           "root_powers_logn1": [1, 288794978602139552],
           "root_powers_logn2": [1, 288794978602139552, 178930308976060547, 748001537669050592],
           "ntt_logn1": {"in": [[0, 0], [1, 0], [1, 1]],
                         "out": [[0, 0], [1, 1], [288794978602139553, 864126526004445282]]}}
    # prime lists of CoeffModulus::Create at the benchmark parameter sets
    kat["coeff_modulus"] = {f"{n}:{','.join(map(str, b))}": r.coeff_modulus_create(n, b) for n, b in (
        (4096, [36, 36, 37]), (16384, [60] + [40] * 7 + [60]), (16384, [50] * 8), (32768, [50] * 8),
        (8192, [43, 43, 44, 44, 44]), (64, [40, 40, 40, 40]))}
    kat["plain_batching"] = {f"{n}:20": r.plain_modulus_batching(n, 20) for n in (64, 4096, 8192, 16384)}
    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump(kat, f, indent=1)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
