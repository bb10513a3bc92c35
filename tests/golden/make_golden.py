"""Generate the golden fixtures in tests/golden/ from the reference's own CPU build.

The reference (cuFE src/*.c) is compiled unmodified by oracle/ref/build_ref.py into
oracle/_ref/<variant>/libref.so; this script drives that build with fixed seeds and stores
its outputs.  Run in the build container (needs the reference tree):

    python oracle/build.py && python tests/golden/make_golden.py

Outputs:
  ref_n256_l8.npz   full arrays at n=256, l=8: NTT/INTT vectors, AES-CTR streams, sampler
                    streams (4 calls per sigma, keyed and zero-key), sample_polya, setup,
                    encrypt, keygen, decrypt residues and decode
  ref_c2.json       SHA-256 of every array of one setup/encrypt/keygen/decrypt round at the
                    C2 shape (n=4096, l=784), and the decoded inner product; also the
                    ciphertext with the f_i stream keyed by seed3 (the reference draws f_i
                    from an AES context it never initialises; the keyed ciphertext is the
                    reference's ciphertext with its zero-key f_i replaced by the reference
                    sampler's keyed stream, exact since c_i is linear in f_i)
  ref_modeb.npz     the GPU counter-to-sample mapping (mode B) from the reference's own kernel
                    bodies (src/sample_gpu.cu) run on the host by oracle/_ref/modeb/libmodeb.so:
                    polynomial 0 (the first 4096 samples) per sigma for two keys as signed
                    integers, and SHA-256 of the canonical residues of polynomials 1, 7, 63
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.ffi import Q, Reference, ReferenceModeB  # noqa: E402


def canon(a):
    a = np.asarray(a, np.uint64)
    q = np.array(Q, np.uint64).reshape([1] * (a.ndim - 2) + [3, 1])
    return (a % q).astype(np.uint32)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, np.uint32).tobytes()).hexdigest()


def small():
    R = Reference("n256_l8")
    rng = np.random.default_rng(0xC0FE0100)
    out = {}
    key = rng.integers(0, 256, 32, dtype=np.uint8)
    out["ctr_key"] = key
    out["ctr_keyed"] = R.ctr_stream(key, 2)
    out["ctr_zero"] = R.ctr_stream(None, 2)
    for sel in range(3):
        a = (rng.integers(0, 2**32, 256, dtype=np.uint64) % Q[sel]).astype(np.uint32)
        out["ntt_in_%d" % sel] = a
        out["ntt_fwd_%d" % sel] = R.ntt(a, sel)
        out["ntt_inv_%d" % sel] = R.ntt(a, sel, inverse=True)
    for sig in range(3):
        out["gauss_key_%d" % sig] = canon(R.gauss(sig, key, 4))
        out["gauss_zero_%d" % sig] = canon(R.gauss(sig, None, 4))
    seed_a, seed_e, seed2 = rng.integers(0, 256, (3, 32), dtype=np.uint8)
    out["polya_seed"] = seed_a
    out["polya"] = R.sample_polya(seed_a)
    mpk, msk = R.setup(seed_a, seed_e)
    x = rng.integers(0, 5, R.l, dtype=np.uint32)
    y = rng.integers(0, 17, R.l, dtype=np.uint32)
    ct = R.encrypt(x, mpk, seed2)
    sky = R.keygen(y, msk)
    dy, dec = R.decrypt(ct, y, sky)
    out.update(seed_a=seed_a, seed_e=seed_e, seed2=seed2, x=x, y=y, mpk=canon(mpk), msk=canon(msk),
               ct=canon(ct), sky=canon(sky), dy=dy, dec=dec)
    np.savez_compressed(os.path.join(HERE, "ref_n256_l8.npz"), **out)


def c2():
    R = Reference("n4096_l784")
    rng = np.random.default_rng(0xC0FE0002)
    seed_a, seed_e, seed2 = rng.integers(0, 256, (3, 32), dtype=np.uint8)
    x = rng.integers(0, 5, R.l, dtype=np.uint32)
    y = rng.integers(0, 17, R.l, dtype=np.uint32)
    mpk, msk = R.setup(seed_a, seed_e)
    ct = R.encrypt(x, mpk, seed2)
    sky = R.keygen(y, msk)
    dy, dec = R.decrypt(ct, y, sky)
    seed3 = np.random.default_rng(0xC0FE0012).integers(0, 256, 32, dtype=np.uint8)
    q = np.array(Q, np.int64)[None, :, None]
    f_zero = canon(R.gauss(2, None, R.l)).astype(np.int64)
    f_key = canon(R.gauss(2, seed3, R.l)).astype(np.int64)
    ct_keyed = canon(ct).astype(np.int64)
    ct_keyed[:R.l] = (ct_keyed[:R.l] - f_zero + f_key) % q
    doc = {"n": R.n, "l": R.l, "seed_a": seed_a.tolist(), "seed_e": seed_e.tolist(), "seed2": seed2.tolist(),
           "x_sha": sha(x), "y_sha": sha(y), "rng": "numpy default_rng(0xC0FE0002): seeds, then x, then y",
           "mpk": sha(canon(mpk)), "msk": sha(canon(msk)), "ct": sha(canon(ct)), "sky": sha(canon(sky)),
           "dy": sha(dy), "dec": sha(dec), "ip": int(dec[0]),
           "ip_plain": int(x.astype(np.int64) @ y.astype(np.int64)),
           "seed3": seed3.tolist(), "ct_keyed": sha(ct_keyed.astype(np.uint32))}
    with open(os.path.join(HERE, "ref_c2.json"), "w") as f:
        json.dump(doc, f, indent=1)


def signed_from_residues(res):
    """the integer v with |v| < q1 q2 / 2 whose residues mod q1, q2 are res[1], res[2]; checked
    against res[0]"""
    q0, q1, q2 = Q
    r = res.astype(object)
    v = [int(a) + q1 * ((int(b) - int(a)) * pow(q1, -1, q2) % q2) for a, b in zip(r[1], r[2])]
    v = np.array([x - q1 * q2 if x > q1 * q2 // 2 else x for x in v], np.int64)
    assert ((v % q0) == res[0]).all(), "residues are not those of one integer"
    return v


def modeb():
    M = ReferenceModeB()
    keys = np.random.default_rng(0xC0FE0200).integers(0, 256, (2, 32), dtype=np.uint8)
    out = {"keys": keys}
    hashes = {}
    for k in range(2):
        for sig in range(3):
            out["poly0_k%d_s%d" % (k, sig)] = signed_from_residues(canon(M.poly(sig, keys[k], 0)))
            for bid in (1, 7, 63):
                hashes["k%d_s%d_b%d" % (k, sig, bid)] = sha(canon(M.poly(sig, keys[k], bid)))
    out["hashes"] = np.array(json.dumps(hashes, sort_keys=True))
    np.savez_compressed(os.path.join(HERE, "ref_modeb.npz"), **out)


if __name__ == "__main__":
    small()
    c2()
    modeb()
    print("golden fixtures written to", HERE)
