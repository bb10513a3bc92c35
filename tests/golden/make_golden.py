"""Generate the golden fixtures in tests/golden/ from the reference's own CPU build.

The reference (cuFE src/*.c) is compiled unmodified by oracle/ref/build_ref.py into
oracle/_ref/<variant>/libref.so; this script drives that build with fixed seeds and stores
its outputs.  Run in the build container (needs the reference tree):

    python oracle/build.py && python oracle/ref/build_ref.py --root <reference tree> &&
    python tests/golden/make_golden.py <reference tree>

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
  ref_svm_a1a.npz   svm_predict5's path end to end on the reference's shipped model and test
                    set (svm model/a1a.txt.model, a1a.t): the model's arrays as main.c reads
                    them, the 200 test vectors main.c's predict() classifies first (lines
                    101-300: it skips the first 100), the setup and encryption seeds, and per
                    vector the label and decision value of the reference's svm_predict_cpu
                    (main.c:137-267: per support vector keygen, decrypt, GMP decode, vote),
                    run at n = 2048, l = 124 by oracle/_ref/callers/libcallers.so
  ref_svm_small.npz the same prediction on a synthetic three-class model with classes of 1, 3
                    and 6 support vectors (the vote's term loops at odd and even short
                    lengths), written in libsvm's format and read by the reference's own
                    svm_load_model, 12 test vectors
  ref_modeb_setup.json  the drop-in setup at the reference's own shape (n = 4096, l = 785):
                    SHA-256 of msk and mpk when s_i and e_i come from the reference's S1 GPU
                    kernel run on the host (blocks 0..784, keys seed2 and seed3, as
                    src/rlwe_sife_gpu.cu:61-62 launches it), a from the reference CPU
                    sample_polya(seed1), and mpk_i = NTT(a) NTT(s_i) + NTT(e_i) with the
                    reference CPU NTT (src/rlwe_sife_gpu.cu:64-71)
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

from oracle.ffi import Q, Reference, ReferenceCallers, ReferenceModeB  # noqa: E402

SVM_ROWS = 200


def ref_root():
    root = os.environ.get("CUFE_REFERENCE_ROOT") or (sys.argv[1] if len(sys.argv) > 1 else None)
    if not root:
        raise SystemExit("usage: make_golden.py <reference tree> (or set CUFE_REFERENCE_ROOT)")
    return root


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


def svm_small():
    import tempfile
    sys.path.insert(0, ROOT)
    from cufe_b200 import libsvm
    R = ReferenceCallers()
    rng = np.random.default_rng(0xC0FE0301)
    nsv = np.array([1, 3, 6], np.int32)
    sv = np.zeros((int(nsv.sum()), R.l), np.uint32)
    for i in range(len(sv)):
        sv[i, rng.choice(np.arange(1, R.l), 14, replace=False)] = 1
    coef = rng.uniform(-1, 1, (2, len(sv)))
    rho = rng.uniform(-0.5, 0.5, 3)
    label = np.array([5, -2, 9], np.int32)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "small.model")
        libsvm.save_model(path, 3, sv, nsv, coef, rho, label)
        model, arr = R.load_model(path)
    assert (arr["sv"] == sv).all() and (arr["coef"] == coef).all() and (arr["rho"] == rho).all()
    seed_a, seed_e = rng.integers(0, 256, (2, 32), dtype=np.uint8)
    mpk, msk = R.setup(seed_a, seed_e)
    x = np.zeros((12, R.l), np.uint32)
    for t in range(12):
        x[t, rng.choice(np.arange(1, R.l), 14, replace=False)] = 1
    seeds2 = rng.integers(0, 256, (12, 32), dtype=np.uint8)
    labels, decs, kvs = [], [], []
    for t in range(12):
        lab, dec, kv = R.predict(model, R.encrypt(x[t], mpk, seeds2[t]), msk, 3, len(sv))
        labels.append(lab)
        decs.append(dec)
        kvs.append(kv)
    R.L.cl_free_model(model)
    np.savez_compressed(os.path.join(HERE, "ref_svm_small.npz"), n=R.n, l=R.l, label=label, nsv=nsv, rho=rho,
                        coef=coef, sv=sv.astype(np.uint8), x=x.astype(np.uint8), seed_a=seed_a, seed_e=seed_e,
                        seeds2=seeds2, ref_label=np.array(labels), ref_dec=np.array(decs),
                        ref_kvalue=np.array(kvs).astype(np.uint16))


def _modeb_block(args):
    sig, seed, bid = args
    return canon(ReferenceModeB().poly(sig, seed, bid))


def modeb_setup():
    import multiprocessing as mp
    R = Reference("default")
    n, l = R.n, R.l
    seed1, seed2, seed3 = np.random.default_rng(0xC0FE0202).integers(0, 256, (3, 32), dtype=np.uint8)
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        s = np.stack(pool.map(_modeb_block, [(0, seed2, i) for i in range(l)], chunksize=8))
        e = np.stack(pool.map(_modeb_block, [(0, seed3, i) for i in range(l)], chunksize=8))
    q = np.array(Q, np.uint64)[:, None]
    a = R.sample_polya(seed1)
    a_hat = np.stack([R.ntt(a[j], j) for j in range(3)]).astype(np.uint64) % q
    mpk = np.zeros((l + 1, 3, n), np.uint32)
    for i in range(l):
        s_hat = np.stack([R.ntt(s[i][j], j) for j in range(3)]).astype(np.uint64) % q
        e_hat = np.stack([R.ntt(e[i][j], j) for j in range(3)]).astype(np.uint64) % q
        mpk[i] = ((a_hat * s_hat % q + e_hat) % q).astype(np.uint32)
    mpk[l] = a_hat.astype(np.uint32)
    doc = {"n": n, "l": l, "seed1": seed1.tolist(), "seed2": seed2.tolist(), "seed3": seed3.tolist(),
           "a_sha": sha(canon(a)), "msk_sha": sha(s), "mpk_sha": sha(mpk)}
    with open(os.path.join(HERE, "ref_modeb_setup.json"), "w") as f:
        json.dump(doc, f, indent=1)


def _svm_init(model_path, seed_a, seed_e):
    global _R, _M, _MSK, _MPK
    _R = ReferenceCallers()
    _M, _ = _R.load_model(model_path)
    _MPK, _MSK = _R.setup(seed_a, seed_e)


def _svm_one(args):
    x, seed2 = args
    c = _R.encrypt(x, _MPK, seed2)
    label, dec, kv = _R.predict(_M, c, _MSK, 1, 591)
    return label, dec, _R.L.cl_predict_plain(_M, np.ascontiguousarray(x, np.uint32)), kv


def svm(root):
    import multiprocessing as mp
    model_path = os.path.join(root, "svm model", "a1a.txt.model")
    R = ReferenceCallers()
    model, arr = R.load_model(model_path)
    R.L.cl_free_model(model)
    assert len(arr["label"]) == 2 and len(arr["sv"]) == 591, "written for the two-class a1a model"
    rows, target = [], []
    with open(os.path.join(root, "svm model", "a1a.t")) as f:
        for g, line in enumerate(f, 1):
            if g <= 100:  # main.c's predict() skips the first 100 lines
                continue
            parts = line.split()
            x = np.zeros(R.l, np.uint32)
            for tok in parts[1:]:
                i, v = tok.split(":")
                x[int(i)] = int(float(v))
            rows.append(x)
            target.append(int(float(parts[0])))
            if len(rows) == SVM_ROWS:
                break
    rng = np.random.default_rng(0xC0FE0300)
    seed_a, seed_e = rng.integers(0, 256, (2, 32), dtype=np.uint8)
    seeds2 = rng.integers(0, 256, (SVM_ROWS, 32), dtype=np.uint8)
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1), _svm_init, (model_path, seed_a, seed_e)) as pool:
        res = pool.map(_svm_one, list(zip(rows, seeds2)), chunksize=4)
    np.savez_compressed(os.path.join(HERE, "ref_svm_a1a.npz"), n=R.n, l=R.l, label=arr["label"], nsv=arr["nsv"],
                        rho=arr["rho"], coef=arr["coef"], sv=arr["sv"].astype(np.uint8),
                        x=np.stack(rows).astype(np.uint8), target=np.array(target, np.int8), seed_a=seed_a,
                        seed_e=seed_e, seeds2=seeds2, ref_label=np.array([r[0] for r in res]),
                        ref_dec=np.array([r[1] for r in res]), plain_label=np.array([r[2] for r in res]),
                        ref_kvalue=np.array([r[3] for r in res]).astype(np.uint16))


if __name__ == "__main__":
    root = ref_root()
    small()
    c2()
    modeb()
    modeb_setup()
    svm(root)
    svm_small()
    print("golden fixtures written to", HERE)
