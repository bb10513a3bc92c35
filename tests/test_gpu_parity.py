"""Parity of the CUDA path (through the C ABI) with the oracle, on a GPU.

The oracle (oracle/cufe_oracle.c) is pinned bit-for-bit to the reference's own CPU build
(tests/test_oracle.py); residues are compared canonically (the reference's mod_prime may
return q_j for 0).
"""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle.ffi import Oracle, canon, aes256_expand
from tests.conftest import seeds

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import cufe_b200 as cf  # noqa: E402


def dev(a):
    return cf.to_dev(a)


@pytest.fixture(scope="module")
def ctx_small(oracle_built):
    c = cf.Context(256, 8)
    yield c
    c.close()


@pytest.mark.parametrize("variant", list(range(1, cf.NTT_VARIANTS + 1)))
@pytest.mark.parametrize("n", [16, 64, 256, 1024, 2048, 4096, 8192])
@pytest.mark.parametrize("k", [3, 6])
def test_ntt_roundtrip_and_values(n, k, variant, rng, oracle_built):
    ring = cf.Ring(n, k)
    ring.set_variant(variant, variant)
    assert ring.variant == (variant, variant)
    npoly = 5  # odd: variant 2 leaves one residue pair half empty
    q = ring.primes.astype(np.uint64)
    a = (rng.integers(0, 2**31, (npoly, k, n), dtype=np.uint64) % q[None, :, None]).astype(np.uint32)
    d = dev(a)
    ring.forward(d)
    got = cf.u32(d)
    O = Oracle.lib()
    for p in range(npoly):
        for m in range(k):
            ref = a[p, m].copy()
            O.or_ntt_generic(ref, n, int(q[m]), np.ascontiguousarray(ring.psi[m]), 0, 0)
            assert (got[p, m] == ref).all(), (n, k, p, m)
    ring.inverse(d)
    assert (cf.u32(d) == a).all()


def test_ring_tune(rng):
    ring = cf.Ring(4096, 3)
    t = ring.tune(64)
    assert all(v > 0 for v in t["fwd"] + t["inv"])
    best = (1 + int(np.argmin(t["fwd"])), 1 + int(np.argmin(t["inv"])))
    assert ring.variant == best == t["variant"]
    q = ring.primes.astype(np.uint64)
    a = (rng.integers(0, 2**31, (7, 3, 4096), dtype=np.uint64) % q[None, :, None]).astype(np.uint32)
    d = dev(a)
    ring.forward(d)
    ring.inverse(d)
    assert (cf.u32(d) == a).all()


def test_ntt_tables_match_reference_chain(oracle_built):
    # the params.h primes use the reference twiddle chain (consts.h), checked via the oracle
    for n in (256, 4096):
        ring = cf.Ring(n, 3)
        t = Oracle(n, 1).tables()
        assert (ring.psi == t["psi"]).all() and (ring.psi_inv == t["psi_inv"]).all()


def test_sample_polya(ctx_small, rng):
    s = seeds(rng)[0]
    got = cf.u32(ctx_small.sample_polya(s))
    torch.cuda.synchronize()
    assert (got == Oracle(256, 8).sample_polya(s)).all()


@pytest.mark.parametrize("sig", [0, 1, 2])
def test_sampler_cpu_map(sig, rng, oracle_built):
    n = 1024
    c = cf.Context(n, 4)
    keys = seeds(rng, 3)
    calls = 5
    got = cf.u32(c.sample_cpu_map(sig, keys, calls))
    zero = cf.u32(c.sample_cpu_map(sig, None, calls, nstreams=2))
    c.sync()
    O = Oracle(n, 4)
    for i in range(3):
        ref, _ = O.gauss(sig, keys[i], calls)
        assert (got[i] == canon(ref)).all(), (sig, i)
    ref, _ = O.gauss(sig, None, calls)
    assert (zero[0] == canon(ref)).all() and (zero[1] == canon(ref)).all()


@pytest.mark.parametrize("sig", [0, 1, 2])
def test_call_search_walk_equals_doubling(sig, rng, oracle_built):
    """the call-start searches (cost rule, walk, doubling) give the same samples (uniform
    streams, and uneven ones through a heterogeneous batch)"""
    L = cf.lib()
    assert L.cufe_sampler_call_search(3) != 0  # modes are 0, 1, 2
    c = cf.Context(1024, 8)
    keys = seeds(rng, 5)
    outs = []
    for mode in (0, 1, 2):
        assert L.cufe_sampler_call_search(mode) == 0
        outs.append(cf.u32(c.sample_cpu_map(sig, keys, 37)))
        c.sync()
    assert L.cufe_sampler_call_search(0) == 0
    assert (outs[0] == outs[1]).all() and (outs[0] == outs[2]).all()
    c.close()
    if sig == 2:
        ns, ls = [256, 1024, 512], [5, 33, 12]
        res = []
        for mode in (1, 2):
            L.cufe_sampler_call_search(mode)
            B = cf.Batch(ns, ls)
            r = np.random.default_rng(9)
            B.setup(r.integers(0, 256, (3, 32), dtype=np.uint8), None, r.integers(0, 256, (3, 32), dtype=np.uint8))
            x = dev(B.pack([r.integers(0, 5, l) for l in ls]).astype(np.uint32))
            y = dev(B.pack([r.integers(-16, 17, l) for l in ls]).astype(np.int32))
            d0 = dev(np.zeros((3, 3), np.uint32))
            B.bind(x, y, cf.bytes_to_dev(r.integers(0, 256, (3, 32), dtype=np.uint8)),
                   cf.bytes_to_dev(r.integers(0, 256, (3, 32), dtype=np.uint8)), d0=d0)
            B.run()
            torch.cuda.synchronize()
            res.append([B.fetch(B.instance(i)[3], (l + 1) * 3 * n) for i, (n, l) in enumerate(zip(ns, ls))])
            B.close()
        L.cufe_sampler_call_search(0)
        for a, b in zip(*res):
            assert (a == b).all()


@pytest.mark.parametrize("sig", [0, 1, 2])
def test_sampler_gpu_map(sig, rng, oracle_built):
    n = 4096
    c = cf.Context(n, 4)
    key = seeds(rng)[0]
    got = cf.u32(c.sample_gpu_map(sig, key, 2, 3))
    c.sync()
    O = Oracle(n, 4)
    rk = aes256_expand(key)
    for p in range(3):
        assert (got[p] == canon(O.gauss_modeB(rk, sig, 2 + p))).all(), (sig, p)


@pytest.mark.parametrize("n,l", [(256, 8), (1024, 16), (2048, 124), (4096, 16), (8192, 8)])
def test_scheme_cpu_map(n, l, rng, oracle_built):
    c = cf.Context(n, l)
    O = Oracle(n, l)
    sa, se, ss = seeds(rng, 3)
    mpk, msk = c.setup(sa, None, se)
    rmpk, rmsk = O.setup(sa, None, se)
    assert (cf.u32(mpk) == canon(rmpk)).all()
    assert (cf.u32(msk) == canon(rmsk)).all()
    # seeded secret stream too
    mpk2, msk2 = c.setup(sa, ss, se)
    r2mpk, r2msk = O.setup(sa, ss, se)
    assert (cf.u32(mpk2) == canon(r2mpk)).all() and (cf.u32(msk2) == canon(r2msk)).all()
    B = 3
    x = rng.integers(0, 5, (B, l), dtype=np.uint32)
    s2 = seeds(rng, B)
    s3 = seeds(rng, B)
    ct = c.encrypt(dev(x), mpk, s2, None)
    ct3 = c.encrypt(dev(x), mpk, s2, s3)
    got, got3 = cf.u32(ct), cf.u32(ct3)
    y = rng.integers(0, 17, (2, l), dtype=np.uint32)
    sky = c.keygen(dev(y), msk)
    gsky = cf.u32(sky)
    dy = c.decrypt(ct, dev(y), sky)
    gdy = cf.u32(dy)
    dec = cf.u32(c.decode(dy))
    c.sync()
    for b in range(B):
        rct = O.encrypt(x[b], rmpk, s2[b], None)
        assert (got[b] == canon(rct)).all(), ("ct", b)
        assert (got3[b] == canon(O.encrypt(x[b], rmpk, s2[b], s3[b]))).all(), ("ct3", b)
        for k in range(2):
            rsk = O.keygen(y[k], rmsk)
            if b == 0:
                assert (gsky[k] == canon(rsk)).all()
            rdy = O.decrypt(rct, y[k], rsk)
            assert (gdy[b, k] == canon(rdy)).all(), ("dy", b, k)
            rdec = O.decode(rdy)
            assert (dec[b * 2 + k] == rdec).all()
            assert int(rdec[0]) == int(x[b].astype(np.int64) @ y[k].astype(np.int64))


def test_c2_shape_golden_hashes():
    """setup / encrypt / keygen / decrypt / decode at n = 4096, l = 784 against the SHA-256 of
    the reference CPU build's outputs for the same seeds (tests/golden/ref_c2.json)"""
    doc = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ref_c2.json")))
    n, l = doc["n"], doc["l"]
    rng = np.random.default_rng(0xC0FE0002)
    seed_a, seed_e, seed2 = rng.integers(0, 256, (3, 32), dtype=np.uint8)
    x = rng.integers(0, 5, l, dtype=np.uint32)
    y = rng.integers(0, 17, l, dtype=np.uint32)
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a, np.uint32).tobytes()).hexdigest()  # noqa: E731
    c = cf.Context(n, l)
    mpk, msk = c.setup(seed_a, None, seed_e)
    ct = c.encrypt(dev(x[None]), mpk, seed2[None], None)
    sky = c.keygen(dev(y[None]), msk)
    dy = c.decrypt(ct, dev(y[None]), sky)
    dec = c.decode(dy)
    c.sync()
    assert sha(cf.u32(mpk)) == doc["mpk"] and sha(cf.u32(msk)) == doc["msk"]
    assert sha(cf.u32(ct)[0]) == doc["ct"]
    assert sha(cf.u32(sky)[0]) == doc["sky"]
    assert sha(cf.u32(dy)[0, 0]) == doc["dy"]
    d = cf.u32(dec)
    assert sha(d[0]) == doc["dec"] and int(d[0][0]) == doc["ip"]
    # the same encryption with f_i drawn from the sigma_3 stream keyed by seed3 (as in the bench)
    ct3 = c.encrypt(dev(x[None]), mpk, seed2[None], np.array(doc["seed3"], np.uint8)[None])
    c.sync()
    assert sha(cf.u32(ct3)[0]) == doc["ct_keyed"]
    c.close()


def test_sampler_gpu_map_golden():
    """k_gauss_gpu_map against the reference's own GPU sampler kernels run on the host
    (tests/golden/ref_modeb.npz): polynomial 0 in full, polynomials 1, 7, 63 by hash, every
    sigma, two keys"""
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_modeb.npz"))
    hashes = json.loads(str(g["hashes"]))
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a, np.uint32).tobytes()).hexdigest()  # noqa: E731
    q = np.array([16760833, 2147352577, 2130706433], np.int64)
    c = cf.Context(4096, 4)
    for k in range(2):
        for sig in range(3):
            got = cf.u32(c.sample_gpu_map(sig, g["keys"][k], 0, 64))
            c.sync()
            v = g["poly0_k%d_s%d" % (k, sig)].astype(np.int64)
            want = np.stack([(v % qq).astype(np.uint32) for qq in q])
            assert (canon(got[0]) == want).all(), (k, sig)
            for bid in (1, 7, 63):
                assert sha(canon(got[bid])) == hashes["k%d_s%d_b%d" % (k, sig, bid)], (k, sig, bid)
    c.close()


@pytest.mark.parametrize("n,l", [(256, 8), (2048, 124), (4096, 784)])
def test_decrypt_coef0(n, l, rng, oracle_built):
    """the constant-coefficient decrypt equals coefficient 0 of the full decrypt and its decode,
    for uint32 (reference) and signed y; at n = 256 also the oracle's decrypt"""
    c = cf.Context(n, l)
    sa, se = seeds(rng, 2)
    mpk, msk = c.setup(sa, None, se)
    B, K = 3, 4
    x = rng.integers(0, 5, (B, l), dtype=np.uint32)
    s2 = seeds(rng, B)
    ct = c.encrypt(dev(x), mpk, s2, None)
    p = 64 * l + 1
    for signed in (False, True):
        if signed:
            yi = rng.integers(-16, 17, (K, l), dtype=np.int64)
            y = yi.astype(np.int32).view(np.uint32)
        else:
            y = rng.integers(0, 17, (K, l), dtype=np.uint32)
            yi = y.astype(np.int64)
        yd = dev(y)
        sky = c.keygen(yd, msk, y_signed=signed)
        dy = c.decrypt(ct, yd, sky, y_signed=signed)
        full = cf.u32(c.decode(dy, ncoeff=1)).reshape(B, K)
        d0 = dev(np.zeros((B, K, 3), np.uint32))
        got = cf.u32(c.decrypt_coef0(ct, yd, sky, y_signed=signed, d0=d0))
        c.sync()
        assert (cf.u32(d0) == cf.u32(dy)[:, :, :, 0]).all()
        assert (got == full).all()
        assert (got.astype(np.int64) % p == (x.astype(np.int64) @ yi.T) % p).all()
        if n == 256 and not signed:
            O = Oracle(n, l)
            rmpk, rmsk = O.setup(sa, None, se)
            for b in range(B):
                rct = O.encrypt(x[b], rmpk, s2[b], None)
                for k in range(K):
                    assert int(got[b, k]) == int(O.decode(O.decrypt(rct, y[k], O.keygen(y[k], rmsk)))[0])
    c.close()


@pytest.mark.parametrize("n,l,B,K", [(256, 8, 70, 33), (2048, 124, 5, 129), (4096, 40, 65, 64)])
def test_decrypt_coef0_tiled(n, l, B, K, rng, oracle_built):
    """from 32 keys the constant-coefficient decrypt runs as a tiled product over K = l + n;
    its residues and decoded values must equal the one-CTA-per-pair kernel's (keys passed
    one at a time), for ragged tiles and for uint32 and signed y"""
    c = cf.Context(n, l)
    sa, se = seeds(rng, 2)
    mpk, msk = c.setup(sa, None, se)
    x = rng.integers(0, 5, (B, l), dtype=np.uint32)
    ct = c.encrypt(dev(x), mpk, seeds(rng, B), None)
    p = 64 * l + 1
    for signed in (False, True):
        if signed:
            yi = rng.integers(-16, 17, (K, l), dtype=np.int64)
            y = yi.astype(np.int32).view(np.uint32)
        else:
            y = rng.integers(0, 17, (K, l), dtype=np.uint32)
            yi = y.astype(np.int64)
        yd = dev(y)
        sky = c.keygen(yd, msk, y_signed=signed)
        d0 = dev(np.zeros((B, K, 3), np.uint32))
        got = cf.u32(c.decrypt_coef0(ct, yd, sky, y_signed=signed, d0=d0))
        got_nod0 = cf.u32(c.decrypt_coef0(ct, yd, sky, y_signed=signed))  # workspace for the residues
        c.sync()
        d0h = cf.u32(d0)
        for k in range(K):
            r0 = dev(np.zeros((B, 1, 3), np.uint32))
            one = cf.u32(c.decrypt_coef0(ct, yd[k:k + 1], sky[k:k + 1], y_signed=signed, d0=r0))
            c.sync()
            assert (d0h[:, k] == cf.u32(r0)[:, 0]).all(), (signed, k)
            assert (got[:, k] == one[:, 0]).all(), (signed, k)
        assert (got_nod0 == got).all()
        ip = (x.astype(np.int64) @ yi.T) % p
        assert (got.astype(np.int64) % p == ip).all()
    c.close()


def test_scheme_gpu_map(rng, oracle_built):
    n, l = 1024, 16
    c = cf.Context(n, l)
    O = Oracle(n, l)
    a = O.sample_polya(seeds(rng)[0])
    s2, s3 = seeds(rng, 2)
    mpk, msk = c.setup_gpu_map(dev(a), s2, s3)
    rmpk, rmsk = O.setup_modeB(a, s2, s3)
    assert (cf.u32(mpk) == canon(rmpk)).all() and (cf.u32(msk) == canon(rmsk)).all()
    x = rng.integers(0, 5, (3, l), dtype=np.uint32)
    ct = cf.u32(c.encrypt_gpu_map(dev(x), mpk, s2))
    c.sync()
    assert (ct == canon(O.encrypt_modeB(x, rmpk, s2))).all()


def test_decode_random_residues(ctx_small, rng):
    n = 256
    q = np.array(cf.Q, np.uint64)
    dy = (rng.integers(0, 2**62, (4, 3, n), dtype=np.uint64) % q[None, :, None]).astype(np.uint32)
    got = cf.u32(ctx_small.decode(dev(dy)))
    ctx_small.sync()
    O = Oracle(n, 8)
    for i in range(4):
        assert (got[i] == O.decode(dy[i])).all()


def test_dropin_abi(rng, oracle_built):
    """the reference's four GPU symbols, host buffers, GPU counter mapping"""
    import ctypes as C
    n, l = 1024, 16
    L = cf.lib()
    assert L.cufe_dropin_configure(n, l, 0) == 0
    O = Oracle(n, l)
    s2, s3 = seeds(rng, 2)
    mpk = np.zeros((l + 1, 3, n), np.uint32)
    msk = np.zeros((l, 3, n), np.uint32)
    mpk[l] = O.sample_polya(seeds(rng)[0])
    a = mpk[l].copy()
    t = C.c_float(0)
    L.rlwe_sife_setup_gpu(mpk.ctypes.data, msk.ctypes.data, s2.ctypes.data, s3.ctypes.data, C.byref(t))
    assert L.cufe_dropin_status() == 0
    rmpk, rmsk = O.setup_modeB(a, s2, s3)
    assert (mpk == canon(rmpk)).all() and (msk == canon(rmsk)).all()
    assert t.value > 0
    rep = 2
    x = rng.integers(0, 5, (rep, l), dtype=np.uint32)
    ct = np.zeros((rep, l + 1, 3, n), np.uint32)
    L.rlwe_sife_encrypt_gpu(x.ctypes.data, mpk.ctypes.data, ct.ctypes.data, s2.ctypes.data, s2.ctypes.data, rep, None)
    assert (ct == canon(O.encrypt_modeB(x, rmpk, s2))).all()
    y = rng.integers(0, 17, (3, l), dtype=np.uint32)
    sk = np.zeros((3, 3, n), np.uint32)
    L.rlwe_sife_keygen_gpu(y.ctypes.data, msk.ctypes.data, sk.ctypes.data, 3, None)
    dy = np.zeros((3, 3, n), np.uint32)
    L.rlwe_sife_decrypt_gmp_gpu(ct[0].ctypes.data, y.ctypes.data, sk.ctypes.data, dy.ctypes.data, 3, None)
    assert L.cufe_dropin_status() == 0
    for k in range(3):
        rsk = O.keygen(y[k], rmsk)
        assert (sk[k] == canon(rsk)).all()
        rdy = O.decrypt(ct[0], y[k], rsk)
        assert (dy[k] == canon(rdy)).all()
        assert int(O.decode(rdy)[0]) == int(x[0].astype(np.int64) @ y[k].astype(np.int64))


def test_dropin_setup_at_the_reference_shape(oracle_built):
    """rlwe_sife_setup_gpu at the reference's compile-time shape (n 4096, l 785, the default
    configuration) against tests/golden/ref_modeb_setup.json, made from the reference's own S1
    GPU kernel (run on the host), CPU sample_polya and CPU NTT"""
    import ctypes as C
    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ref_modeb_setup.json")))
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a, np.uint32).tobytes()).hexdigest()  # noqa: E731
    n, l = d["n"], d["l"]
    L = cf.lib()
    assert L.cufe_dropin_configure(n, l, 0) == 0
    mpk = np.zeros((l + 1, 3, n), np.uint32)
    msk = np.zeros((l, 3, n), np.uint32)
    mpk[l] = Oracle(n, 1).sample_polya(np.array(d["seed1"], np.uint8))
    assert sha(canon(mpk[l])) == d["a_sha"]
    s2, s3 = np.array(d["seed2"], np.uint8), np.array(d["seed3"], np.uint8)
    t = C.c_float(0)
    L.rlwe_sife_setup_gpu(mpk.ctypes.data, msk.ctypes.data, s2.ctypes.data, s3.ctypes.data, C.byref(t))
    assert L.cufe_dropin_status() == 0
    assert sha(msk) == d["msk_sha"] and sha(mpk) == d["mpk_sha"]


def test_dropin_staged_copies(rng, oracle_built):
    """the drop-in symbols at sizes that take the pinned, chunked host copies (mpk and msk
    of 9.8 MB, two ciphertexts of 19.7 MB: ragged last chunks), against the context API on
    device buffers with the same seeds"""
    n, l = 2048, 400
    L = cf.lib()
    assert L.cufe_dropin_configure(n, l, 0) == 0
    s2, s3 = seeds(rng, 2)
    a = rng.integers(0, 2**31, (3, n), dtype=np.uint64) % np.array(cf.Q, np.uint64)[:, None]
    mpk = np.zeros((l + 1, 3, n), np.uint32)
    msk = np.zeros((l, 3, n), np.uint32)
    mpk[l] = a.astype(np.uint32)
    L.rlwe_sife_setup_gpu(mpk.ctypes.data, msk.ctypes.data, s2.ctypes.data, s3.ctypes.data, None)
    assert L.cufe_dropin_status() == 0
    c = cf.Context(n, l)
    dmpk, dmsk = c.setup_gpu_map(a.astype(np.uint32), s2, s3)
    c.sync()
    assert (mpk == cf.u32(dmpk)).all() and (msk == cf.u32(dmsk)).all()
    rep = 2
    x = rng.integers(0, 5, (rep, l), dtype=np.uint32)
    ct = np.zeros((rep, l + 1, 3, n), np.uint32)
    L.rlwe_sife_encrypt_gpu(x.ctypes.data, mpk.ctypes.data, ct.ctypes.data, s2.ctypes.data, s2.ctypes.data, rep, None)
    assert L.cufe_dropin_status() == 0
    dct = c.encrypt_gpu_map(dev(x), dmpk, s2)
    y = rng.integers(0, 17, (2, l), dtype=np.uint32)
    sk = np.zeros((2, 3, n), np.uint32)
    L.rlwe_sife_keygen_gpu(y.ctypes.data, msk.ctypes.data, sk.ctypes.data, 2, None)
    dy = np.zeros((2, 3, n), np.uint32)
    L.rlwe_sife_decrypt_gmp_gpu(ct[1].ctypes.data, y.ctypes.data, sk.ctypes.data, dy.ctypes.data, 2, None)
    assert L.cufe_dropin_status() == 0
    dsk = c.keygen(dev(y), dmsk)
    ddy = c.decrypt(dct[1:2], dev(y), dsk)
    c.sync()
    assert (ct == cf.u32(dct)).all()
    assert (sk == cf.u32(dsk)).all()
    assert (dy == cf.u32(ddy)[0]).all()
    dec = cf.u32(c.decode(ddy, ncoeff=1)).reshape(2)
    assert (dec.astype(np.int64) == (x[1].astype(np.int64) @ y.T.astype(np.int64))).all()
    c.close()
