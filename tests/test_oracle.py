"""The oracle (oracle/cufe_oracle.c) against the reference's own CPU build: committed golden
fixtures (tests/golden/, made by make_golden.py from oracle/_ref) and, where the compiled
reference is present, fresh random cases.  CPU only."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle.ffi import Oracle, Q, aes256_block, aes256_expand, canon, ctr_stream

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def gold(oracle_built):
    d = np.load(os.path.join(GOLD, "ref_n256_l8.npz"))
    return {k: d[k] for k in d.files}


def test_aes256_fips197_kat(oracle_built):
    # FIPS-197 appendix C.3
    key = np.arange(32, dtype=np.uint8)
    pt = np.frombuffer(bytes.fromhex("00112233445566778899aabbccddeeff"), np.uint8)
    ct = aes256_block(aes256_expand(key), pt)
    assert bytes(ct).hex() == "8ea2b7ca516745bfeafc49904b496089"


def test_aes256_random_keys_match_cryptography(oracle_built):
    mod = pytest.importorskip("cryptography.hazmat.primitives.ciphers")
    rng = np.random.default_rng(1)
    for _ in range(20):
        key = rng.integers(0, 256, 32, dtype=np.uint8)
        pt = rng.integers(0, 256, 16, dtype=np.uint8)
        enc = mod.Cipher(mod.algorithms.AES(bytes(key)), mod.modes.ECB()).encryptor()
        assert bytes(aes256_block(aes256_expand(key), pt)) == enc.update(bytes(pt)) + enc.finalize()


def test_ctr_streams(gold):
    assert (ctr_stream(gold["ctr_key"], 2) == gold["ctr_keyed"]).all()
    assert (ctr_stream(None, 2) == gold["ctr_zero"]).all()


def test_ntt_vectors(gold):
    O = Oracle(256, 8)
    for sel in range(3):
        a = gold["ntt_in_%d" % sel]
        assert (O.ntt(a, sel) == gold["ntt_fwd_%d" % sel]).all()
        assert (O.ntt(a, sel, inverse=True) == gold["ntt_inv_%d" % sel]).all()


@pytest.mark.parametrize("sig", [0, 1, 2])
def test_sampler_streams(gold, sig):
    O = Oracle(256, 8)
    got, _ = O.gauss(sig, gold["ctr_key"], 4)
    assert (canon(got) == gold["gauss_key_%d" % sig]).all()
    got, _ = O.gauss(sig, None, 4)
    assert (canon(got) == gold["gauss_zero_%d" % sig]).all()


def test_scheme_round_trip(gold):
    O = Oracle(256, 8)
    assert (O.sample_polya(gold["polya_seed"]) == gold["polya"]).all()
    mpk, msk = O.setup(gold["seed_a"], None, gold["seed_e"])
    assert (canon(mpk) == gold["mpk"]).all() and (canon(msk) == gold["msk"]).all()
    ct = O.encrypt(gold["x"], mpk, gold["seed2"], None)
    assert (canon(ct) == gold["ct"]).all()
    sky = O.keygen(gold["y"], msk)
    assert (canon(sky) == gold["sky"]).all()
    dy = O.decrypt(ct, gold["y"], sky)
    assert (canon(dy) == gold["dy"]).all()
    dec = O.decode(dy)
    assert (dec == gold["dec"]).all()
    assert int(dec[0]) == int(gold["x"].astype(np.int64) @ gold["y"].astype(np.int64))


@pytest.mark.slow
def test_c2_shape_hashes(oracle_built):
    doc = json.load(open(os.path.join(GOLD, "ref_c2.json")))
    n, l = doc["n"], doc["l"]
    rng = np.random.default_rng(0xC0FE0002)
    seed_a, seed_e, seed2 = rng.integers(0, 256, (3, 32), dtype=np.uint8)
    x = rng.integers(0, 5, l, dtype=np.uint32)
    y = rng.integers(0, 17, l, dtype=np.uint32)
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a, np.uint32).tobytes()).hexdigest()  # noqa: E731
    O = Oracle(n, l)
    mpk, msk = O.setup(seed_a, None, seed_e)
    assert sha(canon(mpk)) == doc["mpk"] and sha(canon(msk)) == doc["msk"]
    ct = O.encrypt(x, mpk, seed2, None)
    assert sha(canon(ct)) == doc["ct"]
    sky = O.keygen(y, msk)
    dy = O.decrypt(ct, y, sky)
    assert sha(canon(sky)) == doc["sky"] and sha(canon(dy)) == doc["dy"]
    dec = O.decode(dy)
    assert sha(dec) == doc["dec"] and int(dec[0]) == doc["ip"] == doc["ip_plain"]
    # f_i drawn from the sigma_3 stream keyed by seed3 (the bench's encryptions)
    ct3 = O.encrypt(x, mpk, seed2, np.array(doc["seed3"], np.uint8))
    assert sha(canon(ct3)) == doc["ct_keyed"]


def _modeb_gold():
    d = np.load(os.path.join(GOLD, "ref_modeb.npz"))
    return {k: d[k] for k in d.files}


def residues(v):
    """canonical residues [3][n] of signed integers v"""
    return np.stack([(v.astype(np.int64) % q).astype(np.uint32) for q in Q])


def test_modeb_golden(oracle_built):
    """the oracle's GPU counter mapping (mode B) against the reference's own GPU sampler kernels
    run on the host (tests/golden/ref_modeb.npz): polynomial 0 of every sigma for two keys in
    full, polynomials 1, 7 and 63 by hash"""
    g = _modeb_gold()
    hashes = json.loads(str(g["hashes"]))
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a, np.uint32).tobytes()).hexdigest()  # noqa: E731
    O = Oracle(4096, 4)
    for k in range(2):
        rk = aes256_expand(g["keys"][k])
        for sig in range(3):
            assert (canon(O.gauss_modeB(rk, sig, 0)) == residues(g["poly0_k%d_s%d" % (k, sig)])).all(), (k, sig)
            for bid in (1, 7, 63):
                assert sha(canon(O.gauss_modeB(rk, sig, bid))) == hashes["k%d_s%d_b%d" % (k, sig, bid)], (k, sig, bid)


@pytest.mark.slow
def test_modeb_setup_reference_shape(oracle_built):
    """setup in the GPU counter mapping at the reference's own shape (n 4096, l 785) against
    tests/golden/ref_modeb_setup.json: s_i, e_i from the reference's S1 GPU kernel run on the
    host, a from its CPU sample_polya, mpk through its CPU NTT"""
    d = json.load(open(os.path.join(GOLD, "ref_modeb_setup.json")))
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a, np.uint32).tobytes()).hexdigest()  # noqa: E731
    O = Oracle(d["n"], d["l"])
    a = O.sample_polya(np.array(d["seed1"], np.uint8))
    assert sha(canon(a)) == d["a_sha"]
    mpk, msk = O.setup_modeB(a, np.array(d["seed2"], np.uint8), np.array(d["seed3"], np.uint8))
    assert sha(canon(msk)) == d["msk_sha"] and sha(canon(mpk)) == d["mpk_sha"]


def _have_modeb():
    return os.path.exists(os.path.join(os.path.dirname(GOLD), "..", "oracle", "_ref", "modeb", "libmodeb.so"))


@pytest.mark.skipif(not _have_modeb(), reason="host build of the reference GPU sampler not present")
def test_modeb_random_keys_against_reference_kernels(oracle_built):
    """fresh keys and polynomial indices: the oracle's mode B equals the reference's kernels
    (src/sample_gpu.cu) run on the host, and its key schedule equals AESPrepareKey"""
    from oracle.ffi import ReferenceModeB
    M = ReferenceModeB()
    O = Oracle(4096, 4)
    rng = np.random.default_rng(0xC0FE0201)
    for trial in range(3):
        key = rng.integers(0, 256, 32, dtype=np.uint8)
        rk = aes256_expand(key)
        for sig in range(3):
            bid = int(rng.integers(0, 64))
            assert (canon(M.poly(sig, key, bid)) == canon(O.gauss_modeB(rk, sig, bid))).all(), (trial, sig, bid)


def test_parameters(oracle_built):
    for n in (16, 256, 2048, 4096):
        t = Oracle(n, 8).tables()
        t4 = Oracle(4096, 8).tables()
        assert (t["psi"] == t4["psi"][:, :n]).all()  # one chain of tables for every n
        for j, q in enumerate(Q):
            assert pow(int(t["psi"][j][n // 2]), n, q) == q - 1  # primitive 2n-th root
            assert int(t["ninv"][j]) * n % q == 1
    t = Oracle(256, 785).tables()
    assert t["p"] == 50241 and t["q"] == 76687145727357674227351553
    assert t["delta"] == 1526385735302993058007  # src/params.h:27-28 values for l = 785
    assert list(t["delta_mod"]) == [13798054, 441557681, 1912932552]


def _have_ref(variant):
    return os.path.exists(os.path.join(os.path.dirname(GOLD), "..", "oracle", "_ref", variant, "libref.so"))


@pytest.mark.skipif(not _have_ref("n1024_l16"), reason="reference CPU build not present")
def test_random_cases_against_reference_build(oracle_built):
    from oracle.ffi import Reference
    R = Reference("n1024_l16")
    O = Oracle(1024, 16)
    rng = np.random.default_rng(99)
    for trial in range(3):
        sa, se, s2 = rng.integers(0, 256, (3, 32), dtype=np.uint8)
        mpk, msk = R.setup(sa, se)
        omp, oms = O.setup(sa, None, se)
        assert (mpk == omp).all() and (msk == oms).all()
        x = rng.integers(0, 5, 16, dtype=np.uint32)
        y = rng.integers(0, 17, 16, dtype=np.uint32)
        ct = R.encrypt(x, mpk, s2)
        assert (ct == O.encrypt(x, omp, s2, None)).all()
        sk = R.keygen(y, msk)
        assert (sk == O.keygen(y, oms)).all()
        dy, dec = R.decrypt(ct, y, sk)
        ody = O.decrypt(ct, y, sk)
        assert (dy == canon(ody)).all() and (dec == O.decode(ody)).all()
    for sig in range(3):
        key = rng.integers(0, 256, 32, dtype=np.uint8)
        assert (R.gauss(sig, key, 20) == O.gauss(sig, key, 20)[0]).all()


def test_sampler_shapes(oracle_built):
    """pins what the reference's samplers draw: sigma_1 is D_{Z,sigma_1}; sigma_2 and sigma_3
    are not (their Bernoulli input conversion is exact only below 2^52), with standard
    deviations 1.13 and 0.73 of K sigma_0"""
    import torch
    from cufe_b200.stats import ChiSquare, sigma_of, signed_samples
    O = Oracle(1024, 8)
    rng = np.random.default_rng(0xC0FE0004)
    ratios = []
    for sig in range(3):
        acc = ChiSquare(sigma_of(sig), 100)
        xs = []
        for _ in range(8):
            r, _ = O.gauss(sig, rng.integers(0, 256, 32, dtype=np.uint8), 32)
            x = signed_samples(torch.from_numpy(r.view(np.int32)))
            acc.add(x)
            xs.append(x.numpy())
        ratios.append(float(np.concatenate(xs).astype(np.float64).std() / sigma_of(sig)))
        p = acc.result()["p_value"]
        assert (p > 1e-6) if sig == 0 else (p < 1e-12), (sig, p)
    assert abs(ratios[0] - 1) < 0.01 and abs(ratios[1] - 1.13) < 0.02 and abs(ratios[2] - 0.73) < 0.02, ratios
