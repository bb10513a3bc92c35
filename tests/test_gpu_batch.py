"""Heterogeneous batches (cufe_batch_*): instances of different ring degree and vector length,
each with its own keys, stepped together.

Per instance the batch must give what the single-instance path gives: keys and ciphertexts
equal to the oracle's for the same seeds (the oracle is pinned to the reference CPU build),
function keys and coefficient-0 residues equal to the context API's signed-y path, and the
decoded inner product equal to the plaintext dot product mod p_i.  Also: several chunks give
the same results as one, and a CUDA-graph replay equals an eager step, including after new
seeds are written into the bound buffers.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle.ffi import Oracle, canon
from tests.conftest import seeds

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import cufe_b200 as cf  # noqa: E402

NS = [256, 1024, 256, 512, 1024, 256, 2048]
LS = [8, 5, 17, 12, 3, 30, 9]


def dev(a):
    return cf.to_dev(a)


def make(rng, chunk_bytes):
    B = cf.Batch(NS, LS, max_chunk_bytes=chunk_bytes)
    cnt = B.count
    sa, se = seeds(rng, cnt), seeds(rng, cnt)
    B.setup(sa, None, se)
    xs = [rng.integers(0, 5, l, dtype=np.int64) for l in LS]
    ys = [rng.integers(-16, 17, l, dtype=np.int64) for l in LS]
    x = dev(B.pack(xs).astype(np.uint32))
    y = dev(B.pack(ys).astype(np.int32))
    s2, s3 = seeds(rng, cnt), seeds(rng, cnt)
    d0 = dev(np.zeros((cnt, 3), np.uint32))
    s2d, s3d = cf.bytes_to_dev(s2), cf.bytes_to_dev(s3)
    out = B.bind(x, y, s2d, s3d, d0=d0)
    return B, (sa, se, xs, ys, s2, s3), (out, d0, s2d, s3d)


@pytest.mark.parametrize("chunked", [False, True])
def test_batch_matches_single_instance_paths(chunked, rng, oracle_built):
    B, (sa, se, xs, ys, s2, s3), (out, d0, _, _) = make(rng, 1 << 20 if chunked else 0)
    assert (B.chunks > 1) == chunked
    B.run()
    torch.cuda.synchronize()
    B.status()
    got, got_d0 = cf.u32(out), cf.u32(d0)
    for i, (n, l) in enumerate(zip(NS, LS)):
        O = Oracle(n, l)
        rmpk, rmsk = O.setup(sa[i], None, se[i])
        mpk_a, msk_a, sky_a, ct_a = B.instance(i)
        assert (B.fetch(mpk_a, (l + 1) * 3 * n).reshape(l + 1, 3, n) == canon(rmpk)).all(), ("mpk", i)
        assert (B.fetch(msk_a, l * 3 * n).reshape(l, 3, n) == canon(rmsk)).all(), ("msk", i)
        rct = O.encrypt(xs[i].astype(np.uint32), rmpk, s2[i], s3[i])
        if not chunked:
            assert (B.fetch(ct_a, (l + 1) * 3 * n).reshape(l + 1, 3, n) == canon(rct)).all(), ("ct", i)
        # function key and coefficient-0 residues: the context API's signed path
        c = cf.Context(n, l)
        yi = dev(ys[i].astype(np.int32)[None])
        sky = c.keygen(yi, dev(canon(rmsk)), y_signed=True)
        r0 = dev(np.zeros((1, 1, 3), np.uint32))
        dec = c.decrypt_coef0(dev(canon(rct)[None]), yi, sky, y_signed=True, d0=r0)
        c.sync()
        assert (B.fetch(sky_a, 3 * n).reshape(3, n) == cf.u32(sky)[0]).all(), ("sky", i)
        assert (got_d0[i] == cf.u32(r0).reshape(3)).all(), ("d0", i)
        assert int(got[i]) == int(cf.u32(dec)[0, 0]), ("out", i)
        p = 64 * l + 1
        assert int(got[i]) % p == int(xs[i] @ ys[i]) % p, ("ip", i)
        c.close()
    B.close()


def test_batch_graph_replay(rng, oracle_built):
    B, (_, _, xs, ys, _, _), (out, d0, s2d, s3d) = make(rng, 0)
    B.run()
    torch.cuda.synchronize()
    eager = cf.u32(out).copy(), cf.u32(d0).copy()
    out.zero_()
    d0.zero_()
    B.replay()  # captures (an eager step ran already) and launches
    torch.cuda.synchronize()
    assert (cf.u32(out) == eager[0]).all() and (cf.u32(d0) == eager[1]).all()
    # new seeds in the bound buffers: the replay must see them
    s2d.copy_(cf.bytes_to_dev(seeds(rng, B.count)))
    s3d.copy_(cf.bytes_to_dev(seeds(rng, B.count)))
    B.replay()
    torch.cuda.synchronize()
    rep = cf.u32(out).copy(), cf.u32(d0).copy()
    assert not (rep[1] == eager[1]).all()  # fresh randomness, different ciphertexts
    B.run()
    torch.cuda.synchronize()
    assert (cf.u32(out) == rep[0]).all() and (cf.u32(d0) == rep[1]).all()
    for i, l in enumerate(LS):
        assert int(rep[0][i]) % (64 * l + 1) == int(xs[i] @ ys[i]) % (64 * l + 1)
    B.status()
    B.close()


def test_batch_real_sizes_and_chunk_boundaries(oracle_built):
    """instances of the heterogeneous-batch shapes (n 2048/4096, l up to 1024); instance 0 is the
    reference's C2 golden round (n 4096, l 784, its seeds and x; f_i keyed by seed3).  One chunk:
    instance 0's ciphertext has the reference's hash, the others equal the oracle's encryption.
    One instance per chunk (chunks hold whole instances, so every boundary falls between two
    instances' streams): the same outputs as one chunk.  Every inner product is checked."""
    doc = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_c2.json")))
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a, np.uint32).tobytes()).hexdigest()  # noqa: E731
    ns, ls = [4096, 2048, 4096, 2048, 4096], [784, 1024, 1024, 33, 300]
    rng = np.random.default_rng(0xC0FE0500)
    cnt = len(ns)
    sa, se, s2, s3 = (seeds(rng, cnt) for _ in range(4))
    gr = np.random.default_rng(0xC0FE0002)  # the golden round's seeds, then x
    g_a, g_e, g_2 = gr.integers(0, 256, (3, 32), dtype=np.uint8)
    sa[0], se[0], s2[0], s3[0] = g_a, g_e, g_2, np.array(doc["seed3"], np.uint8)
    xs = [gr.integers(0, 5, 784, dtype=np.uint32).astype(np.int64)]
    xs += [rng.integers(0, 5, l, dtype=np.int64) for l in ls[1:]]
    ys = [rng.integers(-16, 17, l, dtype=np.int64) for l in ls]
    results = []
    for chunk in (0, 1):  # 0: one chunk (default budget); 1 byte: one instance per chunk
        B = cf.Batch(ns, ls, max_chunk_bytes=chunk)
        assert B.chunks == (1 if chunk == 0 else cnt)
        B.setup(sa, None, se)
        x = dev(B.pack(xs).astype(np.uint32))
        y = dev(B.pack(ys).astype(np.int32))
        d0 = dev(np.zeros((cnt, 3), np.uint32))
        out = B.bind(x, y, cf.bytes_to_dev(s2), cf.bytes_to_dev(s3), d0=d0)
        B.run()
        torch.cuda.synchronize()
        B.status()
        results.append((cf.u32(out).copy(), cf.u32(d0).copy()))
        if chunk == 0:
            ct0 = B.fetch(B.instance(0)[3], 785 * 3 * 4096)
            assert sha(ct0) == doc["ct_keyed"]
            for i in (1, 2, 3):
                n, l = ns[i], ls[i]
                O = Oracle(n, l)
                rmpk, _ = O.setup(sa[i], None, se[i])
                rct = O.encrypt(xs[i].astype(np.uint32), rmpk, s2[i], s3[i])
                assert (B.fetch(B.instance(i)[3], (l + 1) * 3 * n).reshape(l + 1, 3, n) == canon(rct)).all(), i
        B.close()
    assert (results[0][0] == results[1][0]).all() and (results[0][1] == results[1][1]).all()
    for i, l in enumerate(ls):
        p = 64 * l + 1
        assert int(results[0][0][i]) % p == int(xs[i] @ ys[i]) % p, i
