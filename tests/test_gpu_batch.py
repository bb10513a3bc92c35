"""Heterogeneous batches (cufe_batch_*): instances of different ring degree and vector length,
each with its own keys, stepped together.

Per instance the batch must give what the single-instance path gives: keys and ciphertexts
equal to the oracle's for the same seeds (the oracle is pinned to the reference CPU build),
function keys and coefficient-0 residues equal to the context API's signed-y path, and the
decoded inner product equal to the plaintext dot product mod p_i.  Also: several chunks give
the same results as one, and a CUDA-graph replay equals an eager step, including after new
seeds are written into the bound buffers.
"""
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
