"""Encrypted linear-SVM prediction (cufe_svm_*), the svm_predict5 path of main.c:270-390.

kvalue (the decoded coefficient 0 of every (test ciphertext, support vector) decryption) must
equal the plaintext inner product, the device vote must give the labels of the plaintext
libsvm vote (main.c:331-379, restated in numpy below), and for unsigned support vectors the
kvalues must equal the oracle's decryption + decode.
"""
import numpy as np
import pytest

from oracle.ffi import Oracle, canon
from tests.conftest import seeds

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import cufe_b200 as cf  # noqa: E402


def plain_vote(kv, nsv, coef, rho, label):
    """the one-against-one vote of main.c:331-379 on plaintext inner products"""
    nr = len(nsv)
    start = np.concatenate([[0], np.cumsum(nsv)[:-1]])
    out, decs = [], []
    for t in range(kv.shape[0]):
        vote = [0] * nr
        p, dv = 0, []
        for i in range(nr):
            for j in range(i + 1, nr):
                si, sj, ci, cj = start[i], start[j], nsv[i], nsv[j]
                s = float(np.dot(coef[j - 1][si:si + ci], kv[t, si:si + ci]) +
                          np.dot(coef[i][sj:sj + cj], kv[t, sj:sj + cj])) - rho[p]
                dv.append(s)
                vote[i if s > 0 else j] += 1
                p += 1
        out.append(label[int(np.argmax(vote))])
        decs.append(dv)
    return np.array(out), np.array(decs)


@pytest.mark.parametrize("nsv,signed", [([40, 24], True), ([10, 17, 9], True), ([12, 20], False)])
def test_svm_predict(nsv, signed, rng, oracle_built):
    n, l = 2048, 124
    c = cf.Context(n, l)
    sa, se = seeds(rng, 2)
    mpk, msk = c.setup(sa, None, se)
    ntest, lsv, nr = 50, sum(nsv), len(nsv)
    x = np.zeros((ntest, l), np.uint32)
    for t in range(ntest):  # a1a-shaped: ~14 ones at feature indices 1..123
        x[t, rng.choice(np.arange(1, l), 14, replace=False)] = 1
    if signed:
        sv = rng.integers(-16, 17, (lsv, l)).astype(np.int32)
    else:
        sv = rng.integers(0, 2, (lsv, l)).astype(np.int32)
    sv[:, 0] = 0
    coef = rng.uniform(-1, 1, (nr - 1, lsv))
    rho = rng.uniform(-0.5, 0.5, nr * (nr - 1) // 2)
    label = np.arange(nr, dtype=np.int32) * 3 - 1
    m = cf.SvmModel(c, sv, nsv, coef, rho, label, msk, signed=signed)
    s2 = seeds(rng, ntest)
    ct = c.encrypt(cf.to_dev(x), mpk, s2, None)
    kv = torch.empty((ntest, lsv), dtype=torch.int32, device=ct.device)
    dec = torch.empty((ntest, nr * (nr - 1) // 2), dtype=torch.float64, device=ct.device)
    got = m.predict(ct, kvalue=kv, dec=dec)
    c.sync()
    kvh = cf.u32(kv).astype(np.int64)
    p = 64 * l + 1
    if signed:
        kvh = np.where(kvh > p // 2, kvh - p, kvh)
    ip = x.astype(np.int64) @ sv.astype(np.int64).T
    assert (kvh == ip).all()
    want, wdec = plain_vote(ip.astype(np.float64), nsv, coef, rho, label)
    assert (got.cpu().numpy() == want).all()
    assert np.allclose(dec.cpu().numpy(), wdec, rtol=1e-12, atol=1e-9)
    if not signed:  # the reference path (uint32 y) for a few pairs, through the oracle
        O = Oracle(n, l)
        rmpk, rmsk = O.setup(sa, None, se)
        for t in range(2):
            rct = O.encrypt(x[t], rmpk, s2[t], None)
            for i in range(3):
                y = sv[i].astype(np.uint32)
                assert int(O.decode(O.decrypt(rct, y, O.keygen(y, rmsk)))[0]) == int(kvh[t, i])
    m.close()
    c.close()


def test_svm_from_libsvm_file(tmp_path, rng, oracle_built):
    """a model file in libsvm's format, loaded and quantized, predicts like the plaintext vote"""
    from cufe_b200 import libsvm
    n, l = 1024, 40
    nsv = [7, 5, 6]
    sv = rng.uniform(-2, 2, (sum(nsv), l))
    sv[:, 0] = 0
    coef = rng.uniform(-1, 1, (2, sum(nsv)))
    path = str(tmp_path / "m.model")
    libsvm.save_model(path, 3, sv, nsv, coef, rng.uniform(-0.5, 0.5, 3), [1, 2, 3])
    svq, nr_sv, c_, rho, label, _ = libsvm.to_integer(libsvm.load_model(path), l)
    ctx = cf.Context(n, l)
    mpk, msk = ctx.setup(*seeds(rng, 1), None, seeds(rng, 1)[0])
    # binary features (a1a-like): |<x, sv>| <= 16 l < p / 2, where the centred decode is exact
    x = rng.integers(0, 2, (20, l)).astype(np.uint32)
    x[:, 0] = 0
    m = cf.SvmModel(ctx, svq, nr_sv, c_, rho, label, msk, signed=True)
    got = m.predict(ctx.encrypt(cf.to_dev(x), mpk, seeds(rng, 20), None))
    ctx.sync()
    want, _ = plain_vote((x.astype(np.int64) @ svq.astype(np.int64).T).astype(np.float64), nr_sv, c_, rho, label)
    assert (got.cpu().numpy() == want).all()
    m.close()
    ctx.close()
