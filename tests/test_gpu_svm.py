"""Encrypted linear-SVM prediction (cufe_svm_*), the svm_predict5 path of main.c:270-390.

kvalue (the decoded coefficient 0 of every (test ciphertext, support vector) decryption) must
equal the plaintext inner product; the device vote must give the labels and, bit for bit, the
decision values of the reference's vote loop (main.c:331-379) as gcc -O3 compiles it for an AVX2 + FMA host
(each term loop vectorised as an in-order reduction: products rounded, then added one by one,
except the last term of an odd-length loop, which the scalar remainder fuses); for unsigned
support vectors
the kvalues must equal the oracle's decryption + decode.  On the reference's own model and test
set (tests/golden/ref_svm_a1a.npz) labels and decision values must equal those of the
reference's svm_predict_cpu.
"""
import os
from fractions import Fraction

import numpy as np
import pytest

from oracle.ffi import Oracle, canon
from tests.conftest import seeds

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import cufe_b200 as cf  # noqa: E402


GOLD_SVM = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_svm_a1a.npz")


def loop_sum(s, coef, kv):
    """one term loop of the vote (main.c:359-362) as the reference build computes it: in index
    order, s + round(coef * kv) for every term except the last of an odd-length loop, which is
    one fused multiply-add (exact rationals, one rounding)"""
    n = len(coef)
    for k in range(n & ~1):
        s = s + float(coef[k]) * float(kv[k])
    if n & 1:
        s = float(Fraction(float(coef[-1])) * Fraction(float(kv[-1])) + Fraction(s))
    return s


def plain_vote(kv, nsv, coef, rho, label):
    """the one-against-one vote of main.c:331-379 on plaintext inner products, with the
    reference build's arithmetic (loop_sum)"""
    nr = len(nsv)
    start = np.concatenate([[0], np.cumsum(nsv)[:-1]])
    out, decs = [], []
    for t in range(kv.shape[0]):
        vote = [0] * nr
        p, dv = 0, []
        for i in range(nr):
            for j in range(i + 1, nr):
                si, sj, ci, cj = start[i], start[j], nsv[i], nsv[j]
                s = loop_sum(loop_sum(0.0, coef[j - 1][si:si + ci], kv[t, si:si + ci]),
                             coef[i][sj:sj + cj], kv[t, sj:sj + cj]) - rho[p]
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
    assert np.array_equal(dec.cpu().numpy(), wdec)  # bit for bit, the reference build's arithmetic
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


def _against_reference_fixture(name, batch=50):
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", name))
    n, l = int(g["n"]), int(g["l"])
    c = cf.Context(n, l)
    mpk, msk = c.setup(g["seed_a"], None, g["seed_e"])
    x = g["x"].astype(np.uint32)
    lsv, pairs = len(g["sv"]), len(g["rho"])
    m = cf.SvmModel(c, g["sv"].astype(np.int32), g["nsv"], g["coef"], g["rho"], g["label"], msk, signed=False)
    labels, decs, kvs = [], [], []
    for b in range(0, len(x), batch):
        ct = c.encrypt(cf.to_dev(x[b:b + batch]), mpk, g["seeds2"][b:b + batch], None)
        dec = torch.empty((ct.shape[0], pairs), dtype=torch.float64, device=ct.device)
        kv = torch.empty((ct.shape[0], lsv), dtype=torch.int32, device=ct.device)
        labels.append(m.predict(ct, kvalue=kv, dec=dec).cpu().numpy())
        decs.append(dec.cpu().numpy())
        kvs.append(cf.u32(kv))
        del ct
    c.sync()
    assert (np.concatenate(kvs) == g["ref_kvalue"]).all()
    assert (np.concatenate(labels) == g["ref_label"]).all()
    assert np.array_equal(np.concatenate(decs).view(np.uint64), g["ref_dec"].view(np.uint64))
    m.close()
    c.close()
    return g


def test_svm_a1a_reference_model():
    """the reference's shipped a1a model and the 200 test vectors its main.c classifies first:
    setup and encryptions from the same seeds as the reference run (CPU stream mapping), then
    cufe_svm_predict; decoded inner products, labels and decision values equal those of the
    reference's svm_predict_cpu (keygen + decrypt + GMP decode per support vector,
    main.c:137-267), bit for bit"""
    g = _against_reference_fixture("ref_svm_a1a.npz")
    assert (g["ref_label"] == g["plain_label"]).all()


def test_svm_short_class_loops_reference():
    """a three-class model with classes of 1, 3 and 6 support vectors (the vote's term loops at
    short odd and even lengths) against the reference's svm_predict_cpu.  Its decode returns
    values in [0, p] (src/rlwe_sife.c:320-324), so a zero inner product with negative noise
    decodes to p and enters the vote as p: the reference's labels then differ from the
    plaintext vote, and these must too"""
    _against_reference_fixture("ref_svm_small.npz", batch=12)
