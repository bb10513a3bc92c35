"""Shape tuners (cufe_tune_encrypt, cufe_tune_decrypt_coef0, cufe_svm_tune, cufe_batch_tune):
every form a tuner can pick gives the bits of the fixed form, so a tuned call equals an untuned
one; the tuners report a choice among their forms and positive timings."""
import numpy as np
import pytest

from oracle.ffi import Oracle, canon
from tests.conftest import seeds

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import cufe_b200 as cf  # noqa: E402


def dev(a):
    return cf.to_dev(a)


def test_tune_encrypt_gives_the_fixed_ciphertexts(rng, oracle_built):
    n, l = 1024, 40
    c = cf.Context(n, l)
    sa, se = seeds(rng, 2)
    mpk, msk = c.setup(sa, None, se)
    x = rng.integers(0, 5, (5, l), dtype=np.uint32)
    s2, s3 = seeds(rng, 5), seeds(rng, 5)
    fixed = cf.u32(c.encrypt(dev(x), mpk, s2, s3))
    choice, ms = c.tune_encrypt(dev(x), mpk, s2, s3)
    assert choice in (1, 2) and all(t > 0 for t in ms)
    tuned = cf.u32(c.encrypt(dev(x), mpk, s2, s3))
    c.sync()
    assert (tuned == fixed).all()
    O = Oracle(n, l)
    rmpk, _ = O.setup(sa, None, se)
    assert (tuned[0] == canon(O.encrypt(x[0], rmpk, s2[0], s3[0]))).all()
    c.close()


def test_coef0_forms_agree_and_tuner(rng):
    """the per-pair kernel and the four tile shapes at counts that are multiples of no tile"""
    n, l = 1024, 40
    c = cf.Context(n, l)
    sa, se = seeds(rng, 2)
    mpk, msk = c.setup(sa, None, se)
    nct, nkeys = 70, 45
    x = rng.integers(0, 5, (nct, l), dtype=np.uint32)
    ct = c.encrypt(dev(x), mpk, seeds(rng, nct), None)
    y = rng.integers(-16, 17, (nkeys, l), dtype=np.int32)
    yd = torch.from_numpy(y).to(ct.device)
    sky = c.keygen(yd, msk, y_signed=True)
    outs = [cf.u32(c.decrypt_coef0_form(f, ct, yd, sky, y_signed=True)) for f in range(5)]
    c.sync()
    for f in range(1, 5):
        assert (outs[f] == outs[0]).all(), f
    p = 64 * l + 1
    got = outs[0].astype(np.int64)
    got = np.where(got > p // 2, got - p, got)
    assert (got == x.astype(np.int64) @ y.astype(np.int64).T).all()
    form, ms = c.tune_decrypt_coef0(ct, yd, sky, y_signed=True)
    assert 0 <= form < 5 and all(t > 0 for t in ms)
    assert (cf.u32(c.decrypt_coef0(ct, yd, sky, y_signed=True)) == outs[0]).all()
    c.close()


def test_svm_tune_keeps_the_predictions(rng):
    n, l = 2048, 124
    c = cf.Context(n, l)
    sa, se = seeds(rng, 2)
    mpk, msk = c.setup(sa, None, se)
    nsv = [20, 30]
    sv = rng.integers(0, 2, (sum(nsv), l)).astype(np.int32)
    m = cf.SvmModel(c, sv, nsv, rng.uniform(-1, 1, (1, sum(nsv))), [0.1], [1, -1], msk, signed=False)
    x = np.zeros((40, l), np.uint32)
    for t in range(40):
        x[t, rng.choice(np.arange(1, l), 14, replace=False)] = 1
    ct = c.encrypt(dev(x), mpk, seeds(rng, 40), None)
    dec0 = torch.empty((40, 1), dtype=torch.float64, device=ct.device)
    before = m.predict(ct, dec=dec0).cpu().numpy()
    form, ms = m.tune(ct)
    assert 0 <= form < 5
    dec1 = torch.empty_like(dec0)
    after = m.predict(ct, dec=dec1).cpu().numpy()
    c.sync()
    assert (before == after).all() and torch.equal(dec0, dec1)
    m.close()
    c.close()


def test_batch_tune_rechunks_without_changing_results(rng):
    ns, ls = [256, 1024, 512, 2048, 256], [8, 30, 12, 9, 21]
    B = cf.Batch(ns, ls)
    cnt = len(ns)
    B.setup(seeds(rng, cnt), None, seeds(rng, cnt))
    xs = [rng.integers(0, 5, l, dtype=np.int64) for l in ls]
    ys = [rng.integers(-16, 17, l, dtype=np.int64) for l in ls]
    d0 = dev(np.zeros((cnt, 3), np.uint32))
    out = B.bind(dev(B.pack(xs).astype(np.uint32)), dev(B.pack(ys).astype(np.int32)),
                 cf.bytes_to_dev(seeds(rng, cnt)), cf.bytes_to_dev(seeds(rng, cnt)), d0=d0)
    B.run()
    torch.cuda.synchronize()
    ref = cf.u32(out).copy(), cf.u32(d0).copy()
    budgets = [1, 1 << 22, 1 << 30]  # one instance per chunk ... everything in one chunk
    chosen, ms = B.tune(budgets)
    assert chosen in budgets and all(t > 0 for t in ms)
    assert B.chunks == (cnt if chosen == 1 else B.chunks)
    out.zero_()
    d0.zero_()
    B.replay()  # a new graph for the new layout
    torch.cuda.synchronize()
    assert (cf.u32(out) == ref[0]).all() and (cf.u32(d0) == ref[1]).all()
    for i, l in enumerate(ls):
        assert int(ref[0][i]) % (64 * l + 1) == int(xs[i] @ ys[i]) % (64 * l + 1)
    B.status()
    B.close()
