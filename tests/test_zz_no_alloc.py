"""cufe_decrypt_noalloc: decryption for callers that cannot allocate device memory during a
call (fixed GPU memory budgets, serving threads that must not synchronise the device through
cudaMalloc).  Its output must equal cufe_decrypt's, bit for bit, on consecutive calls that
reuse the shared scratch array.  This file is collected last on purpose."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import cufe_b200 as cf  # noqa: E402


def _keys_and_ct(ctx, rng, nkeys):
    sa, ss, se = rng.integers(0, 256, (3, 32), dtype=np.uint8)
    mpk, msk = ctx.setup(sa, ss, se)
    x = rng.integers(0, 5, (2, ctx.l), dtype=np.uint32)
    ct = ctx.encrypt(cf.to_dev(x), mpk, rng.integers(0, 256, (2, 32), dtype=np.uint8),
                     rng.integers(0, 256, (2, 32), dtype=np.uint8))
    y = rng.integers(-16, 17, (nkeys, ctx.l), dtype=np.int32)
    yd = torch.from_numpy(y).to(ctx.dev)
    sky = ctx.keygen(yd, msk, y_signed=True)
    return x, ct, y, yd, sky


@pytest.mark.parametrize("n,l", [(1024, 16), (4096, 784)])
def test_noalloc_matches_decrypt_twice(n, l):
    rng = np.random.default_rng(2024 + n)
    ctx = cf.Context(n, l)
    x, ct, y, yd, sky = _keys_and_ct(ctx, rng, 3)
    for b in range(2):  # two calls in a row on different ciphertexts
        ref = cf.u32(ctx.decrypt(ct[b:b + 1], yd, sky, y_signed=True))
        got = cf.u32(ctx.decrypt_noalloc(ct[b:b + 1], yd, sky, y_signed=True))
        ctx.sync()
        assert (got == ref).all(), b
        dec = cf.u32(ctx.decode(cf.to_dev(got)))[:, 0].astype(np.int64)
        dec = np.where(dec > ctx.p // 2, dec - ctx.p, dec)
        assert (dec == y.astype(np.int64) @ x[b].astype(np.int64)).all()


def test_noalloc_rejects_sizes_beyond_limit():
    rng = np.random.default_rng(7)
    ctx = cf.Context(1024, 16)
    x, ct, y, yd, sky = _keys_and_ct(ctx, rng, 5)
    with pytest.raises(cf.CufeError) as e:
        ctx.decrypt_noalloc(ct[:1], yd, sky, y_signed=True)
    assert e.value.code == -1 and "4 keys" in str(e.value)
    big = cf.Context(8192, 4)
    yb = torch.zeros((1, 4), dtype=torch.int32, device=big.dev)
    with pytest.raises(cf.CufeError):
        big.decrypt_noalloc(big.ct_buf(1), yb, torch.zeros((1, 3, 8192), dtype=torch.int32, device=big.dev))
