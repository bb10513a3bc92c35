"""Request server (cufe_server_*): continuous batching over resident tenants.

Served ciphertexts must equal the oracle's encryption for the same tenant keys and seeds,
decrypted inner products must equal the plaintext dot products mod p, and every result must
be bit-identical whether the request was served in a mixed tick or alone.
"""
import numpy as np
import pytest

from oracle.ffi import Oracle, canon
from tests.conftest import seeds

pytestmark = pytest.mark.gpu

pytest.importorskip("torch")
import cufe_b200 as cf  # noqa: E402

NS = [256, 1024, 512, 256]
LS = [8, 6, 13, 21]


def test_server_parity_and_determinism(rng, oracle_built):
    S = cf.Server(NS, LS, arena_bytes=64 << 20, tick_bytes=256 << 20)
    T = len(NS)
    sa, se = seeds(rng, T), seeds(rng, T)
    S.setup(sa, None, se)
    # a mix: encryptions and keygens for every tenant, submitted together
    enc, kg = [], []
    for rep in range(3):
        for t in range(T):
            x = rng.integers(0, 5, LS[t]).astype(np.uint32)
            s2, s3 = seeds(rng, 2)
            enc.append((t, x, s2, s3, S.encrypt(t, x, s2, s3)))
            y = rng.integers(-16, 17, LS[t]).astype(np.int32)
            kg.append((t, y, S.keygen(t, y)))
    S.drain()
    # decryptions of every (ciphertext, key) pair of each tenant, in one go
    dec = []
    for (t, x, _, _, cid) in enc:
        for (t2, y, kid) in kg:
            if t2 == t:
                dec.append((t, x, y, S.decrypt(cid, kid)))
    S.drain()
    assert S.stats()["ticks"] >= 2
    for (t, x, y, did) in dec:
        st, v, _, _ = S.result(did)
        p = 64 * LS[t] + 1
        assert st == S.DONE and v % p == int(x.astype(np.int64) @ y.astype(np.int64)) % p
    # ciphertexts against the oracle
    for (t, x, s2, s3, cid) in enc[:T]:
        O = Oracle(NS[t], LS[t])
        rmpk, _ = O.setup(sa[t], None, se[t])
        n, l = NS[t], LS[t]
        got = S.read(cid, (l + 1) * 3 * n).reshape(l + 1, 3, n)
        assert (got == canon(O.encrypt(x, rmpk, s2, s3))).all(), t
    # determinism: the same requests alone give the same bits
    for (t, x, s2, s3, cid) in enc[:T]:
        n, l = NS[t], LS[t]
        alone = S.encrypt(t, x, s2, s3)
        S.drain()
        assert (S.read(alone, (l + 1) * 3 * n) == S.read(cid, (l + 1) * 3 * n)).all(), t
        S.release(alone)
    t, x, y, did = dec[0]
    cid = [e[4] for e in enc if e[0] == t][0]
    kid = [k[2] for k in kg if k[0] == t][0]
    solo = S.decrypt(cid, kid)
    S.drain()
    assert S.result(solo)[1] == S.result(dec[0][3])[1]
    # releases free the arena for new work
    free0 = S.stats()["ct_free_bytes"]
    for e in enc:
        S.release(e[4])
    assert S.stats()["ct_free_bytes"] > free0
    S.close()
