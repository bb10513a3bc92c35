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


def _wait_all(S, ids, owned=(), check=None, max_polls=20000):
    """poll until every id is finished (done or shed), releasing finished encrypts/keygens in
    `owned` after `check` saw them; bounded so that a stuck server fails the test"""
    owned = list(owned)
    for _ in range(max_polls):
        S.poll(wait=S.pending()[1] > 0)
        for rid in [r for r in owned if S.result(r)[0] == S.DONE]:
            owned.remove(rid)
            if check:
                check(rid)
            S.release(rid)
        if all(S.result(i)[0] in (S.DONE, S.RELEASED, S.SHED) for i in ids):
            return
    raise AssertionError("server did not finish")


def test_server_real_sizes_and_arena_exhaustion(oracle_built):
    """tenants of the serving shapes (n 4096 / 2048, l up to 1024) and a ciphertext arena that
    holds only three of the largest ciphertexts: encryptions that do not fit wait in the queue
    and are admitted as released slots free up; served ciphertexts equal the oracle's, inner
    products the plaintext ones"""
    ns, ls = [4096, 2048, 4096], [1024, 700, 64]
    big = (1024 + 1) * 3 * 4096 * 4
    S = cf.Server(ns, ls, arena_bytes=3 * big + (8 << 20), tick_bytes=4 << 30)
    rng = np.random.default_rng(0xC0FE0501)
    sa, se = seeds(rng, 3), seeds(rng, 3)
    S.setup(sa, None, se)
    reqs, owned = {}, []
    for t in (0, 0, 1, 0, 2, 0, 0, 1, 0, 2):
        x = rng.integers(0, 5, ls[t]).astype(np.uint32)
        s2, s3 = seeds(rng, 2)
        rid = S.encrypt(t, x, s2, s3)
        reqs[rid] = (t, x, s2, s3)
        owned.append(rid)
    checked = []
    oracles = {}

    def check(rid):
        t, x, s2, s3 = reqs[rid]
        if t in checked:
            return
        n, l = ns[t], ls[t]
        if t not in oracles:
            O = Oracle(n, l)
            oracles[t] = (O, O.setup(sa[t], None, se[t])[0])
        O, rmpk = oracles[t]
        got = S.read(rid, (l + 1) * 3 * n).reshape(l + 1, 3, n)
        assert (got == canon(O.encrypt(x, rmpk, s2, s3))).all(), t
        checked.append(t)

    _wait_all(S, list(reqs), owned, check)
    assert sorted(set(checked)) == [0, 1, 2]
    # the arena holds three of tenant 0's ciphertexts: its six encryptions need three ticks
    assert S.stats()["ticks"] >= 3
    # decrypts of fresh ciphertexts against fresh keys of the largest tenant
    x = rng.integers(0, 5, 1024).astype(np.uint32)
    y = rng.integers(-16, 17, 1024).astype(np.int32)
    cid, kid = S.encrypt(0, x, *seeds(rng, 2)), S.keygen(0, y)
    S.drain()
    did = S.decrypt(cid, kid)
    S.drain()
    p = 64 * 1024 + 1
    assert S.result(did)[1] % p == int(x.astype(np.int64) @ y.astype(np.int64)) % p
    S.close()


def test_server_overload_limits(rng):
    """a per-tick request cap splits a burst over several ticks; requests older than the queue
    deadline when a tick forms are shed (state 4, counted), with the decrypts that read them;
    shed requests cannot be read, released or decrypted; fresh requests still complete"""
    S = cf.Server([1024], [16], arena_bytes=64 << 20, tick_bytes=256 << 20)
    S.setup(seeds(rng, 1), None, seeds(rng, 1))
    y = rng.integers(-16, 17, 16).astype(np.int32)
    kid = S.keygen(0, y)
    S.drain()
    S.limits(2, 0.0)
    t0 = S.stats()["ticks"]
    burst = [S.encrypt(0, rng.integers(0, 5, 16).astype(np.uint32), *seeds(rng, 2)) for _ in range(6)]
    S.drain()
    assert S.stats()["ticks"] - t0 >= 3
    assert all(S.result(i)[0] == S.DONE for i in burst)
    S.limits(0, 0.5)
    past = S.now() - 10.0
    x = rng.integers(0, 5, 16).astype(np.uint32)
    old = [S.encrypt(0, x, *seeds(rng, 2), t_arrival=past) for _ in range(3)]
    dep = S.decrypt(old[0], kid)                       # reads a request that will be shed
    fresh = S.encrypt(0, x, *seeds(rng, 2))
    fdec = S.decrypt(burst[0], kid)
    S.drain()
    assert [S.result(i)[0] for i in old + [dep]] == [S.SHED] * 4
    assert S.result(fresh)[0] == S.DONE and S.result(fdec)[0] == S.DONE
    assert S.stats()["shed"] == 4
    with pytest.raises(cf.CufeError):
        S.read(old[1], 17 * 3 * 1024)
    with pytest.raises(cf.CufeError):
        S.release(old[1])
    with pytest.raises(cf.CufeError):
        S.decrypt(old[1], kid)
    S.close()
