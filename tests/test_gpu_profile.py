"""The context profiler's launch counts (cufe_profile_*): every kernel a call launches is
counted once, in its named group and in the context total that bench.py reports as
gpu_launches."""
import numpy as np
import pytest

from tests.conftest import seeds

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import cufe_b200 as cf  # noqa: E402


def test_profile_counts_kernels(rng, oracle_built):
    n, l = 1024, 16
    c = cf.Context(n, l)
    sa, se = seeds(rng, 2)
    mpk, msk = c.setup(sa, None, se)
    x = cf.to_dev(rng.integers(0, 5, (3, l), dtype=np.uint32))
    ct = c.encrypt(x, mpk, seeds(rng, 3), None)
    y = cf.to_dev(rng.integers(0, 17, (40, l), dtype=np.uint32))
    sky = c.keygen(y, msk)
    c.sync()
    c.profile_reset()
    c.profile(True)
    assert c.profile_launches() == 0
    c.decrypt_coef0(ct, y, sky)  # 40 keys: the tiled product and the decode of every pair
    c.sync()
    got = c.profile_read()
    assert got["decrypt_coef0"][0] == 2 and c.profile_launches() == 2
    c.decrypt_coef0(ct, y[:1], sky[:1])  # one key: one CTA per pair, decode included
    c.sync()
    assert c.profile_read()["decrypt_coef0"][0] == 3 and c.profile_launches() == 3
    c.encrypt(x, mpk, seeds(rng, 3), None)
    c.sync()
    prof = c.profile_read()
    total = c.profile_launches()
    assert total >= sum(v[0] for v in prof.values()) > 3
    c.profile(False)
    c.decrypt_coef0(ct, y[:1], sky[:1])  # off: not counted
    c.sync()
    assert c.profile_launches() == total
    c.profile_reset()
    assert c.profile_launches() == 0 and c.profile_read() == {}
    c.close()
