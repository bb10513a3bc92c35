"""Serialized keys and ciphertexts (cufe_serialize / cufe_deserialize): bit-exact round trips
through device buffers and a file, the packed size, and rejection of corrupt input."""
import numpy as np
import pytest

from tests.conftest import seeds

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import cufe_b200 as cf  # noqa: E402


def roundtrip(c, kind, t, count):
    buf = c.serialize(kind, t)
    back = c.deserialize(kind, buf, count)
    c.sync()
    assert (cf.u32(back).reshape(-1) == cf.u32(t).reshape(-1)).all()
    return buf


def test_serialize_scheme_objects(tmp_path, rng):
    n, l = 1024, 16
    c = cf.Context(n, l)
    sa, se = seeds(rng, 2)
    mpk, msk = c.setup(sa, None, se)
    x = rng.integers(0, 5, (3, l)).astype(np.uint32)
    ct = c.encrypt(cf.to_dev(x), mpk, seeds(rng, 3), None)
    y = rng.integers(0, 17, (2, l)).astype(np.uint32)
    sky = c.keygen(cf.to_dev(y), msk)
    dy = c.decrypt(ct, cf.to_dev(y), sky)
    for kind, t, count in [(cf.OBJ_MPK, mpk, 1), (cf.OBJ_MSK, msk, 1), (cf.OBJ_CT, ct, 3),
                           (cf.OBJ_SKY, sky, 2), (cf.OBJ_DY, dy, 6)]:
        buf = roundtrip(c, kind, t, count)
        raw = t.numel() * 4
        assert buf.numel() == 32 + raw * 86 // 96 and buf.numel() < 0.9 * raw + 64
    # through a file on the host
    buf = c.serialize(cf.OBJ_CT, ct)
    path = tmp_path / "ct.bin"
    path.write_bytes(buf.cpu().numpy().tobytes())
    again = torch.from_numpy(np.frombuffer(path.read_bytes(), np.uint8).copy()).cuda()
    back = c.deserialize(cf.OBJ_CT, again, 3)
    c.sync()
    assert (cf.u32(back) == cf.u32(ct)).all()
    # the decrypted inner products still come out of a deserialized ciphertext
    dec = cf.u32(c.decrypt_coef0(back, cf.to_dev(y), sky))
    assert (dec.astype(np.int64) == x.astype(np.int64) @ y.astype(np.int64).T).all()
    # corrupt input is rejected
    bad = buf.clone()
    bad[0] ^= 1
    with pytest.raises(cf.CufeError):
        c.deserialize(cf.OBJ_CT, bad, 3)
    with pytest.raises(cf.CufeError):
        c.deserialize(cf.OBJ_MPK, buf, 3)  # wrong kind
    bad = buf.clone()
    bad[32:] = 255  # 24-bit residues 0xffffff >= q_0
    with pytest.raises(cf.CufeError):
        c.deserialize(cf.OBJ_CT, bad, 3)
    c.close()


def test_serialize_small_ring_partial_words(rng):
    """n = 16: 16 x 31 bits = 15.5 words, padded"""
    c = cf.Context(16, 4)
    q = np.array(cf.Q, np.uint64)
    r = (rng.integers(0, 2**62, (5, 3, 16), dtype=np.uint64) % q[None, :, None]).astype(np.uint32)
    r[0, :, :] = (q - 1).astype(np.uint32)[:, None]  # largest residues
    roundtrip(c, cf.OBJ_SKY, cf.to_dev(r), 5)
    c.close()
