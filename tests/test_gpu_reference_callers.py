"""The reference's own callers of the GPU entry points, bound to this library's drop-in
symbols (oracle/_ref/callers/libcallers.so: main.c, src/rlwe_sife.c and svm/svm.cpp compiled
unmodified at n = 2048, l = 124 and linked against cufe_b200/libcufe_b200.so).

- rlwe_sife_setup_gui / rlwe_sife_encrypt_gui (src/rlwe_sife.c:85-109, 184-212) call
  rlwe_sife_setup_gpu / rlwe_sife_encrypt_gpu here; their outputs must equal the oracle's GPU
  counter mapping (setup from the same three seeds, every encryption instance keyed by the one
  seed the wrapper passes twice).
- svm_predict_gpu ("svm_predict5", main.c:270-390) calls rlwe_sife_keygen_gpu and
  rlwe_sife_decrypt_gmp_gpu here, then decodes on the host with the reference's GMP code; on
  the reference's a1a model its labels and decision values must equal those of the
  reference's CPU prediction (tests/golden/ref_svm_a1a.npz).
"""
import os

import numpy as np
import pytest

from oracle.ffi import Oracle, ReferenceCallers, canon

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(ReferenceCallers.PATH),
                                 reason="reference callers not built (oracle/ref/build_ref.py)")]

torch = pytest.importorskip("torch")
import cufe_b200 as cf  # noqa: E402

GOLD_SVM = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_svm_a1a.npz")


@pytest.fixture
def callers():
    R = ReferenceCallers()
    L = cf.lib()
    assert L.cufe_dropin_configure(R.n, R.l, 0) == 0
    yield R
    L.cufe_dropin_configure(4096, 785, 0)


def test_reference_gui_wrappers_through_dropin(callers, oracle_built):
    R = callers
    rng = np.random.default_rng(0xC0FE0400)
    seed1, seed2, seed3, seed_enc = rng.integers(0, 256, (4, 32), dtype=np.uint8)
    mpk = np.zeros((R.l + 1, 3, R.n), np.uint32)
    msk = np.zeros((R.l, 3, R.n), np.uint32)
    R.seeds(seed1, seed2, seed3)
    R.L.cl_setup_gui(mpk, msk)
    assert cf.lib().cufe_dropin_status() == 0
    O = Oracle(R.n, R.l)
    a = O.sample_polya(seed1)
    rmpk, rmsk = O.setup_modeB(a, seed2, seed3)
    assert (canon(mpk) == canon(rmpk)).all() and (canon(msk) == canon(rmsk)).all()
    x = rng.integers(0, 5, (2, R.l), dtype=np.uint32)
    c = np.zeros((2, R.l + 1, 3, R.n), np.uint32)
    R.seeds(seed_enc)
    R.L.cl_encrypt_gui(x, mpk, c, 2)
    assert cf.lib().cufe_dropin_status() == 0
    for b in range(2):
        assert (canon(c[b]) == canon(O.encrypt_modeB(x[b], rmpk, seed_enc))).all(), b


def test_reference_svm_predict5_through_dropin(callers, tmp_path):
    from cufe_b200 import libsvm
    R = callers
    g = np.load(GOLD_SVM)
    path = str(tmp_path / "a1a.model")
    libsvm.save_model(path, len(g["label"]), g["sv"], g["nsv"], g["coef"], g["rho"], g["label"])
    model, arr = R.load_model(path)  # the reference's own svm_load_model
    assert (arr["sv"] == g["sv"]).all() and (arr["coef"] == g["coef"]).all() and (arr["rho"] == g["rho"]).all()
    c = cf.Context(R.n, R.l)
    mpk, msk = c.setup(g["seed_a"], None, g["seed_e"])
    rows = range(8)
    ct = cf.u32(c.encrypt(cf.to_dev(g["x"][list(rows)].astype(np.uint32)), mpk, g["seeds2"][list(rows)], None))
    msk_h = cf.u32(msk)
    c.sync()
    for k, t in enumerate(rows):
        label, dec, kv = R.predict(model, ct[k], msk_h, 1, len(g["sv"]), gpu=True)
        assert cf.lib().cufe_dropin_status() == 0
        assert (kv == g["ref_kvalue"][t]).all(), t
        assert label == g["ref_label"][t] and dec.view(np.uint64)[0] == g["ref_dec"][t].view(np.uint64)[0], t
    R.L.cl_free_model(model)
    c.close()
