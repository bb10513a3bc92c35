"""libsvm model files -> the arrays of the encrypted SVM path (CPU only)."""
import os

import numpy as np
import pytest

from cufe_b200 import libsvm

REF_ROOT = os.environ.get("CUFE_REFERENCE_ROOT")
REF_MODEL = os.path.join(REF_ROOT, "svm model", "a1a.txt.model") if REF_ROOT else ""
GOLD_SVM = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_svm_a1a.npz")


def test_round_trip_integer_model(tmp_path, rng):
    sv = rng.integers(-16, 17, (9, 30)).astype(np.int32)
    sv[:, 0] = 0
    coef = rng.uniform(-1, 1, (2, 9))
    p = str(tmp_path / "m.model")
    libsvm.save_model(p, 3, sv, [3, 4, 2], coef, [0.5, -0.25, 0.125], [4, 7, 9])
    m = libsvm.load_model(p)
    assert m["nr_class"] == 3 and m["total_sv"] == 9 and list(m["label"]) == [4, 7, 9]
    svq, nsv, c, rho, label, scale = libsvm.to_integer(m, 30)
    assert scale == 1.0 and (svq == sv).all() and (c == coef).all() and list(nsv) == [3, 4, 2]
    assert np.allclose(rho, [0.5, -0.25, 0.125])


def test_scaling_keeps_decisions(tmp_path, rng):
    sv = rng.uniform(-3, 3, (6, 12))
    coef = rng.uniform(-1, 1, (1, 6))
    p = str(tmp_path / "f.model")
    libsvm.save_model(p, 2, sv, [3, 3], coef, [0.3], [1, -1])
    svq, _, c, rho, _, scale = libsvm.to_integer(libsvm.load_model(p), 12)
    assert np.abs(svq).max() == 16 and scale == pytest.approx(16 / np.abs(sv).max())
    x = rng.integers(0, 2, (50, 12))
    exact = (x @ sv.T) @ coef[0] - 0.3
    quant = (x @ svq.T) @ c[0] - rho[0]
    far = np.abs(exact) > 0.05 * np.abs(exact).max()
    assert (np.sign(exact[far]) == np.sign(quant[far])).all()


def test_rejects_nonlinear(tmp_path):
    p = str(tmp_path / "rbf.model")
    with open(p, "w") as f:
        f.write("svm_type c_svc\nkernel_type rbf\ngamma 0.5\nnr_class 2\ntotal_sv 1\nrho 0\nlabel 1 -1\n"
                "nr_sv 1 0\nSV\n1 1:1\n")
    with pytest.raises(ValueError):
        libsvm.to_integer(libsvm.load_model(p), 4)


def test_reference_model_arrays_round_trip(tmp_path):
    """the arrays the reference's own svm_load_model read from its a1a model (fixture) survive
    this module's writer and parser unchanged"""
    g = np.load(GOLD_SVM)
    p = str(tmp_path / "a1a.model")
    libsvm.save_model(p, 2, g["sv"], g["nsv"], g["coef"], g["rho"], g["label"])
    sv, nsv, coef, rho, label, scale = libsvm.to_integer(libsvm.load_model(p), int(g["l"]))
    assert scale == 1.0 and (sv == g["sv"]).all() and (nsv == g["nsv"]).all()
    assert (coef == g["coef"]).all() and (rho == g["rho"]).all() and (label == g["label"]).all()


@pytest.mark.skipif(not os.path.exists(REF_MODEL), reason="CUFE_REFERENCE_ROOT not set")
def test_reference_model_parses():
    """the reference's bundled linear model, read in place: this parser gives the arrays the
    reference's svm_load_model gave (fixture)"""
    m = libsvm.load_model(REF_MODEL)
    assert m["kernel_type"] == "linear" and m["nr_class"] == 2
    assert m["total_sv"] == int(m["nr_sv"].sum())
    sv, nsv, coef, rho, label, scale = libsvm.to_integer(m, 124)
    g = np.load(GOLD_SVM)
    assert scale == 1.0 and (sv == g["sv"]).all() and (coef == g["coef"]).all() and (rho == g["rho"]).all()
