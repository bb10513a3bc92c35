"""libsvm model files for the encrypted SVM path (cufe_b200.SvmModel).

`load_model` reads the text format that libsvm's svm_save_model writes (svm/svm.cpp:2734-2822):
a header of `key value...` lines (svm_type, kernel_type, nr_class, total_sv, rho, label, nr_sv,
optional probA/probB and kernel parameters) followed by `SV` and one line per support vector,
`coef_1 ... coef_{nr_class-1} index:value ...`.

IPFE computes inner products of integer vectors, so only linear models apply, and the support
vectors must be integers of bounded size (the scheme's p = B_x B_y l + 1 assumes |y_i| <= 16,
src/params.h:24-26).  `to_integer` turns a model into the arrays SvmModel takes: the dense
support-vector matrix (convertToarray's layout, main.c:30-41: column = feature index) and, when
the values are not already integers within the bound, a uniform scaling s = bound / max|v| with
rounding; rho is scaled by the same s so that each decision value keeps its sign up to the
rounding of the support vectors.
"""
import numpy as np


def load_model(path):
    """parse a libsvm model file into a dict of header fields, sv_coef [nr_class-1][total_sv]
    and the support vectors as lists of (index, value)"""
    head, svs, coefs = {}, [], []
    with open(path) as f:
        lines = iter(f)
        for line in lines:
            t = line.split()
            if not t:
                continue
            if t[0] == "SV":
                break
            head[t[0]] = t[1:]
        nr_class = int(head["nr_class"][0])
        for line in lines:
            t = line.split()
            if not t:
                continue
            coefs.append([float(v) for v in t[:nr_class - 1]])
            svs.append([(int(a), float(b)) for a, b in (p.split(":") for p in t[nr_class - 1:])])
    model = {
        "svm_type": head["svm_type"][0],
        "kernel_type": head["kernel_type"][0],
        "nr_class": nr_class,
        "total_sv": int(head["total_sv"][0]),
        "rho": np.array([float(v) for v in head["rho"]]),
        "label": np.array([int(v) for v in head.get("label", [])], np.int32),
        "nr_sv": np.array([int(v) for v in head.get("nr_sv", [])], np.int32),
        "sv_coef": np.array(coefs, np.float64).T.reshape(nr_class - 1, len(svs)),
        "SV": svs,
    }
    if model["total_sv"] != len(svs) or (len(model["nr_sv"]) and model["nr_sv"].sum() != len(svs)):
        raise ValueError("model file: support-vector count does not match its header")
    return model


def to_integer(model, l, bound=16):
    """(sv [total_sv][l] int32, nr_sv, sv_coef, rho, label, scale) for SvmModel; features at
    column `index` (indices must be < l)"""
    if model["kernel_type"] != "linear":
        raise ValueError("encrypted prediction computes inner products: only linear models apply")
    if model["svm_type"] != "c_svc" and model["svm_type"] != "nu_svc":
        raise ValueError("classification models only (c_svc, nu_svc)")
    dense = np.zeros((len(model["SV"]), l), np.float64)
    for i, pairs in enumerate(model["SV"]):
        for idx, val in pairs:
            if idx < 0 or idx >= l:
                raise ValueError("feature index %d outside [0, %d)" % (idx, l))
            dense[i, idx] = val
    vmax = float(np.abs(dense).max()) if dense.size else 0.0
    if np.all(dense == np.round(dense)) and vmax <= bound:
        scale = 1.0
    else:
        scale = bound / vmax if vmax else 1.0
    sv = np.round(dense * scale).astype(np.int32)
    return sv, model["nr_sv"], model["sv_coef"], model["rho"] * scale, model["label"], scale


def save_model(path, nr_class, sv, nr_sv, sv_coef, rho, label):
    """write a linear c_svc model in libsvm's text format (for tests and fixtures)"""
    with open(path, "w") as f:
        f.write("svm_type c_svc\nkernel_type linear\nnr_class %d\ntotal_sv %d\n" % (nr_class, len(sv)))
        f.write("rho %s\n" % " ".join("%.17g" % r for r in rho))
        f.write("label %s\n" % " ".join(str(int(v)) for v in label))
        f.write("nr_sv %s\nSV\n" % " ".join(str(int(v)) for v in nr_sv))
        for i, row in enumerate(sv):
            coefs = " ".join("%.17g" % sv_coef[k][i] for k in range(nr_class - 1))
            feats = " ".join("%d:%.17g" % (j, v) for j, v in enumerate(row) if v != 0)
            f.write("%s %s\n" % (coefs, feats))
