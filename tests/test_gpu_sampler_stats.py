"""Distribution of the GPU samplers: chi-square per sigma.

sigma_1 against the ideal discrete Gaussian D_{Z,sigma_1}.  sigma_2 and sigma_3 reproduce the
reference's samplers, which are not D_{Z,sigma} (their Bernoulli input conversion is exact
only below 2^52; see cufe_b200/stats.py), so they are checked by a two-sample chi-square
against the oracle's samples of the same mapping on independent seeds.  Both mappings: the
CPU stream mapping (gaussian_sampler_S*, src/gauss.c) and the GPU counter mapping
(gaussian_sampler_S*_gpu, src/sample_gpu.cu).
"""
import numpy as np
import pytest

from oracle.ffi import Oracle, aes256_expand
from tests.conftest import seeds

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import cufe_b200 as cf  # noqa: E402
from cufe_b200.stats import ChiSquare, homogeneity, sigma_of, signed_samples  # noqa: E402

N = 4096
P_MIN = 1e-6


def oracle_counts(sig, mapping, rng, nsamp, nbins):
    O = Oracle(N, 8)
    acc = ChiSquare(sigma_of(sig), nbins)
    done = 0
    while done < nsamp:
        key = seeds(rng)[0]
        if mapping == "cpu":
            r, _ = O.gauss(sig, key, 16)
        else:
            rk = aes256_expand(key)
            r = np.stack([O.gauss_modeB(rk, sig, p) for p in range(16)])
        acc.add(signed_samples(torch.from_numpy(r.view(np.int32))))
        done += r.shape[0] * N
    return acc


@pytest.mark.parametrize("mapping", ["cpu", "gpu"])
@pytest.mark.parametrize("sig", [0, 1, 2])
def test_sampler_chi_square(sig, mapping, rng, oracle_built):
    c = cf.Context(N, 8)
    nbins = 200
    acc = ChiSquare(sigma_of(sig), nbins)
    if mapping == "cpu":
        out = c.sample_cpu_map(sig, seeds(rng, 64), 16)  # 64 streams x 16 calls x 4096
    else:
        out = c.sample_gpu_map(sig, seeds(rng)[0], 0, 1024)  # 1024 polynomials x 4096
    c.sync()
    acc.add(signed_samples(out))
    assert acc.counts.sum() == 2 ** 22
    ideal = acc.result()
    if sig == 0:
        assert ideal["p_value"] > P_MIN, ideal
    else:
        assert ideal["p_value"] < 1e-12, ideal  # the reference's sigma_2/sigma_3 shape, reproduced
        ref = oracle_counts(sig, mapping, rng, 2 ** 20, nbins)
        h = homogeneity(acc, ref)
        assert h["p_value"] > P_MIN, h
    c.close()
