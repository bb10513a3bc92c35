"""Distribution checks for the discrete Gaussian samplers.

The samplers emit residues mod the three RNS primes.  `signed_samples` recovers the signed
integer sample from the residues mod q_1 and q_2 (every sample of the three sigmas is far
below q_1 q_2 / 2 in magnitude), and `ChiSquare` bins the samples into equiprobable bins of
the ideal discrete Gaussian D_{Z,sigma}, sigma = K sigma_0 with sigma_0 = 1/sqrt(2 ln 2) and
K = 266, 304214978, 608429953 (the three sampler scale factors, src/gauss.c:11-13).

The reference's sigma_2 and sigma_3 samplers are not D_{Z,sigma}: their Bernoulli step turns
the 64-bit exponent input (2Kx + y mod 2^32) * y into a double by OR-ing the exponent bits of
2^52 into it and subtracting 2^52 (src/gauss.c:418-576, src/sampler.cuh:183-422), which is
exact only below 2^52; for y > 2^26 (sigma_2) the input is larger and the acceptance
probability is wrong.  The kernels reproduce that bit for bit, so for sigma_2 and sigma_3 the
distribution check that can pass is `homogeneity`: GPU samples against samples of the CPU
restatement of the same mapping on independent seeds.

The bin probabilities use the normal CDF with continuity correction,
P(a <= X < b) = Phi((b - 1/2)/sigma) - Phi((a - 1/2)/sigma): for sigma >= 200 the discrete
Gaussian's mass at the integers matches the continuous density to within exp(-2 pi^2 sigma^2)
(Poisson summation), far below any count's sampling error.
"""
import math

import numpy as np

from . import Q

SIGMA0 = 1.0 / math.sqrt(2.0 * math.log(2.0))
SIGMA_K = (266, 304214978, 608429953)


def sigma_of(sig):
    return SIGMA_K[sig] * SIGMA0


def signed_samples(res):
    """int64 samples from residues of shape [..., 3, n] (torch, any device): CRT of the
    residues mod q_1 and q_2, centred into (-q_1 q_2 / 2, q_1 q_2 / 2]"""
    import torch
    q1, q2 = Q[1], Q[2]
    r = res.reshape(-1, 3, res.shape[-1])
    # canonical: the reference's residues may equal q itself
    r1 = torch.remainder(r[:, 1].to(torch.int64) & 0xFFFFFFFF, q1)
    r2 = torch.remainder(r[:, 2].to(torch.int64) & 0xFFFFFFFF, q2)
    inv = pow(q1, -1, q2)
    t = torch.remainder(r2 - torch.remainder(r1, q2), q2)
    t = torch.remainder(t * inv, q2)
    x = r1 + q1 * t
    m = q1 * q2
    return torch.where(x > m // 2, x - m, x).reshape(-1)


def _phi(z):
    return 0.5 * math.erfc(-z / math.sqrt(2.0))


class ChiSquare:
    """Pearson chi-square of integer samples against D_{Z,sigma} on `nbins` bins whose edges
    are the integer quantiles of the ideal distribution (the two outer bins are open)."""

    def __init__(self, sigma, nbins=1000):
        from statistics import NormalDist
        nd = NormalDist(0.0, sigma)
        edges = sorted({int(math.floor(nd.inv_cdf(i / nbins) + 0.5)) for i in range(1, nbins)})
        self.sigma = sigma
        self.edges = np.array(edges, np.int64)  # bin b = [edges[b-1], edges[b])
        cdf = np.array([_phi((e - 0.5) / sigma) for e in edges])
        self.prob = np.diff(np.concatenate([[0.0], cdf, [1.0]]))
        self.counts = np.zeros(len(self.prob), np.int64)
        self._edges_dev = None

    def add(self, x):
        """accumulate a torch int64 tensor of samples (binned on its device)"""
        import torch
        if self._edges_dev is None or self._edges_dev.device != x.device:
            self._edges_dev = torch.from_numpy(self.edges).to(x.device)
        b = torch.bucketize(x, self._edges_dev, right=True)
        self.counts += torch.bincount(b, minlength=len(self.prob)).cpu().numpy()

    def result(self):
        from scipy.stats import chi2
        n = int(self.counts.sum())
        exp = self.prob * n
        dev = (self.counts - exp) / np.sqrt(exp)
        stat = float((dev ** 2).sum())
        df = len(self.prob) - 1
        worst = np.argsort(-np.abs(dev))[:3]
        return {"samples": n, "bins": len(self.prob), "chi2": stat, "df": df,
                "p_value": float(chi2.sf(stat, df)),
                "worst_bins": [{"lo": int(self.edges[b - 1]) if b > 0 else None,
                                "hi": int(self.edges[b]) if b < len(self.edges) else None,
                                "z": float(dev[b])} for b in worst]}


def homogeneity(a, b):
    """two-sample Pearson chi-square of two ChiSquare accumulators with the same bins: are
    both sets of counts draws from one distribution?"""
    from scipy.stats import chi2
    ca, cb = a.counts.astype(np.float64), b.counts.astype(np.float64)
    na, nb = ca.sum(), cb.sum()
    keep = (ca + cb) > 0
    ca, cb = ca[keep], cb[keep]
    stat = float((((ca * math.sqrt(nb / na) - cb * math.sqrt(na / nb)) ** 2) / (ca + cb)).sum())
    df = int(keep.sum()) - 1
    return {"samples": [int(na), int(nb)], "bins": int(keep.sum()), "chi2": stat, "df": df,
            "p_value": float(chi2.sf(stat, df))}
