"""The register/shared-memory plan of the NTT kernels (cufe_b200/csrc/ntt.cuh, NttPlan),
restated in Python and checked on the CPU for every ring size and radix the kernels use:

- in each pass, (thread, register) -> coefficient index is a bijection onto [0, n), and the
  thread's bits and the register's bits are disjoint (idx = idx_th + idx_e), which is what
  lets the kernels address register e with a compile-time offset;
- a pass of rb stages pairs, in its stage LS, registers that differ only in the butterfly
  bit of that stage (a radix-2^rb block is held by one thread);
- the shared-memory layout pad(j) = j + (j >> s) (s = 6 for radix 64, else 5) is injective,
  fits SMEM_WORDS and is additive over the disjoint thread and register bits (so an address
  is a per-thread base plus an immediate);
- with thread bits 4 and 5 swapped in the middle radix-16 passes, every exchange between
  passes is free of shared-memory bank conflicts, for the stores of the pass that ends and
  the loads of the pass that begins (one warp = 32 consecutive threads of a residue group).
"""
from collections import Counter

import pytest


class Plan:
    def __init__(self, logn, le):
        self.logn, self.le = logn, le
        self.E = 1 << le
        self.N = 1 << logn
        self.T = self.N // self.E
        self.NP = (logn + le - 1) // le
        self.R0 = logn - le * (self.NP - 1)

    def rb(self, p):
        return self.R0 if p == 0 else self.le

    def s0(self, p):
        return 0 if p == 0 else self.R0 + self.le * (p - 1)

    def lane_swap(self, p):
        return self.le == 4 and self.logn - self.s0(p) - self.rb(p) == 4 and self.T >= 64

    def vth(self, p, th):
        if not self.lane_swap(p):
            return th
        return (th & ~0x30) | (((th >> 5) & 1) << 4) | (((th >> 4) & 1) << 5)

    def idx_th(self, p, th):
        th = self.vth(p, th)
        plo, phi = self.logn - self.s0(p) - self.rb(p), self.logn - 1 - self.s0(p)
        return ((th >> plo) << (phi + 1)) | (th & ((1 << plo) - 1))

    def idx_e(self, p, e):
        rb = self.rb(p)
        plo, phi = self.logn - self.s0(p) - rb, self.logn - 1 - self.s0(p)
        v = (e >> rb) * self.T
        return ((v >> plo) << (phi + 1)) | ((e & ((1 << rb) - 1)) << plo) | (v & ((1 << plo) - 1))

    def pad(self, j):
        return j + (j >> (6 if self.le == 6 else 5))

    def smem_words(self):
        return self.N + (self.N >> (6 if self.le == 6 else 5))


# (log n, log2 coefficients per thread) of every k_ntt instantiation: radix 16 for all rings,
# radix 32 from n = 1024, radix 64 from n = 2048
PLANS = [(lg, 4) for lg in range(4, 14)] + [(lg, 5) for lg in range(10, 14)] + [(lg, 6) for lg in range(11, 14)]


@pytest.mark.parametrize("logn,le", PLANS)
def test_plan_bijective_and_disjoint(logn, le):
    P = Plan(logn, le)
    assert P.R0 >= 1 and P.T >= 1
    for p in range(P.NP):
        seen = set()
        for th in range(P.T):
            for e in range(P.E):
                a, b = P.idx_th(p, th), P.idx_e(p, e)
                assert a & b == 0
                seen.add(a + b)
        assert seen == set(range(P.N)), (logn, le, p)


@pytest.mark.parametrize("logn,le", PLANS)
def test_plan_stage_pairs(logn, le):
    """stage LS of pass p (global stage s = s0 + LS) pairs e1 and e1 + half, half =
    2^(rb-1-LS): their indices differ exactly in bit logn-1-s"""
    P = Plan(logn, le)
    for p in range(P.NP):
        rb = P.rb(p)
        for ls in range(rb):
            half, bit = 1 << (rb - 1 - ls), logn - 1 - (P.s0(p) + ls)
            for e1 in range(P.E):
                if e1 & half:
                    continue
                assert P.idx_e(p, e1) ^ P.idx_e(p, e1 + half) == 1 << bit


@pytest.mark.parametrize("logn,le", PLANS)
def test_layout_injective_additive(logn, le):
    P = Plan(logn, le)
    img = [P.pad(j) for j in range(P.N)]
    assert len(set(img)) == P.N and max(img) < P.smem_words()
    for p in range(P.NP):
        for th in range(P.T):
            a = P.idx_th(p, th)
            for e in range(P.E):
                b = P.idx_e(p, e)
                assert P.pad(a + b) == P.pad(a) + P.pad(b)


@pytest.mark.parametrize("logn,le", [pl for pl in PLANS if Plan(*pl).logn >= 10])
def test_exchanges_conflict_free(logn, le):
    P = Plan(logn, le)
    for p in range(P.NP):
        for e in range(P.E):
            for w0 in range(0, P.T, 32):
                banks = Counter(P.pad(P.idx_th(p, th) + P.idx_e(p, e)) % 32 for th in range(w0, w0 + 32))
                assert max(banks.values()) == 1, (logn, le, p, e, w0)
