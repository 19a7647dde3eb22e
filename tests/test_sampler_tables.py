"""The device sampler's constant tables (csrc/sampler.cuh) hold what they
claim: the first 128 primes of HaltonSampler::kPrimes, 1.f / prime rounded to
nearest, and ceil(2^64 / prime), whose multiply-high gives floor(n / prime)
for every 32-bit n."""
import os
import re

import numpy as np

SRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "anacapa_b200", "csrc",
                   "sampler.cuh")


def _table(name):
    s = open(SRC).read()
    body = re.search(name + r"\[128\] = \{(.*?)\};", s, re.S).group(1)
    return [v.strip() for v in body.replace("\n", " ").split(",") if v.strip()]


def _primes(k):
    out, c = [], 2
    while len(out) < k:
        if all(c % p for p in out if p * p <= c):
            out.append(c)
        c += 1
    return out


def test_prime_tables():
    primes = [int(v) for v in _table("c_primes")]
    assert primes == _primes(128)
    inv = [float.fromhex(v.rstrip("f")) for v in _table("c_inv_primes")]
    assert inv == [float(np.float32(1.0) / np.float32(p)) for p in primes]
    magic = [int(v.rstrip("ULL"), 16) for v in _table("c_magic")]
    rng = np.random.default_rng(0)
    for p, m in zip(primes, magic):
        assert m == -(-(1 << 64) // p) and m < 1 << 64
        ns = [0, 1, p - 1, p, p + 1, (1 << 32) - 1, (1 << 32) - p] + [int(x) for x in rng.integers(0, 1 << 32, 500)]
        for n in ns:
            assert (n * m) >> 64 == n // p
