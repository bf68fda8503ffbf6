"""The kernels' division by a small integer constant D (common.cuh div_k):
q0 = x RN(1/D), r = x - q0 D (one FMA, exact), q = RN(q0 + r RN(1/D)) (one
more FMA).  Emulated here in exact rational arithmetic and compared with the
correctly rounded x / D for random FP64 and FP32 x and every divisor the
stepper algebra uses; it must never differ (the kernels rely on it to keep the
results of plain division)."""
import random
import struct
from fractions import Fraction as F

import numpy as np
import pytest

DIVISORS = (3, 6, 11, 12, 22, 33, 39, 44, 48)


def _rn32(q):
    d = np.float32(float(q))
    cands = [np.nextafter(d, np.float32(-np.inf)), d, np.nextafter(d, np.float32(np.inf))]
    return min(cands, key=lambda c: (abs(F(float(c)) - q), int(np.float32(c).view(np.uint32)) & 1))


def _random_float(bits, rng):
    while True:
        if bits == 64:
            x = struct.unpack("d", struct.pack("Q", rng.getrandbits(64)))[0]
            if np.isfinite(x) and 1e-300 < abs(x) < 1e300:
                return x
        else:
            x = float(np.frombuffer(struct.pack("I", rng.getrandbits(32)), np.float32)[0])
            if np.isfinite(x) and 1e-35 < abs(x) < 1e35:
                return x


@pytest.mark.parametrize("bits", [64, 32])
@pytest.mark.parametrize("D", DIVISORS)
def test_fma_corrected_division_is_correctly_rounded(D, bits):
    rn = (lambda q: float(q)) if bits == 64 else (lambda q: float(_rn32(q)))
    rng = random.Random(D * 1000 + bits)
    inv = F(rn(F(1, D)))
    for _ in range(3000 if bits == 64 else 1500):
        x = F(_random_float(bits, rng))
        q0 = F(rn(x * inv))
        r = F(rn(x - q0 * D))
        assert r == x - q0 * D                 # the residual is exact
        q = rn(q0 + r * inv)
        assert q == rn(x / D)
