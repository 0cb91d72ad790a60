"""The FP32 state accumulator's renormalisation between two forwards of one
launch (``Acc<float>::renormalize`` in ``goss_b200/csrc/goss_kernels.cuh``).

A forward stores each state as ``double(hi) + double(lo)`` and the next one
loads it back as ``hi = float(v)``, ``lo = float(v - double(hi))``.  When a
launch runs several forwards, the kernel does the same round trip in FP32
arithmetic: a two-sum of hi and lo, then the error rounded (ties to even) to the
FP64 grid of hi + lo.  These tests restate both in numpy (IEEE binary32 and
binary64, round to nearest) and check that they agree bit for bit on random and
adversarial pairs, so that fused forwards equal one launch per forward.
"""
import numpy as np

TINY = np.float32(2.0**-72)  # below this the kernel takes the FP64 round trip itself


def round_trip(hi, lo):
    """What store() then load() do."""
    v = hi.astype(np.float64) + lo.astype(np.float64)
    h = v.astype(np.float32)
    lo2 = (v - h.astype(np.float64)).astype(np.float32)
    return h, lo2


def add_rz(a, b):
    """FP32 a + b rounded toward zero (the sum is exact in FP64 here: |b| is
    at most half an FP32 ulp of a)."""
    v = a.astype(np.float64) + b.astype(np.float64)
    f = v.astype(np.float32)
    away = np.abs(f.astype(np.float64)) > np.abs(v)
    return np.where(away, np.nextafter(f, np.float32(0)), f)


def renormalize_fp32(hi, lo):
    """The kernel's FP32 form, operation for operation."""
    f = np.float32
    t = hi + lo
    bp = t - hi
    ap = t - bp
    e = (hi - ap) + (lo - bp)
    # 2^floor(log2|hi + lo|): the binade of hi + lo rounded toward zero
    pow2 = (add_rz(t, e).view(np.uint32) & np.uint32(0x7F800000)).view(np.float32)
    P = pow2 * f(2.0**-29)  # 2^23 x the FP64 ulp of hi + lo
    C = np.copysign(P, e)
    r = (e + C) - C
    lo2 = np.where(np.abs(e) < P, r, e)
    # tiny or non-finite sums: the FP64 round trip itself
    at = np.abs(t)
    slow = ~((at >= TINY) & (at <= np.finfo(np.float32).max))
    h_rt, l_rt = round_trip(hi, lo)
    return np.where(slow, h_rt, t), np.where(slow, l_rt, lo2)


def check(hi, lo):
    with np.errstate(over="ignore", invalid="ignore"):
        a = round_trip(hi, lo)
        b = renormalize_fp32(hi, lo)
    for x, y in zip(a, b):
        same = (x.view(np.uint32) == y.view(np.uint32)) | (np.isnan(x) & np.isnan(y)) | ((x == 0) & (y == 0))
        bad = np.flatnonzero(~same)
        assert bad.size == 0, [(hi[i], lo[i], a[0][i], a[1][i], b[0][i], b[1][i]) for i in bad[:5]]


def test_random_accumulator_pairs():
    rng = np.random.default_rng(1234)
    n = 1 << 20
    # states of every magnitude, lo from one FP32 ulp of hi down to 2^-60 of it, either sign
    hi = (rng.choice([-1.0, 1.0], n) * 10.0 ** rng.uniform(-20, 6, n)).astype(np.float32)
    ulp = np.spacing(np.abs(hi)).astype(np.float64)
    lo = (rng.uniform(-1.0, 1.0, n) * ulp * 2.0 ** -rng.uniform(0, 60, n)).astype(np.float32)
    check(hi, lo)


def test_adversarial_accumulator_pairs():
    rng = np.random.default_rng(5678)
    n = 1 << 18
    # powers of two with lo of the opposite sign (the sum drops a binade) and
    # lo at exactly half an FP64 ulp (ties), near the tiny threshold, |lo| > |hi|
    k = rng.integers(-70, 40, n)
    hi = np.ldexp(1.0, k).astype(np.float32) * rng.choice([-1.0, 1.0], n).astype(np.float32)
    j = rng.integers(1, 60, n)
    lo = (-np.sign(hi) * np.ldexp(1.0, k - 24 - j) * rng.integers(1, 8, n)).astype(np.float32)
    check(hi, lo)
    ties = (np.ldexp(1.0, k - 53) * np.float64(rng.integers(1, 6, n))).astype(np.float32)
    check(hi, ties * np.sign(hi).astype(np.float32))
    check(hi, -ties * np.sign(hi).astype(np.float32))
    big_lo = (rng.uniform(-1, 1, n) * 10.0 ** rng.uniform(-3, 3, n)).astype(np.float32)
    small_hi = (rng.uniform(-1, 1, n) * 10.0 ** rng.uniform(-40, 0, n)).astype(np.float32)
    check(small_hi, big_lo)
    near = (np.ldexp(1.0, -72) * rng.uniform(0.5, 2.0, n)).astype(np.float32)
    check(near, (near.astype(np.float64) * 2.0 ** -rng.uniform(20, 40, n)).astype(np.float32))
    specials = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1.0, -1.0, 3.4e38], np.float32)
    a, b = np.meshgrid(specials, specials)
    check(a.ravel(), b.ravel())
