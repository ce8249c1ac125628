"""The compensated FP32 sum step of the kernels (Acc2 / Acc2x2,
cup-cfd_b200/csrc/kernels.cuh), restated in exact rational arithmetic.

One step adds a*b to the running sum s with error term e:
    p = fl(a b)            (written fma(a, b, +0) in the kernels)
    t = fl(s + p)
    nbp = fl(s - t)
    ar = fl(s - fl(t + nbp))          Knuth's TwoSum: s's exact low part
    brp = fl(a b + nbp)   (one FMA)   the product's error plus p's low part
    e += fl(ar + brp)
The claim: fl(ar + brp) equals the step's exact error s + a b - t to within
a small multiple of u^2 max(|t|, |s|, |a b|) (u = 2^-24), in every magnitude
relation, cancellation included. And the form the compiler produced when it
fused the packed multiply and add (t = fl(a b + s), one rounding) does not
keep that bound: there the error term is wrong by up to one ulp of the terms.
"""
from fractions import Fraction as F

import numpy as np

U = F(1, 2 ** 24)


def rn(x):
    """Exact rational -> nearest float32, ties to even."""
    if x == 0:
        return np.float32(0.0)
    f = np.float32(float(x))
    best = None
    for c in (np.nextafter(f, np.float32(-np.inf)), f, np.nextafter(f, np.float32(np.inf))):
        err = abs(F(float(c)) - x)
        if best is None or err < best[0] or (err == best[0] and (int(c.view(np.int32)) & 1) == 0):
            best = (err, c)
    return best[1]


def fx(v):
    return F(float(v))


def step_error(a, b, s, fused):
    """(recovered error, exact error, scale) of one step."""
    A, B, S = fx(a), fx(b), fx(s)
    t = rn(A * B + S) if fused else rn(S + fx(rn(A * B)))
    nbp = rn(S - fx(t))
    ar = rn(S - fx(rn(fx(t) + fx(nbp))))
    brp = rn(A * B + fx(nbp))
    return fx(rn(fx(ar) + fx(brp))), S + A * B - fx(t), max(abs(fx(t)), abs(S), abs(A * B))


def cases(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        a = np.float32(rng.uniform(-1, 1))
        b = np.float32(rng.uniform(-1, 1) * 10.0 ** rng.integers(-4, 3))
        k = i % 4
        if k == 0:
            s = np.float32(rng.uniform(-1, 1) * 10.0 ** rng.integers(-6, 4))
        elif k == 1:   # near cancellation
            s = rn(-fx(a) * fx(b) * (1 + F(int(rng.integers(-1000, 1001)), 2 ** 22)))
        elif k == 2:   # s = -fl(a b)
            s = rn(-fx(a) * fx(b))
        else:          # |s| << |a b|
            s = np.float32(rng.uniform(-1, 1) * 10.0 ** rng.integers(-12, -5))
        out.append((a, b, s))
    return out


def test_step_recovers_exact_error_to_second_order():
    worst = F(0)
    for a, b, s in cases(4000, 11):
        rec, exact, scale = step_error(a, b, s, fused=False)
        if scale:
            worst = max(worst, abs(rec - exact) / (U * U * scale))
    assert worst <= 2, float(worst)


def test_fused_product_and_add_loses_the_bound():
    worst = F(0)
    for a, b, s in cases(4000, 11):
        rec, exact, scale = step_error(a, b, s, fused=True)
        if scale:
            worst = max(worst, abs(rec - exact) / (U * scale))
    assert worst > F(1, 4), float(worst)   # first order: a sizeable part of an ulp
