"""The library's software binary64 operations (csrc/softf64.cuh, used by the device SAH build and
the exact fallbacks) against the machine's IEEE-754 doubles: every result bit-identical (NaN-ness
for NaN results), over random operands drawn to cover every exponent range, subnormals, zeros of
both signs, infinities, NaNs, exact cancellations, ties and carries."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N = 400_000


@pytest.fixture(scope="module")
def sf(tmp_path_factory):
    out = tmp_path_factory.mktemp("sf") / "libsoftf64_check.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I",
                    os.path.join(ROOT, "three-mesh-bvh_b200", "csrc"),
                    os.path.join(ROOT, "tests", "native", "softf64_check.cpp"), "-o", str(out)], check=True)
    lib = C.CDLL(str(out))
    lib.sf_eval.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]

    def run(op, a, b=None):
        a = np.ascontiguousarray(a, dtype=np.uint64)
        b = np.ascontiguousarray(a if b is None else b, dtype=np.uint64)
        o = np.empty_like(a)
        lib.sf_eval(op, a.ctypes.data, b.ctypes.data, o.ctypes.data, a.size)
        return o

    return run


def _operands(rng, n):
    """Doubles whose exponents span the whole range (uniform bit patterns), values near 1, float32
    values, subnormals and special values, mixed."""
    parts = [
        rng.integers(0, 2**64, n, dtype=np.uint64),
        (rng.standard_normal(n) * np.exp(rng.uniform(-40, 40, n))).view(np.uint64),
        rng.standard_normal(n).astype(np.float32).astype(np.float64).view(np.uint64),
        (rng.integers(0, 2**52, n, dtype=np.uint64) | (rng.integers(0, 2, n, dtype=np.uint64) << np.uint64(63))),
        rng.choice(np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1.0, -1.0, 2.0**-1022, 2.0**-1074,
                             np.finfo(np.float64).max, 0.5, 3.0]), n).view(np.uint64),
    ]
    x = np.concatenate(parts)
    return x[rng.permutation(x.size)][:n]


def _same(got, want):
    g, w = got.view(np.float64), want.view(np.float64)
    both_nan = np.isnan(g) & np.isnan(w)
    return both_nan | (got == want.view(np.uint64))


@pytest.mark.parametrize("op,fn", [(0, np.add), (1, np.subtract), (2, np.multiply), (3, np.divide)])
def test_binary_ops_match_ieee(sf, op, fn):
    rng = np.random.default_rng(100 + op)
    a, b = _operands(rng, N), _operands(rng, N)
    # close operands: cancellations in add/sub, ratios near 1 in div
    with np.errstate(all="ignore"):
        close = (a.view(np.float64) * (1 + rng.standard_normal(N) * 2.0**-40)).view(np.uint64)
    # 27-bit significands: products of exactly 54 bits, half of them exact ties at binary64 precision
    short = (rng.integers(2**26, 2**27, (2, N)).astype(np.float64) * np.exp2(rng.integers(-60, 60, (2, N))))
    a = np.concatenate([a, a, short[0].view(np.uint64)])
    b = np.concatenate([b, close, short[1].view(np.uint64)])
    with np.errstate(all="ignore"):
        want = fn(a.view(np.float64), b.view(np.float64))
    got = sf(op, a, b)
    bad = ~_same(got, want.view(np.uint64))
    assert not bad.any(), (a[bad][:3].view(np.float64), b[bad][:3].view(np.float64), got[bad][:3].view(np.float64))


def test_products_of_float32_and_small_integers(sf):
    """The SAH cost terms: float32 box extents, their products, integer counts."""
    rng = np.random.default_rng(7)
    f = rng.uniform(-50, 50, (N, 2)).astype(np.float32).astype(np.float64)
    cnt = rng.integers(0, 2**24, N).astype(np.float64)
    for a, b in ((f[:, 0], f[:, 1]), (f[:, 0] * f[:, 1], cnt), (f[:, 0], np.full(N, 1.25))):
        for op, fn in ((0, np.add), (2, np.multiply), (3, np.divide)):
            with np.errstate(all="ignore"):
                want = fn(a, b)
            assert _same(sf(op, a.view(np.uint64), b.view(np.uint64)), want.view(np.uint64)).all()


def test_sqrt_matches_ieee(sf):
    rng = np.random.default_rng(5)
    a = np.concatenate([_operands(rng, N), np.abs(rng.standard_normal(N)).view(np.uint64)])
    with np.errstate(all="ignore"):
        want = np.sqrt(a.view(np.float64))
    assert _same(sf(4, a), want.view(np.uint64)).all()


def test_comparisons_match_ieee(sf):
    rng = np.random.default_rng(6)
    a = _operands(rng, N)
    b = np.where(rng.random(N) < 0.2, a, _operands(rng, N))
    b = np.where(rng.random(N) < 0.05, a ^ np.uint64(1 << 63), b)  # opposite signs, incl. -0 / +0
    x, y = a.view(np.float64), b.view(np.float64)
    got = sf(5, a, b)
    assert np.array_equal(got & 1, (x < y).astype(np.uint64))
    assert np.array_equal((got >> 1) & 1, (x <= y).astype(np.uint64))
    assert np.array_equal((got >> 2) & 1, (x == y).astype(np.uint64))


def test_float32_conversions(sf):
    rng = np.random.default_rng(8)
    a = _operands(rng, N)
    with np.errstate(all="ignore"):
        want = a.view(np.float64).astype(np.float32)
    got = sf(6, a).astype(np.uint32)
    w = want.view(np.uint32)
    ok = (np.isnan(want) & np.isnan(got.view(np.float32))) | (got == w)
    assert ok.all(), a[~ok][:3].view(np.float64)
    # ties at float32 precision (exactly half an ulp away) round to even
    base = rng.standard_normal(N).astype(np.float32).astype(np.float64)
    tie = base + np.spacing(base.astype(np.float32)).astype(np.float64) / 2
    assert np.array_equal(sf(6, tie.view(np.uint64)).astype(np.uint32), tie.astype(np.float32).view(np.uint32))
    u = rng.integers(0, 2**32, N, dtype=np.uint64)
    f = u.astype(np.uint32).view(np.float32)
    with np.errstate(all="ignore"):
        wide = f.astype(np.float64)
    assert _same(sf(7, u), wide.view(np.uint64)).all()


def test_integer_conversions(sf):
    rng = np.random.default_rng(9)
    u = np.concatenate([rng.integers(0, 2**53, N, dtype=np.uint64), rng.integers(0, 2**63, N, dtype=np.uint64),
                        np.arange(0, 4096, dtype=np.uint64)])
    assert np.array_equal(sf(8, u), u.astype(np.float64).view(np.uint64))
    x = np.concatenate([rng.uniform(-2**31 + 1, 2**31 - 1, N), rng.uniform(0, 33, N), np.array([np.nan, -0.0, 0.0])])
    got = sf(9, x.view(np.uint64)).view(np.int64)
    want = np.where(np.isnan(x), 0, np.trunc(np.nan_to_num(x))).astype(np.int64)
    assert np.array_equal(got, want)
