"""The exact-order reduction (pbg_seq_sum): the sequential left-to-right sum
with rounding after every addition, the reference's `for_ijk sum += ...`
(Src/Field/Scalar/scalar.h:296-326), computed in parallel on the GPU.

The checker is numpy's add.accumulate, which adds strictly in order. Every
case must agree bit for bit; the cases cover the paths of the parallel
algorithm: sums that stay in one binade, sums that cross zero over and over
(term-by-term chunks), magnitudes spread over 40 binades, exact ties
(half-ulp terms), zeros, sizes that are not a multiple of the 256-term chunk,
non-finite terms, and a 16.7 M-term sum (the 256^3 grid).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def seq(a):
    return float(np.add.accumulate(a)[-1])


def cases():
    rng = np.random.default_rng(7)
    n = 300_017
    yield "positive", rng.random(n)
    yield "mixed_sign", rng.standard_normal(n)
    yield "drift", rng.standard_normal(n) + 0.01
    yield "spread", rng.standard_normal(n) * np.exp(rng.uniform(-14, 14, n))
    yield "zeros", np.where(rng.random(n) < 0.5, 0.0, rng.random(n))
    yield "ties", rng.integers(-3, 4, n).astype(np.float64) * 0.5
    yield "products", rng.standard_normal(n) * rng.standard_normal(n)
    yield "one", np.array([3.25])
    yield "short", rng.random(255)
    yield "chunk", rng.random(256)
    yield "tail", rng.random(256 * 64 * 3 + 17)
    yield "tiny", rng.random(1000) * 1e-310
    yield "cancel", np.concatenate([np.full(1000, 1e16), rng.random(5000), np.full(1000, -1e16)])


@pytest.mark.parametrize("name,a", list(cases()), ids=[c[0] for c in cases()])
def test_seq_sum_matches_sequential(engine, name, a):
    with engine.Session(4, 4, 4, 0.25) as s:
        b = a[::-1].copy()
        got = s.seq_sum(a, b)
        assert got[0] == seq(a), (name, got[0], seq(a))
        assert got[1] == seq(b), (name, got[1], seq(b))
        # twice in a row: the scratch keeps nothing between calls
        assert s.seq_sum(a)[0] == seq(a)


def test_seq_sum_non_finite(engine):
    a = np.random.default_rng(3).random(70_000)
    with engine.Session(4, 4, 4, 0.25) as s:
        a1 = a.copy()
        a1[5000] = np.nan
        assert np.isnan(s.seq_sum(a1)[0])
        a2 = a.copy()
        a2[60_000] = np.inf
        assert s.seq_sum(a2)[0] == np.inf


def test_seq_sum_device_16m(engine):
    """16.7 M terms (one 256^3 field): r.z-like positive products and
    p.Ap-like products with a positive mean, from device memory."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(11)
    n = 256 ** 3
    r = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    z = r * torch.rand(n, dtype=torch.float64, device="cuda", generator=g)
    q = torch.randn(n, dtype=torch.float64, device="cuda", generator=g) + 0.3 * r
    a, b = r * z, r * q
    torch.cuda.synchronize()  # the library reads them on its own stream
    with engine.Session(4, 4, 4, 0.25) as s:
        got = s.seq_sum(a, b)
    ha, hb = a.cpu().numpy(), b.cpu().numpy()
    assert got[0] == seq(ha)
    assert got[1] == seq(hb)
