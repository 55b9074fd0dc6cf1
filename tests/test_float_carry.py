"""The float tallies' carry (kp_tallies_t::carry), restated on the CPU.

In float mode every deposit is an FP32 atomic add.  The kernel takes the
value the atomic read (old) and the addend v, forms the error of the sum
the atomic stored by TwoSum (Knuth, TAOCP vol. 2, 4.2.2; Moller 1965) and
adds that error to a second float array, which the solve adds into the
tally at its end (atomic_add_carry and k_fold_carry in
kratos_polrad_b200/csrc).  These tests restate that arithmetic in numpy
float32 and check it on the oracle's own image deposits, summed in random
orders as the atomics of the GPU may sum them.
"""
import numpy as np
import pytest

from oracle import port
from transport_cases import case, run_oracle

pytestmark = pytest.mark.skipif(not port.available(), reason="oracle not built")

f32 = np.float32


def two_sum(old, v):
    """s = fl(old + v) and e with old + v = s + e exactly (float32 arrays)."""
    s = f32(old + v)
    bv = f32(s - old)
    e = f32(f32(old - f32(s - bv)) + f32(v - bv))
    return s, e


def test_two_sum_is_error_free():
    rng = np.random.default_rng(0)
    a = (rng.standard_normal(200000) * np.exp(rng.uniform(-30, 30, 200000))).astype(f32)
    b = (rng.standard_normal(200000) * np.exp(rng.uniform(-30, 30, 200000))).astype(f32)
    s, e = two_sum(a, b)
    # float32 values and their pairwise sums are exact in float64
    np.testing.assert_array_equal(s.astype(np.float64) + e.astype(np.float64),
                                  a.astype(np.float64) + b.astype(np.float64))


def _sum_in_order(pix, val, n_pix, order, carry):
    """Sequential float32 sums of the deposits per pixel in `order`, as the
    atomics add them; with `carry` the TwoSum errors go to a second array,
    added in at the end."""
    pix, val = pix[order], val[order]
    srt = np.argsort(pix, kind="stable")
    pix, val = pix[srt], val[srt]
    start = np.searchsorted(pix, np.arange(n_pix))
    count = np.bincount(pix, minlength=n_pix)
    hi = np.zeros((n_pix, 4), f32)
    lo = np.zeros((n_pix, 4), f32)
    for k in range(int(count.max())):
        has = count > k
        v = val[start[has] + k]
        if carry:
            s, e = two_sum(hi[has], v)
            hi[has] = s
            lo[has] = f32(lo[has] + e)
        else:
            hi[has] = f32(hi[has] + v)
    return f32(hi + lo) if carry else hi


def test_carry_holds_every_pixel_within_1e6_of_exact():
    mesh, sig, t = case("amr_point")
    ref = run_oracle(mesh, sig, t, deposits=1 << 20)
    pix, val = ref["deposits"]
    n_pix = t.image_n * t.image_n
    exact = np.zeros((n_pix, 4))
    np.add.at(exact, pix, val.astype(np.float64))
    I = exact[:, 0]
    lit = I > 0
    rng = np.random.default_rng(1)
    worst_plain = 0.0
    for _ in range(3):
        order = rng.permutation(len(pix))
        got = _sum_in_order(pix, val, n_pix, order, carry=True).astype(np.float64)
        rel = np.abs(got - exact)[lit] / I[lit][:, None]
        assert rel.max() <= 1e-7, rel.max()
        plain = _sum_in_order(pix, val, n_pix, order, carry=False).astype(np.float64)
        worst_plain = max(worst_plain, (np.abs(plain - exact)[lit] / I[lit][:, None]).max())
    # the plain sums of the same orders miss 1e-6 (thousands of deposits in
    # the brightest pixels); this is what the carry is for
    assert worst_plain > 1e-6
