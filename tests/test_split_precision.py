"""The split-precision arithmetic of the mixed path's tensor-core products,
modelled in numpy (CPU): the same splits the kernels and the host upload
make, the same three products, exact float16 x float16 products accumulated
in float64 here (the tensor pipe accumulates in float32, which the GPU tests
cover).

Scaled F16 (csrc/m2l_tc.cu k_split_proxy_f16, k_colgemm_tc; csrc/api.cu
split_f16_rows): each row x is scaled by 2^e so that max |x| 2^e lies in
[2^14, 2^15), hi = fp16(x 2^e), lo = fp16(x 2^e - hi); D = A_lo B_hi +
A_hi B_lo + A_hi B_hi, unscaled by 2^-(e_A + e_B).
TF32 (csrc/api.cu tf32_round, m2l_tc.cu to_tf32): hi = tf32(x), lo = tf32(x - hi)."""
import numpy as np
import pytest


def split_f16(x):
    """Rows of x (float32) -> (hi, lo, e) with the kernels' scaling."""
    m = np.abs(x).max(axis=1)
    _, k2 = np.frexp(m)
    e = np.where(m > 0, 15 - k2, 0)
    xs = np.ldexp(x.astype(np.float32), e[:, None]).astype(np.float32)
    hi = xs.astype(np.float16)
    lo = (xs - hi.astype(np.float32)).astype(np.float16)
    return hi, lo, e


def tf32(x):
    """float32 -> TF32 (10 explicit mantissa bits), nearest, ties away."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x1000) & 0xFFFFE000).astype(np.uint32)
    return u.view(np.float32)


def three_products(ah, al, bh, bl):
    f = lambda v: v.astype(np.float64)
    return f(al) @ f(bh).T + f(ah) @ f(bl).T + f(ah) @ f(bh).T


def f16_product(A, B):
    ah, al, ea = split_f16(A)
    bh, bl, eb = split_f16(B)
    D = three_products(ah, al, bh, bl)
    return np.ldexp(D, -(ea[:, None] + eb[None, :]))


def tf32_product(A, B):
    ah = tf32(A)
    al = tf32(A - ah)
    bh = tf32(B)
    bl = tf32(B - bh)
    return three_products(ah, al, bh, bl)


def _mats(rng, m=64, n=48, k=120, spread=0.0):
    A = rng.standard_normal((m, k)).astype(np.float32)
    B = rng.standard_normal((n, k)).astype(np.float32)
    if spread:  # rows of very different magnitudes
        A *= np.exp2(rng.uniform(-spread, spread, (m, 1))).astype(np.float32)
    return A, B


@pytest.mark.parametrize("product", [f16_product, tf32_product], ids=["f16", "tf32"])
def test_three_products_reach_float32_level(product):
    """Row-relative error against float64 A B^T: a few 2^-22 (the dropped
    lo x lo term and the splitting), far below a single TF32/F16 product's
    2^-11."""
    rng = np.random.default_rng(1)
    A, B = _mats(rng)
    exact = A.astype(np.float64) @ B.astype(np.float64).T
    scale = np.abs(A).astype(np.float64) @ np.abs(B).astype(np.float64).T
    err = np.abs(product(A, B) - exact) / scale
    assert err.max() < 2.0 ** -20, err.max()
    single = (A.astype(np.float16).astype(np.float64) @ B.astype(np.float16).astype(np.float64).T)
    assert (np.abs(single - exact) / scale).max() > 2.0 ** -14  # what one product would give


def test_f16_rows_of_any_magnitude():
    """Per-row power-of-two scales: rows spanning 2^-100 .. 2^100 (far outside
    F16's range unscaled) keep the same row-relative accuracy, and scaling the
    rows by 2^k scales the result exactly."""
    rng = np.random.default_rng(2)
    A, B = _mats(rng, spread=100.0)
    exact = A.astype(np.float64) @ B.astype(np.float64).T
    scale = np.abs(A).astype(np.float64) @ np.abs(B).astype(np.float64).T
    D = f16_product(A, B)
    assert (np.abs(D - exact) / scale).max() < 2.0 ** -20
    # exact scaling (rows kept inside float32's range after the 2^+-60)
    A, B = _mats(rng, spread=40.0)
    D = f16_product(A, B)
    for k in (-60, 60):
        Dk = f16_product(np.ldexp(A, k).astype(np.float32), B)
        assert np.array_equal(Dk, np.ldexp(D, k))


def test_f16_split_is_exact_where_it_claims():
    """x 2^e = hi + lo + r with |r| <= 2^-22 |x 2^e| for elements within
    2^-17 of the row's largest (both parts normal F16), and an absolute
    |r| <= 2^-25 (half the F16 subnormal spacing) below that."""
    rng = np.random.default_rng(3)
    x = (rng.standard_normal((16, 256)) * np.exp2(rng.uniform(-30, 0, (16, 256)))).astype(
        np.float32)
    hi, lo, e = split_f16(x)
    xs = np.ldexp(x.astype(np.float64), e[:, None])
    r = np.abs(xs - hi.astype(np.float64) - lo.astype(np.float64))
    big = np.abs(xs) >= 2.0 ** -3  # within 2^-17 of a row max in [2^14, 2^15)
    assert (r[big] <= 2.0 ** -22 * np.abs(xs[big])).all()
    assert (r[~big] <= 2.0 ** -25).all()
    assert (np.abs(xs).max(axis=1) < 2.0 ** 15).all() and (np.abs(xs).max(axis=1) >= 2.0 ** 14).all()
