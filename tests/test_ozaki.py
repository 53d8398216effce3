"""Int8-emulated FP64 products (Ozaki scheme): the device digit split and the
tcgen05 kind::i8 GEMM against a numpy restatement of the same scheme.

The digit split is bit-exact against the restatement (the same IEEE
operations in the same order).  In the GEMM every int32 group product is
exact and pairs of groups combine exactly in int32; the kernel adds each
pair with one FMA (one rounding), the restatement with a product and a sum
(two), so the two agree to a few units in the last place of the terms added;
a second check bounds the distance to the plain FP64 product by the
truncation error of s digits.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KB = 128
BASE = 254.0  # digit base: |D_0| <= 64, |D_p| <= 127


def wpow(j):
    """1 / BASE^j with BASE^j formed by repeated multiplication, as the host
    code forms it."""
    p = 1.0
    for _ in range(j):
        p *= BASE
    return 1.0 / p


def np_exponents(X, block):
    """One exponent e per row (or 128-row block) and 128-column block with
    max|x| < 2^e (frexp's exponent); all-zero domains get -2000."""
    R, C = X.shape
    m = np.abs(X).reshape(R, C // KB, KB).max(axis=2)
    if block:
        rb = (R + 127) // 128
        mp = np.zeros((rb * 128, C // KB))
        mp[:R] = m
        m = mp.reshape(rb, 128, C // KB).max(axis=1)
    e = np.frexp(m)[1].astype(np.int64)
    return np.where(m > 0, e, -2000)


def np_split(X, s, block):
    R, C = X.shape
    E = np_exponents(X, block)
    Er = np.repeat(E, 128, axis=0)[:R] if block else E
    Ee = np.repeat(Er, KB, axis=1)
    t = X * np.ldexp(1.0, (6 - Ee).clip(-1022, 1023))
    t[Ee == -2000] = 0.0
    D = []
    for _ in range(s):
        d = np.rint(t)
        D.append(d)
        t = (t - d) * BASE
    return np.array(D), E


def np_oz_gemm(A, B, C, alpha, beta, s, groups=0, lower=False):
    """The kernel's arithmetic: per 128-column block k and group g an exact
    integer product P_g; groups taken in pairs as 254 P_g + P_{g+1} (exact),
    scaled by 2^(eA + eB - 12) / 254^(g+1) and added in FP64 (a last
    unpaired group as 254 P_g at the same scale).  Returns the result and
    the sum of the magnitudes of the terms added (for the rounding bound)."""
    G = groups or s
    DA, EA = np_split(A, s, False)
    DB, EB = np_split(B, s, True)
    M, N = A.shape[0], B.shape[0]
    acc = np.zeros((M, N))
    mag = np.zeros((M, N))
    ebcol = np.repeat(EB, 128, axis=0)[:N]  # per B row (= C column), per block
    for k in range(A.shape[1] // KB):
        sl = slice(k * KB, (k + 1) * KB)

        def group(g):
            P = np.zeros((M, N))
            for p in range(g + 1):
                P += DA[p][:, sl] @ DB[g - p][:, sl].T
            return P

        # groups in pairs: 128 P_g + P_{g+1} (exact integers), one scaled add per pair
        for g in range(0, G, 2):
            P = BASE * group(g) + (group(g + 1) if g + 1 < G else 0.0)
            e = EA[:, k][:, None] + ebcol[:, k][None, :] - 12
            term = P * np.ldexp(wpow(g + 1), e.clip(-1022, 1023))
            acc += term
            mag += np.abs(term)
    out = alpha * acc
    if beta != 0.0:
        out = C + out
    if lower:
        keep = np.tril(np.ones((M, N), dtype=bool))
        out = np.where(keep, out, C)
        mag = np.where(keep, mag, 0.0)
    return out, abs(alpha) * mag


@pytest.fixture(scope="module")
def capi():
    from gprat_b200 import capi as c

    return c


def graded(rng, rows, cols):
    """Rows of widely different magnitudes (the per-row exponents matter)."""
    X = rng.standard_normal((rows, cols))
    X *= np.exp2(rng.integers(-20, 4, size=(rows, 1)))
    X[:, :KB] *= np.exp2(rng.integers(-6, 6, size=(rows, 1)))  # the first column block differs
    return X


@pytest.mark.parametrize("block", [False, True])
@pytest.mark.parametrize("s", [3, 6, 7])
def test_split_matches_numpy(capi, block, s):
    rng = np.random.default_rng(11)
    X = graded(rng, 300, 256)
    X[7] = 0.0            # an all-zero row
    X[200:210, KB:] = 0.0  # zero in one column block only
    D, E = capi.test_oz_split(X, s, block)
    Dn, En = np_split(X, s, block)
    assert np.array_equal(E, En)
    assert np.array_equal(D.astype(np.float64), Dn)
    assert np.abs(D[0]).max() <= 64 and np.abs(D).max() <= 127
    # reconstruction: error below half a unit of the last digit (plus the
    # roundings of the base-254 products once the remainder fills 53 bits)
    Er = np.repeat(En, 128, axis=0)[:300] if block else En
    Ee = np.repeat(Er, KB, axis=1)
    rec = sum(Dn[p] * wpow(p) for p in range(s)) * np.ldexp(1.0, (Ee - 6).clip(-1022, 1023))
    rec[Ee == -2000] = 0.0
    bound = np.ldexp(0.5 * wpow(s - 1) + 2.0 ** -45, (Ee - 6).clip(-1022, 1023))
    assert np.all(np.abs(rec - X) <= bound)


@pytest.mark.parametrize("M,N,K,beta,lower,s,groups,max_ctas", [
    (300, 200, 384, 0.0, False, 6, 0, 0),
    (300, 200, 384, 1.0, False, 5, 0, 0),
    (384, 384, 256, 1.0, True, 6, 0, 0),
    (640, 640, 128, 1.0, True, 4, 0, 0),
    (1024, 1024, 1024, 1.0, False, 6, 0, 8),   # persistent: 4 pairs loop over 32 tiles
    (512, 128, 256, 0.0, False, 7, 5, 0),      # fewer groups than digits
    (128, 72, 128, 0.0, False, 7, 0, 0),       # ragged N, a single pair tile
])
def test_gemm_matches_restatement(capi, M, N, K, beta, lower, s, groups, max_ctas):
    rng = np.random.default_rng(M + N + K + s)
    A = graded(rng, M, K)
    B = graded(rng, N, K)
    C = rng.standard_normal((M, N))
    if lower:
        B = A.copy()
    out = C.copy()
    capi.test_oz_gemm(A, B, out, -1.0, beta, s, groups, lower, max_ctas=max_ctas)
    ref, mag = np_oz_gemm(A, B, C, -1.0, beta, s, groups, lower)
    # one FMA per pair (kernel) against a product and a sum (restatement)
    tol = 2.0 ** -46 * (mag + (np.abs(C) if beta else 0.0))
    assert np.all(np.abs(out - ref) <= tol), f"max |diff| {np.max(np.abs(out - ref)):.3e}"
    # distance to the plain FP64 product: truncation of s digits, relative to |A| |B|^T
    exact = (C if beta else 0.0) - A @ B.T
    if lower:
        exact = np.where(np.tril(np.ones((M, N), dtype=bool)), exact, C)
    # A has row exponents, B block exponents (the maximum over each 128-row block of B)
    bmax = np.abs(B).max(axis=1)
    bblk = np.array([bmax[(j // 128) * 128:(j // 128 + 1) * 128].max() for j in range(N)])
    scale = np.abs(A).max(axis=1)[:, None] * bblk[None, :] * K
    G = groups or s
    # dropped groups (p + q >= G) and the last digit's truncation, per unit of K
    assert np.all(np.abs(out - exact) <= scale * (16 * (G + 2) * BASE ** -G + 2.0 ** -45) + 1e-300)


def test_gemm_rowsq(capi):
    rng = np.random.default_rng(5)
    M, N, K = 700, 128, 256
    A, B = graded(rng, M, K), graded(rng, N, K)
    C = np.zeros((M, N))
    rs = rng.standard_normal(M) ** 2
    rs0 = rs.copy()
    capi.test_oz_gemm(A, B, C, 1.0, 0.0, 6, rowsq=rs)
    ref, mag = np_oz_gemm(A, B, np.zeros((M, N)), 1.0, 0.0, 6)
    assert np.all(np.abs(C - ref) <= 2.0 ** -46 * mag)
    np.testing.assert_allclose(rs, rs0 + np.sum(ref * ref, axis=1), rtol=1e-14)


def test_gemm_nan_propagates(capi):
    rng = np.random.default_rng(6)
    A, B = rng.standard_normal((256, 256)), rng.standard_normal((128, 256))
    A[3, 200] = np.nan
    C = np.zeros((256, 128))
    capi.test_oz_gemm(A, B, C, 1.0, 0.0, 5)
    assert np.all(np.isnan(C[3]))
    assert np.all(np.isfinite(np.delete(C, 3, axis=0)))


def test_gemm_rejects_bad_shapes(capi):
    A = np.zeros((128, 100))
    B = np.zeros((128, 100))
    C = np.zeros((128, 128))
    with pytest.raises(capi.GpratCudaError):
        capi.test_oz_gemm(A, B, C, 1.0, 0.0, 6)  # K not a multiple of 128
    with pytest.raises(capi.GpratCudaError):
        capi.test_oz_gemm(np.zeros((128, 128)), np.zeros((128, 128)), C, 1.0, 0.0, 9)  # too many digits
