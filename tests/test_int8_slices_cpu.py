"""The int8-slice representation behind the mixed path's transforms
(mshqc_b200/csrc/ozaki_i8.cuh), restated in numpy: per-row power of two,
rounding to a 35-bit integer, five signed base-128 digits, the 15 digit
products with s + t < 5 and their weights, and the UMMA blocked byte layout
the slicing kernels write and the GEMM's bulk copies read.  Checks the error
bound stated there (below 2^-32 of 2^(e_x + e_y) per term) and that a tile
read through the layout formula sees each row's digits."""
import numpy as np

S, KB = 5, 32


def slices(X):
    """digits [S, R, K] (int) and row exponents e with |x| < 2^e."""
    mx = np.abs(X).max(axis=1)
    e = np.where(mx > 0, np.frexp(mx)[1], 0)
    m = np.rint(X * np.ldexp(1.0, 7 * S - e)[:, None]).astype(np.int64)
    m = np.clip(m, -(2 ** (7 * S) - 1), 2 ** (7 * S) - 1)
    am, sg = np.abs(m), np.sign(m)
    d = np.stack([sg * ((am >> (7 * (S - 1 - s))) & 127) for s in range(S)])
    return d, e


def product(dx, ex, dy, ey):
    """sum over s + t < S of 2^(ex+ey) 2^(-7(s+t+2)) dx_s . dy_t (exact ints, one scaling)."""
    T = np.zeros((dx.shape[1], dy.shape[1]), dtype=object)
    for s in range(S):
        for t in range(S - s):
            T = T + (dx[s].astype(object) @ dy[t].T.astype(object)) * (2 ** (7 * (S - 1 - s - t)))
    v = np.array([[float(T[i, j]) for j in range(T.shape[1])] for i in range(T.shape[0])])
    return v * np.ldexp(1.0, -7 * (S + 1)) * np.ldexp(1.0, ex)[:, None] * np.ldexp(1.0, ey)[None, :]


def test_digits_and_representation_error():
    rng = np.random.default_rng(3)
    X = rng.standard_normal((37, 50)) * np.exp(3 * rng.standard_normal((37, 1)))
    X[5] = 0.0
    d, e = slices(X)
    assert np.abs(d).max() <= 127
    back = sum(d[s] * np.ldexp(1.0, -7 * (s + 1)) for s in range(S)) * np.ldexp(1.0, e)[:, None]
    assert np.all(np.abs(back - X) <= np.ldexp(1.0, e - 7 * S - 1)[:, None])
    assert e[5] == 0 and not d[:, 5].any()


def test_per_term_error_bound():
    rng = np.random.default_rng(4)
    x = rng.uniform(-1, 1, (400, 1)) * np.exp(rng.standard_normal((400, 1)))
    y = rng.uniform(-1, 1, (300, 1)) * np.exp(rng.standard_normal((300, 1)))
    dx, ex = slices(x)
    dy, ey = slices(y)
    err = np.abs(product(dx, ex, dy, ey) - x @ y.T)
    bound = np.ldexp(1.0, ex[:, None] + ey[None, :] - 32)
    assert np.all(err <= bound)


def blocked_offset(r, k, Rp):
    return (k // 32) * Rp * KB + ((r // 8) * 2 + (k % 32) // 16) * 128 + (r % 8) * 16 + k % 16


def test_layout_tile_reads_rows():
    rng = np.random.default_rng(5)
    R, K, tile = 70, 45, 96
    Rp, Kp = -(-R // tile) * tile, -(-K // KB) * KB
    d, _ = slices(rng.standard_normal((R, K)))
    buf = np.zeros(S * Kp * Rp, dtype=np.int64)
    for s in range(S):
        for r in range(R):
            for k in range(K):
                buf[s * Kp * Rp + blocked_offset(r, k, Rp)] = d[s, r, k]
    # one 32-wide K chunk of the tile starting at row 0 is a contiguous slab
    # of Rp rows x 32 bytes in core matrices of 8 rows x 16 bytes
    for s in range(S):
        for kc in range(Kp // KB):
            slab = buf[s * Kp * Rp + kc * Rp * KB: s * Kp * Rp + (kc + 1) * Rp * KB]
            for r in range(0, R, 7):
                got = [slab[((r // 8) * 2 + kk // 16) * 128 + (r % 8) * 16 + kk % 16] for kk in range(KB)]
                want = [d[s, r, kc * KB + kk] if kc * KB + kk < K else 0 for kk in range(KB)]
                assert got == want
