"""The numpy restatement of the device vector generator: Philox4x32-10
against the published known-answer vectors of its authors' Random123
distribution, and the recipe's structure (symmetric vectors, N(0,1) draws)."""
import numpy as np

from mshqc_b200 import synthetic as syn

# (counter words, key words) -> output words
KAT = [
    ((0x00000000, 0x00000000, 0x00000000, 0x00000000), (0x00000000, 0x00000000),
     (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff, 0xffffffff, 0xffffffff, 0xffffffff), (0xffffffff, 0xffffffff),
     (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
]


def test_philox_known_answers():
    for ctr, key, out in KAT:
        got = syn.philox4x32_10_words(*(np.array([c], dtype=np.uint32) for c in ctr), *key)
        assert tuple(int(g[0]) for g in got) == out


def test_counter_form_matches_words():
    ctr = np.array([0, 1, 2**40 + 7, 2**64 - 1], dtype=np.uint64)
    a = syn.philox4x32_10(ctr, 0x1234567890ABCDEF)
    b = syn.philox4x32_10_words(ctr & np.uint64(0xFFFFFFFF), ctr >> np.uint64(32), np.zeros(4), np.zeros(4),
                                0x90ABCDEF, 0x12345678)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_normals_and_vectors():
    zc, zs = syn.philox_normal_pair(np.arange(400000, dtype=np.uint64), 9)
    for z in (zc, zs):
        assert abs(z.mean()) < 0.01 and abs(z.var() - 1.0) < 0.01 and abs(np.mean(z ** 4) - 3.0) < 0.05
    assert abs(np.mean(zc * zs)) < 0.01          # the two members are uncorrelated
    L = syn.make_vectors_philox(9, 5, seed=3, sigma=0.5).reshape(5, 9, 9)
    assert np.array_equal(L, L.transpose(0, 2, 1))
    sq = syn.scale_factors(5)[2] * 0.5
    # diagonal element = sigma s_Q X_{mu mu} (cosine member)
    x = syn.philox_normal(np.array([(2 * 9 + 4) * 9 + 4], dtype=np.uint64), 3)[0]
    assert L[2, 4, 4] == sq * (0.5 * (x + x))
    # off-diagonal (mu < nu): both members of the block at counter (Q N + mu) N + nu
    c, s = syn.philox_normal_pair(np.array([(2 * 9 + 1) * 9 + 6], dtype=np.uint64), 3)
    assert L[2, 1, 6] == L[2, 6, 1] == sq * (0.5 * (c[0] + s[0]))
