"""The step's orientation index of a nucleated grain id, id % num_theta + 1
(APTPhaseField.cu:259-273), is formed without a divide instruction:
div_invariant / invariant_divisor in cupf_b200/csrc/apt_common.cuh restate
Granlund and Montgomery's division by an invariant integer (PLDI 1994, fig.
4.1).  The same arithmetic in Python (64-bit products, 32-bit words) against
Python's integer division over every divisor up to 5000, assorted large ones,
and dividends at the edges and at random; on the GPU, the melt-pool tests step
nucleated ids past num_theta bit for bit against the oracle."""
import numpy as np

M32 = (1 << 32) - 1


def invariant_divisor(d):
    l = 0
    while (1 << l) < d:
        l += 1
    m = (((1 << 32) * ((1 << l) - d)) // d + 1) & M32
    return m, min(l, 1), max(l - 1, 0)


def div_invariant(n, m, s1, s2):
    t = (m * n) >> 32
    return ((t + ((n - t) >> s1)) & M32) >> s2


def test_matches_integer_division():
    rng = np.random.default_rng(0)
    divisors = list(range(1, 5001)) + [2 ** k for k in range(13, 31)] + \
        [2 ** k - 1 for k in range(13, 31)] + [2 ** k + 1 for k in range(13, 31)] + \
        [int(x) for x in rng.integers(5001, 2 ** 31 - 1, 300)]
    for d in divisors:
        m, s1, s2 = invariant_divisor(d)
        assert 0 <= m <= M32
        ns = [0, 1, d - 1, d, d + 1, 2 * d - 1, 2 * d, 2 ** 31 - 1, 2 ** 32 - 1] + \
            [int(x) for x in rng.integers(0, 2 ** 31, 40)]
        for n in ns:
            if n > M32:
                continue
            assert div_invariant(n, m, s1, s2) == n // d, (n, d)


def test_orientation_index_wrap():
    for ng in (1, 3, 20, 150, 600, 4095, 32767):
        m, s1, s2 = invariant_divisor(ng)
        for i in list(range(ng + 1, ng + 50)) + [5 * ng + 3, 32767, 2 ** 30]:
            assert i - div_invariant(i, m, s1, s2) * ng + 1 == i % ng + 1
