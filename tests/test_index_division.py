"""The x kernels' multiply-high division (fdiv in csrc/bld_kernels.cuh).

The kernels split flat task indices with divisors known only at run time (the
number of modes per row K1, the row length P1): n / d = floor(n * m / 2^32) with
m = ceil(2^32 / d) (and n itself for d = 1).  For n = q d + r < 2^16 and
d < 2^16 the product exceeds n / d by less than 2^-16 <= 1 / d, so the floor is
q.  This checks that claim exhaustively over every index the kernels form
(n < 2^16) for every divisor up to 1200 (K1 <= 513 and P1 <= 1024 here), with
the same 32-bit arithmetic as the device code.
"""

import numpy as np


def fdiv_magic(d):
    return 0 if d <= 1 else ((1 << 32) + d - 1) // d


def test_multiply_high_division_is_exact():
    n = np.arange(1 << 16, dtype=np.uint64)
    for d in range(1, 1201):
        m = fdiv_magic(d)
        got = n if m == 0 else (n * np.uint64(m)) >> np.uint64(32)
        assert m < (1 << 32)
        assert np.array_equal(got, n // np.uint64(d)), d
