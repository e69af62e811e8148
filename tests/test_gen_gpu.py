"""The device workload generators produce the oracle's keys bit for bit."""
import numpy as np
import pytest

import oracle
from tests.conftest import from_np_u, to_np_u

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kb", [4, 8])
def test_gen_uniform_matches_oracle(hg, kb):
    for n, seed in ((0, 1), (1, 2), (100_003, 3), (1 << 20, 1)):
        got = to_np_u(hg.gen_uniform(n, kb, seed), kb)
        np.testing.assert_array_equal(got, oracle.gen_uniform(n, kb, seed))


@pytest.mark.parametrize("kb", [4, 8])
def test_gen_overlap_matches_oracle(hg, kb):
    a = oracle.gen_uniform(70_000, kb, 5)
    for n, frac, seed in ((1 << 16, 0.5, 2), (99_999, 0.25, 7), (5000, 1.0, 3), (80_000, 0.1, 4)):
        got = to_np_u(hg.gen_overlap(n, from_np_u(a), frac, seed), kb)
        np.testing.assert_array_equal(got, oracle.gen_overlap(n, a, frac, seed))


def test_gen_zipf_matches_oracle(hg):
    cdf_np = oracle.zipf_cdf(1 << 16, 1.1)
    cdf = hg.zipf_cdf(1 << 16, 1.1)
    np.testing.assert_array_equal(to_np_u(cdf, 8), cdf_np)
    for kb in (4, 8):
        got = to_np_u(hg.gen_zipf(200_000, kb, cdf, 5), kb)
        np.testing.assert_array_equal(got, oracle.gen_zipf(200_000, kb, cdf_np, 5))
