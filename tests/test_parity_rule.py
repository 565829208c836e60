"""The parity rule of the GPU tests (conftest.assert_parity), checked on the
CPU with mistakes planted in synthetic results: a point whose FP64 rounding
samples stay within an eighth of the bound is held to the bound itself; a
listed point to ten times its samples, measured from the long-double
solution."""
import numpy as np
import pytest

from conftest import assert_parity


def _case(rng, P=6, M=40, scatter=None):
    x = rng.uniform(0.1, 1.0, (P, M))                # long-double solution
    s = np.full((P, M), 1e-13) if scatter is None else scatter
    ref = x + s * rng.choice([-1.0, 1.0], (P, M))    # the oracle: one FP64 rounding sample
    d = x - 0.5 * s                                  # two more restatements
    g = x + 0.25 * s
    return x, ref, d, g


def test_strict_points_are_held_to_the_bound():
    rng = np.random.default_rng(0)
    x, ref, d, g = _case(rng)
    got = ref.copy()
    got[2, 5] += 0.9e-10
    assert_parity(got, ref, 1e-10, ref_x=x, others=(d, g), rows=True)
    got[2, 5] += 0.2e-10
    with pytest.raises(AssertionError, match="beyond the strict bound"):
        assert_parity(got, ref, 1e-10, ref_x=x, others=(d, g), rows=True)


def test_listed_entries_are_held_to_ten_times_the_point_scatter():
    rng = np.random.default_rng(1)
    sc = np.full((6, 40), 1e-13)
    sc[3] = 2e-11                                    # above an eighth of the bound: listed
    sc[3, 7] = 1e-9                                  # the point's largest sample
    x, ref, d, g = _case(rng, scatter=sc)
    got = x.copy()
    got[3, 0] = x[3, 0] + 5e-9                       # within 10 x the point's scatter (1e-8)
    listed = assert_parity(got, ref, 1e-10, ref_x=x, others=(d, g), rows=True)
    assert listed.size == 40                         # every entry of point 3 is listed, no other
    # per entry, entry 0's own samples (2e-11) would not cover it
    with pytest.raises(AssertionError, match="listed points farther"):
        assert_parity(got, ref, 1e-10, ref_x=x, others=(d, g), rows=False)
    got[3, 0] = x[3, 0] + 2e-8                       # beyond 10 x the point's scatter
    with pytest.raises(AssertionError, match="listed points farther"):
        assert_parity(got, ref, 1e-10, ref_x=x, others=(d, g), rows=True)


def test_perturbation_spread_lists_a_point():
    rng = np.random.default_rng(2)
    x, ref, d, g = _case(rng, P=4, M=1)
    x, ref, d, g = x[:, 0], ref[:, 0], d[:, 0], g[:, 0]
    spread = np.array([0.0, 0.0, 5e-10, 0.0])
    got = ref.copy()
    got[2] = x[2] + 3e-9
    listed = assert_parity(got, ref, 1e-10, ref_x=x, others=(d, g), spread=spread)
    assert list(listed) == [2]
    got[1] += 2e-10
    with pytest.raises(AssertionError, match="beyond the strict bound"):
        assert_parity(got, ref, 1e-10, ref_x=x, others=(d, g), spread=spread)
