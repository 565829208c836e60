"""The bench's work model and parity summary on CPU (no GPU): the flop counts
follow the reference operation sequence the roofline divides, and the
parity summary applies the tests' bound."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402
from libnegf_b200 import generators as G  # noqa: E402


def test_c1_point_model():
    wl = bench.WORKLOADS["c1"]
    n3 = 256.0 ** 3
    f = bench.flops_per_point(wl, 47)
    expect = 47 * (176 / 3) * n3 + 2 * (32 / 3) * n3 + 2 * 16 * n3 + (80 / 3) * 100 * n3 + 40 * 99 * n3 + 32 * n3
    assert abs(f - expect) < 1e-6 * expect
    assert 150e9 < f < 170e9                               # about 159 GFLOP per c1 point
    assert bench.executed_flops_per_point(wl, 47) < f     # Gauss-Jordan 8 n^3 < zgetrf + zgetrs 32/3 n^3


def test_scba_point_model():
    wl = bench.WORKLOADS["c3"]
    n3 = 128.0 ** 3
    f0 = bench.scba_flops_per_point(wl, 50, 0)
    f10 = bench.scba_flops_per_point(wl, 50, 10)
    assert abs((f10 - f0) - 10 * (80 / 3 + 40 + 128) * 40 * n3) < 1e-6 * f10
    assert bench.scba_executed_flops_per_point(wl, 50, 10) < f10


def test_parity_summary_applies_the_test_bound():
    wl = dict(bench.WORKLOADS["c0"], nbl=4, n=6, dos=False)
    devs = [G.transport_c0(nbl=4, n=6, seed=0)]
    E = np.linspace(-2.5, 2.5, 8)
    ids = np.zeros(E.size, dtype=np.int32)
    from oracle import oracle as O
    Tc = O.transmission(devs[0], E, eta=wl["eta"])[0]
    same = bench.parity_summary(wl, devs, ids, E, Tc.copy(), Tc, cores=2)
    assert same["all_within_test_bound"] and same["within_1e-10_rel_or_1e-13_abs"] == E.size
    off = Tc.copy()
    off[3] += 1e-3                                        # far beyond rounding and the oracle's spread
    bad = bench.parity_summary(wl, devs, ids, E, off, Tc, cores=2)
    assert not bad["all_within_test_bound"] and bad["beyond_1e-10"] == 1


def test_clock_summary_keeps_the_timed_window():
    """The sampler runs from before the warm-up steps; its summary counts only
    the samples taken inside the timed region, so a throttle reason seen
    during warm-up alone does not mark the timed number."""
    clk = bench.ClockSampler(0)
    row = lambda mhz, cap: [str(mhz), "1965", "900", "0x0", "Not Active", "Not Active", "Not Active",
                            "Active" if cap else "Not Active"]
    clk.rows = [row(1500, True), row(1965, False), row(1965, False), row(1800, True)]
    clk.times = [1.0, 2.0, 3.0, 4.0]
    assert clk.summary()["samples"] == 4 and clk.summary()["reasons"] == ["sw_power_cap"]
    clk.window = (1.5, 3.5)
    s = clk.summary()
    assert s["samples"] == 2 and s["sm_mhz"] == 1965.0 and s["reasons"] == []
    clk.window = (10.0, 11.0)
    assert clk.summary()["reasons"] == ["unsampled"]
