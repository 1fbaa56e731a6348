"""The single-precision filter's error bound, checked on the CPU.

oracle/fp32_filter.py restates the device's estimates in numpy float32 (the
device's operation order, no fused multiply-add) and its bound in float64,
and the reference's double quality and metric edge length in their
operation order. Over 10^7 seeded tets and 10^7 seeded edges of the shapes
that stress a bound (slivers, needles, caps, scales 1e-6..1e6, far from the
origin, edge ratios to 1e4, quality near the 0.3 floor, inverted, within a
few ulps of a threshold), every estimate that carries a bound is within it
of the double value, and every side the edge test decides is the double
comparison's side. The GPU tests check that the device produces the same
estimates bit for bit and a bound at least this large."""
import numpy as np
import pytest

from oracle import fp32_filter as F
from oracle import oracle as O

# the bound holds against the float64 evaluation with this much to spare;
# the device rounds every step of it upward
SLACK = 1.0 - 2.0 ** -40


def test_double_restatement_is_the_oracle_quality():
    coords, conn, _ = O.box(6, 3, 0.3)
    m = O.Oracle(3, coords, conn)
    x = coords.reshape(-1, 3)[conn.reshape(-1, 4)]
    assert np.array_equal(m.qualities(), F.tet_quality64(x))


def test_double_restatement_is_the_oracle_edge_length():
    coords, conn, _ = O.box(5, 2, 0.3)
    m = O.Oracle(3, coords, conn)
    h = np.random.default_rng(0).uniform(0.05, 0.3, size=coords.size // 3)
    m.add_field(0, "adapt_size", h)
    ev = m.down(1, 0).reshape(-1, 2)
    x = coords.reshape(-1, 3)
    got = F.edge_ratio64(x[ev[:, 0]], x[ev[:, 1]], h[ev[:, 0]], h[ev[:, 1]])
    assert np.array_equal(m.edge_lengths(), got)


@pytest.mark.parametrize("chunk", range(10))
def test_quality_bound_holds(chunk):
    x = F.stress_tets(10 ** 6, 1000 + chunk)
    est, bound = F.tet_quality32(x)
    q64 = F.tet_quality64(x)
    fin = np.isfinite(bound)
    assert fin.mean() > 0.99   # nearly every shape gets a usable bound
    err = np.abs(est.astype(np.float64) - q64)
    over = fin & ~(err <= bound * SLACK)
    assert not over.any(), x[over][:3]
    # and the bound is not vacuous: within 10x of the worst observed error
    assert (err[fin] / bound[fin]).max() > 0.1


@pytest.mark.parametrize("thr", [1.0, 1.0 / 3.0, 0.3])
def test_edge_side_matches_double(thr):
    for chunk in range(3):
        xa, xb, ha, hb = F.stress_edges(10 ** 6, 2000 + chunk, thr)
        side = F.edge_ratio_side32(xa, xb, ha, hb, thr)
        r64 = F.edge_ratio64(xa, xb, ha, hb)
        assert (side != 0).mean() > 0.9
        assert not ((side > 0) & ~(r64 > thr)).any()
        assert not ((side < 0) & ~(r64 < thr)).any()


def test_a_planted_overly_tight_bound_is_caught():
    """The check itself can fail: a bound scaled down 100x is exceeded."""
    x = F.stress_tets(10 ** 5, 7)
    est, bound = F.tet_quality32(x)
    q64 = F.tet_quality64(x)
    fin = np.isfinite(bound)
    err = np.abs(est.astype(np.float64) - q64)
    assert (fin & ~(err <= bound * 0.01)).any()
