"""The single-precision filter with double recheck: the same meshes as the
double path (identical digests, so identical decisions), candidates
actually decided on the estimate, and, with the audit switch on, every
decision taken on an estimate taken again in double with no difference and
every estimate within its bound. The device's estimates are the CPU
restatement's bit for bit (oracle/fp32_filter.py, where the bound is
checked over 10^7 stress shapes), and its bounds at least as large."""
import numpy as np
import pytest

from conftest import build_gpu

pytestmark = pytest.mark.gpu

ARGS = (1 / 3., 0.3, 4, 50)


@pytest.fixture(autouse=True)
def audit_on():
    import omega_h_v1_b200 as G
    G.set_fp32_audit(True)
    G.fp32_stats(reset=True)
    yield
    G.set_fp32_audit(False)


def _audit_clean():
    import omega_h_v1_b200 as G
    au = G.fp32_audit_stats()
    st = G.fp32_stats(reset=True)
    assert au["flips"] == 0, au
    assert st["bound_exceeded"] == 0, st
    return st, au


def test_device_estimates_are_the_restatement():
    import omega_h_v1_b200 as G
    from oracle import fp32_filter as F
    x = F.stress_tets(10 ** 6, 11)
    est, err, q64 = G.fp32_probe_tets(x)
    e_np, b_np = F.tet_quality32(x)
    assert np.array_equal(est.view(np.uint32), e_np.view(np.uint32))
    assert np.array_equal(q64, F.tet_quality64(x))
    fin = np.isfinite(err)
    assert fin.mean() > 0.99
    # the device rounds its bound upward: never below the float64 evaluation
    assert (err[fin].astype(np.float64) >= b_np[fin] * (1 - 2.0 ** -40)).all()
    assert (np.abs(est[fin].astype(np.float64) - q64[fin]) <= err[fin]).all()


@pytest.mark.parametrize("thr", [1.0, 1.0 / 3.0])
def test_device_edge_sides_are_the_restatement(thr):
    import omega_h_v1_b200 as G
    from oracle import fp32_filter as F
    xa, xb, ha, hb = F.stress_edges(10 ** 6, 12, thr)
    side, r64 = G.fp32_probe_edges(np.stack([xa, xb], 1), np.stack([ha, hb], 1), thr)
    assert np.array_equal(side, F.edge_ratio_side32(xa, xb, ha, hb, thr))
    assert np.array_equal(r64, F.edge_ratio64(xa, xb, ha, hb))
    assert not ((side > 0) & ~(r64 > thr)).any()
    assert not ((side < 0) & ~(r64 < thr)).any()


def _pair(n, **kw):
    a = build_gpu(n, **kw)
    b = a.clone()
    b.set_fp32_filter(True)
    return a, b


@pytest.mark.parametrize("n,kw", [
    (12, dict(seed=4, pert=0.2, size=1 / 12., fields=True)),
    (12, dict(seed=4, pert=0.25, size=1 / 8., parallel=True)),
    (16, dict(seed=0, radial=(0.02, 0.2))),
])
def test_filter_gives_the_same_mesh(n, kw):
    import omega_h_v1_b200 as G
    G.fp32_stats(reset=True)
    a, b = _pair(n, **kw)
    assert a.adapt(*ARGS) == b.adapt(*ARGS)
    assert a.digest() == b.digest()
    st, au = _audit_clean()
    assert st["decided"] > 0 and st["rechecked"] > 0
    assert au["audited"] >= st["decided"] and au["checked"] > 0
    assert st["max_error"] < 1e-4


def test_filter_swap_and_coarsen_slivers():
    import omega_h_v1_b200 as G
    G.fp32_stats(reset=True)
    a, b = _pair(8, seed=1, pert=0.28, size=1 / 8., fields=True)
    assert a.swap_slivers(0.3, 4) == b.swap_slivers(0.3, 4)
    assert a.coarsen_slivers(0.3, 4) == b.coarsen_slivers(0.3, 4)
    assert a.digest() == b.digest()
    st, au = _audit_clean()
    assert au["audited"] >= st["decided"]


def test_filter_in_a_batch():
    import omega_h_v1_b200 as G
    from omega_h_v1_b200 import workloads as W
    jobs = W.batched_boxes(10, seed=3, nmax=9)
    plain = [W.build_job_mesh(G, j) for j in jobs]
    filt = [m.clone() for m in plain]
    for m in filt:
        m.set_fp32_filter(True)
    G.adapt_batch(plain, *ARGS)
    G.adapt_batch(filt, *ARGS)
    for x, y in zip(plain, filt):
        assert x.digest() == y.digest()
    _audit_clean()


def test_filter_in_the_front_warp_flow():
    """Graded Hessian sizes and warped (poorly shaped) elements: the cases
    where most qualities are computed only in single precision."""
    import omega_h_v1_b200 as G
    from conftest import front_warp_run
    a = build_gpu(10, size=0.1)
    b = a.clone()
    b.set_fp32_filter(True)
    G.fp32_stats(reset=True)
    assert front_warp_run(a, angle=0.4) == front_warp_run(b, angle=0.4)
    assert a.digest() == b.digest()
    st, au = _audit_clean()
    assert st["decided"] > 0 and au["audited"] >= st["decided"]
