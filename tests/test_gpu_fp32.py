"""The single-precision filter with double recheck: the same meshes as the
double path (identical digests, so identical decisions), candidates
actually decided on the estimate, and an observed estimate error that never
exceeds the bound that licensed those decisions."""
import numpy as np
import pytest

from conftest import build_gpu

pytestmark = pytest.mark.gpu

ARGS = (1 / 3., 0.3, 4, 50)


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
    st = G.fp32_stats(reset=True)
    assert st["decided"] > 0 and st["rechecked"] > 0
    assert st["bound_exceeded"] == 0
    assert st["max_error"] < 1e-4


def test_filter_swap_and_coarsen_slivers():
    import omega_h_v1_b200 as G
    G.fp32_stats(reset=True)
    a, b = _pair(8, seed=1, pert=0.28, size=1 / 8., fields=True)
    assert a.swap_slivers(0.3, 4) == b.swap_slivers(0.3, 4)
    assert a.coarsen_slivers(0.3, 4) == b.coarsen_slivers(0.3, 4)
    assert a.digest() == b.digest()
    assert G.fp32_stats(reset=True)["bound_exceeded"] == 0


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
    st = G.fp32_stats(reset=True)
    assert st["bound_exceeded"] == 0 and st["decided"] > 0
