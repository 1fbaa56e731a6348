"""Parity of the CUDA adaptation pass with the oracle (our C restatement,
itself pinned to the reference): stage-by-stage selections and whole passes
must be bit-identical in connectivity, classification, global numbers and
selected sets; f64 fields within 1e-12 relative (mesh_diff)."""
import numpy as np
import pytest

from conftest import build_cpu, build_gpu

pytestmark = pytest.mark.gpu

REL = 1e-12


def _oracle():
    from oracle import oracle as O
    return O


def _same(a, b, what):
    O = _oracle()
    errs = O.mesh_diff(a.snapshot(), b.snapshot(), rel_tol=REL)
    assert not errs, "%s: %s" % (what, errs[:5])


@pytest.mark.parametrize("n", [2, 3, 8])
def test_input_and_adjacency(n):
    O = _oracle()
    g = build_gpu(n)
    o = build_cpu(O.Oracle, n)
    _same(g, o, "input")
    for lo, hi in [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]:
        for x, y in zip(g.up(lo, hi), o.up(lo, hi)):
            assert np.array_equal(x, y), "up(%d,%d)" % (lo, hi)
    for hi, lo in [(2, 1), (3, 1), (3, 2)]:
        assert np.array_equal(g.down(hi, lo), o.down(hi, lo)), "down(%d,%d)" % (hi, lo)
    for lo, hi in [(0, 1), (1, 2), (1, 3), (0, 3)]:
        for x, y in zip(g.star(lo, hi), o.star(lo, hi)):
            assert np.array_equal(x, y), "star(%d,%d)" % (lo, hi)
    assert np.array_equal(g.dual(), o.dual())
    assert np.array_equal(g.qualities(), o.qualities())
    assert g.min_quality() == o.min_quality()
    assert np.array_equal(g.edge_lengths(), o.edge_lengths())


def test_config1_passes():
    """3072 tets, h = 0.05: refine, coarsen and swap with floor 0.3."""
    O = _oracle()
    g, o = build_gpu(8), build_cpu(O.Oracle, 8)
    qf = min(0.3, o.min_quality())
    sg, so = g.refine_sets(qf), o.refine_sets(qf)
    for k in so:
        assert np.array_equal(sg[k], so[k]), "refine set " + k
    assert g.refine_by_size(qf) == o.refine_by_size(qf) == 1
    _same(g, o, "refine")
    cg, co = g.coarsen_sets(qf, 1 / 3.), o.coarsen_sets(qf, 1 / 3.)
    for k in co:
        assert np.array_equal(cg[k], co[k]), "coarsen set " + k
    assert g.coarsen_by_size(qf, 1 / 3.) == o.coarsen_by_size(qf, 1 / 3.)
    _same(g, o, "coarsen")
    wg, wo = g.swap_sets(0.3, 4), o.swap_sets(0.3, 4)
    for k in wo:
        assert np.array_equal(wg[k], wo[k]), "swap set " + k
    assert g.swap_slivers(0.3, 4) == o.swap_slivers(0.3, 4)
    _same(g, o, "swap")


@pytest.mark.parametrize("n,seed,pert", [(6, 0, 0.3), (8, 1, 0.28), (12, 3, 0.27)])
def test_swap_and_coarsen_slivers(n, seed, pert):
    O = _oracle()
    kw = dict(seed=seed, pert=pert, size=1.0 / n, fields=True)
    g, o = build_gpu(n, **kw), build_cpu(O.Oracle, n, **kw)
    wg, wo = g.swap_sets(0.3, 4), o.swap_sets(0.3, 4)
    for k in wo:
        assert np.array_equal(wg[k], wo[k]), "swap set " + k
    assert g.swap_slivers(0.3, 4) == o.swap_slivers(0.3, 4)
    _same(g, o, "swap")
    assert g.coarsen_slivers(0.3, 4) == o.coarsen_slivers(0.3, 4)
    _same(g, o, "coarsen slivers")


@pytest.mark.parametrize("n,seed,h", [(8, 5, 0.4), (10, 6, 0.3)])
def test_coarsen_by_size(n, seed, h):
    O = _oracle()
    kw = dict(seed=seed, size=h, fields=True)
    g, o = build_gpu(n, **kw), build_cpu(O.Oracle, n, **kw)
    qf = min(0.3, o.min_quality())
    cg, co = g.coarsen_sets(qf, 1 / 3.), o.coarsen_sets(qf, 1 / 3.)
    for k in co:
        assert np.array_equal(cg[k], co[k]), "coarsen set " + k
    assert g.coarsen_by_size(qf, 1 / 3.) == o.coarsen_by_size(qf, 1 / 3.)
    _same(g, o, "coarsen")


@pytest.mark.parametrize("parallel", [False, True])
@pytest.mark.parametrize("pert,size", [(0.2, 1 / 12.), (0.25, 1 / 8.)])
def test_adapt_loop_small(parallel, pert, size):
    """Full mesh_adapt on a sliver-prone box with fields: refines, coarsens,
    swaps and collapses slivers before it converges."""
    O = _oracle()
    kw = dict(seed=4, pert=pert, size=size, fields=True, parallel=parallel)
    g, o = build_gpu(12, **kw), build_cpu(O.Oracle, 12, **kw)
    assert g.adapt(1 / 3., 0.3, 4, 50) == o.adapt(1 / 3., 0.3, 4, 50)
    assert o.L.lib.or_error(o.h) == 0
    _same(g, o, "adapt")


def test_max_passes_reported():
    """A mesh that needs more than max_passes: the reference aborts
    (adapt.cpp:36-45); this build raises E_MAXOPS after the same passes."""
    import omega_h_v1_b200 as G
    O = _oracle()
    kw = dict(seed=4, pert=0.25, size=1 / 12., fields=True)
    g, o = build_gpu(12, **kw), build_cpu(O.Oracle, 12, **kw)
    o.adapt(1 / 3., 0.3, 4, 50)
    assert o.L.lib.or_error(o.h) == 2
    with pytest.raises(G.OshError) as e:
        g.adapt(1 / 3., 0.3, 4, 50)
    assert e.value.code == 3
    _same(g, o, "state at the pass cap")


def test_config2_full_adapt():
    """48^3 box (663,552 tets), h = 0.01 + 0.04 |x - c|, mesh_adapt(1/3, 0.3,
    4, 50) to convergence: the headline workload, compared whole."""
    O = _oracle()
    kw = dict(seed=0, radial=(0.01, 0.04))
    g, o = build_gpu(48, **kw), build_cpu(O.Oracle, 48, **kw)
    assert g.adapt(1 / 3., 0.3, 4, 50) == o.adapt(1 / 3., 0.3, 4, 50) == 1
    _same(g, o, "config 2 adapt")
