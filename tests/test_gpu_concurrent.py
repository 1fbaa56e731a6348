"""osh_b200_adapt_concurrent: mesh_adapt of many meshes by several host
threads, each on a CUDA stream of its own. Each mesh runs the unchanged
single-mesh code, so it must end exactly as osh_adapt leaves it alone
(digest, return value, pass count, E_MAXOPS outcome), whatever the thread
count and memory budget, and must come back on the stream it had."""
import ctypes as C

import pytest

from conftest import build_gpu
from test_gpu_batch import ARGS, _alone, _cases

pytestmark = pytest.mark.gpu


def _check(cases, nthreads, budget=0, **extra):
    import omega_h_v1_b200 as G
    alone = [_alone(kw, **extra) for kw in cases]
    ms = [build_gpu(kw["n"], seed=kw["seed"], pert=kw["pert"], size=kw["size"], **extra)
          for kw in cases]
    changed, status, per = G.adapt_concurrent(ms, *ARGS, nthreads=nthreads,
                                              budget_bytes=budget)
    for i, (m, r, st, passes) in enumerate(alone):
        assert status[i] == st, "mesh %d status" % i
        if st == 0:
            assert changed[i] == r, "mesh %d return value" % i
            assert per[i][0] == passes, "mesh %d passes" % i
        assert ms[i].digest() == m.digest(), "mesh %d (%s) digest" % (i, cases[i])
    return ms


@pytest.mark.parametrize("nthreads", [1, 3, 8])
def test_concurrent_equals_each_mesh_alone(nthreads):
    _check(_cases(14, seed=5, nmin=3, nmax=14), nthreads)


def test_concurrent_with_fields_parallel_and_a_pass_cap_failure():
    cases = [dict(n=12, seed=4, pert=0.25, size=1 / 12.),
             dict(n=6, seed=0, pert=0.3, size=1 / 6.),
             dict(n=12, seed=4, pert=0.2, size=1 / 12.),
             dict(n=5, seed=2, pert=0.1, size=0.08)]
    _check(cases, 4, fields=True, parallel=True)


def test_concurrent_under_a_one_byte_budget_runs_one_at_a_time():
    _check(_cases(6, seed=6), 4, budget=1)


def test_concurrent_meshes_keep_their_streams():
    import torch
    import omega_h_v1_b200 as G
    s = torch.cuda.Stream()
    a = build_gpu(4, size=0.2)
    b = build_gpu(5, size=0.15)
    G.lib().osh_b200_set_stream(a.h, C.c_void_p(s.cuda_stream))
    G.lib().osh_b200_set_stream(b.h, C.c_void_p(0))
    ref_a, ref_b = a.clone(), b.clone()
    ref_a.adapt(*ARGS)
    ref_b.adapt(*ARGS)
    G.adapt_concurrent([a, b], *ARGS, nthreads=2)
    assert a.digest() == ref_a.digest() and b.digest() == ref_b.digest()
    # further work still runs (on the streams the meshes had)
    a.adapt(*ARGS)
    b.adapt(*ARGS)
    torch.cuda.synchronize()


def test_concurrent_rejects_a_mesh_twice():
    import omega_h_v1_b200 as G
    a = build_gpu(3, size=0.2)
    with pytest.raises(G.OshError) as e:
        G.adapt_concurrent([a, a], *ARGS)
    assert e.value.code == 4
    G.lib().osh_b200_clear_error()


@pytest.mark.parametrize("small", [25000, 200000])
def test_concurrent_with_small_meshes_grouped_into_unions(small):
    """Meshes estimated below small_mesh_elems run through the batched path
    inside the concurrent driver; each still ends as osh_adapt alone."""
    import omega_h_v1_b200 as G
    from omega_h_v1_b200 import tune
    L = tune._lib(G)
    before = tune.table(L)["small_mesh_elems"]
    assert L.osh_b200_tuning_set(b"small_mesh_elems", small) == 0
    try:
        _check(_cases(14, seed=7, nmin=3, nmax=14), 3)
        cases = [dict(n=12, seed=4, pert=0.25, size=1 / 12.),
                 dict(n=6, seed=0, pert=0.3, size=1 / 6.),
                 dict(n=5, seed=2, pert=0.1, size=0.08)]
        _check(cases, 2, fields=True, parallel=True)
    finally:
        L.osh_b200_tuning_set(b"small_mesh_elems", before)
