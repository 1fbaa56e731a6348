"""osh_b200_adapt_batch: many meshes adapted together as disjoint unions,
one launch per stage for all of them. Each mesh must come out exactly as
osh_adapt leaves it alone (connectivity, classification, global numbers and
tags bit-identical; f64 fields within 1e-12 relative), with the same return
value, the same pass count and the same E_MAXOPS outcome, however the
meshes are grouped into unions."""
import math

import numpy as np
import pytest

from conftest import build_cpu, build_gpu

pytestmark = pytest.mark.gpu

REL = 1e-12
ARGS = (1 / 3., 0.3, 4, 50)


def _oracle():
    from oracle import oracle as O
    return O


def _cases(count, seed, nmin=3, nmax=10):
    """Boxes with n log-uniform in [nmin, nmax] and a uniform size h drawn in
    [0.3/n, 1.5/n], the batched workload's distribution at test sizes."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        h = rng.uniform(0.3 / n, 1.5 / n)
        out.append(dict(n=n, seed=i, pert=0.1, size=h))
    return out


def _alone(kw, **extra):
    import omega_h_v1_b200 as G
    m = build_gpu(kw["n"], seed=kw["seed"], pert=kw["pert"], size=kw["size"], **extra)
    try:
        r = m.adapt(*ARGS)
        st = 0
    except G.OshError as e:
        r, st = 0, e.code
        G.lib().osh_b200_clear_error()
    import ctypes as C
    p, e = C.c_uint(), C.c_double()
    G.lib().osh_b200_adapt_stats(C.byref(p), C.byref(e))
    return m, r, st, p.value


def _check_batch(cases, max_union_elems, **extra):
    import omega_h_v1_b200 as G
    O = _oracle()
    alone = [_alone(kw, **extra) for kw in cases]
    batch = [build_gpu(kw["n"], seed=kw["seed"], pert=kw["pert"], size=kw["size"], **extra)
             for kw in cases]
    changed, status, stats = G.adapt_batch(batch, *ARGS, max_union_elems=max_union_elems)
    for i, (m, r, st, passes) in enumerate(alone):
        assert status[i] == st, "mesh %d status" % i
        if st == 0:
            assert changed[i] == r, "mesh %d return value" % i
            assert stats["per_mesh"][i][0] == passes, "mesh %d passes" % i
        errs = O.mesh_diff(batch[i].snapshot(), m.snapshot(), rel_tol=REL)
        assert not errs, "mesh %d (%s): %s" % (i, cases[i], errs[:5])
        assert batch[i].digest() == m.digest(), "mesh %d digest" % i
    return stats


def test_batch_equals_each_mesh_alone():
    """Whatever the union size limit (one union per pass, or many small
    ones), every mesh ends as it would alone."""
    cases = _cases(14, seed=1)
    one = _check_batch(cases, 0)
    many = _check_batch(cases, 4000)
    assert one["mesh_passes"] == many["mesh_passes"] > 0
    assert many["union_passes"] > one["union_passes"] > 0


def test_batch_with_fields_parallel_and_a_pass_cap_failure():
    """Fields of every transfer kind, global numbers, and one mesh that needs
    more than max_passes (E_MAXOPS for it alone, the others unaffected)."""
    cases = [dict(n=12, seed=4, pert=0.25, size=1 / 12.),
             dict(n=6, seed=0, pert=0.3, size=1 / 6.),
             dict(n=12, seed=4, pert=0.2, size=1 / 12.),
             dict(n=5, seed=2, pert=0.1, size=0.08)]
    _check_batch(cases, 0, fields=True, parallel=True)


def test_batch_against_oracle():
    """Two meshes of one union straight against the oracle's mesh_adapt."""
    import omega_h_v1_b200 as G
    O = _oracle()
    cases = [dict(n=4, seed=0, pert=0.1, size=0.09), dict(n=6, seed=3, pert=0.1, size=0.3)]
    batch = [build_gpu(kw["n"], seed=kw["seed"], pert=kw["pert"], size=kw["size"])
             for kw in cases]
    changed, status, _ = G.adapt_batch(batch, *ARGS)
    for i, kw in enumerate(cases):
        o = build_cpu(O.Oracle, kw["n"], seed=kw["seed"], pert=kw["pert"], size=kw["size"])
        assert changed[i] == o.adapt(*ARGS)
        assert status[i] == 0
        errs = O.mesh_diff(batch[i].snapshot(), o.snapshot(), rel_tol=REL)
        assert not errs, "mesh %d: %s" % (i, errs[:5])


def test_batch_rejects_mixed_tags():
    import omega_h_v1_b200 as G
    a = build_gpu(3, size=0.2)
    b = build_gpu(3, size=0.2, fields=True)
    with pytest.raises(G.OshError) as e:
        G.adapt_batch([a, b], *ARGS)
    assert e.value.code == 4
    G.lib().osh_b200_clear_error()


def test_batch_rejects_vertex_labels_refinement_would_drop():
    import omega_h_v1_b200 as G
    a = build_gpu(3, size=0.2)
    a.add_tag(0, "flag", np.zeros(a.count(0), dtype=np.uint32), type_=G.T_U32)
    with pytest.raises(G.OshError) as e:
        G.adapt_batch([a], *ARGS)
    assert e.value.code == 4
    G.lib().osh_b200_clear_error()


def test_digest_tracks_content():
    a = build_gpu(4, size=0.2, fields=True)
    b = a.clone()
    assert a.digest() == b.digest()
    b.refine_by_size(0.0)
    assert a.digest() != b.digest()
    c = build_gpu(4, size=0.2, fields=True, seed=1)
    assert a.digest() != c.digest()
