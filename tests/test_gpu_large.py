"""Full-size parity against the reference itself: digests recorded from the
reference's OpenMP build (tests/golden/make_large_digests.py) for

* every box with n <= 16 of the seeded 512-box set and its three largest
  boxes, each adapted by mesh_adapt(1/3, 0.3, 4, 50): here adapted together
  by the batched path with the single-precision filter, and the largest
  ones also by the concurrent path;
* the 96^3 anisotropic front workload after its first mesh_adapt and after
  its first warp step.

Every mesh must be the reference's bit for bit (counts, connectivity, every
tag, global numbers)."""
import json
import os

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
DIGESTS = os.path.join(ROOT, "tests", "golden", "large_digests.json")


def _want():
    with open(DIGESTS) as f:
        return json.load(f)


def _flows():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import large_flows
    return large_flows


def _make(dim, coords, conn):
    import omega_h_v1_b200 as G
    return G.Mesh.reduced(dim, coords, conn)


def test_box_set_subset_batched_filtered_matches_reference():
    import omega_h_v1_b200 as G
    from oracle import oracle as O
    F = _flows()
    want = _want()["batched_subset"]["jobs"]
    jobs = F.batched_subset()
    assert len(jobs) == len(want)
    G.pool_reserve(8 << 30)
    # calls of a bounded estimated output, as bench.py cuts the whole set
    chunks, cur, est = [], [], 0.0
    for j in jobs:
        if cur and est + j.estimated_output_tets() > 30e6:
            chunks.append(cur)
            cur, est = [], 0.0
        cur.append(j)
        est += j.estimated_output_tets()
    chunks.append(cur)
    for chunk in chunks:
        ms = [F.box_job_mesh(_make, G.box, j) for j in chunk]
        for m in ms:
            m.set_fp32_filter(True)
        G.adapt_batch(ms, *F.BOX_ADAPT, max_union_elems=1000000)
        for j, m in zip(chunk, ms):
            s = m.snapshot()
            w = want[str(j.index)]
            assert s.counts == w["counts"], j.index
            assert O.snapshot_digest(s) == w["sha256"], j.index
            m.close()


def test_largest_boxes_concurrent_match_reference():
    import omega_h_v1_b200 as G
    from oracle import oracle as O
    F = _flows()
    want = _want()["batched_subset"]["jobs"]
    jobs = F.batched_subset()[-3:]
    ms = [F.box_job_mesh(_make, G.box, j) for j in jobs]
    G.adapt_concurrent(ms, *F.BOX_ADAPT, nthreads=3)
    for j, m in zip(jobs, ms):
        s = m.snapshot()
        assert O.snapshot_digest(s) == want[str(j.index)]["sha256"], j.index
        m.close()


def test_front_workload_matches_reference():
    import omega_h_v1_b200 as G
    from oracle import oracle as O
    F = _flows()
    want = _want()
    G.pool_reserve(16 << 30)
    m = F.front_mesh(_make, G.box)
    m.adapt(*F.FRONT_ADAPT)
    s = m.snapshot()
    assert s.counts == want["front_first_adapt"]["counts"]
    assert O.snapshot_digest(s) == want["front_first_adapt"]["sha256"]
    del s
    tries = F.front_warp_step(m)
    assert tries == want["front_warp_step1"]["tries"]
    s = m.snapshot()
    assert s.counts == want["front_warp_step1"]["counts"]
    assert O.snapshot_digest(s) == want["front_warp_step1"]["sha256"]
    m.close()
