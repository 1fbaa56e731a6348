"""The serving loop (osh_b200_server_*): jobs submitted while others run
join the running batch at the next step and leave it when their own pass
loop ends. Each job's result must be the same alone and in the mix: equal to
osh_adapt of the same input (bit-identical connectivity, classification and
tags; f64 fields within 1e-12 relative, here identical digests), whatever
else shares its steps, and whatever the memory budget admits."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ARGS = (1 / 3., 0.3, 4, 50)
REL = 1e-12


def _jobs():
    import omega_h_v1_b200 as G
    from omega_h_v1_b200 import workloads as W
    jobs = [W.BoxJob(0, 4, 0.2, 0), W.BoxJob(1, 6, 0.12, 1),
            W.BoxJob(2, 5, 0.0, 2, (0.05, 0.2, 0.4, 0.5, 0.6)),
            W.BoxJob(3, 3, 0.09, 3), W.BoxJob(4, 7, 0.3, 4),
            W.BoxJob(5, 6, 0.0, 5, (0.08, 0.3, 0.6, 0.4, 0.5)),
            # the front's Hessian size field, computed on the GPU
            W.BoxJob(6, 8, 0.0, 6, None, 0.0, (0.45, (2 / 8 - 0.5 / 8) / 2000, 0.5 / 8, 2 / 8))]
    return [(j,) + W.job_host_input(G, j) for j in jobs]


def _alone(coords, conn, h):
    import omega_h_v1_b200 as G
    m = G.Mesh.reduced(3, coords, conn)
    m.derive_model_full()
    m.add_field(0, "adapt_size", h, transfer=G.X_POINTWISE)
    r = m.adapt(*ARGS)
    return m, r


def _serve(inputs, budget, schedule):
    """Submit inputs in groups (schedule = list of group sizes), stepping the
    server once between groups, then step to the end."""
    import omega_h_v1_b200 as G
    sv = G.Server(*ARGS, budget)
    ids, i, max_active = [], 0, 0
    for g in schedule:
        for _ in range(g):
            _, coords, conn, h = inputs[i]
            ids.append(sv.submit(coords, conn, h))
            i += 1
        sv.step()
        max_active = max(max_active, sv.stats()["active"])
    while sv.step() > 0:
        max_active = max(max_active, sv.stats()["active"])
    done = sv.poll()
    assert sorted(done) == sorted(ids)
    out = {j: sv.take(j) for j in ids}
    info = {j: sv.job_info(j) for j in ids}
    return sv, out, info, max_active


def test_results_equal_alone_and_in_the_mix():
    from oracle import oracle as O
    inputs = _jobs()
    alone = [_alone(c, k, h) for _, c, k, h in inputs]
    sv, out, info, max_active = _serve(inputs, 1 << 40, [2, 1, 4])
    assert max_active >= 3, "jobs should overlap on the device"
    for i, (m, r) in enumerate(alone):
        g = out[i]
        assert info[i]["status"] == 0
        errs = O.mesh_diff(g.snapshot(), m.snapshot(), rel_tol=REL)
        assert not errs, "job %d: %s" % (i, errs[:5])
        assert g.digest() == m.digest(), "job %d digest" % i
    # each job alone in its own server gives the same result
    for i in (1, 2, 6):
        _, out1, _, _ = _serve([inputs[i]], 1 << 40, [1])
        assert out1[0].digest() == out[i].digest()
    sv.close()


def test_memory_budget_admits_one_job_at_a_time():
    inputs = _jobs()[:3]
    sv, out, info, max_active = _serve(inputs, 1, [3])
    assert max_active == 1
    for i, (_, c, k, h) in enumerate(inputs):
        m, _ = _alone(c, k, h)
        assert out[i].digest() == m.digest()
        assert info[i]["t_admit"] >= info[i]["t_submit"]
        assert info[i]["t_done"] >= info[i]["t_admit"]
    # admitted in submission order, one after another
    assert info[1]["t_admit"] >= info[0]["t_done"]
    sv.close()


def test_engine_thread_results_equal_alone():
    """The server's own engine thread runs the steps while jobs are still
    being submitted from this thread; every result equals osh_adapt alone."""
    import time
    import omega_h_v1_b200 as G
    inputs = _jobs()
    sv = G.Server(*ARGS, 1 << 40)
    sv.start()
    ids = []
    for k, (_, coords, conn, h) in enumerate(inputs):
        ids.append(sv.submit(coords, conn, h))
        time.sleep(0.002 * k)
    assert sv.wait(120.0) == 0
    for i, (_, c, k, h) in enumerate(inputs):
        m, _ = _alone(c, k, h)
        assert sv.take(ids[i]).digest() == m.digest(), "job %d" % i
    sv.stop()
    sv.close()
