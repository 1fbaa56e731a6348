"""The CUDA path pinned directly to outputs of the reference itself (golden
fixtures and digests in tests/golden/, made by tests/golden/make_golden.py),
independently of the oracle."""
import json
import os

import pytest

from conftest import ROOT, build_gpu

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _cases():
    import sys
    sys.path.insert(0, GOLDEN)
    import make_golden
    return make_golden.CASES, make_golden.DIGESTS


def _run(m, script):
    qf = min(0.3, m.min_quality())
    out = []
    for step in script.split(","):
        out.append({"refine": lambda: m.refine_by_size(qf),
                    "coarsen": lambda: m.coarsen_by_size(qf, 1 / 3.),
                    "swap": lambda: m.swap_slivers(0.3, 4),
                    "coarsen_slivers": lambda: m.coarsen_slivers(0.3, 4),
                    "adapt": lambda: m.adapt(1 / 3., 0.3, 4, 50)}[step]())
    return out


@pytest.mark.parametrize("name", ["cfg1_passes", "swap_slivers_n6", "coarsen_n8",
                                  "adapt_n6_parallel"])
def test_gpu_matches_reference_fixture(name):
    from oracle import oracle as O
    cases, _ = _cases()
    kw, script = cases[name]
    kw = dict(kw)
    n = kw.pop("n")
    g = build_gpu(n, **kw)
    rets = _run(g, script)
    want, extra = O.snapshot_from_npz(os.path.join(GOLDEN, name + ".npz"))
    assert rets == extra["returns"].tolist()
    errs = O.mesh_diff(g.snapshot(), want, rel_tol=0.0)
    assert not errs, errs[:5]


@pytest.mark.parametrize("name", ["adapt_n12_fields", "cfg2_adapt_box48"])
def test_gpu_matches_reference_digest(name):
    from oracle import oracle as O
    _, digests = _cases()
    kw, script = digests[name]
    kw = dict(kw)
    n = kw.pop("n")
    g = build_gpu(n, **kw)
    _run(g, script)
    with open(os.path.join(GOLDEN, "digests.json")) as f:
        want = json.load(f)[name]
    s = g.snapshot()
    assert s.counts == want["counts"]
    assert O.snapshot_digest(s) == want["sha256"]
