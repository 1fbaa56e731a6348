"""Regenerates the golden fixtures in this folder from the reference itself.

Run where the reference sources are present (oracle/Makefile builds them into
oracle/_ref/): `python tests/golden/make_golden.py`. Each fixture is the
reference's output for one seeded input and pass sequence; the CPU tests pin
the oracle to them and the GPU tests pin the CUDA path to the digests, so
both checks work on machines without the reference.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from conftest import build_cpu  # noqa: E402
from oracle import oracle as O  # noqa: E402


class Quiet:
    """Silence the reference's printf output."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)

    def __exit__(self, *a):
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


# name -> (builder kwargs, box n, pass script)
CASES = {
    # 3,072 tets, h = 0.05: one refine (512 splits), coarsen and swap no-ops
    "cfg1_passes": (dict(n=8, size=0.05), "refine,coarsen,swap"),
    # sliver-prone box with fields: a swap pass then a sliver collapse pass
    "swap_slivers_n6": (dict(n=6, seed=0, pert=0.3, size=1 / 6., fields=True),
                        "swap,coarsen_slivers"),
    # coarsening of an over-resolved box with fields
    "coarsen_n8": (dict(n=8, seed=5, size=0.4, fields=True), "coarsen"),
    # full mesh_adapt with refine, coarsen, swap and sliver collapse, parallel
    "adapt_n6_parallel": (dict(n=6, seed=4, pert=0.25, size=1 / 4., fields=True,
                               parallel=True), "adapt"),
}

# larger cases kept as digests only: (builder kwargs, pass script)
DIGESTS = {
    "cfg2_adapt_box48": (dict(n=48, seed=0, radial=(0.01, 0.04)), "adapt"),
    "adapt_n12_fields": (dict(n=12, seed=4, pert=0.2, size=1 / 12., fields=True), "adapt"),
}


def run(m, script):
    qf = min(0.3, m.min_quality())
    rets = []
    for step in script.split(","):
        if step == "refine":
            rets.append(m.refine_by_size(qf))
        elif step == "coarsen":
            rets.append(m.coarsen_by_size(qf, 1 / 3.))
        elif step == "swap":
            rets.append(m.swap_slivers(0.3, 4))
        elif step == "coarsen_slivers":
            rets.append(m.coarsen_slivers(0.3, 4))
        elif step == "adapt":
            rets.append(m.adapt(1 / 3., 0.3, 4, 50))
    return np.asarray(rets, np.uint32)


def main():
    assert O.have_reference(), "build oracle/_ref first (make -C oracle)"
    digests = {}
    for name, (kw, script) in CASES.items():
        kw = dict(kw)
        n = kw.pop("n")
        m = build_cpu(O.Reference, n, **kw)
        with Quiet():
            rets = run(m, script)
        s = m.snapshot()
        O.snapshot_to_npz(s, os.path.join(HERE, name + ".npz"), returns=rets)
        digests[name] = {"sha256": O.snapshot_digest(s), "counts": s.counts,
                         "returns": rets.tolist(), "script": script}
        print(name, s.counts, rets.tolist())
    for name, (kw, script) in DIGESTS.items():
        kw = dict(kw)
        n = kw.pop("n")
        m = build_cpu(O.Reference, n, **kw)
        with Quiet():
            rets = run(m, script)
        s = m.snapshot()
        digests[name] = {"sha256": O.snapshot_digest(s), "counts": s.counts,
                         "returns": rets.tolist(), "script": script}
        print(name, s.counts, rets.tolist())
    with open(os.path.join(HERE, "digests.json"), "w") as f:
        json.dump(digests, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
