"""Records the reference's own digests of the full-size parity cases
(tests/large_flows.py) into large_digests.json.

Run where the reference sources are present (oracle/Makefile builds the
reference's OpenMP library into oracle/_ref/):

    python tests/golden/make_large_digests.py [boxes] [front]

* boxes: mesh_adapt(1/3, 0.3, 4, 50) of every box with n <= 16 of the
  seeded 512-box set, and of its three largest boxes;
* front: the 96^3 anisotropic front workload after its first mesh_adapt and
  after its first warp step.

Each digest is oracle.snapshot_digest of the adapted mesh (counts,
connectivity, every tag in order, global numbers), so the GPU tests can
compare without the reference being present.
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import large_flows as F  # noqa: E402
from make_golden import Quiet  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(HERE, "large_digests.json")


def load():
    if os.path.exists(OUT):
        with open(OUT) as f:
            return json.load(f)
    return {}


def save(d):
    with open(OUT, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)


def record(s, extra=None):
    r = {"sha256": O.snapshot_digest(s), "counts": s.counts}
    if extra:
        r.update(extra)
    return r


def boxes(out):
    res = {}
    t0 = time.time()
    for j in F.batched_subset():
        m = F.box_job_mesh(O.Reference, O.box, j)
        with Quiet():
            ret = m.adapt(*F.BOX_ADAPT)
        res[str(j.index)] = record(m.snapshot(), {"n": j.n, "size": j.size,
                                                  "returns": int(ret)})
        m.close()
    out["batched_subset"] = {"jobs": res, "adapt": list(F.BOX_ADAPT),
                             "seconds": round(time.time() - t0, 1)}
    print("boxes: %d meshes in %.0f s" % (len(res), time.time() - t0), flush=True)


def front(out):
    t0 = time.time()
    m = F.front_mesh(O.Reference, O.box)
    with Quiet():
        m.adapt(*F.FRONT_ADAPT)
    out["front_first_adapt"] = record(m.snapshot(), {"seconds": round(time.time() - t0, 1)})
    save(out)
    print("front first adapt: %s in %.0f s" % (m.count(3), time.time() - t0), flush=True)
    t1 = time.time()
    with Quiet():
        tries = F.front_warp_step(m)
    out["front_warp_step1"] = record(m.snapshot(), {"tries": tries,
                                                    "seconds": round(time.time() - t1, 1)})
    print("front warp step 1: %s tets, %d tries in %.0f s" % (m.count(3), tries,
                                                            time.time() - t1), flush=True)
    m.close()


def main():
    assert O.have_reference(), "build oracle/_ref first (make -C oracle)"
    which = sys.argv[1:] or ["boxes", "front"]
    out = load()
    if "boxes" in which:
        boxes(out)
        save(out)
    if "front" in which:
        front(out)
        save(out)


if __name__ == "__main__":
    main()
