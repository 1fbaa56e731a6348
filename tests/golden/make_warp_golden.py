"""Records the SHA-256 of every VTU step the reference's 2D and 3D warp
tests (test_warp.cpp, test_warp_3d.cpp) write, run through the reference's own library
(oracle/_ref, oracle/Makefile) with tests/warp_flows.py:
`python tests/golden/make_warp_golden.py`. The GPU test compares this
library's files with these digests (and with a live reference run where
oracle/_ref is present)."""
import hashlib
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, HERE)

import warp_flows as W  # noqa: E402
from make_golden import Quiet  # noqa: E402
from oracle import oracle as O  # noqa: E402


def quiet(f, *a):
    with Quiet():
        return f(*a)


def record(dim, flow, coords, conn, name):
    m = O.ReferenceVariant(dim, coords, conn, "serial")
    m.derive_model_full()
    with tempfile.TemporaryDirectory() as d:
        files = flow(m, d, adapt=quiet)
        out = {os.path.basename(f): hashlib.sha256(open(f, "rb").read()).hexdigest()
               for f in files}
    json.dump(out, open(os.path.join(HERE, name), "w"), indent=1, sort_keys=True)
    print(name, len(out), "steps")


def main():
    record(2, W.run, W.BOX_2D_COORDS, W.BOX_2D_CONN, "warp2d_sha256.json")
    record(3, W.run3d, W.BOX_3D_COORDS, W.BOX_3D_CONN, "warp3d_sha256.json")


if __name__ == "__main__":
    main()
