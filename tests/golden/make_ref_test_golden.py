"""Records the SHA-256 of every VTU file the reference's own tests write
(test_warp.cpp, test_warp_3d.cpp, test_refine_by_size.cpp,
test_coarsen_by_size.cpp, test_box.cpp, test_grad.cpp), run through the
reference's library (oracle/_ref, oracle/Makefile) with the flows of
tests/ref_test_flows.py: `python tests/golden/make_ref_test_golden.py`.
The GPU test compares this library's files with these digests, and with a
live reference run where oracle/_ref is present."""
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

import ref_test_flows as W  # noqa: E402
from make_golden import Quiet  # noqa: E402
from oracle import oracle as O  # noqa: E402


def quiet(f, *a):
    with Quiet():
        return f(*a)


def main():
    out = {}
    for name in sorted(W.CASES):
        dim, flow, coords, conn, full = W.CASES[name]
        m = O.ReferenceVariant(dim, coords, conn, "serial")
        if full:
            m.derive_model_full()
        with tempfile.TemporaryDirectory() as d:
            files = flow(m, d, adapt=quiet)
            out[name] = {os.path.basename(f): hashlib.sha256(open(f, "rb").read()).hexdigest()
                         for f in files}
            print(name, len(files), "files", sum(os.path.getsize(f) for f in files), "bytes")
    json.dump(out, open(os.path.join(HERE, "ref_test_steps_sha256.json"), "w"), indent=1,
              sort_keys=True)


if __name__ == "__main__":
    main()
