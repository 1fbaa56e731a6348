"""The reference's own 2D warp test (test_warp.cpp) run through this
library on the GPU: a 2D box refined to size 0.1, a dye field whose
recovered Hessian sets the size field, eight rotation warps each applied
up to the quality limit with adaptation in between. Every VTU step written
must equal, byte for byte, the step the reference writes on the same calls
(the reference's run_tests.sh diffs warp_0008.vtu against its gold copy):
against recorded digests, and against a live reference run when
oracle/_ref is built."""
import hashlib
import json
import os

import pytest

import warp2d_flow as W

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                    "warp2d_sha256.json")


def _sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def test_2d_warp_steps_equal_the_reference(tmp_path):
    import omega_h_v1_b200 as G
    m = G.Mesh.reduced(2, W.BOX_2D_COORDS, W.BOX_2D_CONN)
    m.derive_model_full()
    ours = tmp_path / "ours"
    ours.mkdir()
    files = W.run(m, str(ours))
    want = json.load(open(GOLD))
    assert [os.path.basename(f) for f in files] == sorted(want)
    for f in files:
        assert _sha(f) == want[os.path.basename(f)], os.path.basename(f)
    from oracle import oracle as O
    if not O.have_reference(serial=True):
        return
    import sys

    def quiet(f, *a):
        # the reference prints a line per pass
        sys.stdout.flush()
        saved, null = os.dup(1), os.open(os.devnull, os.O_WRONLY)
        os.dup2(null, 1)
        try:
            return f(*a)
        finally:
            os.dup2(saved, 1)
            os.close(saved)
            os.close(null)

    r = O.ReferenceVariant(2, W.BOX_2D_COORDS, W.BOX_2D_CONN, "serial")
    r.derive_model_full()
    ref = tmp_path / "ref"
    ref.mkdir()
    rfiles = W.run(r, str(ref), adapt=quiet)
    for a, b in zip(files, rfiles):
        assert open(a, "rb").read() == open(b, "rb").read(), os.path.basename(a)
