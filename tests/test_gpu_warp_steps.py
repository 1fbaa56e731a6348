"""The reference's own warp tests run through this library on the GPU.
2D (test_warp.cpp): a box refined to size 0.1, a dye field whose recovered
Hessian sets the size field, eight rotation warps each applied up to the
quality limit with adaptation in between. 3D (test_warp_3d.cpp): a box
refined to size 0.2 with a conserved and a pointwise element field, eight
rotation warps with sliver layers. Every VTU step written
must equal, byte for byte, the step the reference writes on the same calls
(the reference's run_tests.sh diffs warp_0008.vtu against its gold copy):
against recorded digests, and against a live reference run when
oracle/_ref is built."""
import hashlib
import json
import os

import pytest

import warp_flows as W

pytestmark = pytest.mark.gpu

GOLD_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def _quiet(f, *a):
    import sys
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


CASES = {
    "2d": (2, W.run, W.BOX_2D_COORDS, W.BOX_2D_CONN, "warp2d_sha256.json"),
    "3d": (3, W.run3d, W.BOX_3D_COORDS, W.BOX_3D_CONN, "warp3d_sha256.json"),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_warp_steps_equal_the_reference(case, tmp_path):
    import omega_h_v1_b200 as G
    dim, flow, coords, conn, gold = CASES[case]
    m = G.Mesh.reduced(dim, coords, conn)
    m.derive_model_full()
    ours = tmp_path / "ours"
    ours.mkdir()
    files = flow(m, str(ours))
    want = json.load(open(os.path.join(GOLD_DIR, gold)))
    assert [os.path.basename(f) for f in files] == sorted(want)
    for f in files:
        assert _sha(f) == want[os.path.basename(f)], os.path.basename(f)
    from oracle import oracle as O
    if not O.have_reference(serial=True):
        return
    r = O.ReferenceVariant(dim, coords, conn, "serial")
    r.derive_model_full()
    ref = tmp_path / "ref"
    ref.mkdir()
    rfiles = flow(r, str(ref), adapt=_quiet)
    for a, b in zip(files, rfiles):
        assert open(a, "rb").read() == open(b, "rb").read(), os.path.basename(a)
