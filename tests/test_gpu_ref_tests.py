"""The reference's own tests, run through this library on the GPU:
test_warp.cpp (2D: Hessian size fields, eight rotation warps),
test_warp_3d.cpp (3D: conserved and pointwise element fields, warps with
sliver layers), test_refine_by_size.cpp and test_coarsen_by_size.cpp (2D,
radial size fields), test_box.cpp (uniform refinement, the arguments of
run_tests.sh) and test_grad.cpp (3D unclassified mesh, gradient recovery,
size from Hessian), test_one_refine.cpp and test_one_coarsen.cpp (a
parallel mesh through .pvtu files). Every VTU file a flow writes must
equal, byte for byte,
the file the reference writes on the same calls (the reference's own
run_tests.sh diffs warp_0008.vtu against a gold copy): against digests
recorded from the reference (tests/golden/make_ref_test_golden.py), and
against a live reference run when oracle/_ref is built."""
import hashlib
import json
import os
import sys

import pytest

import ref_test_flows as W

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                    "ref_test_steps_sha256.json")


def _sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def _quiet(f, *a):
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


@pytest.mark.parametrize("case", sorted(W.CASES))
def test_reference_test_files_equal(case, tmp_path):
    import omega_h_v1_b200 as G
    dim, flow, coords, conn, full = W.CASES[case]
    m = G.Mesh.reduced(dim, coords, conn)
    if full:
        m.derive_model_full()
    ours = tmp_path / "ours"
    ours.mkdir()
    files = flow(m, str(ours))
    want = json.load(open(GOLD))[case]
    assert sorted(os.path.basename(f) for f in files) == sorted(want)
    for f in files:
        assert _sha(f) == want[os.path.basename(f)], os.path.basename(f)
    from oracle import oracle as O
    if not O.have_reference(serial=True):
        return
    r = O.ReferenceVariant(dim, coords, conn, "serial")
    if full:
        r.derive_model_full()
    ref = tmp_path / "ref"
    ref.mkdir()
    rfiles = flow(r, str(ref), adapt=_quiet)
    for a, b in zip(sorted(files), sorted(rfiles)):
        assert open(a, "rb").read() == open(b, "rb").read(), os.path.basename(a)
