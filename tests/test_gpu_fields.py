"""Size-field producers on the device (element_gradients,
recover_by_volume, size_from_hessian, warp_to_limit) and the warp-adapt
flow built on them, against the oracle (itself pinned to the reference):
bit-identical meshes, fields and warp outcomes."""
import numpy as np
import pytest

from conftest import build_cpu, build_gpu, front_warp_run

pytestmark = pytest.mark.gpu


def _oracle():
    from oracle import oracle as O
    return O


@pytest.mark.parametrize("n,angle,adapt", [(6, 0.25, True), (6, 1.6, False), (10, 0.4, True)])
def test_front_warp_flow_matches_oracle(n, angle, adapt):
    O = _oracle()
    g, o = build_gpu(n, size=0.1), build_cpu(O.Oracle, n, size=0.1)
    rg = front_warp_run(g, angle=angle, adapt=adapt)
    ro = front_warp_run(o, angle=angle, adapt=adapt)
    assert rg == ro
    errs = O.mesh_diff(g.snapshot(), o.snapshot(), rel_tol=0.0)
    assert not errs, errs[:5]


def test_size_chain_fields_match_oracle():
    """Each intermediate field of the chain, compared before adaptation."""
    from omega_h_v1_b200 import workloads as W
    from conftest import vertex_field
    O = _oracle()
    g, o = build_gpu(8, size=0.1, seed=3, pert=0.2), build_cpu(O.Oracle, 8, size=0.1, seed=3,
                                                              pert=0.2)
    for m in (g, o):
        m.add_field(0, "dye", W.front_field(vertex_field(m, "coordinates"), offset=0.45))
        m.element_gradients("dye")
        m.recover_by_volume("grad_dye")
        m.element_gradients("grad_dye")
        m.recover_by_volume("grad_grad_dye")
        m.free_tag(0, "adapt_size")
        m.size_from_hessian("grad_grad_dye", [3e-4], 0.01, 0.2)
    sg, so = g.snapshot(), o.snapshot()
    for d in (0, 3):
        names = [t.name for t in so.tags[d]]
        assert [t.name for t in sg.tags[d]] == names
        for t in so.tags[d]:
            assert np.array_equal(sg.tag(d, t.name).data, t.data), (d, t.name)
