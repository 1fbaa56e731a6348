"""The scans' bounded wait: a look-back that never sees its predecessor
publish gives up after its limit, the stream's check reports E_TIMEOUT, and
the device stays usable (a pass run afterwards is exact)."""
import pytest

from conftest import build_cpu, build_gpu

pytestmark = pytest.mark.gpu


def test_scan_wait_gives_up_and_reports_timeout():
    import torch
    import omega_h_v1_b200 as G
    torch.cuda.set_device(0)
    L = G.lib()
    L.osh_b200_selftest_scan_wait.restype = G.C.c_int
    L.osh_b200_selftest_scan_wait.argtypes = [G.C.c_uint]
    assert L.osh_b200_selftest_scan_wait(1000) == 7   # OSH_B200_E_TIMEOUT
    L.osh_b200_clear_error()
    # the context is intact: a refinement pass still matches the oracle
    from oracle import oracle as O
    g, o = build_gpu(4, size=0.2), build_cpu(O.Oracle, 4, size=0.2)
    qf = min(0.3, o.min_quality())
    assert g.refine_by_size(qf) == o.refine_by_size(qf)
    assert not O.mesh_diff(g.snapshot(), o.snapshot())
