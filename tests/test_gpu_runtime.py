"""The passes' scan: exact at sizes from empty to 2^25 items (one tile,
ragged last tiles, thousands of tiles), and its bounded wait: a look-back
that never sees its predecessor publish gives up after its limit, the
stream's check reports E_TIMEOUT, and the device stays usable (a pass run
afterwards is exact)."""
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


@pytest.mark.parametrize("n", [0, 1, 4095, 4096, 8193, 100003, 1 << 22, (1 << 25) + 7])
def test_exscan_matches_numpy(n):
    import numpy as np
    import torch
    import omega_h_v1_b200 as G
    torch.cuda.set_device(0)
    L = G.lib()
    rng = np.random.default_rng(n)
    # counts like the passes' (0..12 per item), and wrap-around at 2^25 items
    hi = 13 if n < (1 << 25) else 300
    a = rng.integers(0, hi, size=n, dtype=np.uint32)
    d_in = torch.from_numpy(a.view(np.int32)).cuda() if n else torch.empty(1, dtype=torch.int32,
                                                                           device="cuda")
    d_out = torch.full((n + 1,), -1, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    for _ in range(2):   # twice: the scratch is returned to zero after a scan
        assert L.osh_b200_exscan_u32(d_in.data_ptr(), d_out.data_ptr(), n, s, 1) == 0
        got = d_out.cpu().numpy().view(np.uint32)
        want = np.zeros(n + 1, dtype=np.uint64)
        np.cumsum(a, dtype=np.uint64, out=want[1:])
        assert np.array_equal(got, (want & 0xffffffff).astype(np.uint32))


def test_exscan_rejects_overlap():
    import torch
    import omega_h_v1_b200 as G
    torch.cuda.set_device(0)
    L = G.lib()
    buf = torch.zeros(100, dtype=torch.int32, device="cuda")
    p = buf.data_ptr()
    assert L.osh_b200_exscan_u32(p, p + 4 * 10, 50, None, 1) == 4   # OSH_B200_E_ARG
    L.osh_b200_clear_error()


def test_released_stream_leaves_meshes_usable():
    """A mesh adapted on a caller's stream, whose scratch is then released
    (osh_b200_release_stream) and the stream destroyed, keeps working on
    another stream, and matches the oracle: the library kept nothing of
    the released stream. Repeated over several streams, as a caller that
    makes one per request would."""
    import torch
    import omega_h_v1_b200 as G
    from oracle import oracle as O
    torch.cuda.set_device(0)
    L = G.lib()
    g, o = build_gpu(5, size=0.2), build_cpu(O.Oracle, 5, size=0.2)
    for _ in range(3):
        st = torch.cuda.Stream()
        L.osh_b200_set_stream(g.h, G.C.c_void_p(st.cuda_stream))
        G.check()
        qf = min(0.3, o.min_quality())
        assert g.refine_by_size(qf) == o.refine_by_size(qf)
        L.osh_b200_set_stream(g.h, G.C.c_void_p(0))
        G.check()
        L.osh_b200_release_stream(G.C.c_void_p(st.cuda_stream))
        G.check()
        st.synchronize()
        del st
    qf = min(0.3, o.min_quality())
    assert g.coarsen_by_size(qf, 1 / 3.) == o.coarsen_by_size(qf, 1 / 3.)
    assert not O.mesh_diff(g.snapshot(), o.snapshot())
