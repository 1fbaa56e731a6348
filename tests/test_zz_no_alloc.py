"""osh_b200_up_from_down_noalloc: upward adjacency without device allocation.

The entry point exists for callers that cannot allocate device memory when
they need the adjacency (work issued during CUDA graph capture, host
callbacks, codes with a fixed device-memory budget). Its output must equal
what the allocating getters osh_up_offs / osh_up / osh_up_dirs return for the
same mesh, on two calls in a row (the calls share one scratch array), and it
must refuse sizes above its stated maxima without launching anything.

This file is collected last so that a failure here leaves every other test
already run; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mesh(n=20):
    import omega_h_v1_b200 as G
    coords, conn, _ = G.box(n, 7, 0.1)
    m = G.Mesh.reduced(3, coords, conn)
    m.derive_model_full()
    return G, m


def _bind(L):
    fn = L.osh_b200_up_from_down_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_void_p, C.c_void_p,
                   C.c_void_p, C.c_void_p, C.c_void_p]
    return fn


@pytest.mark.parametrize("high,low", [(3, 0), (3, 1)])
def test_noalloc_matches_allocating_getters(high, low):
    import torch
    torch.cuda.set_device(0)
    G, m = _mesh()
    L = G.lib()
    fn = _bind(L)
    deg = G.DEG[high][low]
    nh, nl = m.count(high), m.count(low)
    assert nh * deg <= 1 << 20 and nl <= 1 << 20
    want_offs, want_adj, want_dirs = m.up(low, high)   # allocating path
    loh = L.osh_down(m.h, high, low)
    G.check()
    stream = torch.cuda.current_stream()
    for call in range(2):  # two calls in a row share the scratch array
        offs = torch.full((nl + 1,), -1, dtype=torch.int32, device="cuda")
        adj = torch.full((nh * deg,), -1, dtype=torch.int32, device="cuda")
        dirs = torch.full((nh * deg,), -1, dtype=torch.int32, device="cuda")
        rc = fn(high, low, nh, nl, loh, C.c_void_p(offs.data_ptr()),
                C.c_void_p(adj.data_ptr()), C.c_void_p(dirs.data_ptr()),
                C.c_void_p(stream.cuda_stream))
        assert rc == 0, L.osh_b200_last_error_message()
        stream.synchronize()
        got = [t.cpu().numpy().view(np.uint32) for t in (offs, adj, dirs)]
        assert np.array_equal(got[0], want_offs), "offsets, call %d" % call
        assert np.array_equal(got[1], want_adj), "highs_of_lows, call %d" % call
        assert np.array_equal(got[2], want_dirs), "directions, call %d" % call
    m.close()


def test_noalloc_rejects_sizes_above_maximum():
    import torch
    import omega_h_v1_b200 as G
    torch.cuda.set_device(0)
    L = G.lib()
    fn = _bind(L)
    # 2^18 + 1 tets * 4 uses is above the 2^20-use cap: refused, nothing runs
    rc = fn(3, 0, (1 << 18) + 1, 1000, None, None, None, None, None)
    assert rc == 4
    assert "OSH_B200_NOALLOC_MAX_USES" in L.osh_b200_last_error_message().decode()
    L.osh_b200_clear_error()
    rc = fn(3, 0, 10, (1 << 20) + 1, None, None, None, None, None)
    assert rc == 4
    L.osh_b200_clear_error()
