"""osh_b200_up_from_down_noalloc: upward adjacency without device allocation.

The entry point exists for callers that cannot allocate device memory when
they need the adjacency (host callbacks and real-time loops that must not
wait on the allocator, codes that hand the GPU a fixed memory budget). Its
output must equal what the allocating getters osh_up_offs / osh_up /
osh_up_dirs return for the same mesh, on two calls in a row (the calls share
one scratch array), up to and including its stated maximum of 2^20 uses; it
must refuse sizes above its maxima without launching anything, and report
an input it cannot use in offsets[nlows] without writing through it.

This file is collected last so that a failure here leaves every other test
already run; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(L):
    fn = L.osh_b200_up_from_down_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_void_p, C.c_void_p,
                   C.c_void_p, C.c_void_p, C.c_void_p]
    return fn


def _call_twice(G, fn, high, low, nh, nl, loh, want):
    import torch
    L = G.lib()
    deg = G.DEG[high][low]
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
        assert got[0][nl] == nh * deg, "offsets[nlows] holds nuses, call %d" % call
        assert np.array_equal(got[0], want[0]), "offsets, call %d" % call
        assert np.array_equal(got[1], want[1]), "highs_of_lows, call %d" % call
        assert np.array_equal(got[2], want[2]), "directions, call %d" % call


@pytest.mark.parametrize("high,low", [(3, 0), (3, 1)])
def test_noalloc_matches_allocating_getters(high, low):
    import torch
    import omega_h_v1_b200 as G
    torch.cuda.set_device(0)
    coords, conn, _ = G.box(20, 7, 0.1)
    m = G.Mesh.reduced(3, coords, conn)
    m.derive_model_full()
    L = G.lib()
    nh, nl = m.count(high), m.count(low)
    assert nh * G.DEG[high][low] <= 1 << 20 and nl <= 1 << 20
    want = m.up(low, high)   # allocating path
    loh = L.osh_down(m.h, high, low)
    G.check()
    _call_twice(G, _bind(L), high, low, nh, nl, loh, want)
    m.close()


def test_noalloc_at_its_maximum_of_uses():
    """2^18 tets, vertices as the low entities: exactly 2^20 uses."""
    import torch
    import omega_h_v1_b200 as G
    torch.cuda.set_device(0)
    coords, conn, _ = G.box(36, 3, 0.1)
    nt = 1 << 18
    m = G.Mesh.reduced(3, coords, np.ascontiguousarray(conn[: nt * 4]))
    L = G.lib()
    nh, nl = m.count(3), m.count(0)
    assert nh * 4 == 1 << 20
    want = m.up(0, 3)
    loh = L.osh_down(m.h, 3, 0)
    G.check()
    _call_twice(G, _bind(L), 3, 0, nh, nl, loh, want)
    m.close()


def test_noalloc_reports_an_unusable_input_in_offsets():
    """An entry of lows_of_highs not below nlows: no write through it, the
    outputs untouched, 0xffffffff in offsets[nlows]; the next good call on
    the shared scratch is exact again."""
    import torch
    import omega_h_v1_b200 as G
    torch.cuda.set_device(0)
    L = G.lib()
    fn = _bind(L)
    loh = torch.tensor([0, 1, 2, 3, 1, 2, 3, 9], dtype=torch.int32, device="cuda")
    offs = torch.zeros(5, dtype=torch.int32, device="cuda")
    adj = torch.full((8,), -1, dtype=torch.int32, device="cuda")
    dirs = torch.full((8,), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    rc = fn(3, 0, 2, 4, C.c_void_p(loh.data_ptr()), C.c_void_p(offs.data_ptr()),
            C.c_void_p(adj.data_ptr()), C.c_void_p(dirs.data_ptr()),
            C.c_void_p(stream.cuda_stream))
    assert rc == 0
    stream.synchronize()
    assert offs.cpu().numpy().view(np.uint32)[4] == 0xFFFFFFFF
    assert (adj.cpu().numpy() == -1).all() and (dirs.cpu().numpy() == -1).all()
    loh[7] = 0
    rc = fn(3, 0, 2, 4, C.c_void_p(loh.data_ptr()), C.c_void_p(offs.data_ptr()),
            C.c_void_p(adj.data_ptr()), C.c_void_p(dirs.data_ptr()),
            C.c_void_p(stream.cuda_stream))
    assert rc == 0
    stream.synchronize()
    assert offs.cpu().tolist() == [0, 2, 4, 6, 8]
    assert adj.cpu().tolist() == [0, 1, 0, 1, 0, 1, 0, 1]
    assert dirs.cpu().tolist() == [0, 3, 1, 0, 2, 1, 3, 2]


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
