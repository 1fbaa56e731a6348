"""The public C ABI used the way an Omega_h v1 caller uses it
(omega_h.cpp:177-1054): osh_new, osh_build_ents, fields, labels, global
numbers, then osh_adapt; plus the getters and small entry points."""
import ctypes as C

import numpy as np
import pytest

from conftest import build_cpu

pytestmark = pytest.mark.gpu


def _G():
    import omega_h_v1_b200 as G
    return G


def _upload(G, L, ptr, arr):
    arr = np.ascontiguousarray(arr)
    L.osh_b200_copy_to_device(ptr, arr.ctypes.data_as(C.c_void_p), arr.nbytes)
    G.check()


def _mesh_from_snapshot(G, snap):
    """Build a full-topology parallel mesh through osh_new / osh_build_ents
    exactly as a C caller would, from a host snapshot."""
    L = G.lib()
    h = L.osh_new(3)
    G.check()
    L.osh_build_ents(h, 0, snap.counts[0])
    for d in (1, 2, 3):
        p = L.osh_build_ents(h, d, snap.counts[d])
        _upload(G, L, p, snap.conn[d].astype(np.uint32))
    for d in range(4):
        for t in snap.tags[d]:
            if t.type == G.T_F64:
                p = L.osh_new_field(h, d, t.name.encode(), t.ncomps, t.transfer)
            else:
                p = L.osh_new_label(h, d, t.name.encode(), t.ncomps)
            G.check()
            _upload(G, L, p, t.data)
        if d in snap.globals:
            p = L.osh_new_global(h, d)
            _upload(G, L, p, snap.globals[d].astype(np.uint64))
    return G.Mesh(h)


@pytest.mark.parametrize("kw", [dict(n=6, seed=4, pert=0.25, size=0.25, fields=True),
                                dict(n=10, seed=1, size=0.07, fields=True)])
def test_osh_adapt_through_c_abi_matches_oracle(kw):
    from oracle import oracle as O
    G = _G()
    kw = dict(kw)
    n = kw.pop("n")
    o = build_cpu(O.Oracle, n, parallel=True, **kw)
    g = _mesh_from_snapshot(G, o.snapshot())
    assert g.adapt(1 / 3., 0.3, 4, 50) == o.adapt(1 / 3., 0.3, 4, 50)
    errs = O.mesh_diff(g.snapshot(), o.snapshot(), rel_tol=1e-12)
    assert not errs, errs[:5]


def test_getters_and_small_entry_points():
    from oracle import oracle as O
    G = _G()
    L = G.lib()
    o = build_cpu(O.Oracle, 4)
    g = _mesh_from_snapshot(G, o.snapshot())
    h = g.h
    assert L.osh_dim(h) == 3
    assert L.osh_count(h, 3) == o.count(3)
    # identity size: longest adjacent edge per vertex (size.cpp:90-135)
    L.osh_identity_size(h, b"ident")
    G.check()
    x = o.snapshot().tag(0, "coordinates").data.reshape(-1, 3)
    ev = o.down(1, 0).reshape(-1, 2)
    # same summation order as vector_squared_distance(x_other, x_self)
    want = np.zeros(len(x))
    for e, (a, b) in enumerate(ev):
        for i, j in ((a, b), (b, a)):
            dx = x[j] - x[i]
            s = 0.0
            s += dx[0] * dx[0]
            s += dx[1] * dx[1]
            s += dx[2] * dx[2]
            want[i] = max(want[i], np.sqrt(s))
    got = [t for t in g.tags(0) if t.name == "ident"][0].data
    assert np.array_equal(got, want)
    # mark_classified: OR into a caller array (omega_h.cpp:890-903)
    cd = o.snapshot().tag(1, "class_dim").data
    import torch
    marked = torch.zeros(o.count(1), dtype=torch.int32, device="cuda")
    L.osh_mark_classified(h, 1, 2, 0xFFFFFFFF, C.c_void_p(marked.data_ptr()))
    G.check()
    assert np.array_equal(marked.cpu().numpy().astype(np.uint32), (cd == 2).astype(np.uint32))
    # own ranks / ids on one rank
    L.osh_own_rank.restype = C.c_void_p
    L.osh_own_id.restype = C.c_void_p
    pr = L.osh_own_rank(h, 0)
    pi = L.osh_own_id(h, 0)
    r = np.empty(o.count(0), np.uint32)
    i = np.empty(o.count(0), np.uint32)
    L.osh_b200_copy_to_host(r.ctypes.data_as(C.c_void_p), pr, r.nbytes)
    L.osh_b200_copy_to_host(i.ctypes.data_as(C.c_void_p), pi, i.nbytes)
    assert not r.any() and np.array_equal(i, np.arange(o.count(0)))
    # a missing VTU file is reported (OSH_B200_E_IO), not aborted on
    L.osh_read_vtk.restype = C.c_void_p
    assert not L.osh_read_vtk(b"missing.vtu")
    assert L.osh_b200_last_error() == 9
    L.osh_b200_clear_error()


def test_async_copies_round_trip():
    """osh_b200_copy_to_device_async / _to_host_async run on the mesh's own
    stream (a non-blocking one here, as osh_new makes it) in order with its
    work: a field uploaded and copied back, read after
    osh_b200_synchronize, equals what was sent; the array osh_new_field
    returns takes the copies at once."""
    import torch
    G = _G()
    L = G.lib()
    h = L.osh_new(3)
    G.check()
    L.osh_build_ents(h, 0, 1000)
    L.osh_build_ents(h, 3, 0)
    p = L.osh_new_field(h, 0, b"u", 3, 0)
    G.check()
    src = torch.arange(3000, dtype=torch.float64).pin_memory()
    dst = torch.full((3000,), -1.0, dtype=torch.float64).pin_memory()
    L.osh_b200_copy_to_device_async(h, p, C.c_void_p(src.data_ptr()), 3000 * 8)
    L.osh_b200_copy_to_host_async(h, C.c_void_p(dst.data_ptr()), p, 3000 * 8)
    L.osh_b200_synchronize(h)
    G.check()
    assert torch.equal(src, dst)
    # and the synchronous copy sees the same array
    back = np.empty(3000)
    L.osh_b200_copy_to_host(back.ctypes.data_as(C.c_void_p), p, back.nbytes)
    G.check()
    assert np.array_equal(back, np.arange(3000, dtype=np.float64))
    L.osh_free(h)
