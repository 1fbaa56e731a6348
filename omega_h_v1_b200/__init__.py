"""Python front-end of libosh_b200.so, the sm_100a mesh-adaptation library.

Everything here calls the library's C ABI (include/omega_h.h and
include/omega_h_b200.h) through ctypes; the library itself is CUDA + C++.
There is no CPU fallback: importing works without a GPU (for symbol checks),
but creating a mesh needs a CUDA device and raises if the library is missing.

``Mesh`` mirrors the reference's C++ entry points for the adaptation pass
(refine_by_size, coarsen_by_size, coarsen_slivers, swap_slivers, mesh_adapt)
and the getters of the public C API, with host copies for inspection.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libosh_b200.so")
INCLUDE_DIR = os.path.join(os.path.dirname(HERE), "include")

T_U8, T_U32, T_U64, T_F64 = 0, 1, 2, 3
X_NOT, X_POINTWISE, X_CONSERVE, X_INHERIT = 0, 1, 2, 3
DEG = [[1, 0, 0, 0], [2, 1, 0, 0], [3, 3, 1, 0], [4, 6, 4, 1]]
_NP = {T_U8: np.uint8, T_U32: np.uint32, T_U64: np.uint64, T_F64: np.float64}
ERRORS = {0: "ok", 1: "cuda", 2: "no convergence", 3: "max passes", 4: "argument",
          5: "out of memory", 6: "unsupported", 7: "timeout", 8: "inverted element",
          9: "file"}

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


class OshError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "?"), code, msg))
        self.code = code


def exported_symbols():
    """Names declared in the public headers, in declaration order."""
    import re
    names = []
    for h in ("omega_h.h", "omega_h_b200.h"):
        txt = open(os.path.join(INCLUDE_DIR, h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names += re.findall(r"\b(osh_\w+)\s*\(", txt)
    seen, out = set(), []
    for n in names:
        if n not in seen:
            seen.add(n)
            out.append(n)
    return out


_lib = None


def lib():
    """Load libosh_b200.so (built in place by ``build()``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libosh_b200.so is not built; run __graft_entry__.build()")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p

    def f(name, res, *args):
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = list(args)

    f("osh_init", None, vp, vp)
    f("osh_free", None, vp)
    f("osh_new", vp, C.c_uint)
    f("osh_build_ents", vp, vp, C.c_uint, C.c_uint)
    f("osh_dim", C.c_uint, vp)
    f("osh_count", C.c_uint, vp, C.c_uint)
    f("osh_down", vp, vp, C.c_uint, C.c_uint)
    f("osh_up", vp, vp, C.c_uint, C.c_uint)
    f("osh_up_offs", vp, vp, C.c_uint, C.c_uint)
    f("osh_up_dirs", vp, vp, C.c_uint, C.c_uint)
    f("osh_star", vp, vp, C.c_uint, C.c_uint)
    f("osh_star_offs", vp, vp, C.c_uint, C.c_uint)
    f("osh_coords", vp, vp)
    f("osh_global", vp, vp, C.c_uint)
    f("osh_new_field", vp, vp, C.c_uint, C.c_char_p, C.c_uint, C.c_int)
    f("osh_get_field", vp, vp, C.c_uint, C.c_char_p)
    f("osh_new_label", vp, vp, C.c_uint, C.c_char_p, C.c_uint)
    f("osh_new_global", vp, vp, C.c_uint)
    f("osh_adapt", C.c_uint, vp, C.c_double, C.c_double, C.c_uint, C.c_uint)
    f("osh_identity_size", None, vp, C.c_char_p)
    f("osh_mark_classified", None, vp, C.c_uint, C.c_uint, C.c_uint, vp)
    f("osh_b200_last_error", C.c_int)
    f("osh_b200_last_error_message", C.c_char_p)
    f("osh_b200_clear_error", None)
    f("osh_b200_refine_by_size", C.c_uint, vp, C.c_double)
    f("osh_b200_uniformly_refine", None, vp)
    f("osh_b200_coarsen_by_size", C.c_uint, vp, C.c_double, C.c_double)
    f("osh_b200_coarsen_slivers", C.c_uint, vp, C.c_double, C.c_uint)
    f("osh_b200_swap_slivers", C.c_uint, vp, C.c_double, C.c_uint)
    f("osh_b200_mesh_adapt", C.c_uint, vp, C.c_double, C.c_double, C.c_uint, C.c_uint)
    f("osh_b200_min_quality", C.c_double, vp)
    f("osh_b200_last_pass", None, *([C.POINTER(C.c_uint)] * 5))
    f("osh_b200_refine_sets", C.c_uint, vp, C.c_double, _u32p, _u32p, _f64p, _u32p)
    f("osh_b200_coarsen_sets", C.c_uint, vp, C.c_double, C.c_double, _u32p, _u32p,
      _u32p, _f64p, _u32p, _f64p, _u32p, _u32p)
    f("osh_b200_swap_sets", C.c_uint, vp, C.c_double, C.c_uint, _u32p, _u32p,
      _u32p, _u32p, _f64p, _u32p, _u32p)
    f("osh_b200_new_reduced", vp, C.c_uint, C.c_uint, _f64p, C.c_uint, _u32p)
    f("osh_b200_derive_model", None, vp, C.c_double)
    f("osh_b200_make_parallel", None, vp)
    f("osh_b200_box", None, C.c_uint, C.c_ulong, C.c_double, _f64p, _u32p, _f64p)
    f("osh_b200_add_tag", None, vp, C.c_uint, C.c_char_p, C.c_uint, C.c_uint, C.c_uint, vp)
    f("osh_b200_ntags", C.c_uint, vp, C.c_uint)
    f("osh_b200_tag_name", C.c_char_p, vp, C.c_uint, C.c_uint)
    f("osh_b200_tag_info", None, vp, C.c_uint, C.c_uint, C.POINTER(C.c_uint),
      C.POINTER(C.c_uint), C.POINTER(C.c_uint))
    f("osh_b200_tag_data", vp, vp, C.c_uint, C.c_uint)
    f("osh_b200_set_globals", None, vp, C.c_uint, _u64p)
    f("osh_b200_dual", vp, vp)
    f("osh_b200_qualities", None, vp, _f64p)
    f("osh_b200_edge_lengths", None, vp, _f64p)
    f("osh_b200_copy_to_host", None, vp, vp, C.c_size_t)
    f("osh_b200_copy_to_device", None, vp, vp, C.c_size_t)
    f("osh_b200_copy_to_host_async", None, vp, vp, vp, C.c_size_t)
    f("osh_b200_copy_to_device_async", None, vp, vp, vp, C.c_size_t)
    f("osh_b200_synchronize", None, vp)
    f("osh_b200_clone", vp, vp)
    f("osh_b200_set_stream", None, vp, vp)
    f("osh_b200_release_stream", None, vp)
    f("osh_b200_adapt_stats", None, C.POINTER(C.c_uint), C.POINTER(C.c_double))
    f("osh_b200_adapt_batch", C.c_int, C.POINTER(vp), C.c_uint, C.c_double, C.c_double,
      C.c_uint, C.c_uint, C.c_ulonglong, C.POINTER(C.c_uint), C.POINTER(C.c_int))
    f("osh_b200_adapt_concurrent", C.c_int, C.POINTER(vp), C.c_uint, C.c_double, C.c_double,
      C.c_uint, C.c_uint, C.c_uint, C.c_ulonglong, C.POINTER(C.c_uint), C.POINTER(C.c_int))
    f("osh_b200_batch_stats", None, *([C.POINTER(C.c_uint)] * 4), C.POINTER(C.c_double))
    f("osh_b200_batch_mesh_stats", None, C.c_uint, C.POINTER(C.c_uint), C.POINTER(C.c_double))
    f("osh_b200_batch_times", None, *([C.POINTER(C.c_double)] * 3))
    f("osh_b200_digest", C.c_ulonglong, vp)
    f("osh_b200_has_dim", C.c_uint, vp, C.c_uint)
    f("osh_ghost", None, vp, C.c_uint)
    f("osh_num_ghost_layers", C.c_uint, vp)
    f("osh_read_vtk", vp, C.c_char_p)
    f("osh_write_vtk", None, vp, C.c_char_p)
    f("osh_b200_write_vtk_opts", None, vp, C.c_char_p, C.c_int, C.c_int)
    f("osh_b200_pool_reserve", None, C.c_ulonglong)
    f("osh_b200_pool_stats", None, *([C.POINTER(C.c_ulonglong)] * 3), C.c_int)
    f("osh_b200_set_fp32_filter", None, vp, C.c_int)
    f("osh_b200_element_gradients", None, vp, C.c_char_p)
    f("osh_b200_recover_by_volume", None, vp, C.c_char_p)
    f("osh_b200_size_from_hessian", None, vp, C.c_char_p, C.c_void_p, C.c_double, C.c_double)
    f("osh_b200_warp_to_limit", C.c_uint, vp, C.c_double)
    f("osh_free_field", None, vp, C.c_uint, C.c_char_p)
    f("osh_b200_fp32_stats", None, C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong),
      C.POINTER(C.c_double), C.POINTER(C.c_uint))
    f("osh_b200_fp32_stats_reset", None)
    f("osh_b200_set_fp32_audit", None, C.c_int)
    f("osh_b200_fp32_audit_stats", None, *([C.POINTER(C.c_ulonglong)] * 3))
    f("osh_b200_fp32_probe_tets", None, C.c_uint, _f64p, np.ctypeslib.ndpointer(np.float32),
      np.ctypeslib.ndpointer(np.float32), _f64p)
    f("osh_b200_fp32_probe_edges", None, C.c_uint, _f64p, _f64p, C.c_double,
      np.ctypeslib.ndpointer(np.int32), _f64p)
    f("osh_b200_selftest_scan_wait", C.c_int, C.c_uint)
    f("osh_b200_exscan_u32", C.c_int, vp, vp, C.c_uint, vp, C.c_int)
    f("osh_b200_server_new", vp, C.c_double, C.c_double, C.c_uint, C.c_uint, C.c_ulonglong)
    f("osh_b200_server_free", None, vp)
    f("osh_b200_server_submit", C.c_int, vp, C.c_uint, C.c_uint, _f64p, C.c_uint, _u32p, _f64p)
    f("osh_b200_server_step", C.c_int, vp)
    f("osh_b200_server_start", None, vp)
    f("osh_b200_server_stop", None, vp)
    f("osh_b200_server_wait", C.c_int, vp, C.c_double)
    f("osh_b200_server_set_union_elems", None, vp, C.c_ulonglong)
    f("osh_b200_server_poll", C.c_uint, vp, C.POINTER(C.c_uint), C.c_uint)
    f("osh_b200_server_take", vp, vp, C.c_uint)
    f("osh_b200_server_job_info", C.c_int, vp, C.c_uint, *([C.POINTER(C.c_double)] * 3),
      C.POINTER(C.c_uint), C.POINTER(C.c_double), C.POINTER(C.c_int))
    f("osh_b200_server_stats", None, vp, *([C.POINTER(C.c_uint)] * 3),
      C.POINTER(C.c_ulonglong), C.POINTER(C.c_double))
    f("osh_b200_server_times", None, vp, *([C.POINTER(C.c_double)] * 4))
    f("osh_b200_launch_count", C.c_ulonglong)
    f("osh_b200_sync_count", C.c_ulonglong)
    f("osh_b200_host_stats", None, C.POINTER(C.c_ulonglong), C.POINTER(C.c_double))
    f("osh_b200_probe_enable", None, C.c_uint)
    f("osh_b200_probe_reset", None)
    f("osh_b200_probe_count", C.c_uint)
    f("osh_b200_probe_name", C.c_char_p, C.c_uint)
    f("osh_b200_probe_read", None, C.c_uint, C.POINTER(C.c_uint), C.POINTER(C.c_double),
      C.POINTER(C.c_double))
    f("osh_b200_swap_table", C.c_uint, C.c_uint, C.POINTER(C.c_uint),
      C.POINTER(C.c_uint), C.POINTER(C.c_uint), _u32p, _u32p)
    _lib = L
    return L


def check():
    L = lib()
    code = L.osh_b200_last_error()
    if code:
        msg = L.osh_b200_last_error_message().decode()
        L.osh_b200_clear_error()
        raise OshError(code, msg)


def box(n: int, seed: int = 0, pert: float = 0.1):
    """The library's own n^3 six-tet box generator (host code)."""
    nv = (n + 1) ** 3
    coords = np.empty(nv * 3, np.float64)
    conn = np.empty(6 * n ** 3 * 4, np.uint32)
    center = np.empty(3, np.float64)
    lib().osh_b200_box(n, seed, pert, coords, conn, center)
    return coords, conn, center


def swap_table(ring_size):
    nt, nm, ni = C.c_uint(), C.c_uint(), C.c_uint()
    tris = np.zeros(42 * 5 * 3, np.uint32)
    ied = np.zeros(42 * 4 * 2, np.uint32)
    lib().osh_b200_swap_table(ring_size, C.byref(nt), C.byref(nm), C.byref(ni), tris, ied)
    nt, nm, ni = nt.value, nm.value, ni.value
    return (tris[: nm * nt * 3].reshape(nm, nt, 3), ied[: nm * ni * 2].reshape(nm, ni, 2))


@dataclass
class Tag:
    name: str
    type: int
    ncomps: int
    transfer: int
    data: np.ndarray


@dataclass
class MeshSnapshot:
    dim: int
    counts: list
    conn: dict
    tags: dict
    globals: dict = field(default_factory=dict)

    def tag(self, dim, name):
        for t in self.tags[dim]:
            if t.name == name:
                return t
        return None


class Mesh:
    """A mesh resident on the current GPU, driven through the C ABI."""

    def __init__(self, handle):
        self.L = lib()
        self.h = handle
        if not self.h:
            check()
            raise OshError(4, "null mesh")

    @classmethod
    def reduced(cls, dim, coords, conn):
        coords = np.ascontiguousarray(coords, dtype=np.float64).ravel()
        conn = np.ascontiguousarray(conn, dtype=np.uint32).ravel()
        h = lib().osh_b200_new_reduced(dim, coords.size // 3, coords,
                                       conn.size // DEG[dim][0], conn)
        check()
        return cls(h)

    def clone(self):
        """A deep copy on the same GPU (connectivity, tags, global numbers)."""
        h = self.L.osh_b200_clone(self.h)
        self._chk()
        return Mesh(h)

    def has_tag(self, dim, name):
        n = self.L.osh_b200_ntags(self.h, dim)
        return any(self.L.osh_b200_tag_name(self.h, dim, i).decode() == name for i in range(n))

    # size-field producers ----------------------------------------------------
    def element_gradients(self, name):
        self.L.osh_b200_element_gradients(self.h, name.encode())
        self._chk()

    def recover_by_volume(self, name):
        self.L.osh_b200_recover_by_volume(self.h, name.encode())
        self._chk()

    def size_from_hessian(self, hess_name, weights, min_h, max_h):
        w = None
        if weights is not None:
            w = np.ascontiguousarray(weights, dtype=np.float64)
        self.L.osh_b200_size_from_hessian(self.h, hess_name.encode(),
                                          None if w is None else w.ctypes.data_as(C.c_void_p),
                                          min_h, max_h)
        self._chk()

    def warp_to_limit(self, qual_floor):
        return self._chk(self.L.osh_b200_warp_to_limit(self.h, qual_floor))

    def free_tag(self, dim, name):
        self.L.osh_free_field(self.h, dim, name.encode())
        self._chk()

    def set_fp32_filter(self, on=True):
        """Decide far-from-threshold candidates on single-precision estimates
        (double recheck near thresholds; results unchanged)."""
        self.L.osh_b200_set_fp32_filter(self.h, 1 if on else 0)
        self._chk()

    def ghost(self, nlayers):
        """osh_ghost: on one rank, records the layers (and owner caches)."""
        self.L.osh_ghost(self.h, nlayers)
        self._chk()

    def ghost_layers(self):
        return self.L.osh_num_ghost_layers(self.h)

    @classmethod
    def read_vtk(cls, path):
        """osh_read_vtk: a ".vtu" file, or the one piece of a ".pvtu" file
        (as a parallel mesh)."""
        h = lib().osh_read_vtk(os.fsencode(path))
        check()
        return cls(h)

    def write_vtk(self, path, ascii=False, compress=False):
        """osh_write_vtk (binary) or, with ascii / compress,
        osh_b200_write_vtk_opts; a ".pvtu" path also writes "<stem>.vtu"."""
        if ascii or compress:
            self.L.osh_b200_write_vtk_opts(self.h, os.fsencode(path), int(bool(ascii)),
                                           int(bool(compress)))
        else:
            self.L.osh_write_vtk(self.h, os.fsencode(path))
        self._chk()

    def has_dim(self, dim):
        """mesh_has_dim: entities of dimension dim are held (not derived)"""
        return bool(self._chk(self.L.osh_b200_has_dim(self.h, dim)))

    def digest(self):
        """Order-sensitive 64-bit hash of every array of the mesh (device)."""
        return self._chk(self.L.osh_b200_digest(self.h))

    def close(self):
        if self.h:
            self.L.osh_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, r=None):
        check()
        return r

    # set-up ------------------------------------------------------------------
    def derive_model_full(self, crease=3.14159265359 / 4):
        self.L.osh_b200_derive_model(self.h, crease)
        self._chk()

    def make_parallel(self):
        self.L.osh_b200_make_parallel(self.h)
        self._chk()

    def add_tag(self, dim, name, data, type_=T_F64, ncomps=1, transfer=X_NOT):
        arr = np.ascontiguousarray(data, dtype=_NP[type_])
        self.L.osh_b200_add_tag(self.h, dim, name.encode(), type_, ncomps, transfer,
                                arr.ctypes.data_as(C.c_void_p))
        self._chk()

    def add_field(self, dim, name, data, ncomps=1, transfer=X_NOT):
        self.add_tag(dim, name, data, T_F64, ncomps, transfer)

    def set_globals(self, dim, g):
        self.L.osh_b200_set_globals(self.h, dim, np.ascontiguousarray(g, dtype=np.uint64))
        self._chk()

    # queries -------------------------------------------------------------------
    @property
    def dim(self):
        return self.L.osh_dim(self.h)

    def count(self, dim):
        return self._chk(self.L.osh_count(self.h, dim))

    def _d2h(self, ptr, n, dtype):
        out = np.empty(n, dtype)
        if n:
            self.L.osh_b200_copy_to_host(out.ctypes.data_as(C.c_void_p), ptr,
                                         out.nbytes)
            self._chk()
        return out

    def down(self, high, low):
        p = self.L.osh_down(self.h, high, low)
        self._chk()
        return self._d2h(p, self.count(high) * DEG[high][low], np.uint32)

    def up(self, low, high):
        n = self.count(low)
        po = self.L.osh_up_offs(self.h, low, high)
        pa = self.L.osh_up(self.h, low, high)
        pd = self.L.osh_up_dirs(self.h, low, high)
        self._chk()
        offs = self._d2h(po, n + 1, np.uint32)
        nadj = int(offs[-1])
        return offs, self._d2h(pa, nadj, np.uint32), self._d2h(pd, nadj, np.uint32)

    def star(self, low, high):
        n = self.count(low)
        po = self.L.osh_star_offs(self.h, low, high)
        pa = self.L.osh_star(self.h, low, high)
        self._chk()
        offs = self._d2h(po, n + 1, np.uint32)
        return offs, self._d2h(pa, int(offs[-1]), np.uint32)

    def dual(self):
        d = self.dim
        p = self.L.osh_b200_dual(self.h)
        self._chk()
        return self._d2h(p, self.count(d) * DEG[d][d - 1], np.uint32)

    def min_quality(self):
        return self._chk(self.L.osh_b200_min_quality(self.h))

    def qualities(self):
        out = np.empty(self.count(self.dim), np.float64)
        self.L.osh_b200_qualities(self.h, out)
        return self._chk(out)

    def edge_lengths(self):
        out = np.empty(self.count(1), np.float64)
        self.L.osh_b200_edge_lengths(self.h, out)
        return self._chk(out)

    def tags(self, dim):
        out = []
        n = self.count(dim)
        for i in range(self.L.osh_b200_ntags(self.h, dim)):
            ty, nc, tr = C.c_uint(), C.c_uint(), C.c_uint()
            self.L.osh_b200_tag_info(self.h, dim, i, C.byref(ty), C.byref(nc), C.byref(tr))
            name = self.L.osh_b200_tag_name(self.h, dim, i).decode()
            p = self.L.osh_b200_tag_data(self.h, dim, i)
            self._chk()
            out.append(Tag(name, ty.value, nc.value, tr.value,
                           self._d2h(p, n * nc.value, _NP[ty.value])))
        return out

    def globals(self, dim):
        p = self.L.osh_global(self.h, dim)
        self._chk()
        if not p:
            return None
        return self._d2h(p, self.count(dim), np.uint64)

    def snapshot(self) -> MeshSnapshot:
        d = self.dim
        counts = [self.count(k) for k in range(d + 1)]
        conn = {k: self.down(k, 0) for k in range(1, d + 1)}
        tags = {k: self.tags(k) for k in range(d + 1)}
        glob = {}
        for k in range(d + 1):
            g = self.globals(k)
            if g is not None:
                glob[k] = g
        return MeshSnapshot(d, counts, conn, tags, glob)

    # passes ----------------------------------------------------------------------
    def refine_by_size(self, qual_floor):
        return self._chk(self.L.osh_b200_refine_by_size(self.h, qual_floor))

    def uniformly_refine(self):
        self.L.osh_b200_uniformly_refine(self.h)
        self._chk()

    def coarsen_by_size(self, qual_floor, size_floor):
        return self._chk(self.L.osh_b200_coarsen_by_size(self.h, qual_floor, size_floor))

    def coarsen_slivers(self, qual_floor, nlayers):
        return self._chk(self.L.osh_b200_coarsen_slivers(self.h, qual_floor, nlayers))

    def swap_slivers(self, good_qual, nlayers):
        return self._chk(self.L.osh_b200_swap_slivers(self.h, good_qual, nlayers))

    def adapt(self, size_floor, good_qual, nlayers, max_ops):
        return self._chk(self.L.osh_adapt(self.h, size_floor, good_qual, nlayers, max_ops))

    def last_pass(self):
        v = [C.c_uint() for _ in range(5)]
        self.L.osh_b200_last_pass(*[C.byref(x) for x in v])
        return dict(zip(("op", "elems_in", "elems_out", "nselected", "rounds"),
                        [x.value for x in v]))

    def refine_sets(self, qual_floor):
        ne = self.count(1)
        cand, good, ind = (np.zeros(ne, np.uint32) for _ in range(3))
        quals = np.zeros(ne, np.float64)
        self.L.osh_b200_refine_sets(self.h, qual_floor, cand, good, quals, ind)
        self._chk()
        return dict(candidate=cand, good=good, quals=quals, indset=ind)

    def coarsen_sets(self, qual_floor, size_floor):
        ne, nv = self.count(1), self.count(0)
        cs, cc, cq = (np.zeros(ne, np.uint32) for _ in range(3))
        q2 = np.zeros(ne * 2, np.float64)
        cand, ind, gv = (np.zeros(nv, np.uint32) for _ in range(3))
        colq = np.zeros(nv, np.float64)
        self.L.osh_b200_coarsen_sets(self.h, qual_floor, size_floor, cs, cc, cq, q2,
                                     cand, colq, ind, gv)
        self._chk()
        return dict(codes_size=cs, codes_class=cc, codes_qual=cq, quals2=q2,
                    candidates=cand, col_qual=colq, indset=ind, gen_vert=gv)

    def swap_sets(self, good_qual, nlayers):
        ne, nel = self.count(1), self.count(self.dim)
        sl = np.zeros(nel, np.uint32)
        cand, inter, good, rs, ind = (np.zeros(ne, np.uint32) for _ in range(5))
        q = np.zeros(ne, np.float64)
        self.L.osh_b200_swap_sets(self.h, good_qual, nlayers, sl, cand, inter, good, q,
                                  rs, ind)
        self._chk()
        return dict(slivers=sl, candidates=cand, interior=inter, good=good, quals=q,
                    ring_sizes=rs, indset=ind)

    def synchronize(self):
        self.L.osh_b200_synchronize(self.h)
        self._chk()


def fp32_stats(reset=False):
    """(decided on the estimate, rechecked in double, max |estimate - double|,
    times the bound was exceeded) since the last reset."""
    L = lib()
    d, r = C.c_ulonglong(), C.c_ulonglong()
    e, b = C.c_double(), C.c_uint()
    L.osh_b200_fp32_stats(C.byref(d), C.byref(r), C.byref(e), C.byref(b))
    check()
    if reset:
        L.osh_b200_fp32_stats_reset()
        check()
    return dict(decided=d.value, rechecked=r.value, max_error=e.value, bound_exceeded=b.value)


def set_fp32_audit(on=True):
    """Audit mode of the filter (device-wide): every decision taken on an
    estimate is also taken in double and compared."""
    lib().osh_b200_set_fp32_audit(1 if on else 0)
    check()


def fp32_audit_stats():
    """(decisions audited, audited decisions the double path takes
    differently, estimates checked against their double value)."""
    L = lib()
    a, f, c = C.c_ulonglong(), C.c_ulonglong(), C.c_ulonglong()
    L.osh_b200_fp32_audit_stats(C.byref(a), C.byref(f), C.byref(c))
    check()
    return dict(audited=a.value, flips=f.value, checked=c.value)


def fp32_probe_tets(tets_xyz):
    """Device estimates for tets given as an (n, 4, 3) array: (estimate,
    bound, double quality)."""
    x = np.ascontiguousarray(tets_xyz, dtype=np.float64).reshape(-1)
    n = x.size // 12
    est = np.empty(n, np.float32)
    err = np.empty(n, np.float32)
    q64 = np.empty(n, np.float64)
    lib().osh_b200_fp32_probe_tets(n, x, est, err, q64)
    check()
    return est, err, q64


def fp32_probe_edges(ends_xyz, sizes, thr):
    """Device side decisions for edges given as an (n, 2, 3) array of end
    points and (n, 2) sizes: (side, double metric length)."""
    x = np.ascontiguousarray(ends_xyz, dtype=np.float64).reshape(-1)
    h = np.ascontiguousarray(sizes, dtype=np.float64).reshape(-1)
    n = x.size // 6
    side = np.empty(n, np.int32)
    r64 = np.empty(n, np.float64)
    lib().osh_b200_fp32_probe_edges(n, x, h, float(thr), side, r64)
    check()
    return side, r64


def pool_reserve(nbytes):
    """Grow the device memory pool to at least nbytes now."""
    lib().osh_b200_pool_reserve(int(nbytes))
    check()


def pool_stats(reset_high=False):
    """Bytes the device pool holds, bytes in use, and the peak in use."""
    r, u, h = C.c_ulonglong(), C.c_ulonglong(), C.c_ulonglong()
    lib().osh_b200_pool_stats(C.byref(r), C.byref(u), C.byref(h), 1 if reset_high else 0)
    check()
    return dict(reserved=r.value, used=u.value, peak=h.value)


def adapt_batch(meshes, size_floor, good_qual, nlayers, max_ops, max_union_elems=0):
    """mesh_adapt of every mesh, adapted together in disjoint unions of at most
    ``max_union_elems`` input elements (0 = one union). Returns (changed, status)
    per mesh and the batch statistics."""
    L = lib()
    n = len(meshes)
    hs = (C.c_void_p * max(n, 1))(*[m.h for m in meshes])
    changed = (C.c_uint * max(n, 1))()
    status = (C.c_int * max(n, 1))()
    rc = L.osh_b200_adapt_batch(hs, n, size_floor, good_qual, nlayers, max_ops,
                                max_union_elems, changed, status)
    if rc:
        check()
        raise OshError(rc, "osh_b200_adapt_batch failed")
    u, st, up, mp = (C.c_uint() for _ in range(4))
    e = C.c_double()
    L.osh_b200_batch_stats(C.byref(u), C.byref(st), C.byref(up), C.byref(mp), C.byref(e))
    per = []
    for i in range(n):
        p, ei = C.c_uint(), C.c_double()
        L.osh_b200_batch_mesh_stats(i, C.byref(p), C.byref(ei))
        per.append((p.value, ei.value))
    stats = dict(unions=u.value, steps=st.value, union_passes=up.value,
                 mesh_passes=mp.value, elems_in=e.value, per_mesh=per)
    return list(changed[:n]), list(status[:n]), stats


def adapt_concurrent(meshes, size_floor, good_qual, nlayers, max_ops, nthreads=0,
                     budget_bytes=0):
    """mesh_adapt of every mesh, unchanged, by ``nthreads`` host threads on
    streams of their own (0 = 4), largest first within a device-memory
    budget (0 = 70% of free memory). Returns (changed, status) per mesh and
    the per-mesh (passes, elements in)."""
    L = lib()
    n = len(meshes)
    hs = (C.c_void_p * max(n, 1))(*[m.h for m in meshes])
    changed = (C.c_uint * max(n, 1))()
    status = (C.c_int * max(n, 1))()
    rc = L.osh_b200_adapt_concurrent(hs, n, size_floor, good_qual, nlayers, max_ops,
                                     nthreads, budget_bytes, changed, status)
    if rc:
        check()
        raise OshError(rc, "osh_b200_adapt_concurrent failed")
    per = []
    for i in range(n):
        p, ei = C.c_uint(), C.c_double()
        L.osh_b200_batch_mesh_stats(i, C.byref(p), C.byref(ei))
        per.append((p.value, ei.value))
    return list(changed[:n]), list(status[:n]), per


class Server:
    """Continuous-batching adaptation server (osh_b200_server_*): jobs are
    host arrays (coords, element connectivity, vertex size field)."""

    def __init__(self, size_floor, good_qual, nlayers, max_ops, budget_bytes):
        self.L = lib()
        self.h = self.L.osh_b200_server_new(size_floor, good_qual, nlayers, max_ops,
                                            int(budget_bytes))
        if not self.h:
            check()

    def submit(self, coords, conn, size, dim=3):
        coords = np.ascontiguousarray(coords, dtype=np.float64).ravel()
        conn = np.ascontiguousarray(conn, dtype=np.uint32).ravel()
        size = np.ascontiguousarray(size, dtype=np.float64).ravel()
        r = self.L.osh_b200_server_submit(self.h, dim, coords.size // 3, coords,
                                          conn.size // (dim + 1), conn, size)
        if r < 0:
            check()
        return r

    def start(self):
        """Run steps on the server's own engine thread."""
        self.L.osh_b200_server_start(self.h)
        check()

    def wait(self, timeout=-1.0):
        """Block until every submitted job finished (or timeout seconds);
        returns the jobs not finished."""
        r = self.L.osh_b200_server_wait(self.h, timeout)
        if r < 0:
            check()
        return r

    def stop(self):
        self.L.osh_b200_server_stop(self.h)
        check()

    def set_union_elems(self, n):
        self.L.osh_b200_server_set_union_elems(self.h, int(n))
        check()

    def step(self):
        r = self.L.osh_b200_server_step(self.h)
        if r < 0:
            check()
        return r

    def poll(self, max_ids=4096):
        ids = (C.c_uint * max_ids)()
        n = self.L.osh_b200_server_poll(self.h, ids, max_ids)
        check()
        return list(ids[:n])

    def take(self, job):
        h = self.L.osh_b200_server_take(self.h, job)
        check()
        return Mesh(h)

    def job_info(self, job):
        ts, ta, td, e = (C.c_double() for _ in range(4))
        p, st = C.c_uint(), C.c_int()
        r = self.L.osh_b200_server_job_info(self.h, job, C.byref(ts), C.byref(ta),
                                            C.byref(td), C.byref(p), C.byref(e), C.byref(st))
        if r < 0:
            check()
        return dict(finished=bool(r), t_submit=ts.value, t_admit=ta.value, t_done=td.value,
                    passes=p.value, elems_in=e.value, status=st.value)

    def stats(self):
        steps, active, queued = C.c_uint(), C.c_uint(), C.c_uint()
        res, now = C.c_ulonglong(), C.c_double()
        self.L.osh_b200_server_stats(self.h, C.byref(steps), C.byref(active), C.byref(queued),
                                     C.byref(res), C.byref(now))
        check()
        a, j, p, r = (C.c_double() for _ in range(4))
        self.L.osh_b200_server_times(self.h, C.byref(a), C.byref(j), C.byref(p), C.byref(r))
        return dict(steps=steps.value, active=active.value, queued=queued.value,
                    reserved=res.value, now=now.value, secs_admit=a.value, secs_join=j.value,
                    secs_passes=p.value, secs_retire=r.value)

    def close(self):
        if self.h:
            self.L.osh_b200_server_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def new_box_mesh(n, seed=0, pert=0.1, size=None, radial=None, parallel=False):
    """A classified, full-topology n^3 box on the GPU with an adapt_size field:
    uniform ``size`` or radial h = h0 + h1 |x - c| from ``radial=(h0, h1)``."""
    coords, conn, center = box(n, seed, pert)
    m = Mesh.reduced(3, coords, conn)
    m.derive_model_full()
    nv = coords.size // 3
    if radial is not None:
        h0, h1 = radial
        d = coords.reshape(-1, 3) - center
        h = h0 + h1 * np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
    else:
        h = np.full(nv, 0.05 if size is None else size)
    m.add_field(0, "adapt_size", h)
    if parallel:
        m.make_parallel()
    return m
