"""TEST INFRASTRUCTURE ONLY: ctypes front-ends for the two CPU checkers.

* ``Oracle``    -- our C restatement of the adaptation pass (liboracle.so,
                  built from oracle/osh_oracle.c).
* ``Reference`` -- the reference implementation itself, compiled from its own
                  sources into oracle/_ref/ by oracle/Makefile (OpenMP or
                  serial loop mode) and driven through oracle/ref_driver.cpp.

Both expose the same methods, so tests can run one seeded input through each
and compare with ``mesh_diff``. Nothing in the product imports this module;
it is loaded only by tests/, ``__graft_entry__.smoke()`` and the CPU leg of
bench.py.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_OMP_SO = os.path.join(HERE, "_ref", "libosh_ref_omp.so")
REF_SERIAL_SO = os.path.join(HERE, "_ref", "libosh_ref_serial.so")
REF_ZLIB_SO = os.path.join(HERE, "_ref", "libosh_ref_zlib.so")

T_U8, T_U32, T_U64, T_F64 = 0, 1, 2, 3
X_NOT, X_POINTWISE, X_CONSERVE, X_INHERIT = 0, 1, 2, 3
INVALID = 0xFFFFFFFF
DEG = [[1, 0, 0, 0], [2, 1, 0, 0], [3, 3, 1, 0], [4, 6, 4, 1]]
_NP = {T_U8: np.uint8, T_U32: np.uint32, T_U64: np.uint64, T_F64: np.float64}

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def have_reference(serial: bool = False) -> bool:
    return os.path.exists(REF_SERIAL_SO if serial else REF_OMP_SO)


@dataclass
class Tag:
    name: str
    type: int
    ncomps: int
    transfer: int
    data: np.ndarray


@dataclass
class MeshSnapshot:
    """Host copy of everything a pass produces (per dimension)."""

    dim: int
    counts: list
    conn: dict                      # dim -> uint32[n * verts_per_ent]
    tags: dict                      # dim -> list[Tag] (in mesh order)
    globals: dict = field(default_factory=dict)  # dim -> uint64[n]

    def tag(self, dim, name):
        for t in self.tags[dim]:
            if t.name == name:
                return t
        return None


class _Lib:
    """Shared binding for the oracle ("or_") and reference driver ("refd_")."""

    def __init__(self, path: str, prefix: str):
        self.lib = C.CDLL(path)
        self.p = prefix
        L, p = self.lib, prefix
        vp = C.c_void_p

        def f(name, res, *args):
            fn = getattr(L, p + name)
            fn.restype = res
            fn.argtypes = list(args)
            return fn

        self.new_reduced = f("new_reduced", vp, C.c_uint, C.c_uint, _f64p, C.c_uint, _u32p)
        self.derive_model_full = f("derive_model_full", None, vp)
        self.make_parallel = f("make_parallel", None, vp)
        self.free = f("free", None, vp)
        self.dim = f("dim", C.c_uint, vp)
        self.count = f("count", C.c_uint, vp, C.c_uint)
        self.add_tag = f("add_tag", None, vp, C.c_uint, C.c_char_p, C.c_uint, C.c_uint, C.c_uint, C.c_void_p)
        self.free_tag = f("free_tag", None, vp, C.c_uint, C.c_char_p)
        self.ntags = f("ntags", C.c_uint, vp, C.c_uint)
        self.tag_name = f("tag_name", C.c_char_p, vp, C.c_uint, C.c_uint)
        self.tag_type = f("tag_type", C.c_uint, vp, C.c_uint, C.c_uint)
        self.tag_ncomps = f("tag_ncomps", C.c_uint, vp, C.c_uint, C.c_uint)
        self.tag_transfer = f("tag_transfer", C.c_uint, vp, C.c_uint, C.c_uint)
        self.tag_data = f("tag_data", None, vp, C.c_uint, C.c_uint, C.c_void_p)
        self.down = f("down", None, vp, C.c_uint, C.c_uint, _u32p)
        self.up_size = f("up_size", C.c_uint, vp, C.c_uint, C.c_uint)
        self.up = f("up", None, vp, C.c_uint, C.c_uint, _u32p, _u32p, _u32p)
        self.star_size = f("star_size", C.c_uint, vp, C.c_uint, C.c_uint)
        self.star = f("star", None, vp, C.c_uint, C.c_uint, _u32p, _u32p)
        self.dual = f("dual", None, vp, _u32p)
        self.has_globals = f("has_globals", C.c_uint, vp, C.c_uint)
        self.globals_ = f("globals", None, vp, C.c_uint, _u64p)
        self.set_globals = f("set_globals", None, vp, C.c_uint, _u64p)
        self.min_quality = f("min_quality", C.c_double, vp)
        self.qualities = f("qualities", None, vp, _f64p)
        self.edge_lengths = f("edge_lengths", None, vp, _f64p)
        self.refine_by_size = f("refine_by_size", C.c_uint, vp, C.c_double)
        self.uniformly_refine = f("uniformly_refine", None, vp)
        self.coarsen_by_size = f("coarsen_by_size", C.c_uint, vp, C.c_double, C.c_double)
        self.coarsen_slivers = f("coarsen_slivers", C.c_uint, vp, C.c_double, C.c_uint)
        self.swap_slivers = f("swap_slivers", C.c_uint, vp, C.c_double, C.c_uint)
        self.adapt = f("adapt", C.c_uint, vp, C.c_double, C.c_double, C.c_uint, C.c_uint)
        self.refine_sets = f("refine_sets", C.c_uint, vp, C.c_double, _u32p, _u32p, _f64p, _u32p)
        self.coarsen_sets = f("coarsen_sets", C.c_uint, vp, C.c_double, C.c_double,
                              _u32p, _u32p, _u32p, _f64p, _u32p, _f64p, _u32p, _u32p)
        self.swap_sets = f("swap_sets", C.c_uint, vp, C.c_double, C.c_uint,
                           _u32p, _u32p, _u32p, _u32p, _f64p, _u32p, _u32p)
        self.element_gradients = f("element_gradients", None, vp, C.c_char_p)
        self.recover_by_volume = f("recover_by_volume", None, vp, C.c_char_p)
        self.size_from_hessian = f("size_from_hessian", None, vp, C.c_char_p, C.c_void_p,
                                   C.c_double, C.c_double)
        self.warp_to_limit = f("warp_to_limit", C.c_uint, vp, C.c_double)
        if prefix == "refd_":
            # VTU files (vtk_io.cpp), only in the reference driver
            self.read_vtk = f("read_vtk", vp, C.c_char_p)
            self.write_vtk = f("write_vtk", None, vp, C.c_char_p, C.c_uint)
            self.is_full = f("is_full", C.c_uint, vp)
            self.is_parallel = f("is_parallel", C.c_uint, vp)
            self.ghost_layers = f("ghost_layers", C.c_uint, vp)


_LIBS: dict = {}


def _lib(path, prefix):
    key = (path, prefix)
    if key not in _LIBS:
        _LIBS[key] = _Lib(path, prefix)
    return _LIBS[key]


class CpuMesh:
    """One mesh living inside a CPU checker library."""

    def __init__(self, lib: _Lib, dim: int, coords: np.ndarray, conn: np.ndarray):
        self.L = lib
        coords = np.ascontiguousarray(coords, dtype=np.float64)
        conn = np.ascontiguousarray(conn, dtype=np.uint32)
        nverts = coords.size // 3
        nelems = conn.size // DEG[dim][0]
        self.h = lib.new_reduced(dim, nverts, coords.ravel(), nelems, conn.ravel())

    @classmethod
    def adopt(cls, lib: _Lib, handle):
        m = cls.__new__(cls)
        m.L, m.h = lib, handle
        return m

    def close(self):
        if self.h:
            self.L.free(self.h)
            self.h = None

    def write_vtk(self, path, ascii=False):
        """write_mesh_vtk_opts of the reference (binary is zlib-compressed in
        the zlib build)."""
        self.L.write_vtk(self.h, os.fsencode(path), 1 if ascii else 0)

    def is_full(self):
        return bool(self.L.is_full(self.h))

    def is_parallel(self):
        return bool(self.L.is_parallel(self.h))

    def ghost_layers(self):
        return self.L.ghost_layers(self.h)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- set-up ---------------------------------------------------------------
    def derive_model_full(self):
        self.L.derive_model_full(self.h)

    def make_parallel(self):
        self.L.make_parallel(self.h)

    def add_tag(self, dim, name, data, type_=T_F64, ncomps=1, transfer=X_NOT):
        arr = np.ascontiguousarray(data, dtype=_NP[type_])
        self.L.add_tag(self.h, dim, name.encode(), type_, ncomps, transfer,
                       arr.ctypes.data_as(C.c_void_p))

    def add_field(self, dim, name, data, ncomps=1, transfer=X_NOT):
        self.add_tag(dim, name, data, T_F64, ncomps, transfer)

    def free_tag(self, dim, name):
        self.L.free_tag(self.h, dim, name.encode())

    def set_globals(self, dim, g):
        self.L.set_globals(self.h, dim, np.ascontiguousarray(g, dtype=np.uint64))

    # -- queries --------------------------------------------------------------
    @property
    def dim(self):
        return self.L.dim(self.h)

    def count(self, dim):
        return self.L.count(self.h, dim)

    def down(self, high, low):
        out = np.empty(self.count(high) * DEG[high][low], np.uint32)
        self.L.down(self.h, high, low, out)
        return out

    def up(self, low, high):
        n = self.count(low)
        nadj = self.L.up_size(self.h, low, high)
        offs = np.empty(n + 1, np.uint32)
        adj = np.empty(nadj, np.uint32)
        dirs = np.empty(nadj, np.uint32)
        self.L.up(self.h, low, high, offs, adj, dirs)
        return offs, adj, dirs

    def star(self, low, high):
        n = self.count(low)
        nadj = self.L.star_size(self.h, low, high)
        offs = np.empty(n + 1, np.uint32)
        adj = np.empty(nadj, np.uint32)
        self.L.star(self.h, low, high, offs, adj)
        return offs, adj

    def dual(self):
        d = self.dim
        out = np.empty(self.count(d) * DEG[d][d - 1], np.uint32)
        self.L.dual(self.h, out)
        return out

    def min_quality(self):
        return self.L.min_quality(self.h)

    def qualities(self):
        out = np.empty(self.count(self.dim), np.float64)
        self.L.qualities(self.h, out)
        return out

    def edge_lengths(self):
        out = np.empty(self.count(1), np.float64)
        self.L.edge_lengths(self.h, out)
        return out

    def tags(self, dim):
        out = []
        n = self.count(dim)
        for i in range(self.L.ntags(self.h, dim)):
            ty = self.L.tag_type(self.h, dim, i)
            nc = self.L.tag_ncomps(self.h, dim, i)
            arr = np.empty(n * nc, _NP[ty])
            self.L.tag_data(self.h, dim, i, arr.ctypes.data_as(C.c_void_p))
            out.append(Tag(self.L.tag_name(self.h, dim, i).decode(), ty, nc,
                           self.L.tag_transfer(self.h, dim, i), arr))
        return out

    def globals(self, dim):
        if not self.L.has_globals(self.h, dim):
            return None
        out = np.empty(self.count(dim), np.uint64)
        self.L.globals_(self.h, dim, out)
        return out

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

    # -- passes ---------------------------------------------------------------
    def refine_by_size(self, qual_floor):
        return self.L.refine_by_size(self.h, qual_floor)

    def uniformly_refine(self):
        self.L.uniformly_refine(self.h)

    def coarsen_by_size(self, qual_floor, size_floor):
        return self.L.coarsen_by_size(self.h, qual_floor, size_floor)

    def coarsen_slivers(self, qual_floor, nlayers):
        return self.L.coarsen_slivers(self.h, qual_floor, nlayers)

    def swap_slivers(self, good_qual, nlayers):
        return self.L.swap_slivers(self.h, good_qual, nlayers)

    def adapt(self, size_floor, good_qual, nlayers, max_ops):
        return self.L.adapt(self.h, size_floor, good_qual, nlayers, max_ops)

    def has_tag(self, dim, name):
        n = self.L.ntags(self.h, dim)
        return any(self.L.tag_name(self.h, dim, i).decode() == name for i in range(n))

    # size-field producers ----------------------------------------------------
    def element_gradients(self, name):
        self.L.element_gradients(self.h, name.encode())

    def recover_by_volume(self, name):
        self.L.recover_by_volume(self.h, name.encode())

    def size_from_hessian(self, hess_name, weights, min_h, max_h):
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        self.L.size_from_hessian(self.h, hess_name.encode(),
                                 None if w is None else w.ctypes.data_as(C.c_void_p),
                                 min_h, max_h)

    def warp_to_limit(self, qual_floor):
        return self.L.warp_to_limit(self.h, qual_floor)

    def refine_sets(self, qual_floor):
        ne = self.count(1)
        cand, good, ind = (np.zeros(ne, np.uint32) for _ in range(3))
        quals = np.zeros(ne, np.float64)
        self.L.refine_sets(self.h, qual_floor, cand, good, quals, ind)
        return dict(candidate=cand, good=good, quals=quals, indset=ind)

    def coarsen_sets(self, qual_floor, size_floor):
        ne, nv = self.count(1), self.count(0)
        cs, cc, cq = (np.zeros(ne, np.uint32) for _ in range(3))
        q2 = np.zeros(ne * 2, np.float64)
        cand, ind, gv = (np.zeros(nv, np.uint32) for _ in range(3))
        colq = np.zeros(nv, np.float64)
        self.L.coarsen_sets(self.h, qual_floor, size_floor, cs, cc, cq, q2,
                            cand, colq, ind, gv)
        return dict(codes_size=cs, codes_class=cc, codes_qual=cq, quals2=q2,
                    candidates=cand, col_qual=colq, indset=ind, gen_vert=gv)

    def swap_sets(self, good_qual, nlayers):
        ne, nel = self.count(1), self.count(self.dim)
        sl = np.zeros(nel, np.uint32)
        cand, inter, good, rs, ind = (np.zeros(ne, np.uint32) for _ in range(5))
        q = np.zeros(ne, np.float64)
        self.L.swap_sets(self.h, good_qual, nlayers, sl, cand, inter, good, q, rs, ind)
        return dict(slivers=sl, candidates=cand, interior=inter, good=good,
                    quals=q, ring_sizes=rs, indset=ind)


def Oracle(dim, coords, conn) -> CpuMesh:
    return CpuMesh(_lib(ORACLE_SO, "or_"), dim, coords, conn)


def Reference(dim, coords, conn, serial=False) -> CpuMesh:
    return CpuMesh(_lib(REF_SERIAL_SO if serial else REF_OMP_SO, "refd_"),
                   dim, coords, conn)


def reference_read_vtk(path, variant="serial") -> CpuMesh:
    """read_mesh_vtk of the reference; variant "serial", "omp" or "zlib"."""
    so = {"serial": REF_SERIAL_SO, "omp": REF_OMP_SO, "zlib": REF_ZLIB_SO}[variant]
    lib = _lib(so, "refd_")
    return CpuMesh.adopt(lib, lib.read_vtk(os.fsencode(path)))


def reference_lib(variant="serial") -> _Lib:
    so = {"serial": REF_SERIAL_SO, "omp": REF_OMP_SO, "zlib": REF_ZLIB_SO}[variant]
    return _lib(so, "refd_")


def ReferenceVariant(dim, coords, conn, variant="serial") -> CpuMesh:
    return CpuMesh(reference_lib(variant), dim, coords, conn)


# -- seeded synthetic inputs ---------------------------------------------------

def box(n: int, seed: int = 0, pert: float = 0.1):
    """n^3 hexahedra, 6 tets each, interior vertices perturbed by +-pert*h0.

    Returns (coords f64[V*3], conn u32[T*4], center f64[3])."""
    lib = _lib(ORACLE_SO, "or_").lib
    fn = lib.or_box
    fn.restype = None
    fn.argtypes = [C.c_uint, C.c_uint64, C.c_double, _f64p, _u32p, _f64p]
    nv = (n + 1) ** 3
    coords = np.empty(nv * 3, np.float64)
    conn = np.empty(6 * n ** 3 * 4, np.uint32)
    center = np.empty(3, np.float64)
    fn(n, seed, pert, coords, conn, center)
    return coords, conn, center


def radial_size(coords, center, h0=0.01, h1=0.04):
    lib = _lib(ORACLE_SO, "or_").lib
    fn = lib.or_radial_size
    fn.restype = None
    fn.argtypes = [C.c_uint, _f64p, _f64p, C.c_double, C.c_double, _f64p]
    nv = coords.size // 3
    out = np.empty(nv, np.float64)
    fn(nv, np.ascontiguousarray(coords), np.ascontiguousarray(center), h0, h1, out)
    return out


def swap_table(ring_size):
    lib = _lib(ORACLE_SO, "or_").lib
    fn = lib.or_swap_table
    fn.restype = C.c_uint
    fn.argtypes = [C.c_uint, C.POINTER(C.c_uint), C.POINTER(C.c_uint),
                   C.POINTER(C.c_uint), _u32p, _u32p]
    nt, nm, ni = C.c_uint(), C.c_uint(), C.c_uint()
    tris = np.zeros(42 * 5 * 3, np.uint32)
    ied = np.zeros(42 * 4 * 2, np.uint32)
    fn(ring_size, C.byref(nt), C.byref(nm), C.byref(ni), tris, ied)
    nt, nm, ni = nt.value, nm.value, ni.value
    return (tris[: nm * nt * 3].reshape(nm, nt, 3),
            ied[: nm * ni * 2].reshape(nm, ni, 2))


# -- fixtures ----------------------------------------------------------------------

def snapshot_digest(s: MeshSnapshot) -> str:
    """SHA-256 over a mesh's counts, connectivity, tags (name, type, ncomps,
    transfer, raw bytes in order) and global numbers."""
    import hashlib
    h = hashlib.sha256()
    h.update(np.asarray(s.counts, np.uint64).tobytes())
    for d in range(1, s.dim + 1):
        h.update(np.ascontiguousarray(s.conn[d], np.uint32).tobytes())
    for d in range(s.dim + 1):
        for t in s.tags[d]:
            h.update(t.name.encode())
            h.update(np.asarray([t.type, t.ncomps, t.transfer], np.uint32).tobytes())
            h.update(np.ascontiguousarray(t.data).tobytes())
    for d in sorted(s.globals):
        h.update(np.ascontiguousarray(s.globals[d], np.uint64).tobytes())
    return h.hexdigest()


def snapshot_to_npz(s: MeshSnapshot, path: str, **extra):
    arrays = {"counts": np.asarray(s.counts, np.uint32)}
    names = []
    for d in range(1, s.dim + 1):
        arrays["conn%d" % d] = s.conn[d]
    for d in range(s.dim + 1):
        for i, t in enumerate(s.tags[d]):
            key = "tag%d_%d" % (d, i)
            arrays[key] = t.data
            names.append("%d|%d|%s|%d|%d|%d" % (d, i, t.name, t.type, t.ncomps, t.transfer))
    for d, g in s.globals.items():
        arrays["glob%d" % d] = g
    arrays["tagmeta"] = np.asarray(names)
    for k, v in extra.items():
        arrays["x_" + k] = v
    np.savez_compressed(path, **arrays)


def snapshot_from_npz(path: str):
    z = np.load(path, allow_pickle=False)
    counts = [int(c) for c in z["counts"]]
    dim = len(counts) - 1
    conn = {d: z["conn%d" % d] for d in range(1, dim + 1)}
    tags = {d: [] for d in range(dim + 1)}
    for meta in z["tagmeta"]:
        d, i, name, ty, nc, tr = str(meta).split("|")
        tags[int(d)].append(Tag(name, int(ty), int(nc), int(tr), z["tag%s_%s" % (d, i)]))
    glob = {int(k[4:]): z[k] for k in z.files if k.startswith("glob")}
    extra = {k[2:]: z[k] for k in z.files if k.startswith("x_")}
    return MeshSnapshot(dim, counts, conn, tags, glob), extra


# -- comparison ------------------------------------------------------------------

def mesh_diff(a: MeshSnapshot, b: MeshSnapshot, rel_tol=1e-12, floor=0.0,
              check_tag_order=True):
    """Differences between two meshes, following mesh_diff.cpp:135-180 but
    taking the maximum over every entry (no serial index-0 skip).

    Connectivity and integer tags must match exactly; f64 tags may differ by
    ``rel_tol`` relative unless both values are below ``floor``. Returns a
    list of human-readable differences (empty when the meshes agree)."""
    errs = []
    if a.dim != b.dim:
        return ["dim %d != %d" % (a.dim, b.dim)]
    if list(a.counts) != list(b.counts):
        errs.append("counts %s != %s" % (a.counts, b.counts))
        return errs
    for d in range(1, a.dim + 1):
        if not np.array_equal(a.conn[d], b.conn[d]):
            bad = np.nonzero(a.conn[d] != b.conn[d])[0]
            errs.append("conn dim %d: %d entries differ (first at %d)"
                        % (d, bad.size, bad[0]))
    for d in range(a.dim + 1):
        na = [t.name for t in a.tags[d]]
        nb = [t.name for t in b.tags[d]]
        if check_tag_order and na != nb:
            errs.append("tags dim %d: %s != %s" % (d, na, nb))
        for ta in a.tags[d]:
            tb = b.tag(d, ta.name)
            if tb is None:
                if not check_tag_order:
                    errs.append("tag %s missing on dim %d" % (ta.name, d))
                continue
            if (ta.type, ta.ncomps, ta.transfer) != (tb.type, tb.ncomps, tb.transfer):
                errs.append("tag %s dim %d: meta %s != %s" % (
                    ta.name, d, (ta.type, ta.ncomps, ta.transfer),
                    (tb.type, tb.ncomps, tb.transfer)))
                continue
            if ta.type == T_F64:
                x, y = ta.data, tb.data
                if x.shape != y.shape:
                    errs.append("tag %s dim %d: shape" % (ta.name, d))
                    continue
                mag = np.maximum(np.abs(x), np.abs(y))
                diff = np.abs(x - y)
                with np.errstate(invalid="ignore", divide="ignore"):
                    rel = np.where(mag > 0, diff / np.where(mag > 0, mag, 1), 0.0)
                ok = (rel <= rel_tol) | ((np.abs(x) < floor) & (np.abs(y) < floor))
                ok |= (x == y)
                if not ok.all():
                    i = int(np.nonzero(~ok)[0][0])
                    errs.append("tag %s dim %d: max rel %.3g at %d (%r vs %r)" % (
                        ta.name, d, float(rel.max()), i, x[i], y[i]))
            elif not np.array_equal(ta.data, tb.data):
                bad = np.nonzero(ta.data != tb.data)[0]
                errs.append("tag %s dim %d: %d entries differ (first %d)" % (
                    ta.name, d, bad.size, bad[0]))
    for d in sorted(set(a.globals) | set(b.globals)):
        ga, gb = a.globals.get(d), b.globals.get(d)
        if ga is None or gb is None or not np.array_equal(ga, gb):
            errs.append("globals dim %d differ" % d)
    return errs
