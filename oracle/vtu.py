"""TEST INFRASTRUCTURE ONLY: a Python restatement of the reference's VTU
format (vtk_io.cpp, base64.cpp, compress.cpp), used to check the library's
reader and writer byte for byte. Never imported by the product.

Layout (write_vtu_opts, vtk_io.cpp:487-538): VTKFile / UnstructuredGrid /
Piece with NumberOfPoints, NumberOfCells, NumberOfEdges and NumberOfFaces
(when the mesh holds them) and Rep; Points (the coordinates), Edges, Faces,
Cells (connectivity, offsets, types); PointData, EdgeData, FaceData,
CellData with every tag in list order (a parallel mesh appends
global_number / own_rank / own_id, parallel_mesh.cpp:219-228).

Arrays (write_array, vtk_io.cpp:319-336): binary = base64(UInt32 byte count)
+ base64(values), two separately padded strings (vtk_io.cpp:149-171); zlib =
base64 of the header {1, size, size, compressed size} + base64(zlib block);
ASCII = one entity per line, each value as " %u" / " %lu" / " %.15e".
"""
from __future__ import annotations

import base64
import re
import struct
import zlib
from dataclasses import dataclass, field

import numpy as np

T_U8, T_U32, T_U64, T_F64 = 0, 1, 2, 3
TYPE_NAMES = ["UInt8", "UInt32", "UInt64", "Float64"]
NP = {T_U8: np.uint8, T_U32: np.uint32, T_U64: np.uint64, T_F64: np.float64}
CELL_TYPES = [1, 3, 5, 10]      # VTK_VERTEX, VTK_LINE, VTK_TRIANGLE, VTK_TETRA
DEG0 = [1, 2, 3, 4]             # vertices per entity of each dimension


@dataclass
class VtuTag:
    name: str
    type: int
    ncomps: int
    data: np.ndarray


@dataclass
class VtuMesh:
    dim: int
    full: bool
    counts: list                                # per dimension 0..dim
    conn: dict                                  # dim -> uint32 (dims present)
    tags: dict = field(default_factory=dict)    # dim -> [VtuTag] (coordinates first at 0)
    ghost_level: int | None = None              # from a .pvtu


# ---------------------------------------------------------------------------
# writing

def _array(out, t, name, ncomps, data, fmt, compress):
    out.append('<DataArray type="%s" Name="%s" NumberOfComponents="%u" format="%s">\n'
               % (TYPE_NAMES[t], name, ncomps, "ascii" if fmt == "ascii" else "binary"))
    a = np.ascontiguousarray(data, dtype=NP[t]).ravel()
    if fmt == "ascii":
        conv = " %.15e" if t == T_F64 else " %u"
        rows = a.reshape(-1, ncomps) if a.size else np.zeros((0, ncomps), NP[t])
        for r in rows:
            out.append("".join(conv % (float(v) if t == T_F64 else int(v)) for v in r) + "\n")
    else:
        raw = a.astype(a.dtype.newbyteorder("<")).tobytes()
        if compress:
            comp = zlib.compress(raw)
            out.append(base64.b64encode(struct.pack("<4I", 1, len(raw), len(raw),
                                                    len(comp))).decode())
            out.append(base64.b64encode(comp).decode())
        else:
            out.append(base64.b64encode(struct.pack("<I", len(raw))).decode())
            out.append(base64.b64encode(raw).decode())
        out.append("\n")
    out.append("</DataArray>\n")


def render(m: VtuMesh, fmt="binary", compress=False) -> str:
    """The text the reference writes for mesh m (little-endian host)."""
    d = m.dim
    o = ['<VTKFile type="UnstructuredGrid"']
    if fmt != "ascii":
        o.append(' byte_order="LittleEndian" header_type="UInt32"')
        if compress:
            o.append(' compressor="vtkZLibDataCompressor"')
    o.append(">\n<UnstructuredGrid>\n")
    do_edges = d > 1 and 1 in m.conn
    do_faces = d > 2 and 2 in m.conn
    o.append('<Piece NumberOfPoints="%u" NumberOfCells="%u"' % (m.counts[0], m.counts[d]))
    if do_edges:
        o.append(' NumberOfEdges="%u"' % m.counts[1])
    if do_faces:
        o.append(' NumberOfFaces="%u"' % m.counts[2])
    o.append(' Rep="%s">\n' % ("Full" if m.full else "Reduced"))
    coords = next(t for t in m.tags[0] if t.name == "coordinates")
    o.append("<Points>\n")
    _array(o, coords.type, coords.name, coords.ncomps, coords.data, fmt, compress)
    o.append("</Points>\n")
    for k, sec in ((1, "Edges"), (2, "Faces")):
        if (k == 1 and do_edges) or (k == 2 and do_faces):
            o.append("<%s>\n" % sec)
            _array(o, T_U32, "connectivity", 1, m.conn[k], fmt, compress)
            o.append("</%s>\n" % sec)
    o.append("<Cells>\n")
    _array(o, T_U32, "connectivity", 1, m.conn[d], fmt, compress)
    n = m.counts[d]
    _array(o, T_U32, "offsets", 1, (np.arange(n, dtype=np.uint64) + 1) * DEG0[d], fmt, compress)
    _array(o, T_U8, "types", 1, np.full(n, CELL_TYPES[d], np.uint8), fmt, compress)
    o.append("</Cells>\n")
    secs = [(0, "PointData")]
    if do_edges:
        secs.append((1, "EdgeData"))
    if do_faces:
        secs.append((2, "FaceData"))
    secs.append((d, "CellData"))
    for k, sec in secs:
        o.append("<%s>\n" % sec)
        for t in m.tags.get(k, []):
            if not (k == 0 and t is coords):
                _array(o, t.type, t.name, t.ncomps, t.data, fmt, compress)
        o.append("</%s>\n" % sec)
    o.append("</Piece>\n</UnstructuredGrid>\n</VTKFile>\n")
    return "".join(o)


# ---------------------------------------------------------------------------
# reading (read_vtu_opts, vtk_io.cpp:726-737)

_B64 = set(b"ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/=")
_TOKEN = re.compile(rb"\s*(\S+)")


def _attr(line, name):
    key = name + '="'
    p = line.find(key)
    if p < 0:
        return None
    e = line.find('"', p + len(key))
    return line[p + len(key):e]


class _Cursor:
    def __init__(self, text: bytes):
        self.t = text
        self.pos = 0

    def line(self):
        if self.pos >= len(self.t):
            return None
        e = self.t.find(b"\n", self.pos)
        e = len(self.t) if e < 0 else e
        s = self.t[self.pos:e].decode("latin-1")
        self.pos = min(e + 1, len(self.t))
        return s

    def seek(self, prefix):
        while True:
            s = self.line()
            if s is None:
                raise ValueError("no %s" % prefix)
            if s.startswith(prefix):
                return s

    def array(self, head, nents, little, compressed):
        t = TYPE_NAMES.index(_attr(head, "type"))
        nc = int(_attr(head, "NumberOfComponents") or 1)
        n = nents * nc
        dt = np.dtype(NP[t]).newbyteorder("<" if little else ">")
        if _attr(head, "format") == "ascii":
            vals = []
            for _ in range(n):
                mt = _TOKEN.match(self.t, self.pos)
                vals.append(mt.group(1))
                self.pos = mt.end()
            a = np.array([float(v) if t == T_F64 else int(v) for v in vals], dtype=NP[t])
        else:
            e = self.pos
            while e < len(self.t) and self.t[e] in _B64:
                e += 1
            run = self.t[self.pos:e]
            self.pos = e
            if compressed:
                hdr = struct.unpack(("<" if little else ">") + "4I", base64.b64decode(run[:24]))
                comp = base64.b64decode(run[24:24 + (hdr[3] + 2) // 3 * 4])[:hdr[3]]
                raw = zlib.decompress(comp)
            else:
                nb = n * dt.itemsize
                raw = base64.b64decode(run[8:8 + (nb + 2) // 3 * 4])[:nb]
            a = np.frombuffer(raw, dtype=dt).astype(NP[t])
        self.seek("</DataArray")
        return VtuTag(_attr(head, "Name"), t, nc, a)


def parse(text: bytes, ghost_level=None) -> VtuMesh:
    c = _Cursor(text)
    vh = c.seek("<VTKFile")
    little = (_attr(vh, "byte_order") or "LittleEndian") == "LittleEndian"
    compressed = _attr(vh, "compressor") is not None
    ph = c.seek("<Piece")
    nv, ne = int(_attr(ph, "NumberOfPoints")), int(_attr(ph, "NumberOfCells"))
    nedges, nfaces = _attr(ph, "NumberOfEdges"), _attr(ph, "NumberOfFaces")
    full = _attr(ph, "Rep") == "Full"
    c.seek("<Cells")
    while True:
        h = c.seek("<DataArray")
        if _attr(h, "Name") == "types":
            break
    types = c.array(h, ne, little, compressed).data
    d = CELL_TYPES.index(int(types[0]))
    assert (types == CELL_TYPES[d]).all()
    counts = [nv] + [0] * d
    counts[d] = ne
    m = VtuMesh(d, full, counts, {}, {})
    c.pos = 0
    c.seek("<Points")
    m.tags[0] = [c.array(c.seek("<DataArray"), nv, little, compressed)]
    for k, n, name in ((1, nedges, "<Edge"), (2, nfaces, "<Face"), (d, ne, "<Cell")):
        if name != "<Cell" and (n is None or k >= d):
            continue
        n = int(n)
        m.counts[k] = n
        c.seek(name)
        m.conn[k] = c.array(c.seek("<DataArray"), n * DEG0[k], little, compressed).data
    secs = [(0, "<PointData")]
    if d > 1 and 1 in m.conn:
        secs.append((1, "<EdgeData"))
    if d > 2 and 2 in m.conn:
        secs.append((2, "<FaceData"))
    secs.append((d, "<CellData"))
    for k, sec in secs:
        c.seek(sec)
        lst = m.tags.setdefault(k, [])
        while True:
            s = c.line()
            if s is None or not s.startswith("<DataArray"):
                break
            lst.append(c.array(s, m.counts[k], little, compressed))
    m.ghost_level = ghost_level
    return m


def read(path: str) -> VtuMesh:
    with open(path, "rb") as f:
        return parse(f.read())


def from_snapshot(snap, full: bool, dims_present=None) -> VtuMesh:
    """A VtuMesh of an oracle / library MeshSnapshot; dims_present lists the
    intermediate dimensions whose connectivity the mesh holds (the element
    dimension is always written)."""
    d = snap.dim
    conn = {d: snap.conn[d]}
    for k in dims_present or ():
        conn[k] = snap.conn[k]
    tags = {k: [VtuTag(t.name, t.type, t.ncomps, t.data) for t in snap.tags[k]]
            for k in range(d + 1)}
    return VtuMesh(d, full, list(snap.counts), conn, tags)
