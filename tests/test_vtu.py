"""VTU files on the CPU: the Python restatement of the reference's format
(oracle/vtu.py) against the reference-written fixtures in tests/golden/vtu/,
and against the reference itself where oracle/_ref/ is built."""
import os
import re

import numpy as np
import pytest

from oracle import oracle as O
from oracle import vtu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "vtu")
FIXTURES = sorted(f for f in os.listdir(GOLD) if f.endswith(".vtu"))


def fmt_of(text: bytes):
    head = text.split(b"\n", 1)[0]
    ascii_ = b'format="ascii"' in text[:4096] and b"byte_order" not in head
    return ("ascii" if ascii_ else "binary"), b"compressor=" in head


@pytest.mark.parametrize("name", FIXTURES)
def test_restatement_reproduces_fixture(name):
    """parse -> render gives the reference's bytes back, for every format."""
    raw = open(os.path.join(GOLD, name), "rb").read()
    m = vtu.parse(raw)
    fmt, comp = fmt_of(raw)
    assert vtu.render(m, fmt, comp).encode() == raw


def test_fixture_contents():
    """What the fixtures hold (pins the parser on known facts)."""
    m = vtu.read(os.path.join(GOLD, "square4_binary.vtu"))
    assert m.dim == 2 and m.counts[0] == 25 and m.counts[2] == 32 and not m.full
    assert [t.name for t in m.tags[0]] == ["coordinates", "speed"]
    assert np.allclose(m.tags[0][1].data, np.linspace(0.0, 1.0, 25))
    m = vtu.read(os.path.join(GOLD, "box2_tags_zlib.vtu"))
    assert m.dim == 3 and m.full and set(m.conn) == {1, 2, 3}
    names = {k: [t.name for t in m.tags[k]] for k in m.tags}
    assert names[3][-1] == "region" and m.tags[3][-1].type == vtu.T_U8
    assert names[1][-1] == "edge_key" and m.tags[1][-1].type == vtu.T_U64
    assert np.array_equal(m.tags[1][-1].data,
                          np.arange(m.counts[1], dtype=np.uint64) * 2654435761)
    a = vtu.read(os.path.join(GOLD, "box2_fields_ascii.vtu"))
    assert [t.name for t in a.tags[3]][-2:] == ["mass", "pointwise"]
    assert a.tags[3][-1].ncomps == 3
    p = vtu.read(os.path.join(GOLD, "box2_parallel.vtu"))
    for k in range(4):
        g = [t for t in p.tags[k] if t.name == "global_number"]
        assert len(g) == 1 and np.array_equal(g[0].data, np.arange(p.counts[k]))
    pv = open(os.path.join(GOLD, "box2_parallel.pvtu")).read()
    assert '<Piece Source="box2_parallel.vtu"/>' in pv and 'GhostLevel="0"' in pv


def test_reduced_mesh_has_no_intermediate_sections():
    raw = open(os.path.join(GOLD, "box3_reduced_binary.vtu"), "rb").read()
    assert b"<Edges>" not in raw and b"NumberOfEdges" not in raw and b'Rep="Reduced"' in raw


needs_ref = pytest.mark.skipif(not O.have_reference(serial=True)
                               or not os.path.exists(O.REF_ZLIB_SO),
                               reason="reference not built (oracle/Makefile)")


@needs_ref
@pytest.mark.parametrize("name", FIXTURES)
def test_reference_reads_fixture_as_restated(name, tmp_path):
    """The reference reads each fixture into the mesh the restatement parses,
    and writes it back byte for byte."""
    path = os.path.join(GOLD, name)
    raw = open(path, "rb").read()
    fmt, comp = fmt_of(raw)
    r = O.reference_read_vtk(path, "zlib" if comp else "serial")
    out = str(tmp_path / name)
    r.write_vtk(out, ascii=(fmt == "ascii"))
    assert open(out, "rb").read() == raw
    m = vtu.parse(raw)
    s = r.snapshot()  # derives what a reduced mesh lacks: compare what the file holds
    assert s.counts[0] == m.counts[0]
    for k, c in m.conn.items():
        assert s.counts[k] == m.counts[k]
        assert np.array_equal(s.conn[k], c)
    for k in range(m.dim + 1):
        mine = [t for t in m.tags.get(k, []) if t.name != "coordinates"]
        theirs = [t for t in s.tags[k] if t.name != "coordinates"]
        assert [t.name for t in theirs] == [t.name for t in mine]
        for a, b in zip(theirs, mine):
            assert a.type == b.type and a.ncomps == b.ncomps
            assert np.array_equal(a.data, b.data)


@needs_ref
def test_reference_parallel_round_trip(tmp_path):
    """A .pvtu reads as a parallel mesh: global_number becomes the global
    numbers and leaves the tag lists; the GhostLevel is kept."""
    r = O.reference_read_vtk(os.path.join(GOLD, "box2_parallel.pvtu"))
    assert r.is_parallel() and r.ghost_layers() == 0
    for k in range(4):
        assert not r.has_tag(k, "global_number")
        assert np.array_equal(r.globals(k), np.arange(r.count(k)))
    r.write_vtk(str(tmp_path / "box2_parallel.pvtu"))
    for f in ("box2_parallel.vtu", "box2_parallel.pvtu"):
        assert open(tmp_path / f, "rb").read() == open(os.path.join(GOLD, f), "rb").read()


def test_render_of_restated_arrays_matches_format_rules():
    """Known bytes: a 1-triangle mesh in binary (base64 of the UInt32 count,
    then of the values, separately padded) and in ASCII."""
    m = vtu.VtuMesh(2, False, [3, 0, 1], {2: np.array([0, 1, 2], np.uint32)},
                    {0: [vtu.VtuTag("coordinates", vtu.T_F64, 3,
                                    np.array([0, 0, 0, 1, 0, 0, 0, 1, 0], float))],
                     1: [], 2: []})
    txt = vtu.render(m, "binary")
    # connectivity: 12 bytes -> "DAAAAA==" then base64 of 0,1,2 as uint32
    assert "DAAAAA==AAAAAAEAAAACAAAA\n" in txt
    # offsets 3 and types 5 (VTK_TRIANGLE)
    assert "BAAAAA==AwAAAA==\n" in txt and "AQAAAA==BQ==\n" in txt
    a = vtu.render(m, "ascii")
    assert " 1.000000000000000e+00 0.000000000000000e+00 0.000000000000000e+00\n" in a
    assert re.search(r'Name="types" NumberOfComponents="1" format="ascii">\n 5\n', a)
