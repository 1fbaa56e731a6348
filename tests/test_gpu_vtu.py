"""VTU files through the library (osh_read_vtk / osh_write_vtk /
osh_b200_write_vtk_opts): the reference-written fixtures read and written
back byte for byte, adapted meshes written exactly as the reference writes
them (serial and parallel, binary / ASCII / zlib), reference-written meshes
adapted further with results identical to the reference's, and malformed
files reported as OSH_B200_E_IO."""
import os

import numpy as np
import pytest

from conftest import build_cpu, build_gpu

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "vtu")
FIXTURES = sorted(f for f in os.listdir(GOLD) if f.endswith(".vtu"))


def _fmt(raw):
    head = raw.split(b"\n", 1)[0]
    return (b"byte_order" not in head), (b"compressor=" in head)


def _ref_ok():
    from oracle import oracle as O
    return O.have_reference(serial=True) and os.path.exists(O.REF_ZLIB_SO)


needs_ref = pytest.mark.skipif(not _ref_ok(), reason="reference not built (oracle/Makefile)")


def _quiet(fn, *a):
    import sys
    sys.stdout.flush()
    saved = os.dup(1)
    null = os.open(os.devnull, os.O_WRONLY)
    os.dup2(null, 1)
    try:
        return fn(*a)
    finally:
        os.dup2(saved, 1)
        os.close(saved)
        os.close(null)


@pytest.mark.parametrize("name", FIXTURES)
def test_fixture_read_and_written_back(name, tmp_path):
    import omega_h_v1_b200 as G
    from oracle import vtu
    path = os.path.join(GOLD, name)
    raw = open(path, "rb").read()
    ascii_, comp = _fmt(raw)
    m = G.Mesh.read_vtk(path)
    out = str(tmp_path / name)
    m.write_vtk(out, ascii=ascii_, compress=comp)
    assert open(out, "rb").read() == raw
    # and the mesh holds what the file says (read after writing: a snapshot
    # derives the intermediate entities a reduced mesh lacks)
    want = vtu.parse(raw)
    s = m.snapshot()
    assert s.counts[0] == want.counts[0]
    for k, c in want.conn.items():
        assert np.array_equal(s.conn[k], c)
    for k in range(want.dim + 1):
        got = [t for t in s.tags[k] if t.name != "coordinates"]
        exp = [t for t in want.tags.get(k, []) if t.name != "coordinates"]
        assert [t.name for t in got] == [t.name for t in exp]
        for a, b in zip(got, exp):
            assert a.type == b.type and a.ncomps == b.ncomps
            assert np.array_equal(a.data, b.data)


def test_pvtu_fixture(tmp_path):
    import omega_h_v1_b200 as G
    m = G.Mesh.read_vtk(os.path.join(GOLD, "box2_parallel.pvtu"))
    assert m.ghost_layers() == 0
    for k in range(4):
        assert not m.has_tag(k, "global_number")
        assert np.array_equal(m.globals(k), np.arange(m.count(k)))
    m.write_vtk(str(tmp_path / "box2_parallel.pvtu"))
    for f in ("box2_parallel.vtu", "box2_parallel.pvtu"):
        assert open(tmp_path / f, "rb").read() == open(os.path.join(GOLD, f), "rb").read()


# (n, seed, pert, size, fields, parallel): the parallel n=4 case ends ghosted
# in the reference (a refine that found nothing after ghosting)
ADAPT_CASES = [
    (4, 4, 0.25, 0.2, False, False),
    (4, 4, 0.25, 0.2, False, True),
    (6, 4, 0.25, 0.25, True, True),
    (5, 1, 0.3, 0.3, True, False),
]


@needs_ref
@pytest.mark.parametrize("case", ADAPT_CASES)
def test_adapted_mesh_written_as_reference_writes_it(case, tmp_path):
    from oracle import oracle as O
    n, seed, pert, size, fields, parallel = case
    r = build_cpu(lambda d, c, k: O.ReferenceVariant(d, c, k, "serial"), n, seed=seed,
                  pert=pert, size=size, fields=fields, parallel=parallel)
    g = build_gpu(n, seed=seed, pert=pert, size=size, fields=fields, parallel=parallel)
    rr = _quiet(r.adapt, 0.3, 0.3, 4, 50)
    gr = g.adapt(0.3, 0.3, 4, 50)
    assert rr == gr
    if parallel:
        assert g.ghost_layers() == r.ghost_layers()
    ext = "pvtu" if parallel else "vtu"
    r.write_vtk(str(tmp_path / ("ref." + ext)))
    g.write_vtk(str(tmp_path / ("ours." + ext)))
    assert open(tmp_path / "ours.vtu", "rb").read() == open(tmp_path / "ref.vtu", "rb").read()
    if parallel:
        a = open(tmp_path / "ours.pvtu").read().replace("ours.vtu", "X")
        b = open(tmp_path / "ref.pvtu").read().replace("ref.vtu", "X")
        assert a == b
    # ASCII, and zlib against the reference's zlib build
    r.write_vtk(str(tmp_path / "ref_a.vtu"), ascii=True)
    g.write_vtk(str(tmp_path / "ours_a.vtu"), ascii=True)
    assert open(tmp_path / "ours_a.vtu", "rb").read() == open(tmp_path / "ref_a.vtu", "rb").read()
    zl = O.reference_lib("zlib")
    zm = O.CpuMesh.adopt(zl, zl.read_vtk(os.fsencode(str(tmp_path / "ref.vtu"))))
    zm.write_vtk(str(tmp_path / "ref_z.vtu"))
    g2 = type(g).read_vtk(str(tmp_path / "ours.vtu"))
    g2.write_vtk(str(tmp_path / "ours_z.vtu"), compress=True)
    assert open(tmp_path / "ours_z.vtu", "rb").read() == open(tmp_path / "ref_z.vtu", "rb").read()


@needs_ref
def test_reference_file_adapted_further_identically(tmp_path):
    """Interop: the reference adapts and writes; both libraries read that
    file, get a finer size field, adapt again and write identical files."""
    from oracle import oracle as O
    import omega_h_v1_b200 as G
    r = build_cpu(lambda d, c, k: O.ReferenceVariant(d, c, k, "serial"), 5, seed=2,
                  pert=0.2, size=0.3, fields=True)
    _quiet(r.adapt, 0.3, 0.3, 4, 50)
    src = str(tmp_path / "stage1.vtu")
    r.write_vtk(src)
    a = O.reference_read_vtk(src)
    b = G.Mesh.read_vtk(src)
    h = np.full(a.count(0), 0.12)
    for m in (a, b):
        m.free_tag(0, "adapt_size")
        m.add_field(0, "adapt_size", h)
    ra = _quiet(a.adapt, 0.3, 0.3, 4, 60)
    rb = b.adapt(0.3, 0.3, 4, 60)
    assert ra == rb == 1
    a.write_vtk(str(tmp_path / "ref2.vtu"))
    b.write_vtk(str(tmp_path / "ours2.vtu"))
    assert open(tmp_path / "ours2.vtu", "rb").read() == open(tmp_path / "ref2.vtu", "rb").read()


@needs_ref
def test_reference_reads_our_files(tmp_path):
    from oracle import oracle as O
    g = build_gpu(4, seed=3, pert=0.2, size=0.2, fields=True)
    g.adapt(0.3, 0.3, 4, 50)
    for asc in (False, True):
        p = str(tmp_path / ("g%d.vtu" % asc))
        g.write_vtk(p, ascii=asc)
        r = O.reference_read_vtk(p)
        sg, sr = g.snapshot(), r.snapshot()
        # files carry no transfer kinds: the reference reads every tag as
        # OSH_TRANSFER_NOT
        for s in (sg, sr):
            for lst in s.tags.values():
                for t in lst:
                    t.transfer = 0
        # binary is exact; ASCII prints 16 significant digits (" %.15e"),
        # one short of a double's round trip
        errs = O.mesh_diff(sg, sr, rel_tol=2e-15 if asc else 0.0)
        assert not errs, errs[:5]


def test_ghosting_api():
    import omega_h_v1_b200 as G
    m = build_gpu(2, parallel=True)
    assert m.ghost_layers() == 0
    m.ghost(1)
    assert m.ghost_layers() == 1
    m.ghost(0)
    assert m.ghost_layers() == 0
    s = build_gpu(2)
    with pytest.raises(G.OshError) as e:
        s.ghost(1)
    assert e.value.code == 4


def _corrupt(tmp_path, name, fn, tag):
    raw = open(os.path.join(GOLD, name), "rb").read()
    p = tmp_path / ("bad_%s_%s" % (tag, name))
    p.write_bytes(fn(raw))
    return str(p)


def _star_in_first_binary_array(raw):
    """a '*' ten characters into the first binary array's base64 run"""
    p = raw.index(b'format="binary">\n') + len(b'format="binary">\n') + 10
    return raw[:p] + b"*" + raw[p + 1:]


def test_malformed_files_are_reported(tmp_path):
    import omega_h_v1_b200 as G
    bad = [
        str(tmp_path / "missing.vtu"),
        # truncated in the middle of the data
        _corrupt(tmp_path, "box2_adapt_binary.vtu", lambda r: r[: len(r) // 2], "cut"),
        # a character outside base64 inside an array
        _corrupt(tmp_path, "square4_binary.vtu", _star_in_first_binary_array, "star"),
        # an unknown array type
        _corrupt(tmp_path, "square4_ascii.vtu",
                 lambda r: r.replace(b'type="Float64"', b'type="Int16"', 1), "type"),
        # a vertex index past NumberOfPoints
        _corrupt(tmp_path, "square4_ascii.vtu",
                 lambda r: r.replace(b'Name="connectivity" NumberOfComponents="1" '
                                     b'format="ascii">\n 0\n',
                                     b'Name="connectivity" NumberOfComponents="1" '
                                     b'format="ascii">\n 4000\n', 1), "vertex"),
        # no cells
        _corrupt(tmp_path, "square4_ascii.vtu",
                 lambda r: r.replace(b'NumberOfCells="32"', b'NumberOfCells="0"', 1), "empty"),
    ]
    for p in bad:
        with pytest.raises(G.OshError) as e:
            G.Mesh.read_vtk(p)
        assert e.value.code == 9, (p, str(e.value))
    # the library still works afterwards
    m = G.Mesh.read_vtk(os.path.join(GOLD, "square4_binary.vtu"))
    assert m.count(2) == 32


def test_large_round_trip(tmp_path):
    """A 384,000-tet mesh: write -> read -> write gives the same bytes, and
    the read mesh adapts to the same result as the original."""
    import omega_h_v1_b200 as G
    g = build_gpu(40, seed=1, pert=0.1, size=1 / 30.)
    p1, p2 = str(tmp_path / "a.vtu"), str(tmp_path / "b.vtu")
    g.write_vtk(p1)
    h = G.Mesh.read_vtk(p1)
    h.write_vtk(p2)
    assert open(p1, "rb").read() == open(p2, "rb").read()
    g.adapt(0.3, 0.3, 4, 50)
    h.adapt(0.3, 0.3, 4, 50)
    g.write_vtk(p1)
    h.write_vtk(p2)
    assert open(p1, "rb").read() == open(p2, "rb").read()
