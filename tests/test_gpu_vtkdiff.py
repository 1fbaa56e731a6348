"""omega_h_v1_b200.vtkdiff, the reference's vtkdiff tool (test_vtkdiff.cpp,
mesh_diff.cpp:135-180) over this library's VTU reader: exit 0 for meshes
that agree, 2 for ones that differ, with the reference's messages; relative
tolerance and floor on f64 tags, exact integers and connectivity, and the
-superset option."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "vtu")
SRC = os.path.join(GOLD, "box2_adapt_binary.vtu")


def _variant(tmp_path, name, edit):
    from oracle import vtu
    m = vtu.read(SRC)
    edit(m)
    p = tmp_path / name
    p.write_text(vtu.render(m, "binary"))
    return str(p)


def test_same_and_copies_agree(tmp_path, capsys):
    from omega_h_v1_b200 import vtkdiff
    import omega_h_v1_b200 as G
    assert vtkdiff.main([SRC, SRC]) == 0
    copy = str(tmp_path / "copy.vtu")
    G.Mesh.read_vtk(SRC).write_vtk(copy)
    assert vtkdiff.main(["-tolerance", "0", copy, SRC]) == 0


def test_tolerance_and_floor(tmp_path, capsys):
    from omega_h_v1_b200 import vtkdiff

    def nudge(m):
        x = m.tags[0][0].data
        i = int(np.flatnonzero(x)[0])
        x[i] = x[i] * (1 + 1e-9)

    p = _variant(tmp_path, "nudged.vtu", nudge)
    assert vtkdiff.main([p, SRC]) == 0                       # 1e-6 default
    assert vtkdiff.main(["-tolerance", "1e-12", p, SRC]) == 2
    out = capsys.readouterr().out
    assert "max relative difference" in out and 'tag "coordinates" contents differ' in out

    def tiny(m):
        m.tags[0][0].data[0] = 1e-20   # was 0: relative difference 1
    q = _variant(tmp_path, "tiny.vtu", tiny)
    assert vtkdiff.main(["-tolerance", "1e-12", q, SRC]) == 2
    assert vtkdiff.main(["-tolerance", "1e-12", "-Floor", "1e-15", q, SRC]) == 0


def test_connectivity_and_labels(tmp_path, capsys):
    from omega_h_v1_b200 import vtkdiff

    def swap_conn(m):
        c = m.conn[3]
        c[0], c[1] = c[1], c[0]
    p = _variant(tmp_path, "conn.vtu", swap_conn)
    assert vtkdiff.main([p, SRC]) == 2
    assert "connectivity differs for dimension 3" in capsys.readouterr().out

    def relabel(m):
        t = [t for t in m.tags[3] if t.name == "class_id"][0]
        t.data[0] += 1
    q = _variant(tmp_path, "label.vtu", relabel)
    assert vtkdiff.main(["-tolerance", "1", q, SRC]) == 2
    assert 'tag "class_id" contents differ' in capsys.readouterr().out


def test_superset(tmp_path, capsys):
    from omega_h_v1_b200 import vtkdiff
    from oracle import vtu

    def extra(m):
        m.tags[3].append(vtu.VtuTag("extra", vtu.T_F64, 1, np.zeros(m.counts[3])))
    p = _variant(tmp_path, "extra.vtu", extra)
    assert vtkdiff.main([SRC, p]) == 2
    assert 'tag "extra" only on second mesh' in capsys.readouterr().out
    assert vtkdiff.main(["-superset", SRC, p]) == 0
    # as in the reference (mesh_diff.cpp:111-118), -superset also lets a tag
    # stand on the first mesh alone
    assert vtkdiff.main(["-superset", p, SRC]) == 0
    assert vtkdiff.main([p, SRC]) == 2
    assert 'tag "extra" only on first mesh' in capsys.readouterr().out
