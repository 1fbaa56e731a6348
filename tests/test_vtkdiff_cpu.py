"""The comparison logic of omega_h_v1_b200.vtkdiff (mesh_diff.cpp:135-180
semantics) on the CPU, over meshes parsed from the reference-written VTU
fixtures by the Python restatement of the format: no GPU needed."""
import os

import numpy as np

from oracle import vtu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "vtu")


class Fake:
    """The mesh interface vtkdiff.mesh_diff reads, over a parsed VTU file."""

    def __init__(self, vm):
        self.vm = vm
        self.dim = vm.dim

    def has_dim(self, d):
        return d == 0 or d in self.vm.conn

    def count(self, d):
        return self.vm.counts[d]

    def down(self, d, low):
        assert low == 0
        return self.vm.conn[d]

    def tags(self, d):
        return self.vm.tags.get(d, [])


def _load(name="box2_adapt_binary.vtu"):
    return vtu.read(os.path.join(GOLD, name))


def test_identical_meshes_agree():
    from omega_h_v1_b200.vtkdiff import mesh_diff
    differ, msgs = mesh_diff(Fake(_load()), Fake(_load()), tol=0.0)
    assert not differ and not msgs


def test_messages_follow_the_reference():
    from omega_h_v1_b200.vtkdiff import mesh_diff
    a, b = _load(), _load()
    b.conn[3][:2] = b.conn[3][1::-1].copy()
    differ, msgs = mesh_diff(Fake(a), Fake(b))
    assert differ and msgs == ["connectivity differs for dimension 3"]
    a, b = _load(), _load()
    b.tags[0][0].data[np.flatnonzero(b.tags[0][0].data)[0]] *= 1 + 1e-3
    differ, msgs = mesh_diff(Fake(a), Fake(b))
    assert differ and msgs[0].startswith("max relative difference")
    assert msgs[-2:] == ['tag "coordinates" contents differ', "tags for dimension 0 differ"]
    differ, _ = mesh_diff(Fake(a), Fake(b), tol=1e-2)
    assert not differ
    sq = _load("square4_binary.vtu")
    differ, msgs = mesh_diff(Fake(a), Fake(sq))
    assert differ and msgs == ["mesh dimensionalities 3 and 2 differ"]


def test_floor_and_dimensions():
    from omega_h_v1_b200.vtkdiff import mesh_diff
    a, b = _load(), _load()
    b.tags[0][0].data[0] = 1e-20            # an exact zero in a
    assert mesh_diff(Fake(a), Fake(b), tol=1e-9)[0]
    assert not mesh_diff(Fake(a), Fake(b), tol=1e-9, floor=1e-12)[0]
    r = _load("box3_reduced_binary.vtu")
    f = _load("box3_reduced_binary.vtu")
    f.conn[1] = np.zeros(0, np.uint32)      # the second mesh holds edges too
    f.counts[1] = 0
    differ, msgs = mesh_diff(Fake(r), Fake(f))
    assert differ and msgs == ["only second mesh has dimension 1"]
    assert not mesh_diff(Fake(r), Fake(f), superset=True)[0]
    assert mesh_diff(Fake(f), Fake(r), superset=True)[1] == ["only first mesh has dimension 1"]
