"""vtkdiff: compare two VTU meshes as the reference's vtkdiff tool does
(test_vtkdiff.cpp, mesh_diff.cpp:135-180), reading them with this library.

    python -m omega_h_v1_b200.vtkdiff [-tolerance T] [-Floor F] [-superset] a.vtu b.vtu

Exit status 0 when the meshes agree, 2 when they differ (as the reference).
For every dimension either mesh holds: counts and vertex connectivity must
be equal, and every tag equal by name, type and size; integer tags exactly,
f64 tags within relative tolerance T (default 1e-6) unless both values are
below F in magnitude (default 0). With -superset the second mesh may hold
dimensions and tags the first does not. One difference from the serial
reference: the maximum relative difference is taken over every entry (the
reference's serial doubles_max starts its scan after entry 0).
"""
from __future__ import annotations

import sys

import numpy as np

from . import T_F64, Mesh


def _tag_diff(ta, tb, tol, floor, out):
    if ta.ncomps != tb.ncomps:
        out.append('tag "%s" sizes %u and %u differ' % (ta.name, ta.ncomps, tb.ncomps))
        return True
    if ta.type != tb.type:
        out.append('tag "%s" types differ' % ta.name)
        return True
    a, b = ta.data, tb.data
    if ta.type != T_F64:
        if not np.array_equal(a, b):
            out.append('tag "%s" contents differ' % ta.name)
            return True
        return False
    fa, fb = np.abs(a), np.abs(b)
    fm = np.maximum(fa, fb)
    with np.errstate(invalid="ignore", divide="ignore"):
        d = np.where((fa < floor) & (fb < floor), 0.0, np.abs(a - b) / fm)
    d = np.nan_to_num(d, nan=0.0)
    mx = float(d.max()) if d.size else 0.0
    if mx > tol:
        i = int(np.argmax(d))
        out.append("max relative difference %e" % mx)
        out.append("max difference pair is (%e, %e), #%u" % (a[i], b[i], i))
        out.append('tag "%s" contents differ' % ta.name)
        return True
    return False


def mesh_diff(a: Mesh, b: Mesh, tol=1e-6, floor=0.0, superset=False):
    """(differ, messages) with the semantics of mesh_diff.cpp:135-180"""
    out = []
    if a.dim != b.dim:
        out.append("mesh dimensionalities %u and %u differ" % (a.dim, b.dim))
        return True, out
    for d in range(a.dim + 1):
        ha, hb = a.has_dim(d), b.has_dim(d)
        if not ha and not hb:
            continue
        if ha and not hb:
            out.append("only first mesh has dimension %u" % d)
            return True, out
        if hb and not ha:
            if superset:
                continue
            out.append("only second mesh has dimension %u" % d)
            return True, out
        na, nb = a.count(d), b.count(d)
        if na != nb:
            out.append("counts %u and %u differ for dimension %u" % (na, nb, d))
            return True, out
        if d and not np.array_equal(a.down(d, 0), b.down(d, 0)):
            out.append("connectivity differs for dimension %u" % d)
            return True, out
        tas = {t.name: t for t in a.tags(d)}
        tbs = {t.name: t for t in b.tags(d)}
        for name, ta in tas.items():
            tb = tbs.get(name)
            if tb is None:
                if superset:
                    continue
                out.append('tag "%s" only on first mesh' % name)
                out.append("tags for dimension %u differ" % d)
                return True, out
            if _tag_diff(ta, tb, tol, floor, out):
                out.append("tags for dimension %u differ" % d)
                return True, out
        if not superset:
            for name in tbs:
                if name not in tas:
                    out.append('tag "%s" only on second mesh' % name)
                    out.append("tags for dimension %u differ" % d)
                    return True, out
    return False, out


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    tol, floor, superset, files = 1e-6, 0.0, False, []
    i = 0
    while i < len(argv):
        x = argv[i]
        if x == "-tolerance" and i + 1 < len(argv):
            tol = float(argv[i + 1])
            i += 2
            continue
        if x == "-Floor" and i + 1 < len(argv):
            floor = float(argv[i + 1])
            i += 2
            continue
        if x == "-superset":
            superset = True
        elif x == "-help":
            files = []
            break
        else:
            files.append(x)
        i += 1
    if len(files) != 2:
        print(__doc__)
        return 0
    a, b = Mesh.read_vtk(files[0]), Mesh.read_vtk(files[1])
    differ, msgs = mesh_diff(a, b, tol, floor, superset)
    for m in msgs:
        print(m)
    return 2 if differ else 0


if __name__ == "__main__":
    sys.exit(main())
