"""The reference's 2D and 3D warp tests (test_warp.cpp, test_warp_3d.cpp) as
flows that run
on either library: the reference driven through oracle/ref_driver.cpp, or
this library on the GPU. Both expose the same mesh methods, so the same
calls produce the VTU steps the reference's test writes (warp_0000.vtu,
...), and the two sets of files can be compared byte for byte, as the
reference's own run_tests.sh compares warp_0008.vtu with its gold copy.

Vertex fields are evaluated on the host with Python's math module, which
calls the same C library functions (atan2, cos, sin, sqrt) as the
reference's eval_field, in the reference's operation order."""
import math
import os

import numpy as np

PI = 3.14159265359                    # algebra.hpp:8
WARP_QUAL_FLOOR = 0.1                 # test_warp.cpp:20-24
GOOD_QUAL_FLOOR = 0.4
SIZE_FLOOR = 1. / 3.
NSLIVER_LAYERS = 0
MAX_OPS = 50

BOX_2D_COORDS = np.array([0, 0, 0, 1, 0, 0, 1, 1, 0, 0, 1, 0], np.float64)  # tables.cpp:22-27
BOX_2D_CONN = np.array([0, 1, 2, 2, 3, 0], np.uint32)                      # tables.cpp:17-20
X_NOT = 0


def _norm3(x):
    d = 0.0
    for k in range(3):
        d += x[k] * x[k]
    return math.sqrt(d)


def dye_fun(c):
    """test_warp.cpp:53-70"""
    l, r = (.25, .5, 0.0), (.75, .5, 0.0)
    d = 1.0
    x = [c[k] - l[k] for k in range(3)]
    if _norm3(x) > .25:
        d = -1.0
        x = [c[k] - r[k] for k in range(3)]
    if _norm3(x) > .25:
        return [0.0]
    return [4 * d * (.25 - _norm3(x))]


def warp_fun(c, rotation):
    """test_warp.cpp:34-51"""
    mid = (.5, .5, 0.0)
    x = [c[k] - mid[k] for k in range(3)]
    polar_a = math.atan2(x[1], x[0])
    polar_r = _norm3(x)
    rot_a = 0.0
    if polar_r < .5:
        rot_a = rotation * (2 * (.5 - polar_r))
    dest_a = polar_a + rot_a
    dst = [math.cos(dest_a) * polar_r, math.sin(dest_a) * polar_r, 0.0]
    return [dst[k] - x[k] for k in range(3)]


def _coords(m):
    for t in m.tags(0):
        if t.name == "coordinates":
            return t.data.reshape(-1, 3)
    raise KeyError("coordinates")


def eval_field(m, name, ncomps, fun):
    """mesh_eval_field (eval_field.cpp:34-40): fun at every vertex"""
    x = _coords(m)
    out = np.empty((x.shape[0], ncomps), np.float64)
    for i in range(x.shape[0]):
        out[i] = fun([float(x[i, 0]), float(x[i, 1]), float(x[i, 2])])
    m.add_field(0, name, out.ravel(), ncomps, X_NOT)


def set_size_field(m):
    """test_warp.cpp:72-85"""
    dim = 2
    m.free_tag(0, "adapt_size")
    m.element_gradients("dye")
    m.recover_by_volume("grad_dye")
    m.free_tag(dim, "grad_dye")
    m.element_gradients("grad_dye")
    m.free_tag(0, "grad_dye")
    m.recover_by_volume("grad_grad_dye")
    m.free_tag(dim, "grad_grad_dye")
    m.size_from_hessian("grad_grad_dye", [0.075 / 100.0], 0.025, 0.1)
    m.free_tag(0, "grad_grad_dye")


def run(m, outdir, adapt=None):
    """main() and warped_adapt() of test_warp.cpp on mesh m (the 2D box,
    already made full and classified); writes outdir/warp_%04u.vtu as
    write_vtk_step does and returns the file names. `adapt` wraps calls that
    print (the reference's passes)."""
    call = adapt or (lambda f, *a: f(*a))
    files = []

    def step():
        name = os.path.join(outdir, "warp_%04u.vtu" % len(files))
        m.write_vtk(name)
        files.append(name)

    eval_field(m, "adapt_size", 1, lambda c: [0.1])
    while call(m.refine_by_size, 0.0):
        pass
    eval_field(m, "dye", 1, dye_fun)
    set_size_field(m)
    step()
    call(m.adapt, SIZE_FLOOR, GOOD_QUAL_FLOOR, NSLIVER_LAYERS, MAX_OPS)
    rotation = PI / 4.
    for _ in range(2):
        for _ in range(4):
            eval_field(m, "warp", 3, lambda c: warp_fun(c, rotation))
            for it in range(3):
                done = m.warp_to_limit(WARP_QUAL_FLOOR)
                set_size_field(m)
                step()
                call(m.adapt, SIZE_FLOOR, GOOD_QUAL_FLOOR, NSLIVER_LAYERS, MAX_OPS)
                if done:
                    break
            else:
                raise RuntimeError("warped_adapt still not done after 3 iters")
            m.free_tag(0, "warp")
        rotation = -rotation
    return files


# ---------------------------------------------------------------------------
# test_warp_3d.cpp

BOX_3D_COORDS = np.array([0, 0, 0, 1, 0, 0, 1, 1, 0, 0, 1, 0,
                          0, 0, 1, 1, 0, 1, 1, 1, 1, 0, 1, 1], np.float64)  # tables.cpp:38-47
BOX_3D_CONN = np.array([0, 1, 2, 6, 2, 3, 0, 6, 0, 3, 7, 6,
                        7, 4, 0, 6, 0, 4, 5, 6, 5, 1, 0, 6], np.uint32)     # tables.cpp:29-36
X_CONSERVE, X_POINTWISE = 2, 1


def dye_fun_3d(c):
    """test_warp_3d.cpp:57-74"""
    l, r = (.25, .5, .5), (.75, .5, .5)
    d = 1.0
    x = [c[k] - l[k] for k in range(3)]
    if _norm3(x) > .25:
        d = -1.0
        x = [c[k] - r[k] for k in range(3)]
    if _norm3(x) > .25:
        return [0.0]
    return [4 * d * (.25 - _norm3(x))]


def warp_fun_3d(c, rotation):
    """test_warp_3d.cpp:36-55 (rotation about the z axis)"""
    mid = (.5, .5, 0.0)
    x = [c[k] - mid[k] for k in range(3)]
    x[2] = 0.0
    polar_a = math.atan2(x[1], x[0])
    polar_r = _norm3(x)
    rot_a = 0.0
    if polar_r < .5:
        rot_a = rotation * (2 * (.5 - polar_r))
    dest_a = polar_a + rot_a
    dst = [math.cos(dest_a) * polar_r, math.sin(dest_a) * polar_r, 0.0]
    return [dst[k] - x[k] for k in range(3)]


def element_centroids(m):
    """mesh_interp_to_elems of the coordinates (element_field.cpp:9-44):
    the vertices' sum in element order, divided by the vertex count"""
    x = _coords(m)
    c = m.down(3, 0).reshape(-1, 4)
    s = np.zeros((c.shape[0], 3))
    for j in range(4):
        s = s + x[c[:, j]]
    return s / 4


def run3d(m, outdir, adapt=None):
    """main() and warped_adapt() of test_warp_3d.cpp on the 3D box (already
    full and classified); returns the VTU steps written."""
    call = adapt or (lambda f, *a: f(*a))
    files = []

    def step():
        name = os.path.join(outdir, "warp_%04u.vtu" % len(files))
        m.write_vtk(name)
        files.append(name)

    eval_field(m, "adapt_size", 1, lambda c: [0.2])
    while call(m.refine_by_size, 0.0):
        pass
    eval_field(m, "dye", 1, dye_fun_3d)
    ec = element_centroids(m)
    nel = ec.shape[0]
    mass = np.where(ec[:, 0] > 0.5, 1.0 / nel, 0.0)
    m.add_field(3, "mass", mass, 1, X_CONSERVE)
    m.add_field(3, "pointwise", ec.ravel().copy(), 3, X_POINTWISE)
    step()
    rotation = PI / 4
    for _ in range(2):
        for _ in range(4):
            eval_field(m, "warp", 3, lambda c: warp_fun_3d(c, rotation))
            for it in range(6):
                done = m.warp_to_limit(0.2)
                call(m.adapt, 1. / 3., 0.3, 4, 50)
                step()
                if done:
                    break
            else:
                raise RuntimeError("warped_adapt still not done after 6 iters")
            m.free_tag(0, "warp")
        rotation = -rotation
    return files


# ---------------------------------------------------------------------------
# test_refine_by_size.cpp, test_coarsen_by_size.cpp, test_box.cpp, test_grad.cpp

def _radial_size(fine):
    """size_fun of test_refine_by_size.cpp:13-20 / fine_fun of
    test_coarsen_by_size.cpp:15-22"""
    def f(c):
        coarse = 0.5
        radius = _norm3(c)
        d = abs(radius - 0.5)
        return [coarse * d + fine * (1 - d)]
    return f


def _write(m, outdir, name, files):
    p = os.path.join(outdir, name)
    m.write_vtk(p)
    files.append(p)


def run_refine_by_size(m, outdir, adapt=None):
    """test_refine_by_size.cpp on the 2D box (full, classified)"""
    call = adapt or (lambda f, *a: f(*a))
    files = []
    size = _radial_size(0.1)
    eval_field(m, "adapt_size", 1, size)
    nel = m.count(2)
    m.add_field(2, "mass", np.full(nel, 1.0 / nel), 1, X_NOT)
    _write(m, outdir, "out_0.vtu", files)
    it = 1
    while call(m.refine_by_size, 0.0):
        _write(m, outdir, "out_%u.vtu" % it, files)
        it += 1
        m.free_tag(0, "adapt_size")
        eval_field(m, "adapt_size", 1, size)
    return files


def run_coarsen_by_size(m, outdir, adapt=None):
    """test_coarsen_by_size.cpp on the 2D box (full, classified)"""
    call = adapt or (lambda f, *a: f(*a))
    files = []
    fine = _radial_size(0.2)
    eval_field(m, "adapt_size", 1, fine)
    nel = m.count(2)
    m.add_field(2, "mass", np.full(nel, 1.0 / nel), 1, X_NOT)
    it = 0
    while call(m.refine_by_size, 0.0):
        _write(m, outdir, "ref_%u.vtu" % it, files)
        it += 1
        m.free_tag(0, "adapt_size")
        eval_field(m, "adapt_size", 1, fine)
    m.free_tag(0, "adapt_size")
    eval_field(m, "adapt_size", 1, lambda c: [4.0])
    it = 0
    while call(m.coarsen_by_size, 0.1, 0.5):
        _write(m, outdir, "cor_%u.vtu" % it, files)
        it += 1
    return files


def run_box(m, outdir, nrefs, adapt=None):
    """test_box.cpp: uniformly_refine nrefs times, write box.vtu"""
    call = adapt or (lambda f, *a: f(*a))
    for _ in range(nrefs):
        call(m.uniformly_refine)
    files = []
    _write(m, outdir, "box.vtu", files)
    return files


def run_grad(m, outdir, adapt=None):
    """test_grad.cpp on the 3D box (reduced, unclassified)"""
    call = adapt or (lambda f, *a: f(*a))
    eval_field(m, "adapt_size", 1, lambda c: [0.1])
    while call(m.refine_by_size, 0.0):
        pass
    eval_field(m, "dye", 1, dye_fun_3d)
    m.element_gradients("dye")
    m.recover_by_volume("grad_dye")
    m.element_gradients("grad_dye")
    m.recover_by_volume("grad_grad_dye")
    m.free_tag(0, "adapt_size")
    m.size_from_hessian("grad_grad_dye", [0.05 / 75.0], 0.05, 0.1)
    files = []
    _write(m, outdir, "grad.vtu", files)
    return files


# ---------------------------------------------------------------------------
# test_one_refine.cpp, test_one_coarsen.cpp on a parallel mesh read from a
# .pvtu, as run_tests.sh chains them (split -> one_ref -> two_ref, split ->
# one_cor -> two_cor), on one rank

def _read_like(m, path):
    """read_mesh_vtk in the library m belongs to"""
    if type(m).__name__ == "CpuMesh":
        from oracle import oracle as O
        return O.CpuMesh.adopt(m.L, m.L.read_vtk(os.fsencode(path)))
    return type(m).read_vtk(path)


def _pvtu_files(outdir, stem):
    return [os.path.join(outdir, stem + ".pvtu"), os.path.join(outdir, stem + ".vtu")]


def run_one_ops(m, outdir, adapt=None):
    """the 2D box refined uniformly three times and made parallel is the
    split mesh; then one_refine twice and one_coarsen twice from it"""
    call = adapt or (lambda f, *a: f(*a))
    for _ in range(3):
        call(m.uniformly_refine)
    m.make_parallel()
    m.write_vtk(os.path.join(outdir, "split.pvtu"))
    files = _pvtu_files(outdir, "split")
    src = "split"
    for stem in ("one_ref", "two_ref"):
        r = _read_like(m, os.path.join(outdir, src + ".pvtu"))
        call(r.uniformly_refine)
        r.write_vtk(os.path.join(outdir, stem + ".pvtu"))
        files += _pvtu_files(outdir, stem)
        src = stem
    src = "split"
    for stem in ("one_cor", "two_cor"):
        c = _read_like(m, os.path.join(outdir, src + ".pvtu"))
        c.add_field(0, "adapt_size", np.full(c.count(0), 2.0), 1, X_NOT)
        call(c.coarsen_by_size, 0.1, 0.7)
        c.free_tag(0, "adapt_size")
        c.write_vtk(os.path.join(outdir, stem + ".pvtu"))
        files += _pvtu_files(outdir, stem)
        src = stem
    return files


# name -> (dim, flow, box coordinates, box connectivity, classified full mesh)
CASES = {
    "warp_2d": (2, run, BOX_2D_COORDS, BOX_2D_CONN, True),
    "warp_3d": (3, run3d, BOX_3D_COORDS, BOX_3D_CONN, True),
    "refine_by_size_2d": (2, run_refine_by_size, BOX_2D_COORDS, BOX_2D_CONN, True),
    "coarsen_by_size_2d": (2, run_coarsen_by_size, BOX_2D_COORDS, BOX_2D_CONN, True),
    # run_tests.sh: box.exe --dim 2 --refinements 6
    "box_2d_6": (2, lambda m, d, adapt=None: run_box(m, d, 6, adapt), BOX_2D_COORDS,
                 BOX_2D_CONN, True),
    "box_3d_3": (3, lambda m, d, adapt=None: run_box(m, d, 3, adapt), BOX_3D_COORDS,
                 BOX_3D_CONN, True),
    "grad_3d": (3, run_grad, BOX_3D_COORDS, BOX_3D_CONN, False),
    "one_ops_pvtu_2d": (2, run_one_ops, BOX_2D_COORDS, BOX_2D_CONN, True),
}
